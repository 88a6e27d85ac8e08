// Known-answer tests of the C++ host API (hpgb::Gridder) on the device,
// in the manner of the reference's GridderState unit tests
// (tests/GridderStateUnitTests.cc): a constant CF makes every footprint
// cell receive the same value, so sums over the grid and the weights have
// closed forms independent of where the visibility lands.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hpgb/gridder.hpp"

static int failures = 0;
#define CHECK(cond)                                                   \
  do {                                                                \
    if (!(cond)) {                                                    \
      std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);   \
      ++failures;                                                     \
    }                                                                 \
  } while (0)

// one group, constant CF value, support radius r, oversampling os
class ConstCF : public hpgb::CFArray {
 public:
  ConstCF(unsigned os, unsigned radius, std::complex<float> value)
      : m_os(os), m_r(radius), m_v(value) {}
  unsigned oversampling() const override { return m_os; }
  unsigned num_groups() const override { return 1; }
  std::array<unsigned, 4> extents(unsigned) const override {
    const unsigned e = (2 * m_r + 1 + 2 * padding) * m_os;
    return {e, e, 1, 1};
  }
  std::complex<float> operator()(unsigned, unsigned, unsigned, unsigned,
                                 unsigned) const override {
    return m_v;
  }

 private:
  unsigned m_os, m_r;
  std::complex<float> m_v;
};

static hpgb::VisData<1> one_vis(double u, double v, std::complex<float> val,
                                float weight) {
  hpgb::VisData<1> d{};
  d.visibilities[0][0] = val.real();
  d.visibilities[0][1] = val.imag();
  d.weights[0] = weight;
  d.frequency = 299792458.0;  // inverse wavelength 1 per metre
  d.phase = 0.0;
  d.uvw[0] = u;
  d.uvw[1] = v;
  d.uvw[2] = 0.0;
  d.grid_cube = 0;
  d.cf_index[0] = d.cf_index[1] = 0;
  return d;
}

int main() {
  int ndev = 0;
  hpgb_device_count(&ndev);
  if (ndev < 1) {
    std::printf("no device\n");
    return 2;
  }
  const std::array<unsigned, 4> gs{64, 64, 1, 1};
  const std::array<double, 2> scale{1.0, 1.0};
  auto rg = hpgb::Gridder::create(0, 0, 4, gs, scale, {{0}}, {{0}});
  CHECK(hpgb::is_value(rg));
  if (!hpgb::is_value(rg)) return 1;
  hpgb::Gridder g = std::move(hpgb::get_value(rg));
  CHECK(g.num_polarizations() == 1);
  const unsigned radius = 2, taps = 2 * radius + 1;
  ConstCF cf(4, radius, {1.0f, 0.0f});
  CHECK(!g.set_convolution_function(cf));

  // gridding: every one of the taps^2 cells gets vis * weight
  {
    std::vector<hpgb::VisData<1>> vis{one_vis(3.2, -7.6, {2.0f, 1.0f}, 0.5f)};
    CHECK(!g.grid_visibilities(std::move(vis)));
    g.fence();
    auto grid = g.grid_values();
    std::complex<double> sum = 0;
    int nonzero = 0;
    for (size_t i = 0; i < grid->size(); ++i) {
      sum += grid->data()[i];
      nonzero += grid->data()[i] != 0.0;
    }
    CHECK(nonzero == int(taps * taps));
    CHECK(std::abs(sum - std::complex<double>(25.0, 12.5)) < 1e-12);
    auto w = g.grid_weights();
    CHECK(std::abs((*w)(0, 0) - 12.5) < 1e-12);
  }

  // a deep copy is independent of its source
  {
    hpgb::Gridder c(g);
    c.reset_grid();
    auto a = g.grid_values();
    auto b = c.grid_values();
    double na = 0, nb = 0;
    for (size_t i = 0; i < a->size(); ++i) {
      na += std::norm(a->data()[i]);
      nb += std::norm(b->data()[i]);
    }
    CHECK(na > 0 && nb == 0);
  }

  // degridding a constant model predicts that constant (the normaliser is
  // the sum of the CF), residual = vis - prediction
  {
    hpgb::GridValueArray model(gs);
    for (size_t i = 0; i < model.size(); ++i) model.data()[i] = {3.0, -1.0};
    CHECK(!g.set_model(model));
    std::vector<hpgb::VisData<1>> vis{one_vis(-11.3, 4.1, {5.0f, 2.0f}, 1.0f)};
    auto rf = g.degrid_grid_get_residual_visibilities(std::move(vis));
    CHECK(hpgb::is_value(rf));
    if (hpgb::is_value(rf)) {
      auto& out = hpgb::get_value(rf).get();
      CHECK(out[0].visibilities[0][0] == 2.0f && out[0].visibilities[0][1] == 3.0f);
    }
    std::vector<hpgb::VisData<1>> vis2{one_vis(8.0, 8.0, {0.0f, 0.0f}, 1.0f)};
    auto pf = g.degrid_get_predicted_visibilities(std::move(vis2));
    CHECK(hpgb::is_value(pf));
    if (hpgb::is_value(pf)) {
      auto& out = hpgb::get_value(pf).get();
      CHECK(out[0].visibilities[0][0] == 3.0f && out[0].visibilities[0][1] == -1.0f);
    }
  }

  // FFT with POSITIVE sign then NEGATIVE with norm nx*ny restores the grid;
  // a shift forward then backward too
  {
    auto before = g.grid_values();
    CHECK(!g.apply_grid_fft(1.0, hpgb::FFTSign::POSITIVE));
    CHECK(!g.apply_grid_fft(double(gs[0]) * gs[1], hpgb::FFTSign::NEGATIVE));
    g.shift_grid(hpgb::ShiftDirection::FORWARD);
    g.shift_grid(hpgb::ShiftDirection::BACKWARD);
    auto after = g.grid_values();
    double err = 0, ref = 0;
    for (size_t i = 0; i < before->size(); ++i) {
      err += std::norm(after->data()[i] - before->data()[i]);
      ref += std::norm(before->data()[i]);
    }
    CHECK(ref > 0 && std::sqrt(err / ref) < 1e-12);
  }

  // errors are values of the reference's types
  {
    std::vector<hpgb::VisData<2>> v2(1);
    auto e = g.grid_visibilities(std::move(v2));
    CHECK(e && e->type() == hpgb::ErrorType::InvalidNumberPolarizations);
    std::vector<hpgb::VisData<1>> many(5, one_vis(0, 0, {1, 0}, 1));
    e = g.grid_visibilities(std::move(many));
    CHECK(e && e->type() == hpgb::ErrorType::ExcessiveNumberVisibilities);
    auto bad = hpgb::Gridder::create(0, 0, 1, gs, scale, {{0}, {0}}, {{0}});
    CHECK(!hpgb::is_value(bad) &&
          hpgb::get_error(bad).type() ==
              hpgb::ErrorType::InvalidNumberMuellerIndexRows);
  }

  // batched launch over two gridders of different sizes; plan controls
  {
    auto ra = hpgb::Gridder::create(0, 0, 4, {64, 64, 1, 1}, scale, {{0}}, {{0}});
    auto rb = hpgb::Gridder::create(0, 0, 4, {96, 80, 1, 1}, scale, {{0}}, {{0}});
    CHECK(hpgb::is_value(ra) && hpgb::is_value(rb));
    hpgb::Gridder a = std::move(hpgb::get_value(ra));
    hpgb::Gridder b = std::move(hpgb::get_value(rb));
    CHECK(!a.set_convolution_function(cf) && !b.set_convolution_function(cf));
    hpgb_tiled_plan plan{4, 64, 0, 0};
    CHECK(!a.set_tiled_plan(plan));
    CHECK(a.tiled_plan().ring_parts == 4 && a.tiled_plan().chunk_vis == 64);
    std::vector<std::vector<hpgb::VisData<1>>> batches{
        {one_vis(3.2, -7.6, {2.0f, 1.0f}, 0.5f)},
        {one_vis(-5.1, 4.4, {1.0f, -1.0f}, 2.0f)}};
    CHECK(!hpgb::grid_visibilities_batch<hpgb::VisData<1>>({&a, &b}, batches));
    a.fence();
    CHECK(a.last_gridding_kernel() == HPGB_KERNEL_TILED);
    auto ga = a.grid_values();
    auto gb = b.grid_values();
    std::complex<double> sa = 0, sb = 0;
    for (size_t i = 0; i < ga->size(); ++i) sa += ga->data()[i];
    for (size_t i = 0; i < gb->size(); ++i) sb += gb->data()[i];
    // taps^2 cells of vis * weight each
    CHECK(std::abs(sa - double(taps * taps) * std::complex<double>(1.0, 0.5)) < 1e-12);
    CHECK(std::abs(sb - double(taps * taps) * std::complex<double>(2.0, -2.0)) < 1e-12);
  }

  if (failures == 0) std::printf("OK\n");
  return failures == 0 ? 0 : 1;
}
