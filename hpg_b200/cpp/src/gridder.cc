// gridder.cc -- hpgb::Gridder over the C ABI (include/hpgb.h).

#include "hpgb/gridder.hpp"

#include <algorithm>

namespace hpgb {

opt_error_t error_of(int status) {
  if (status == HPGB_SUCCESS) return std::nullopt;
  const int t = status - 1;
  const ErrorType type = (t >= 0 && t <= int(ErrorType::Other))
                             ? ErrorType(t)
                             : ErrorType::Other;
  return Error(hpgb_last_error_message(), type);
}

rval_t<Gridder> Gridder::create(
    int device, unsigned max_added_tasks, size_t max_visibility_batch_size,
    const std::array<unsigned, 4>& grid_size,
    const std::array<double, 2>& grid_scale,
    const std::vector<std::vector<int>>& mueller_indexes,
    const std::vector<std::vector<int>>& conjugate_mueller_indexes) {
  // src/hpg.cc:226-264: the rows of both index sets match the grid's rows
  if (mueller_indexes.size() != grid_size[2] ||
      conjugate_mueller_indexes.size() != grid_size[2])
    return Error("Number of rows of Mueller indexes does not match grid",
                 ErrorType::InvalidNumberMuellerIndexRows);
  const unsigned npol =
      mueller_indexes.empty() ? 0 : unsigned(mueller_indexes[0].size());
  std::vector<int> m(size_t(grid_size[2]) * npol), c(m.size());
  for (unsigned r = 0; r < grid_size[2]; ++r) {
    if (mueller_indexes[r].size() != npol ||
        conjugate_mueller_indexes[r].size() != npol)
      return Error("Mueller index rows differ in length",
                   ErrorType::InvalidNumberPolarizations);
    std::copy(mueller_indexes[r].begin(), mueller_indexes[r].end(),
              m.begin() + size_t(r) * npol);
    std::copy(conjugate_mueller_indexes[r].begin(),
              conjugate_mueller_indexes[r].end(), c.begin() + size_t(r) * npol);
  }
  hpgb_gridder* h = nullptr;
  if (auto e = error_of(hpgb_create(device, max_added_tasks,
                                    max_visibility_batch_size, grid_size.data(),
                                    grid_scale.data(), npol, m.data(), c.data(),
                                    &h)))
    return *e;
  Gridder g;
  g.m_h = h;
  g.m_device = device;
  g.m_max_added_tasks = max_added_tasks;
  g.m_max_batch = max_visibility_batch_size;
  g.m_grid_size = grid_size;
  g.m_grid_scale = grid_scale;
  g.m_npol = npol;
  return g;
}

Gridder::Gridder(Gridder&& o) noexcept { *this = std::move(o); }

Gridder& Gridder::operator=(Gridder&& o) noexcept {
  if (this != &o) {
    if (m_h) hpgb_destroy(m_h);
    m_h = std::exchange(o.m_h, nullptr);
    m_device = o.m_device;
    m_max_added_tasks = o.m_max_added_tasks;
    m_max_batch = o.m_max_batch;
    m_grid_size = o.m_grid_size;
    m_grid_scale = o.m_grid_scale;
    m_npol = o.m_npol;
  }
  return *this;
}

Gridder::Gridder(const Gridder& o)
    : m_device(o.m_device),
      m_max_added_tasks(o.m_max_added_tasks),
      m_max_batch(o.m_max_batch),
      m_grid_size(o.m_grid_size),
      m_grid_scale(o.m_grid_scale),
      m_npol(o.m_npol) {
  if (o.m_h) hpgb_clone(o.m_h, &m_h);
}

Gridder& Gridder::operator=(const Gridder& o) {
  if (this != &o) {
    Gridder tmp(o);
    *this = std::move(tmp);
  }
  return *this;
}

Gridder::~Gridder() {
  if (m_h) hpgb_destroy(m_h);
}

opt_error_t Gridder::set_precision(int precision) {
  return error_of(hpgb_set_precision(m_h, precision));
}

opt_error_t Gridder::set_gridding_kernel(int kind) {
  return error_of(hpgb_set_gridding_kernel(m_h, kind));
}

opt_error_t Gridder::set_tiled_plan(const hpgb_tiled_plan& plan) {
  return error_of(hpgb_set_tiled_plan_ex(m_h, &plan));
}

hpgb_tiled_plan Gridder::tiled_plan() const {
  hpgb_tiled_plan p{0, 0, 0, 0};
  hpgb_get_tiled_plan(m_h, &p);
  return p;
}

int Gridder::last_gridding_kernel() const {
  int k = HPGB_KERNEL_AUTO;
  hpgb_last_gridding_kernel(m_h, &k);
  return k;
}

namespace {
std::vector<unsigned> shape_extents(const CFArrayShape* s) {
  std::vector<unsigned> ext;
  if (!s) return ext;
  for (unsigned g = 0; g < s->num_groups(); ++g) {
    const auto e = s->extents(g);
    ext.insert(ext.end(), e.begin(), e.end());
  }
  return ext;
}
}  // namespace

size_t Gridder::convolution_function_region_size(
    const CFArrayShape* shape) const noexcept {
  size_t n = 0;
  const auto ext = shape_extents(shape);
  hpgb_cf_region_size(m_h, shape ? shape->oversampling() : 0,
                      shape ? shape->num_groups() : 0, ext.data(), &n);
  return n;
}

opt_error_t Gridder::allocate_convolution_function_region(
    const CFArrayShape* shape) {
  const auto ext = shape_extents(shape);
  return error_of(hpgb_allocate_cf_region(m_h, shape ? shape->oversampling() : 0,
                                          shape ? shape->num_groups() : 0,
                                          ext.data()));
}

opt_error_t Gridder::set_convolution_function(const CFArray& cf) {
  // the logical CFArray order, rightmost index fastest: one buffer per group
  // with element (x, y, mueller, cube) at ((x*ny + y)*nm + m)*nc + c
  const unsigned ng = cf.num_groups();
  const auto ext = shape_extents(&cf);
  std::vector<std::vector<std::complex<float>>> bufs(ng);
  std::vector<const void*> ptrs(ng);
  for (unsigned g = 0; g < ng; ++g) {
    const auto e = cf.extents(g);
    auto& b = bufs[g];
    b.resize(size_t(e[0]) * e[1] * e[2] * e[3]);
    size_t k = 0;
    for (unsigned x = 0; x < e[0]; ++x)
      for (unsigned y = 0; y < e[1]; ++y)
        for (unsigned m = 0; m < e[2]; ++m)
          for (unsigned c = 0; c < e[3]; ++c) b[k++] = cf(x, y, m, c, g);
    ptrs[g] = b.data();
  }
  return error_of(hpgb_set_cf(m_h, cf.oversampling(), ng, ext.data(),
                              ptrs.data(), HPGB_CF_LAYOUT_LOGICAL, 0));
}

opt_error_t Gridder::set_model(const GridValueArray& gv) {
  const auto e = gv.extents();
  return error_of(hpgb_set_model(m_h, gv.data(), e.data(), HPGB_LAYOUT_LEFT, 0));
}

opt_error_t Gridder::grid_raw(void* vis, size_t n, unsigned npol,
                              unsigned flags, void* returned) {
  return error_of(hpgb_grid_visibilities(m_h, vis, n, npol, flags, 0, returned));
}

void Gridder::fence() const { hpgb_fence(m_h); }

std::unique_ptr<GridWeightArray> Gridder::grid_weights() const {
  auto w = std::make_unique<GridWeightArray>(m_grid_size[2], m_grid_size[3]);
  hpgb_copy_weights(m_h, w->data(), HPGB_LAYOUT_LEFT);
  return w;
}

std::unique_ptr<GridValueArray> Gridder::grid_values() const {
  auto g = std::make_unique<GridValueArray>(m_grid_size);
  hpgb_copy_grid(m_h, g->data(), HPGB_LAYOUT_LEFT);
  return g;
}

std::unique_ptr<GridValueArray> Gridder::model_values() const {
  auto g = std::make_unique<GridValueArray>(m_grid_size);
  hpgb_copy_model(m_h, g->data(), HPGB_LAYOUT_LEFT);
  return g;
}

void Gridder::reset_grid() { hpgb_reset_grid(m_h); }
void Gridder::reset_model() { hpgb_reset_model(m_h); }

void Gridder::normalize_by_weights(double wfactor) {
  hpgb_normalize_by_weights(m_h, wfactor);
}

opt_error_t Gridder::apply_grid_fft(double norm, FFTSign sign, bool in_place) {
  return error_of(hpgb_apply_grid_fft(m_h, norm, int(sign), in_place));
}

opt_error_t Gridder::apply_model_fft(double norm, FFTSign sign, bool in_place) {
  return error_of(hpgb_apply_model_fft(m_h, norm, int(sign), in_place));
}

void Gridder::shift_grid(ShiftDirection direction) {
  hpgb_shift_grid(m_h, int(direction));
}

void Gridder::shift_model(ShiftDirection direction) {
  hpgb_shift_model(m_h, int(direction));
}

}  // namespace hpgb
