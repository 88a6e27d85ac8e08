// gridder.hpp -- C++ host API of the B200 gridding library, over the C ABI
// of include/hpgb.h.
//
// It mirrors the value API of the reference's hpg::Gridder
// (src/hpg.hpp:2206-2700, src/hpg.cc:974-1400) for the gridding path: the
// same names, argument meanings and error behaviour (errors are values,
// hpg::ErrorType order), so that code written against hpg::Gridder reads
// the same against hpgb::Gridder:
//
//   auto g = hpgb::Gridder::create(0, 0, batch, grid_size, grid_scale,
//                                  mueller, conj_mueller);
//   g.set_convolution_function(cf);           // an hpgb::CFArray
//   g.set_model(model);                       // hpgb::GridValueArray
//   g.degrid_grid_visibilities(std::move(vis));
//   g.normalize_by_weights();
//   g.apply_grid_fft();
//   g.shift_grid();
//   auto grid = g.grid_values();
#pragma once

#include <array>
#include <complex>
#include <memory>
#include <optional>
#include <string>
#include <type_traits>
#include <utility>
#include <variant>
#include <vector>

#include "hpgb.h"

namespace hpgb {

// hpg::ErrorType (src/hpg_error.hpp:26-38)
enum class ErrorType {
  DisabledDevice,
  DisabledHostDevice,
  OutOfBoundsCFIndex,
  InvalidNumberMuellerIndexRows,
  InvalidNumberPolarizations,
  InvalidCFLayout,
  InvalidModelGridSize,
  ExcessiveNumberVisibilities,
  UpdateWeightsWithoutGridding,
  CFSupportExceedsGrid,
  Other
};

// hpg::Error (src/hpg_error.hpp:43-75)
class Error {
 public:
  Error(std::string msg, ErrorType type = ErrorType::Other)
      : m_msg(std::move(msg)), m_type(type) {}
  const std::string& message() const { return m_msg; }
  ErrorType type() const { return m_type; }

 private:
  std::string m_msg;
  ErrorType m_type;
};

// hpg::rval_t (src/hpg_rval.hpp:35): a value or an error
template <typename T>
using rval_t = std::variant<Error, T>;
using opt_error_t = std::optional<Error>;

template <typename T>
bool is_value(const rval_t<T>& r) {
  return std::holds_alternative<T>(r);
}
template <typename T>
T& get_value(rval_t<T>& r) {
  return std::get<T>(r);
}
template <typename T>
const Error& get_error(const rval_t<T>& r) {
  return std::get<Error>(r);
}

// hpg::Layout, hpg::FFTSign, hpg::ShiftDirection (src/hpg.hpp:611-614,
// :965-968, :989-992)
enum class Layout { Right = HPGB_LAYOUT_RIGHT, Left = HPGB_LAYOUT_LEFT };
enum class FFTSign { POSITIVE = HPGB_FFT_POSITIVE, NEGATIVE = HPGB_FFT_NEGATIVE };
enum class ShiftDirection { FORWARD = HPGB_SHIFT_FORWARD, BACKWARD = HPGB_SHIFT_BACKWARD };

// hpg::VisData<N> (src/hpg.hpp:236-311): the C records of include/hpgb.h
template <unsigned N> struct VisDataOf;
template <> struct VisDataOf<1> { using type = hpgb_visdata1; };
template <> struct VisDataOf<2> { using type = hpgb_visdata2; };
template <> struct VisDataOf<3> { using type = hpgb_visdata3; };
template <> struct VisDataOf<4> { using type = hpgb_visdata4; };
template <unsigned N>
using VisData = typename VisDataOf<N>::type;
// the polarization count of a record type
template <typename V> struct VisNpol;
template <> struct VisNpol<hpgb_visdata1> { static constexpr unsigned value = 1; };
template <> struct VisNpol<hpgb_visdata2> { static constexpr unsigned value = 2; };
template <> struct VisNpol<hpgb_visdata3> { static constexpr unsigned value = 3; };
template <> struct VisNpol<hpgb_visdata4> { static constexpr unsigned value = 4; };

// hpg::CFArrayShape / hpg::CFArray (src/hpg.hpp:615-704): extents in
// oversampled units including the two-cell padding on each edge, element
// access by (x, y, mueller, cube, group)
class CFArrayShape {
 public:
  virtual unsigned oversampling() const = 0;
  virtual unsigned num_groups() const = 0;
  virtual std::array<unsigned, 4> extents(unsigned grp) const = 0;
  virtual ~CFArrayShape() = default;
};

class CFArray : public CFArrayShape {
 public:
  static constexpr unsigned padding = 2;
  virtual std::complex<float> operator()(unsigned x, unsigned y,
                                         unsigned mueller, unsigned cube,
                                         unsigned grp) const = 0;
  std::array<unsigned, 2> radii(unsigned grp) const {
    const unsigned os = oversampling();
    const auto ext = extents(grp);
    return {((ext[0] - 2 * padding * os) / os) / 2,
            ((ext[1] - 2 * padding * os) / os) / 2};
  }
};

// hpg::GridValueArray / GridWeightArray (src/hpg.hpp:780-960): host copies
// with element access (x, y, mrow, cube) and (mrow, cube)
class GridValueArray {
 public:
  GridValueArray(std::array<unsigned, 4> ext)
      : m_ext(ext), m_v(size_t(ext[0]) * ext[1] * ext[2] * ext[3]) {}
  std::complex<double>& operator()(unsigned x, unsigned y, unsigned mrow,
                                   unsigned cube) {
    return m_v[index(x, y, mrow, cube)];
  }
  const std::complex<double>& operator()(unsigned x, unsigned y,
                                         unsigned mrow, unsigned cube) const {
    return m_v[index(x, y, mrow, cube)];
  }
  std::array<unsigned, 4> extents() const { return m_ext; }
  // [cube][mrow][y][x], x fastest (Layout::Left)
  std::complex<double>* data() { return m_v.data(); }
  const std::complex<double>* data() const { return m_v.data(); }
  size_t size() const { return m_v.size(); }

 private:
  size_t index(unsigned x, unsigned y, unsigned mrow, unsigned cube) const {
    return ((size_t(cube) * m_ext[2] + mrow) * m_ext[1] + y) * m_ext[0] + x;
  }
  std::array<unsigned, 4> m_ext;
  std::vector<std::complex<double>> m_v;
};

class GridWeightArray {
 public:
  GridWeightArray(unsigned nrow, unsigned ncube)
      : m_nrow(nrow), m_v(size_t(nrow) * ncube) {}
  double operator()(unsigned mrow, unsigned cube) const {
    return m_v[size_t(cube) * m_nrow + mrow];
  }
  double* data() { return m_v.data(); }
  size_t size() const { return m_v.size(); }

 private:
  unsigned m_nrow;
  std::vector<double> m_v;
};

// hpg::future (src/hpg.hpp:167-210): the value is ready after a fence
template <typename T>
class future {
 public:
  future() = default;
  future(hpgb_gridder* g, std::shared_ptr<T> value)
      : m_g(g), m_value(std::move(value)) {}
  T& get() {
    if (m_g) hpgb_fence(m_g);
    return *m_value;
  }

 private:
  hpgb_gridder* m_g = nullptr;
  std::shared_ptr<T> m_value;
};

// hpg::Gridder: a mutable gridder on one B200
class Gridder {
 public:
  // Gridder::create (src/hpg.hpp:2265-2300, GridderState::create
  // src/hpg.cc:226-264)
  static rval_t<Gridder> create(
      int device, unsigned max_added_tasks, size_t max_visibility_batch_size,
      const std::array<unsigned, 4>& grid_size,
      const std::array<double, 2>& grid_scale,
      const std::vector<std::vector<int>>& mueller_indexes,
      const std::vector<std::vector<int>>& conjugate_mueller_indexes);

  Gridder() = default;
  Gridder(Gridder&&) noexcept;
  Gridder& operator=(Gridder&&) noexcept;
  Gridder(const Gridder&);             // deep copy after a fence
  Gridder& operator=(const Gridder&);
  ~Gridder();

  bool is_null() const noexcept { return m_h == nullptr; }
  int device() const noexcept { return m_device; }
  unsigned max_added_tasks() const noexcept { return m_max_added_tasks; }
  size_t max_visibility_batch_size() const noexcept { return m_max_batch; }
  std::array<unsigned, 4> grid_size() const noexcept { return m_grid_size; }
  std::array<double, 2> grid_scale() const noexcept { return m_grid_scale; }
  unsigned num_polarizations() const noexcept { return m_npol; }

  // choice of arithmetic and kernels (no counterpart in the reference)
  opt_error_t set_precision(int precision);
  opt_error_t set_gridding_kernel(int kind);
  // the tiled kernel's plan (hpgb_set_tiled_plan_ex) and the kernel that
  // took the last batch (hpgb_last_gridding_kernel)
  opt_error_t set_tiled_plan(const hpgb_tiled_plan& plan);
  hpgb_tiled_plan tiled_plan() const;
  int last_gridding_kernel() const;

  size_t convolution_function_region_size(const CFArrayShape* shape) const noexcept;
  opt_error_t allocate_convolution_function_region(const CFArrayShape* shape);
  opt_error_t set_convolution_function(const CFArray& cf);
  opt_error_t set_model(const GridValueArray& gv);

  template <typename V>
  opt_error_t grid_visibilities(std::vector<V>&& vis,
                                bool update_grid_weights = true) {
    return grid_raw(vis.data(), vis.size(), VisNpol<V>::value,
                    HPGB_DO_GRID | (update_grid_weights ? HPGB_UPDATE_GRID_WEIGHTS : 0),
                    nullptr);
  }
  template <typename V>
  opt_error_t degrid_grid_visibilities(std::vector<V>&& vis,
                                       bool update_grid_weights = true) {
    return grid_raw(vis.data(), vis.size(), VisNpol<V>::value,
                    HPGB_DO_DEGRID | HPGB_DO_GRID |
                        (update_grid_weights ? HPGB_UPDATE_GRID_WEIGHTS : 0),
                    nullptr);
  }
  template <typename V>
  rval_t<future<std::vector<V>>> degrid_get_predicted_visibilities(
      std::vector<V>&& vis) {
    return returning(std::move(vis), HPGB_DO_DEGRID | HPGB_RETURN_VISIBILITIES);
  }
  template <typename V>
  rval_t<future<std::vector<V>>> degrid_grid_get_residual_visibilities(
      std::vector<V>&& vis, bool update_grid_weights = true) {
    return returning(std::move(vis),
                     HPGB_DO_DEGRID | HPGB_DO_GRID | HPGB_RETURN_VISIBILITIES |
                         (update_grid_weights ? HPGB_UPDATE_GRID_WEIGHTS : 0));
  }

  void fence() const;
  std::unique_ptr<GridWeightArray> grid_weights() const;
  std::unique_ptr<GridValueArray> grid_values() const;
  std::unique_ptr<GridValueArray> model_values() const;
  void reset_grid();
  void reset_model();
  void normalize_by_weights(double wfactor = 1.0);
  opt_error_t apply_grid_fft(double norm = 1.0, FFTSign sign = FFTSign::POSITIVE,
                             bool in_place = true);
  opt_error_t apply_model_fft(double norm = 1.0, FFTSign sign = FFTSign::NEGATIVE,
                              bool in_place = true);
  void shift_grid(ShiftDirection direction = ShiftDirection::FORWARD);
  void shift_model(ShiftDirection direction = ShiftDirection::FORWARD);

  hpgb_gridder* handle() const { return m_h; }

 private:
  opt_error_t grid_raw(void* vis, size_t n, unsigned npol, unsigned flags,
                       void* returned);
  template <typename V>
  rval_t<future<std::vector<V>>> returning(std::vector<V>&& vis,
                                           unsigned flags) {
    auto out = std::make_shared<std::vector<V>>(std::move(vis));
    auto err = grid_raw(out->data(), out->size(), VisNpol<V>::value, flags,
                        out->data());
    if (err) return *err;
    return future<std::vector<V>>(m_h, out);
  }

  hpgb_gridder* m_h = nullptr;
  int m_device = 0;
  unsigned m_max_added_tasks = 0;
  size_t m_max_batch = 0;
  std::array<unsigned, 4> m_grid_size{};
  std::array<double, 2> m_grid_scale{};
  unsigned m_npol = 0;
};

// the error of a status code (nullopt for success)
opt_error_t error_of(int status);

// The batches of many gridders in one launch of the tiled kernel
// (hpgb_grid_visibilities_batch; no counterpart in the reference):
// gridders[j] grids batches[j] as its grid_visibilities /
// degrid_grid_visibilities would.  The gridders share polarizations, grid
// rows, Mueller tables and arithmetic form; grids, CFs and batch sizes may
// differ.  The work runs on gridders[0]'s stream; fence it for the results.
template <typename V>
opt_error_t grid_visibilities_batch(const std::vector<Gridder*>& gridders,
                                    std::vector<std::vector<V>>& batches,
                                    bool do_degrid = false,
                                    bool update_grid_weights = true) {
  if (gridders.size() != batches.size())
    return Error("one batch per gridder", ErrorType::Other);
  std::vector<hpgb_gridder*> hs;
  std::vector<const void*> vs;
  std::vector<size_t> ns;
  for (size_t j = 0; j < gridders.size(); ++j) {
    hs.push_back(gridders[j]->handle());
    vs.push_back(batches[j].data());
    ns.push_back(batches[j].size());
  }
  const unsigned flags = HPGB_DO_GRID | (do_degrid ? HPGB_DO_DEGRID : 0) |
                         (update_grid_weights ? HPGB_UPDATE_GRID_WEIGHTS : 0);
  return error_of(hpgb_grid_visibilities_batch(
      hs.data(), hs.size(), vs.data(), ns.data(), VisNpol<V>::value, flags, 0,
      nullptr));
}

}  // namespace hpgb
