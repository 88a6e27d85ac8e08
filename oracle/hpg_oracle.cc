// hpg_oracle.cc -- CPU restatement of HPG's gridding / degridding arithmetic.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the
// sm_100a device library (hpg_b200/csrc) and the timed CPU baseline of the
// benchmark.  Nothing in the product path links, loads or calls it; only the
// tests, the smoke check and the benchmark's CPU-baseline leg do.
//
// It restates, in plain C++17, the arithmetic of the reference library
// hannajonathan/hpg (v2.0.1):
//   - coordinate math        src/hpg_core.hpp:422-446 (compute_vis_coord)
//   - per-visibility setup   src/hpg_core.hpp:493-550 (Vis ctor)
//   - phase to complex       src/hpg_core.hpp:448-479 (sincos / cphase)
//   - degridding             src/hpg_core.hpp:580-682 (degrid_vis)
//   - gridding (+ weights)   src/hpg_core.hpp:791-886 (grid_vis)
//   - gridding (no weights)  src/hpg_core.hpp:994-1068 (grid_vis_no_weights)
//   - footprint test         src/hpg_core.hpp:1070-1080 (all_within_grid)
//   - launch semantics       src/hpg_core.hpp:1082-1253 (VisibilityGridder::kernel:
//                            degrid -> residual/predicted -> gvis scaling -> grid)
//   - normalisation          src/hpg_core.hpp:1829-1890 (GridNormalizer)
//   - grid shift             src/hpg_core.hpp:2303-2542 (GridShifter)
//   - Mueller index padding  src/hpg_runtime.hpp:1590-1637 (-1 = inactive)
//   - CF radius              src/hpg.hpp:687-694 (CFArray::radii)
//   - cone CF test fixture   tests/GridderStateUnitTests.cc:198-259 (ConeCFArray)
//
// Complex arithmetic follows Kokkos::complex (Kokkos >= 4.0, the reference's
// third-party dependency, not vendored in the reference tree): products are
// (ar*br - ai*bi, ar*bi + ai*br) in the common type of the operands, and
// complex division scales both operands by the 1-norm |yr|+|yi| of the divisor
// before multiplying by the conjugate (Kokkos_Complex.hpp, operator/).
//
// Build with -std=c++17 -ffp-contract=off (the reference builds its host
// devices in ISO mode, CMakeLists.txt:52-59, so GCC does not contract a*b+c).
//
// Summation order: nthreads == 1 reproduces the Kokkos Serial device order
// exactly (visibility-major, then grid row, then X, then Y, then visibility
// polarisation); nthreads > 1 mirrors the reference's OpenMP device (one task
// per visibility and grid row, atomic FP64 accumulation into grid and
// weights), on std::thread workers so that any C++17 compiler builds it.

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

using cf32 = std::complex<float>;
using c64 = std::complex<double>;

constexpr int kPadding = 2;                  // CFArray::padding, src/hpg.hpp:655
constexpr double kLightSpeed = 299792458.0;  // src/hpg_core.hpp:528

// ---------------------------------------------------------------------------
// Kokkos::complex arithmetic, written out so that operation order is explicit

template <typename A, typename B>
inline auto kmul(const std::complex<A>& x, const std::complex<B>& y) {
  using T = std::common_type_t<A, B>;
  T xr = x.real(), xi = x.imag(), yr = y.real(), yi = y.imag();
  return std::complex<T>(xr * yr - xi * yi, xr * yi + xi * yr);
}

template <typename A, typename B>
inline auto kmul_r(const std::complex<A>& x, B y) {
  using T = std::common_type_t<A, B>;
  return std::complex<T>(T(x.real()) * T(y), T(x.imag()) * T(y));
}

inline c64 kdiv(const c64& x, const c64& y) {
  const double s = std::fabs(y.real()) + std::fabs(y.imag());
  if (s == 0.0) return c64(x.real() / s, x.imag() / s);
  const c64 xs(x.real() / s, x.imag() / s);
  const c64 ycs(y.real() / s, -y.imag() / s);
  const double a = ycs.real() * ycs.real() + ycs.imag() * ycs.imag();
  c64 r = kmul(xs, ycs);
  return c64(r.real() / a, r.imag() / a);
}

// cphase(): (cos ph, sin ph), host branch of src/hpg_core.hpp:451-456
inline c64 cphase(double ph) { return c64(std::cos(ph), std::sin(ph)); }

// ---------------------------------------------------------------------------
// VisData<N> binary layout (src/hpg.hpp:236-311); identical to the device ABI

template <int N>
struct VisData {
  float vis[N][2];
  float weights[N];
  double freq;
  double phase;
  double uvw[3];
  unsigned grid_cube;
  unsigned cf_index[2];
  double cf_phase_gradient[2];
};
static_assert(sizeof(VisData<1>) == 88, "VisData<1> layout");
static_assert(sizeof(VisData<2>) == 96, "VisData<2> layout");
static_assert(sizeof(VisData<3>) == 112, "VisData<3> layout");
static_assert(sizeof(VisData<4>) == 120, "VisData<4> layout");

}  // namespace

extern "C" {

// Gridder configuration seen by the oracle.  CF values of group g are
// complex<float> in the CFArray logical index order (x, y, mueller, cube),
// rightmost index fastest: ((x*ext[1] + y)*ext[2] + m)*ext[3] + cube.
struct oracle_params {
  int grid_size[4];          // x, y, mrow, cube
  double grid_scale[2];
  int npol;                  // visibility polarisations N
  int mueller[4][4];         // [mrow][vpol], -1 = inactive
  int conj_mueller[4][4];
  int oversampling;
  int ngroups;
  const unsigned* cf_extents;      // [ngroups][4]
  const float* const* cf_values;   // [ngroups] -> interleaved complex<float>
};

// per-visibility coordinate record, the values the device must reproduce
// bit-for-bit
struct oracle_coords {
  int32_t grid_coord[2];
  int32_t cf_major[2];
  int32_t cf_minor[2];
  int32_t fine_offset[2];
  int32_t cf_size[2];
  int32_t pos_w;
  int32_t in_grid;
  int32_t grid_mueller[4][4];    // Mueller plane of the gridding products
  int32_t degrid_mueller[4][4];  // and of the degridding products
};

}  // extern "C"

namespace {

struct Coord {
  long grid_coord, cf_major, cf_minor, fine_offset;
};

// src/hpg_core.hpp:422-446
inline Coord compute_vis_coord(int g_size, int oversampling, int cf_radius,
                               double coord, double inv_lambda,
                               double grid_scale) {
  const double position = grid_scale * coord * inv_lambda + g_size / 2.0;
  long grid_coord = std::lrint(position);
  const long fine_offset = std::lrint((grid_coord - position) * oversampling);
  grid_coord -= cf_radius;
  long cf_minor, cf_major;
  if (fine_offset >= 0) {
    cf_minor = fine_offset;
    cf_major = kPadding;
  } else {
    cf_minor = oversampling + fine_offset;
    cf_major = kPadding - 1;
  }
  return {grid_coord, cf_major, cf_minor, fine_offset};
}

inline unsigned cf_radius(unsigned ext, unsigned os) {
  // src/hpg.hpp:687-694 (unsigned arithmetic)
  return ((ext - 2 * unsigned(kPadding) * os) / os) / 2;
}

template <int N>
struct Vis {
  int grid_coord[2], cf_minor[2], cf_major[2], fine_offset[2], cf_size[2];
  cf32 values[N];
  float weights[N];
  c64 phasor;
  int grid_cube, cf_cube, cf_grp;
  bool pos_w;
  double phi0[2], dphi[2];
};

// src/hpg_core.hpp:513-550
template <int N>
inline Vis<N> make_vis(const oracle_params& p, const VisData<N>& vd,
                       const cf32* vals) {
  Vis<N> v;
  for (int i = 0; i < N; ++i) {
    v.values[i] = vals[i];
    v.weights[i] = vd.weights[i];
  }
  v.phasor = cphase(vd.phase);
  v.grid_cube = int(vd.grid_cube);
  v.cf_cube = int(vd.cf_index[0]);
  v.cf_grp = int(vd.cf_index[1]);
  v.pos_w = vd.uvw[2] > 0;
  const double inv_lambda = vd.freq / kLightSpeed;
  const unsigned* ext = p.cf_extents + 4 * v.cf_grp;
  for (int d = 0; d < 2; ++d) {
    v.cf_size[d] = 2 * int(cf_radius(ext[d], unsigned(p.oversampling))) + 1;
    Coord c = compute_vis_coord(p.grid_size[d], p.oversampling,
                                v.cf_size[d] / 2, vd.uvw[d], inv_lambda,
                                p.grid_scale[d]);
    v.grid_coord[d] = int(c.grid_coord);
    v.cf_major[d] = int(c.cf_major);
    v.cf_minor[d] = int(c.cf_minor);
    v.fine_offset[d] = int(c.fine_offset);
    v.phi0[d] = -vd.cf_phase_gradient[d] *
                ((v.cf_size[d] / 2) * p.oversampling - v.fine_offset[d]);
    v.dphi[d] = vd.cf_phase_gradient[d] * p.oversampling;
  }
  return v;
}

// src/hpg_core.hpp:1070-1080
template <int N>
inline bool all_within_grid(const Vis<N>& v, const int* gs) {
  return 0 <= v.grid_coord[0] && v.grid_coord[0] + v.cf_size[0] <= gs[0] &&
         0 <= v.grid_coord[1] && v.grid_coord[1] + v.cf_size[1] <= gs[1];
}

// CF value for tap (X, Y) of a visibility, Mueller element m: logical CFArray
// coordinates x = (cf_major + X)*os + cf_minor (the device view indexing of
// src/hpg_core.hpp:623-631 expressed through src/hpg_impl.hpp:1040-1046).
// Coordinates beyond the group's extents read as zero.
template <int N>
inline cf32 cf_at(const oracle_params& p, const Vis<N>& v, int X, int Y,
                  int m) {
  const unsigned* ext = p.cf_extents + 4 * v.cf_grp;
  const long x = long(v.cf_major[0] + X) * p.oversampling + v.cf_minor[0];
  const long y = long(v.cf_major[1] + Y) * p.oversampling + v.cf_minor[1];
  if (x < 0 || y < 0 || x >= long(ext[0]) || y >= long(ext[1])) return cf32(0);
  const size_t idx =
      ((size_t(x) * ext[1] + size_t(y)) * ext[2] + size_t(m)) * ext[3] +
      size_t(v.cf_cube);
  const float* f = p.cf_values[v.cf_grp] + 2 * idx;
  return cf32(f[0], f[1]);
}

inline size_t grid_index(const int* gs, int x, int y, int r, int c) {
  return ((size_t(c) * gs[2] + size_t(r)) * gs[1] + size_t(y)) * gs[0] +
         size_t(x);
}

inline void add_to(double* a, double v, bool atomic) {
  if (atomic) {
    double old;
    __atomic_load(a, &old, __ATOMIC_RELAXED);
    double nw;
    do {
      nw = old + v;
    } while (!__atomic_compare_exchange(a, &old, &nw, true, __ATOMIC_RELAXED,
                                        __ATOMIC_RELAXED));
  } else {
    *a += v;
  }
}

// dynamic-chunk parallel loop over [0, n); sequential, in order, when
// nthreads <= 1
template <typename F>
void parallel_for(long n, int nthreads, long chunk, F&& f) {
  if (nthreads <= 1 || n <= chunk) {
    for (long i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<long> next{0};
  std::vector<std::thread> workers;
  workers.reserve(nthreads);
  for (int t = 0; t < nthreads; ++t)
    workers.emplace_back([&]() {
      for (;;) {
        const long s = next.fetch_add(chunk);
        if (s >= n) break;
        const long e = std::min(n, s + chunk);
        for (long i = s; i < e; ++i) f(i);
      }
    });
  for (auto& w : workers) w.join();
}

// src/hpg_core.hpp:580-682; returns predicted visibilities
template <int N>
void degrid_vis(const oracle_params& p, const Vis<N>& v, const double* model,
                cf32* out) {
  for (int i = 0; i < N; ++i) out[i] = cf32(0);
  if (!model) return;  // model not allocated: prediction is zero (:614)
  const int NX = v.cf_size[0], NY = v.cf_size[1], NR = p.grid_size[2];
  const auto& mi = v.pos_w ? p.conj_mueller : p.mueller;
  const float im_factor = v.pos_w ? 1.0f : -1.0f;
  c64 acc_vis[N], acc_wgt[N];
  for (int i = 0; i < N; ++i) acc_vis[i] = acc_wgt[i] = c64(0);
  std::vector<double> phi_Y(NY);
  for (int Y = 0; Y < NY; ++Y) phi_Y[Y] = v.phi0[1] + Y * v.dphi[1];
  for (int gpol = 0; gpol < NR; ++gpol) {
    c64 va_vis[N], va_wgt[N];
    for (int i = 0; i < N; ++i) va_vis[i] = va_wgt[i] = c64(0);
    for (int X = 0; X < NX; ++X) {
      const double phi_X = v.phi0[0] + X * v.dphi[0];
      for (int Y = 0; Y < NY; ++Y) {
        const c64 screen = cphase(-phi_X - phi_Y[Y]);
        const double* g =
            model + 2 * grid_index(p.grid_size, v.grid_coord[0] + X,
                                   v.grid_coord[1] + Y, gpol, v.grid_cube);
        const c64 mv = kmul(c64(g[0], g[1]), screen);
        for (int vpol = 0; vpol < N; ++vpol) {
          const int m = mi[gpol][vpol];
          if (m >= 0) {
            cf32 cfv = cf_at(p, v, X, Y, m);
            cfv.imag(cfv.imag() * im_factor);
            va_vis[vpol] += kmul(cfv, mv);
            va_wgt[vpol] += c64(cfv.real(), cfv.imag());
          }
        }
      }
    }
    for (int i = 0; i < N; ++i) {
      acc_vis[i] += va_vis[i];
      acc_wgt[i] += va_wgt[i];
    }
  }
  const c64 conj_phasor(v.phasor.real(), -v.phasor.imag());
  for (int i = 0; i < N; ++i) {
    const c64 den = (acc_wgt[i] != c64(0)) ? acc_wgt[i] : c64(1);
    const c64 r = kmul(kdiv(acc_vis[i], den), conj_phasor);
    out[i] = cf32(float(r.real()), float(r.imag()));
  }
}

// src/hpg_core.hpp:791-886 and :994-1068 (one grid row gpol)
template <int N>
void grid_vis(const oracle_params& p, const Vis<N>& v, int gpol, double* grid,
              double* weights, bool update_weights, bool atomic) {
  const int NX = v.cf_size[0], NY = v.cf_size[1];
  const int* mi = (v.pos_w ? p.mueller : p.conj_mueller)[gpol];
  const float im_factor = v.pos_w ? -1.0f : 1.0f;
  std::vector<double> phi_Y(NY);
  for (int Y = 0; Y < NY; ++Y) phi_Y[Y] = v.phi0[1] + Y * v.dphi[1];
  c64 grid_wgt[N];
  for (int i = 0; i < N; ++i) grid_wgt[i] = c64(0);
  for (int X = 0; X < NX; ++X) {
    const double phi_X = v.phi0[0] + X * v.dphi[0];
    for (int Y = 0; Y < NY; ++Y) {
      const c64 sc = cphase(phi_X + phi_Y[Y]);
      const cf32 screen(float(sc.real()), float(sc.imag()));
      c64 gv(0);
      for (int vpol = 0; vpol < N; ++vpol) {
        const int m = mi[vpol];
        if (m >= 0) {
          cf32 cfv = cf_at(p, v, X, Y, m);
          cfv.imag(cfv.imag() * im_factor);
          const cf32 prod = kmul(kmul(cfv, screen), v.values[vpol]);
          gv += c64(prod.real(), prod.imag());
          grid_wgt[vpol] += c64(cfv.real(), cfv.imag());
        }
      }
      double* g = grid + 2 * grid_index(p.grid_size, v.grid_coord[0] + X,
                                        v.grid_coord[1] + Y, gpol, v.grid_cube);
      // pseudo_atomic_add: real and imaginary parts separately (:360-384)
      add_to(g, gv.real(), atomic);
      add_to(g + 1, gv.imag(), atomic);
    }
  }
  if (update_weights) {
    double twgt = 0;
    for (int i = 0; i < N; ++i)
      twgt += double(std::hypot(grid_wgt[i].real(), grid_wgt[i].imag()) *
                     v.weights[i]);
    add_to(weights + size_t(v.grid_cube) * p.grid_size[2] + gpol, twgt,
           atomic);
  }
}

// src/hpg_core.hpp:1082-1253, for one batch of VisData<N>
template <int N>
void grid_visibilities(const oracle_params& p, VisData<N>* vis, size_t n,
                       bool update_weights, bool do_degrid, bool return_vis,
                       bool do_grid, double* grid, double* weights,
                       const double* model, int nthreads) {
  std::vector<cf32> gvis(n * N);
  std::vector<VisData<N>> work(vis, vis + n);
  const bool atomic = nthreads > 1;
  if (do_degrid) {
    parallel_for(long(n), nthreads, 64, [&](long i) {
      VisData<N>& vd = work[i];
      cf32 vals[N];
      for (int k = 0; k < N; ++k) vals[k] = cf32(vd.vis[k][0], vd.vis[k][1]);
      const Vis<N> v = make_vis<N>(p, vd, vals);
      if (!all_within_grid(v, p.grid_size)) return;
      cf32 pred[N];
      degrid_vis<N>(p, v, model, pred);
      for (int k = 0; k < N; ++k) {
        if (do_grid) {
          // residual, then rescale for gridding (:1153-1159)
          cf32 r = vals[k] - pred[k];
          vd.vis[k][0] = r.real();
          vd.vis[k][1] = r.imag();
          const c64 g = kmul_r(kmul(r, v.phasor), v.weights[k]);
          gvis[i * N + k] = cf32(float(g.real()), float(g.imag()));
        } else {
          vd.vis[k][0] = pred[k].real();
          vd.vis[k][1] = pred[k].imag();
        }
      }
    });
  } else {
    // "gvis_init" (:1171-1183)
    parallel_for(long(n), nthreads, 4096, [&](long i) {
      const VisData<N>& vd = work[i];
      const c64 phasor = cphase(vd.phase);
      for (int k = 0; k < N; ++k) {
        const cf32 val(vd.vis[k][0], vd.vis[k][1]);
        const c64 g = kmul_r(kmul(val, phasor), vd.weights[k]);
        gvis[i * N + k] = cf32(float(g.real()), float(g.imag()));
      }
    });
  }
  if (do_grid) {
    const int NR = p.grid_size[2];
    parallel_for(long(n) * NR, nthreads, 16, [&](long t) {
      const long i = t / NR;
      const int gpol = int(t % NR);
      const Vis<N> v = make_vis<N>(p, work[i], &gvis[i * N]);
      if (!all_within_grid(v, p.grid_size)) return;
      grid_vis<N>(p, v, gpol, grid, weights, update_weights, atomic);
    });
  }
  if (return_vis)
    std::memcpy(static_cast<void*>(vis), work.data(), n * sizeof(VisData<N>));
}

// Degridding normaliser of each visibility polarization, the den of
// degrid_vis (src/hpg_core.hpp:598-600, :659-661): the sum over grid rows
// and footprint of the degridding CF, 1 where that sum is 0 or the
// visibility is off the grid.  out: complex<double> [n][N].
template <int N>
void normalisers(const oracle_params& p, const VisData<N>* vis, size_t n,
                 double* out) {
  for (size_t i = 0; i < n; ++i) {
    cf32 vals[N];
    const Vis<N> v = make_vis<N>(p, vis[i], vals);
    c64 den[N];
    for (int k = 0; k < N; ++k) den[k] = c64(0);
    if (all_within_grid(v, p.grid_size)) {
      const auto& mi = v.pos_w ? p.conj_mueller : p.mueller;
      const float im_factor = v.pos_w ? 1.0f : -1.0f;
      for (int gpol = 0; gpol < p.grid_size[2]; ++gpol)
        for (int X = 0; X < v.cf_size[0]; ++X)
          for (int Y = 0; Y < v.cf_size[1]; ++Y)
            for (int k = 0; k < N; ++k) {
              const int m = mi[gpol][k];
              if (m >= 0) {
                cf32 cfv = cf_at(p, v, X, Y, m);
                cfv.imag(cfv.imag() * im_factor);
                den[k] += c64(cfv.real(), cfv.imag());
              }
            }
    }
    for (int k = 0; k < N; ++k) {
      const c64 d = den[k] != c64(0) ? den[k] : c64(1);
      out[2 * (i * N + k)] = d.real();
      out[2 * (i * N + k) + 1] = d.imag();
    }
  }
}

template <int N>
void coords(const oracle_params& p, const VisData<N>* vis, size_t n,
            oracle_coords* out) {
  for (size_t i = 0; i < n; ++i) {
    cf32 vals[N];
    const Vis<N> v = make_vis<N>(p, vis[i], vals);
    oracle_coords& o = out[i];
    for (int d = 0; d < 2; ++d) {
      o.grid_coord[d] = v.grid_coord[d];
      o.cf_major[d] = v.cf_major[d];
      o.cf_minor[d] = v.cf_minor[d];
      o.fine_offset[d] = v.fine_offset[d];
      o.cf_size[d] = v.cf_size[d];
    }
    o.pos_w = v.pos_w;
    o.in_grid = all_within_grid(v, p.grid_size);
    // Mueller routing: src/hpg_core.hpp:808-817 (gridding), :598-600
    // (degridding)
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        o.grid_mueller[r][c] = (v.pos_w ? p.mueller : p.conj_mueller)[r][c];
        o.degrid_mueller[r][c] = (v.pos_w ? p.conj_mueller : p.mueller)[r][c];
      }
  }
}

}  // namespace

extern "C" {

int oracle_num_threads(void) {
  const unsigned n = std::thread::hardware_concurrency();
  return n > 0 ? int(n) : 1;
}

// Per-visibility coordinates (src/hpg_core.hpp:493-550).
int oracle_vis_coords(const oracle_params* p, const void* vis, size_t n,
                      int npol, oracle_coords* out) {
  switch (npol) {
    case 1: coords<1>(*p, static_cast<const VisData<1>*>(vis), n, out); break;
    case 2: coords<2>(*p, static_cast<const VisData<2>*>(vis), n, out); break;
    case 3: coords<3>(*p, static_cast<const VisData<3>*>(vis), n, out); break;
    case 4: coords<4>(*p, static_cast<const VisData<4>*>(vis), n, out); break;
    default: return -1;
  }
  return 0;
}

// Degridding normalisers, complex<double> [n][npol] (see normalisers()).
int oracle_normalisers(const oracle_params* p, const void* vis, size_t n,
                       int npol, double* out) {
  switch (npol) {
    case 1: normalisers<1>(*p, static_cast<const VisData<1>*>(vis), n, out); break;
    case 2: normalisers<2>(*p, static_cast<const VisData<2>*>(vis), n, out); break;
    case 3: normalisers<3>(*p, static_cast<const VisData<3>*>(vis), n, out); break;
    case 4: normalisers<4>(*p, static_cast<const VisData<4>*>(vis), n, out); break;
    default: return -1;
  }
  return 0;
}

// One call of VisibilityGridder<N>::kernel (src/hpg_core.hpp:1082-1253) on a
// batch.  grid, model: complex<double> [cube][mrow][y][x] (x fastest);
// weights: double [cube][mrow]; model may be NULL (no model set).  When
// return_vis is set, the (residual or predicted) visibility values are written
// back into vis.
int oracle_grid_visibilities(const oracle_params* p, void* vis, size_t n,
                             int npol, int update_weights, int do_degrid,
                             int return_vis, int do_grid, double* grid,
                             double* weights, const double* model,
                             int nthreads) {
#define HPG_ORACLE_CASE(N)                                                   \
  case N:                                                                    \
    grid_visibilities<N>(*p, static_cast<VisData<N>*>(vis), n,              \
                         update_weights != 0, do_degrid != 0,               \
                         return_vis != 0, do_grid != 0, grid, weights,      \
                         model, nthreads);                                   \
    break;
  switch (npol) {
    HPG_ORACLE_CASE(1)
    HPG_ORACLE_CASE(2)
    HPG_ORACLE_CASE(3)
    HPG_ORACLE_CASE(4)
    default: return -1;
  }
#undef HPG_ORACLE_CASE
  return 0;
}

// GridNormalizer, weights form (src/hpg_core.hpp:1832-1861)
void oracle_normalize_by_weights(double* grid, const double* weights,
                                 const int* gs, double wfactor) {
  for (int c = 0; c < gs[3]; ++c)
    for (int r = 0; r < gs[2]; ++r) {
      const double d = wfactor * weights[size_t(c) * gs[2] + r];
      for (int y = 0; y < gs[1]; ++y)
        for (int x = 0; x < gs[0]; ++x) {
          double* g = grid + 2 * grid_index(gs, x, y, r, c);
          g[0] /= d;
          g[1] /= d;
        }
    }
}

// GridNormalizer, norm form (src/hpg_core.hpp:1863-1889)
void oracle_normalize(double* grid, const int* gs, double norm) {
  const double inv = 1.0 / norm;
  const size_t n = size_t(gs[0]) * gs[1] * gs[2] * gs[3];
  for (size_t i = 0; i < 2 * n; ++i) grid[i] *= inv;
}

// GridShifter (src/hpg_core.hpp:2303-2542): the reference's in-place swap and
// rotation loops, planes processed one after another.  direction 0 = FORWARD,
// 1 = BACKWARD.
void oracle_shift(double* grid, const int* gs, int direction) {
  const int nx = gs[0], ny = gs[1];
  const int mx = nx / 2, my = ny / 2;
  auto at = [&](double* pl, int x, int y) -> c64* {
    return reinterpret_cast<c64*>(pl) + size_t(y) * nx + x;
  };
  for (int c = 0; c < gs[3]; ++c)
    for (int r = 0; r < gs[2]; ++r) {
      double* pl = grid + 2 * grid_index(gs, 0, 0, r, c);
      if (nx % 2 == 0 && ny % 2 == 0) {
        for (int x = 0; x < nx / 2; ++x)
          for (int y = 0; y < ny / 2; ++y) {
            std::swap(*at(pl, x, y), *at(pl, x + mx, y + my));
            std::swap(*at(pl, x + mx, y), *at(pl, x, y + my));
          }
      } else if (nx == ny) {
        for (int x0 = 0; x0 < nx; ++x0) {
          c64 tmp(0);
          int x = x0, y = 0;
          for (int i = 0; i <= ny; ++i) {
            std::swap(tmp, *at(pl, x, y));
            if (direction == 0) {
              x += mx; if (x >= nx) x -= nx;
              y += my; if (y >= ny) y -= ny;
            } else {
              x -= mx; if (x < 0) x += nx;
              y -= my; if (y < 0) y += ny;
            }
          }
        }
      } else {
        // first pass along y, for each x
        for (int x = 0; x < nx; ++x) {
          if (ny % 2 == 1) {
            c64 tmp(0);
            int y = 0;
            for (int i = 0; i <= ny; ++i) {
              std::swap(tmp, *at(pl, x, y));
              if (direction == 0) { y += my; if (y >= ny) y -= ny; }
              else { y -= my; if (y < 0) y += ny; }
            }
          } else if (direction == 0) {
            for (int y = 0; y < my; ++y) std::swap(*at(pl, x, y), *at(pl, x, y + my));
          } else {
            for (int y = my; y < ny; ++y) std::swap(*at(pl, x, y), *at(pl, x, y - my));
          }
        }
        // second pass along x, for each y
        for (int y = 0; y < ny; ++y) {
          if (nx % 2 == 1) {
            c64 tmp(0);
            int x = 0;
            for (int i = 0; i <= nx; ++i) {
              std::swap(tmp, *at(pl, x, y));
              if (direction == 0) { x += mx; if (x >= nx) x -= nx; }
              else { x -= mx; if (x < 0) x += nx; }
            }
          } else if (direction == 0) {
            for (int x = 0; x < mx; ++x) std::swap(*at(pl, x, y), *at(pl, x + mx, y));
          } else {
            for (int x = mx; x < nx; ++x) std::swap(*at(pl, x, y), *at(pl, x - mx, y));
          }
        }
      }
    }
}

// ConeCFArray::operator() of the reference's unit tests
// (tests/GridderStateUnitTests.cc:198-259), host float arithmetic through
// std::polar / std::abs / std::arg.  Writes the one-group CF in the logical
// (x, y, mueller, cube=1) order used by oracle_params.
void oracle_cone_cf(unsigned nmueller, unsigned oversampling, unsigned radius,
                    float* out) {
  const int osr = int((radius + kPadding) * oversampling);
  const unsigned w = 2 * unsigned(osr) + 1;
  for (unsigned x = 0; x < w; ++x)
    for (unsigned y = 0; y < w; ++y)
      for (unsigned m = 0; m < nmueller; ++m) {
        std::complex<float> pt((-osr + int(x)) + 0.5f, (-osr + int(y)) + 0.5f);
        using namespace std::complex_literals;
        const std::complex<float> v = std::polar(
            (m + 1) * std::max(osr - std::abs(pt), 0.0f),
            std::arg(std::abs(pt.real()) + 1.0if * std::abs(pt.imag())));
        const size_t idx = (size_t(x) * w + y) * nmueller + m;
        out[2 * idx] = v.real();
        out[2 * idx + 1] = v.imag();
      }
}

}  // extern "C"
