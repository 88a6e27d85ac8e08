// common.cuh -- types and exact-rounding helpers shared by the hpgb kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "hpgb.h"

namespace hpgb {

// ---------------------------------------------------------------------------
// error plumbing (host)

void set_last_error(const std::string& msg);

struct Status {
  int code = HPGB_SUCCESS;
  std::string msg;
  static Status ok() { return Status(); }
  static Status err(int c, std::string m) { Status s; s.code = c; s.msg = std::move(m); return s; }
  explicit operator bool() const { return code == HPGB_SUCCESS; }
};

#define HPGB_CUDA_TRY(expr)                                                  \
  do {                                                                       \
    cudaError_t hpgb_e_ = (expr);                                            \
    if (hpgb_e_ != cudaSuccess)                                              \
      return ::hpgb::Status::err(                                            \
          HPGB_ERROR_OTHER, std::string(#expr " failed: ") +                 \
                                cudaGetErrorString(hpgb_e_));                \
  } while (0)

#define HPGB_TRY(expr)                                                       \
  do {                                                                       \
    ::hpgb::Status hpgb_s_ = (expr);                                         \
    if (!hpgb_s_) return hpgb_s_;                                            \
  } while (0)

// ---------------------------------------------------------------------------
// visibility record, byte-identical to hpg::VisData<N> (src/hpg.hpp:236-311)

template <int N>
struct VisData {
  float2 vis[N];
  float weights[N];
  double freq;
  double phase;
  double uvw[3];
  unsigned grid_cube;
  unsigned cf_index[2];
  double cf_phase_gradient[2];
};
static_assert(sizeof(VisData<1>) == sizeof(hpgb_visdata1), "VisData<1>");
static_assert(sizeof(VisData<2>) == sizeof(hpgb_visdata2), "VisData<2>");
static_assert(sizeof(VisData<3>) == sizeof(hpgb_visdata3), "VisData<3>");
static_assert(sizeof(VisData<4>) == sizeof(hpgb_visdata4), "VisData<4>");
static_assert(sizeof(VisData<4>) == 120, "VisData<4>");

inline size_t visdata_size(unsigned npol) {
  switch (npol) {
    case 1: return sizeof(VisData<1>);
    case 2: return sizeof(VisData<2>);
    case 3: return sizeof(VisData<3>);
    case 4: return sizeof(VisData<4>);
    default: return 0;
  }
}

// ---------------------------------------------------------------------------
// device-resident CF group descriptor
//
// Device CF layout (this library's own, layout version 1): for each group, a
// table of "slices", one per (cube, fine_y, fine_x) with fine = fine_offset +
// os/2 in [0, nfine), nfine = 2*(os/2) + 1.  A slice holds every value one
// visibility reads: [mueller][Y][X] complex<float>, Y < taps_y, X < taps_x,
// value = CF(x = (2 + X)*os + fine_offset_x, y = (2 + Y)*os + fine_offset_y),
// i.e. the reference's (cf_major + X, cf_minor) indexing of
// src/hpg_core.hpp:623-631 with both cf_major branches folded into the fine
// offset.  Each Mueller plane is padded to an even number of elements, so
// every plane and every slice starts 16-byte aligned and is a whole number of
// 16-byte units (the unit of bulk copies).  wsum holds, per slice and Mueller element, the FP64 sum
// of the slice's CF values (the visibility-independent part of both the
// degridding normaliser and the gridding weight).

struct CFGroup {
  const float2* data;      // slices
  const double2* wsum;     // [slice][mueller]
  int taps_x, taps_y;      // 2*radius + 1
  int nmueller, ncube;
  int plane_stride;        // float2 elements per Mueller plane (even)
  long long slice_stride;  // float2 elements per slice = nmueller*plane_stride
};

struct MuellerTables {
  int m[4][4];   // mueller_indexes, -1 padded (src/hpg_runtime.hpp:1590-1637)
  int c[4][4];   // conjugate_mueller_indexes
};

// Parameters every gridding kernel launch needs, passed by value.
struct GridGeom {
  int nx, ny, nrow, ncube;
  double scale_x, scale_y;
  int os, nfine;
  int ngroups;
  MuellerTables mt;
  unsigned* status;  // device word; bit 0 set when a visibility's cf_index or
                     // grid_cube is out of range (the visibility is skipped)
};

enum : unsigned { kStatusBadIndex = 1u, kStatusWaitTimeout = 2u };

// ---------------------------------------------------------------------------
// exact-rounding arithmetic: every operation rounds once, no FMA contraction,
// operand order as in Kokkos::complex (the reference's complex type)

__device__ __forceinline__ float2 cmul_f(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

__device__ __forceinline__ double2 cmul_d(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

__device__ __forceinline__ double2 cadd_d(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}

// Kokkos::complex division: scale by the 1-norm of the divisor, multiply by
// its conjugate, divide by the squared magnitude.
__device__ __forceinline__ double2 cdiv_d(double2 x, double2 y) {
  const double s = __dadd_rn(fabs(y.x), fabs(y.y));
  if (s == 0.0) return make_double2(__ddiv_rn(x.x, s), __ddiv_rn(x.y, s));
  const double2 xs = make_double2(__ddiv_rn(x.x, s), __ddiv_rn(x.y, s));
  const double2 ys = make_double2(__ddiv_rn(y.x, s), __ddiv_rn(-y.y, s));
  const double a = __dadd_rn(__dmul_rn(ys.x, ys.x), __dmul_rn(ys.y, ys.y));
  const double2 r = cmul_d(xs, ys);
  return make_double2(__ddiv_rn(r.x, a), __ddiv_rn(r.y, a));
}

// cphase(): (cos ph, sin ph) (src/hpg_core.hpp:473-479)
__device__ __forceinline__ double2 cphase_d(double ph) {
  double s, c;
  sincos(ph, &s, &c);
  return make_double2(c, s);
}

// gvis = complex<float>((value * phasor) * weight): complex<float> times
// complex<double> in double, times float weight in double, rounded to float
// (src/hpg_core.hpp:1155-1158, :1179-1180)
__device__ __forceinline__ float2 scale_for_gridding(float2 v, double2 phasor,
                                                     float w) {
  const double2 p = cmul_d(make_double2(v.x, v.y), phasor);
  const double wd = w;
  return make_float2(__double2float_rn(__dmul_rn(p.x, wd)),
                     __double2float_rn(__dmul_rn(p.y, wd)));
}

// ---------------------------------------------------------------------------
// per-visibility coordinates, bit-exact with compute_vis_coord()
// (src/hpg_core.hpp:422-446) and the Vis constructor (:513-550)

struct VisCoord {
  int grid_coord[2];
  int cf_major[2];
  int cf_minor[2];
  int fine[2];
  int taps[2];
  bool pos_w;
  bool in_grid;
  int grp, cf_cube, grid_cube;
  double phi0[2], dphi[2];
};

__device__ __forceinline__ void vis_coords(const GridGeom& g,
                                           const CFGroup* groups, double freq,
                                           const double* uvw, unsigned gcube,
                                           const unsigned* cfi,
                                           const double* grad, VisCoord& vc) {
  const double inv_lambda = __ddiv_rn(freq, 299792458.0);
  vc.grp = int(cfi[1]);
  vc.cf_cube = int(cfi[0]);
  vc.grid_cube = int(gcube);
  vc.pos_w = uvw[2] > 0;
  // index checks the reference leaves to the caller
  // (src/hpg_runtime.hpp:1093-1100): an out-of-range index skips the
  // visibility and flags the gridder's status word instead of reading
  // outside the CF or grid
  if (cfi[1] >= unsigned(g.ngroups) || gcube >= unsigned(g.ncube) ||
      cfi[0] >= unsigned(groups[cfi[1]].ncube)) {
    vc.in_grid = false;
    for (int d = 0; d < 2; ++d) {
      vc.grid_coord[d] = vc.cf_major[d] = vc.cf_minor[d] = vc.fine[d] = 0;
      vc.taps[d] = 0;
      vc.phi0[d] = vc.dphi[d] = 0.0;
    }
    if (g.status) atomicOr(g.status, kStatusBadIndex);
    return;
  }
  const CFGroup& G = groups[vc.grp];
  const int gsz[2] = {g.nx, g.ny};
  const double scl[2] = {g.scale_x, g.scale_y};
  const int taps[2] = {G.taps_x, G.taps_y};
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const int radius = taps[d] / 2;
    const double position =
        __dadd_rn(__dmul_rn(__dmul_rn(scl[d], uvw[d]), inv_lambda),
                  double(gsz[d]) / 2.0);
    long long gc = __double2ll_rn(position);
    const long long fo = __double2ll_rn(
        __dmul_rn(__dsub_rn(double(gc), position), double(g.os)));
    gc -= radius;
    vc.taps[d] = taps[d];
    vc.grid_coord[d] = int(gc);
    vc.fine[d] = int(fo);
    if (fo >= 0) {
      vc.cf_minor[d] = int(fo);
      vc.cf_major[d] = 2;
    } else {
      vc.cf_minor[d] = g.os + int(fo);
      vc.cf_major[d] = 1;
    }
    vc.phi0[d] = __dmul_rn(-grad[d], double(radius * g.os - int(fo)));
    vc.dphi[d] = __dmul_rn(grad[d], double(g.os));
  }
  // all_within_grid (src/hpg_core.hpp:1070-1080); the fine-offset bound
  // holds for every finite position and keeps the CF slice index in range
  // for non-finite ones
  vc.in_grid = 0 <= vc.grid_coord[0] && vc.grid_coord[0] + taps[0] <= g.nx &&
               0 <= vc.grid_coord[1] && vc.grid_coord[1] + taps[1] <= g.ny &&
               abs(vc.fine[0]) <= g.os / 2 && abs(vc.fine[1]) <= g.os / 2;
}

__device__ __forceinline__ long long slice_index(const GridGeom& g,
                                                 const VisCoord& vc) {
  const int fx = vc.fine[0] + g.os / 2;
  const int fy = vc.fine[1] + g.os / 2;
  return (static_cast<long long>(vc.cf_cube) * g.nfine + fy) * g.nfine + fx;
}

}  // namespace hpgb
