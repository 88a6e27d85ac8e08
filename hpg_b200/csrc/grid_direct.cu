// grid_direct.cu -- per-visibility gridding and degridding kernels with
// global FP64 atomics: the reference's launch structure
// (VisibilityGridder<N, Cuda, 0>::kernel, src/hpg_core.hpp:1082-1253) done as
// one CTA per visibility covering every grid row, used for the exact-parity
// path and for CFs whose support is too wide for the shared-memory tiles.
//
// Arithmetic is the reference's:
//  - degridding (src/hpg_core.hpp:580-682): FP64 products model*screen and
//    cf*mv, FP64 sums, prediction = sum / (normaliser != 0 ? normaliser : 1)
//    * conj(phasor), rounded to complex<float>;
//  - gridding (src/hpg_core.hpp:791-886): FP32 products cf*screen*gvis (no
//    contraction), FP64 sum over visibility polarisations, FP64 atomic add
//    of real and imaginary parts (pseudo_atomic_add, :360-384); grid weight
//    += sum_vpol |sum_XY cf| * w (:877-885).
// The normaliser sum_XY cf and the weight sums come from the per-slice FP64
// sums computed when the CF is set (CFGroup::wsum).

#include <mutex>
#include <string>

#include "gridder.cuh"

namespace hpgb {

namespace {

constexpr int kThreads = 128;

// sum 2N doubles over the CTA; result valid in thread 0
template <int N>
__device__ void block_sum(double (&v)[2 * N], double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 2 * N; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 2 * N; ++k) sh[warp * 2 * N + k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < int(blockDim.x >> 5); ++w) {
#pragma unroll
      for (int k = 0; k < 2 * N; ++k) v[k] += sh[w * 2 * N + k];
    }
  }
}

template <int N>
__global__ void __launch_bounds__(kThreads)
degrid_direct_kernel(VisData<N>* vis, size_t n, GridGeom g,
                     const CFGroup* groups, const double2* model,
                     float2* gvis, bool do_grid) {
  __shared__ double sh[(kThreads / 32) * 2 * N];
  const size_t i = blockIdx.x;
  if (i >= n) return;
  VisData<N>& vd = vis[i];
  VisCoord vc;
  vis_coords(g, groups, vd.freq, vd.uvw, vd.grid_cube, vd.cf_index,
             vd.cf_phase_gradient, vc);
  if (!vc.in_grid) return;
  const CFGroup& G = groups[vc.grp];
  const int (*dmi)[4] = vc.pos_w ? g.mt.c : g.mt.m;  // degridding indexes
  const float im = vc.pos_w ? 1.0f : -1.0f;
  const bool screen_on = vc.phi0[0] != 0.0 || vc.phi0[1] != 0.0 ||
                         vc.dphi[0] != 0.0 || vc.dphi[1] != 0.0;
  const long long sidx = slice_index(g, vc);
  const float2* slice = G.data + sidx * G.slice_stride;
  const int tx = vc.taps[0], ty = vc.taps[1], ncell = tx * ty;
  double acc[2 * N];
#pragma unroll
  for (int k = 0; k < 2 * N; ++k) acc[k] = 0.0;
  if (model) {
    const size_t plane = size_t(g.nx) * g.ny;
    for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
      const int Y = c / tx, X = c - Y * tx;
      double2 screen = make_double2(1.0, 0.0);
      if (screen_on) {
        const double phx = __dadd_rn(vc.phi0[0], __dmul_rn(double(X), vc.dphi[0]));
        const double phy = __dadd_rn(vc.phi0[1], __dmul_rn(double(Y), vc.dphi[1]));
        screen = cphase_d(__dsub_rn(-phx, phy));
      }
      const size_t gidx = (size_t(vc.grid_cube) * g.nrow * g.ny +
                           size_t(vc.grid_coord[1] + Y)) * g.nx +
                          size_t(vc.grid_coord[0] + X);
      for (int gpol = 0; gpol < g.nrow; ++gpol) {
        const double2 mv = cmul_d(model[gidx + size_t(gpol) * plane], screen);
#pragma unroll
        for (int vpol = 0; vpol < N; ++vpol) {
          const int m = dmi[gpol][vpol];
          if (m >= 0) {
            float2 cf = slice[m * G.plane_stride + c];
            cf.y *= im;
            const double2 p = cmul_d(make_double2(cf.x, cf.y), mv);
            acc[2 * vpol] = __dadd_rn(acc[2 * vpol], p.x);
            acc[2 * vpol + 1] = __dadd_rn(acc[2 * vpol + 1], p.y);
          }
        }
      }
    }
  }
  block_sum<N>(acc, sh);
  if (threadIdx.x != 0) return;
  const double2* ws = G.wsum + sidx * G.nmueller;
  const double2 phasor = cphase_d(vd.phase);
  const double2 cph = make_double2(phasor.x, -phasor.y);
#pragma unroll
  for (int vpol = 0; vpol < N; ++vpol) {
    float2 pred = make_float2(0.f, 0.f);
    if (model) {
      double2 den = make_double2(0.0, 0.0);
      for (int gpol = 0; gpol < g.nrow; ++gpol) {
        const int m = dmi[gpol][vpol];
        if (m >= 0) {
          const double2 w = ws[m];
          den = cadd_d(den, make_double2(w.x, vc.pos_w ? w.y : -w.y));
        }
      }
      if (den.x == 0.0 && den.y == 0.0) den = make_double2(1.0, 0.0);
      const double2 q =
          cmul_d(cdiv_d(make_double2(acc[2 * vpol], acc[2 * vpol + 1]), den), cph);
      pred = make_float2(__double2float_rn(q.x), __double2float_rn(q.y));
    }
    if (do_grid) {
      const float2 r = make_float2(__fsub_rn(vd.vis[vpol].x, pred.x),
                                   __fsub_rn(vd.vis[vpol].y, pred.y));
      vd.vis[vpol] = r;
      gvis[i * N + vpol] = scale_for_gridding(r, phasor, vd.weights[vpol]);
    } else {
      vd.vis[vpol] = pred;
    }
  }
}

template <int N>
__global__ void gvis_init_kernel(const VisData<N>* vis, size_t n,
                                 float2* gvis) {
  const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const VisData<N>& vd = vis[i];
  const double2 phasor = cphase_d(vd.phase);
#pragma unroll
  for (int k = 0; k < N; ++k)
    gvis[i * N + k] = scale_for_gridding(vd.vis[k], phasor, vd.weights[k]);
}

template <int N>
__global__ void __launch_bounds__(kThreads)
grid_direct_kernel(const VisData<N>* vis, size_t n, GridGeom g,
                   const CFGroup* groups, const float2* gvis, double2* grid,
                   double* weights) {
  const size_t i = blockIdx.x;
  if (i >= n) return;
  const VisData<N>& vd = vis[i];
  VisCoord vc;
  vis_coords(g, groups, vd.freq, vd.uvw, vd.grid_cube, vd.cf_index,
             vd.cf_phase_gradient, vc);
  if (!vc.in_grid) return;
  const CFGroup& G = groups[vc.grp];
  const int (*gmi)[4] = vc.pos_w ? g.mt.m : g.mt.c;  // gridding indexes
  const float im = vc.pos_w ? -1.0f : 1.0f;
  const bool screen_on = vc.phi0[0] != 0.0 || vc.phi0[1] != 0.0 ||
                         vc.dphi[0] != 0.0 || vc.dphi[1] != 0.0;
  const long long sidx = slice_index(g, vc);
  const float2* slice = G.data + sidx * G.slice_stride;
  const int tx = vc.taps[0], ty = vc.taps[1], ncell = tx * ty;
  float2 gv_in[N];
#pragma unroll
  for (int k = 0; k < N; ++k) gv_in[k] = gvis[i * N + k];
  const size_t plane = size_t(g.nx) * g.ny;
  for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
    const int Y = c / tx, X = c - Y * tx;
    float2 screen = make_float2(1.0f, 0.0f);
    if (screen_on) {
      const double phx = __dadd_rn(vc.phi0[0], __dmul_rn(double(X), vc.dphi[0]));
      const double phy = __dadd_rn(vc.phi0[1], __dmul_rn(double(Y), vc.dphi[1]));
      const double2 s = cphase_d(__dadd_rn(phx, phy));
      screen = make_float2(__double2float_rn(s.x), __double2float_rn(s.y));
    }
    const size_t gidx = (size_t(vc.grid_cube) * g.nrow * g.ny +
                         size_t(vc.grid_coord[1] + Y)) * g.nx +
                        size_t(vc.grid_coord[0] + X);
    for (int gpol = 0; gpol < g.nrow; ++gpol) {
      double gx = 0.0, gy = 0.0;
#pragma unroll
      for (int vpol = 0; vpol < N; ++vpol) {
        const int m = gmi[gpol][vpol];
        if (m >= 0) {
          float2 cf = slice[m * G.plane_stride + c];
          cf.y *= im;
          const float2 p = cmul_f(cmul_f(cf, screen), gv_in[vpol]);
          gx = __dadd_rn(gx, double(p.x));
          gy = __dadd_rn(gy, double(p.y));
        }
      }
      double2* dst = grid + gidx + size_t(gpol) * plane;
      atomicAdd(&dst->x, gx);
      atomicAdd(&dst->y, gy);
    }
  }
  if (weights && threadIdx.x == 0) {
    const double2* ws = G.wsum + sidx * G.nmueller;
    for (int gpol = 0; gpol < g.nrow; ++gpol) {
      double twgt = 0.0;
#pragma unroll
      for (int vpol = 0; vpol < N; ++vpol) {
        const int m = gmi[gpol][vpol];
        if (m >= 0) {
          const double2 w = ws[m];
          twgt = __dadd_rn(twgt, __dmul_rn(hypot(w.x, w.y), double(vd.weights[vpol])));
        }
      }
      atomicAdd(weights + size_t(vc.grid_cube) * g.nrow + gpol, twgt);
    }
  }
}

template <int N>
__global__ void coords_kernel(const VisData<N>* vis, size_t n, GridGeom g,
                              const CFGroup* groups, hpgb_vis_coords* out) {
  const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const VisData<N>& vd = vis[i];
  VisCoord vc;
  vis_coords(g, groups, vd.freq, vd.uvw, vd.grid_cube, vd.cf_index,
             vd.cf_phase_gradient, vc);
  hpgb_vis_coords& o = out[i];
  for (int d = 0; d < 2; ++d) {
    o.grid_coord[d] = vc.grid_coord[d];
    o.cf_major[d] = vc.cf_major[d];
    o.cf_minor[d] = vc.cf_minor[d];
    o.fine_offset[d] = vc.fine[d];
    o.cf_size[d] = vc.taps[d];
  }
  o.pos_w = vc.pos_w;
  o.in_grid = vc.in_grid;
  const int(*gm)[4] = vc.pos_w ? g.mt.m : g.mt.c;
  const int(*dm)[4] = vc.pos_w ? g.mt.c : g.mt.m;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      o.grid_mueller[r][c] = gm[r][c];
      o.degrid_mueller[r][c] = dm[r][c];
    }
}

template <int N>
Status grid_direct_n(hpgb_gridder* g, void* d_vis, size_t n, unsigned flags) {
  if (n == 0) return Status::ok();
  VisData<N>* vis = static_cast<VisData<N>*>(d_vis);
  const GridGeom geom = g->geom();
  const CFGroup* groups = g->cf.desc.as<const CFGroup>();
  HPGB_TRY(g->vb.gvis.reserve(n * N * sizeof(float2)));
  float2* gvis = g->vb.gvis.as<float2>();
  const bool do_grid = flags & HPGB_DO_GRID;
  if (flags & HPGB_DO_DEGRID) {
    degrid_direct_kernel<N><<<unsigned(n), kThreads, 0, g->stream>>>(
        vis, n, geom, groups,
        g->has_model ? g->model.as<const double2>() : nullptr, gvis, do_grid);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
  } else if (do_grid) {
    gvis_init_kernel<N><<<unsigned((n + 255) / 256), 256, 0, g->stream>>>(
        vis, n, gvis);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
  }
  if (do_grid) {
    grid_direct_kernel<N><<<unsigned(n), kThreads, 0, g->stream>>>(
        vis, n, geom, groups, gvis, g->grid.as<double2>(),
        (flags & HPGB_UPDATE_GRID_WEIGHTS) ? g->weights.as<double>() : nullptr);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
  }
  return Status::ok();
}

}  // namespace

Status grid_direct(hpgb_gridder* g, const void* d_vis, size_t n,
                   unsigned flags) {
  void* v = const_cast<void*>(d_vis);
  switch (g->npol) {
    case 1: return grid_direct_n<1>(g, v, n, flags);
    case 2: return grid_direct_n<2>(g, v, n, flags);
    case 3: return grid_direct_n<3>(g, v, n, flags);
    case 4: return grid_direct_n<4>(g, v, n, flags);
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
}

Status debug_coords(hpgb_gridder* g, const void* d_vis, size_t n,
                    hpgb_vis_coords* d_out) {
  if (n == 0) return Status::ok();
  const GridGeom geom = g->geom();
  const CFGroup* groups = g->cf.desc.as<const CFGroup>();
  const unsigned blocks = unsigned((n + 255) / 256);
  switch (g->npol) {
    case 1: coords_kernel<1><<<blocks, 256, 0, g->stream>>>(static_cast<const VisData<1>*>(d_vis), n, geom, groups, d_out); break;
    case 2: coords_kernel<2><<<blocks, 256, 0, g->stream>>>(static_cast<const VisData<2>*>(d_vis), n, geom, groups, d_out); break;
    case 3: coords_kernel<3><<<blocks, 256, 0, g->stream>>>(static_cast<const VisData<3>*>(d_vis), n, geom, groups, d_out); break;
    case 4: coords_kernel<4><<<blocks, 256, 0, g->stream>>>(static_cast<const VisData<4>*>(d_vis), n, geom, groups, d_out); break;
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  return Status::ok();
}

// ---------------------------------------------------------------------------
// Allocation-free form of the direct path (hpgb_grid_visibilities_noalloc).
//
// Some callers cannot allocate device memory when they grid: cudaMalloc and
// cudaFree can synchronize the whole device, which stalls every other stream
// of a pipeline that overlaps gridding with transfers, and they fail outright
// in a process that handed nearly all device memory to its own pool when it
// started.  For them the only per-call scratch of the direct path, the
// gridding values of each visibility (float2 [n][N]), lives in a fixed
// device array compiled into this library instead of a gridder buffer.
//
// The array needs no initial value: the degridding kernel (or
// gvis_init_kernel when only gridding) writes the entry of every visibility
// that lies on the grid before grid_direct_kernel reads it in the same call,
// and visibilities off the grid are skipped by both.  There is one array per
// device, shared by every gridder: two calls that can run at the same time
// on one device (different streams with no ordering between them) race on
// it.

namespace {

__device__ __align__(256) float2 g_noalloc_gvis[kNoAllocMaxValues];

constexpr int kNoAllocMaxDevices = 64;
std::mutex noalloc_mtx;
float2* noalloc_addr[kNoAllocMaxDevices] = {};

// device address of g_noalloc_gvis on `device`, looked up once per device
// with that device current
Status noalloc_scratch(int device, float2** out) {
  if (device < 0 || device >= kNoAllocMaxDevices)
    return Status::err(HPGB_ERROR_OTHER, "device index out of range");
  std::lock_guard<std::mutex> lock(noalloc_mtx);
  if (!noalloc_addr[device]) {
    void* p = nullptr;
    HPGB_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_gvis));
    noalloc_addr[device] = static_cast<float2*>(p);
  }
  *out = noalloc_addr[device];
  return Status::ok();
}

template <int N>
Status grid_direct_noalloc_n(hpgb_gridder* g, void* d_vis, size_t n,
                             unsigned flags) {
  if (n == 0) return Status::ok();
  const bool do_grid = flags & HPGB_DO_GRID;
  if (do_grid && n * N > kNoAllocMaxValues)
    return Status::err(
        HPGB_ERROR_EXCESSIVE_NUMBER_VISIBILITIES,
        "allocation-free gridding holds at most " +
            std::to_string(kNoAllocMaxValues) +
            " visibility polarization values per call (" +
            std::to_string(kNoAllocMaxValues / N) + " visibilities of " +
            std::to_string(N) + " polarizations)");
  float2* gvis = nullptr;
  HPGB_TRY(noalloc_scratch(g->device, &gvis));
  VisData<N>* vis = static_cast<VisData<N>*>(d_vis);
  const GridGeom geom = g->geom();
  const CFGroup* groups = g->cf.desc.as<const CFGroup>();
  if (flags & HPGB_DO_DEGRID) {
    degrid_direct_kernel<N><<<unsigned(n), kThreads, 0, g->stream>>>(
        vis, n, geom, groups,
        g->has_model ? g->model.as<const double2>() : nullptr, gvis, do_grid);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
  } else if (do_grid) {
    gvis_init_kernel<N><<<unsigned((n + 255) / 256), 256, 0, g->stream>>>(
        vis, n, gvis);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
  }
  if (do_grid) {
    grid_direct_kernel<N><<<unsigned(n), kThreads, 0, g->stream>>>(
        vis, n, geom, groups, gvis, g->grid.as<double2>(),
        (flags & HPGB_UPDATE_GRID_WEIGHTS) ? g->weights.as<double>() : nullptr);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
  }
  return Status::ok();
}

}  // namespace

Status grid_direct_noalloc(hpgb_gridder* g, void* d_vis, size_t n,
                           unsigned flags) {
  switch (g->npol) {
    case 1: return grid_direct_noalloc_n<1>(g, d_vis, n, flags);
    case 2: return grid_direct_noalloc_n<2>(g, d_vis, n, flags);
    case 3: return grid_direct_noalloc_n<3>(g, d_vis, n, flags);
    case 4: return grid_direct_noalloc_n<4>(g, d_vis, n, flags);
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
}

}  // namespace hpgb
