// adjoint.cu -- the degridding and gridding maps as FP64 linear operators,
// and their adjoints, for differentiable imaging.
//
// For a batch of visibility records (only their geometry is used: uvw,
// frequency, phase, weights, cf_index, grid_cube, cf_phase_gradient):
//
//   D  (degridding, src/hpg_core.hpp:580-682):
//        y[i][v] = conj(phasor_i) / den_iv *
//                  sum_{r, X, Y} cfd_i[d(r, v)](X, Y) * sd_i(X, Y) * x[r](cell)
//      with d = (pos_w ? conjugate Mueller : Mueller) indexes, cfd the CF
//      with its imaginary part times (pos_w ? +1 : -1), sd = exp(-i phi(X, Y))
//      and den_iv = sum_r sum_XY cfd_i[d(r, v)] (1 where that is 0);
//   D^H (degridding adjoint): x[r](cell) += sum_v conj(cfd[d(r, v)]) *
//        conj(sd) * phasor / conj(den_v) * y[v] -- gridding of the cotangent
//        with the degridding indexes and the conjugate CF;
//   G  (gridding, src/hpg_core.hpp:791-886):
//        g[r](cell) += sum_v cfg_i[m(r, v)](X, Y) * sg_i(X, Y) * phasor_i *
//                      w_iv * u[i][v]
//      with m = (pos_w ? Mueller : conjugate Mueller) indexes, cfg the CF with
//      its imaginary part times (pos_w ? -1 : +1), sg = exp(+i phi(X, Y));
//   G^H (gridding adjoint): u[i][v] = conj(phasor_i) * w_iv *
//        sum_{r, X, Y} conj(cfg[m(r, v)]) * conj(sg) * g[r](cell) --
//        degridding of the cotangent without the normaliser.
//
// All arithmetic is FP64 (the CF values are converted exactly), so
// <D x, y> = <x, D^H y> and <G u, g> = <u, G^H g> hold to FP64 rounding.
// Visibilities whose footprint leaves the grid contribute nothing (the
// reference skips them).  Grid-shaped arrays use the gridder's device grid
// layout, double2 [cube][mrow][y][x]; per-visibility arrays are
// double2 [n][npol].  The kernels here take one CTA per visibility and
// accumulate grid outputs with FP64 global atomics; adjoint_tiled.cu runs
// the same operators on the tile sort of the batch (the default).

#include "gridder.cuh"

namespace hpgb {

namespace {

constexpr int kThreadsAdj = 128;

__device__ __forceinline__ double2 conj_d(double2 a) {
  return make_double2(a.x, -a.y);
}

// sum 2N doubles over the CTA; result valid in thread 0
template <int N>
__device__ void block_sum_adj(double (&v)[2 * N], double* sh) {
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

__device__ __forceinline__ double screen_phase(const VisCoord& vc, int X,
                                               int Y) {
  const double phx = __dadd_rn(vc.phi0[0], __dmul_rn(double(X), vc.dphi[0]));
  const double phy = __dadd_rn(vc.phi0[1], __dmul_rn(double(Y), vc.dphi[1]));
  return __dadd_rn(phx, phy);
}

// degridding normaliser den_v (src/hpg_core.hpp:598-600, :659-661)
template <int N>
__device__ void normalisers(const GridGeom& g, const CFGroup& G,
                            const VisCoord& vc, double2 (&den)[N]) {
  const int(*dmi)[4] = vc.pos_w ? g.mt.c : g.mt.m;
  const double2* ws = G.wsum + slice_index(g, vc) * G.nmueller;
#pragma unroll
  for (int v = 0; v < N; ++v) {
    double2 d = make_double2(0.0, 0.0);
    for (int r = 0; r < g.nrow; ++r) {
      const int m = dmi[r][v];
      if (m >= 0) {
        const double2 w = ws[m];
        d = cadd_d(d, make_double2(w.x, vc.pos_w ? w.y : -w.y));
      }
    }
    if (d.x == 0.0 && d.y == 0.0) d = make_double2(1.0, 0.0);
    den[v] = d;
  }
}

// D x and G^H g share one shape: a per-visibility reduction over the
// footprint of sum_v c[r][v](X, Y) * s(X, Y) * grid[r](cell)
template <int N, bool ADJ_GRID>
__global__ void __launch_bounds__(kThreadsAdj)
reduce_kernel(const VisData<N>* vis, size_t n, GridGeom g,
              const CFGroup* groups, const double2* grid, double2* out) {
  __shared__ double sh[(kThreadsAdj / 32) * 2 * N];
  const size_t i = blockIdx.x;
  if (i >= n) return;
  const VisData<N>& vd = vis[i];
  VisCoord vc;
  vis_coords(g, groups, vd.freq, vd.uvw, vd.grid_cube, vd.cf_index,
             vd.cf_phase_gradient, vc);
  if (!vc.in_grid) {
    if (threadIdx.x < N) out[i * N + threadIdx.x] = make_double2(0.0, 0.0);
    return;
  }
  const CFGroup& G = groups[vc.grp];
  // D: degridding indexes, CF imaginary part x (pos_w ? +1 : -1), screen
  //    exp(-i phi).  G^H: gridding indexes, conj of the gridding CF (imag x
  //    (pos_w ? +1 : -1)), conj of the gridding screen (exp(-i phi)).
  const int(*mi)[4] = ADJ_GRID ? (vc.pos_w ? g.mt.m : g.mt.c)
                               : (vc.pos_w ? g.mt.c : g.mt.m);
  const double im = vc.pos_w ? 1.0 : -1.0;
  const float2* slice = G.data + slice_index(g, vc) * G.slice_stride;
  const int tx = vc.taps[0], ncell = tx * vc.taps[1];
  const size_t plane = size_t(g.nx) * g.ny;
  double acc[2 * N];
#pragma unroll
  for (int k = 0; k < 2 * N; ++k) acc[k] = 0.0;
  for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
    const int Y = c / tx, X = c - Y * tx;
    const double2 s = cphase_d(-screen_phase(vc, X, Y));
    const size_t gidx = (size_t(vc.grid_cube) * g.nrow * g.ny +
                         size_t(vc.grid_coord[1] + Y)) * g.nx +
                        size_t(vc.grid_coord[0] + X);
    for (int r = 0; r < g.nrow; ++r) {
      const double2 gs = cmul_d(grid[gidx + size_t(r) * plane], s);
#pragma unroll
      for (int v = 0; v < N; ++v) {
        const int m = mi[r][v];
        if (m >= 0) {
          const float2 cf = slice[m * G.plane_stride + c];
          const double2 p = cmul_d(make_double2(cf.x, im * double(cf.y)), gs);
          acc[2 * v] += p.x;
          acc[2 * v + 1] += p.y;
        }
      }
    }
  }
  block_sum_adj<N>(acc, sh);
  if (threadIdx.x != 0) return;
  const double2 phasor = cphase_d(vd.phase);
  double2 den[N];
  if (!ADJ_GRID) normalisers<N>(g, G, vc, den);
#pragma unroll
  for (int v = 0; v < N; ++v) {
    const double2 sum = make_double2(acc[2 * v], acc[2 * v + 1]);
    out[i * N + v] =
        ADJ_GRID ? cmul_d(sum, make_double2(phasor.x * double(vd.weights[v]),
                                            -phasor.y * double(vd.weights[v])))
                 : cmul_d(cdiv_d(sum, den[v]), conj_d(phasor));
  }
}

// G u and D^H y share one shape: per visibility, add
// sum_v c[r][v](X, Y) * s(X, Y) * a_v to grid[r](cell)
template <int N, bool ADJ_DEGRID>
__global__ void __launch_bounds__(kThreadsAdj)
scatter_kernel(const VisData<N>* vis, size_t n, GridGeom g,
               const CFGroup* groups, const double2* vals, double2* grid) {
  const size_t i = blockIdx.x;
  if (i >= n) return;
  const VisData<N>& vd = vis[i];
  VisCoord vc;
  vis_coords(g, groups, vd.freq, vd.uvw, vd.grid_cube, vd.cf_index,
             vd.cf_phase_gradient, vc);
  if (!vc.in_grid) return;
  const CFGroup& G = groups[vc.grp];
  // G: gridding indexes, CF imag x (pos_w ? -1 : +1), screen exp(+i phi),
  //    a_v = phasor * w_v * u_v.  D^H: degridding indexes, conj of the
  //    degridding CF (imag x (pos_w ? -1 : +1)), conj of its screen
  //    (exp(+i phi)), a_v = phasor / conj(den_v) * y_v.
  const int(*mi)[4] = ADJ_DEGRID ? (vc.pos_w ? g.mt.c : g.mt.m)
                                 : (vc.pos_w ? g.mt.m : g.mt.c);
  const double im = vc.pos_w ? -1.0 : 1.0;
  const double2 phasor = cphase_d(vd.phase);
  double2 a[N];
  if (ADJ_DEGRID) {
    double2 den[N];
    normalisers<N>(g, G, vc, den);
#pragma unroll
    for (int v = 0; v < N; ++v)
      a[v] = cmul_d(cdiv_d(phasor, conj_d(den[v])), vals[i * N + v]);
  } else {
#pragma unroll
    for (int v = 0; v < N; ++v)
      a[v] = cmul_d(make_double2(phasor.x * double(vd.weights[v]),
                                 phasor.y * double(vd.weights[v])),
                    vals[i * N + v]);
  }
  const float2* slice = G.data + slice_index(g, vc) * G.slice_stride;
  const int tx = vc.taps[0], ncell = tx * vc.taps[1];
  const size_t plane = size_t(g.nx) * g.ny;
  for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
    const int Y = c / tx, X = c - Y * tx;
    const double2 s = cphase_d(screen_phase(vc, X, Y));
    const size_t gidx = (size_t(vc.grid_cube) * g.nrow * g.ny +
                         size_t(vc.grid_coord[1] + Y)) * g.nx +
                        size_t(vc.grid_coord[0] + X);
    for (int r = 0; r < g.nrow; ++r) {
      double2 sum = make_double2(0.0, 0.0);
#pragma unroll
      for (int v = 0; v < N; ++v) {
        const int m = mi[r][v];
        if (m >= 0) {
          const float2 cf = slice[m * G.plane_stride + c];
          sum = cadd_d(sum, cmul_d(make_double2(cf.x, im * double(cf.y)), a[v]));
        }
      }
      sum = cmul_d(sum, s);
      double2* dst = grid + gidx + size_t(r) * plane;
      atomicAdd(&dst->x, sum.x);
      atomicAdd(&dst->y, sum.y);
    }
  }
}

template <int N>
Status linear_n(hpgb_gridder* g, const void* d_vis, size_t n, int op,
                const void* in, void* out) {
  const VisData<N>* vis = static_cast<const VisData<N>*>(d_vis);
  const GridGeom geom = g->geom();
  const CFGroup* groups = g->cf.desc.as<const CFGroup>();
  const unsigned blocks = unsigned(n);
  const double2* src = static_cast<const double2*>(in);
  double2* dst = static_cast<double2*>(out);
  switch (op) {
    case 0:  // D
      reduce_kernel<N, false><<<blocks, kThreadsAdj, 0, g->stream>>>(
          vis, n, geom, groups, src, dst);
      break;
    case 1:  // D^H
      scatter_kernel<N, true><<<blocks, kThreadsAdj, 0, g->stream>>>(
          vis, n, geom, groups, src, dst);
      break;
    case 2:  // G
      scatter_kernel<N, false><<<blocks, kThreadsAdj, 0, g->stream>>>(
          vis, n, geom, groups, src, dst);
      break;
    default:  // G^H
      reduce_kernel<N, true><<<blocks, kThreadsAdj, 0, g->stream>>>(
          vis, n, geom, groups, src, dst);
      break;
  }
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  return Status::ok();
}

}  // namespace

Status linear_op(hpgb_gridder* g, const void* d_vis, size_t n, int op,
                 const void* in, void* out) {
  if (n == 0) return Status::ok();
  if (n > size_t(0x7fffffff))
    return Status::err(HPGB_ERROR_EXCESSIVE_NUMBER_VISIBILITIES,
                       "too many visibilities for one launch");
  // the tile-sorted kernels (adjoint_tiled.cu) unless the per-visibility
  // kernels are selected or the CF's region does not fit shared memory
  if (g->kernel_kind != HPGB_KERNEL_DIRECT) {
    bool used = false;
    HPGB_TRY(linear_op_tiled(g, d_vis, n, op, in, out, &used));
    if (used) {
      g->last_kernel = HPGB_KERNEL_TILED;
      return Status::ok();
    }
    if (g->kernel_kind == HPGB_KERNEL_TILED)
      return Status::err(HPGB_ERROR_OTHER,
                         "the tiled operators cannot take this CF or grid");
  }
  g->last_kernel = HPGB_KERNEL_DIRECT;
  switch (g->npol) {
    case 1: return linear_n<1>(g, d_vis, n, op, in, out);
    case 2: return linear_n<2>(g, d_vis, n, op, in, out);
    case 3: return linear_n<3>(g, d_vis, n, op, in, out);
    case 4: return linear_n<4>(g, d_vis, n, op, in, out);
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
}

}  // namespace hpgb
