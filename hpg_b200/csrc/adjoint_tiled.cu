// adjoint_tiled.cu -- the FP64 linear operators D, D^H, G and G^H
// (definitions in adjoint.cu) on the tile sort of the batch, for the
// differentiable-imaging workloads: degridding D (src/hpg_core.hpp:580-682)
// and its adjoint, gridding G (:791-886) and its adjoint.
//
// The batch is sorted into uv tiles of T x T footprint origins (tiles.cuh),
// a tile's visibilities in descending footprint size with every other block
// of 16 reversed (kOrderSnake16): the 16 warps of a CTA take visibilities
// r = warp, warp + 16, ... of a pass and meet at its end, so their shares
// of footprint cells come out nearly even (measured at 10M visibilities:
// 43.4 against 35.2 Mvis/s per gradient step in batch order).
// A persistent CTA takes one tile pass at a time from a device work counter
// and keeps the pass's grid region -- R x R cells (R = T + taps - 1) of
// every grid row -- in shared memory as FP64:
//   - D and G^H (gathers): the model / grid-cotangent region is loaded once
//     per pass; each warp then reduces one visibility at a time over its
//     footprint (lane = cell), reading the CF slice from global memory with
//     coalesced loads and the grid values from the shared region, and a
//     warp butterfly gives the visibility's values;
//   - D^H and G (scatters): each warp adds one visibility's contributions
//     into the shared region with FP64 shared-memory atomics (warps take
//     different visibilities, whose footprints may overlap); the pass ends
//     with one FP64 global atomic per region cell and row.
// The region is held as two planes, real and imaginary parts, so that a
// warp's atomics on consecutive cells touch consecutive 8-byte words (half
// the shared-memory wavefronts of interleaved complex values).
// Each CF value crosses HBM once per visibility, each grid cell once per
// pass (plus the region's halo of taps - 1 cells).  Arithmetic and signs are
// those of the per-visibility kernels in adjoint.cu, so both satisfy the
// dot-product identities to FP64 rounding.

#include <algorithm>
#include <cmath>

#include "gridder.cuh"
#include "tiles.cuh"

namespace hpgb {

namespace {

constexpr int kAdjThreads = 512;
constexpr int kAdjWarps = kAdjThreads / 32;
// visibilities per tile pass: FP64 regions carry no accumulation error, so
// passes are long; the cap keeps the passes of crowded tiles spread over
// several CTAs
constexpr int kAdjChunk = 2048;
// shared memory for the region (bytes)
constexpr int kAdjSmemBudget = 220 * 1024;

struct AdjParams {
  int nx, ny, nrow, ncube;
  int R, T, ntx, nty;
  int op;  // 0 D, 1 D^H, 2 G, 3 G^H
  int npol;
  MuellerTables mt;
  const TileDesc* descs;
  const SliceRef* srefs;
  const Chunk* chunks;
  const unsigned* num_chunks;
  unsigned* next_chunk;  // work counter, zero at launch
  const float2* cf;
  const double2* grid_in;  // gathers: model / grid cotangent
  double2* grid_out;       // scatters: accumulated
  const double2* vals_in;  // scatters: [n][npol]
  double2* vals_out;       // gathers: [n][npol]
};

__device__ __forceinline__ double2 conj2(double2 a) {
  return make_double2(a.x, -a.y);
}

// the descriptor fields one warp needs for one visibility
struct AdjVis {
  int index, cx, cy, tx, ty, pst;
  bool pos_w, screen;
  double2 phasor;
  double phi0x, phi0y, dphix, dphiy;
  long long cfoff;
};

__device__ __forceinline__ AdjVis adj_vis(const TileDesc* d, const SliceRef* s) {
  AdjVis v;
  v.index = d->index;
  v.cx = d->cx;
  v.cy = d->cy;
  v.tx = d->taps_x;
  v.ty = d->taps_y;
  v.pst = d->pstride;
  v.pos_w = d->flags & kPosW;
  v.screen = d->flags & kScreen;
  v.phasor = d->phasor;
  v.phi0x = d->phi0[0];
  v.phi0y = d->phi0[1];
  v.dphix = d->dphi[0];
  v.dphiy = d->dphi[1];
  v.cfoff = s->off;
  return v;
}

// One visibility's footprint cells (lane = cell, U cells per lane at a
// time, their CF loads issued together so that each warp keeps several HBM
// reads in flight -- the slices stream from HBM once, nothing to reuse).
// GATHER: acc += CF' * (region * screen) per polarization, the region
// values read from shared memory as each plane's products are formed (held
// across the planes they took the registers of 4 more cells per lane: D at
// 10M visibilities 82 -> 72 ms); otherwise region += screen * CF' * a[q],
// plane by plane, with shared-memory atomics.  (Issuing the next row's or
// plane's loads before the current ones are used was measured slower: 82 ->
// 89 ms for D, 114 -> 130 ms for D^H.)
// STRIDE threads share the visibility's cells (a warp); ATOMIC: scatters
// add with shared-memory atomics (warps take different visibilities, whose
// footprints may overlap).  A CTA-wide scatter (every thread on one
// visibility, plain read-modify-writes, a barrier between visibilities) was
// measured 1.8x slower at 10M visibilities: each visibility's CF loads then
// wait in turn.
template <int N, bool GATHER, bool SCREEN, int STRIDE, bool ATOMIC>
__device__ __forceinline__ void vis_cells(const AdjVis& v, const int (*mi)[4],
                                          double im, const float2* slice,
                                          double* re_plane, double* im_plane,
                                          int R, int RR, int nrow, int lane,
                                          const double2 (&a)[N],
                                          double (&acc)[2 * N]) {
  // cells per lane whose CF loads are issued together
  constexpr int U = (!SCREEN && N <= 2) ? 12 : 4;
  const int ncell = v.tx * v.ty;
  const double sph = GATHER ? -1.0 : 1.0;
  for (int base = lane; base < ncell; base += STRIDE * U) {
    int rc[U];
    double2 s[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int c = base + STRIDE * u;
      const int cu = c < ncell ? c : 0;
      const int Y = cu / v.tx, X = cu - Y * v.tx;
      if constexpr (SCREEN) {
        const double phx = __dadd_rn(v.phi0x, __dmul_rn(double(X), v.dphix));
        const double phy = __dadd_rn(v.phi0y, __dmul_rn(double(Y), v.dphiy));
        s[u] = cphase_d(sph * __dadd_rn(phx, phy));
      }
      rc[u] = (v.cy + Y) * R + v.cx + X;
    }
    for (int r = 0; r < nrow; ++r) {
      if constexpr (GATHER) {
#pragma unroll
        for (int q = 0; q < N; ++q) {
          const int m = mi[r][q];
          if (m < 0) continue;
          const float2* plane = slice + size_t(m) * v.pst;
          float2 cf[U];
#pragma unroll
          for (int u = 0; u < U; ++u)
            cf[u] = base + STRIDE * u < ncell
                        ? __ldg(plane + base + STRIDE * u)
                        : make_float2(0.f, 0.f);
#pragma unroll
          for (int u = 0; u < U; ++u) {
            double2 gs = make_double2(re_plane[r * RR + rc[u]],
                                      im_plane[r * RR + rc[u]]);
            if constexpr (SCREEN) gs = cmul_d(gs, s[u]);
            const double2 pr =
                cmul_d(make_double2(cf[u].x, im * double(cf[u].y)), gs);
            acc[2 * q] += pr.x;
            acc[2 * q + 1] += pr.y;
          }
        }
      } else {
        // each plane's products are added as soon as they are formed (the
        // shared-memory atomics are fire-and-forget reductions), so no
        // per-cell sum is held across the planes: measured 145 -> 114 ms
        // for D^H at 10M visibilities, against a sum over the planes
        // before one addition per cell
#pragma unroll
        for (int q = 0; q < N; ++q) {
          const int m = mi[r][q];
          if (m < 0) continue;
          const float2* plane = slice + size_t(m) * v.pst;
          float2 cf[U];
#pragma unroll
          for (int u = 0; u < U; ++u)
            cf[u] = base + STRIDE * u < ncell
                        ? __ldg(plane + base + STRIDE * u)
                        : make_float2(0.f, 0.f);
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (base + STRIDE * u >= ncell) continue;
            const double2 pr =
                cmul_d(make_double2(cf[u].x, im * double(cf[u].y)), a[q]);
            const double2 t = SCREEN ? cmul_d(pr, s[u]) : pr;
            double* dre = re_plane + r * RR + rc[u];
            double* dim = im_plane + r * RR + rc[u];
            if constexpr (ATOMIC) {
              atomicAdd(dre, t.x);
              atomicAdd(dim, t.y);
            } else {
              *dre += t.x;
              *dim += t.y;
            }
          }
        }
      }
    }
  }
}

template <int N>
__global__ void __launch_bounds__(kAdjThreads, 1)
adj_tiled_kernel(const __grid_constant__ AdjParams p) {
  // [nrow][R][R] real parts, then [nrow][R][R] imaginary parts
  extern __shared__ __align__(16) double region[];
  __shared__ unsigned cur_chunk;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool gather = p.op == 0 || p.op == 3;
  const bool degrid_set = p.op == 0 || p.op == 1;
  const int R = p.R, RR = R * R;
  double* const re_plane = region;
  double* const im_plane = region + size_t(p.nrow) * RR;
  const unsigned nchunks = *p.num_chunks;
  for (;;) {
    __syncthreads();  // the previous pass is done with the region
    if (threadIdx.x == 0) cur_chunk = atomicAdd(p.next_chunk, 1u);
    __syncthreads();
    const unsigned c = cur_chunk;
    if (c >= nchunks) break;
    const Chunk ch = p.chunks[c];
    const int tile = ch.tile;
    const int x0 = (tile % p.ntx) * p.T, y0 = ((tile / p.ntx) % p.nty) * p.T;
    const int cube = tile / (p.ntx * p.nty);
    // region: gathers load the grid values, scatters start from zero
    for (int i = threadIdx.x; i < RR * p.nrow; i += kAdjThreads) {
      const int r = i / RR, j = i - r * RR;
      const int gx = x0 + j % R, gy = y0 + j / R;
      double2 v = make_double2(0.0, 0.0);
      if (gather && gx < p.nx && gy < p.ny)
        v = p.grid_in[(size_t(cube * p.nrow + r) * p.ny + gy) * p.nx + gx];
      re_plane[i] = v.x;
      im_plane[i] = v.y;
    }
    __syncthreads();
    for (int k = warp; k < ch.count; k += kAdjWarps) {
      const AdjVis v = adj_vis(p.descs + ch.start + k, p.srefs + ch.start + k);
      const TileDesc* d = p.descs + ch.start + k;
      // Mueller routing and CF sign: gathers use the CF with its imaginary
      // part times (pos_w ? +1 : -1) and the screen exp(-i phi); scatters
      // the conjugates of both
      const int(*mi)[4] = degrid_set ? (v.pos_w ? p.mt.c : p.mt.m)
                                     : (v.pos_w ? p.mt.m : p.mt.c);
      const double im = (v.pos_w == gather) ? 1.0 : -1.0;
      const float2* slice = p.cf + v.cfoff;
      double2 a[N];  // scatters: per-polarization factors
      if (!gather) {
#pragma unroll
        for (int q = 0; q < N; ++q) {
          const double2 in = p.vals_in[size_t(v.index) * N + q];
          // D^H: phasor / conj(den) = conj(conj(phasor) / den);  G: phasor * w
          const double2 f =
              p.op == 1 ? conj2(d->wfac[q])
                        : make_double2(v.phasor.x * double(d->weights[q]),
                                       v.phasor.y * double(d->weights[q]));
          a[q] = cmul_d(f, in);
        }
      }
      double acc[2 * N];
#pragma unroll
      for (int t = 0; t < 2 * N; ++t) acc[t] = 0.0;
      // the cell loop: separate instantiations with and without phase
      // screen, for gathers and scatters (each keeps only its registers)
      if (gather) {
        if (v.screen)
          vis_cells<N, true, true, 32, false>(v, mi, im, slice, re_plane,
                                              im_plane, R, RR, p.nrow, lane,
                                              a, acc);
        else
          vis_cells<N, true, false, 32, false>(v, mi, im, slice, re_plane,
                                               im_plane, R, RR, p.nrow, lane,
                                               a, acc);
      } else {
        if (v.screen)
          vis_cells<N, false, true, 32, true>(v, mi, im, slice, re_plane,
                                              im_plane, R, RR, p.nrow, lane,
                                              a, acc);
        else
          vis_cells<N, false, false, 32, true>(v, mi, im, slice, re_plane,
                                               im_plane, R, RR, p.nrow, lane,
                                               a, acc);
      }
      if (gather) {
#pragma unroll
        for (int t = 0; t < 2 * N; ++t)
#pragma unroll
          for (int o = 16; o > 0; o >>= 1)
            acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], o);
        if (lane < N) {
          double2 sum = make_double2(0.0, 0.0);
#pragma unroll
          for (int q = 0; q < N; ++q)
            if (q == lane) sum = make_double2(acc[2 * q], acc[2 * q + 1]);
          // D: conj(phasor) / den;  G^H: conj(phasor) * w
          const double2 f =
              p.op == 0 ? d->wfac[lane]
                        : make_double2(v.phasor.x * double(d->weights[lane]),
                                       -v.phasor.y * double(d->weights[lane]));
          p.vals_out[size_t(v.index) * N + lane] = cmul_d(sum, f);
        }
      }
    }
    if (!gather) {
      __syncthreads();
      for (int i = threadIdx.x; i < RR * p.nrow; i += kAdjThreads) {
        const int r = i / RR, j = i - r * RR;
        const int gx = x0 + j % R, gy = y0 + j / R;
        const double2 v = make_double2(re_plane[i], im_plane[i]);
        if (gx < p.nx && gy < p.ny && (v.x != 0.0 || v.y != 0.0)) {
          double2* dst =
              p.grid_out + (size_t(cube * p.nrow + r) * p.ny + gy) * p.nx + gx;
          atomicAdd(&dst->x, v.x);
          atomicAdd(&dst->y, v.y);
        }
      }
    }
  }
}

// gathers write every visibility's values; those off the grid (never in a
// tile pass) get zero first
__global__ void zero_vals_kernel(double2* v, size_t n) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x)
    v[i] = make_double2(0.0, 0.0);
}

}  // namespace

// Runs op on the tile sort of the batch; *used is false when the region of
// the largest CF does not fit shared memory (the caller then uses the
// per-visibility kernels).
Status linear_op_tiled(hpgb_gridder* g, const void* d_vis, size_t n, int op,
                       const void* in, void* out, bool* used) {
  *used = false;
  const int nrow = int(g->grid_size[2]);
  const int taps = std::max(g->cf.max_taps_x, g->cf.max_taps_y);
  int R = int(std::sqrt(double(kAdjSmemBudget) / (16.0 * nrow)));
  R = std::min(R, 128) & ~1;
  const int T = R - taps + 1;
  if (T < 4 || n > size_t(0x7fffffff)) return Status::ok();
  *used = true;
  const int ntx = (int(g->grid_size[0]) + T - 1) / T;
  const int nty = (int(g->grid_size[1]) + T - 1) / T;
  TilePrep prep;
  HPGB_TRY(prepare_tiles(g, const_cast<void*>(d_vis), n, T, ntx, nty,
                         kAdjChunk, &prep, nullptr, kOrderSnake16));
  AdjParams p{};
  p.nx = int(g->grid_size[0]);
  p.ny = int(g->grid_size[1]);
  p.nrow = nrow;
  p.ncube = int(g->grid_size[3]);
  p.R = R;
  p.T = T;
  p.ntx = ntx;
  p.nty = nty;
  p.op = op;
  p.npol = int(g->npol);
  p.mt = g->mt;
  p.descs = prep.descs;
  p.srefs = prep.srefs;
  p.chunks = prep.chunks;
  p.num_chunks = prep.num_chunks;
  // the work counter: word 2 of the gridder's counters (word 0 is the
  // status, word 1 the chunk count)
  p.next_chunk = g->vb.counters.as<unsigned>() + 2;
  HPGB_CUDA_TRY(cudaMemsetAsync(p.next_chunk, 0, sizeof(unsigned), g->stream));
  p.cf = g->cf.data.as<const float2>();
  const bool gather = op == 0 || op == 3;
  if (gather) {
    p.grid_in = static_cast<const double2*>(in);
    p.vals_out = static_cast<double2*>(out);
    const size_t nv = n * g->npol;
    zero_vals_kernel<<<unsigned(std::min<size_t>((nv + 255) / 256, 148 * 16)),
                       256, 0, g->stream>>>(p.vals_out, nv);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
  } else {
    p.vals_in = static_cast<const double2*>(in);
    p.grid_out = static_cast<double2*>(out);
  }
  const int smem = nrow * R * R * int(sizeof(double2));
  int sms = 0;
  HPGB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount,
                                       g->device));
  auto launch = [&](auto kern) -> Status {
    HPGB_CUDA_TRY(cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kern<<<unsigned(sms), kAdjThreads, size_t(smem), g->stream>>>(p);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
    return Status::ok();
  };
  switch (g->npol) {
    case 1: return launch(adj_tiled_kernel<1>);
    case 2: return launch(adj_tiled_kernel<2>);
    case 3: return launch(adj_tiled_kernel<3>);
    case 4: return launch(adj_tiled_kernel<4>);
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
}

}  // namespace hpgb
