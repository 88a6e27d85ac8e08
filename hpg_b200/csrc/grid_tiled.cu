// grid_tiled.cu -- fused degrid -> residual -> grid over shared-memory uv
// tiles: the hot path of State::grid_visibilities
// (src/hpg_runtime.hpp:965-1001 -> VisibilityGridder::kernel,
// src/hpg_core.hpp:1082-1253), designed for sm_100a.
//
// Pipeline of one batch (all on the gridder's stream, no host sync):
//   1. tile_keys_kernel   coordinates of every visibility (bit-exact with
//                         compute_vis_coord) -> key = (cube, tile row, tile
//                         col) of the tile holding the footprint origin;
//                         histogram of keys
//   2. cub radix sort     stable sort of (key, visibility index)
//   3. scans + chunks     tile starts; work chunks of <= kChunkVis visibilities
//   4. tile_desc_kernel   one 256-byte descriptor per visibility in sorted
//                         order (tile-relative footprint origin, phasor,
//                         phase screen, degridding normaliser and grid-row
//                         weights from the per-slice CF sums, gridding
//                         values) + the address of its CF slice
//   5. tiled_kernel       persistent, one thread-block cluster per tile with
//                         one CTA per grid row (Mueller row) r; 20 warps:
//                         - two producer warps stream each visibility's
//                           descriptor and the CF planes row r needs
//                           (Mueller row r of both index sets) into a ring of
//                           shared-memory slots with cp.async.bulk and
//                           mbarrier completion (16 visibilities in flight
//                           at most, bounded by the ring's bytes);
//                         - the model tile of row r is loaded once per chunk
//                           with a 3-D TMA tensor copy (FP64 form: the next
//                           chunk's as soon as the degridding warps are
//                           done with the current one);
//                         - 8 degridding warps in two groups of 4 take
//                           alternate visibilities: partial sums of row r
//                           over the footprint, reduced per warp;
//                         - 2 exchange warps (alternate visibilities) send
//                           the partials to every CTA of the cluster through
//                           distributed shared memory and a remote mbarrier,
//                           and form the prediction, residual and gridding
//                           values (identically in every CTA) as soon as
//                           the other rows' partials arrive;
//                         - 8 gridding warps add the scaled residual of one
//                           visibility at a time into the row's
//                           shared-memory grid tile (mixed form: two groups
//                           of 4 take alternate visibilities, each with a
//                           tile of its own);
//                         - at the end of a chunk the tile (the sum of the
//                           groups' tiles) is added to the FP64 grid with
//                           red.global.add.f64, and the row's
//                           weight sum to the weights.
// Each CF value therefore crosses HBM once per visibility, the model and grid
// tiles once per chunk.
//
// Arithmetic forms:
//   FP64  (reference arithmetic): FP64 model tile, FP64 degridding products
//         (FMA), gridding products in FP32 with the reference's rounding
//         (cf*screen*gvis, no contraction), FP64 sum over polarizations, FP64
//         shared-memory tile.
//   MIXED FP32 model tile, FP32 products, per-thread and per-warp FP32
//         partial sums (merged in FP64 across warps, rows and in the
//         normalisation),
//         FP32 shared-memory tile flushed into the FP64 grid every chunk.
//         Coordinates, phases, normalisers and weight sums stay FP64.

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cub/cub.cuh>
#include <type_traits>

#include "gridder.cuh"
#include "ptx.cuh"
#include "tiles.cuh"

namespace hpgb {

namespace {

// warp roles of the tiled kernel: kDG degridding warps, kX exchange warps
// (alternating visibilities), kGR gridding warps, one producer warp
constexpr int kDG = 8;
// the degridding warps form two groups of four that take alternate
// visibilities, as the two exchange warps do: two visibilities are degridded
// at once, so a group's per-visibility latency (loads, warp reduction,
// hand-off) overlaps the other group's work
constexpr int kDGGroups = 2;
constexpr int kDGPer = kDG / kDGGroups;
constexpr int kX = 2;
constexpr int kGR = 8;
constexpr int kXBase = kDG;
constexpr int kGRBase = kXBase + kX;
constexpr int kPWarp = kGRBase + kGR;
constexpr int kXSlots = 8;  // exchange buffers (visibility q uses q % 8)
constexpr int kConsumers = (kDG + kX + kGR) * 32;
static_assert(kDGGroups == kX, "degridding group g hands visibilities to exchange warp g");
// two producer warps: a warp's bulk copies are taken up one after another
// (measured on B200: one warp streams ~21 B/clk per SM in ~18 KB copies, two
// warps ~37 B/clk), so kPWarp allocates ring space for every visibility and
// issues the copies of the even ones, kPWarp + 1 those of the odd ones
constexpr int kProducers = 2;
constexpr int kThreadsTiled = kConsumers + 32 * kProducers;
constexpr int kSlots = 16;  // descriptor slots (visibilities in flight)
constexpr int kChunkVisFP64 = 2048;
constexpr int kChunkVisMixed = 256;
// compensated tiles accumulate without FP32 error: longer passes
constexpr int kChunkVisMixedComp = 2048;
constexpr int kMaxRuns = 8;

struct TiledParams {
  int nx, ny, nrow, ncube;
  int R, T, ntx, nty;
  int ring_bytes, model_bytes;  // CF ring size (bytes, multiple of 128)
  int esize_model, esize_grid;  // bytes per tile element; 0 when unused
  int grid_tiles;  // grid tiles: one per gridding group, two when compensated
  int compensated;  // mixed form: high/low tile pairs updated by two-sum
  int nplanes[4];
  int nruns[4];
  int run_plane[4][kMaxRuns];
  int run_len[4][kMaxRuns];
  int run_dst[4][kMaxRuns];
  int dpos[4][2][4];  // [row][pos_w][vpol] -> plane position in the slot
  int gpos[4][2][4];
  int do_degrid, do_grid, update_weights, has_model;
  const TileDesc* descs;
  const SliceRef* srefs;
  const Chunk* chunks;
  const unsigned* num_chunks;
  const float2* cf;
  double2* grid;
  double* weights;
  unsigned char* records;  // VisData<N> records (values written back)
  int rec_stride;
  unsigned* status;
  unsigned long long wait_limit_ns;  // bound of every wait in the kernel
  // test hook: CTA 0 never issues the copies of this visibility (its ring
  // position in CTA 0's sequence), so that the waits for them run out; -1:
  // none
  long long withhold_vis;
};

struct SmemLayout {
  int bars, xbuf, wred, bcast, slots, desc, ring, model, grid, total;
};

__host__ __device__ inline int align_up(int v, int a) { return (v + a - 1) / a * a; }

__host__ __device__ inline SmemLayout smem_layout(int ring_bytes, int R,
                                                  int esize_model,
                                                  int esize_grid,
                                                  int grid_tiles) {
  SmemLayout L;
  // mbarriers full[kSlots] empty[kSlots] model xchg[kXSlots] dgfull[2]
  // dgempty[2] gvfull[kSlots] req[kSlots], then the abort flag
  L.bars = 0;
  // + the WaitCtl block (abort flag, wait limit)
  L.xbuf = align_up((4 * kSlots + kXSlots + 5) * 8 + int(sizeof(ptx::WaitCtl)),
                    16);  // [kXSlots][4 rows][4 pol] complex double
  L.wred = L.xbuf + kXSlots * 4 * 4 * 16;  // [2][kDG][8] double (degrid partials)
  L.bcast = L.wred + 2 * kDG * 8 * 8; // [kSlots][4] float2 (gridding values)
  // slot_end[kSlots] u64, req_src[kSlots] i64, ring_off[kSlots] int,
  // req_off[kSlots] int, req_pst[kSlots] int, req_desc[kSlots] int,
  // issued[kSlots] int
  L.slots = L.bcast + kSlots * 4 * 8;
  L.desc = align_up(L.slots + kSlots * (8 + 8 + 4 + 4 + 4 + 4 + 4), 128);
  L.ring = align_up(L.desc + kSlots * int(sizeof(TileDesc)), 1024);
  L.model = align_up(L.ring + ring_bytes, 1024);
  L.grid = align_up(L.model + R * R * esize_model, 128);
  L.total = L.grid + R * R * esize_grid * grid_tiles;
  return L;
}

// ---------------------------------------------------------------------------
// preparation kernels

template <int N>
__global__ void tile_keys_kernel(const VisData<N>* vis, size_t n, GridGeom g,
                                 const CFGroup* groups, TileGeom tg,
                                 unsigned* keys, unsigned* order,
                                 unsigned* counts) {
  const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const VisData<N>& vd = vis[i];
  VisCoord vc;
  vis_coords(g, groups, vd.freq, vd.uvw, vd.grid_cube, vd.cf_index,
             vd.cf_phase_gradient, vc);
  unsigned key = unsigned(tg.ntiles);
  if (vc.in_grid) {
    key = unsigned((vc.grid_cube * tg.nty + vc.grid_coord[1] / tg.T) * tg.ntx +
                   vc.grid_coord[0] / tg.T);
    atomicAdd(&counts[key], 1u);
  }
  keys[i] = key;
  order[i] = unsigned(i);
}

__global__ void chunk_count_kernel(const unsigned* counts, int ntiles, int K,
                                   unsigned* nch) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ntiles) nch[t] = (counts[t] + K - 1) / K;
}

__global__ void chunk_write_kernel(const unsigned* counts,
                                   const unsigned* tstart,
                                   const unsigned* nch, const unsigned* cstart,
                                   int ntiles, int K, Chunk* chunks,
                                   unsigned* num_chunks) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  for (unsigned k = 0; k < nch[t]; ++k) {
    Chunk c;
    c.tile = t;
    c.start = int(tstart[t] + k * K);
    c.count = int(min(unsigned(K), counts[t] - k * K));
    c.pad = 0;
    chunks[cstart[t] + k] = c;
  }
  if (t == ntiles - 1) *num_chunks = cstart[t] + nch[t];
}

template <int N>
__global__ void tile_desc_kernel(const VisData<N>* vis, const unsigned* order,
                                 const unsigned* keys, size_t n, GridGeom g,
                                 const CFGroup* groups, TileGeom tg,
                                 const float2* cf_base, TileDesc* descs,
                                 SliceRef* srefs) {
  const size_t pidx = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (pidx >= n) return;
  const unsigned key = keys[pidx];
  if (key >= unsigned(tg.ntiles)) return;
  const unsigned i = order[pidx];
  const VisData<N>& vd = vis[i];
  VisCoord vc;
  vis_coords(g, groups, vd.freq, vd.uvw, vd.grid_cube, vd.cf_index,
             vd.cf_phase_gradient, vc);
  const CFGroup& G = groups[vc.grp];
  const int tx = int(key % unsigned(tg.ntx));
  const int ty = int((key / unsigned(tg.ntx)) % unsigned(tg.nty));
  TileDesc d;
  d.index = int(i);
  d.cx = int16_t(vc.grid_coord[0] - tx * tg.T);
  d.cy = int16_t(vc.grid_coord[1] - ty * tg.T);
  d.taps_x = uint8_t(vc.taps[0]);
  d.taps_y = uint8_t(vc.taps[1]);
  const bool screen_on = vc.phi0[0] != 0.0 || vc.phi0[1] != 0.0 ||
                         vc.dphi[0] != 0.0 || vc.dphi[1] != 0.0;
  d.flags = (vc.pos_w ? kPosW : 0) | (screen_on ? kScreen : 0);
  d.pad0 = 0;
  d.pstride = G.plane_stride;
  d.phasor = cphase_d(vd.phase);
  for (int k = 0; k < 2; ++k) {
    d.phi0[k] = vc.phi0[k];
    d.dphi[k] = vc.dphi[k];
  }
  const long long sidx = slice_index(g, vc);
  const double2* ws = G.wsum + sidx * G.nmueller;
  const int(*dmi)[4] = vc.pos_w ? g.mt.c : g.mt.m;
  const int(*gmi)[4] = vc.pos_w ? g.mt.m : g.mt.c;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    d.vals[v] = v < N ? vd.vis[v] : make_float2(0.f, 0.f);
    d.weights[v] = v < N ? vd.weights[v] : 0.f;
    d.gvis[v] = v < N ? scale_for_gridding(vd.vis[v], d.phasor, vd.weights[v])
                      : make_float2(0.f, 0.f);
    // normaliser: sum over grid rows of the slice sums, conjugated for
    // non-positive w (src/hpg_core.hpp:598-600, :659-661)
    double2 den = make_double2(0.0, 0.0);
    if (v < N)
      for (int r = 0; r < g.nrow; ++r) {
        const int m = dmi[r][v];
        if (m >= 0) {
          const double2 w = ws[m];
          den = cadd_d(den, make_double2(w.x, vc.pos_w ? w.y : -w.y));
        }
      }
    // prediction = sum * conj(phasor) / normaliser (src/hpg_core.hpp:670-679),
    // with the factor formed here once per visibility
    if (den.x == 0.0 && den.y == 0.0) den = make_double2(1.0, 0.0);
    d.wfac[v] = cdiv_d(make_double2(d.phasor.x, -d.phasor.y), den);
  }
  // grid weight per row: sum_vpol |sum_XY cf| * w (src/hpg_core.hpp:877-885)
  for (int r = 0; r < 4; ++r) {
    double tw = 0.0;
    if (r < g.nrow)
      for (int v = 0; v < N; ++v) {
        const int m = gmi[r][v];
        if (m >= 0) {
          const double2 w = ws[m];
          tw = __dadd_rn(tw, __dmul_rn(hypot(w.x, w.y), double(vd.weights[v])));
        }
      }
    d.twgt[r] = tw;
  }
  d.inv_tx = 1.0f / float(vc.taps[0]);
  for (int k = 0; k < 3; ++k) d.pad1[k] = 0;
  descs[pidx] = d;
  SliceRef s;
  s.off = (G.data - cf_base) + sidx * G.slice_stride;
  s.pstride = G.plane_stride;
  s.ncell = vc.taps[0] * vc.taps[1];
  srefs[pidx] = s;
}

__global__ void model_to_f32_kernel(const double2* __restrict__ in,
                                    float2* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const double2 v = in[i];
    out[i] = make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
  }
}

// ---------------------------------------------------------------------------
// the tiled kernel

template <bool MIXED>
struct Form;

// gridding groups, each with a grid tile of its own: two in the mixed form
// (8-byte tiles leave room for a second one), one in the FP64 form
template <bool MIXED>
constexpr int kGridTiles = MIXED ? 2 : 1;
// gridding groups of the compensated mixed form (each with a high and a low
// tile)
constexpr int kCompGroups = 1;
// gridding groups of a form
template <bool MIXED, bool COMP>
constexpr int kGroups = COMP ? kCompGroups : kGridTiles<MIXED>;

template <>
struct Form<false> {
  using model_t = double2;
  using grid_t = double2;
};

template <>
struct Form<true> {
  using model_t = float2;
  using grid_t = float2;
};

// Per-visibility values the cell loops need, copied out of the descriptor
// into registers once per visibility.
struct VisGeom {
  int cx, cy, tx, ty, pst;
  float inv_tx;
  bool pos_w, screen_on;
  double phi0x, phi0y, dphix, dphiy;
};

__device__ __forceinline__ VisGeom vis_geom(const TileDesc& d) {
  VisGeom v;
  v.cx = d.cx;
  v.cy = d.cy;
  v.tx = d.taps_x;
  v.ty = d.taps_y;
  v.pst = d.pstride;
  v.inv_tx = d.inv_tx;
  v.pos_w = d.flags & kPosW;
  v.screen_on = d.flags & kScreen;
  v.phi0x = v.phi0y = v.dphix = v.dphiy = 0.0;
  if (v.screen_on) {
    v.phi0x = d.phi0[0];
    v.phi0y = d.phi0[1];
    v.dphix = d.dphi[0];
    v.dphiy = d.dphi[1];
  }
  return v;
}

// Footprint cells c = first, first + stride, ... with their (X, Y) and the
// shared-memory address of their tile cell (row pitch R elements of `esize`
// bytes), advanced without integer division: the start and the step are
// split with the float reciprocal of taps_x, exact here because with
// c + 0.5 < 2^14 and taps_x < 128 the two float roundings (relative error
// < 2^-23) leave an absolute error below 2^14 / taps_x * 2^-23 < 2^-9 /
// taps_x, under the distance of (c + 0.5) / taps_x to the nearest integer
// (>= 0.5 / taps_x).  Footprints reach 65^2 = 4225 < 2^14 cells.
struct CellWalk {
  int X, Y, dX, dY;
  uint32_t tile, dtile, wrap;  // tile-cell address, its step, row wrap
  __device__ __forceinline__ CellWalk(int first, int stride, int tx,
                                      float inv_tx, uint32_t tile0, int R,
                                      uint32_t esize) {
    Y = int((float(first) + 0.5f) * inv_tx);
    X = first - Y * tx;
    dY = int((float(stride) + 0.5f) * inv_tx);
    dX = stride - dY * tx;
    tile = tile0 + uint32_t(Y * R + X) * esize;
    dtile = uint32_t(dY * R + dX) * esize;
    wrap = uint32_t(R - tx) * esize;
  }
  __device__ __forceinline__ void next(int tx) {
    X += dX;
    Y += dY;
    tile += dtile;
    if (X >= tx) {
      X -= tx;
      ++Y;
      tile += wrap;
    }
  }
};

// Partial degridding sums of this CTA's row over the footprint cells
// c = first, first + stride, ... of one visibility (src/hpg_core.hpp:642-668).
// pp[v]: slot plane of Mueller element dmi[row][v] (-1 if inactive; never
// when DENSE).  The sign of the CF imaginary part (+1 for w > 0, else -1)
// is moved onto the model value's imaginary part and the sum's imaginary
// part: sgn*(cf * m) with cf' = (cr, sgn*ci) equals the sum taken with
// (cr, ci) and (mx, sgn*my), imaginary part times sgn, bit for bit.
template <int N, bool MIXED, bool DENSE, bool SCREEN>
__device__ __forceinline__ void degrid_cells(
    const VisGeom& g, const int (&pp)[N], uint32_t cfs, uint32_t mtile, int R,
    int first, int stride, double (&acc)[2 * N]) {
  using MT = typename Form<MIXED>::model_t;
  const int tx = g.tx, ncell = g.tx * g.ty;
  CellWalk w(first, stride, tx, g.inv_tx,
             mtile + uint32_t(g.cy * R + g.cx) * uint32_t(sizeof(MT)), R,
             uint32_t(sizeof(MT)));
  uint32_t po[N];  // plane offsets in bytes
#pragma unroll
  for (int v = 0; v < N; ++v) po[v] = uint32_t((pp[v] >= 0 ? pp[v] : 0) * g.pst) * 8u;
  uint32_t ca = cfs + uint32_t(first) * 8u;
  const uint32_t dca = uint32_t(stride) * 8u;
  if constexpr (!MIXED) {
    const double sgn = g.pos_w ? 1.0 : -1.0;
    for (int c = first; c < ncell; c += stride) {
      double2 mv = ptx::lds_d2(w.tile);
      if constexpr (SCREEN) {
        const double phx = __dadd_rn(g.phi0x, __dmul_rn(double(w.X), g.dphix));
        const double phy = __dadd_rn(g.phi0y, __dmul_rn(double(w.Y), g.dphiy));
        mv = cmul_d(mv, cphase_d(__dsub_rn(-phx, phy)));
      }
      const double my = sgn * mv.y;
#pragma unroll
      for (int v = 0; v < N; ++v) {
        if (DENSE || pp[v] >= 0) {
          const float2 cf = ptx::lds_f2(ca + po[v]);
          const double cr = cf.x, ci = cf.y;
          acc[2 * v] = fma(cr, mv.x, fma(-ci, my, acc[2 * v]));
          acc[2 * v + 1] = fma(cr, my, fma(ci, mv.x, acc[2 * v + 1]));
        }
      }
      w.next(tx);
      ca += dca;
    }
#pragma unroll
    for (int v = 0; v < N; ++v) acc[2 * v + 1] *= sgn;
  } else {
    // Packed FP32 products (two per instruction): per plane v the thread
    // sums P = sum cf * (mx, mx) and Q = sum cf * (my, my) componentwise;
    // then Re = P.x - sgn Q.y and Im = Q.x + sgn P.y are the real and
    // imaginary parts of sum cf' * m (the imaginary part already times sgn).
    const float sgn = g.pos_w ? 1.0f : -1.0f;
    float2 P[N], Q[N];
#pragma unroll
    for (int v = 0; v < N; ++v) {
      P[v] = make_float2(0.f, 0.f);
      Q[v] = make_float2(0.f, 0.f);
    }
    for (int c = first; c < ncell; c += stride) {
      float2 mv = ptx::lds_f2(w.tile);
      if constexpr (SCREEN) {
        const double phx = __dadd_rn(g.phi0x, __dmul_rn(double(w.X), g.dphix));
        const double phy = __dadd_rn(g.phi0y, __dmul_rn(double(w.Y), g.dphiy));
        const double2 sc = cphase_d(__dsub_rn(-phx, phy));
        const float sx = float(sc.x), sy = float(sc.y);
        mv = make_float2(mv.x * sx - mv.y * sy, mv.x * sy + mv.y * sx);
      }
      const float2 xx = make_float2(mv.x, mv.x), yy = make_float2(mv.y, mv.y);
#pragma unroll
      for (int v = 0; v < N; ++v) {
        if (DENSE || pp[v] >= 0) {
          const float2 cf = ptx::lds_f2(ca + po[v]);
          P[v] = __ffma2_rn(cf, xx, P[v]);
          Q[v] = __ffma2_rn(cf, yy, Q[v]);
        }
      }
      w.next(tx);
      ca += dca;
    }
#pragma unroll
    for (int v = 0; v < N; ++v) {
      acc[2 * v] = fmaf(-sgn, Q[v].y, P[v].x);
      acc[2 * v + 1] = fmaf(sgn, P[v].y, Q[v].x);
    }
  }
}

// Gridding of one visibility's footprint cells c = first, first + stride,
// ... < end into the row's shared-memory grid tile (src/hpg_core.hpp:856-873).
// The gridding warps cover every cell of one visibility between two
// barriers, so no two threads add to a tile cell at once (measured faster
// than shared-memory atomics with two visibilities in flight).  pp[v]: slot
// plane of Mueller element gmi[row][v] (-1 if inactive; never when DENSE).
// gv[v] arrive conjugated when w > 0 (the CF imaginary part is negated
// then): conj(cf)*s*g = conj(cf*conj(s)*conj(g)), bit for bit in the
// reference's FP32 products, so only the sum's imaginary part flips.
// Loop state of grid_cells, formed from the descriptor alone: the gridding
// warps set it up while they still wait for the visibility's gridding
// values, so its address arithmetic is off the critical path.
template <int N>
struct GridCursor {
  CellWalk w;
  uint32_t po[N];  // plane offsets in bytes
  uint32_t ca, dca;
  int first, stride, end;
};

// a - b rounded once (an FMA with -1: the product is exact), two lanes
__device__ __forceinline__ float2 fsub2_rn(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}

// Compensated add of x into the tile cell (hi, lo) at shared address a,
// with the low part lo_off bytes further: hi + x = s + err exactly (Knuth's
// two-sum in round-to-nearest), hi <- s, lo <- lo + err.  The pair holds the
// cell's sum to within the rounding of lo, so a tile pass of any length
// adds no FP32 accumulation error beyond that.
__device__ __forceinline__ void two_sum_add(uint32_t a, uint32_t lo_off,
                                            float2 x) {
  const float2 hi = ptx::lds_f2(a);
  const float2 lo = ptx::lds_f2(a + lo_off);
  const float2 sum = __fadd2_rn(hi, x);
  const float2 bp = fsub2_rn(sum, hi);
  const float2 err = __fadd2_rn(fsub2_rn(hi, fsub2_rn(sum, bp)),
                                fsub2_rn(x, bp));
  ptx::sts_f2(a, sum);
  ptx::sts_f2(a + lo_off, __fadd2_rn(lo, err));
}

template <int N, bool MIXED>
__device__ __forceinline__ GridCursor<N> grid_prepare(
    const VisGeom& g, const int (&pp)[N], uint32_t cfs, uint32_t gtile, int R,
    int first, int stride, int end) {
  using GT = typename Form<MIXED>::grid_t;
  GridCursor<N> k{CellWalk(first, stride, g.tx, g.inv_tx,
                           gtile + uint32_t(g.cy * R + g.cx) * uint32_t(sizeof(GT)),
                           R, uint32_t(sizeof(GT)))};
#pragma unroll
  for (int v = 0; v < N; ++v)
    k.po[v] = uint32_t((pp[v] >= 0 ? pp[v] : 0) * g.pst) * 8u;
  k.ca = cfs + uint32_t(first) * 8u;
  k.dca = uint32_t(stride) * 8u;
  k.first = first;
  k.stride = stride;
  k.end = end;
  return k;
}

template <int N, bool MIXED, bool DENSE, bool SCREEN, bool COMP>
__device__ __forceinline__ void grid_cells(const VisGeom& g, const int (&pp)[N],
                                           GridCursor<N> k,
                                           const float2 (&gv)[N],
                                           uint32_t lo_off) {
  const int tx = g.tx, ncell = k.end, first = k.first, stride = k.stride;
  CellWalk& w = k.w;
  const uint32_t(&po)[N] = k.po;
  uint32_t ca = k.ca;
  const uint32_t dca = k.dca;
  // mixed form: with s = -1 for w > 0 (else +1) and g' = gv[v], the cell
  // gains (sum cf.x g'.x - cf.y g'.y, s * sum cf.x g'.y + cf.y g'.x), which
  // is (s1.x + s2.y, s1.y + s2.x) for ga = (g'.x, s g'.x), gb = (s g'.y, -g'.y)
  float2 ga[N], gb[N];
  if constexpr (MIXED) {
    const float sg = g.pos_w ? -1.0f : 1.0f;
#pragma unroll
    for (int v = 0; v < N; ++v) {
      ga[v] = make_float2(gv[v].x, sg * gv[v].x);
      gb[v] = make_float2(sg * gv[v].y, -gv[v].y);
    }
  }
  for (int c = first; c < ncell; c += stride) {
    float2 screen = make_float2(1.0f, 0.0f);
    if constexpr (SCREEN) {
      const double phx = __dadd_rn(g.phi0x, __dmul_rn(double(w.X), g.dphix));
      const double phy = __dadd_rn(g.phi0y, __dmul_rn(double(w.Y), g.dphiy));
      const double2 sc = cphase_d(__dadd_rn(phx, phy));
      screen = make_float2(__double2float_rn(sc.x),
                           g.pos_w ? -__double2float_rn(sc.y)
                                   : __double2float_rn(sc.y));
    }
    if constexpr (!MIXED) {
      double sx = 0.0, sy = 0.0;
#pragma unroll
      for (int v = 0; v < N; ++v) {
        if (DENSE || pp[v] >= 0) {
          const float2 cf = ptx::lds_f2(ca + po[v]);
          const float2 prod = SCREEN ? cmul_f(cmul_f(cf, screen), gv[v])
                                     : cmul_f(cf, gv[v]);
          sx = __dadd_rn(sx, double(prod.x));
          sy = __dadd_rn(sy, double(prod.y));
        }
      }
      double2 t = ptx::lds_d2(w.tile);
      t.x += sx;
      t.y = g.pos_w ? t.y - sy : t.y + sy;
      ptx::sts_d2(w.tile, t);
    } else {
      // packed FP32 products: s1 = sum cf * ga[v], s2 = sum cf * gb[v]
      // componentwise, and the cell's increment is (s1.x + s2.y, s1.y + s2.x)
      float2 s1 = make_float2(0.f, 0.f), s2 = make_float2(0.f, 0.f);
#pragma unroll
      for (int v = 0; v < N; ++v) {
        if (DENSE || pp[v] >= 0) {
          float2 cf = ptx::lds_f2(ca + po[v]);
          if constexpr (SCREEN)
            cf = make_float2(cf.x * screen.x - cf.y * screen.y,
                             cf.x * screen.y + cf.y * screen.x);
          s1 = __ffma2_rn(cf, ga[v], s1);
          s2 = __ffma2_rn(cf, gb[v], s2);
        }
      }
      const float2 inc = make_float2(s1.x + s2.y, s1.y + s2.x);
      if constexpr (COMP) {
        two_sum_add(w.tile, lo_off, inc);
      } else {
        const float2 t = ptx::lds_f2(w.tile);
        ptx::sts_f2(w.tile, __fadd2_rn(t, inc));
      }
    }
    w.next(tx);
    ca += dca;
  }
}

// COMP (mixed form only): compensated grid tiles, a low-part tile beside
// each group's tile, updated by two-sum
template <int N, bool MIXED, bool DENSE, bool COMP>
__global__ void __launch_bounds__(kThreadsTiled, 1)
tiled_kernel(const __grid_constant__ TiledParams p,
             const __grid_constant__ CUtensorMap model_map) {
  using MT = typename Form<MIXED>::model_t;
  using GT = typename Form<MIXED>::grid_t;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  // TMA destinations want 1024-byte alignment; the launch adds 1 KB of slack
  unsigned char* sm =
      sm_raw + ((1024u - (ptx::smem(sm_raw) & 1023u)) & 1023u);
  // same layout the host sized the launch with (tiles absent when unused)
  const SmemLayout L =
      smem_layout(p.ring_bytes, p.R, p.esize_model, p.esize_grid, p.grid_tiles);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + L.bars);
  uint64_t* empty = full + kSlots;
  uint64_t* model_bar = empty + kSlots;
  uint64_t* xchg = model_bar + 1;  // [kXSlots]
  uint64_t* dgfull = xchg + kXSlots;  // [2]
  uint64_t* dgempty = dgfull + 2;  // [2]
  uint64_t* gvfull = dgempty + 2;  // [kSlots]
  // copy requests of odd visibilities, from kPWarp to kPWarp + 1
  uint64_t* req = gvfull + kSlots;  // [kSlots]
  volatile int* abort = reinterpret_cast<volatile int*>(req + kSlots);
  double* xbuf = reinterpret_cast<double*>(sm + L.xbuf);  // [8][4][4][2]
  double* dgpart = reinterpret_cast<double*>(sm + L.wred);  // [2][kDG][8]
  // gridding values of visibility q in entry q % kSlots: the exchange warp
  // runs at most kSlots - 1 visibilities ahead of the gridding warps (the
  // producer reclaims a slot only after they are done with it)
  float2* gvring = reinterpret_cast<float2*>(sm + L.bcast);  // [kSlots][4]
  unsigned long long* slot_end =
      reinterpret_cast<unsigned long long*>(sm + L.slots);  // [kSlots]
  long long* req_src = reinterpret_cast<long long*>(slot_end + kSlots);
  int* ring_off = reinterpret_cast<int*>(req_src + kSlots);  // [kSlots]
  int* req_off = ring_off + kSlots;   // ring offset of a requested copy
  int* req_pst = req_off + kSlots;    // its CF plane stride
  int* req_desc = req_pst + kSlots;   // its descriptor index
  // last visibility whose copies were issued into slot s (-1: none), for the
  // drain before exit
  int* issued = req_desc + kSlots;
  TileDesc* descs = reinterpret_cast<TileDesc*>(sm + L.desc);
  unsigned char* ring = sm + L.ring;
  MT* mtile = reinterpret_cast<MT*>(sm + L.model);
  GT* gtile = reinterpret_cast<GT*>(sm + L.grid);

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int row = int(ptx::cluster_rank());
  const unsigned cid = ptx::cluster_id_x(), ncl = ptx::num_clusters_x();
  const bool exchange = p.do_degrid && p.has_model;
  // Slot q is released by the last roles to read it.  With gridding those
  // are the warps of the gridding group that takes q alone: they read it
  // after their wait on gvfull[q], which the exchange warp arrives on after
  // its own last read, and the exchange warp started only after the
  // degridding warps' hand-off (dgfull) that followed their last read.
  // Without gridding the exchange warp releases it too (the gridding warps
  // then only wait for the copies).
  constexpr int kGT = kGroups<MIXED, COMP>;
  constexpr int kTiles = kGT * (COMP ? 2 : 1);  // grid tiles in shared memory
  static_assert(MIXED || !COMP, "compensated tiles are a mixed-form option");
  const uint32_t empty_count = uint32_t(kGR / kGT + (p.do_grid ? 0 : 1));

  if (tid == 0) {
    for (int s = 0; s < kSlots; ++s) {
      ptx::mbar_init(&full[s], 1);
      ptx::mbar_init(&empty[s], empty_count);
    }
    ptx::mbar_init(model_bar, 1);
    for (int x = 0; x < kXSlots; ++x) ptx::mbar_init(&xchg[x], 1);
    for (int x = 0; x < 2; ++x) {
      ptx::mbar_init(&dgfull[x], kDGPer);
      ptx::mbar_init(&dgempty[x], 1);
    }
    for (int x = 0; x < kSlots; ++x) ptx::mbar_init(&gvfull[x], 1);
    for (int x = 0; x < kSlots; ++x) ptx::mbar_init(&req[x], 1);
    for (int x = 0; x < kSlots; ++x) issued[x] = -1;
    *abort = 0;
    reinterpret_cast<ptx::WaitCtl*>(const_cast<int*>(abort))->limit_ns =
        p.wait_limit_ns;
    ptx::fence_mbar_init();
  }
  __syncthreads();
  ptx::cluster_sync();  // every CTA's barriers exist before remote traffic

  const unsigned nchunks = *p.num_chunks;
  bool ok = true;
  const int R = p.R;
  const int RR = R * R;
  // slot planes of this row's Mueller elements for w <= 0 and w > 0, one
  // signed byte per element (-1: inactive), packed four to a register
  uint32_t dpk[2] = {0u, 0u}, gpk[2] = {0u, 0u};
#pragma unroll
  for (int w = 0; w < 2; ++w)
#pragma unroll
    for (int v = 0; v < N; ++v) {
      dpk[w] |= uint32_t(p.dpos[row][w][v] & 0xff) << (8 * v);
      gpk[w] |= uint32_t(p.gpos[row][w][v] & 0xff) << (8 * v);
    }

  int model_loads = 0;  // model-tile copies issued (thread 0 issues them)
  if (warp >= kPWarp) {
    // ---------------- producer warps ----------------
    // kPWarp: lane k holds the slice reference of visibility base+k of the
    // current chunk; per visibility the warp reserves a descriptor slot and
    // room in the byte ring, and lane 0 issues the bulk copies of its
    // descriptor and of the CF planes of this CTA's row for even
    // visibilities, or hands the copies of odd ones to kPWarp + 1 (req).
    // (An L2 prefetch of later slices was measured to slow the kernel: the
    // ring already keeps enough copies in flight to cover the HBM latency.)
    // this row's plane runs, held in registers (loops below are unrolled)
    const int nruns = p.nruns[row];
    const int nplanes = p.nplanes[row];
    int run_plane[kMaxRuns], run_len[kMaxRuns], run_dst[kMaxRuns];
#pragma unroll
    for (int u = 0; u < kMaxRuns; ++u) {
      run_plane[u] = p.run_plane[row][u];
      run_len[u] = p.run_len[row][u];
      run_dst[u] = p.run_dst[row][u];
    }
    const bool cf_needed = exchange || p.do_grid;
    // the copies of one visibility into slot s (one thread)
    auto issue = [&](int s, int roff, long long off, int pstride, int dindex,
                     uint32_t qv) {
      // test hook: CTA 0 never issues the copies of one visibility, so that
      // the waits for them run out (the slot's phase never completes)
      if (blockIdx.x == 0 && (long long)qv == p.withhold_vis) return;
      const uint32_t pbytes = uint32_t(pstride) * 8u;
      const uint32_t need = cf_needed ? uint32_t(nplanes) * pbytes : 0u;
      ring_off[s] = roff;
      ptx::mbar_expect_tx(&full[s], uint32_t(sizeof(TileDesc)) + need);
      ptx::bulk_g2s(&descs[s], &p.descs[dindex], uint32_t(sizeof(TileDesc)),
                    &full[s]);
      if (cf_needed) {
        unsigned char* dst = ring + roff;
        const float2* slice = p.cf + off;
#pragma unroll
        for (int u = 0; u < kMaxRuns; ++u)
          if (u < nruns)
            ptx::bulk_g2s(dst + run_dst[u] * pbytes,
                          slice + size_t(run_plane[u]) * pstride,
                          uint32_t(run_len[u]) * pbytes, &full[s]);
      }
      issued[s] = int(qv);
    };
    uint32_t q = 0;
    if (warp != kPWarp) {
      // second producer warp: the odd visibilities' copies, in order, as
      // kPWarp requests them (it never waits for this warp)
      for (unsigned c = cid; c < nchunks; c += ncl) {
        const int count = p.chunks[c].count;
        for (int k = int((q + 1) & 1); k < count; k += 2) {
          const uint32_t qq = q + uint32_t(k);
          const int s = int(qq % uint32_t(kSlots));
          ok &= ptx::mbar_wait(&req[s], (qq / kSlots) & 1, abort);
          if (lane == 0 && !*abort)
            issue(s, req_off[s], req_src[s], req_pst[s], req_desc[s], qq);
          __syncwarp();
        }
        q += uint32_t(count);
      }
    } else {
      uint32_t q_old = 0;               // oldest visibility not yet reclaimed
      unsigned long long head = 0;      // ring bytes allocated (monotonic)
      uint32_t pos = 0;                 // head modulo the ring size
      unsigned long long tail = 0;      // ring bytes released (monotonic)
      for (unsigned c = cid; c < nchunks; c += ncl) {
        const Chunk ch = p.chunks[c];
        SliceRef cur{};
        for (int k = 0; k < ch.count; ++k, ++q) {
          if ((k & 31) == 0) {
            cur = SliceRef{};
            if (k + lane < ch.count) cur = p.srefs[ch.start + k + lane];
          }
          const int kk = k & 31;
          const long long off = __shfl_sync(0xffffffffu, cur.off, kk);
          const int pstride = __shfl_sync(0xffffffffu, cur.pstride, kk);
          // Reclaim the oldest visibilities' slots until a descriptor slot
          // is free and the CF part fits in the byte ring (allocations never
          // straddle the ring end; they are released in order).
          const uint32_t pbytes = uint32_t(pstride) * 8u;
          const uint32_t need = cf_needed ? uint32_t(nplanes) * pbytes : 0u;
          const uint32_t rb = uint32_t(p.ring_bytes);
          for (;;) {
            unsigned long long h = head;
            uint32_t ps = pos;
            if (need > 0 && ps + need > rb) {
              h += rb - ps;
              ps = 0;
            }
            const bool need_slot = (q - q_old) >= uint32_t(kSlots);
            const bool need_space = need > 0 && h + need - tail > rb;
            if (!need_slot && !need_space) {
              head = h;
              pos = ps;
              break;
            }
            if (q_old == q) {  // cannot happen: the plan keeps need <= ring
              ok = false;
              break;
            }
            const int so = int(q_old % uint32_t(kSlots));
            ok &= ptx::mbar_wait(&empty[so], (q_old / kSlots) & 1, abort);
            tail = slot_end[so];
            ++q_old;
          }
          const int s = int(q % uint32_t(kSlots));
          // after an abort nothing is copied into slots that may still be read
          if (lane == 0 && !*abort) {
            slot_end[s] = head + need;
            if ((q & 1) == 0) {
              issue(s, int(pos), off, pstride, ch.start + k, q);
            } else {
              req_off[s] = int(pos);
              req_src[s] = off;
              req_pst[s] = pstride;
              req_desc[s] = ch.start + k;
              ptx::mbar_arrive(&req[s]);
            }
          }
          head += need;
          pos += need;
          __syncwarp();
        }
      }
    }
  } else {
    // ---------------- consumer roles ----------------
    // degridding warps [0, kDG), exchange warps [kXBase, kGRBase), gridding
    // warps [kGRBase, kGRBase + kGR).  Roles hand visibilities to each other
    // through mbarriers; all of them meet at chunk boundaries.
    uint32_t q = 0;
    uint32_t model_phase = 0;
    // the model tile of this cluster's chunk cc, copied by one thread.  FP64
    // form: the first chunk's here, each next one's as soon as the
    // degridding warps (its only readers) are done with the current one, so
    // the copy runs while the other roles finish the chunk and flush the
    // grid tile.  Mixed form: at the start of each chunk (loading early
    // there costs registers the mixed cell loops need: measured slower).
    constexpr bool kEarlyModel = !MIXED;
    auto load_model = [&](unsigned cc) {
      const int t = p.chunks[cc].tile;
      const int mx = (t % p.ntx) * p.T, my = ((t / p.ntx) % p.nty) * p.T;
      const int mc = t / (p.ntx * p.nty);
      // earlier generic-proxy reads of the tile precede this async write
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      ptx::mbar_expect_tx(model_bar, uint32_t(p.model_bytes));
      ptx::tma_load_3d(mtile, &model_map, 2 * mx, my, mc * p.nrow + row,
                       model_bar);
      ++model_loads;
    };
    if (kEarlyModel && exchange && tid == 0 && cid < nchunks && !*abort)
      load_model(cid);
    for (unsigned c = cid; c < nchunks; c += ncl) {
      const Chunk ch = p.chunks[c];
      const int tile = ch.tile;
      const int tx = tile % p.ntx;
      const int ty = (tile / p.ntx) % p.nty;
      const int cube = tile / (p.ntx * p.nty);
      const int x0 = tx * p.T, y0 = ty * p.T;
      ptx::named_sync(1, kConsumers);
      if (!kEarlyModel && exchange && tid == 0 && !*abort) load_model(c);
      if (p.do_grid)
        for (int i = tid; i < RR * kTiles; i += kConsumers) {
          GT z;
          z.x = 0;
          z.y = 0;
          gtile[i] = z;
        }
      if (exchange) {
        ok &= ptx::mbar_wait(model_bar, model_phase, abort);
        model_phase ^= 1;
      }
      ptx::named_sync(1, kConsumers);
      double wchunk = 0.0;

      if (warp < kDG) {
        // -------- degridding warps --------
        const int grp = warp / kDGPer;
        for (int k = 0; k < ch.count; ++k, ++q) {
          const int s = int(q % uint32_t(kSlots));
          if (!exchange || int(q % kDGGroups) != grp) continue;
          ok &= ptx::mbar_wait(&full[s], (q / kSlots) & 1, abort);
          if (ptx::warp_flag(abort)) continue;
          double acc[2 * N];
#pragma unroll
          for (int t = 0; t < 2 * N; ++t) acc[t] = 0.0;
          {
            const VisGeom vg = vis_geom(descs[s]);
            int pp[N];
#pragma unroll
            for (int v = 0; v < N; ++v)
              pp[v] = int(int8_t((vg.pos_w ? dpk[1] : dpk[0]) >> (8 * v)));
            // the phase screen is a separate instantiation: its code in
            // the loop costs instructions even when it is skipped
            if (vg.screen_on)
              degrid_cells<N, MIXED, DENSE, true>(
                  vg, pp, ptx::smem(ring) + uint32_t(ring_off[s]),
                  ptx::smem(mtile), R, (warp % kDGPer) * 32 + lane,
                  kDGPer * 32, acc);
            else
              degrid_cells<N, MIXED, DENSE, false>(
                  vg, pp, ptx::smem(ring) + uint32_t(ring_off[s]),
                  ptx::smem(mtile), R, (warp % kDGPer) * 32 + lane,
                  kDGPer * 32, acc);
          }
          // warp sum of the 8 (padded) partials: halve the values held per
          // lane at each of the first three levels, then butterfly; lane
          // L ends with the sum of value ((L>>4)&1)*4 + ((L>>3)&1)*2 + ((L>>2)&1).
          // The mixed form's partials are FP32 (exact in acc) and are summed
          // across the warp in FP32, the FP64 form's in FP64.
          using RR = typename std::conditional<MIXED, float, double>::type;
          RR v8[8];
#pragma unroll
          for (int t = 0; t < 8; ++t) v8[t] = t < 2 * N ? RR(acc[t]) : RR(0);
          RR v4[4], v2[2], v1;
          {
            const bool hi = lane & 16;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const RR give = hi ? v8[i] : v8[i + 4];
              const RR keep = hi ? v8[i + 4] : v8[i];
              v4[i] = keep + __shfl_xor_sync(0xffffffffu, give, 16);
            }
          }
          {
            const bool hi = lane & 8;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const RR give = hi ? v4[i] : v4[i + 2];
              const RR keep = hi ? v4[i + 2] : v4[i];
              v2[i] = keep + __shfl_xor_sync(0xffffffffu, give, 8);
            }
          }
          {
            const bool hi = lane & 4;
            const RR give = hi ? v2[0] : v2[1];
            const RR keep = hi ? v2[1] : v2[0];
            v1 = keep + __shfl_xor_sync(0xffffffffu, give, 4);
          }
          v1 += __shfl_xor_sync(0xffffffffu, v1, 2);
          v1 += __shfl_xor_sync(0xffffffffu, v1, 1);
          const int vidx = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 +
                           ((lane >> 2) & 1);
          const int b = int(q & 1);
          if (q >= 2) ok &= ptx::mbar_wait(&dgempty[b], ((q >> 1) & 1) ^ 1, abort);
          if (ptx::warp_flag(abort)) continue;
          if ((lane & 3) == 0) dgpart[(b * kDG + warp) * 8 + vidx] = double(v1);
          __syncwarp();
          if (lane == 0) ptx::mbar_arrive(&dgfull[b]);
          __syncwarp();
        }
        if constexpr (kEarlyModel) {
          // every degridding warp is done with this chunk's model tile
          ptx::named_sync(4, kDG * 32);
          if (exchange && tid == 0 && c + ncl < nchunks && !*abort)
            load_model(c + ncl);
        }
      } else if (warp < kGRBase) {
        // -------- exchange warps --------
        // Exchange warp xw takes the visibilities q with q % 2 == xw (the
        // degrid partial buffer q % 2 is its own).  For each of them it
        // sends this row's partials to every CTA of the cluster, waits for
        // the other rows' partials and finishes the visibility at once, so
        // that the gridding warps can take it up (and release its ring part)
        // as early as possible (the other exchange warp meanwhile takes the
        // next visibility).  A remote CTA
        // sends into exchange buffer q % 8 again only for q + 8, after it
        // finished q + 6, which needed this CTA's partials of q + 6, sent
        // after this warp finished q: the buffer is never overwritten while
        // it is read.
        const int xw = warp - kXBase;
        for (int k = 0; k < ch.count; ++k, ++q) {
          if ((q & 1) != uint32_t(xw)) continue;
          {
            // with degridding, the degridding warps' hand-off (dgfull)
            // follows their own wait on the slot's copies and covers it
            const int s = int(q % uint32_t(kSlots));
            if (!exchange) ok &= ptx::mbar_wait(&full[s], (q / kSlots) & 1, abort);
            if (exchange && !ptx::warp_flag(abort)) {
              const int xs = int(q % uint32_t(kXSlots));
              const int b = xw;
              ok &= ptx::mbar_wait(&dgfull[b], (q >> 1) & 1, abort);
              const bool live = !ptx::warp_flag(abort);
              double tot = 0.0;
              if (live && lane < 2 * N)
                for (int w = b * kDGPer; w < (b + 1) * kDGPer; ++w)
                  tot += dgpart[(b * kDG + w) * 8 + lane];
              __syncwarp();
              if (live && lane == 0) {
                ptx::mbar_arrive(&dgempty[b]);
                // this CTA expects every row's partials for visibility q
                ptx::mbar_expect_tx(&xchg[xs], uint32_t(p.nrow * 2 * N * 8));
              }
              // lane r*2N + t sends component t of this row's partial to CTA r
              const int r = lane / (2 * N), t = lane % (2 * N);
              const double v = __shfl_sync(0xffffffffu, tot, t);
              if (live && r < p.nrow)
                ptx::st_async_f64(&xbuf[((xs * 4 + row) * 4) * 2 + t],
                                  uint32_t(r), v, &xchg[xs]);
            }
          }
          {
            const int s = int(q % uint32_t(kSlots));
            const uint32_t qq = q;
            const TileDesc& d = descs[s];
            const int xs = int(qq % uint32_t(kXSlots));
            const int gs = int(qq % uint32_t(kSlots));
            // everything the finish needs from the descriptor is read
            // before the wait, so only the partial sums remain after it
            const int v = lane < N ? lane : 0;
            const double2 wfac = d.wfac[v];
            const float2 val = d.vals[v];
            const float wgt = d.weights[v];
            const double2 phasor = d.phasor;
            const float2 gv0 = d.gvis[v];
            const int vis_index = d.index;
            const double twgt = d.twgt[row];
            if (exchange)
              ok &= ptx::mbar_wait_cluster(&xchg[xs], (qq / kXSlots) & 1, abort);
            const bool live = !ptx::warp_flag(abort);
            float2 gout = make_float2(0.f, 0.f);
            if (live && lane < N) {
              if (p.do_degrid) {
                float2 pred = make_float2(0.f, 0.f);
                if (exchange) {
                  const double2* x =
                      reinterpret_cast<const double2*>(xbuf) + (xs * 4) * 4 + v;
                  double2 part[4];
#pragma unroll
                  for (int r = 0; r < 4; ++r)
                    part[r] = r < p.nrow ? x[r * 4] : make_double2(0.0, 0.0);
                  double2 num = make_double2(0.0, 0.0);
#pragma unroll
                  for (int r = 0; r < 4; ++r)
                    if (r < p.nrow) {
                      num.x += part[r].x;
                      num.y += part[r].y;
                    }
                  const double2 qv = cmul_d(num, wfac);
                  pred = make_float2(__double2float_rn(qv.x),
                                     __double2float_rn(qv.y));
                }
                float2* out = reinterpret_cast<float2*>(
                    p.records + size_t(vis_index) * p.rec_stride);
                if (p.do_grid) {
                  const float2 rr = make_float2(__fsub_rn(val.x, pred.x),
                                                __fsub_rn(val.y, pred.y));
                  if (row == 0) out[v] = rr;
                  gout = scale_for_gridding(rr, phasor, wgt);
                } else if (row == 0) {
                  out[v] = pred;
                }
              } else {
                gout = gv0;
              }
              if (p.do_grid) gvring[gs * 4 + v] = gout;
            }
            if (live && lane == 0 && p.do_grid) wchunk += twgt;
            __syncwarp();
            if (live && lane == 0) {
              if (p.do_grid)
                ptx::mbar_arrive(&gvfull[gs]);
              else
                ptx::mbar_arrive(&empty[s]);
            }
            __syncwarp();
          }
        }
      } else {
        // -------- gridding warps --------
        // The gridding warps form kGT groups: group g takes the
        // visibilities q with q % kGT == g and adds them into a grid
        // tile of its own, so two groups never touch the same tile.  The
        // warps of a group cover the cells of one visibility between two
        // barriers (id 2 + g), so footprints of the group's consecutive
        // visibilities that overlap are never added at the same time.
        const int gw = warp - kGRBase;
        constexpr int gper = kGR / kGT;  // warps per group
        const int grp = gw / gper;
        const uint32_t mytile =
            ptx::smem(gtile) + uint32_t(grp * RR) * uint32_t(sizeof(GT));
        // compensated tiles: the low parts of the groups' tiles follow their
        // high parts
        const uint32_t lo_off = uint32_t(kGT * RR) * uint32_t(sizeof(GT));
        bool first = true;  // the group's first visibility of the chunk
        for (int k = 0; k < ch.count; ++k, ++q) {
          if (int(q % uint32_t(kGT)) != grp) continue;
          const int s = int(q % uint32_t(kSlots));
          if (p.do_grid) {
            const int gs = int(q % uint32_t(kSlots));
            // The exchange warp arrives on gvfull only after it has seen
            // the slot's copies land (its own wait on full, or the
            // degridding warps' hand-off that followed theirs), so this one
            // wait also covers the slot: a wait on an mbarrier whose phase
            // is already complete still costs ~100 cycles here.
            ok &= ptx::mbar_wait(&gvfull[gs], (q / kSlots) & 1, abort);
            // loop state from the descriptor, formed while the other
            // gridding warps may still work on the previous visibility
            const VisGeom vg = vis_geom(descs[s]);
            int pp[N];
#pragma unroll
            for (int v = 0; v < N; ++v)
              pp[v] = int(int8_t((vg.pos_w ? gpk[1] : gpk[0]) >> (8 * v)));
            const GridCursor<N> cur = grid_prepare<N, MIXED>(
                vg, pp, ptx::smem(ring) + uint32_t(ring_off[s]), mytile, R,
                (gw % gper) * 32 + lane, gper * 32, vg.tx * vg.ty);
            if (!first) {
              if constexpr (kGT == 1)
                ptx::named_sync(2, gper * 32);
              else
                ptx::named_sync(2 + grp, gper * 32);
            }
            first = false;
            if (!ptx::warp_flag(abort)) {
              float2 gv[N];
#pragma unroll
              for (int v = 0; v < N; ++v) {
                gv[v] = gvring[gs * 4 + v];
                if (vg.pos_w) gv[v].y = -gv[v].y;
              }
              if (vg.screen_on)
                grid_cells<N, MIXED, DENSE, true, COMP>(vg, pp, cur, gv, lo_off);
              else
                grid_cells<N, MIXED, DENSE, false, COMP>(vg, pp, cur, gv, lo_off);
            }
          } else {
            // nothing to grid: release the slot once its copies landed
            ok &= ptx::mbar_wait(&full[s], (q / kSlots) & 1, abort);
          }
          __syncwarp();
          if (lane == 0) ptx::mbar_arrive(&empty[s]);
        }
      }
      ptx::named_sync(1, kConsumers);
      if (p.do_grid && !*abort) {
        double2* plane = p.grid + size_t(cube * p.nrow + row) * p.ny * p.nx;
        for (int i = tid; i < RR; i += kConsumers) {
          const int gx = x0 + i % R, gy = y0 + i / R;
          if (gx < p.nx && gy < p.ny) {
            // the gridding groups' tiles (with their low parts), summed in
            // FP64
            double vx = 0.0, vy = 0.0;
#pragma unroll
            for (int t = 0; t < kTiles; ++t) {
              const GT v = gtile[t * RR + i];
              vx += double(v.x);
              vy += double(v.y);
            }
            if (vx != 0 || vy != 0) {
              double2* dst = plane + size_t(gy) * p.nx + gx;
              atomicAdd(&dst->x, vx);
              atomicAdd(&dst->y, vy);
            }
          }
        }
        if (warp >= kXBase && warp < kGRBase && lane == 0 && p.update_weights &&
            wchunk != 0.0)
          atomicAdd(p.weights + size_t(cube) * p.nrow + row, wchunk);
      }
    }
  }
  // Drain: after an abort the waits return early, so bulk copies issued
  // into this CTA's shared memory may still be in flight; each has landed
  // before the CTA leaves (on the normal path each was waited for already,
  // and these waits return at once).  The exchange's st.async stores into
  // peers are weak memory operations of their issuing threads, ordered
  // before the release of the cluster barrier below.
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < kSlots; ++s)
      if (issued[s] >= 0)
        ok &= ptx::mbar_drain(&full[s], (uint32_t(issued[s]) / kSlots) & 1,
                              abort);
    if (model_loads > 0)
      ok &= ptx::mbar_drain(model_bar, uint32_t(model_loads - 1) & 1, abort);
  }
  if (!ok) atomicOr(p.status, kStatusWaitTimeout);
  __syncwarp();
  ptx::cluster_sync();  // no CTA leaves while peers may still address it
}

// ---------------------------------------------------------------------------
// host side


PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

struct Plan {
  bool ok = false;
  std::string why;
  int R = 0, T = 0, ring_bytes = 0, K = 0;
  TiledParams p{};
  int smem = 0;
};

Plan make_plan(const hpgb_gridder* g, unsigned flags, bool mixed,
               size_t nvis) {
  Plan pl;
  const CFRegion& cf = g->cf;
  const int nrow = int(g->grid_size[2]);
  if (cf.groups.empty()) {
    pl.why = "no CF groups";
    return pl;
  }
  if (nrow < 1 || nrow > 4) {
    pl.why = "rows";
    return pl;
  }
  TiledParams& p = pl.p;
  std::memset(&p, 0, sizeof(p));
  for (int r = 0; r < 4; ++r)
    for (int v = 0; v < 4; ++v)
      if (g->mt.m[r][v] >= 64 || g->mt.c[r][v] >= 64) {
        pl.why = "Mueller index beyond 63";
        return pl;
      }
  // planes each row's CTA needs: Mueller row r of both index sets
  int max_planes = 0;
  for (int r = 0; r < nrow; ++r) {
    bool need[64] = {false};
    for (int v = 0; v < 4; ++v) {
      if (g->mt.m[r][v] >= 0) need[g->mt.m[r][v]] = true;
      if (g->mt.c[r][v] >= 0) need[g->mt.c[r][v]] = true;
    }
    int pos[64];
    int np = 0, nr = 0;
    for (int m = 0; m < 64; ++m) {
      pos[m] = -1;
      if (!need[m]) continue;
      pos[m] = np;
      if (m > 0 && need[m - 1]) {
        p.run_len[r][nr - 1]++;
      } else {
        if (nr == kMaxRuns) {
          pl.why = "too many plane runs";
          return pl;
        }
        p.run_plane[r][nr] = m;
        p.run_len[r][nr] = 1;
        p.run_dst[r][nr] = np;
        ++nr;
      }
      ++np;
    }
    p.nplanes[r] = np;
    p.nruns[r] = nr;
    max_planes = std::max(max_planes, np);
    for (int w = 0; w < 2; ++w)
      for (int v = 0; v < 4; ++v) {
        // pos_w (w = 1): degrid uses conjugate indexes, grid uses indexes
        const int dm = w ? g->mt.c[r][v] : g->mt.m[r][v];
        const int gm = w ? g->mt.m[r][v] : g->mt.c[r][v];
        p.dpos[r][w][v] = dm >= 0 ? pos[dm] : -1;
        p.gpos[r][w][v] = gm >= 0 ? pos[gm] : -1;
      }
  }
  int max_plane_bytes = 0;
  for (const CFGroup& G : cf.groups)
    max_plane_bytes = std::max(max_plane_bytes, G.plane_stride * 8);
  const int part = align_up(std::max(max_planes * max_plane_bytes, 16), 128);
  const int esize = mixed ? 8 : 16;
  const bool do_degrid = flags & HPGB_DO_DEGRID;
  const bool do_grid = flags & HPGB_DO_GRID;
  const int em = (do_degrid && g->has_model) ? esize : 0;
  const int eg = do_grid ? esize : 0;
  const int budget = 227 * 1024;
  const int taps = std::max(cf.max_taps_x, cf.max_taps_y);
  // CF byte ring: five of the largest parts if the tiles still fit, else
  // four (more visibilities in flight when parts are smaller); the tiles
  // take the rest.  The deeper ring is taken only while the smaller tiles it
  // leaves still hold kMinVisPerTile visibilities of the batch on average
  // (measured: the deeper ring wins at 10M visibilities on a 2048^2 grid in
  // both forms, loses at 1M in the FP64 form, whose 16-byte tiles shrink to
  // 5x5 cells).  CF slices too wide for four parts (supports up to 64 with
  // one or two Mueller planes per row: 65^2 taps are 33 KB a plane) get a
  // ring of three or two: no role waits for a later visibility before it
  // hands on or releases visibility q, so any ring that holds the largest
  // part keeps the pipeline moving; a shallower one only keeps fewer
  // visibilities in flight, which the longer per-visibility work of wide
  // footprints covers.  kMinRingParts is the least the plan takes.
  constexpr int kMinRingParts = 2;
  constexpr size_t kMinVisPerTile = 32;
  const hpgb_tiled_plan& tp = g->tplan;
  const bool fixed = tp.ring_parts > 0;
  const int m_hi = fixed ? tp.ring_parts : 5;
  const int m_lo = fixed ? tp.ring_parts : kMinRingParts;
  if (m_lo < kMinRingParts) {
    pl.why = "the CF ring must hold at least two parts";
    return pl;
  }
  // grid tiles: one per gridding group, and in the compensated mixed form
  // a low-part tile beside each
  const bool comp = mixed && do_grid && tp.compensated == HPGB_COMPENSATED_ON;
  const int gt = comp ? 2 * kCompGroups : mixed ? kGridTiles<true> : kGridTiles<false>;
  for (int m = m_hi; m >= m_lo; --m) {
    const int rb = m * part;
    const SmemLayout L0 = smem_layout(rb, 0, em, eg, gt);
    const int left = budget - L0.total - 1024 - 1024;
    if (left <= 0) continue;
    const int per_cell = em + eg * gt;
    int R = per_cell > 0 ? int(std::sqrt(double(left) / double(per_cell))) : 128;
    R = std::min(R, 128) & ~1;
    if (tp.tile_side > 0) {
      if (tp.tile_side > R) continue;  // no room for the requested side
      R = tp.tile_side;
    }
    if (R - taps + 1 < 4) continue;
    if (!fixed && m > m_lo) {
      const size_t T = size_t(R - taps + 1);
      const size_t ntiles = ((g->grid_size[0] + T - 1) / T) *
                            ((g->grid_size[1] + T - 1) / T) * g->grid_size[3];
      if (nvis < kMinVisPerTile * ntiles) continue;
    }
    pl.ring_bytes = rb;
    pl.R = R;
    break;
  }
  if (pl.ring_bytes == 0) {
    pl.why = "CF slice part too large for the shared-memory ring";
    return pl;
  }
  pl.T = pl.R - taps + 1;
  pl.K = tp.chunk_vis > 0
             ? tp.chunk_vis
             : (!mixed ? kChunkVisFP64 : comp ? kChunkVisMixedComp : kChunkVisMixed);
  pl.smem = smem_layout(pl.ring_bytes, pl.R, em, eg, gt).total + 1024;
  if (em > 0 && (2 * size_t(g->grid_size[0]) * (mixed ? 4 : 8)) % 16 != 0) {
    pl.why = "model row pitch not a 16-byte multiple";
    return pl;
  }
  p.nx = int(g->grid_size[0]);
  p.ny = int(g->grid_size[1]);
  p.nrow = nrow;
  p.ncube = int(g->grid_size[3]);
  p.R = pl.R;
  p.T = pl.T;
  p.ntx = (p.nx + pl.T - 1) / pl.T;
  p.nty = (p.ny + pl.T - 1) / pl.T;
  p.ring_bytes = pl.ring_bytes;
  p.model_bytes = pl.R * pl.R * esize;
  p.esize_model = em;
  p.esize_grid = eg;
  p.grid_tiles = gt;
  p.compensated = comp;
  p.do_degrid = do_degrid;
  p.do_grid = do_grid;
  p.update_weights = (flags & HPGB_UPDATE_GRID_WEIGHTS) != 0;
  p.has_model = g->has_model;
  pl.ok = true;
  return pl;
}

template <int N, bool MIXED>
Status launch_tiled(hpgb_gridder* g, const TiledParams& p, int smem,
                    const CUtensorMap& map) {
  using MT = typename Form<MIXED>::model_t;
  using GT = typename Form<MIXED>::grid_t;
  // the kernel places its tiles with these sizes; they must match the form
  const bool comp = MIXED && p.compensated;
  if ((p.esize_model != 0 && p.esize_model != int(sizeof(MT))) ||
      p.grid_tiles != (comp ? 2 * kCompGroups : kGridTiles<MIXED>) ||
      (p.esize_grid != 0 && p.esize_grid != int(sizeof(GT))) ||
      smem_layout(p.ring_bytes, p.R, p.esize_model, p.esize_grid,
                  p.grid_tiles).total +
              1024 > smem)
    return Status::err(HPGB_ERROR_OTHER, "tiled kernel layout mismatch");
  if ((p.do_degrid && p.has_model && p.esize_model == 0) ||
      (p.do_grid && p.esize_grid == 0))
    return Status::err(HPGB_ERROR_OTHER, "tiled kernel tile missing");
  // every Mueller element of every row active: the cell loops skip the
  // per-element activity test
  bool dense = true;
  for (int r = 0; r < p.nrow; ++r)
    for (int w = 0; w < 2; ++w)
      for (int v = 0; v < N; ++v)
        dense = dense && p.dpos[r][w][v] >= 0 && p.gpos[r][w][v] >= 0;
  auto kern = dense ? (comp ? tiled_kernel<N, MIXED, true, MIXED>
                            : tiled_kernel<N, MIXED, true, false>)
                   : (comp ? tiled_kernel<N, MIXED, false, MIXED>
                           : tiled_kernel<N, MIXED, false, false>);
  HPGB_CUDA_TRY(cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = unsigned(p.nrow);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.blockDim = dim3(kThreadsTiled);  // 20 warps
  cfg.dynamicSmemBytes = size_t(smem);
  cfg.stream = g->stream;
  int sms = 0;
  HPGB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount,
                                       g->device));
  cfg.gridDim = dim3(unsigned(sms / p.nrow * p.nrow));
  int max_clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg) == cudaSuccess &&
      max_clusters > 0)
    cfg.gridDim = dim3(unsigned(max_clusters * p.nrow));
  else
    cudaGetLastError();
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (g->profile) {
    HPGB_CUDA_TRY(cudaEventCreate(&ev[0]));
    HPGB_CUDA_TRY(cudaEventCreate(&ev[1]));
    HPGB_CUDA_TRY(cudaEventRecord(ev[0], g->stream));
  }
  HPGB_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, p, map));
  ++g->launches;
  if (g->profile) {
    HPGB_CUDA_TRY(cudaEventRecord(ev[1], g->stream));
    g->prof_events.emplace_back(ev[0], ev[1]);
  }
  return Status::ok();
}

template <int N>
Status prepare_tiles_n(hpgb_gridder* g, void* d_vis, size_t n, int T, int ntx,
                       int nty, int K, TilePrep* out) {
  VisBuffers& vb = g->vb;
  const GridGeom geom = g->geom();
  const CFGroup* groups = g->cf.desc.as<const CFGroup>();
  TileGeom tg;
  tg.T = T;
  tg.ntx = ntx;
  tg.nty = nty;
  tg.ntiles = tg.ntx * tg.nty * int(g->grid_size[3]);
  const int ntiles = tg.ntiles;
  const size_t max_chunks = n / K + size_t(ntiles) + 1;
  // scratch
  HPGB_TRY(vb.keys.reserve(n * 4));
  HPGB_TRY(vb.keys_alt.reserve(n * 4));
  HPGB_TRY(vb.order.reserve(n * 4));
  HPGB_TRY(vb.order_alt.reserve(n * 4));
  HPGB_TRY(vb.buckets.reserve(size_t(ntiles + 1) * 4 * 4));
  HPGB_TRY(vb.items.reserve(max_chunks * sizeof(Chunk)));
  HPGB_TRY(vb.prep.reserve(n * (sizeof(TileDesc) + sizeof(SliceRef))));
  unsigned* counts = vb.buckets.as<unsigned>();
  unsigned* tstart = counts + (ntiles + 1);
  unsigned* nch = tstart + (ntiles + 1);
  unsigned* cstart = nch + (ntiles + 1);
  unsigned* num_chunks = vb.counters.as<unsigned>() + 1;
  TileDesc* descs = vb.prep.as<TileDesc>();
  SliceRef* srefs = reinterpret_cast<SliceRef*>(vb.prep.as<char>() +
                                                n * sizeof(TileDesc));
  // CUB scratch sizing
  int end_bit = 1;
  while ((1ll << end_bit) <= (long long)ntiles) ++end_bit;
  size_t sort_bytes = 0, scan_bytes = 0;
  cub::DoubleBuffer<unsigned> kbuf(vb.keys.as<unsigned>(), vb.keys_alt.as<unsigned>());
  cub::DoubleBuffer<unsigned> vbuf(vb.order.as<unsigned>(), vb.order_alt.as<unsigned>());
  HPGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, kbuf, vbuf,
                                                int(n), 0, end_bit, g->stream));
  HPGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts,
                                              tstart, ntiles, g->stream));
  HPGB_TRY(vb.sort_tmp.reserve(std::max(sort_bytes, scan_bytes) + 16));

  HPGB_CUDA_TRY(cudaMemsetAsync(counts, 0, size_t(ntiles + 1) * 4, g->stream));
  const unsigned blocks = unsigned((n + 255) / 256);
  tile_keys_kernel<N><<<blocks, 256, 0, g->stream>>>(
      static_cast<const VisData<N>*>(d_vis), n, geom, groups, tg,
      vb.keys.as<unsigned>(), vb.order.as<unsigned>(), counts);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  size_t tmp_bytes = vb.sort_tmp.bytes;
  HPGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(vb.sort_tmp.ptr, tmp_bytes, kbuf,
                                                vbuf, int(n), 0, end_bit,
                                                g->stream));
  tmp_bytes = vb.sort_tmp.bytes;
  HPGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(vb.sort_tmp.ptr, tmp_bytes, counts,
                                              tstart, ntiles, g->stream));
  const unsigned tblocks = unsigned((ntiles + 255) / 256);
  chunk_count_kernel<<<tblocks, 256, 0, g->stream>>>(counts, ntiles, K, nch);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  tmp_bytes = vb.sort_tmp.bytes;
  HPGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(vb.sort_tmp.ptr, tmp_bytes, nch,
                                              cstart, ntiles, g->stream));
  chunk_write_kernel<<<tblocks, 256, 0, g->stream>>>(
      counts, tstart, nch, cstart, ntiles, K, vb.items.as<Chunk>(), num_chunks);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  tile_desc_kernel<N><<<blocks, 256, 0, g->stream>>>(
      static_cast<const VisData<N>*>(d_vis), vbuf.Current(), kbuf.Current(), n,
      geom, groups, tg, g->cf.data.as<const float2>(), descs, srefs);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;

  out->descs = descs;
  out->srefs = srefs;
  out->chunks = vb.items.as<Chunk>();
  out->num_chunks = num_chunks;
  out->max_chunks = max_chunks;
  return Status::ok();
}

template <int N>
Status grid_tiled_n(hpgb_gridder* g, void* d_vis, size_t n, unsigned flags,
                    const Plan& plan, bool mixed) {
  TilePrep prep;
  HPGB_TRY(prepare_tiles_n<N>(g, d_vis, n, plan.T, plan.p.ntx, plan.p.nty,
                              plan.K, &prep));
  VisBuffers& vb = g->vb;
  TileDesc* descs = const_cast<TileDesc*>(prep.descs);
  SliceRef* srefs = const_cast<SliceRef*>(prep.srefs);
  unsigned* num_chunks = const_cast<unsigned*>(prep.num_chunks);
  TiledParams p = plan.p;
  p.descs = descs;
  p.srefs = srefs;
  p.chunks = vb.items.as<Chunk>();
  p.num_chunks = num_chunks;
  p.cf = g->cf.data.as<const float2>();
  p.grid = g->grid.as<double2>();
  p.weights = g->weights.as<double>();
  p.records = static_cast<unsigned char*>(d_vis);
  p.rec_stride = int(sizeof(VisData<N>));
  p.status = vb.counters.as<unsigned>();
  p.wait_limit_ns = g->wait_limit_ns;
  p.withhold_vis = g->withhold_vis;

  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  if (p.do_degrid && p.has_model) {
    const void* base = g->model.ptr;
    size_t esize = 8;
    CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    if (mixed) {
      const size_t ne = g->grid_elems();
      if (!g->model32_valid) {
        HPGB_TRY(g->model32.reserve(std::max<size_t>(ne, 1) * sizeof(float2)));
        model_to_f32_kernel<<<148 * 8, 256, 0, g->stream>>>(
            g->model.as<const double2>(), g->model32.as<float2>(), ne);
        HPGB_CUDA_TRY(cudaGetLastError());
        ++g->launches;
        g->model32_valid = true;
      }
      base = g->model32.ptr;
      esize = 4;
      dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    }
    auto enc = tensor_map_encoder();
    if (!enc) return Status::err(HPGB_ERROR_OTHER, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[3] = {cuuint64_t(2 * p.nx), cuuint64_t(p.ny),
                          cuuint64_t(p.nrow * p.ncube)};
    cuuint64_t strides[2] = {cuuint64_t(2 * p.nx) * esize,
                             cuuint64_t(2 * p.nx) * p.ny * esize};
    cuuint32_t box[3] = {cuuint32_t(2 * p.R), cuuint32_t(p.R), 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&map, dt, 3, const_cast<void*>(base), dims, strides, box,
                     estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      return Status::err(HPGB_ERROR_OTHER,
                         "cuTensorMapEncodeTiled failed: " + std::to_string(int(r)));
  }
  if (mixed) return launch_tiled<N, true>(g, p, plan.smem, map);
  return launch_tiled<N, false>(g, p, plan.smem, map);
}

}  // namespace

Status prepare_tiles(hpgb_gridder* g, void* d_vis, size_t n, int T, int ntx,
                     int nty, int K, TilePrep* out) {
  switch (g->npol) {
    case 1: return prepare_tiles_n<1>(g, d_vis, n, T, ntx, nty, K, out);
    case 2: return prepare_tiles_n<2>(g, d_vis, n, T, ntx, nty, K, out);
    case 3: return prepare_tiles_n<3>(g, d_vis, n, T, ntx, nty, K, out);
    case 4: return prepare_tiles_n<4>(g, d_vis, n, T, ntx, nty, K, out);
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
}

bool tiled_plan_side(const hpgb_gridder* g, unsigned flags, size_t n,
                     int* side) {
  const Plan plan =
      make_plan(g, flags, g->precision == HPGB_PRECISION_MIXED, n);
  *side = plan.ok ? plan.R : 0;
  return plan.ok;
}

Status grid_tiled(hpgb_gridder* g, void* d_vis, size_t n, unsigned flags,
                  bool* used) {
  *used = false;
  if (n == 0) return Status::ok();
  if (!(flags & (HPGB_DO_DEGRID | HPGB_DO_GRID))) {
    *used = true;
    return Status::ok();
  }
  if (n > size_t(0x7fffffff)) return Status::ok();
  const bool mixed = g->precision == HPGB_PRECISION_MIXED;
  const Plan plan = make_plan(g, flags, mixed, n);
  if (!plan.ok) return Status::ok();
  *used = true;
  switch (g->npol) {
    case 1: return grid_tiled_n<1>(g, d_vis, n, flags, plan, mixed);
    case 2: return grid_tiled_n<2>(g, d_vis, n, flags, plan, mixed);
    case 3: return grid_tiled_n<3>(g, d_vis, n, flags, plan, mixed);
    case 4: return grid_tiled_n<4>(g, d_vis, n, flags, plan, mixed);
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
}

}  // namespace hpgb

