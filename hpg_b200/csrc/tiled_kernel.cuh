// tiled_kernel.cuh -- the fused degrid -> residual -> grid kernel over
// shared-memory uv tiles (the hot path; pipeline and arithmetic forms are
// described in grid_tiled.cu), its launch parameters and shared-memory
// layout.  Included by grid_tiled.cu (launches for one gridder) and
// grid_batch.cu (one launch over the batches of many gridders).
#pragma once

#include <cuda.h>

#include <string>
#include <type_traits>
#include <vector>

#include "gridder.cuh"
#include "ptx.cuh"
#include "tiles.cuh"

namespace hpgb {
namespace tiled {


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
// issues the copies of visibilities q with q % kProducers == 0, helper warp
// kPWarp + h those with q % kProducers == h
#ifndef HPGB_TILED_PRODUCERS
#define HPGB_TILED_PRODUCERS 2
#endif
constexpr int kProducers = HPGB_TILED_PRODUCERS;
constexpr int kThreadsTiled = kConsumers + 32 * kProducers;
constexpr int kSlots = 16;  // descriptor slots (visibilities in flight)
constexpr int kChunkVisFP64 = 2048;
constexpr int kChunkVisMixed = 256;
// compensated tiles accumulate without FP32 error: longer passes
constexpr int kChunkVisMixedComp = 2048;
constexpr int kMaxRuns = 8;

// The per-gridder part of a batched launch (grid_batch.cu): what differs
// between the gridders whose tile passes one launch takes.  Tile passes
// name their gridder in Chunk::pad.  In global memory, 64-byte aligned (the
// model's tensor map comes first).
constexpr int kMaxBatchJobs = 96;  // gridders one batched launch takes
struct alignas(64) BatchJob {
  CUtensorMap model_map;
  const TileDesc* descs;
  const SliceRef* srefs;
  const float2* cf;
  double2* grid;
  double* weights;
  unsigned char* records;
  int nx, ny, T, ntx, nty, pad;
};

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
  const BatchJob* jobs;  // batched launches: the gridders' job table
  unsigned long long wait_limit_ns;  // bound of every wait in the kernel
  // test hook: the CTA of row 0 that takes this visibility (its position in
  // the tile-sorted batch; of the first gridder in a batched launch) never
  // issues its copies, so that the waits for them run out; -1: none
  long long withhold_vis;
};

// single fields of a tile pass's gridder: from the launch parameters (the
// constant bank), or in a batched launch from the job table in global
// memory.  The consumer roles read them where they are used, once per pass
// (holding them across a pass would add register pressure to the cell
// loops); the producer warps, which need the descriptor and CF bases for
// every visibility, read those once per pass into registers.
#define HPGB_JOB(BATCH, p, j, field) ((BATCH) ? (p).jobs[j].field : (p).field)

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
// the tiled kernel

template <bool MIXED>
struct Form;

// gridding groups, each with a grid tile of its own: two in the mixed form
// (8-byte tiles leave room for a second one), one in the FP64 form
template <bool MIXED>
constexpr int kGridTiles = MIXED ? 2 : 1;
// gridding groups of the compensated mixed form (each with a high and a low
// tile: four tiles, so the ring gets less room than in the plain form;
// measured 7.9% faster than one group of eight warps with its two tiles)
constexpr int kCompGroups = 2;
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
template <int N, bool MIXED, bool DENSE, bool COMP, bool BATCH>
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
  // copy requests from kPWarp to its helper warps
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
    reinterpret_cast<ptx::WaitCtl*>(const_cast<int*>(abort))->copies = 0;
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

  // model-tile copies issued (thread 0 issues them), kept in shared memory
  volatile int* model_loads = &reinterpret_cast<ptx::WaitCtl*>(
                                   const_cast<int*>(abort))->copies;
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
    // the withholding test hook applies to the current pass (row 0, the
    // first gridder's passes)
    bool hook_job = false;
    // the copies of one visibility into slot s (one thread); jdescs, jcf:
    // the descriptors and CF of the pass's gridder (read from the job table
    // once per pass in a batched launch)
    auto issue = [&](const TileDesc* jdescs, const float2* jcf, int s,
                     int roff, long long off, int pstride, int dindex,
                     uint32_t qv) {
      // test hook: row 0 never issues the copies of one visibility, so
      // that the waits for them run out (the slot's phase never completes)
      if (hook_job && (long long)dindex == p.withhold_vis) return;
      const uint32_t pbytes = uint32_t(pstride) * 8u;
      const uint32_t need = cf_needed ? uint32_t(nplanes) * pbytes : 0u;
      ring_off[s] = roff;
      ptx::mbar_expect_tx(&full[s], uint32_t(sizeof(TileDesc)) + need);
      ptx::bulk_g2s(&descs[s], &jdescs[dindex], uint32_t(sizeof(TileDesc)),
                    &full[s]);
      if (cf_needed) {
        unsigned char* dst = ring + roff;
        const float2* slice = jcf + off;
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
      // helper producer warp h: the copies of the visibilities q with
      // q % kProducers == h, in order, as kPWarp requests them (kPWarp never
      // waits for a helper)
      const uint32_t h = uint32_t(warp - kPWarp);
      for (unsigned c = cid; c < nchunks; c += ncl) {
        const int count = p.chunks[c].count;
        const int cjob = BATCH ? p.chunks[c].pad : 0;
        hook_job = p.withhold_vis >= 0 && row == 0 && cjob == 0;
        const TileDesc* jdescs = HPGB_JOB(BATCH, p, cjob, descs);
        const float2* jcf = HPGB_JOB(BATCH, p, cjob, cf);

        for (int k = int((h + kProducers - q % kProducers) % kProducers);
             k < count; k += kProducers) {
          const uint32_t qq = q + uint32_t(k);
          const int s = int(qq % uint32_t(kSlots));
          ok &= ptx::mbar_wait(&req[s], (qq / kSlots) & 1, abort);
          if (lane == 0 && !*abort)
            issue(jdescs, jcf, s, req_off[s], req_src[s], req_pst[s],
                  req_desc[s], qq);
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
        hook_job = p.withhold_vis >= 0 && row == 0 && (!BATCH || ch.pad == 0);
        const TileDesc* jdescs = HPGB_JOB(BATCH, p, ch.pad, descs);
        const float2* jcf = HPGB_JOB(BATCH, p, ch.pad, cf);
        const SliceRef* jsrefs = HPGB_JOB(BATCH, p, ch.pad, srefs);
        SliceRef cur{};
        for (int k = 0; k < ch.count; ++k, ++q) {
          if ((k & 31) == 0) {
            cur = SliceRef{};
            if (k + lane < ch.count) cur = jsrefs[ch.start + k + lane];
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
            if (q % kProducers == 0) {
              issue(jdescs, jcf, s, int(pos), off, pstride, ch.start + k, q);
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
    // through mbarriers and never wait for one another at chunk boundaries:
    // the degridding warps meet there among themselves (model tile), the
    // gridding warps among themselves (zeroing and flush of their tiles).
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
      const Chunk chm = p.chunks[cc];
      const int mj = chm.pad;
      const int t = chm.tile;
      const int mntx = HPGB_JOB(BATCH, p, mj, ntx);
      const int mnty = HPGB_JOB(BATCH, p, mj, nty);
      const int mT = HPGB_JOB(BATCH, p, mj, T);
      const int mx = (t % mntx) * mT, my = ((t / mntx) % mnty) * mT;
      const int mc = t / (mntx * mnty);
      const CUtensorMap* mmap = BATCH ? &p.jobs[mj].model_map : &model_map;
      // earlier generic-proxy reads of the tile precede this async write
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      ptx::mbar_expect_tx(model_bar, uint32_t(p.model_bytes));
      ptx::tma_load_3d(mtile, mmap, 2 * mx, my, mc * p.nrow + row,
                       model_bar);
      *model_loads = *model_loads + 1;
    };
    if (kEarlyModel && exchange && tid == 0 && cid < nchunks && !*abort)
      load_model(cid);
    for (unsigned c = cid; c < nchunks; c += ncl) {
      const Chunk ch = p.chunks[c];
      const int job = ch.pad;
      const int tile = ch.tile;
      const int jntx = HPGB_JOB(BATCH, p, job, ntx);
      const int jnty = HPGB_JOB(BATCH, p, job, nty);
      const int jT = HPGB_JOB(BATCH, p, job, T);
      const int tx = tile % jntx;
      const int ty = (tile / jntx) % jnty;
      const int cube = tile / (jntx * jnty);
      const int x0 = tx * jT, y0 = ty * jT;

      if (warp < kDG) {
        // -------- degridding warps --------
        // the chunk's model tile: mixed form, loaded here once every
        // degridding warp (its only readers) is done with the previous one
        if constexpr (!kEarlyModel) {
          ptx::named_sync(4, kDG * 32);
          if (exchange && tid == 0 && !*abort) load_model(c);
        }
        if (exchange) {
          ok &= ptx::mbar_wait(model_bar, model_phase, abort);
          model_phase ^= 1;
        }
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
        double wchunk = 0.0;  // this warp's share of the row's weight sum
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
                    HPGB_JOB(BATCH, p, job, records) +
                    size_t(vis_index) * p.rec_stride);
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
        if (lane == 0 && p.do_grid && p.update_weights && wchunk != 0.0 &&
            !*abort)
          atomicAdd(HPGB_JOB(BATCH, p, job, weights) + size_t(cube) * p.nrow + row,
                    wchunk);
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
        // Thread gt of the gridding warps zeroes, and after the chunk
        // flushes, the tile cells gt, gt + kGR * 32, ... of every tile; a
        // barrier of the gridding warps alone (id 5) separates the zeroing
        // from the chunk's first additions and the last additions from the
        // flush, so the other roles run on into the next chunk meanwhile.
        const int gt = tid - kGRBase * 32;
        if (p.do_grid)
          for (int i = gt; i < RR; i += kGR * 32)
#pragma unroll
            for (int t = 0; t < kTiles; ++t) {
              GT z;
              z.x = 0;
              z.y = 0;
              gtile[t * RR + i] = z;
            }
        ptx::named_sync(5, kGR * 32);
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
        ptx::named_sync(5, kGR * 32);
        if (p.do_grid && !*abort) {
          const int jnx = HPGB_JOB(BATCH, p, job, nx);
          const int jny = HPGB_JOB(BATCH, p, job, ny);
          double2* plane = HPGB_JOB(BATCH, p, job, grid) +
                           size_t(cube * p.nrow + row) * jny * jnx;
          for (int i = gt; i < RR; i += kGR * 32) {
            const int gx = x0 + i % R, gy = y0 + i / R;
            if (gx < jnx && gy < jny) {
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
                double2* dst = plane + size_t(gy) * jnx + gx;
                atomicAdd(&dst->x, vx);
                atomicAdd(&dst->y, vy);
              }
            }
          }
        }
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
    if (*model_loads > 0)
      ok &= ptx::mbar_drain(model_bar, uint32_t(*model_loads - 1) & 1, abort);
  }
  if (!ok) atomicOr(p.status, kStatusWaitTimeout);
  __syncwarp();
  ptx::cluster_sync();  // no CTA leaves while peers may still address it
}

// ---------------------------------------------------------------------------
// host side shared by grid_tiled.cu and grid_batch.cu

// the shape of a batched launch: the largest CF plane and support over its
// gridders, and per gridder its grid (width, height, cubes), widest CF
// (taps) and batch size, from which the plan counts the launch's tiles
struct BatchShape {
  struct Job {
    long long nx, ny, ncube, taps, nvis;
  };
  int max_plane_bytes = 0;
  int max_taps = 0;
  std::vector<Job> jobs;
};

struct Plan {
  bool ok = false;
  std::string why;
  int R = 0, T = 0, ring_bytes = 0, K = 0;
  TiledParams p{};
  int smem = 0;
};

// the tiled kernel's plan for a batch of g (or, with `batch`, for a launch
// over many gridders that share g's Mueller tables and polarizations)
Plan make_plan(const hpgb_gridder* g, unsigned flags, bool mixed, size_t nvis,
               const BatchShape* batch);

// the 3-D tensor map of g's model (FP32 copy made on st when mixed) with a
// box of R x R cells of one grid row
Status encode_model_map(hpgb_gridder* g, bool mixed, int R, CUtensorMap* map,
                        cudaStream_t st);

// Launches the tiled kernel on g's stream: one cluster of nrow CTAs per
// tile pass at a time, as many clusters as fit the device at once.  BATCH:
// p holds the job table of a launch over many gridders (g is the first).
template <int N, bool MIXED, bool BATCH>
Status launch_tiled_kernel(hpgb_gridder* g, const TiledParams& p, int smem,
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
  auto kern = dense ? (comp ? tiled_kernel<N, MIXED, true, MIXED, BATCH>
                            : tiled_kernel<N, MIXED, true, false, BATCH>)
                   : (comp ? tiled_kernel<N, MIXED, false, MIXED, BATCH>
                           : tiled_kernel<N, MIXED, false, false, BATCH>);
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

}  // namespace tiled
}  // namespace hpgb
