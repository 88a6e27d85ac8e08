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
//   2. cub radix sort     stable sort of (key, visibility index); the key's
//                         low bits are the footprint's size class
//   3. scans + chunks     tile starts; work chunks of <= kChunkVis visibilities
//   4. tile_desc_kernel   one 256-byte descriptor per visibility
//                         (tile-relative footprint origin, phasor, phase
//                         screen, degridding normaliser and grid-row
//                         weights from the per-slice CF sums, gridding
//                         values) + the address of its CF slice, a tile's
//                         visibilities interleaved large/small
//                         (tile_order_source: measured 2.8% faster in the
//                         mixed form, 1.5% in the FP64 form, than input
//                         order; sorted by size alone, 3% slower)
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
//                         - at the end of a chunk the gridding warps add
//                           the tile (the sum of the groups' tiles, with
//                           their low parts in the compensated form) to the
//                           FP64 grid and zero it, between barriers of
//                           their own, while the other roles run on into
//                           the next chunk: two scalar FP64 reductions per
//                           cell (an atomicAdd whose result is unused
//                           compiles to a reduction; PTX has no vector FP64
//                           reduction); the exchange warps add the row's
//                           weight sum to the weights.  The
//                           reductions take under 3% of the L2's reduction
//                           throughput (lts__t_sectors_srcunit_tex_op_red in
//                           the kernel's ncu capture): one per tile cell per
//                           pass, never per visibility.
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
#include "tiled_kernel.cuh"

namespace hpgb {

namespace {

using namespace tiled;

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
  unsigned key = unsigned(tg.ntiles) << tg.sbits;
  if (vc.in_grid) {
    const unsigned tile =
        unsigned((vc.grid_cube * tg.nty + vc.grid_coord[1] / tg.T) * tg.ntx +
                 vc.grid_coord[0] / tg.T);
    // footprint size class in the key's low bits (cells / 128, capped)
    const unsigned top = (1u << tg.sbits) - 1u;
    const unsigned sc = min(top, unsigned(vc.taps[0] * vc.taps[1]) >> 7);
    key = (tile << tg.sbits) | sc;
    atomicAdd(&counts[tile], 1u);
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
                                 SliceRef* srefs, const unsigned* tstart,
                                 const unsigned* tcount) {
  const size_t pidx = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (pidx >= n) return;
  const unsigned key = keys[pidx] >> tg.sbits;  // the tile
  if (key >= unsigned(tg.ntiles)) return;
  // the tile's visibilities are sorted by footprint size; descriptor
  // position pidx takes the one tile_order_source picks
  const unsigned t0 = tstart[key];
  const unsigned r = unsigned(pidx) - t0;
  const unsigned i = order[t0 + tile_order_source(r, tcount[key], tg.order)];
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
// host side


}  // namespace

namespace tiled {

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

Status encode_model_map(hpgb_gridder* g, bool mixed, int R, CUtensorMap* map,
                        cudaStream_t st) {
  std::memset(map, 0, sizeof(*map));
  const int nx = int(g->grid_size[0]), ny = int(g->grid_size[1]);
  const int nrow = int(g->grid_size[2]), ncube = int(g->grid_size[3]);
  const void* base = g->model.ptr;
  size_t esize = 8;
  CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  if (mixed) {
    const size_t ne = g->grid_elems();
    if (!g->model32_valid) {
      HPGB_TRY(g->model32.reserve(std::max<size_t>(ne, 1) * sizeof(float2)));
      model_to_f32_kernel<<<148 * 8, 256, 0, st>>>(
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
  cuuint64_t dims[3] = {cuuint64_t(2 * nx), cuuint64_t(ny),
                        cuuint64_t(nrow * ncube)};
  cuuint64_t strides[2] = {cuuint64_t(2 * nx) * esize,
                           cuuint64_t(2 * nx) * ny * esize};
  cuuint32_t box[3] = {cuuint32_t(2 * R), cuuint32_t(R), 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, dt, 3, const_cast<void*>(base), dims, strides, box,
                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return Status::err(HPGB_ERROR_OTHER,
                       "cuTensorMapEncodeTiled failed: " + std::to_string(int(r)));
  return Status::ok();
}

Plan make_plan(const hpgb_gridder* g, unsigned flags, bool mixed,
               size_t nvis, const BatchShape* batch) {
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
  // a batched launch sizes its ring and tiles for every gridder's CF
  if (batch) max_plane_bytes = std::max(max_plane_bytes, batch->max_plane_bytes);
  const int part = align_up(std::max(max_planes * max_plane_bytes, 16), 128);
  const int esize = mixed ? 8 : 16;
  const bool do_degrid = flags & HPGB_DO_DEGRID;
  const bool do_grid = flags & HPGB_DO_GRID;
  const int em = (do_degrid && g->has_model) ? esize : 0;
  const int eg = do_grid ? esize : 0;
  const int budget = 227 * 1024;
  const int taps = std::max(std::max(cf.max_taps_x, cf.max_taps_y),
                            batch ? batch->max_taps : 0);
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
  // the ring depth that few visibilities per tile still keep when it fits:
  // two parts are for CF slices too wide for three (measured on a 2048^2
  // grid with dense Mueller: at 50k visibilities 2.21 -> 1.58 ms mixed,
  // 2.76 -> 1.95 ms FP64; at 200k 7.51 -> 5.73 ms in the compensated form,
  // whose four tiles leave the least room)
  constexpr int kFewVisParts = 3;
  constexpr int kSideTrim = 6;
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
    // automatic plans at four parts or fewer: a side up to kSideTrim cells
    // below the largest, whose freed bytes deepen the ring (the autotuner
    // picks 4 to 12 cells below there on the 2048^2 full-polarization
    // workload; measured with the automatic plan: 1M visibilities mixed
    // 22.95 -> 19.22 ms, 200k FP64 6.71 -> 6.13 ms, the batched benchmark
    // 71.7 -> 74.2 Mvis/s), while tile strides stay >= 8
    if (!fixed && tp.tile_side <= 0 && m <= 4)
      R -= std::max(0, std::min(kSideTrim, (R - taps + 1 - 8) & ~1));
    if (!fixed && m > std::max(m_lo, kFewVisParts)) {
      // tiles of the batch (of every gridder of a batched launch, each
      // with the largest tile its own CF allows in the region)
      auto tiles = [R](size_t nx, size_t ny, size_t ncube, int t) {
        const size_t T = size_t(R - t + 1);
        return ((nx + T - 1) / T) * ((ny + T - 1) / T) * ncube;
      };
      size_t ntiles = 0;
      if (batch) {
        for (const BatchShape::Job& j : batch->jobs)
          if (j.nvis > 0) ntiles += tiles(j.nx, j.ny, j.ncube, int(j.taps));
      } else {
        ntiles = tiles(g->grid_size[0], g->grid_size[1], g->grid_size[3], taps);
      }
      if (nvis < kMinVisPerTile * ntiles) continue;
    }
    // the ring takes every whole KB the tiles leave (the ring's bytes, not
    // its part count, set how many visibilities are in flight; a tile side
    // below the largest thus deepens the ring)
    const int spare = left - per_cell * R * R;
    pl.ring_bytes = rb + (spare >= 1024 ? spare / 1024 * 1024 : 0);
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

}  // namespace tiled

namespace {

template <int N, bool MIXED>
Status launch_tiled(hpgb_gridder* g, const TiledParams& p, int smem,
                    const CUtensorMap& map) {
  return launch_tiled_kernel<N, MIXED, false>(g, p, smem, map);
}

template <int N>
Status prepare_tiles_n(hpgb_gridder* g, void* d_vis, size_t n, int T, int ntx,
                       int nty, int K, TilePrep* out, cudaStream_t st,
                       int order) {
  VisBuffers& vb = g->vb;
  const GridGeom geom = g->geom();
  const CFGroup* groups = g->cf.desc.as<const CFGroup>();
  TileGeom tg;
  tg.T = T;
  tg.ntx = ntx;
  tg.nty = nty;
  tg.ntiles = tg.ntx * tg.nty * int(g->grid_size[3]);
  // five bits of footprint size class below the tile while keys fit 32 bits
  tg.sbits = (unsigned(tg.ntiles) + 1u) <= (1u << 27) ? 5 : 0;
  tg.order = tg.sbits ? order : kOrderBatch;
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
  while ((1ll << end_bit) <= ((long long)ntiles << tg.sbits)) ++end_bit;
  size_t sort_bytes = 0, scan_bytes = 0;
  cub::DoubleBuffer<unsigned> kbuf(vb.keys.as<unsigned>(), vb.keys_alt.as<unsigned>());
  cub::DoubleBuffer<unsigned> vbuf(vb.order.as<unsigned>(), vb.order_alt.as<unsigned>());
  HPGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, kbuf, vbuf,
                                                int(n), 0, end_bit, st));
  HPGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts,
                                              tstart, ntiles, st));
  HPGB_TRY(vb.sort_tmp.reserve(std::max(sort_bytes, scan_bytes) + 16));

  HPGB_CUDA_TRY(cudaMemsetAsync(counts, 0, size_t(ntiles + 1) * 4, st));
  const unsigned blocks = unsigned((n + 255) / 256);
  tile_keys_kernel<N><<<blocks, 256, 0, st>>>(
      static_cast<const VisData<N>*>(d_vis), n, geom, groups, tg,
      vb.keys.as<unsigned>(), vb.order.as<unsigned>(), counts);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  size_t tmp_bytes = vb.sort_tmp.bytes;
  HPGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(vb.sort_tmp.ptr, tmp_bytes, kbuf,
                                                vbuf, int(n), 0, end_bit,
                                                st));
  tmp_bytes = vb.sort_tmp.bytes;
  HPGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(vb.sort_tmp.ptr, tmp_bytes, counts,
                                              tstart, ntiles, st));
  const unsigned tblocks = unsigned((ntiles + 255) / 256);
  chunk_count_kernel<<<tblocks, 256, 0, st>>>(counts, ntiles, K, nch);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  tmp_bytes = vb.sort_tmp.bytes;
  HPGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(vb.sort_tmp.ptr, tmp_bytes, nch,
                                              cstart, ntiles, st));
  chunk_write_kernel<<<tblocks, 256, 0, st>>>(
      counts, tstart, nch, cstart, ntiles, K, vb.items.as<Chunk>(), num_chunks);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  tile_desc_kernel<N><<<blocks, 256, 0, st>>>(
      static_cast<const VisData<N>*>(d_vis), vbuf.Current(), kbuf.Current(), n,
      geom, groups, tg, g->cf.data.as<const float2>(), descs, srefs, tstart,
      counts);
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
                              plan.K, &prep, g->stream, kOrderPairs));
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
  if (p.do_degrid && p.has_model)
    HPGB_TRY(encode_model_map(g, mixed, p.R, &map, g->stream));
  if (mixed) return launch_tiled<N, true>(g, p, plan.smem, map);
  return launch_tiled<N, false>(g, p, plan.smem, map);
}

}  // namespace

Status prepare_tiles(hpgb_gridder* g, void* d_vis, size_t n, int T, int ntx,
                     int nty, int K, TilePrep* out, cudaStream_t st,
                     int order) {
  if (!st) st = g->stream;
  switch (g->npol) {
    case 1: return prepare_tiles_n<1>(g, d_vis, n, T, ntx, nty, K, out, st, order);
    case 2: return prepare_tiles_n<2>(g, d_vis, n, T, ntx, nty, K, out, st, order);
    case 3: return prepare_tiles_n<3>(g, d_vis, n, T, ntx, nty, K, out, st, order);
    case 4: return prepare_tiles_n<4>(g, d_vis, n, T, ntx, nty, K, out, st, order);
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
}

bool tiled_plan_side(const hpgb_gridder* g, unsigned flags, size_t n,
                     int* side) {
  const Plan plan =
      make_plan(g, flags, g->precision == HPGB_PRECISION_MIXED, n, nullptr);
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
  const Plan plan = make_plan(g, flags, mixed, n, nullptr);
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

