// tiles.cuh -- the tile sort of a visibility batch, shared by the tiled
// gridding kernel (grid_tiled.cu) and the tiled linear operators
// (adjoint_tiled.cu).
//
// A batch is sorted by the uv tile (T x T cells of footprint origins, per
// grid cube) that holds each visibility's footprint origin, and within a
// tile by footprint size, then reordered (tile_order_source);
// each tile's visibilities are cut into passes ("chunks") of at most K;
// every visibility in that order gets a 256-byte descriptor of what the
// kernels need and the offset of its CF slice.
#pragma once

#include "gridder.cuh"

namespace hpgb {

struct alignas(16) TileDesc {
  int32_t index;         // visibility index in the batch
  int16_t cx, cy;        // footprint origin relative to the tile region
  uint8_t taps_x, taps_y, flags, pad0;
  int32_t pstride;       // CF plane stride (float2 elements)
  double2 phasor;        // cphase(phase)
  double phi0[2], dphi[2];
  float2 vals[4];
  float weights[4];
  double2 wfac[4];       // conj(phasor) / normaliser, per polarization
  double twgt[4];        // grid weight increment per grid row
  float2 gvis[4];        // values scaled for gridding (used without degrid)
  float inv_tx;          // 1 / taps_x, rounded to float
  int32_t pad1[3];
};
static_assert(sizeof(TileDesc) == 256, "TileDesc is one 256-byte bulk copy");

enum : uint8_t { kPosW = 1, kScreen = 2 };

struct SliceRef {
  long long off;  // float2 offset of the slice in the CF region
  int pstride;
  int ncell;
};

struct Chunk {
  int tile, start, count, pad;
};

struct TileGeom {
  int T, ntx, nty, ntiles;  // ntiles = ncube * nty * ntx (also the invalid key)
  // bits of the sort key below the tile: the footprint's size class (0 when
  // the key has no room, or in batch order)
  int sbits;
  int order;  // TileOrder: how a tile's visibilities are ordered
};

// How a tile's visibilities are ordered (each from the tile's visibilities
// sorted by footprint size, ascending; position r of the tile's n takes the
// sorted position tile_order_source gives):
//  - kOrderBatch: as in the batch;
//  - kOrderPairs (the tiled gridding kernel): large, small, small, large,
//    large, small, ... (n - 1 - r/2 when large, r/2 when small): each
//    consecutive pair holds one large and one small footprint, so the CF
//    ring keeps a mix of large and small parts in flight, and each of two
//    groups that take alternate visibilities alternates between them;
//  - kOrderSnake16 (the tiled linear operators, whose 16 warps take
//    visibilities r = warp, warp + 16, ... of a pass and meet at its end):
//    descending size, every other block of 16 reversed, so that each warp's
//    share of the footprints comes out nearly even.
enum TileOrder : int { kOrderBatch = 0, kOrderPairs = 1, kOrderSnake16 = 2 };

__host__ __device__ inline unsigned tile_order_source(unsigned r, unsigned n,
                                                      int order) {
  if (order == kOrderPairs) {
    const unsigned k = r >> 1;
    const bool large = ((k & 1u) == 0u) == ((r & 1u) == 0u);
    return large ? n - 1u - k : k;
  }
  if (order == kOrderSnake16) {
    const unsigned b = r >> 4, i = r & 15u;
    const unsigned m = n - (b << 4) < 16u ? n - (b << 4) : 16u;  // block size
    const unsigned d = (b << 4) + ((b & 1u) ? m - 1u - i : i);  // descending
    return n - 1u - d;
  }
  return r;
}

// where prepare_tiles leaves its results (the gridder's batch buffers)
struct TilePrep {
  const TileDesc* descs;   // [n] in sorted order (off-grid ones unused)
  const SliceRef* srefs;   // [n]
  const Chunk* chunks;     // [num_chunks] tile passes
  const unsigned* num_chunks;  // device word
  size_t max_chunks;       // bound on *num_chunks
};

// Sorts the batch d_vis (n VisData<npol> records in device memory) into
// tiles of T x T origins, ntx x nty tiles per grid cube, passes of at most
// K visibilities; all on stream st (the gridder's stream when null).
// order: TileOrder of a tile's visibilities (kOrderPairs for the tiled
// gridding kernel, whose pipeline runs best on a mix of footprint sizes;
// kOrderSnake16 for the tiled linear operators).
Status prepare_tiles(hpgb_gridder* g, void* d_vis, size_t n, int T, int ntx,
                     int nty, int K, TilePrep* out, cudaStream_t st = nullptr,
                     int order = kOrderPairs);

}  // namespace hpgb
