// tiles.cuh -- the tile sort of a visibility batch, shared by the tiled
// gridding kernel (grid_tiled.cu) and the tiled linear operators
// (adjoint_tiled.cu).
//
// A batch is sorted by the uv tile (T x T cells of footprint origins, per
// grid cube) that holds each visibility's footprint origin, and within a
// tile by footprint size, then interleaved large/small (tile_order_source);
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
  // the key has no room, or without interleaving)
  int sbits;
  int interleave;  // order a tile's visibilities by tile_order_source
};

// Order of a tile's visibilities: sorted by footprint size, then taken as
// large, small, small, large, large, small, ... (position r of the tile's n
// takes sorted position n - 1 - r/2 when large, r/2 when small).  Each
// consecutive pair holds one large and one small footprint, so the CF ring
// keeps a mix of large and small parts in flight, and each of two groups
// that take alternate visibilities alternates between large and small.
__host__ __device__ inline unsigned tile_order_source(unsigned r, unsigned n) {
  const unsigned k = r >> 1;
  const bool large = ((k & 1u) == 0u) == ((r & 1u) == 0u);
  return large ? n - 1u - k : k;
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
// interleave: a tile's visibilities in tile_order_source's large/small
// order (the tiled gridding kernel, whose pipeline runs best on a mix of
// footprint sizes); otherwise in batch order (the tiled linear operators,
// whose warps take every 16th visibility of a pass: a periodic size pattern
// would give some warps only large footprints).
Status prepare_tiles(hpgb_gridder* g, void* d_vis, size_t n, int T, int ntx,
                     int nty, int K, TilePrep* out, cudaStream_t st = nullptr,
                     bool interleave = true);

}  // namespace hpgb
