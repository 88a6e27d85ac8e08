// autotune.cu -- choice of the tiled kernel's plan by measurement.
//
// The tiled kernel's free parameters trade against each other: a deeper CF
// ring keeps more visibilities in flight but leaves less shared memory for
// the uv tiles (more tiles, more halo and flush traffic); a smaller tile
// side than the largest that fits shortens the model-tile loads and flushes
// of a pass but multiplies the passes; a longer tile pass amortises the tile
// flush but delays it.  Which balance wins depends on the CF supports, the
// arithmetic form and the number and spread of the visibilities, so the
// autotuner times the candidates on the caller's own batch and keeps the
// fastest for the gridder:
//   1. CF ring depths 2..8 (largest per-row parts), tile side and pass
//      length automatic;
//   2. at the best depth, tile sides 8 and 16 cells below the largest;
//   3. at the best depth and side, pass lengths around the default.
// The mixed form's compensation setting is kept as the caller set it (it is
// a precision choice, not a speed one).  Every candidate runs three times and
// is ranked by its median time; a candidate whose launch reported a device
// wait timeout counts as not fitting.  Results are cached per workload key
// (grid shape, polarizations, Mueller tables, CF group shapes, precision and
// compensation, flags, model present, log2 of the batch size): a later call
// with the same key applies the cached plan without timing anything.  The
// grid and weights are restored on every exit path: tuning leaves the
// gridder's data as it found it.

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <mutex>
#include <vector>

#include "gridder.cuh"

namespace hpgb {

namespace {

struct Trial {
  int ring_parts, chunk_vis, tile_side;
};

std::vector<long long> tune_key(const hpgb_gridder* g, unsigned flags,
                                size_t n) {
  std::vector<long long> k;
  for (unsigned d : g->grid_size) k.push_back(d);
  k.push_back(g->npol);
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      k.push_back(g->mt.m[r][c]);
      k.push_back(g->mt.c[r][c]);
    }
  k.push_back(g->precision);
  k.push_back(g->tplan.compensated);
  k.push_back(flags & (HPGB_DO_DEGRID | HPGB_DO_GRID | HPGB_UPDATE_GRID_WEIGHTS));
  k.push_back(g->has_model);
  k.push_back(n > 0 ? (long long)std::floor(std::log2(double(n))) : -1);
  k.push_back(g->cf.os);
  for (const CFGroup& G : g->cf.groups) {
    k.push_back(G.taps_x);
    k.push_back(G.taps_y);
    k.push_back(G.nmueller);
    k.push_back(G.plane_stride);
  }
  return k;
}

std::mutex g_cache_mtx;
std::map<std::vector<long long>, Trial> g_cache;

// copies the saved grid and weights back when it goes out of scope
struct RestoreGrid {
  hpgb_gridder* g;
  const DevBuf& grid;
  const DevBuf& weights;
  ~RestoreGrid() {
    cudaMemcpyAsync(g->grid.ptr, grid.ptr, grid.bytes, cudaMemcpyDeviceToDevice,
                    g->stream);
    cudaMemcpyAsync(g->weights.ptr, weights.ptr, weights.bytes,
                    cudaMemcpyDeviceToDevice, g->stream);
    cudaStreamSynchronize(g->stream);
  }
};

// reads and clears the wait-timeout bit of the gridder's status word (the
// bad-index bit stays for the caller's next fence)
Status take_timeout_bit(hpgb_gridder* g, bool* timed_out) {
  unsigned h = 0;
  HPGB_CUDA_TRY(cudaMemcpy(&h, g->vb.counters.ptr, sizeof(unsigned),
                           cudaMemcpyDeviceToHost));
  *timed_out = (h & kStatusWaitTimeout) != 0;
  if (*timed_out) {
    h &= ~unsigned(kStatusWaitTimeout);
    HPGB_CUDA_TRY(cudaMemcpy(g->vb.counters.ptr, &h, sizeof(unsigned),
                             cudaMemcpyHostToDevice));
  }
  return Status::ok();
}

}  // namespace

Status autotune_tiled(hpgb_gridder* g, const void* vis, size_t n,
                      unsigned flags, bool on_device, int* best_ring,
                      int* best_chunk) {
  const std::vector<long long> key = tune_key(g, flags, n);
  {
    std::lock_guard<std::mutex> lk(g_cache_mtx);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) {
      g->tplan.ring_parts = it->second.ring_parts;
      g->tplan.chunk_vis = it->second.chunk_vis;
      g->tplan.tile_side = it->second.tile_side;
      *best_ring = it->second.ring_parts;
      *best_chunk = it->second.chunk_vis;
      return Status::ok();
    }
  }
  const size_t bytes = n * visdata_size(g->npol);
  HPGB_TRY(g->vb.vis.reserve(std::max(g->max_batch, n) * visdata_size(g->npol)));
  DevBuf saved_grid, saved_weights;
  HPGB_TRY(saved_grid.reserve(g->grid_elems() * sizeof(double2)));
  HPGB_TRY(saved_weights.reserve(g->weight_elems() * sizeof(double)));
  saved_grid.bytes = g->grid_elems() * sizeof(double2);
  saved_weights.bytes = g->weight_elems() * sizeof(double);
  HPGB_CUDA_TRY(cudaMemcpyAsync(saved_grid.ptr, g->grid.ptr, saved_grid.bytes,
                                cudaMemcpyDeviceToDevice, g->stream));
  HPGB_CUDA_TRY(cudaMemcpyAsync(saved_weights.ptr, g->weights.ptr,
                                saved_weights.bytes, cudaMemcpyDeviceToDevice,
                                g->stream));
  RestoreGrid restore{g, saved_grid, saved_weights};
  const hpgb_tiled_plan plan0 = g->tplan;

  cudaEvent_t e0 = nullptr, e1 = nullptr;
  HPGB_CUDA_TRY(cudaEventCreate(&e0));
  const cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return Status::err(HPGB_ERROR_OTHER, cudaGetErrorString(ce));
  }
  struct Events {
    cudaEvent_t a, b;
    ~Events() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } events{e0, e1};

  // one run of candidate t: the batch is copied afresh (a degrid+grid run
  // writes residuals into the records), the tiled kernel's work timed;
  // ms < 0 when the plan does not fit or the kernel timed out
  auto run = [&](const Trial& t, float* ms) -> Status {
    g->tplan.ring_parts = t.ring_parts;
    g->tplan.chunk_vis = t.chunk_vis;
    g->tplan.tile_side = t.tile_side;
    HPGB_CUDA_TRY(cudaMemcpyAsync(
        g->vb.vis.ptr, vis, bytes,
        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
        g->stream));
    HPGB_CUDA_TRY(cudaEventRecord(e0, g->stream));
    bool used = false;
    HPGB_TRY(grid_tiled(g, g->vb.vis.ptr, n, flags, &used));
    HPGB_CUDA_TRY(cudaEventRecord(e1, g->stream));
    HPGB_CUDA_TRY(cudaEventSynchronize(e1));
    *ms = -1.f;
    bool timed_out = false;
    HPGB_TRY(take_timeout_bit(g, &timed_out));
    if (used && !timed_out) HPGB_CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
    return Status::ok();
  };
  Trial best{0, 0, 0};
  float best_ms = std::numeric_limits<float>::max();
  auto trial = [&](const Trial& t) -> Status {
    float m[3];
    for (float& x : m) {
      HPGB_TRY(run(t, &x));
      if (x < 0.f) return Status::ok();  // does not fit
    }
    std::sort(m, m + 3);
    if (m[1] < best_ms) {
      best_ms = m[1];
      best = t;
    }
    return Status::ok();
  };
  Status st = Status::ok();
  auto finish = [&](Status s) -> Status {
    if (!s || best_ms == std::numeric_limits<float>::max()) {
      g->tplan = plan0;
      return s ? Status::err(HPGB_ERROR_OTHER, "no tiled plan fits") : s;
    }
    g->tplan.ring_parts = best.ring_parts;
    g->tplan.chunk_vis = best.chunk_vis;
    g->tplan.tile_side = best.tile_side;
    *best_ring = best.ring_parts;
    *best_chunk = best.chunk_vis;
    std::lock_guard<std::mutex> lk(g_cache_mtx);
    g_cache[key] = best;
    return Status::ok();
  };
  // warm-up (one-time set-up costs) with the automatic plan
  float ms = -1.f;
  st = run(Trial{0, 0, 0}, &ms);
  if (!st) return finish(st);
  if (ms < 0.f)
    return finish(Status::err(HPGB_ERROR_OTHER,
                              "the tiled kernel cannot take this CF or grid"));
  // 1. ring depth
  for (int ring = 2; st && ring <= 8; ++ring) st = trial(Trial{ring, 0, 0});
  if (!st || best_ms == std::numeric_limits<float>::max()) return finish(st);
  // 2. tile sides below the largest that fits at that depth and one part
  // shallower: a smaller side gives the bytes it frees to the ring, so
  // these trials fill in ring sizes between whole parts (more visibilities
  // in flight against more, shorter tile passes)
  {
    const int taps = std::max(g->cf.max_taps_x, g->cf.max_taps_y);
    const int deepest = best.ring_parts;
    for (int ring = deepest; st && ring >= std::max(2, deepest - 1); --ring) {
      g->tplan.ring_parts = ring;
      g->tplan.tile_side = 0;
      int side = 0;
      if (!tiled_plan_side(g, flags, n, &side) || side <= 0) continue;
      for (int d : {0, 4, 8, 12, 16})
        if (st && side - d - taps + 1 >= 4)
          st = trial(Trial{ring, 0, side - d});
    }
  }
  // 3. tile-pass length
  const bool mixed = g->precision == HPGB_PRECISION_MIXED;
  const bool comp = g->tplan.compensated == HPGB_COMPENSATED_ON;
  const std::vector<int> chunks =
      !mixed ? std::vector<int>{1024, 4096, 8192}
      : comp ? std::vector<int>{512, 1024, 4096, 8192}
             // plain FP32 tiles: the tile's rounding error grows with the
             // visibilities summed between flushes, so passes stay short
             : std::vector<int>{128, 512};
  const Trial base = best;
  for (int chunk : chunks)
    if (st) st = trial(Trial{base.ring_parts, chunk, base.tile_side});
  return finish(st);
}

}  // namespace hpgb
