// autotune.cu -- choice of the tiled kernel's plan by measurement.
//
// The tiled kernel's two free parameters trade against each other: a
// deeper CF ring keeps more visibilities in flight but leaves less shared
// memory for the uv tiles (more tiles, more halo and flush traffic), and a
// longer tile pass amortises the tile flush but delays it.  Which balance
// wins depends on the CF supports, the arithmetic form and the number and
// spread of the visibilities, so the autotuner times the candidates on the
// caller's own batch and keeps the fastest for the gridder.  The grid and
// weights are restored after every trial: tuning leaves the gridder's data
// as it found it.

#include <limits>
#include <vector>

#include "gridder.cuh"

namespace hpgb {

namespace {

struct Trial {
  int ring_parts, chunk_vis;
};

// one timed run of the tiled kernel on the staged batch; ms < 0 when the
// plan does not fit
Status run_trial(hpgb_gridder* g, const void* src, size_t bytes, bool on_device,
                 size_t n, unsigned flags, const Trial& t, cudaEvent_t e0,
                 cudaEvent_t e1, const DevBuf& saved_grid,
                 const DevBuf& saved_weights, float* ms) {
  g->tiled_ring_parts = t.ring_parts;
  g->tiled_chunk_vis = t.chunk_vis;
  HPGB_CUDA_TRY(cudaMemcpyAsync(
      g->vb.vis.ptr, src, bytes,
      on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
      g->stream));
  HPGB_CUDA_TRY(cudaEventRecord(e0, g->stream));
  bool used = false;
  HPGB_TRY(grid_tiled(g, g->vb.vis.ptr, n, flags, &used));
  HPGB_CUDA_TRY(cudaEventRecord(e1, g->stream));
  HPGB_CUDA_TRY(cudaEventSynchronize(e1));
  *ms = -1.f;
  if (used) HPGB_CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
  HPGB_CUDA_TRY(cudaMemcpyAsync(g->grid.ptr, saved_grid.ptr, saved_grid.bytes,
                                cudaMemcpyDeviceToDevice, g->stream));
  HPGB_CUDA_TRY(cudaMemcpyAsync(g->weights.ptr, saved_weights.ptr,
                                saved_weights.bytes, cudaMemcpyDeviceToDevice,
                                g->stream));
  HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return Status::ok();
}

}  // namespace

Status autotune_tiled(hpgb_gridder* g, const void* vis, size_t n,
                      unsigned flags, bool on_device, int* best_ring,
                      int* best_chunk) {
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
  cudaEvent_t e0, e1;
  HPGB_CUDA_TRY(cudaEventCreate(&e0));
  HPGB_CUDA_TRY(cudaEventCreate(&e1));
  const int ring0 = g->tiled_ring_parts, chunk0 = g->tiled_chunk_vis;
  Status st = Status::ok();
  Trial best{ring0, chunk0};
  float best_ms = std::numeric_limits<float>::max();
  auto trial = [&](const Trial& t) -> Status {
    float ms = -1.f;
    HPGB_TRY(run_trial(g, vis, bytes, on_device, n, flags, t, e0, e1,
                       saved_grid, saved_weights, &ms));
    if (ms >= 0.f && ms < best_ms) {
      best_ms = ms;
      best = t;
    }
    return Status::ok();
  };
  // warm-up (one-time set-up costs) with the plan's own choice, then the
  // ring depths, then tile-pass lengths around the best depth
  float ms = -1.f;
  st = run_trial(g, vis, bytes, on_device, n, flags, Trial{0, 0}, e0, e1,
                 saved_grid, saved_weights, &ms);
  if (st && ms < 0.f)
    st = Status::err(HPGB_ERROR_OTHER,
                     "the tiled kernel cannot take this CF or grid");
  for (int ring = 4; st && ring <= 8; ++ring) st = trial(Trial{ring, 0});
  if (st && best_ms < std::numeric_limits<float>::max()) {
    // the mixed form's FP32 tile holds at most 512 visibilities between
    // flushes: its rounding error grows with the number summed
    const bool mixed = g->precision == HPGB_PRECISION_MIXED;
    const std::vector<int> chunks =
        mixed ? std::vector<int>{128, 512} : std::vector<int>{1024, 4096, 8192};
    for (int chunk : chunks)
      if (st) st = trial(Trial{best.ring_parts, chunk});
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!st || best_ms == std::numeric_limits<float>::max()) {
    g->tiled_ring_parts = ring0;
    g->tiled_chunk_vis = chunk0;
    return st ? Status::err(HPGB_ERROR_OTHER, "no tiled plan fits") : st;
  }
  g->tiled_ring_parts = best.ring_parts;
  g->tiled_chunk_vis = best.chunk_vis;
  *best_ring = best.ring_parts;
  *best_chunk = best.chunk_vis;
  return Status::ok();
}

}  // namespace hpgb
