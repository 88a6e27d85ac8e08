// dispatch.cu -- choice of gridding kernel for one batch.
//
// The tiled kernel (grid_tiled.cu) takes every batch whose CF fits its
// shared-memory ring; the per-visibility kernels (grid_direct.cu) take the
// rest, or every batch when selected with hpgb_set_gridding_kernel.

#include "gridder.cuh"

namespace hpgb {

Status grid_batch(hpgb_gridder* g, const void* d_vis, size_t n,
                  unsigned flags) {
  if (g->kernel_kind != HPGB_KERNEL_DIRECT) {
    bool used = false;
    HPGB_TRY(grid_tiled(g, const_cast<void*>(d_vis), n, flags, &used));
    if (used) {
      if (n > 0) g->last_kernel = HPGB_KERNEL_TILED;
      return Status::ok();
    }
    if (g->kernel_kind == HPGB_KERNEL_TILED)
      return Status::err(HPGB_ERROR_OTHER,
                         "the tiled kernel cannot take this CF or grid");
  }
  if (n > 0) g->last_kernel = HPGB_KERNEL_DIRECT;
  return grid_direct(g, d_vis, n, flags);
}

}  // namespace hpgb
