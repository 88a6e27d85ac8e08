// dispatch.cu -- choice of gridding kernel for one batch.

#include "gridder.cuh"

namespace hpgb {

Status grid_batch(hpgb_gridder* g, const void* d_vis, size_t n,
                  unsigned flags) {
  return grid_direct(g, d_vis, n, flags);
}

}  // namespace hpgb
