// gridder.cuh -- host-side state of one hpgb_gridder (one hpg::GridderState).
#pragma once

#include <cufft.h>

#include <array>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include "common.cuh"

namespace hpgb {

// device buffer owned by the gridder
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  Status reserve(size_t n);   // grows, contents not preserved
  void release();
  template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// the CF region: slices of every group plus their sums
struct CFRegion {
  unsigned os = 0;
  std::vector<std::array<unsigned, 4>> extents;  // per group, as given
  std::vector<CFGroup> groups;                   // host copy of descriptors
  DevBuf data;      // all slices of all groups
  DevBuf wsum;      // all slice sums
  DevBuf desc;      // device copy of groups
  int max_taps_x = 0, max_taps_y = 0, max_mueller = 0;
  bool set = false;
};

// scratch and staging for one visibility batch
struct VisBuffers {
  DevBuf vis;       // VisData<N> records (device copy / returned values)
  DevBuf gvis;      // float2 [n][N] visibility values scaled for gridding
  // tiled path: sorted work description
  DevBuf keys, keys_alt, order, order_alt, sort_tmp, buckets, items, counters;
  DevBuf prep;      // per-visibility prepared records (sorted order)
  // batched launches led by this gridder: job table and combined pass list
  DevBuf batch_jobs, batch_chunks;
  // host batches outside a stream capture: two staging buffers, used in
  // turn, so that one call's host->device copy overlaps the previous call's
  // work
  DevBuf staged[2];
};

struct hpgb_gridder_impl;

}  // namespace hpgb

// an instantiated CUDA graph of work captured on a gridder's stream
struct hpgb_graph {
  cudaGraphExec_t exec = nullptr;
  int device = 0;
  uint64_t launches = 0;  // kernels in the graph
};

struct hpgb_gridder {
  int device = 0;
  unsigned max_added_tasks = 0;
  size_t max_batch = 0;
  unsigned grid_size[4] = {0, 0, 0, 0};
  double grid_scale[2] = {0, 0};
  unsigned npol = 0;
  hpgb::MuellerTables mt;
  int precision = HPGB_PRECISION_FP64;

  cudaStream_t stream = nullptr;
  // copies of host batches into vb.staged[staged_next]: on copy_stream,
  // after the buffer's previous batch is done with it (staged_free[b],
  // recorded on `stream`); `stream` waits for the copy (staged_copied)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t staged_copied = nullptr;
  cudaEvent_t staged_free[2] = {nullptr, nullptr};
  int staged_next = 0;

  hpgb::DevBuf grid;      // double2 [cube][mrow][y][x]
  hpgb::DevBuf weights;   // double  [cube][mrow]
  hpgb::DevBuf model;     // double2, empty when no model is set
  bool has_model = false;
  hpgb::DevBuf model32;   // float2 copy of the model for the mixed form
  bool model32_valid = false;
  int kernel_kind = HPGB_KERNEL_AUTO;
  int last_kernel = HPGB_KERNEL_AUTO;  // kernel of the last non-empty batch
  // tiled-kernel plan overrides (fields 0: chosen by the plan)
  hpgb_tiled_plan tplan = {0, 0, 0, 0};
  // bound of every device-side wait of the tiled kernel, and its test hook
  // (a visibility whose copies CTA 0 never issues; -1: none)
  unsigned long long wait_limit_ns = 500000000ull;
  long long withhold_vis = -1;

  hpgb::CFRegion cf;
  hpgb::VisBuffers vb;

  // returned-visibility copy pending until the next fence
  void* pending_dst = nullptr;
  size_t pending_bytes = 0;
  bool pending_on_device = false;

  // cuFFT plans by (nx, ny, batch)
  std::map<std::tuple<int, int, int>, cufftHandle> fft_plans;

  mutable std::mutex mtx;
  uint64_t launches = 0;  // kernels launched by this gridder
  uint64_t capture_launches0 = 0;  // launches when the stream capture began

  // event pairs around each launch of the tiled gridding kernel, recorded
  // while profiling is on (benchmark instrumentation)
  bool profile = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;

  size_t grid_elems() const {
    return size_t(grid_size[0]) * grid_size[1] * grid_size[2] * grid_size[3];
  }
  size_t weight_elems() const { return size_t(grid_size[2]) * grid_size[3]; }
  hpgb::GridGeom geom() const;
};

namespace hpgb {

// cf_layout.cu
Status cf_region_bytes(unsigned os, unsigned ngroups, const unsigned* extents,
                       size_t* data_bytes, size_t* wsum_bytes);
Status set_cf(hpgb_gridder* g, unsigned os, unsigned ngroups,
              const unsigned* extents, const void* const* values, int layout,
              bool on_device);
Status copy_cf(hpgb_gridder* dst, const hpgb_gridder* src);

// grid_tiled.cu: *used is false when the tiled kernel cannot take the batch
Status grid_tiled(hpgb_gridder* g, void* d_vis, size_t n, unsigned flags,
                  bool* used);

// grid_tiled.cu: the uv tile side of the plan the tiled kernel would take
// for the batch (false when no plan fits)
bool tiled_plan_side(const hpgb_gridder* g, unsigned flags, size_t n,
                     int* side);

// grid_batch.cu: one tiled launch over the device batches of many gridders
// (validated by the caller: same polarizations, rows, Mueller tables, form)
Status grid_batch_tiled(hpgb_gridder* const* gs, size_t njobs,
                        void* const* d_vis, const size_t* nvis, unsigned flags);

// autotune.cu: times tiled plans on the batch, keeps the fastest
Status autotune_tiled(hpgb_gridder* g, const void* vis, size_t n,
                      unsigned flags, bool on_device, int* best_ring,
                      int* best_chunk);

// grid_direct.cu
Status grid_direct(hpgb_gridder* g, const void* d_vis, size_t n,
                   unsigned flags);
// direct path with its per-visibility scratch in a fixed device array of
// kNoAllocMaxValues complex<float> values: allocates no device memory
constexpr size_t kNoAllocMaxValues = HPGB_NOALLOC_MAX_VALUES;
Status grid_direct_noalloc(hpgb_gridder* g, void* d_vis, size_t n,
                           unsigned flags);
Status debug_coords(hpgb_gridder* g, const void* d_vis, size_t n,
                    hpgb_vis_coords* d_out);

// adjoint.cu: FP64 linear operators on device arrays; op 0 = degridding D
// (model -> values), 1 = its adjoint (values -> model, accumulated),
// 2 = gridding G (values -> grid, accumulated), 3 = its adjoint (grid ->
// values)
Status linear_op(hpgb_gridder* g, const void* d_vis, size_t n, int op,
                 const void* in, void* out);
// adjoint_tiled.cu: the same on the tile sort of the batch; *used is false
// when the CF's tile region does not fit shared memory
Status linear_op_tiled(hpgb_gridder* g, const void* d_vis, size_t n, int op,
                       const void* in, void* out, bool* used);

// imaging.cu
Status normalize_by_weights(hpgb_gridder* g, double wfactor);
Status scale_grid(hpgb_gridder* g, double2* grid, double norm);
Status shift(hpgb_gridder* g, double2* grid, int direction);
Status fft(hpgb_gridder* g, DevBuf& grid, double norm, int sign, bool in_place);
Status to_layout(hpgb_gridder* g, const double2* src, double2* dst,
                 int layout, bool to_device_layout, const unsigned* ext);
Status weights_to_layout(hpgb_gridder* g, const double* src, double* dst,
                         int layout);
void release_fft_plans(hpgb_gridder* g);
Status image_tail(hpgb_gridder* g, double wfactor, double norm, int sign,
                  int direction);

}  // namespace hpgb
