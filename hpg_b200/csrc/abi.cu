// abi.cu -- the extern "C" entry points of libhpgb.so (include/hpgb.h).
//
// Each entry point replaces one virtual of hpg::runtime::State
// (src/hpg_runtime.hpp:80-207) as implemented by StateT<Device::Cuda>
// (src/hpg_runtime.hpp:721-1750); the header names the virtual for each.

#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "gridder.cuh"

namespace hpgb {

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

Status grid_batch(hpgb_gridder* g, const void* d_vis, size_t n,
                  unsigned flags);  // grid_tiled.cu

namespace {

int finish(const Status& s) {
  if (!s) set_last_error(s.msg);
  else set_last_error("");
  return s.code;
}

template <typename F>
int guarded(F&& f) {
  try {
    return finish(f());
  } catch (const std::bad_alloc&) {
    return finish(Status::err(HPGB_ERROR_OTHER, "host allocation failed"));
  } catch (const std::exception& e) {
    return finish(Status::err(HPGB_ERROR_OTHER, e.what()));
  } catch (...) {
    return finish(Status::err(HPGB_ERROR_OTHER, "unknown exception"));
  }
}

Status check_status_word(hpgb_gridder* g) {
  // status word lives in the first bytes of vb.counters
  unsigned h = 0;
  if (!g->vb.counters.ptr) return Status::ok();
  HPGB_CUDA_TRY(cudaMemcpy(&h, g->vb.counters.ptr, sizeof(unsigned),
                           cudaMemcpyDeviceToHost));
  if (h != 0) {
    HPGB_CUDA_TRY(cudaMemsetAsync(g->vb.counters.ptr, 0, sizeof(unsigned),
                                  g->stream));
    HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
  }
  if (h & kStatusWaitTimeout)
    return Status::err(HPGB_ERROR_OTHER,
                       "a device-side wait gave up after its iteration limit; "
                       "results of the last batch are incomplete");
  if (h & kStatusBadIndex)
    return Status::err(HPGB_ERROR_OUT_OF_BOUNDS_CF_INDEX,
                       "visibility cf_index or grid_cube out of bounds; "
                       "the visibility was skipped");
  return Status::ok();
}

Status fence_impl(const hpgb_gridder* cg) {
  hpgb_gridder* g = const_cast<hpgb_gridder*>(cg);
  HPGB_CUDA_TRY(cudaSetDevice(g->device));
  HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
  g->pending_dst = nullptr;
  g->pending_bytes = 0;
  return check_status_word(g);
}

Status alloc_grid(hpgb_gridder* g, bool zero_weights) {
  HPGB_TRY(g->grid.reserve(std::max<size_t>(g->grid_elems(), 1) * sizeof(double2)));
  HPGB_CUDA_TRY(cudaMemsetAsync(g->grid.ptr, 0, g->grid_elems() * sizeof(double2),
                                g->stream));
  if (zero_weights) {
    HPGB_TRY(g->weights.reserve(std::max<size_t>(g->weight_elems(), 1) * sizeof(double)));
    HPGB_CUDA_TRY(cudaMemsetAsync(g->weights.ptr, 0,
                                  g->weight_elems() * sizeof(double), g->stream));
  }
  return Status::ok();
}

// host-side index validation (the check the reference leaves commented out,
// src/hpg_runtime.hpp:1093-1100)
template <int N>
Status validate_host_indexes(const hpgb_gridder* g, const void* vis, size_t n) {
  const VisData<N>* v = static_cast<const VisData<N>*>(vis);
  const CFRegion& cf = g->cf;
  for (size_t i = 0; i < n; ++i) {
    const unsigned grp = v[i].cf_index[1], cube = v[i].cf_index[0];
    if (grp >= cf.extents.size() || cube >= cf.extents[grp][3] ||
        v[i].grid_cube >= g->grid_size[3])
      return Status::err(
          HPGB_ERROR_OUT_OF_BOUNDS_CF_INDEX,
          "visibility " + std::to_string(i) + ": cf_index (" +
              std::to_string(cube) + "," + std::to_string(grp) +
              ") or grid_cube " + std::to_string(v[i].grid_cube) +
              " is out of bounds");
  }
  return Status::ok();
}

Status validate_range(const hpgb_gridder* g, const void* vis, size_t n) {
  switch (g->npol) {
    case 1: return validate_host_indexes<1>(g, vis, n);
    case 2: return validate_host_indexes<2>(g, vis, n);
    case 3: return validate_host_indexes<3>(g, vis, n);
    case 4: return validate_host_indexes<4>(g, vis, n);
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
}

// large batches are checked by several host threads (the first error in
// batch order is reported, as a sequential check would)
Status validate_indexes(const hpgb_gridder* g, const void* vis, size_t n) {
  constexpr size_t kPerThread = size_t(1) << 18;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>(std::min<size_t>(hw, 32),
                                     (n + kPerThread - 1) / kPerThread);
  if (nt <= 1) return validate_range(g, vis, n);
  const size_t rec = visdata_size(g->npol);
  const size_t per = (n + nt - 1) / nt;
  std::vector<Status> res(nt);
  std::vector<std::thread> th;
  th.reserve(nt);
  for (size_t t = 0; t < nt; ++t)
    th.emplace_back([&, t]() {
      const size_t a = t * per, b = std::min(n, a + per);
      if (a < b) {
        res[t] = validate_range(
            g, static_cast<const char*>(vis) + a * rec, b - a);
        if (!res[t]) {  // report the batch index, not the chunk index
          size_t i = a;
          while (i < b && validate_range(g, static_cast<const char*>(vis) + i * rec, 1))
            ++i;
          res[t] = validate_range(g, static_cast<const char*>(vis) + i * rec, 1);
          res[t].msg = "visibility " + std::to_string(i) +
                       res[t].msg.substr(res[t].msg.find(':'));
        }
      }
    });
  for (auto& x : th) x.join();
  for (auto& r : res)
    if (!r) return r;
  return Status::ok();
}

// every Mueller index must address a Mueller plane of every CF group (the
// reference indexes the CF view without a check, src/hpg_core.hpp:656, :865)
Status validate_mueller(const hpgb_gridder* g) {
  int max_index = -1;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c)
      max_index = std::max(max_index, std::max(g->mt.m[r][c], g->mt.c[r][c]));
  for (size_t grp = 0; grp < g->cf.groups.size(); ++grp)
    if (max_index >= g->cf.groups[grp].nmueller)
      return Status::err(HPGB_ERROR_OTHER,
                         "Mueller index " + std::to_string(max_index) +
                             " exceeds the Mueller extent of CF group " +
                             std::to_string(grp));
  return Status::ok();
}

}  // namespace
}  // namespace hpgb

using namespace hpgb;

hpgb::GridGeom hpgb_gridder::geom() const {
  GridGeom g;
  g.nx = int(grid_size[0]);
  g.ny = int(grid_size[1]);
  g.nrow = int(grid_size[2]);
  g.ncube = int(grid_size[3]);
  g.scale_x = grid_scale[0];
  g.scale_y = grid_scale[1];
  g.os = int(cf.os);
  g.nfine = 2 * int(cf.os / 2) + 1;
  g.ngroups = int(cf.groups.size());
  g.mt = mt;
  g.status = vb.counters.as<unsigned>();
  return g;
}

extern "C" {

int hpgb_abi_version(void) { return HPGB_ABI_VERSION; }

const char* hpgb_last_error_message(void) { return g_last_error.c_str(); }

int hpgb_device_count(int* count) {
  return guarded([&]() -> Status {
    if (!count) return Status::err(HPGB_ERROR_OTHER, "null argument");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
      cudaGetLastError();
      c = 0;
    }
    *count = c;
    return Status::ok();
  });
}

int hpgb_create(int device_id, unsigned max_added_tasks,
                size_t max_visibility_batch_size, const unsigned grid_size[4],
                const double grid_scale[2], unsigned num_polarizations,
                const int* mueller_indexes,
                const int* conjugate_mueller_indexes, hpgb_gridder** out) {
  return guarded([&]() -> Status {
    if (!out || !grid_size || !grid_scale || !mueller_indexes ||
        !conjugate_mueller_indexes)
      return Status::err(HPGB_ERROR_OTHER, "null argument");
    *out = nullptr;
    if (num_polarizations < 1 || num_polarizations > 4)
      return Status::err(HPGB_ERROR_INVALID_NUMBER_POLARIZATIONS,
                         "number of polarizations must be 1..4");
    if (grid_size[2] < 1 || grid_size[2] > 4)
      return Status::err(HPGB_ERROR_INVALID_NUMBER_MUELLER_INDEX_ROWS,
                         "number of Mueller index rows must be 1..4");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
      cudaGetLastError();
      count = 0;
    }
    const int dev = device_id < 0 ? 0 : device_id;
    if (dev >= count)
      return Status::err(HPGB_ERROR_DISABLED_DEVICE,
                         "Requested device is not enabled");
    HPGB_CUDA_TRY(cudaSetDevice(dev));
    std::unique_ptr<hpgb_gridder> g(new hpgb_gridder);
    g->device = dev;
    g->max_added_tasks = max_added_tasks;
    g->max_batch = max_visibility_batch_size;
    std::copy(grid_size, grid_size + 4, g->grid_size);
    std::copy(grid_scale, grid_scale + 2, g->grid_scale);
    g->npol = num_polarizations;
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        const bool in = r < int(grid_size[2]) && c < int(num_polarizations);
        g->mt.m[r][c] = in ? mueller_indexes[r * num_polarizations + c] : -1;
        g->mt.c[r][c] = in ? conjugate_mueller_indexes[r * num_polarizations + c] : -1;
      }
    HPGB_CUDA_TRY(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    HPGB_TRY(g->vb.counters.reserve(256));
    HPGB_CUDA_TRY(cudaMemsetAsync(g->vb.counters.ptr, 0, 256, g->stream));
    HPGB_TRY(alloc_grid(g.get(), true));
    HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    *out = g.release();
    return Status::ok();
  });
}

int hpgb_clone(const hpgb_gridder* src, hpgb_gridder** out) {
  return guarded([&]() -> Status {
    if (!src || !out) return Status::err(HPGB_ERROR_OTHER, "null argument");
    *out = nullptr;
    HPGB_TRY(fence_impl(src));
    std::unique_ptr<hpgb_gridder> g(new hpgb_gridder);
    g->device = src->device;
    g->max_added_tasks = src->max_added_tasks;
    g->max_batch = src->max_batch;
    std::copy(src->grid_size, src->grid_size + 4, g->grid_size);
    std::copy(src->grid_scale, src->grid_scale + 2, g->grid_scale);
    g->npol = src->npol;
    g->mt = src->mt;
    g->precision = src->precision;
    g->kernel_kind = src->kernel_kind;
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    HPGB_CUDA_TRY(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    HPGB_TRY(g->vb.counters.reserve(256));
    HPGB_CUDA_TRY(cudaMemsetAsync(g->vb.counters.ptr, 0, 256, g->stream));
    HPGB_TRY(g->grid.reserve(src->grid.bytes));
    HPGB_CUDA_TRY(cudaMemcpyAsync(g->grid.ptr, src->grid.ptr, src->grid.bytes,
                                  cudaMemcpyDeviceToDevice, g->stream));
    HPGB_TRY(g->weights.reserve(src->weights.bytes));
    HPGB_CUDA_TRY(cudaMemcpyAsync(g->weights.ptr, src->weights.ptr,
                                  src->weights.bytes, cudaMemcpyDeviceToDevice,
                                  g->stream));
    if (src->has_model) {
      HPGB_TRY(g->model.reserve(src->model.bytes));
      HPGB_CUDA_TRY(cudaMemcpyAsync(g->model.ptr, src->model.ptr,
                                    src->model.bytes, cudaMemcpyDeviceToDevice,
                                    g->stream));
      g->has_model = true;
    }
    HPGB_TRY(copy_cf(g.get(), src));
    HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    *out = g.release();
    return Status::ok();
  });
}

int hpgb_destroy(hpgb_gridder* g) {
  return guarded([&]() -> Status {
    if (!g) return Status::ok();
    cudaSetDevice(g->device);
    cudaStreamSynchronize(g->stream);
    release_fft_plans(g);
    for (auto& e : g->prof_events) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    if (g->copy_stream) {
      cudaStreamSynchronize(g->copy_stream);
      cudaStreamDestroy(g->copy_stream);
    }
    if (g->staged_copied) cudaEventDestroy(g->staged_copied);
    for (cudaEvent_t e : g->staged_free)
      if (e) cudaEventDestroy(e);
    cudaStream_t s = g->stream;
    delete g;  // DevBuf destructors free device memory
    if (s) cudaStreamDestroy(s);
    return Status::ok();
  });
}

int hpgb_set_precision(hpgb_gridder* g, int precision) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    if (precision != HPGB_PRECISION_FP64 && precision != HPGB_PRECISION_MIXED)
      return Status::err(HPGB_ERROR_OTHER, "unknown precision");
    g->precision = precision;
    return Status::ok();
  });
}

int hpgb_set_gridding_kernel(hpgb_gridder* g, int kind) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    if (kind != HPGB_KERNEL_AUTO && kind != HPGB_KERNEL_DIRECT &&
        kind != HPGB_KERNEL_TILED)
      return Status::err(HPGB_ERROR_OTHER, "unknown kernel kind");
    g->kernel_kind = kind;
    return Status::ok();
  });
}

int hpgb_get_stream(const hpgb_gridder* g, void** stream) {
  return guarded([&]() -> Status {
    if (!g || !stream) return Status::err(HPGB_ERROR_OTHER, "null argument");
    *stream = static_cast<void*>(g->stream);
    return Status::ok();
  });
}

int hpgb_cf_region_size(const hpgb_gridder* g, unsigned os, unsigned ngroups,
                        const unsigned* extents, size_t* bytes) {
  return guarded([&]() -> Status {
    if (!bytes) return Status::err(HPGB_ERROR_OTHER, "null argument");
    if (ngroups == 0 || !extents) {
      *bytes = g ? g->cf.data.bytes + g->cf.wsum.bytes : 0;
      return Status::ok();
    }
    if (os == 0) return Status::err(HPGB_ERROR_OTHER, "oversampling must be > 0");
    size_t d = 0, w = 0;
    HPGB_TRY(cf_region_bytes(os, ngroups, extents, &d, &w));
    *bytes = d + w;
    return Status::ok();
  });
}

int hpgb_allocate_cf_region(hpgb_gridder* g, unsigned os, unsigned ngroups,
                            const unsigned* extents) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    HPGB_TRY(fence_impl(g));
    if (ngroups == 0 || !extents) return Status::ok();
    if (os == 0) return Status::err(HPGB_ERROR_OTHER, "oversampling must be > 0");
    size_t d = 0, w = 0;
    HPGB_TRY(cf_region_bytes(os, ngroups, extents, &d, &w));
    HPGB_TRY(g->cf.data.reserve(std::max<size_t>(d, 16)));
    HPGB_TRY(g->cf.wsum.reserve(std::max<size_t>(w, 16)));
    return Status::ok();
  });
}

int hpgb_set_cf(hpgb_gridder* g, unsigned os, unsigned ngroups,
                const unsigned* extents, const void* const* values, int layout,
                int values_on_device) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    if (ngroups > 0 && (!extents || !values))
      return Status::err(HPGB_ERROR_OTHER, "null argument");
    return set_cf(g, os, ngroups, extents, values, layout, values_on_device != 0);
  });
}

int hpgb_set_model(hpgb_gridder* g, const void* values, const unsigned ext[4],
                   int layout, int on_device) {
  return guarded([&]() -> Status {
    if (!g || !values || !ext) return Status::err(HPGB_ERROR_OTHER, "null argument");
    if (!std::equal(ext, ext + 4, g->grid_size))
      return Status::err(
          HPGB_ERROR_INVALID_MODEL_GRID_SIZE,
          "model grid size [" + std::to_string(ext[0]) + "," +
              std::to_string(ext[1]) + "," + std::to_string(ext[2]) + "," +
              std::to_string(ext[3]) + "] is different from visibility grid size [" +
              std::to_string(g->grid_size[0]) + "," + std::to_string(g->grid_size[1]) +
              "," + std::to_string(g->grid_size[2]) + "," +
              std::to_string(g->grid_size[3]) + "]");
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    HPGB_TRY(fence_impl(g));
    const size_t n = g->grid_elems();
    HPGB_TRY(g->model.reserve(std::max<size_t>(n, 1) * sizeof(double2)));
    if (layout == HPGB_LAYOUT_LEFT) {
      HPGB_CUDA_TRY(cudaMemcpyAsync(g->model.ptr, values, n * sizeof(double2),
                                    on_device ? cudaMemcpyDeviceToDevice
                                              : cudaMemcpyHostToDevice,
                                    g->stream));
    } else {
      DevBuf tmp;
      const void* src = values;
      if (!on_device) {
        HPGB_TRY(tmp.reserve(n * sizeof(double2)));
        HPGB_CUDA_TRY(cudaMemcpyAsync(tmp.ptr, values, n * sizeof(double2),
                                      cudaMemcpyHostToDevice, g->stream));
        src = tmp.ptr;
      }
      HPGB_TRY(to_layout(g, static_cast<const double2*>(src),
                         g->model.as<double2>(), layout, true, g->grid_size));
      HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    g->has_model = true;
    g->model32_valid = false;
    return Status::ok();
  });
}

// copy stream and events of the staged host-batch path, made on first use
static Status ensure_staging(hpgb_gridder* g) {
  if (g->copy_stream) return Status::ok();
  HPGB_CUDA_TRY(cudaEventCreateWithFlags(&g->staged_copied, cudaEventDisableTiming));
  for (int b = 0; b < 2; ++b)
    HPGB_CUDA_TRY(cudaEventCreateWithFlags(&g->staged_free[b], cudaEventDisableTiming));
  HPGB_CUDA_TRY(cudaStreamCreateWithFlags(&g->copy_stream, cudaStreamNonBlocking));
  return Status::ok();
}

int hpgb_grid_visibilities(hpgb_gridder* g, const void* vis, size_t n,
                           unsigned npol, unsigned flags, int vis_on_device,
                           void* returned) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    // validation order of src/hpg_runtime.hpp:1816-1828
    if (n > g->max_batch)
      return Status::err(HPGB_ERROR_EXCESSIVE_NUMBER_VISIBILITIES,
                         "Number of visibilities exceeds maximum batch size");
    if (npol != g->npol)
      return Status::err(HPGB_ERROR_INVALID_NUMBER_POLARIZATIONS,
                         "Number of visibility polarizations does not match "
                         "Mueller matrix");
    const bool do_grid = flags & HPGB_DO_GRID;
    if (!do_grid && (flags & HPGB_UPDATE_GRID_WEIGHTS))
      return Status::err(HPGB_ERROR_UPDATE_WEIGHTS_WITHOUT_GRIDDING,
                         "Unable to update grid weights during degridding only");
    if (n == 0) return Status::ok();
    if (!vis) return Status::err(HPGB_ERROR_OTHER, "null visibilities");
    if ((flags & HPGB_RETURN_VISIBILITIES) && !returned)
      return Status::err(HPGB_ERROR_OTHER, "null buffer for returned visibilities");
    if (!g->cf.set)
      return Status::err(HPGB_ERROR_OTHER, "no convolution function set");
    HPGB_TRY(validate_mueller(g));
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    const size_t rec = visdata_size(npol);
    const size_t bytes = n * rec;
    // A host batch outside a stream capture is copied on the copy stream
    // into the staging buffer not used by the previous call, so that the
    // copy overlaps the previous call's work (the work on the gridder's
    // stream waits for it).  Device batches and captured calls copy into
    // vb.vis on the gridder's stream.
    bool staged = false;
    if (!vis_on_device) {
      cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
      HPGB_CUDA_TRY(cudaStreamIsCapturing(g->stream, &cap));
      staged = cap == cudaStreamCaptureStatusNone;
    }
    const int b = g->staged_next;
    void* dvis = nullptr;
    cudaStream_t cs = g->stream;
    if (staged) {
      HPGB_TRY(ensure_staging(g));
      HPGB_TRY(g->vb.staged[b].reserve(g->max_batch * rec));
      dvis = g->vb.staged[b].ptr;
      cs = g->copy_stream;
      // the buffer's batch of two calls ago must be done with it
      HPGB_CUDA_TRY(cudaStreamWaitEvent(cs, g->staged_free[b], 0));
    } else {
      HPGB_TRY(g->vb.vis.reserve(g->max_batch * rec));
      dvis = g->vb.vis.ptr;
    }
    // the copy is queued first, so that checking the indexes of host
    // records overlaps the transfer; a batch that fails the check is
    // copied (the call waits for that copy, the caller may free its
    // buffer on return) but never gridded
    HPGB_CUDA_TRY(cudaMemcpyAsync(
        dvis, vis, bytes,
        vis_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, cs));
    if (staged) {
      HPGB_CUDA_TRY(cudaEventRecord(g->staged_copied, cs));
      HPGB_CUDA_TRY(cudaStreamWaitEvent(g->stream, g->staged_copied, 0));
    }
    Status st = Status::ok();
    if (!vis_on_device) {
      st = validate_indexes(g, vis, n);
      if (!st) cudaStreamSynchronize(g->stream);
    }
    if (st) st = grid_batch(g, dvis, n, flags);
    if (st && (flags & HPGB_RETURN_VISIBILITIES)) {
      const cudaError_t e = cudaMemcpyAsync(
          returned, dvis, bytes,
          vis_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
          g->stream);
      if (e != cudaSuccess) {
        st = Status::err(HPGB_ERROR_OTHER, cudaGetErrorString(e));
      } else {
        g->pending_dst = returned;
        g->pending_bytes = bytes;
        g->pending_on_device = vis_on_device != 0;
      }
    }
    if (staged) {
      // everything queued that reads the buffer precedes this record
      const cudaError_t e = cudaEventRecord(g->staged_free[b], g->stream);
      if (e != cudaSuccess && st)
        st = Status::err(HPGB_ERROR_OTHER, cudaGetErrorString(e));
      g->staged_next = b ^ 1;
    }
    return st;
  });
}

int hpgb_grid_visibilities_noalloc(hpgb_gridder* g, void* vis, size_t n,
                                   unsigned npol, unsigned flags) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    // validation order of src/hpg_runtime.hpp:1816-1828
    if (n > g->max_batch)
      return Status::err(HPGB_ERROR_EXCESSIVE_NUMBER_VISIBILITIES,
                         "Number of visibilities exceeds maximum batch size");
    if (npol != g->npol)
      return Status::err(HPGB_ERROR_INVALID_NUMBER_POLARIZATIONS,
                         "Number of visibility polarizations does not match "
                         "Mueller matrix");
    if (!(flags & HPGB_DO_GRID) && (flags & HPGB_UPDATE_GRID_WEIGHTS))
      return Status::err(HPGB_ERROR_UPDATE_WEIGHTS_WITHOUT_GRIDDING,
                         "Unable to update grid weights during degridding only");
    if (n == 0) return Status::ok();
    if (!vis) return Status::err(HPGB_ERROR_OTHER, "null visibilities");
    if (!g->cf.set)
      return Status::err(HPGB_ERROR_OTHER, "no convolution function set");
    HPGB_TRY(validate_mueller(g));
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    return grid_direct_noalloc(g, vis, n, flags);
  });
}

static int linear_entry(hpgb_gridder* g, const void* vis, size_t n,
                        unsigned npol, int op, const void* in, void* out) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    if (n > g->max_batch)
      return Status::err(HPGB_ERROR_EXCESSIVE_NUMBER_VISIBILITIES,
                         "Number of visibilities exceeds maximum batch size");
    if (npol != g->npol)
      return Status::err(HPGB_ERROR_INVALID_NUMBER_POLARIZATIONS,
                         "Number of visibility polarizations does not match "
                         "Mueller matrix");
    if (n == 0) return Status::ok();
    if (!vis || !in || !out) return Status::err(HPGB_ERROR_OTHER, "null argument");
    if (!g->cf.set)
      return Status::err(HPGB_ERROR_OTHER, "no convolution function set");
    HPGB_TRY(validate_mueller(g));
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    return linear_op(g, vis, n, op, in, out);
  });
}

int hpgb_degrid_linear(hpgb_gridder* g, const void* vis, size_t n,
                       unsigned npol, const void* model, void* values) {
  return linear_entry(g, vis, n, npol, 0, model, values);
}

int hpgb_degrid_adjoint(hpgb_gridder* g, const void* vis, size_t n,
                        unsigned npol, const void* values_cotangent,
                        void* model_cotangent) {
  return linear_entry(g, vis, n, npol, 1, values_cotangent, model_cotangent);
}

int hpgb_grid_linear(hpgb_gridder* g, const void* vis, size_t n,
                     unsigned npol, const void* values, void* grid) {
  return linear_entry(g, vis, n, npol, 2, values, grid);
}

int hpgb_grid_adjoint(hpgb_gridder* g, const void* vis, size_t n,
                      unsigned npol, const void* grid_cotangent,
                      void* values_cotangent) {
  return linear_entry(g, vis, n, npol, 3, grid_cotangent, values_cotangent);
}

int hpgb_fence(const hpgb_gridder* g) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    return fence_impl(g);
  });
}

int hpgb_copy_weights(const hpgb_gridder* cg, double* dst, int layout) {
  return guarded([&]() -> Status {
    if (!cg || !dst) return Status::err(HPGB_ERROR_OTHER, "null argument");
    hpgb_gridder* g = const_cast<hpgb_gridder*>(cg);
    HPGB_TRY(fence_impl(g));
    std::vector<double> h(g->weight_elems());
    HPGB_CUDA_TRY(cudaMemcpy(h.data(), g->weights.ptr, h.size() * sizeof(double),
                             cudaMemcpyDeviceToHost));
    return weights_to_layout(g, h.data(), dst, layout);
  });
}

static Status copy_values(hpgb_gridder* g, const DevBuf& buf, bool present,
                          void* dst, int layout) {
  HPGB_TRY(fence_impl(g));
  const size_t n = g->grid_elems();
  if (!present) {
    std::memset(dst, 0, n * sizeof(double2));
    return Status::ok();
  }
  if (layout == HPGB_LAYOUT_LEFT) {
    HPGB_CUDA_TRY(cudaMemcpy(dst, buf.ptr, n * sizeof(double2),
                             cudaMemcpyDeviceToHost));
    return Status::ok();
  }
  DevBuf tmp;
  HPGB_TRY(tmp.reserve(std::max<size_t>(n, 1) * sizeof(double2)));
  HPGB_TRY(to_layout(g, buf.as<const double2>(), tmp.as<double2>(), layout,
                     false, g->grid_size));
  HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
  HPGB_CUDA_TRY(cudaMemcpy(dst, tmp.ptr, n * sizeof(double2),
                           cudaMemcpyDeviceToHost));
  return Status::ok();
}

int hpgb_copy_grid(const hpgb_gridder* cg, void* dst, int layout) {
  return guarded([&]() -> Status {
    if (!cg || !dst) return Status::err(HPGB_ERROR_OTHER, "null argument");
    hpgb_gridder* g = const_cast<hpgb_gridder*>(cg);
    return copy_values(g, g->grid, true, dst, layout);
  });
}

int hpgb_copy_model(const hpgb_gridder* cg, void* dst, int layout) {
  return guarded([&]() -> Status {
    if (!cg || !dst) return Status::err(HPGB_ERROR_OTHER, "null argument");
    hpgb_gridder* g = const_cast<hpgb_gridder*>(cg);
    return copy_values(g, g->model, g->has_model, dst, layout);
  });
}

int hpgb_weights_device_ptr(const hpgb_gridder* g, void** ptr, size_t* span) {
  return guarded([&]() -> Status {
    if (!g || !ptr) return Status::err(HPGB_ERROR_OTHER, "null argument");
    *ptr = g->weights.ptr;
    if (span) *span = g->weight_elems();
    return Status::ok();
  });
}

int hpgb_grid_device_ptr(const hpgb_gridder* g, void** ptr, size_t* span) {
  return guarded([&]() -> Status {
    if (!g || !ptr) return Status::err(HPGB_ERROR_OTHER, "null argument");
    *ptr = g->grid.ptr;
    if (span) *span = g->grid_elems();
    return Status::ok();
  });
}

int hpgb_model_device_ptr(const hpgb_gridder* g, void** ptr, size_t* span) {
  return guarded([&]() -> Status {
    if (!g || !ptr) return Status::err(HPGB_ERROR_OTHER, "null argument");
    *ptr = g->has_model ? g->model.ptr : nullptr;
    if (span) *span = g->has_model ? g->grid_elems() : 0;
    return Status::ok();
  });
}

int hpgb_reset_grid(hpgb_gridder* g) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    HPGB_TRY(fence_impl(g));
    HPGB_TRY(alloc_grid(g, true));
    HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return Status::ok();
  });
}

int hpgb_reset_model(hpgb_gridder* g) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    HPGB_TRY(fence_impl(g));
    g->model.release();
    g->has_model = false;
    g->model32_valid = false;
    return Status::ok();
  });
}

int hpgb_normalize_by_weights(hpgb_gridder* g, double wfactor) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    return normalize_by_weights(g, wfactor);
  });
}

int hpgb_apply_grid_fft(hpgb_gridder* g, double norm, int sign, int in_place) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    return fft(g, g->grid, norm, sign, in_place != 0);
  });
}

int hpgb_apply_model_fft(hpgb_gridder* g, double norm, int sign, int in_place) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    if (!g->has_model) return Status::ok();  // src/hpg_runtime.hpp:1369
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    g->model32_valid = false;
    return fft(g, g->model, norm, sign, in_place != 0);
  });
}

int hpgb_image_grid(hpgb_gridder* g, double wfactor, double norm, int sign,
                    int direction) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    return image_tail(g, wfactor, norm, sign, direction);
  });
}

int hpgb_shift_grid(hpgb_gridder* g, int direction) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    return shift(g, g->grid.as<double2>(), direction);
  });
}

int hpgb_shift_model(hpgb_gridder* g, int direction) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    if (!g->has_model) return Status::ok();
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    g->model32_valid = false;
    return shift(g, g->model.as<double2>(), direction);
  });
}

int hpgb_kernel_launches(const hpgb_gridder* g, uint64_t* count) {
  return guarded([&]() -> Status {
    if (!g || !count) return Status::err(HPGB_ERROR_OTHER, "null argument");
    *count = g->launches;
    return Status::ok();
  });
}

int hpgb_set_tiled_plan(hpgb_gridder* g, int ring_parts, int chunk_vis) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    if (ring_parts < 0 || (ring_parts > 0 && ring_parts < 2) ||
        ring_parts > 16 || chunk_vis < 0 || chunk_vis > (1 << 20))
      return Status::err(HPGB_ERROR_OTHER,
                         "ring_parts must be 0 or 2..16 and chunk_vis 0..2^20");
    g->tplan = hpgb_tiled_plan{ring_parts, chunk_vis, 0, 0};
    return Status::ok();
  });
}

int hpgb_set_tiled_plan_ex(hpgb_gridder* g, const hpgb_tiled_plan* plan) {
  return guarded([&]() -> Status {
    if (!g || !plan) return Status::err(HPGB_ERROR_OTHER, "null argument");
    const hpgb_tiled_plan& t = *plan;
    if (t.ring_parts < 0 || (t.ring_parts > 0 && t.ring_parts < 2) ||
        t.ring_parts > 16 || t.chunk_vis < 0 || t.chunk_vis > (1 << 20))
      return Status::err(HPGB_ERROR_OTHER,
                         "ring_parts must be 0 or 2..16 and chunk_vis 0..2^20");
    if (t.tile_side < 0 || t.tile_side > 128 || (t.tile_side & 1))
      return Status::err(HPGB_ERROR_OTHER,
                         "tile_side must be 0 or an even number up to 128");
    if (t.compensated < 0 || t.compensated > HPGB_COMPENSATED_ON)
      return Status::err(HPGB_ERROR_OTHER, "compensated takes 0, 1 or 2");
    g->tplan = t;
    return Status::ok();
  });
}

int hpgb_get_tiled_plan(const hpgb_gridder* g, hpgb_tiled_plan* plan) {
  return guarded([&]() -> Status {
    if (!g || !plan) return Status::err(HPGB_ERROR_OTHER, "null argument");
    *plan = g->tplan;
    return Status::ok();
  });
}

int hpgb_grid_visibilities_batch(hpgb_gridder* const* gridders, size_t num,
                                 const void* const* vis, const size_t* nvis,
                                 unsigned npol, unsigned flags,
                                 int vis_on_device, void* const* returned) {
  return guarded([&]() -> Status {
    if (!gridders || !vis || !nvis || num == 0)
      return Status::err(HPGB_ERROR_OTHER, "null argument");
    if (num > 96)
      return Status::err(HPGB_ERROR_OTHER, "at most 96 gridders per batch");
    hpgb_gridder* g0 = gridders[0];
    if (!g0) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    const bool do_grid = flags & HPGB_DO_GRID;
    const bool ret = flags & HPGB_RETURN_VISIBILITIES;
    for (size_t j = 0; j < num; ++j) {
      hpgb_gridder* g = gridders[j];
      if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
      for (size_t i = 0; i < j; ++i)
        if (gridders[i] == g)
          return Status::err(HPGB_ERROR_OTHER, "a gridder appears twice");
      // validation order of src/hpg_runtime.hpp:1816-1828, per gridder
      if (nvis[j] > g->max_batch)
        return Status::err(HPGB_ERROR_EXCESSIVE_NUMBER_VISIBILITIES,
                           "Number of visibilities exceeds maximum batch size");
      if (npol != g->npol)
        return Status::err(HPGB_ERROR_INVALID_NUMBER_POLARIZATIONS,
                           "Number of visibility polarizations does not match "
                           "Mueller matrix");
      if (!do_grid && (flags & HPGB_UPDATE_GRID_WEIGHTS))
        return Status::err(HPGB_ERROR_UPDATE_WEIGHTS_WITHOUT_GRIDDING,
                           "Unable to update grid weights during degridding only");
      if (nvis[j] > 0 && !vis[j])
        return Status::err(HPGB_ERROR_OTHER, "null visibilities");
      if (ret && nvis[j] > 0 && (!returned || !returned[j]))
        return Status::err(HPGB_ERROR_OTHER,
                           "null buffer for returned visibilities");
      if (!g->cf.set)
        return Status::err(HPGB_ERROR_OTHER, "no convolution function set");
      HPGB_TRY(validate_mueller(g));
      bool same = g->device == g0->device &&
                  g->grid_size[2] == g0->grid_size[2] &&
                  g->precision == g0->precision &&
                  g->tplan.compensated == g0->tplan.compensated &&
                  (!(flags & HPGB_DO_DEGRID) || g->has_model == g0->has_model);
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
          same = same && g->mt.m[r][c] == g0->mt.m[r][c] &&
                 g->mt.c[r][c] == g0->mt.c[r][c];
      if (!same)
        return Status::err(HPGB_ERROR_OTHER,
                           "the gridders of a batch must share their device, "
                           "grid rows, Mueller tables, precision, compensation "
                           "and (when degridding) whether a model is set");
    }
    if (!(flags & (HPGB_DO_DEGRID | HPGB_DO_GRID))) return Status::ok();
    HPGB_CUDA_TRY(cudaSetDevice(g0->device));
    const cudaStream_t st = g0->stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    HPGB_CUDA_TRY(cudaStreamIsCapturing(st, &cap));
    const bool capturing = cap != cudaStreamCaptureStatusNone;
    // the others' queued work comes first
    if (!capturing)
      for (size_t j = 1; j < num; ++j) {
        cudaEvent_t e;
        HPGB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        cudaEventRecord(e, gridders[j]->stream);
        cudaStreamWaitEvent(st, e, 0);
        cudaEventDestroy(e);
      }
    const size_t rec = visdata_size(npol);
    std::vector<void*> dvis(num, nullptr);
    for (size_t j = 0; j < num; ++j) {
      hpgb_gridder* g = gridders[j];
      if (!vis_on_device && nvis[j] > 0)
        HPGB_TRY(validate_indexes(g, vis[j], nvis[j]));
      HPGB_TRY(g->vb.vis.reserve(std::max<size_t>(g->max_batch, 1) * rec));
      dvis[j] = g->vb.vis.ptr;
      if (nvis[j] > 0)
        HPGB_CUDA_TRY(cudaMemcpyAsync(
            dvis[j], vis[j], nvis[j] * rec,
            vis_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
            st));
    }
    HPGB_TRY(grid_batch_tiled(gridders, num, dvis.data(), nvis, flags));
    for (size_t j = 0; j < num; ++j) {
      if (nvis[j] > 0) gridders[j]->last_kernel = HPGB_KERNEL_TILED;
      if (ret && nvis[j] > 0)
        HPGB_CUDA_TRY(cudaMemcpyAsync(
            returned[j], dvis[j], nvis[j] * rec,
            vis_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
            st));
    }
    // work queued on the others later comes after the batch
    if (!capturing) {
      cudaEvent_t e;
      HPGB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      HPGB_CUDA_TRY(cudaEventRecord(e, st));
      for (size_t j = 1; j < num; ++j)
        cudaStreamWaitEvent(gridders[j]->stream, e, 0);
      cudaEventDestroy(e);
    }
    return Status::ok();
  });
}

int hpgb_set_wait_limit(hpgb_gridder* g, double seconds) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    if (!(seconds >= 1e-4 && seconds <= 60.0))
      return Status::err(HPGB_ERROR_OTHER, "wait limit must be 1e-4..60 s");
    g->wait_limit_ns = static_cast<unsigned long long>(seconds * 1e9);
    return Status::ok();
  });
}

int hpgb_debug_withhold_copy(hpgb_gridder* g, long long visibility) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    if (visibility < -1)
      return Status::err(HPGB_ERROR_OTHER, "visibility position must be >= -1");
    g->withhold_vis = visibility;
    return Status::ok();
  });
}

int hpgb_last_gridding_kernel(const hpgb_gridder* g, int* kind) {
  return guarded([&]() -> Status {
    if (!g || !kind) return Status::err(HPGB_ERROR_OTHER, "null argument");
    *kind = g->last_kernel;
    return Status::ok();
  });
}

int hpgb_autotune_tiled(hpgb_gridder* g, const void* vis, size_t n,
                        unsigned npol, unsigned flags, int vis_on_device,
                        int* ring_parts, int* chunk_vis) {
  return guarded([&]() -> Status {
    if (!g || !ring_parts || !chunk_vis)
      return Status::err(HPGB_ERROR_OTHER, "null argument");
    if (n > g->max_batch)
      return Status::err(HPGB_ERROR_EXCESSIVE_NUMBER_VISIBILITIES,
                         "Number of visibilities exceeds maximum batch size");
    if (npol != g->npol)
      return Status::err(HPGB_ERROR_INVALID_NUMBER_POLARIZATIONS,
                         "Number of visibility polarizations does not match "
                         "Mueller matrix");
    if (!(flags & HPGB_DO_GRID) && (flags & HPGB_UPDATE_GRID_WEIGHTS))
      return Status::err(HPGB_ERROR_UPDATE_WEIGHTS_WITHOUT_GRIDDING,
                         "Unable to update grid weights during degridding only");
    if (n == 0 || !vis)
      return Status::err(HPGB_ERROR_OTHER, "autotuning needs visibilities");
    if (!g->cf.set)
      return Status::err(HPGB_ERROR_OTHER, "no convolution function set");
    HPGB_TRY(validate_mueller(g));
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    HPGB_TRY(fence_impl(g));
    return autotune_tiled(g, vis, n, flags & ~HPGB_RETURN_VISIBILITIES,
                          vis_on_device != 0, ring_parts, chunk_vis);
  });
}

int hpgb_begin_capture(hpgb_gridder* g) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    HPGB_TRY(fence_impl(g));
    HPGB_CUDA_TRY(
        cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeRelaxed));
    g->capture_launches0 = g->launches;
    return Status::ok();
  });
}

int hpgb_end_capture(hpgb_gridder* g, hpgb_graph** out) {
  return guarded([&]() -> Status {
    if (!g || !out) return Status::err(HPGB_ERROR_OTHER, "null argument");
    *out = nullptr;
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    cudaGraph_t graph = nullptr;
    HPGB_CUDA_TRY(cudaStreamEndCapture(g->stream, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t rc = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (rc != cudaSuccess)
      return Status::err(HPGB_ERROR_OTHER,
                         std::string("cudaGraphInstantiate: ") +
                             cudaGetErrorString(rc));
    auto* h = new hpgb_graph;
    h->exec = exec;
    h->device = g->device;
    h->launches = g->launches - g->capture_launches0;
    *out = h;
    return Status::ok();
  });
}

int hpgb_graph_launch(hpgb_gridder* g, const hpgb_graph* graph) {
  return guarded([&]() -> Status {
    if (!g || !graph) return Status::err(HPGB_ERROR_OTHER, "null argument");
    if (graph->device != g->device)
      return Status::err(HPGB_ERROR_OTHER, "graph captured on another device");
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    HPGB_CUDA_TRY(cudaGraphLaunch(graph->exec, g->stream));
    g->launches += graph->launches;
    return Status::ok();
  });
}

int hpgb_graph_destroy(hpgb_graph* graph) {
  return guarded([&]() -> Status {
    if (!graph) return Status::ok();
    cudaSetDevice(graph->device);
    cudaGraphExecDestroy(graph->exec);
    delete graph;
    return Status::ok();
  });
}

int hpgb_profile_tiled_kernel(hpgb_gridder* g, int enable) {
  return guarded([&]() -> Status {
    if (!g) return Status::err(HPGB_ERROR_OTHER, "null gridder");
    g->profile = enable != 0;
    return Status::ok();
  });
}

int hpgb_tiled_kernel_time(hpgb_gridder* g, double* total_ms,
                           uint64_t* count) {
  return guarded([&]() -> Status {
    if (!g || !total_ms || !count)
      return Status::err(HPGB_ERROR_OTHER, "null argument");
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    double sum = 0.0;
    Status st = Status::ok();
    for (auto& e : g->prof_events) {
      float ms = 0.f;
      const cudaError_t rc = cudaEventElapsedTime(&ms, e.first, e.second);
      if (rc != cudaSuccess && st)
        st = Status::err(HPGB_ERROR_OTHER,
                         std::string("cudaEventElapsedTime: ") +
                             cudaGetErrorString(rc));
      sum += ms;
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    *count = g->prof_events.size();
    *total_ms = sum;
    g->prof_events.clear();
    return st;
  });
}

int hpgb_debug_coords(hpgb_gridder* g, const void* vis, size_t n,
                      unsigned npol, hpgb_vis_coords* out) {
  return guarded([&]() -> Status {
    if (!g || (n > 0 && (!vis || !out)))
      return Status::err(HPGB_ERROR_OTHER, "null argument");
    if (npol != g->npol)
      return Status::err(HPGB_ERROR_INVALID_NUMBER_POLARIZATIONS,
                         "Number of visibility polarizations does not match "
                         "Mueller matrix");
    if (!g->cf.set) return Status::err(HPGB_ERROR_OTHER, "no convolution function set");
    if (n == 0) return Status::ok();
    HPGB_CUDA_TRY(cudaSetDevice(g->device));
    HPGB_TRY(fence_impl(g));
    const size_t rec = visdata_size(npol);
    DevBuf dv, dout;
    HPGB_TRY(dv.reserve(n * rec));
    HPGB_TRY(dout.reserve(n * sizeof(hpgb_vis_coords)));
    HPGB_CUDA_TRY(cudaMemcpyAsync(dv.ptr, vis, n * rec, cudaMemcpyHostToDevice,
                                  g->stream));
    HPGB_TRY(debug_coords(g, dv.ptr, n, dout.as<hpgb_vis_coords>()));
    HPGB_CUDA_TRY(cudaMemcpyAsync(out, dout.ptr, n * sizeof(hpgb_vis_coords),
                                  cudaMemcpyDeviceToHost, g->stream));
    HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    // an out-of-range index shows as in_grid = 0; clear the status bit
    HPGB_CUDA_TRY(cudaMemset(g->vb.counters.ptr, 0, sizeof(unsigned)));
    return Status::ok();
  });
}

}  // extern "C"
