// cf_layout.cu -- CF ingestion: host or device values in any of the
// reference's CF layouts -> this device's slice layout (see common.cuh), plus
// the per-slice FP64 sums.
//
// Replaces CFPool::add_host_cfs / add_device_cfs (src/hpg_runtime.hpp:458-551)
// and the host-side element-by-element layout loop init_cf_host
// (src/hpg_impl.hpp:1013-1047) with one device kernel per group.

#include <algorithm>
#include <cstring>

#include "gridder.cuh"

namespace hpgb {

namespace {

struct GroupShape {
  int taps_x, taps_y, nmueller, ncube, nfine, plane_stride;
  long long nslices, slice_stride;
};

// CFArray::radii (src/hpg.hpp:687-694), unsigned arithmetic as in the reference
inline unsigned cf_radius(unsigned ext, unsigned os) {
  return ((ext - 4u * os) / os) / 2u;
}

GroupShape group_shape(unsigned os, const unsigned* ext) {
  GroupShape s;
  s.taps_x = 2 * int(cf_radius(ext[0], os)) + 1;
  s.taps_y = 2 * int(cf_radius(ext[1], os)) + 1;
  s.nmueller = int(ext[2]);
  s.ncube = int(ext[3]);
  s.nfine = 2 * int(os / 2) + 1;
  s.nslices = (long long)s.ncube * s.nfine * s.nfine;
  s.plane_stride = (s.taps_x * s.taps_y + 1) & ~1;  // 16-byte multiple
  s.slice_stride = (long long)s.nmueller * s.plane_stride;
  return s;
}

struct LayoutArgs {
  const float2* in;
  float2* out;
  int layout;
  int os, nfine;
  unsigned ext[4];
  int taps_x, taps_y, nmueller, ncube, plane_stride;
  long long slice_stride;
  long long total;  // nslices * nmueller * taps_y * taps_x
};

__global__ void cf_layout_kernel(LayoutArgs a) {
  const long long per_slice = (long long)a.nmueller * a.taps_y * a.taps_x;
  const long long xm = (a.ext[0] + a.os - 1) / a.os;
  const long long ym = (a.ext[1] + a.os - 1) / a.os;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
       i < a.total; i += (long long)gridDim.x * blockDim.x) {
    const long long s = i / per_slice;
    long long r = i - s * per_slice;
    const int m = int(r / ((long long)a.taps_y * a.taps_x));
    r -= (long long)m * a.taps_y * a.taps_x;
    const int Y = int(r / a.taps_x);
    const int X = int(r - (long long)Y * a.taps_x);
    const int fx = int(s % a.nfine);
    const int fy = int((s / a.nfine) % a.nfine);
    const int cube = int(s / ((long long)a.nfine * a.nfine));
    const long long x = (long long)(2 + X) * a.os + (fx - a.os / 2);
    const long long y = (long long)(2 + Y) * a.os + (fy - a.os / 2);
    float2 v = make_float2(0.f, 0.f);
    if (x >= 0 && y >= 0 && x < a.ext[0] && y < a.ext[1]) {
      long long idx;
      if (a.layout == HPGB_CF_LAYOUT_LOGICAL) {
        idx = ((x * a.ext[1] + y) * a.ext[2] + m) * a.ext[3] + cube;
      } else {
        const long long xmaj = x / a.os, xmin = x % a.os;
        const long long ymaj = y / a.os, ymin = y % a.os;
        const long long minor = xmin + (long long)a.os * ymin;
        if (a.layout == HPGB_CF_LAYOUT_CUDA_V0)
          idx = xmaj + xm * (ymaj + ym * (m + (long long)a.ext[2] *
                                                  (cube + a.ext[3] * minor)));
        else
          idx = m + (long long)a.ext[2] *
                        (ymaj + ym * (xmaj + xm * (cube + a.ext[3] * minor)));
      }
      v = a.in[idx];
    }
    a.out[s * a.slice_stride + (long long)m * a.plane_stride + r] = v;
  }
}

// one warp per (slice, mueller): FP64 sum of the taps_x*taps_y values
__global__ void cf_wsum_kernel(const float2* data, double2* wsum,
                               long long nslices, int nmueller, int taps,
                               int plane_stride, long long slice_stride) {
  const long long warp =
      (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nslices * nmueller) return;
  const long long s = warp / nmueller;
  const int m = int(warp - s * nmueller);
  const float2* p = data + s * slice_stride + (long long)m * plane_stride;
  double sx = 0, sy = 0;
  for (int i = lane; i < taps; i += 32) {
    const float2 v = p[i];
    sx += v.x;
    sy += v.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_down_sync(0xffffffffu, sx, o);
    sy += __shfl_down_sync(0xffffffffu, sy, o);
  }
  if (lane == 0) wsum[warp] = make_double2(sx, sy);
}

long long input_elems(int layout, unsigned os, const unsigned* ext) {
  if (layout == HPGB_CF_LAYOUT_LOGICAL)
    return (long long)ext[0] * ext[1] * ext[2] * ext[3];
  const long long xm = (ext[0] + os - 1) / os, ym = (ext[1] + os - 1) / os;
  return xm * ym * (long long)ext[2] * ext[3] * os * os;
}

}  // namespace

Status DevBuf::reserve(size_t n) {
  if (n <= bytes && ptr) return Status::ok();
  release();
  if (n == 0) return Status::ok();
  HPGB_CUDA_TRY(cudaMalloc(&ptr, n));
  bytes = n;
  return Status::ok();
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

Status cf_region_bytes(unsigned os, unsigned ngroups, const unsigned* extents,
                       size_t* data_bytes, size_t* wsum_bytes) {
  size_t d = 0, w = 0;
  for (unsigned g = 0; g < ngroups; ++g) {
    const GroupShape s = group_shape(os, extents + 4 * g);
    d += size_t(s.nslices) * size_t(s.slice_stride) * sizeof(float2);
    w += size_t(s.nslices) * size_t(s.nmueller) * sizeof(double2);
  }
  *data_bytes = d;
  *wsum_bytes = w;
  return Status::ok();
}

Status set_cf(hpgb_gridder* g, unsigned os, unsigned ngroups,
              const unsigned* extents, const void* const* values, int layout,
              bool on_device) {
  if (os == 0) return Status::err(HPGB_ERROR_OTHER, "oversampling must be > 0");
  if (layout != HPGB_CF_LAYOUT_LOGICAL && layout != HPGB_CF_LAYOUT_CUDA_V0 &&
      layout != HPGB_CF_LAYOUT_HOST_V0)
    return Status::err(HPGB_ERROR_INVALID_CF_LAYOUT, "unknown CF layout");
  // src/hpg_runtime.hpp:893-902
  for (unsigned grp = 0; grp < ngroups; ++grp) {
    const unsigned* e = extents + 4 * grp;
    if (e[0] > g->grid_size[0] * os || e[1] > g->grid_size[1] * os)
      return Status::err(HPGB_ERROR_CF_SUPPORT_EXCEEDS_GRID,
                         "CF support size exceeds grid size");
  }
  for (unsigned grp = 0; grp < ngroups; ++grp) {
    const unsigned* e = extents + 4 * grp;
    if (e[0] < 4 * os || e[1] < 4 * os)
      return Status::err(HPGB_ERROR_OTHER,
                         "CF extents smaller than the padded minimum");
  }
  HPGB_CUDA_TRY(cudaSetDevice(g->device));
  size_t data_bytes = 0, wsum_bytes = 0;
  HPGB_TRY(cf_region_bytes(os, ngroups, extents, &data_bytes, &wsum_bytes));
  CFRegion& cf = g->cf;
  // the previous CF may still be read by queued kernels
  HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
  HPGB_TRY(cf.data.reserve(std::max<size_t>(data_bytes, 16)));
  HPGB_TRY(cf.wsum.reserve(std::max<size_t>(wsum_bytes, 16)));
  HPGB_TRY(cf.desc.reserve(std::max<size_t>(ngroups, 1) * sizeof(CFGroup)));
  cf.os = os;
  cf.extents.assign(ngroups, {0, 0, 0, 0});
  cf.groups.assign(ngroups, CFGroup{});
  cf.max_taps_x = cf.max_taps_y = cf.max_mueller = 0;

  DevBuf staging;
  size_t doff = 0, woff = 0;
  for (unsigned grp = 0; grp < ngroups; ++grp) {
    const unsigned* e = extents + 4 * grp;
    std::copy(e, e + 4, cf.extents[grp].begin());
    const GroupShape s = group_shape(os, e);
    float2* out = reinterpret_cast<float2*>(cf.data.as<char>() + doff);
    double2* ws = reinterpret_cast<double2*>(cf.wsum.as<char>() + woff);
    const long long nin = input_elems(layout, os, e);
    const float2* in = static_cast<const float2*>(values[grp]);
    if (!on_device && nin > 0) {
      HPGB_TRY(staging.reserve(size_t(nin) * sizeof(float2)));
      HPGB_CUDA_TRY(cudaMemcpyAsync(staging.ptr, values[grp],
                                    size_t(nin) * sizeof(float2),
                                    cudaMemcpyHostToDevice, g->stream));
      in = staging.as<float2>();
    }
    const size_t out_bytes =
        size_t(s.nslices) * size_t(s.slice_stride) * sizeof(float2);
    HPGB_CUDA_TRY(cudaMemsetAsync(out, 0, out_bytes, g->stream));
    LayoutArgs a;
    a.in = in;
    a.out = out;
    a.layout = layout;
    a.os = int(os);
    a.nfine = s.nfine;
    std::copy(e, e + 4, a.ext);
    a.taps_x = s.taps_x;
    a.taps_y = s.taps_y;
    a.nmueller = s.nmueller;
    a.ncube = s.ncube;
    a.plane_stride = s.plane_stride;
    a.slice_stride = s.slice_stride;
    a.total = s.nslices * s.nmueller * s.taps_x * s.taps_y;
    if (a.total > 0) {
      const int threads = 256;
      const long long blocks =
          std::min<long long>((a.total + threads - 1) / threads, 148LL * 64);
      cf_layout_kernel<<<unsigned(blocks), threads, 0, g->stream>>>(a);
      HPGB_CUDA_TRY(cudaGetLastError());
      ++g->launches;
      const long long warps = s.nslices * s.nmueller;
      const long long wblocks = (warps * 32 + threads - 1) / threads;
      cf_wsum_kernel<<<unsigned(wblocks), threads, 0, g->stream>>>(
          out, ws, s.nslices, s.nmueller, s.taps_x * s.taps_y, s.plane_stride,
          s.slice_stride);
      HPGB_CUDA_TRY(cudaGetLastError());
      ++g->launches;
    }
    if (!on_device) {
      // staging is reused by the next group: wait for this group's kernels
      HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    CFGroup& d = cf.groups[grp];
    d.data = out;
    d.wsum = ws;
    d.taps_x = s.taps_x;
    d.taps_y = s.taps_y;
    d.nmueller = s.nmueller;
    d.ncube = s.ncube;
    d.plane_stride = s.plane_stride;
    d.slice_stride = s.slice_stride;
    cf.max_taps_x = std::max(cf.max_taps_x, s.taps_x);
    cf.max_taps_y = std::max(cf.max_taps_y, s.taps_y);
    cf.max_mueller = std::max(cf.max_mueller, s.nmueller);
    doff += out_bytes;
    woff += size_t(s.nslices) * size_t(s.nmueller) * sizeof(double2);
  }
  if (ngroups > 0)
    HPGB_CUDA_TRY(cudaMemcpyAsync(cf.desc.ptr, cf.groups.data(),
                                  ngroups * sizeof(CFGroup),
                                  cudaMemcpyHostToDevice, g->stream));
  HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
  cf.set = true;
  return Status::ok();
}

Status copy_cf(hpgb_gridder* dst, const hpgb_gridder* src) {
  const CFRegion& s = src->cf;
  CFRegion& d = dst->cf;
  d.os = s.os;
  d.extents = s.extents;
  d.max_taps_x = s.max_taps_x;
  d.max_taps_y = s.max_taps_y;
  d.max_mueller = s.max_mueller;
  d.set = s.set;
  d.groups = s.groups;
  if (!s.set) return Status::ok();
  HPGB_TRY(d.data.reserve(s.data.bytes));
  HPGB_TRY(d.wsum.reserve(s.wsum.bytes));
  HPGB_TRY(d.desc.reserve(std::max<size_t>(s.groups.size(), 1) * sizeof(CFGroup)));
  HPGB_CUDA_TRY(cudaMemcpyAsync(d.data.ptr, s.data.ptr, s.data.bytes,
                                cudaMemcpyDeviceToDevice, dst->stream));
  HPGB_CUDA_TRY(cudaMemcpyAsync(d.wsum.ptr, s.wsum.ptr, s.wsum.bytes,
                                cudaMemcpyDeviceToDevice, dst->stream));
  for (size_t i = 0; i < d.groups.size(); ++i) {
    d.groups[i].data = reinterpret_cast<const float2*>(
        d.data.as<const char>() +
        (reinterpret_cast<const char*>(s.groups[i].data) - s.data.as<const char>()));
    d.groups[i].wsum = reinterpret_cast<const double2*>(
        d.wsum.as<const char>() +
        (reinterpret_cast<const char*>(s.groups[i].wsum) - s.wsum.as<const char>()));
  }
  if (!d.groups.empty())
    HPGB_CUDA_TRY(cudaMemcpyAsync(d.desc.ptr, d.groups.data(),
                                  d.groups.size() * sizeof(CFGroup),
                                  cudaMemcpyHostToDevice, dst->stream));
  HPGB_CUDA_TRY(cudaStreamSynchronize(dst->stream));
  return Status::ok();
}

}  // namespace hpgb
