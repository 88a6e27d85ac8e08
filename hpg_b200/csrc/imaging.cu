// imaging.cu -- elementwise passes over the grid and the cuFFT call:
// normalize_by_weights and norm scaling (GridNormalizer,
// src/hpg_core.hpp:1829-1890), quadrant shift / cyclic rotation
// (GridShifter, src/hpg_core.hpp:2303-2542), the 2-D FFT of every
// (mrow, cube) plane (FFT<Cuda>, src/hpg_core.hpp:2192-2276), and the
// Left/Right layout conversions of GridValueArray / GridWeightArray copies.
//
// All passes are HBM-bound streams over complex<double>: each thread handles
// 16-byte elements with coalesced loads and stores, grids sized to a few
// waves of the 148 SMs.

#include <algorithm>

#include "gridder.cuh"

namespace hpgb {

namespace {

inline unsigned blocks_for(size_t n, int threads) {
  const size_t b = (n + threads - 1) / threads;
  return unsigned(std::min<size_t>(std::max<size_t>(b, 1), 148 * 32));
}

// grid(x,y,mrow,cube) /= (wfactor * weights(mrow,cube))
__global__ void normalize_weights_kernel(double2* __restrict__ grid,
                                         const double* __restrict__ weights,
                                         size_t plane, size_t nplanes,
                                         double wfactor) {
  const size_t n = plane * nplanes;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const double d = __dmul_rn(wfactor, weights[i / plane]);
    double2 v = grid[i];
    v.x = __ddiv_rn(v.x, d);
    v.y = __ddiv_rn(v.y, d);
    grid[i] = v;
  }
}

// grid *= 1/norm
__global__ void scale_kernel(double2* __restrict__ grid, size_t n, double inv) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    double2 v = grid[i];
    v.x = __dmul_rn(v.x, inv);
    v.y = __dmul_rn(v.y, inv);
    grid[i] = v;
  }
}

// both sides even: swap quadrants (x,y)<->(x+mx,y+my), (x+mx,y)<->(x,y+my)
__global__ void shift_even_kernel(double2* __restrict__ grid, int nx, int ny,
                                  size_t nplanes) {
  const int mx = nx / 2, my = ny / 2;
  const size_t quarter = size_t(mx) * my;
  const size_t plane = size_t(nx) * ny;
  const size_t n = quarter * nplanes;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const size_t p = i / quarter;
    const size_t r = i - p * quarter;
    const int y = int(r / mx), x = int(r - size_t(y) * mx);
    double2* pl = grid + p * plane;
    const size_t a = size_t(y) * nx + x, b = size_t(y + my) * nx + (x + mx);
    const size_t c = size_t(y) * nx + (x + mx), d = size_t(y + my) * nx + x;
    const double2 va = pl[a], vb = pl[b], vc = pl[c], vd = pl[d];
    pl[a] = vb;
    pl[b] = va;
    pl[c] = vd;
    pl[d] = vc;
  }
}

// per-plane factor of the imaging tail: 1 / (wfactor * weight) then 1 / norm
__device__ __forceinline__ double2 tail_scale(double2 v, const double* weights,
                                              size_t p, double wfactor,
                                              double inv_norm) {
  const double d = __dmul_rn(wfactor, weights[p]);
  v.x = __dmul_rn(__ddiv_rn(v.x, d), inv_norm);
  v.y = __dmul_rn(__ddiv_rn(v.y, d), inv_norm);
  return v;
}

// shift_even_kernel with the imaging tail's per-plane scaling folded in
__global__ void shift_even_scale_kernel(double2* __restrict__ grid, int nx,
                                        int ny, size_t nplanes,
                                        const double* __restrict__ weights,
                                        double wfactor, double inv_norm) {
  const int mx = nx / 2, my = ny / 2;
  const size_t quarter = size_t(mx) * my;
  const size_t plane = size_t(nx) * ny;
  const size_t n = quarter * nplanes;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const size_t p = i / quarter;
    const size_t r = i - p * quarter;
    const int y = int(r / mx), x = int(r - size_t(y) * mx);
    double2* pl = grid + p * plane;
    const size_t a = size_t(y) * nx + x, b = size_t(y + my) * nx + (x + mx);
    const size_t c = size_t(y) * nx + (x + mx), d = size_t(y + my) * nx + x;
    const double2 va = pl[a], vb = pl[b], vc = pl[c], vd = pl[d];
    pl[a] = tail_scale(vb, weights, p, wfactor, inv_norm);
    pl[b] = tail_scale(va, weights, p, wfactor, inv_norm);
    pl[c] = tail_scale(vd, weights, p, wfactor, inv_norm);
    pl[d] = tail_scale(vc, weights, p, wfactor, inv_norm);
  }
}

// roll_kernel with the imaging tail's per-plane scaling folded in
__global__ void roll_scale_kernel(const double2* __restrict__ in,
                                  double2* __restrict__ out, int nx, int ny,
                                  int sx, int sy, size_t nplanes,
                                  const double* __restrict__ weights,
                                  double wfactor, double inv_norm) {
  const size_t plane = size_t(nx) * ny;
  const size_t n = plane * nplanes;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const size_t p = i / plane;
    const size_t r = i - p * plane;
    const int y = int(r / nx), x = int(r - size_t(y) * nx);
    int xs = x - sx, ys = y - sy;
    xs = ((xs % nx) + nx) % nx;
    ys = ((ys % ny) + ny) % ny;
    out[i] = tail_scale(in[p * plane + size_t(ys) * nx + xs], weights, p,
                        wfactor, inv_norm);
  }
}

// general sizes: out(x, y) = in(x - sx mod nx, y - sy mod ny)
__global__ void roll_kernel(const double2* __restrict__ in,
                            double2* __restrict__ out, int nx, int ny, int sx,
                            int sy, size_t nplanes) {
  const size_t plane = size_t(nx) * ny;
  const size_t n = plane * nplanes;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const size_t p = i / plane;
    const size_t r = i - p * plane;
    const int y = int(r / nx), x = int(r - size_t(y) * nx);
    int xs = x - sx, ys = y - sy;
    xs = ((xs % nx) + nx) % nx;
    ys = ((ys % ny) + ny) % ny;
    out[i] = in[p * plane + size_t(ys) * nx + xs];
  }
}

// Left [x,y,mrow,cube] <-> Right (cube fastest) element copy
__global__ void layout_kernel(const double2* __restrict__ src,
                              double2* __restrict__ dst, unsigned nx,
                              unsigned ny, unsigned nr, unsigned nc,
                              bool to_left) {
  const size_t n = size_t(nx) * ny * nr * nc;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    size_t t = i;
    const unsigned x = unsigned(t % nx); t /= nx;
    const unsigned y = unsigned(t % ny); t /= ny;
    const unsigned r = unsigned(t % nr); t /= nr;
    const unsigned c = unsigned(t);
    const size_t right = ((size_t(x) * ny + y) * nr + r) * nc + c;
    if (to_left)
      dst[i] = src[right];
    else
      dst[right] = src[i];
  }
}

}  // namespace

Status normalize_by_weights(hpgb_gridder* g, double wfactor) {
  const size_t plane = size_t(g->grid_size[0]) * g->grid_size[1];
  const size_t np = size_t(g->grid_size[2]) * g->grid_size[3];
  normalize_weights_kernel<<<blocks_for(plane * np, 256), 256, 0, g->stream>>>(
      g->grid.as<double2>(), g->weights.as<double>(), plane, np, wfactor);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  return Status::ok();
}

Status scale_grid(hpgb_gridder* g, double2* grid, double norm) {
  const size_t n = g->grid_elems();
  const double inv = 1.0 / norm;
  scale_kernel<<<blocks_for(n, 256), 256, 0, g->stream>>>(grid, n, inv);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  return Status::ok();
}

Status shift(hpgb_gridder* g, double2* grid, int direction) {
  const int nx = int(g->grid_size[0]), ny = int(g->grid_size[1]);
  const size_t np = size_t(g->grid_size[2]) * g->grid_size[3];
  if (nx % 2 == 0 && ny % 2 == 0) {
    const size_t n = size_t(nx / 2) * (ny / 2) * np;
    if (n == 0) return Status::ok();
    shift_even_kernel<<<blocks_for(n, 256), 256, 0, g->stream>>>(grid, nx, ny, np);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
    return Status::ok();
  }
  // FORWARD rolls each axis by +n/2, BACKWARD by -(n/2): the net effect of
  // the reference's swap chains (src/hpg_core.hpp:2356-2540)
  const int sx = direction == HPGB_SHIFT_FORWARD ? nx / 2 : -(nx / 2);
  const int sy = direction == HPGB_SHIFT_FORWARD ? ny / 2 : -(ny / 2);
  const size_t n = g->grid_elems();
  DevBuf tmp;
  HPGB_TRY(tmp.reserve(n * sizeof(double2)));
  roll_kernel<<<blocks_for(n, 256), 256, 0, g->stream>>>(
      grid, tmp.as<double2>(), nx, ny, sx, sy, np);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  HPGB_CUDA_TRY(cudaMemcpyAsync(grid, tmp.ptr, n * sizeof(double2),
                                cudaMemcpyDeviceToDevice, g->stream));
  HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return Status::ok();
}

// The imaging tail normalize_by_weights(wfactor) -> apply_grid_fft(norm,
// sign, in place) -> shift_grid(direction) (src/hpg_runtime.hpp:1293-1441)
// as the FFT followed by one pass: the normalisation is a factor per
// (mrow, cube) plane and the FFT transforms each plane linearly, so the
// factor is applied after the FFT, together with 1/norm, in the pass that
// shifts (results equal the three calls' to FP64 rounding).
Status image_tail(hpgb_gridder* g, double wfactor, double norm, int sign,
                  int direction) {
  HPGB_TRY(fft(g, g->grid, 1.0, sign, true));
  const int nx = int(g->grid_size[0]), ny = int(g->grid_size[1]);
  const size_t np = size_t(g->grid_size[2]) * g->grid_size[3];
  const double inv_norm = 1.0 / norm;
  double2* grid = g->grid.as<double2>();
  const double* w = g->weights.as<const double>();
  if (nx % 2 == 0 && ny % 2 == 0) {
    const size_t n = size_t(nx / 2) * (ny / 2) * np;
    if (n == 0) return Status::ok();
    shift_even_scale_kernel<<<blocks_for(n, 256), 256, 0, g->stream>>>(
        grid, nx, ny, np, w, wfactor, inv_norm);
    HPGB_CUDA_TRY(cudaGetLastError());
    ++g->launches;
    return Status::ok();
  }
  const int sx = direction == HPGB_SHIFT_FORWARD ? nx / 2 : -(nx / 2);
  const int sy = direction == HPGB_SHIFT_FORWARD ? ny / 2 : -(ny / 2);
  const size_t n = g->grid_elems();
  DevBuf tmp;
  HPGB_TRY(tmp.reserve(n * sizeof(double2)));
  roll_scale_kernel<<<blocks_for(n, 256), 256, 0, g->stream>>>(
      grid, tmp.as<double2>(), nx, ny, sx, sy, np, w, wfactor, inv_norm);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  HPGB_CUDA_TRY(cudaMemcpyAsync(grid, tmp.ptr, n * sizeof(double2),
                                cudaMemcpyDeviceToDevice, g->stream));
  HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return Status::ok();
}

static const char* cufft_msg(cufftResult r) {
  switch (r) {
    case CUFFT_SUCCESS: return "success";
    case CUFFT_INVALID_PLAN: return "invalid plan";
    case CUFFT_ALLOC_FAILED: return "allocation failed";
    case CUFFT_INVALID_VALUE: return "invalid value";
    case CUFFT_INTERNAL_ERROR: return "internal error";
    case CUFFT_EXEC_FAILED: return "exec failed";
    case CUFFT_SETUP_FAILED: return "setup failed";
    case CUFFT_INVALID_SIZE: return "invalid size";
    default: return "cufft error";
  }
}

Status fft(hpgb_gridder* g, DevBuf& grid, double norm, int sign,
           bool in_place) {
  const int nx = int(g->grid_size[0]), ny = int(g->grid_size[1]);
  const int batch = int(g->grid_size[2] * g->grid_size[3]);
  const auto key = std::make_tuple(nx, ny, batch);
  cufftHandle plan;
  auto it = g->fft_plans.find(key);
  if (it == g->fft_plans.end()) {
    // planes are contiguous, x fastest: n = {ny, nx} (src/hpg_core.hpp:2209)
    int n[2] = {ny, nx};
    cufftResult r =
        cufftPlanMany(&plan, 2, n, nullptr, 1, nx * ny, nullptr, 1, nx * ny,
                      CUFFT_Z2Z, batch);
    if (r != CUFFT_SUCCESS)
      return Status::err(HPGB_ERROR_OTHER,
                         std::string("cufftPlanMany: ") + cufft_msg(r));
    g->fft_plans[key] = plan;
  } else {
    plan = it->second;
  }
  cufftResult r = cufftSetStream(plan, g->stream);
  if (r != CUFFT_SUCCESS)
    return Status::err(HPGB_ERROR_OTHER,
                       std::string("cufftSetStream: ") + cufft_msg(r));
  const int dir = sign == HPGB_FFT_NEGATIVE ? CUFFT_FORWARD : CUFFT_INVERSE;
  double2* src = grid.as<double2>();
  if (in_place) {
    r = cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(src),
                     reinterpret_cast<cufftDoubleComplex*>(src), dir);
  } else {
    // the reference transforms into a newly allocated grid
    // (src/hpg_runtime.hpp:1331-1346)
    DevBuf fresh;
    HPGB_TRY(fresh.reserve(g->grid_elems() * sizeof(double2)));
    r = cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(src),
                     reinterpret_cast<cufftDoubleComplex*>(fresh.as<double2>()),
                     dir);
    if (r == CUFFT_SUCCESS) {
      HPGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
      std::swap(grid.ptr, fresh.ptr);
      std::swap(grid.bytes, fresh.bytes);
    }
  }
  if (r != CUFFT_SUCCESS)
    return Status::err(HPGB_ERROR_OTHER,
                       std::string("cufftExecZ2Z: ") + cufft_msg(r));
  if (norm != 1) HPGB_TRY(scale_grid(g, grid.as<double2>(), norm));
  return Status::ok();
}

void release_fft_plans(hpgb_gridder* g) {
  for (auto& kv : g->fft_plans) cufftDestroy(kv.second);
  g->fft_plans.clear();
}

Status to_layout(hpgb_gridder* g, const double2* src, double2* dst,
                 int layout, bool to_device_layout, const unsigned* ext) {
  const size_t n = size_t(ext[0]) * ext[1] * ext[2] * ext[3];
  if (n == 0) return Status::ok();
  if (layout == HPGB_LAYOUT_LEFT) {
    HPGB_CUDA_TRY(cudaMemcpyAsync(dst, src, n * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, g->stream));
    return Status::ok();
  }
  layout_kernel<<<blocks_for(n, 256), 256, 0, g->stream>>>(
      src, dst, ext[0], ext[1], ext[2], ext[3], to_device_layout);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g->launches;
  return Status::ok();
}

Status weights_to_layout(hpgb_gridder* g, const double* src, double* dst,
                         int layout) {
  const unsigned nr = g->grid_size[2], nc = g->grid_size[3];
  if (layout == HPGB_LAYOUT_LEFT) {
    std::copy(src, src + size_t(nr) * nc, dst);
  } else {
    for (unsigned c = 0; c < nc; ++c)
      for (unsigned r = 0; r < nr; ++r)
        dst[size_t(r) * nc + c] = src[size_t(c) * nr + r];
  }
  return Status::ok();
}

}  // namespace hpgb
