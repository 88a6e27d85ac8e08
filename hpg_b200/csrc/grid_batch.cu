// grid_batch.cu -- one launch of the tiled kernel over the batches of many
// gridders (hpgb_grid_visibilities_batch): many independent grids of
// uneven sizes, each with its own CF set and batch, in one persistent
// launch, so that the device stays full however small each job is and the
// whole step is one kernel (and one CUDA graph).
//
// Every gridder's batch is sorted into uv tiles on its own buffers
// (tiles.cuh), with the tile side its own CF allows under the launch's
// common shared-memory plan; a small kernel then concatenates the gridders'
// tile-pass lists into one work list, each pass tagged with its gridder,
// and the tiled kernel reads each pass's grid, weights, CF, records, tile
// geometry and model tensor map from a job table in device memory
// (BatchJob).  The sorts run on the gridders' own streams, forked from the
// first gridder's stream and joined back before the launch, which runs
// there; the others' streams are ordered before and after the whole call.
// The gridders must share the
// number of polarizations and grid rows, the Mueller tables, the arithmetic
// form and (when degridding) whether a model is set.

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "tiled_kernel.cuh"

namespace hpgb {

using namespace tiled;

namespace {

struct ChunkSrc {
  const Chunk* chunks;
  const unsigned* num_chunks;
};

// The job table and the gridders' pass lists travel as the parameters of
// the kernel that places them (kernel parameters are copied at launch, and
// by value into a CUDA graph that captures the call): no host buffer has to
// outlive the call.  BatchJob entries are carried as raw 16-byte words.
struct BatchTable {
  int njobs;
  int pad[3];
  ChunkSrc src[kMaxBatchJobs];
  uint4 jobs[kMaxBatchJobs * sizeof(BatchJob) / 16];
};
static_assert(sizeof(BatchJob) % 16 == 0, "BatchJob is whole 16-byte words");
static_assert(sizeof(BatchTable) <= 32000, "kernel parameter limit");

// block j writes gridder j's job-table entry and copies its tile passes
// behind those of gridders < j, tagged with j; the last block writes the
// total
__global__ void place_batch_kernel(const __grid_constant__ BatchTable t,
                                   BatchJob* jobs, Chunk* out,
                                   unsigned* total) {
  const int j = blockIdx.x;
  constexpr int kWords = int(sizeof(BatchJob) / 16);
  uint4* dst = reinterpret_cast<uint4*>(jobs + j);
  for (int w = threadIdx.x; w < kWords; w += blockDim.x)
    dst[w] = t.jobs[j * kWords + w];
  unsigned off = 0;
  for (int i = 0; i < j; ++i) off += *t.src[i].num_chunks;
  const unsigned nj = *t.src[j].num_chunks;
  for (unsigned k = threadIdx.x; k < nj; k += blockDim.x) {
    Chunk c = t.src[j].chunks[k];
    c.pad = j;
    out[off + k] = c;
  }
  if (j == t.njobs - 1 && threadIdx.x == 0) *total = off + nj;
}

template <bool MIXED>
Status launch_batch_n(hpgb_gridder* g0, unsigned npol, const TiledParams& p,
                      int smem, const CUtensorMap& map) {
  switch (npol) {
    case 1: return launch_tiled_kernel<1, MIXED, true>(g0, p, smem, map);
    case 2: return launch_tiled_kernel<2, MIXED, true>(g0, p, smem, map);
    case 3: return launch_tiled_kernel<3, MIXED, true>(g0, p, smem, map);
    case 4: return launch_tiled_kernel<4, MIXED, true>(g0, p, smem, map);
    default: return Status::err(HPGB_ERROR_OTHER, "bad polarization count");
  }
}

}  // namespace

// One launch over the gridders gs[0..njobs) on gs[0]'s stream, with gs[0]'s
// buffers; a wait timeout is reported in `status`.
Status grid_batch_launch(hpgb_gridder* const* gs, size_t njobs,
                         void* const* d_vis, const size_t* nvis,
                         unsigned flags, unsigned* status) {
  hpgb_gridder* g0 = gs[0];
  const cudaStream_t st = g0->stream;
  const bool mixed = g0->precision == HPGB_PRECISION_MIXED;
  BatchShape shape;
  size_t total = 0;
  for (size_t j = 0; j < njobs; ++j) {
    const hpgb_gridder* g = gs[j];
    for (const CFGroup& G : g->cf.groups)
      shape.max_plane_bytes = std::max(shape.max_plane_bytes, G.plane_stride * 8);
    const int taps = std::max(g->cf.max_taps_x, g->cf.max_taps_y);
    shape.max_taps = std::max(shape.max_taps, taps);
    shape.jobs.push_back({(long long)g->grid_size[0], (long long)g->grid_size[1],
                          (long long)g->grid_size[3], taps, (long long)nvis[j]});
    total += nvis[j];
  }
  if (total == 0) return Status::ok();
  if (total > size_t(0x7fffffff))
    return Status::err(HPGB_ERROR_EXCESSIVE_NUMBER_VISIBILITIES,
                       "too many visibilities for one launch");
  const Plan plan = make_plan(g0, flags, mixed, total, &shape);
  if (!plan.ok)
    return Status::err(HPGB_ERROR_OTHER,
                       "the tiled kernel cannot take this batch: " + plan.why);
  const int R = plan.R;
  if (njobs > size_t(kMaxBatchJobs))
    return Status::err(HPGB_ERROR_OTHER, "more gridders than one launch takes");
  std::vector<BatchJob> jobs(njobs);
  std::vector<ChunkSrc> srcs(njobs);
  size_t max_chunks = 0;
  const bool model = plan.p.do_degrid && plan.p.has_model;
  // every model's rows must start on 16-byte boundaries for its tensor map
  // (an odd grid width in the mixed form's FP32 copy does not)
  if (model)
    for (size_t j = 0; j < njobs; ++j)
      if ((2 * size_t(gs[j]->grid_size[0]) * (mixed ? 4 : 8)) % 16 != 0)
        return Status::err(HPGB_ERROR_OTHER,
                           "gridder " + std::to_string(j) +
                               ": model row pitch not a 16-byte multiple "
                               "(odd grid width in the mixed form)");
  // Each gridder's tile sort (and FP32 model copy) runs on the gridder's own
  // stream, forked from st and joined back before the launch, so that the
  // gridders' short preparation kernels overlap one another instead of
  // queueing one after another on st.  Their buffers are the gridder's own.
  cudaEvent_t fork = nullptr;
  HPGB_CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  std::vector<cudaEvent_t> joins;
  struct Release {
    cudaEvent_t& f;
    std::vector<cudaEvent_t>& j;
    ~Release() {
      cudaEventDestroy(f);
      for (cudaEvent_t e : j) cudaEventDestroy(e);
    }
  } release{fork, joins};
  HPGB_CUDA_TRY(cudaEventRecord(fork, st));
  for (size_t j = 0; j < njobs; ++j) {
    hpgb_gridder* g = gs[j];
    BatchJob& b = jobs[j];
    std::memset(&b, 0, sizeof(b));
    const cudaStream_t js = g->stream;
    if (js != st) HPGB_CUDA_TRY(cudaStreamWaitEvent(js, fork, 0));
    const int taps = std::max(g->cf.max_taps_x, g->cf.max_taps_y);
    // the largest tile this gridder's CF allows in the launch's region
    b.T = R - taps + 1;
    b.nx = int(g->grid_size[0]);
    b.ny = int(g->grid_size[1]);
    b.ntx = (b.nx + b.T - 1) / b.T;
    b.nty = (b.ny + b.T - 1) / b.T;
    b.cf = g->cf.data.as<const float2>();
    b.grid = g->grid.as<double2>();
    b.weights = g->weights.as<double>();
    b.records = static_cast<unsigned char*>(d_vis[j]);
    if (nvis[j] > 0) {
      TilePrep prep;
      HPGB_TRY(prepare_tiles(g, d_vis[j], nvis[j], b.T, b.ntx, b.nty, plan.K,
                             &prep, js));
      b.descs = prep.descs;
      b.srefs = prep.srefs;
      srcs[j] = ChunkSrc{prep.chunks, prep.num_chunks};
      max_chunks += prep.max_chunks;
    } else {
      // no passes: point at a zero count
      srcs[j] = ChunkSrc{nullptr, g->vb.counters.as<unsigned>() + 3};
      HPGB_CUDA_TRY(cudaMemsetAsync(g->vb.counters.as<unsigned>() + 3, 0,
                                    sizeof(unsigned), js));
    }
    if (model) HPGB_TRY(encode_model_map(g, mixed, R, &b.model_map, js));
    if (js != st) {
      cudaEvent_t e = nullptr;
      HPGB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      joins.push_back(e);
      HPGB_CUDA_TRY(cudaEventRecord(e, js));
      HPGB_CUDA_TRY(cudaStreamWaitEvent(st, e, 0));
    }
  }
  // job table and the combined work list, in g0's buffers
  VisBuffers& vb = g0->vb;
  HPGB_TRY(vb.batch_jobs.reserve(njobs * sizeof(BatchJob)));
  HPGB_TRY(vb.batch_chunks.reserve(std::max<size_t>(max_chunks, 1) * sizeof(Chunk)));
  std::unique_ptr<BatchTable> table(new BatchTable);
  std::memset(table.get(), 0, sizeof(BatchTable));
  table->njobs = int(njobs);
  std::memcpy(table->src, srcs.data(), njobs * sizeof(ChunkSrc));
  std::memcpy(table->jobs, jobs.data(), njobs * sizeof(BatchJob));
  unsigned* total_chunks = vb.counters.as<unsigned>() + 4;
  place_batch_kernel<<<unsigned(njobs), 128, 0, st>>>(
      *table, vb.batch_jobs.as<BatchJob>(), vb.batch_chunks.as<Chunk>(),
      total_chunks);
  HPGB_CUDA_TRY(cudaGetLastError());
  ++g0->launches;
  TiledParams p = plan.p;
  p.jobs = vb.batch_jobs.as<const BatchJob>();
  p.chunks = vb.batch_chunks.as<Chunk>();
  p.num_chunks = total_chunks;
  p.rec_stride = int(visdata_size(g0->npol));
  p.status = status;
  p.wait_limit_ns = g0->wait_limit_ns;
  p.withhold_vis = g0->withhold_vis;
  CUtensorMap unused;
  std::memset(&unused, 0, sizeof(unused));
  if (mixed) return launch_batch_n<true>(g0, g0->npol, p, plan.smem, unused);
  return launch_batch_n<false>(g0, g0->npol, p, plan.smem, unused);
}

// The gridders are grouped by their widest CF (taps up to 17, 33, 65, more)
// and by the tile side their own plan would take: one launch's plan -- ring
// depth and tile side -- is sized for its widest CF and its gridders' tiles
// together, so a gridder with narrow CFs in a launch with a wide one would
// get a shallow ring and small tiles, and a sparse gridder in a launch with
// dense ones a deep ring and passes of few visibilities (measured on the
// 64-job benchmark: the four-polarization class 229 -> 217 ms against
// grouping by support alone).  Each group takes one launch on the stream of
// its first gridder, forked from and joined back to gs[0]'s stream, so that
// the groups' launches overlap where the device has room.
Status grid_batch_tiled(hpgb_gridder* const* gs, size_t njobs,
                        void* const* d_vis, const size_t* nvis,
                        unsigned flags) {
  const bool mixed = gs[0]->precision == HPGB_PRECISION_MIXED;
  // every model's rows must start on 16-byte boundaries for its tensor map
  // (an odd grid width in the mixed form's FP32 copy does not); checked for
  // every gridder before the grouping, whatever its batch size
  if ((flags & HPGB_DO_DEGRID) && gs[0]->has_model && mixed)
    for (size_t j = 0; j < njobs; ++j)
      if ((2 * size_t(gs[j]->grid_size[0]) * 4) % 16 != 0)
        return Status::err(HPGB_ERROR_OTHER,
                           "gridder " + std::to_string(j) +
                               ": model row pitch not a 16-byte multiple "
                               "(odd grid width in the mixed form)");
  auto taps_class = [](const hpgb_gridder* g) {
    const int t = std::max(g->cf.max_taps_x, g->cf.max_taps_y);
    return t <= 17 ? 0 : t <= 33 ? 1 : t <= 65 ? 2 : 3;
  };
  std::map<std::pair<int, int>, std::vector<size_t>> groups;
  for (size_t j = 0; j < njobs; ++j) {
    const Plan own = nvis[j] > 0 ? make_plan(gs[j], flags, mixed, nvis[j], nullptr)
                                 : Plan();
    groups[{taps_class(gs[j]), own.ok ? own.R : 0}].push_back(j);
  }
  std::vector<std::vector<size_t>> cls;
  for (auto& kv : groups) cls.push_back(kv.second);
  const cudaStream_t st = gs[0]->stream;
  unsigned* status = gs[0]->vb.counters.as<unsigned>();
  const int used = int(cls.size());
  if (used <= 1) return grid_batch_launch(gs, njobs, d_vis, nvis, flags, status);
  cudaEvent_t fork = nullptr;
  HPGB_CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  std::vector<cudaEvent_t> joins;
  auto cleanup = [&]() {
    cudaEventDestroy(fork);
    for (cudaEvent_t e : joins) cudaEventDestroy(e);
  };
  Status result = Status::ok();
  cudaError_t ce = cudaEventRecord(fork, st);
  for (auto& c : cls) {
    if (c.empty() || ce != cudaSuccess || !result) continue;
    std::vector<hpgb_gridder*> sub;
    std::vector<void*> sv;
    std::vector<size_t> sn;
    for (size_t j : c) {
      sub.push_back(gs[j]);
      sv.push_back(d_vis[j]);
      sn.push_back(nvis[j]);
    }
    const cudaStream_t cs = sub[0]->stream;
    if (cs != st) ce = cudaStreamWaitEvent(cs, fork, 0);
    if (ce != cudaSuccess) break;
    result = grid_batch_launch(sub.data(), sub.size(), sv.data(), sn.data(),
                               flags, status);
    if (cs != st) {
      cudaEvent_t e = nullptr;
      ce = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      if (ce != cudaSuccess) break;
      joins.push_back(e);
      ce = cudaEventRecord(e, cs);
      if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st, e, 0);
    }
  }
  cleanup();
  if (ce != cudaSuccess && result)
    result = Status::err(HPGB_ERROR_OTHER, cudaGetErrorString(ce));
  return result;
}

}  // namespace hpgb
