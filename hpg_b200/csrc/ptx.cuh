// ptx.cuh -- thin wrappers over the sm_90+/sm_100a PTX used by the tiled
// kernel: mbarriers (with bounded waits), bulk and tensor TMA copies into
// shared memory, shared-memory loads and stores at 32-bit addresses and
// distributed-shared-memory access within a thread-block cluster.  No
// multicast form is used anywhere.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace hpgb {
namespace ptx {

__device__ __forceinline__ uint32_t smem(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem(bar)),
               "r"(bytes)
               : "memory");
}

// arrive on the mbarrier at the same shared-memory offset in CTA `rank` of
// this cluster, with release semantics at cluster scope (orders this
// thread's earlier shared::cluster stores before the arrival)
__device__ __forceinline__ void mbar_arrive_remote(uint64_t* bar,
                                                   uint32_t rank) {
  uint32_t remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
               : "=r"(remote)
               : "r"(smem(bar)), "r"(rank));
  asm volatile(
      "mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(
          remote)
      : "memory");
}

// Waits for the completion of the mbarrier phase with the given parity.
// Every lane of the calling warp waits (the warp stays converged).  After a
// first plain test, each try_wait carries a suspend-time hint, so the warp
// sleeps in hardware until the phase completes (or the hint runs out)
// instead of spinning.  The wait is bounded by the global timer: after the
// CTA's wait limit it sets the CTA-wide abort flag and returns false, and
// the caller records the timeout instead of hanging.
constexpr uint32_t kSuspendHintNs = 20000;
constexpr uint64_t kWaitLimitNs = 500000000ull;  // default limit: 0.5 s

// The CTA's wait-control block in shared memory: the abort flag, a count of
// the tensor copies issued (for the drain before exit), then (8 bytes in)
// the wait limit in nanoseconds.  Waits take the flag's address.
struct WaitCtl {
  int flag;
  int copies;
  unsigned long long limit_ns;
};

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
      "selp.u32 %0, 1, 0, p; }"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ bool mbar_try_suspend(uint32_t a, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, "
      "%3; selp.u32 %0, 1, 0, p; }"
      : "=r"(done)
      : "r"(a), "r"(parity), "r"(kSuspendHintNs)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ bool mbar_try_cluster(uint32_t a, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.acquire.cluster.shared::cta."
      "b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ bool mbar_try_cluster_suspend(uint32_t a,
                                                         uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.acquire.cluster.shared::cta."
      "b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
      : "=r"(done)
      : "r"(a), "r"(parity), "r"(kSuspendHintNs)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ uint64_t wait_limit(volatile int* abort) {
  return *reinterpret_cast<volatile unsigned long long*>(
      reinterpret_cast<volatile char*>(abort) + 8);
}

// `abort` is the flag of the CTA's WaitCtl block: a wait that gives up sets
// it, and every later wait returns false at once, so a broken pipeline ends
// quickly with an error status instead of timing out wait after wait.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          volatile int* abort) {
  const uint32_t a = smem(bar);
  if (mbar_try(a, parity)) return true;
  const uint64_t t0 = global_ns();
  const uint64_t limit = wait_limit(abort);
  for (;;) {
    if (mbar_try_suspend(a, parity)) return true;
    if (*abort) return false;
    if (global_ns() - t0 > limit) break;
  }
  *abort = 1;
  return false;
}

// acquire at cluster scope, for barriers that remote CTAs complete
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar,
                                                  uint32_t parity,
                                                  volatile int* abort) {
  const uint32_t a = smem(bar);
  if (mbar_try_cluster(a, parity)) return true;
  const uint64_t t0 = global_ns();
  const uint64_t limit = wait_limit(abort);
  for (;;) {
    if (mbar_try_cluster_suspend(a, parity)) return true;
    if (*abort) return false;
    if (global_ns() - t0 > limit) break;
  }
  *abort = 1;
  return false;
}

// Wait for a phase whose transfer was issued (a bulk copy into this CTA's
// shared memory), ignoring the abort flag: used before the CTA exits so
// that no copy still lands in memory the CTA no longer owns.  Bounded by the
// wait limit; returns false if it ran out.
__device__ __forceinline__ bool mbar_drain(uint64_t* bar, uint32_t parity,
                                           volatile int* abort) {
  const uint32_t a = smem(bar);
  if (mbar_try(a, parity)) return true;
  const uint64_t t0 = global_ns();
  const uint64_t limit = wait_limit(abort);
  for (;;) {
    if (mbar_try_suspend(a, parity)) return true;
    if (global_ns() - t0 > limit) return false;
  }
}

// warp-uniform read of a shared-memory flag (lane 0's view)
__device__ __forceinline__ bool warp_flag(volatile int* flag) {
  return __shfl_sync(0xffffffffu, *flag, 0) != 0;
}

// shared-memory loads and stores at 32-bit shared-window addresses
__device__ __forceinline__ float2 lds_f2(uint32_t a) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];"
               : "=f"(v.x), "=f"(v.y)
               : "r"(a));
  return v;
}

__device__ __forceinline__ double2 lds_d2(uint32_t a) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
               : "=d"(v.x), "=d"(v.y)
               : "r"(a));
  return v;
}

__device__ __forceinline__ void sts_f2(uint32_t a, float2 v) {
  asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x),
               "f"(v.y));
}

__device__ __forceinline__ void sts_d2(uint32_t a, double2 v) {
  asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.x),
               "d"(v.y));
}


// bulk copy global -> this CTA's shared memory, completion counted in bytes
// on bar; dst, src and bytes are 16-byte multiples
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src,
                                        uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], "
      "[%1], %2, [%3];" ::"r"(smem(dst)),
      "l"(src), "r"(bytes), "r"(smem(bar))
      : "memory");
}

// 3-D tiled tensor load (no multicast); c0 is the innermost coordinate
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map,
                                            int c0, int c1, int c2,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_"
      "tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2),
      "r"(smem(bar))
      : "memory");
}

// store a double into CTA `rank`'s shared memory at the offset of p
__device__ __forceinline__ void st_cluster_f64(double* p, uint32_t rank,
                                               double v) {
  uint32_t remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
               : "=r"(remote)
               : "r"(smem(p)), "r"(rank));
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(remote), "d"(v)
               : "memory");
}

// asynchronous store of a double into CTA `rank`'s shared memory; its
// completion is counted (8 bytes) on the mbarrier at bar's offset in that CTA
__device__ __forceinline__ void st_async_f64(double* p, uint32_t rank, double v,
                                             uint64_t* bar) {
  uint32_t rp, rb;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
               : "=r"(rp)
               : "r"(smem(p)), "r"(rank));
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
               : "=r"(rb)
               : "r"(smem(bar)), "r"(rank));
  asm volatile(
      "st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, "
      "[%2];" ::"r"(rp),
      "d"(v), "r"(rb)
      : "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint32_t num_clusters_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}

// full barrier over every thread of every CTA of the cluster
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// named barrier over `count` threads (multiple of 32)
__device__ __forceinline__ void named_sync(uint32_t id, uint32_t count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

}  // namespace ptx
}  // namespace hpgb
