// tma.cuh -- Blackwell bulk-copy (TMA) and mbarrier primitives as inline PTX.
//
// Loads land in shared memory and complete on an mbarrier with a transaction
// byte count; stores are bulk groups.  Every wait on an mbarrier is bounded:
// after kMaxSpins polls the waiting thread records the failure in a global
// status word and returns false, so a kernel never spins forever.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace gpe {

constexpr uint32_t kMaxSpins = 1u << 22;
enum : uint32_t { kErrTmaTimeout = 1u };

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

// Programmatic dependent launch.  pdl_trigger lets the next kernel of the
// stream be scheduled once every CTA of this grid has started; pdl_wait
// returns once the previous kernel has completed and its memory is visible.
// Every step kernel calls both before its first global-memory access, so a
// kernel launched with the attribute can occupy SMs freed by the tail of its
// predecessor without reading or writing anything early.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Asynchronous 8-byte global -> shared copies (cp.async); cp_async_wait_all
// returns once all of this thread's copies have landed (each thread then
// still needs a barrier before others read them).
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
   asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// orders this thread's generic-proxy shared-memory writes before later
// async-proxy (bulk copy) reads of the same memory
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
   uint32_t ok;
   asm volatile(
       "{\n\t.reg .pred p;\n\t"
       "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
       "selp.u32 %0, 1, 0, p;\n\t}"
       : "=r"(ok)
       : "r"(smem_u32(bar)), "r"(parity)
       : "memory");
   return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
   asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Named barrier 1 over the nthreads consumer threads of a warp-specialised
// CTA (the producer warp never takes part).
__device__ __forceinline__ void consumer_sync(int nthreads) {
   asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Consumer barrier that also ORs a flag across the consumer threads.
__device__ __forceinline__ bool consumer_any(bool flag, int nthreads) {
   uint32_t r;
   asm volatile(
       "{\n\t.reg .pred p, q;\n\t"
       "setp.ne.u32 p, %1, 0;\n\t"
       "bar.red.or.pred q, 1, %2, p;\n\t"
       "selp.u32 %0, 1, 0, q;\n\t}"
       : "=r"(r)
       : "r"((uint32_t) flag), "r"(nthreads)
       : "memory");
   return r != 0;
}

// Bounded wait for phase `parity` of `bar`: at most `spins` polls.  Returns
// false (and sets bit kErrTmaTimeout in *err) when the phase did not complete
// in time.
__device__ __forceinline__ bool mbar_wait_n(uint64_t *bar, uint32_t parity, uint32_t *err, uint32_t spins) {
   for (uint32_t i = 0; i < spins; i++)
      if (mbar_try_wait(bar, parity)) return true;
   if (err) atomicOr(err, kErrTmaTimeout);
   return false;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t *err) {
   return mbar_wait_n(bar, parity, err, kMaxSpins);
}

// 3D tiled tensor load global -> shared, completing on bar.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar) {
   asm volatile(
       "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
       ::"r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
       : "memory");
}

// 3D tiled tensor store shared -> global (out-of-range elements are clipped).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, int c0, int c1, int c2, const void *src) {
   asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];"
                ::"l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(src))
                : "memory");
}

// Contiguous bulk copy global -> shared (16-byte aligned, size % 16 == 0).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
   asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                : "memory");
}

// Contiguous bulk copy shared -> global.
__device__ __forceinline__ void bulk_store(void *dst, const void *src, uint32_t bytes) {
   asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)), "r"(bytes)
                : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// all committed bulk stores of this thread have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// all committed bulk stores of this thread are complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// all but the newest N committed bulk-store groups have finished reading
// shared memory (N = pipeline stages - 2, an immediate)
template <int N> __device__ __forceinline__ void bulk_wait_read() {
   asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// In an S-stage pipeline (one store group per tile): the stage about to be
// reloaded has been read out by its store.
template <int S> __device__ __forceinline__ void wait_stage_free() {
   if constexpr (S == 2) bulk_wait_read<0>();
   else if constexpr (S == 3) bulk_wait_read<1>();
   else bulk_wait_read<2>();
}

}  // namespace gpe
