// Tensor-memory-access (TMA) staging helpers for sm_100a: mbarrier
// handling and the tiled 4-D bulk tensor load, written as inline PTX.
//
// Rules the callers keep (checked on the host before a tensor map is made):
// the global base address is 16-byte aligned, every global stride is a
// multiple of 16 bytes, the innermost box extent times the element size is a
// multiple of 16 bytes, and the innermost start coordinate times the element
// size is a multiple of 16 bytes.  Loads are never multicast.  Every wait is
// bounded: a wait that runs out reports failure and the caller raises a bit
// of the device error word instead of spinning on.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace dn {

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

// retires an mbarrier whose every phase has completed, so that its shared
// memory can be initialised again (the next work item of a CTA)
__device__ __forceinline__ void mbar_inval(uint64_t* bar)
{
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" :: "r"(smem_u32(bar)) : "memory");
}

// makes the initialised mbarriers visible to the async proxy
__device__ __forceinline__ void mbar_init_fence()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// arrival of the issuing thread plus the byte count the transfer will deliver
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
  unsigned ok;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity to complete; false after about
// 2^18 unsuccessful polls (each poll may itself suspend the thread for a
// bounded, hardware-defined time), far beyond any transfer's latency.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity)
{
  for (int n = 0; n < (1 << 18); ++n)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) accesses of the same memory
__device__ __forceinline__ void fence_proxy_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Tiled 4-D load of one box of `map` at coordinates (c0 innermost .. c3)
// into shared memory at dst (128-byte aligned), completing on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2, int c3)
{
  asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
               " [%0], [%1, {%2, %3, %4, %5}], [%6];"
               :: "r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
                  "r"(smem_u32(bar))
               : "memory");
}

} // namespace dn
