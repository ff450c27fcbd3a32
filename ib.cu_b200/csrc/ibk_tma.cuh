// Tensor-memory-accelerator (TMA) staging of grid boxes into shared memory.
//
// One elected thread arms an mbarrier with the expected byte count and issues
// a tiled bulk-tensor copy (cp.async.bulk.tensor, no multicast: the source is
// always this GPU's own memory); every thread then waits on the mbarrier.
// Waits are bounded: after kTmaSpinLimit polls the kernel records an error in
// the plan's status word and skips the box (the host reports
// IBK_ERR_DEVICE_CHECK).  Copies start on 16-byte boundaries by construction
// (even x origin, even box width for 8-byte elements).
#pragma once
#include <cstdint>
#include <cuda.h>
#include "ibk_device.cuh"

namespace ibk {

struct TmaMaps {
	CUtensorMap map[kMaxDims];   // one per grid component
};

constexpr unsigned kTmaSpinLimit = 1u << 22;

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
	return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Ends the barrier object so its memory can be initialised again (a
// persistent CTA reuses one barrier for every tile it stages).
__device__ __forceinline__ void mbar_inval(uint64_t* bar)
{
	asm volatile("mbarrier.inval.shared::cta.b64 [%0];" :: "r"(smem_addr(bar)) : "memory");
}

// Orders this thread's earlier generic-proxy accesses to shared memory
// (reads of a staged box, patches, in-place rounding) before a later
// tensor copy that overwrites the same bytes.
__device__ __forceinline__ void fence_proxy_async_smem()
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// A tensor map in global memory written before the launch (by a copy from
// the host) is made visible to the tensor-copy proxy before its first use.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map)
{
	asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;"
	             :: "l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
	             :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
	unsigned ok;
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	             "selp.u32 %0, 1, 0, p;\n\t}"
	             : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
	return ok != 0;
}

// Bounded wait for phase `parity`; false (and an error recorded) on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int* status)
{
	for (unsigned i = 0; i < kTmaSpinLimit; ++i)
		if (mbar_try_wait(bar, parity)) return true;
	if (status) atomicExch(status, 1);
	return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar)
{
	asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
	             " [%0], [%1, {%2, %3, %4}], [%5];"
	             :: "r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z),
	                "r"(smem_addr(bar))
	             : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar)
{
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
	             " [%0], [%1, {%2, %3}], [%4];"
	             :: "r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y),
	                "r"(smem_addr(bar))
	             : "memory");
}

} // namespace ibk
