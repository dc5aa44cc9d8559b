// Tensor-memory-access (TMA) and mbarrier primitives for sm_100a, written as
// inline PTX.  Only plain CTA-local forms are used: no cluster multicast.
#pragma once
#include <cstdint>

namespace cbm {
namespace tma {

__device__ __forceinline__ uint32_t smemAddr(const void *p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbarInit(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fenceBarrierInit()
{
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void arriveExpectTx(uint64_t *bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void arrive(uint64_t *bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}

__device__ __forceinline__ bool tryWait(uint64_t *bar, uint32_t parity)
{
	uint32_t done;
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(done)
		: "r"(smemAddr(bar)), "r"(parity)
		: "memory");
	return done != 0;
}

__device__ __forceinline__ uint64_t globalTimerNs()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Wait for the phase of `bar` with the given parity, giving up after
// limitNs nanoseconds.  Returns false on time-out.
__device__ __forceinline__ bool waitBounded(uint64_t *bar, uint32_t parity, uint64_t limitNs)
{
	if (tryWait(bar, parity)) return true;
	const uint64_t t0 = globalTimerNs();
	while (!tryWait(bar, parity))
		if (globalTimerNs() - t0 > limitNs) return false;
	return true;
}

__device__ __forceinline__ void prefetchMap(const void *map)
{
	asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

// Tiled 2D / 3D loads global -> this CTA's shared memory, completing on bar.
// The innermost coordinate x times the element size must be a multiple of 16
// bytes (callers pass x = 32-element multiples).
__device__ __forceinline__ void load2d(void *dst, const void *map, int32_t x, int32_t y, uint64_t *bar)
{
	asm volatile(
		"cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
		::"r"(smemAddr(dst)), "l"(map), "r"(x), "r"(y), "r"(smemAddr(bar))
		: "memory");
}

__device__ __forceinline__ void load3d(void *dst, const void *map, int32_t x, int32_t y, int32_t z, uint64_t *bar)
{
	asm volatile(
		"cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
		::"r"(smemAddr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smemAddr(bar))
		: "memory");
}

}  // namespace tma
}  // namespace cbm
