// Shared-memory barriers and bulk asynchronous copies (sm_90+ PTX, used on
// sm_100a): mbarrier phases with transaction counts, one-dimensional
// cp.async.bulk from global to shared memory (no multicast), and bounded
// waits that give up - setting an error flag - instead of spinning forever.
#pragma once
#include <cuda_runtime.h>

namespace tval3g {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
	return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
	unsigned ok;
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	    "selp.u32 %0, 1, 0, p;\n\t}"
	    : "=r"(ok)
	    : "r"(bar), "r"(parity)
	    : "memory");
	return ok != 0;
}
// generic-proxy accesses of shared memory before async-proxy ones (a bulk
// copy into a buffer that was just read)
__device__ __forceinline__ void fence_proxy_async_smem() {
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// barrier initialisation visible to the async proxy
__device__ __forceinline__ void fence_mbar_init() {
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// bytes (a multiple of 16) from global src to shared dst (both 16-byte
// aligned); completion is signalled on bar as a transaction count
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
	             "l"(src), "r"(bytes), "r"(bar)
	             : "memory");
}

// L2 cache policies (createpolicy): evict_last keeps lines that will be read
// again soon; evict_first marks lines at their last use
__device__ __forceinline__ unsigned long long l2_policy_evict_last() {
	unsigned long long p;
	asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
	return p;
}
__device__ __forceinline__ unsigned long long l2_policy_evict_first() {
	unsigned long long p;
	asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
	return p;
}
// bulk_g2s with an L2 cache policy for the source lines
__device__ __forceinline__ void bulk_g2s_hint(unsigned dst, const void *src, unsigned bytes, unsigned bar,
                                              unsigned long long policy) {
	asm volatile(
	    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
	        dst),
	    "l"(src), "r"(bytes), "r"(bar), "l"(policy)
	    : "memory");
}
// a 16-byte global load with an L2 cache policy
__device__ __forceinline__ float4 ld_f4_hint(const float *p, unsigned long long policy) {
	float4 v;
	asm volatile("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
	             : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
	             : "l"(p), "l"(policy));
	return v;
}

constexpr unsigned ASYNC_WAIT_LIMIT = 1u << 22;   // polls before a wait gives up

// every lane of the warp polls phase `parity` of bar; false (after raising
// *err from lane 0) if it does not complete within `limit` polls
__device__ __forceinline__ bool mbar_wait_warp(unsigned bar, unsigned parity, int *err,
                                               unsigned limit = ASYNC_WAIT_LIMIT) {
	for (unsigned i = 0; i < limit; i++)
		if (__all_sync(0xffffffffu, mbar_try(bar, parity))) return true;
	if ((threadIdx.x & 31) == 0) atomicExch(err, 1);
	return false;
}

}  // namespace tval3g
