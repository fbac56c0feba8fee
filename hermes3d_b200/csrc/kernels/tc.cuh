// Minimal tcgen05 (5th-generation tensor core) layer for sm_100a: TMEM
// allocation, shared-memory matrix descriptors, kind::tf32 / kind::f16 MMA
// issue, commit to an mbarrier and accumulator loads.
//
// Operand layout used throughout (K-major, no swizzle): an R x K tile of
// 32-bit (tf32) or 16-bit (bf16) elements is stored as 16-byte "core
// matrix" rows: element (r, k) lives at
//     ((k / E) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % E) * sizeof(elem)
// with E = 16 bytes / sizeof(elem).  In descriptor terms: stride between
// 8-row groups (SBO) = 128 B, stride between 16-byte K chunks (LBO) =
// (R / 8) * 128 B.  One MMA consumes 32 bytes of K (8 tf32 / 16 bf16), i.e.
// two K chunks; the next K step starts 2 * LBO further.
//
// Descriptor bit fields follow the sm100 UMMA definitions (SmemDescriptor:
// start>>4 [0,14), LBO>>4 [16,30), SBO>>4 [32,46), version 1 [46,48),
// layout type [61,64) = 0 for no swizzle; InstrDescriptor: c_format [4,6),
// a_format [7,10), b_format [10,13), a/b major [15]/[16], N>>3 [17,23),
// M>>4 [24,29)).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace h3dg {
namespace tc {

__device__ __forceinline__ uint64_t smem_desc(const void *base, uint32_t lbo_bytes, uint32_t sbo_bytes) {
	const uint32_t a = smem_u32(base);
	uint64_t d = 0;
	d |= (uint64_t) ((a >> 4) & 0x3FFF);
	d |= (uint64_t) ((lbo_bytes >> 4) & 0x3FFF) << 16;
	d |= (uint64_t) ((sbo_bytes >> 4) & 0x3FFF) << 32;
	d |= (uint64_t) 1 << 46;                       // version (sm100)
	// base offset 0, lbo mode 0, layout type 0 (no swizzle)
	return d;
}

// formats: 0 F16, 1 BF16, 2 TF32 (inputs); c: 1 = F32 accumulator
__host__ __device__ constexpr uint32_t instr_desc(int M, int N, int ab_format) {
	return (1u << 4)                                // D/C format F32
	       | ((uint32_t) ab_format << 7)            // A format
	       | ((uint32_t) ab_format << 10)           // B format
	       | (0u << 15) | (0u << 16)                // A, B K-major
	       | ((uint32_t) (N >> 3) << 17)
	       | ((uint32_t) (M >> 4) << 24);
}

constexpr int kTF32 = 2, kBF16 = 1;
constexpr int kI8 = 8;   // selects kind::i8 (signed int8 operands, int32 accumulator)

// kind::i8: c_format S32 (2), a / b format signed int8 (1)
__host__ __device__ constexpr uint32_t instr_desc_i8(int M, int N) {
	return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (N >> 3) << 17) | ((uint32_t) (M >> 4) << 24);
}

// Allocate ncols TMEM columns (power of two >= 32); warp-wide, one warp.
// The address is written to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols) : "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T ; issued by a single thread.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, bool accumulate) {
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d_tmem),
		"l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t) accumulate), "r"(0u)
		: "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, bool accumulate) {
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d_tmem),
		"l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t) accumulate), "r"(0u)
		: "memory");
}

// int8 x int8 -> int32, K = 32 per instruction
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, bool accumulate) {
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d_tmem),
		"l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t) accumulate), "r"(0u)
		: "memory");
}

// Arrive on an mbarrier once all previously issued MMAs of this thread complete.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 lanes x 32 bit, 16 consecutive columns per thread (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
	uint32_t r[16];
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
		  "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
		: "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// same without the wait: issue several, then tmem_wait_ld() once
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, float *v) {
	uint32_t *r = reinterpret_cast<uint32_t *>(v);
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
		  "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
		: "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// byte offset of element (r, k) in a K-major no-swizzle tile with R rows
// (R a multiple of 8) and 4-byte elements
__host__ __device__ __forceinline__ uint32_t kmaj_off32(int r, int k, int R) {
	return (uint32_t) ((((k >> 2) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 3) << 2));
}

// same for 2-byte elements
__host__ __device__ __forceinline__ uint32_t kmaj_off16(int r, int k, int R) {
	return (uint32_t) ((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// same for 1-byte elements
__host__ __device__ __forceinline__ uint32_t kmaj_off8(int r, int k, int R) {
	return (uint32_t) ((((k >> 4) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + (k & 15));
}

// round to tf32 (nearest, ties away) and return as float
__device__ __forceinline__ float to_tf32(float x) {
	uint32_t r;
	asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
	return __uint_as_float(r);
}

} // namespace tc
} // namespace h3dg
