// Self-test of the tcgen05 layer: C = A B^T for one 128 x 128 tile with
// K = 32 (tf32) or K = 64 (bf16, int8), operands staged K-major without swizzle,
// accumulator in TMEM, read back with tcgen05.ld.  Used by the parity tests
// to check descriptors and layouts against exact integer products before
// any assembly kernel relies on them.
#pragma once

#include <cuda_bf16.h>

#include "tc.cuh"

namespace h3dg {

// A: 128 x K row-major floats, B: 128 x K row-major floats (values exact in
// the MMA input type), C: 128 x 128 row-major.  One CTA of 128 threads.
template <int KIND>
__global__ void __launch_bounds__(128) k_tc_selftest(const float *A, const float *B, float *C, int *status) {
	constexpr int M = 128, N = 128;
	constexpr int K = KIND == tc::kTF32 ? 32 : 64;
	constexpr int ESZ = KIND == tc::kTF32 ? 4 : KIND == tc::kBF16 ? 2 : 1;
	__shared__ __align__(128) unsigned char sa[M * K * ESZ];
	__shared__ __align__(128) unsigned char sb[N * K * ESZ];
	__shared__ uint64_t bar;
	__shared__ uint32_t tslot;
	const int tid = threadIdx.x, warp = tid >> 5;
	if (warp == 0) tc::tmem_alloc(&tslot, 128);
	if (tid == 0) {
		mbar_init(&bar, 1);
		fence_mbar_init();
	}
	for (int i = tid; i < M * K; i += 128) {
		const int r = i / K, k = i % K;
		if (KIND == tc::kTF32) {
			*reinterpret_cast<float *>(sa + tc::kmaj_off32(r, k, M)) = A[i];
			*reinterpret_cast<float *>(sb + tc::kmaj_off32(r, k, N)) = B[i];
		}
		else if (KIND == tc::kBF16) {
			*reinterpret_cast<__nv_bfloat16 *>(sa + tc::kmaj_off16(r, k, M)) = __float2bfloat16(A[i]);
			*reinterpret_cast<__nv_bfloat16 *>(sb + tc::kmaj_off16(r, k, N)) = __float2bfloat16(B[i]);
		}
		else {
			*reinterpret_cast<int8_t *>(sa + tc::kmaj_off8(r, k, M)) = (int8_t) (int) A[i];
			*reinterpret_cast<int8_t *>(sb + tc::kmaj_off8(r, k, N)) = (int8_t) (int) B[i];
		}
	}
	tc::fence_async_smem();
	tc::fence_before_sync();
	__syncthreads();
	tc::fence_after_sync();
	const uint32_t tmem = tslot;
	if (tid == 0) {
		constexpr uint32_t idesc = KIND == tc::kI8 ? tc::instr_desc_i8(M, N) : tc::instr_desc(M, N, KIND);
		constexpr uint32_t lbo_a = (M / 8) * 128, lbo_b = (N / 8) * 128;
		for (int s = 0; s < K * ESZ / 32; s++) {
			const uint64_t da = tc::smem_desc(sa + s * 2 * lbo_a, lbo_a, 128);
			const uint64_t db = tc::smem_desc(sb + s * 2 * lbo_b, lbo_b, 128);
			if (KIND == tc::kTF32) tc::mma_tf32(tmem, da, db, idesc, s > 0);
			else if (KIND == tc::kBF16) tc::mma_bf16(tmem, da, db, idesc, s > 0);
			else tc::mma_i8(tmem, da, db, idesc, s > 0);
		}
		tc::mma_commit(&bar);
	}
	bool ok = mbar_wait_bounded(&bar, 0, status);
	// never free TMEM under an MMA still in flight: a second, longer bounded wait
	if (!ok) mbar_wait_bounded(&bar, 0, nullptr, 1u << 26);
	ok = __syncthreads_and(ok ? 1 : 0) != 0;
	tc::fence_after_sync();
	if (ok) {
		for (int c = 0; c < N; c += 16) {
			float v[16];
			tc::tmem_ld16(tmem + ((uint32_t) (32 * warp) << 16) + c, v);
#pragma unroll
			for (int j = 0; j < 16; j++)
				C[(32 * warp + (tid & 31)) * N + c + j] = KIND == tc::kI8 ? (float) __float_as_int(v[j]) : v[j];
		}
	}
	tc::fence_before_sync();
	__syncthreads();
	if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

} // namespace h3dg
