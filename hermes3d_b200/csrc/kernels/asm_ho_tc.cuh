// Split-precision high-order assembly on the 5th-generation tensor cores.
//
// Same element matrix as k_assemble_fp64_ho (src/integrals/h1.h:115-177 per
// pair, restated as sum factorisation), with the precision split the way the
// error budget allows:
//   * FP64: the reference map, its determinant and inverse, the geometric
//     factors G, the load vector and the Dirichlet lifting (matrix-free
//     element operator, shared with the FP64 kernel), the CSC positions and
//     the final coefficient products c_i c_j K_ij;
//   * FP32: stage 1 (G folded with the z tables) and stage 2 (the y tables),
//     i.e. the per-column vectors V_f[q1], f = 4 x-classes;
//   * tcgen05 kind::tf32 with three products (3xTF32, hi*hi + hi*lo +
//     lo*hi, FP32 accumulation in TMEM): stage 3,
//         K[(a,b,c)][(a',b',c')] = sum_{f,q1} V_f[(b,b',c')][q1] E_f[(a,a')][q1]
//     with E_f[(a,a')][q1] = E_x^(f>>1)[a][q1] E_x^(f&1)[a'][q1] (E^0 = values,
//     E^1 = derivatives of the x-direction Lobatto functions).  Per test z
//     index c this is a GEMM with M = the (b,b',c') columns (tiles of 128), N =
//     the (a,a') pairs padded to a multiple of 16, K = 4 NQX padded to 8.  The
//     E operand is constant and staged once per CTA; the V operand of each
//     tile is written to shared memory by stage 2 and consumed by the MMA.
// The epilogue reads the accumulator tile from TMEM (one row = one column
// set (b,b',c') per thread) and posts c_i c_j K_ij into the CSC matrix with
// the same colour-exclusive, stream-ordered adds as the FP64 kernels, so the
// split result is also bitwise reproducible run to run.
// Operand layout: K-major, no swizzle (see tc.cuh).  One mbarrier tracks MMA
// completion; every wait is bounded and on timeout the kernel records
// kErrTimeout, drains, frees its TMEM and leaves.
#pragma once

#include "asm_fp64_ho.cuh"
#include "tc.cuh"

namespace h3dg {

__host__ __device__ constexpr int ho_tc_align(int x, int a) { return (x + a - 1) / a * a; }
__host__ __device__ constexpr int ho_tc_max(int a, int b) { return a > b ? a : b; }

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ>
struct HoTcShape {
	using B = HoShape<PX, PY, PZ, NQX, NQY, NQZ>;
	static constexpr int NX = B::NX, NY = B::NY, NZ = B::NZ, NL = B::NL, NQ = B::NQ;
	static constexpr int NPAIR = NX * NX;                     // (a, a') pairs
	static constexpr int NB = ho_tc_align(NPAIR, 16);         // MMA N
	static constexpr int KD = ho_tc_align(4 * NQX, 8);        // MMA K (tf32: 8 per instruction)
	static constexpr int NCOL = NY * NY * NZ;                 // columns (b, b', c') per test z index
	static constexpr int TM = 128;                            // MMA M
	static constexpr int NTILE = (NCOL + TM - 1) / TM;
	static constexpr int TMEM_COLS = NB <= 32 ? 32 : NB <= 64 ? 64 : NB <= 128 ? 128 : 256;
	static constexpr int H0 = (NQX + 1) / 2;                  // q1 split between the two stage-2 threads of a column
	static constexpr int T1F = 9 * NQX * NQY * NZ;            // stage-1 products (floats)
	// dynamic shared memory, byte offsets
	static constexpr int O_TAB = 0;                                          // FP64 tables
	static constexpr int O_TAB32 = O_TAB + 8 * B::TABP;                      // FP32 copy
	static constexpr int O_BOP = ho_tc_align(O_TAB32 + 4 * B::TABP, 128);    // E operand: hi, lo (NB x KD each)
	static constexpr int BOP_HALF = NB * KD * 4;
	static constexpr int O_G32 = O_BOP + 2 * BOP_HALF;                       // 7 x NQ floats
	static constexpr int O_U = ho_tc_align(O_G32 + 7 * NQ * 4, 128);         // union, see below
	//   FP64 phase: G (8 NQ doubles) + matrix-free work (MF doubles)
	//   matrix phase: T1 (T1F floats), then the V operand hi, lo (TM x KD each)
	static constexpr int U_FP64 = 8 * (8 * NQ + B::MF);
	static constexpr int O_AOP_REL = ho_tc_align(4 * T1F, 128);
	static constexpr int AOP_HALF = TM * KD * 4;
	static constexpr int U_MAT = O_AOP_REL + 2 * AOP_HALF;
	static constexpr int O_X = O_U + ho_tc_align(ho_tc_max(U_FP64, U_MAT), 16);
	static constexpr int O_M = O_X + 24 * 8;
	static constexpr int O_C = O_M + 24 * 8;
	static constexpr int O_CS = O_C + NL * 8;
	static constexpr int O_CE = O_CS + NL * 8;
	static constexpr int O_D = O_CE + NL * 8;
	static constexpr size_t SMEM_BYTES = (size_t) O_D + (size_t) NL * 4 + 16;
	static_assert(NB <= 256 && TM == 128, "MMA shape");
	static_assert(SMEM_BYTES <= 227 * 1024, "shared memory");
};

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ>
__global__ void __launch_bounds__(256, 1) k_assemble_ho_tc(KArgsHO args, int64_t kbeg, int64_t kend) {
	constexpr int NT = 256;
	using S = HoTcShape<PX, PY, PZ, NQX, NQY, NQZ>;
	using SB = typename S::B;
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NL = S::NL, NQ = S::NQ;
	constexpr int NB = S::NB, KD = S::KD, TM = S::TM, H0 = S::H0;
	extern __shared__ __align__(128) unsigned char smb[];
	__shared__ uint64_t bar_tab, bar_mma;
	__shared__ int s_nlift;
	__shared__ uint32_t s_tmem;

	double *tab = reinterpret_cast<double *>(smb + S::O_TAB);
	float *tab32 = reinterpret_cast<float *>(smb + S::O_TAB32);
	unsigned char *bop_hi = smb + S::O_BOP, *bop_lo = bop_hi + S::BOP_HALF;
	float *G32 = reinterpret_cast<float *>(smb + S::O_G32);
	double *G64 = reinterpret_cast<double *>(smb + S::O_U);
	double *MFw = G64 + 8 * NQ;
	float *T1 = reinterpret_cast<float *>(smb + S::O_U);
	unsigned char *aop_hi = smb + S::O_U + S::O_AOP_REL, *aop_lo = aop_hi + S::AOP_HALF;
	double *X = reinterpret_cast<double *>(smb + S::O_X), *Mo = reinterpret_cast<double *>(smb + S::O_M);
	double *cc = reinterpret_cast<double *>(smb + S::O_C);
	int64_t *cs = reinterpret_cast<int64_t *>(smb + S::O_CS), *ce = reinterpret_cast<int64_t *>(smb + S::O_CE);
	int *cd = reinterpret_cast<int *>(smb + S::O_D);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

	if (!stage_tables(tab, args.tables, args.table_bytes, &bar_tab, args.status)) return;
	if (warp == 0) tc::tmem_alloc(&s_tmem, S::TMEM_COLS);
	if (tid == 0) {
		mbar_init(&bar_mma, 1);
		fence_mbar_init();
	}
	for (int i = tid; i < SB::TABP; i += NT) tab32[i] = (float) tab[i];
	// constant E operand, split hi / lo
	for (int e = tid; e < NB * KD; e += NT) {
		const int n = e / KD, kq = e % KD;
		double v = 0.0;
		if (n < S::NPAIR && kq < 4 * NQX) {
			const int a = n / NX, a2 = n % NX, f = kq / NQX, q1 = kq % NQX;
			const double ea = (f >> 1) ? tab[SB::ODX + a * NQX + q1] : tab[SB::OVX + a * NQX + q1];
			const double eb = (f & 1) ? tab[SB::ODX + a2 * NQX + q1] : tab[SB::OVX + a2 * NQX + q1];
			v = ea * eb;
		}
		const float hi = tc::to_tf32((float) v);
		const float lo = tc::to_tf32((float) (v - (double) hi));
		*reinterpret_cast<float *>(bop_hi + tc::kmaj_off32(n, kq, NB)) = hi;
		*reinterpret_cast<float *>(bop_lo + tc::kmaj_off32(n, kq, NB)) = lo;
	}
	tc::fence_async_smem();
	tc::fence_before_sync();
	__syncthreads();
	tc::fence_after_sync();
	const uint32_t tmem = s_tmem;
	const float *Vy = tab32 + SB::OVY, *Dy = tab32 + SB::ODY, *Vz = tab32 + SB::OVZ, *Dz = tab32 + SB::ODZ;
	const bool do_rhs = args.rhs && args.lf;
	uint32_t mma_phase = 0;
	bool alive = true;

	for (int64_t k = kbeg + blockIdx.x; k < kend && alive; k += gridDim.x) {
		// ---- FP64: set-up, geometry, load vector with lifting
		const double cgrad = ho_element_setup<SB, NT>(args, k, X, Mo, cc, cd, cs, ce, &s_nlift);
		ho_geometry<SB, NT>(args, tab, Mo, cgrad, G64);
		if (do_rhs) ho_rhs<SB, NT>(args, tab, G64, MFw, cd, cc, s_nlift > 0);
		if (!args.Ax) continue;
		for (int i = tid; i < 7 * NQ; i += NT) G32[i] = (i < 6 * NQ || args.mass) ? (float) G64[i] : 0.0f;
		__syncthreads();

		for (int c = 0; c < NZ && alive; c++) {
			// ---- stage 1 (FP32): T1_kk[q1][q2][c'] = sum_q3 G_g(kk) E_z^alpha[c][q3] E_z^beta[c'][q3] (+ mass into kk = 2)
			for (int i = tid; i < 9 * NQX * NQY; i += NT) {
				const int kk = i / (NQX * NQY), q12 = i % (NQX * NQY);
				const int fz = kHoFz[kk];
				const float *ea = (fz >> 1) ? Dz + c * NQZ : Vz + c * NQZ;
				const float *gp = G32 + kHoG[kk] * NQ + q12 * NQZ;
				const float *gm = G32 + 6 * NQ + q12 * NQZ;
				const bool addm = kk == 2 && args.mass;
				float h[NQZ], hm[NQZ];
#pragma unroll
				for (int q3 = 0; q3 < NQZ; q3++) {
					h[q3] = gp[q3] * ea[q3];
					hm[q3] = addm ? gm[q3] * Vz[c * NQZ + q3] : 0.0f;
				}
				float *out = T1 + (kk * NQX * NQY + q12) * NZ;
				for (int c2 = 0; c2 < NZ; c2++) {
					const float *eb = (fz & 1) ? Dz + c2 * NQZ : Vz + c2 * NQZ;
					float s = 0.0f;
#pragma unroll
					for (int q3 = 0; q3 < NQZ; q3++) s = fmaf(h[q3], eb[q3], s);
					if (addm) {
#pragma unroll
						for (int q3 = 0; q3 < NQZ; q3++) s = fmaf(hm[q3], Vz[c2 * NQZ + q3], s);
					}
					out[c2] = s;
				}
			}
			__syncthreads();

			for (int t = 0; t < S::NTILE; t++) {
				// ---- stage 2 (FP32): V_f[q1] of column col, q1 split between two threads
				{
					const int m = tid & (TM - 1), half = tid >> 7;
					const int col = t * TM + m;
					float V[4][H0];
#pragma unroll
					for (int f = 0; f < 4; f++)
#pragma unroll
						for (int j = 0; j < H0; j++) V[f][j] = 0.0f;
					if (col < S::NCOL) {
						const int b = col / (NY * NZ), b2 = (col / NZ) % NY, c2 = col % NZ;
#pragma unroll
						for (int kk = 0; kk < 9; kk++) {
							// y flag and x class of product kk (compile-time after unrolling)
							constexpr int kFy[9] = { 0, 3, 0, 1, 2, 0, 0, 2, 1 };
							constexpr int kCls[9] = { 3, 0, 0, 2, 1, 2, 1, 0, 0 };
							const int fy = kFy[kk], f = kCls[kk];
							const float *ea = (fy >> 1) ? Dy + b * NQY : Vy + b * NQY;
							const float *eb = (fy & 1) ? Dy + b2 * NQY : Vy + b2 * NQY;
							float wy[NQY];
#pragma unroll
							for (int q2 = 0; q2 < NQY; q2++) wy[q2] = ea[q2] * eb[q2];
							const float *t1 = T1 + kk * NQX * NQY * NZ + c2;
#pragma unroll
							for (int j = 0; j < H0; j++) {
								const int q1 = j + half * H0;
								if (q1 < NQX) {
									float s = V[f][j];
#pragma unroll
									for (int q2 = 0; q2 < NQY; q2++) s = fmaf(wy[q2], t1[(q1 * NQY + q2) * NZ], s);
									V[f][j] = s;
								}
							}
						}
					}
#pragma unroll
					for (int f = 0; f < 4; f++)
#pragma unroll
						for (int j = 0; j < H0; j++) {
							const int q1 = j + half * H0;
							if (q1 < NQX) {
								const float v = V[f][j];
								const float hi = tc::to_tf32(v);
								const float lo = tc::to_tf32(v - hi);
								const uint32_t o = tc::kmaj_off32(m, f * NQX + q1, TM);
								*reinterpret_cast<float *>(aop_hi + o) = hi;
								*reinterpret_cast<float *>(aop_lo + o) = lo;
							}
						}
					if (KD > 4 * NQX && half == 1) {
						for (int kq = 4 * NQX; kq < KD; kq++) {
							const uint32_t o = tc::kmaj_off32(m, kq, TM);
							*reinterpret_cast<float *>(aop_hi + o) = 0.0f;
							*reinterpret_cast<float *>(aop_lo + o) = 0.0f;
						}
					}
				}
				tc::fence_async_smem();
				tc::fence_before_sync();
				__syncthreads();

				// ---- stage 3: 3xTF32 on the tensor cores, one thread issues
				if (tid == 0) {
					tc::fence_after_sync();
					constexpr uint32_t idesc = tc::instr_desc(TM, NB, tc::kTF32);
					constexpr uint32_t lbo_a = (TM / 8) * 128, lbo_b = (NB / 8) * 128;
					// small terms first: lo*hi, hi*lo, then hi*hi
#pragma unroll
					for (int pass = 0; pass < 3; pass++) {
						const unsigned char *pa = pass == 0 ? aop_lo : aop_hi;
						const unsigned char *pb = pass == 1 ? bop_lo : bop_hi;
#pragma unroll
						for (int s = 0; s < KD / 8; s++) {
							const uint64_t da = tc::smem_desc(pa + s * 2 * lbo_a, lbo_a, 128);
							const uint64_t db = tc::smem_desc(pb + s * 2 * lbo_b, lbo_b, 128);
							tc::mma_tf32(tmem, da, db, idesc, pass > 0 || s > 0);
						}
					}
					tc::mma_commit(&bar_mma);
				}
				bool ok = mbar_wait_bounded(&bar_mma, mma_phase, args.status);
				if (!ok) mbar_wait_bounded(&bar_mma, mma_phase, nullptr, 1u << 26);
				mma_phase ^= 1u;
				if (!__syncthreads_and(ok ? 1 : 0)) {
					alive = false;
					break;
				}
				tc::fence_after_sync();

				// ---- epilogue: TMEM row m = column set (b,b',c'), TMEM column n = pair (a,a')
				{
					const int quarter = warp & 3, chalf = warp >> 2;
					const int m = quarter * 32 + lane;
					const int col = t * TM + m;
					const bool live = col < S::NCOL;
					const int b = live ? col / (NY * NZ) : 0, b2 = live ? (col / NZ) % NY : 0, c2 = live ? col % NZ : 0;
					constexpr int NCH = NB / 16;                 // 16-column chunks
					constexpr int CH0 = (NCH + 1) / 2;
					const int ch_beg = chalf ? CH0 : 0, ch_end = chalf ? NCH : CH0;
					const uint16_t *offk = args.offc + (size_t) k * NL * NL;
					for (int ch = ch_beg; ch < ch_end; ch++) {
						float v[16];
						tc::tmem_ld16(tmem + ((uint32_t) (quarter * 32) << 16) + (uint32_t) (ch * 16), v);
						if (!live) continue;
#pragma unroll
						for (int u = 0; u < 16; u++) {
							const int n = ch * 16 + u;
							if (n >= S::NPAIR) break;
							const int a = n / NX, a2 = n % NX;
							const int i = (a * NY + b) * NZ + c, j = (a2 * NY + b2) * NZ + c2;
							const int di = cd[i], dj = cd[j];
							if (di < 0 || dj < 0) continue;
							const int64_t pos = cs[j] + offk[(size_t) i * NL + j];
							if (pos < ce[j]) posted_add(args.Ax + pos, cc[i] * cc[j] * (double) v[u]);
							else atomicOr(args.status, kErrBounds);
						}
					}
				}
				tc::fence_before_sync();
				__syncthreads();
			}
		}
	}
	__syncthreads();
	tc::fence_after_sync();
	if (warp == 0) tc::tmem_dealloc(tmem, S::TMEM_COLS);
}

} // namespace h3dg
