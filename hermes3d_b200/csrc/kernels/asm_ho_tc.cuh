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
//         K[(a,b,c)][(a',b',c')] = sum_{f,q1} V_f[(b',b,c)][q1] E_f[(a',a)][q1]
//     with E_f = E_x^(f>>1)[a][q1] E_x^(f&1)[a'][q1] (E^0 = values, E^1 =
//     derivatives of the x-direction Lobatto functions).  Per TRIAL z index
//     c' this is a GEMM with M = the rows (b', b, c) (tiles of 128, c
//     fastest), N = the pairs n = a' NX + a padded to a multiple of 16, K =
//     4 NQX padded to 8.  The E operand is constant and staged once per CTA;
//     the V operand of each tile is written to shared memory by stage 2 and
//     consumed by the MMA.
// Software pipeline per element: stage 2 of tile t+1 (other operand buffer)
// runs while the MMAs of tile t+1 are queued behind the epilogue of tile t
// (other TMEM accumulator).
// Epilogue: a thread owns one TMEM row (b', b, c) and, for each trial x index
// a', posts the 9 entries of CSC column j = (a', b', c') with rows i = (a, b,
// c).  Lanes of a warp share b' and so post into the same column at nearby
// rows: the adds coalesce in L2.  Positions come from a per-plan stream
// (k_build_offt) validated against the column lengths when it is built.  The
// adds are the same colour-exclusive, stream-ordered posted adds as in the
// FP64 kernels, so the split result is also bitwise reproducible run to run.
// Operand layout: K-major, no swizzle (see tc.cuh).  Every mbarrier wait is
// bounded; on timeout the kernel records kErrTimeout, drains, frees its TMEM
// and leaves.
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
	static constexpr int ACC_COLS = NB <= 32 ? 32 : NB <= 64 ? 64 : 128;   // one accumulator
	static constexpr int TMEM_COLS = 2 * ACC_COLS;                          // two, double-buffered
	static constexpr int NTT = NZ * NTILE;                                  // tiles per element
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
	static constexpr int U_MAT = O_AOP_REL + 4 * AOP_HALF;   // two buffers of (hi, lo)
	static constexpr int O_X = O_U + ho_tc_align(ho_tc_max(U_FP64, U_MAT), 16);
	static constexpr int O_M = O_X + 24 * 8;
	static constexpr int O_C = O_M + 24 * 8;
	static constexpr int O_CS = O_C + NL * 8;
	static constexpr int O_CE = O_CS + NL * 8;
	static constexpr int O_D = O_CE + NL * 8;
	static constexpr size_t SMEM_BYTES = (size_t) O_D + (size_t) NL * 4 + 16;
	static_assert(NB <= 128 && TM == 128, "MMA shape");
	static_assert(SMEM_BYTES <= 227 * 1024, "shared memory");
};

// Scatter stream of the tensor-core epilogue, built once per plan from the
// canonical position map: for element k, trial z index c' and row set col =
// (b', b, c), NB entries in TMEM-column order n = a' NX + a; entry = row
// position of cdof_i in column cdof_j (i = (a,b,c), j = (a',b',c')), or
// kOffSkip where either function has no matrix entry (Dirichlet) or n is
// padding.  Records are NB * 2 bytes (a multiple of 32), so a thread reads
// its half with 16-byte loads.
//
// First touch: built colour by colour (assembly order), an entry whose Ax
// slot no earlier element wrote carries kOffStore; the epilogue stores it
// instead of adding.  When every slot of the pattern is first-touched this
// way the assembly needs no zero-fill of Ax (saving a write and, for each
// first touch, the read of the posted add); 0 + v = v, so the values are
// the same.
constexpr uint16_t kOffSkip = 0xFFFF;
constexpr uint16_t kOffStore = 0x8000;
constexpr uint16_t kOffMask = 0x7FFF;

static __global__ void k_build_offt(const uint16_t *offc, const int32_t *cdof, const int64_t *Ap, int64_t kbeg, int64_t kend,
                                    int nx, int ny, int nz, int nb, uint16_t *offt, int *status, uint8_t *touched,
                                    unsigned long long *stores) {
	const int nl = nx * ny * nz, ncol = ny * ny * nz;
	const int64_t per = (int64_t) nz * ncol * nb;
	const int64_t total = (kend - kbeg) * per;
	unsigned long long nst = 0;
	for (int64_t e0 = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; e0 < total; e0 += (int64_t) gridDim.x * blockDim.x) {
		const int64_t e = kbeg * per + e0;
		const int n = (int) (e % nb);
		int64_t r = e / nb;
		const int col = (int) (r % ncol);
		r /= ncol;
		const int c2 = (int) (r % nz);
		const int64_t k = r / nz;
		uint16_t v = kOffSkip;
		if (n < nx * nx) {
			const int a2 = n / nx, a = n % nx;
			const int b2 = col / (ny * nz), b = (col / nz) % ny, c = col % nz;
			const int i = (a * ny + b) * nz + c, j = (a2 * ny + b2) * nz + c2;
			const int dj = cdof[k * nl + j];
			if (cdof[k * nl + i] >= 0 && dj >= 0) {
				v = offc[(k * nl + i) * nl + j];
				// every position is checked against its column once, here, so the
				// epilogue can post without a bounds test
				const int64_t len = Ap[dj + 1] - Ap[dj];
				if (v == kOffSkip || (int64_t) v >= len || v > kOffMask - 1) {
					if (len > 0) atomicOr(status, kErrBounds);     // an empty column is one this plan does not own
					v = kOffSkip;
				}
				else if (touched) {
					// elements of this launch (one colour) write disjoint slots
					const int64_t slot = Ap[dj] + v;
					if (!touched[slot]) {
						touched[slot] = 1;
						v |= kOffStore;
						nst++;
					}
				}
			}
		}
		offt[e] = v;
	}
	if (stores && nst) atomicAdd(stores, nst);
}

// stage 1 (FP32) for a fixed TRIAL z index c':
//   T1_kk[q1][q2][c] = sum_q3 G_g(kk) E_z^alpha[c][q3] E_z^beta[c'][q3]  (+ mass into kk = 2)
// (alpha / beta select values or derivatives of the test / trial function)
template <class S, int NT>
__device__ __forceinline__ void ho_tc_stage1(const float *G32, const float *tab32, int c2, int mass, float *T1) {
	using SB = typename S::B;
	constexpr int NZ = S::NZ, NQ = S::NQ, NQX = SB::QX, NQY = SB::QY, NQZ = SB::QZ;
	const float *Vz = tab32 + SB::OVZ, *Dz = tab32 + SB::ODZ;
	for (int i = threadIdx.x; i < 9 * NQX * NQY; i += NT) {
		const int kk = i / (NQX * NQY), q12 = i % (NQX * NQY);
		const int fz = kHoFz[kk];
		const float *eb = (fz & 1) ? Dz + c2 * NQZ : Vz + c2 * NQZ;
		const float *gp = G32 + kHoG[kk] * NQ + q12 * NQZ;
		const float *gm = G32 + 6 * NQ + q12 * NQZ;
		const bool addm = kk == 2 && mass;
		float h[NQZ], hm[NQZ];
#pragma unroll
		for (int q3 = 0; q3 < NQZ; q3++) {
			h[q3] = gp[q3] * eb[q3];
			hm[q3] = addm ? gm[q3] * Vz[c2 * NQZ + q3] : 0.0f;
		}
		float *out = T1 + (kk * NQX * NQY + q12) * NZ;
		for (int c = 0; c < NZ; c++) {
			const float *ea = (fz >> 1) ? Dz + c * NQZ : Vz + c * NQZ;
			float s = 0.0f;
#pragma unroll
			for (int q3 = 0; q3 < NQZ; q3++) s = fmaf(h[q3], ea[q3], s);
			if (addm) {
#pragma unroll
				for (int q3 = 0; q3 < NQZ; q3++) s = fmaf(hm[q3], Vz[c * NQZ + q3], s);
			}
			out[c] = s;
		}
	}
}

// stage 2 (FP32) for tile tt: V_f[q1] of row col = tt 128 + (tid mod 128) =
// (b', b, c) (trial y, test y, test z; c fastest), q1 split between the two
// threads of a row; written hi / lo (tf32) into the K-major V operand.
template <class S>
__device__ __forceinline__ void ho_tc_stage2(const float *T1, const float *tab32, int tt, unsigned char *aop_hi,
                                             unsigned char *aop_lo) {
	using SB = typename S::B;
	constexpr int NY = S::NY, NZ = S::NZ, NQX = SB::QX, NQY = SB::QY, TM = S::TM, H0 = S::H0, KD = S::KD;
	const float *Vy = tab32 + SB::OVY, *Dy = tab32 + SB::ODY;
	const int m = threadIdx.x & (TM - 1), half = threadIdx.x >> 7;
	const int col = tt * TM + m;
	float V[4][H0];
#pragma unroll
	for (int f = 0; f < 4; f++)
#pragma unroll
		for (int j = 0; j < H0; j++) V[f][j] = 0.0f;
	if (col < S::NCOL) {
		const int b2 = col / (NY * NZ), b = (col / NZ) % NY, c = col % NZ;
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
			const float *t1 = T1 + kk * NQX * NQY * NZ + c;
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

// stage 3: 3xTF32 MMAs of one tile into the accumulator at tmem_acc, small
// terms first (lo*hi, hi*lo, then hi*hi); one thread issues, commit to bar.
template <class S>
__device__ __forceinline__ void ho_tc_issue(uint32_t tmem_acc, const unsigned char *aop_hi, const unsigned char *aop_lo,
                                            const unsigned char *bop_hi, const unsigned char *bop_lo, uint64_t *bar) {
	constexpr int NB = S::NB, KD = S::KD, TM = S::TM;
	constexpr uint32_t idesc = tc::instr_desc(TM, NB, tc::kTF32);
	constexpr uint32_t lbo_a = (TM / 8) * 128, lbo_b = (NB / 8) * 128;
#pragma unroll
	for (int pass = 0; pass < 3; pass++) {
		const unsigned char *pa = pass == 0 ? aop_lo : aop_hi;
		const unsigned char *pb = pass == 1 ? bop_lo : bop_hi;
#pragma unroll
		for (int s = 0; s < KD / 8; s++) {
			const uint64_t da = tc::smem_desc(pa + s * 2 * lbo_a, lbo_a, 128);
			const uint64_t db = tc::smem_desc(pb + s * 2 * lbo_b, lbo_b, 128);
			tc::mma_tf32(tmem_acc, da, db, idesc, pass > 0 || s > 0);
		}
	}
	tc::mma_commit(bar);
}

// Epilogue of one tile for the threads of column half H: trial x index a'
// in [A2_0, A2_1), all test x indices a.  TMEM column n = a' NX + a, so for
// one a' the thread's CSC column j is fixed and its 9 positions are
// consecutive offsets into the prefetched record.
template <class S, int H>
struct HoTcEpi {
	static constexpr int NX = S::NX;
	static constexpr int A2_0 = H ? (NX + 1) / 2 : 0, A2_1 = H ? NX : (NX + 1) / 2;
	static constexpr int COL0 = A2_0 * NX, COL1 = A2_1 * NX;         // TMEM columns [COL0, COL1)
	static constexpr int CHB = COL0 / 16, CHE = (COL1 + 15) / 16;    // 16-column chunks loaded
	static constexpr int E0 = COL0 / 8 * 8;                          // first record entry prefetched
	static constexpr int NOV = (COL1 - E0 + 7) / 8;                  // 16-byte record pieces
};

template <class S>
struct HoTcEpiMax {
	static constexpr int NOV = HoTcEpi<S, 0>::NOV > HoTcEpi<S, 1>::NOV ? HoTcEpi<S, 0>::NOV : HoTcEpi<S, 1>::NOV;
};

template <class S, int H>
__device__ __forceinline__ void ho_tc_prefetch(const uint16_t *rec, uint4 *offv) {
	using E = HoTcEpi<S, H>;
	const uint4 *r = reinterpret_cast<const uint4 *>(rec + E::E0);
#pragma unroll
	for (int w = 0; w < E::NOV; w++) offv[w] = __ldcs(r + w);
}

template <class S, int H>
__device__ __forceinline__ void ho_tc_epilogue(uint32_t tacc, const uint4 *offv, bool live, int b2, int b, int c, int c2,
                                               const double *cc, const int64_t *cs, double *Ax) {
	using E = HoTcEpi<S, H>;
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ;
	float v[(E::CHE - E::CHB) * 16];
#pragma unroll
	for (int ch = E::CHB; ch < E::CHE; ch++) tc::tmem_ld16_nowait(tacc + (uint32_t) (ch * 16), v + (ch - E::CHB) * 16);
	tc::tmem_wait_ld();
	if (!live) return;
	double cci[NX];
#pragma unroll
	for (int a = 0; a < NX; a++) cci[a] = cc[(a * NY + b) * NZ + c];
	const uint16_t *o16 = reinterpret_cast<const uint16_t *>(offv);
#pragma unroll
	for (int a2 = E::A2_0; a2 < E::A2_1; a2++) {
		const int j = (a2 * NY + b2) * NZ + c2;
		const int64_t csj = cs[j];
		const double ccj = cc[j];
#pragma unroll
		for (int a = 0; a < NX; a++) {
			const int n = a2 * NX + a;
			const uint16_t off = o16[n - E::E0];
			if (off == kOffSkip) continue;
			const double val = cci[a] * ccj * (double) v[n - E::CHB * 16];
			if (off & kOffStore) posted_store(Ax + csj + (off & kOffMask), val);     // first touch of the slot
			else posted_add(Ax + csj + off, val);
		}
	}
}

// MINB > 1 (low orders): several CTAs share an SM; their TMEM allocations fit side by side
template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) k_assemble_ho_tc(KArgsHO args, int64_t kbeg, int64_t kend) {
	constexpr int NT = 256;
	using S = HoTcShape<PX, PY, PZ, NQX, NQY, NQZ>;
	using SB = typename S::B;
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NQ = S::NQ;
	constexpr int NB = S::NB, KD = S::KD, TM = S::TM, NTILE = S::NTILE, NTT = S::NTT;
	extern __shared__ __align__(128) unsigned char smb[];
	__shared__ uint64_t bar_tab, bar_mma[2];
	__shared__ int s_nlift;
	__shared__ uint32_t s_tmem;

	double *tab = reinterpret_cast<double *>(smb + S::O_TAB);
	float *tab32 = reinterpret_cast<float *>(smb + S::O_TAB32);
	unsigned char *bop_hi = smb + S::O_BOP, *bop_lo = bop_hi + S::BOP_HALF;
	float *G32 = reinterpret_cast<float *>(smb + S::O_G32);
	double *G64 = reinterpret_cast<double *>(smb + S::O_U);
	double *MFw = G64 + 8 * NQ;
	float *T1 = reinterpret_cast<float *>(smb + S::O_U);
	unsigned char *aop = smb + S::O_U + S::O_AOP_REL;     // buffer q: hi at aop + 2q AOP_HALF, lo after it
	double *X = reinterpret_cast<double *>(smb + S::O_X), *Mo = reinterpret_cast<double *>(smb + S::O_M);
	double *cc = reinterpret_cast<double *>(smb + S::O_C);
	int64_t *cs = reinterpret_cast<int64_t *>(smb + S::O_CS), *ce = reinterpret_cast<int64_t *>(smb + S::O_CE);
	int *cd = reinterpret_cast<int *>(smb + S::O_D);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

	if (!stage_tables(tab, args.tables, args.table_bytes, &bar_tab, args.status)) return;
	if (warp == 0) tc::tmem_alloc(&s_tmem, S::TMEM_COLS);
	if (tid == 0) {
		mbar_init(&bar_mma[0], 1);
		mbar_init(&bar_mma[1], 1);
		fence_mbar_init();
	}
	for (int i = tid; i < SB::TABP; i += NT) tab32[i] = (float) tab[i];
	// constant E operand, split hi / lo
	for (int e = tid; e < NB * KD; e += NT) {
		const int n = e / KD, kq = e % KD;
		double v = 0.0;
		if (n < S::NPAIR && kq < 4 * NQX) {
			const int a2 = n / NX, a = n % NX, f = kq / NQX, q1 = kq % NQX;
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
	const bool do_rhs = args.rhs && args.lf;
	uint32_t phases = 0u;                 // bit q: parity to wait for on bar_mma[q]
	bool alive = true;
	// epilogue mapping: TMEM lane quarter and column half of this warp
	const int quarter = warp & 3, chalf = warp >> 2;

	for (int64_t k = kbeg + blockIdx.x; k < kend && alive; k += gridDim.x) {
		// ---- FP64: set-up, geometry, load vector with lifting
		const double cgrad = ho_element_setup<SB, NT>(args, k, X, Mo, cc, cd, cs, ce, &s_nlift);
		ho_geometry<SB, NT>(args, tab, Mo, cgrad, G64);
		if (do_rhs) ho_rhs<SB, NT>(args, tab, G64, MFw, cd, cc, cd, cc, s_nlift > 0 && args.Ax);
		if (!args.Ax) continue;
		for (int i = tid; i < 7 * NQ; i += NT) G32[i] = (i < 6 * NQ || args.mass) ? (float) G64[i] : 0.0f;
		__syncthreads();

		// ---- software pipeline over the NTT tiles (c, tile): stage 2 of tile
		// t+1 and the MMAs of tile t+1 overlap the epilogue of tile t
		ho_tc_stage1<S, NT>(G32, tab32, 0, args.mass, T1);
		__syncthreads();
		ho_tc_stage2<S>(T1, tab32, 0, aop, aop + S::AOP_HALF);
		tc::fence_async_smem();
		tc::fence_before_sync();
		__syncthreads();
		if (tid == 0) {
			tc::fence_after_sync();
			ho_tc_issue<S>(tmem, aop, aop + S::AOP_HALF, bop_hi, bop_lo, &bar_mma[0]);
		}
		for (int t = 0; t < NTT; t++) {
			const int c2 = t / NTILE, tt = t % NTILE, q = t & 1;
			const int m = quarter * 32 + lane;
			const int col = tt * TM + m;
			const bool live = col < S::NCOL;
			// prefetch this thread's scatter offsets for tile t (streamed once)
			uint4 offv[HoTcEpiMax<S>::NOV];
			if (live) {
				const uint16_t *rec = args.offt + (((size_t) k * NZ + c2) * S::NCOL + col) * NB;
				if (chalf) ho_tc_prefetch<S, 1>(rec, offv);
				else ho_tc_prefetch<S, 0>(rec, offv);
			}
			// stage 1 / 2 of the next tile into the other buffer
			if (t + 1 < NTT) {
				const int c1 = (t + 1) / NTILE, tt1 = (t + 1) % NTILE;
				if (tt1 == 0) {
					ho_tc_stage1<S, NT>(G32, tab32, c1, args.mass, T1);
					__syncthreads();
				}
				unsigned char *ab = aop + 2 * (q ^ 1) * S::AOP_HALF;
				ho_tc_stage2<S>(T1, tab32, tt1, ab, ab + S::AOP_HALF);
			}
			// accumulator of tile t
			const uint32_t par = (phases >> q) & 1u;
			bool ok = mbar_wait_bounded(&bar_mma[q], par, args.status);
			if (!ok) mbar_wait_bounded(&bar_mma[q], par, nullptr, 1u << 26);
			phases ^= 1u << q;
			if (!__syncthreads_and(ok ? 1 : 0)) {
				alive = false;
				break;
			}
			tc::fence_after_sync();
			{
				const int b2 = live ? col / (NY * NZ) : 0, b = live ? (col / NZ) % NY : 0, c = live ? col % NZ : 0;
				const uint32_t tacc = tmem + ((uint32_t) (quarter * 32) << 16) + (uint32_t) (q * S::ACC_COLS);
				if (chalf) ho_tc_epilogue<S, 1>(tacc, offv, live, b2, b, c, c2, cc, cs, args.Ax);
				else ho_tc_epilogue<S, 0>(tacc, offv, live, b2, b, c, c2, cc, cs, args.Ax);
			}
			tc::fence_async_smem();
			tc::fence_before_sync();
			__syncthreads();
			if (t + 1 < NTT && tid == 0) {
				tc::fence_after_sync();
				const unsigned char *ab = aop + 2 * (q ^ 1) * S::AOP_HALF;
				ho_tc_issue<S>(tmem + (uint32_t) ((q ^ 1) * S::ACC_COLS), ab, ab + S::AOP_HALF, bop_hi, bop_lo,
				               &bar_mma[q ^ 1]);
			}
		}
	}
	__syncthreads();
	tc::fence_after_sync();
	if (warp == 0) tc::tmem_dealloc(tmem, S::TMEM_COLS);
}

} // namespace h3dg
