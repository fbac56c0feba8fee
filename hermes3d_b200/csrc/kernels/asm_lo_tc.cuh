// Split-precision (3xTF32) assembly for low uniform orders, with elements
// batched on the 5th-generation tensor cores.
//
// Same element matrix as k_assemble_fp64 (src/integrals/h1.h:115-177 per
// pair, restated as sum factorisation; K = A + A^T with the 0.5 factors in
// G), with stages 2 and 3 of the sum factorisation fused into one GEMM over
// a batch of elements:
//     A[(a,b,c)][(a',b',c')] = sum_k sum_{q1,q2} T1_k[q1][q2][c][c'] W_k[q1 q2][a a' b b'],
//     W_k[q1 q2][a a' b b'] = Wx_fx(k)[a][a'][q1] Wy_fy(k)[b][b'][q2],
// k the 6 stage-1 products (xx, yy, zz + mass, xy, xz, yz).  GEMM rows are
// (element, c, c') -- (p+1)^2 per element, so 128 / (p+1)^2 elements fill
// one MMA tile (14 at p = 2, 32 at p = 1) --, K = (k, q1, q2), N = (a, a',
// b, b').  W is the same for every element: it is the B operand, staged in
// shared memory once per CTA.  The A operand (T1) is produced per batch by
// stage 1.
// Precision split:
//   * FP64: reference map, determinant, inverse (geometric factors G), load
//     vector, Dirichlet lifting (matrix-free: the lifting function's gradient
//     at the points, G applied, integrated back), coefficient products, CSC
//     positions;
//   * FP32: G for the matrix, stage 1 (G folded with the z tables);
//   * tcgen05 kind::tf32, three products (hi*hi + hi*lo + lo*hi, small terms
//     first) accumulated in FP32 in TMEM: stages 2+3.
// Epilogue: TMEM rows -> A in shared memory (FP64), then the scatter and the
// load vector exactly as k_assemble_fp64 posts them: colour-exclusive,
// stream-ordered posted adds, bitwise reproducible run to run.
// Every mbarrier wait is bounded; on timeout the kernel records kErrTimeout,
// waits (bounded) for the MMAs in flight, frees its TMEM and leaves.
#pragma once

#include "asm_fp64.cuh"
#include "tc.cuh"

namespace h3dg {

__host__ __device__ constexpr int lt_align(int x, int a) { return (x + a - 1) / a * a; }
__host__ __device__ constexpr int lt_max(int a, int b) { return a > b ? a : b; }

template <int P, int NQ>
struct LoTcShape {
	using S = SfShape<P, P, P, NQ, NQ, NQ, 1>;               // 1D table blob layout
	static constexpr int NX = P + 1, NL = NX * NX * NX, NQ3 = NQ * NQ * NQ;
	static constexpr int ROWS = NX * NX;                      // GEMM rows per element: (c, c')
	static constexpr int TM = 128;
	static constexpr int EBT = TM / ROWS;                     // elements per batch
	static constexpr int KREAL = 6 * NQ * NQ, KD = lt_align(KREAL, 8);
	static constexpr int NREAL = NX * NX * NX * NX, NB = lt_align(NREAL, 16);
	static constexpr int ACC = NB <= 32 ? 32 : NB <= 64 ? 64 : NB <= 128 ? 128 : 256;   // TMEM columns
	static constexpr int AOP = TM * KD * 4;                   // bytes of one A half (hi or lo)
	static constexpr int BOP = NB * KD * 4;
	static constexpr int WZN = 4 * NX * NX * NQ;              // Wz^f[c][c'][q3], floats
	// per-element area (doubles): vertices, monomials, coefficients, load
	// vector, DOFs and shape indices (ints), source weights at the points,
	// column bounds
	static constexpr int E_X = 0, E_M = 24, E_C = 48, E_F = E_C + NL, E_I = E_F + NL, E_GS = E_I + NL;
	static constexpr int E_CS = E_GS + NQ3, E_CE = E_CS + NL;  // column bounds (int64) of the element's DOFs
	static constexpr int E_SIZE = lt_align(E_CE + NL, 2);
	// dynamic shared memory, byte offsets
	static constexpr int O_TAB = 0;
	static constexpr int O_WZ = lt_align(O_TAB + 8 * S::TABP, 16);
	static constexpr int O_BOP = lt_align(O_WZ + 4 * WZN, 128);
	static constexpr int O_AOP = O_BOP + 2 * BOP;             // A operand hi, lo; later A (FP64, EBT x NL^2)
	static constexpr int U_A = lt_max(2 * AOP, EBT * NL * NL * 8);
	static constexpr int O_G32 = lt_align(O_AOP + U_A, 16);   // EBT x 7 x NQ3 floats
	static constexpr int O_EL = lt_align(O_G32 + EBT * 7 * NQ3 * 4, 16);
	static constexpr size_t SMEM_BYTES = (size_t) O_EL + (size_t) EBT * E_SIZE * 8;
	static_assert(NB <= 256 && KD % 8 == 0, "MMA shape");
	static_assert(SMEM_BYTES <= 225 * 1024, "shared memory");
};

// N index n = ((a NX + a') NX + b) NX + b'; K index kq = (k NQ + q1) NQ + q2
// x / y table flags of the 6 stage-1 products (alpha = test side
// differentiated, beta = trial side): f = 2 alpha + beta
static __device__ __constant__ int kLtFx[6] = { 3, 0, 0, 2, 2, 0 };
static __device__ __constant__ int kLtFy[6] = { 0, 3, 0, 1, 0, 2 };
static __device__ __constant__ int kLtFz[6] = { 0, 0, 3, 0, 1, 1 };

template <int P, int NQ, int NT>
__global__ void __launch_bounds__(NT, 1) k_assemble_lo_tc(KArgs args, int64_t kbeg, int64_t kend) {
	using L = LoTcShape<P, NQ>;
	using S = typename L::S;
	constexpr int NX = L::NX, NL = L::NL, NL2 = NL * NL, NQ3 = L::NQ3, ROWS = L::ROWS, EBT = L::EBT;
	constexpr int KD = L::KD, NB = L::NB, TM = L::TM;
	static_assert(NT == 256, "two warps per TMEM lane quarter");
	extern __shared__ __align__(128) unsigned char smb[];
	__shared__ uint64_t bar_tab, bar_mma;
	__shared__ uint32_t s_tmem;
	__shared__ int s_m[EBT], s_l[EBT];
	__shared__ double s_cg[EBT];
	double *tab = reinterpret_cast<double *>(smb + L::O_TAB);
	float *wz = reinterpret_cast<float *>(smb + L::O_WZ);
	unsigned char *bop_hi = smb + L::O_BOP, *bop_lo = bop_hi + L::BOP;
	unsigned char *aop_hi = smb + L::O_AOP, *aop_lo = aop_hi + L::AOP;
	double *Afp = reinterpret_cast<double *>(smb + L::O_AOP);     // after the MMAs: A of the batch's elements
	float *G32 = reinterpret_cast<float *>(smb + L::O_G32);
	double *EL = reinterpret_cast<double *>(smb + L::O_EL);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

	if (!stage_tables(tab, args.tables, args.table_bytes, &bar_tab, args.status, args.wait_limit)) return;
	if (warp == 0) tc::tmem_alloc(&s_tmem, L::ACC);
	if (tid == 0) {
		mbar_init(&bar_mma, 1);
		fence_mbar_init();
	}
	// z products (FP32) for stage 1 and the constant B operand W (hi / lo)
	for (int i = tid; i < L::WZN; i += NT) {
		const int q = i % NQ, cp = (i / NQ) % NX, c = (i / (NQ * NX)) % NX, f = i / (NQ * NX * NX);
		const double e0 = (f >> 1) ? tab[S::ODZ + c * NQ + q] : tab[S::OVZ + c * NQ + q];
		const double e1 = (f & 1) ? tab[S::ODZ + cp * NQ + q] : tab[S::OVZ + cp * NQ + q];
		wz[i] = (float) (e0 * e1);
	}
	for (int i = tid; i < NB * KD; i += NT) {
		const int n = i / KD, kq = i % KD;
		double v = 0.0;
		if (n < L::NREAL && kq < L::KREAL) {
			const int bp = n % NX, b = (n / NX) % NX, ap = (n / (NX * NX)) % NX, a = n / (NX * NX * NX);
			const int q2 = kq % NQ, q1 = (kq / NQ) % NQ, k = kq / (NQ * NQ);
			const int fx = kLtFx[k], fy = kLtFy[k];
			const double xa = (fx >> 1) ? tab[S::ODX + a * NQ + q1] : tab[S::OVX + a * NQ + q1];
			const double xb = (fx & 1) ? tab[S::ODX + ap * NQ + q1] : tab[S::OVX + ap * NQ + q1];
			const double ya = (fy >> 1) ? tab[S::ODY + b * NQ + q2] : tab[S::OVY + b * NQ + q2];
			const double yb = (fy & 1) ? tab[S::ODY + bp * NQ + q2] : tab[S::OVY + bp * NQ + q2];
			v = xa * xb * ya * yb;
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
	uint32_t phase = 0;
	const int64_t nbatch = (kend - kbeg + EBT - 1) / EBT;

	for (int64_t bt = blockIdx.x; bt < nbatch; bt += gridDim.x) {
		const int64_t k0 = kbeg + bt * EBT;
		const int ne = (int) (kend - k0 < EBT ? kend - k0 : EBT);
		// ---- element data
		if (tid < EBT) {
			const bool live = tid < ne;
			s_m[tid] = live ? args.el_cnt[2 * (k0 + tid)] : 0;
			s_l[tid] = live ? args.el_cnt[2 * (k0 + tid) + 1] : 0;
			s_cg[tid] = live && args.ecoef ? args.ecoef[args.el_id[k0 + tid]] : 1.0;
		}
		for (int i = tid; i < EBT * 24; i += NT) {
			const int e = i / 24, r = i % 24;
			EL[e * L::E_SIZE + L::E_X + r] = e < ne ? args.xyz[3 * (int64_t) args.el_vtx[8 * (k0 + e) + r / 3] + r % 3] : 0.0;
		}
		for (int i = tid; i < EBT * NL; i += NT) {
			const int e = i / NL, j = i % NL;
			double *Eb = EL + e * L::E_SIZE;
			int *ei = reinterpret_cast<int *>(Eb + L::E_I);
			const int64_t g = (k0 + e) * NL + j;
			const int dof = e < ne ? args.el_dof[g] : -1;
			Eb[L::E_C + j] = e < ne ? args.el_coef[g] : 0.0;
			ei[j] = dof;
			ei[NL + j] = e < ne ? args.el_s[g] : 0;
			int64_t *cs = reinterpret_cast<int64_t *>(Eb + L::E_CS);
			cs[j] = dof >= 0 ? args.Ap[dof] : 0;
			cs[NL + j] = dof >= 0 ? args.Ap[dof + 1] : 0;
		}
		__syncthreads();
		// ---- trilinear map as monomials (as sf_monomials)
		for (int i = tid; i < EBT * 24; i += NT) {
			const int e = i / 24, mr = i % 24, mo = mr / 3, r = mr % 3;
			double *Eb = EL + e * L::E_SIZE;
			const int usex = mo == 1 || mo == 4 || mo == 5 || mo == 7;
			const int usey = mo == 2 || mo == 4 || mo == 6 || mo == 7;
			const int usez = mo == 3 || mo == 5 || mo == 6 || mo == 7;
			double c = 0.0;
#pragma unroll
			for (int v = 0; v < 8; v++) {
				const int bx = ((v + 1) >> 1) & 1, by = (v >> 1) & 1, bz = v >> 2;
				const int neg = (usex && !bx) ^ (usey && !by) ^ (usez && !bz);
				const double xv = Eb[L::E_X + 3 * v + r];
				c += neg ? -xv : xv;
			}
			Eb[L::E_M + mr] = 0.125 * c;
		}
		__syncthreads();
		// ---- geometry (FP64): terms 0..6 kept in FP32 for the matrix, the source in FP64
		for (int i = tid; i < EBT * NQ3; i += NT) {
			const int e = i / NQ3, q = i % NQ3;
			double *Eb = EL + e * L::E_SIZE;
			const int q1 = q / (NQ * NQ), q2 = (q / NQ) % NQ, q3 = q % NQ;
			const double w = tab[S::OWX + q1] * tab[S::OWY + q2] * tab[S::OWZ + q3];
			double t[8];
			sf_point_terms(Eb + L::E_M, tab[S::OQX + q1], tab[S::OQY + q2], tab[S::OQZ + q3], w, s_cg[e], args.lf,
			               args.lf_value, t);
			float *g = G32 + (size_t) e * 7 * NQ3;
#pragma unroll
			for (int r = 0; r < 6; r++) g[r * NQ3 + q] = (float) t[r];
			g[6 * NQ3 + q] = args.mass ? (float) t[6] : 0.0f;
			Eb[L::E_GS + q] = t[7];
		}
		__syncthreads();
		// ---- load vector (FP64) and stage 1 (FP32) into the A operand:
		//      T1_k[q1][q2][c][c'] = sum_q3 G_k(q) Wz_fz(k)[c][c'][q3]  (+ mass into k = 2)
		if (do_rhs)
			for (int i = tid; i < EBT * NX * NX; i += NT) {
				const int e = i / (NX * NX), ab = i % (NX * NX);
				double *Eb = EL + e * L::E_SIZE;
				sf_load_line<S>(tab, Eb + L::E_GS, ab / NX, ab % NX, Eb + L::E_F + ab * NX);
			}
		for (int i = tid; i < EBT * 6 * NQ * NQ; i += NT) {
			const int e = i / (6 * NQ * NQ), kq = i % (6 * NQ * NQ), k = kq / (NQ * NQ), q12 = kq % (NQ * NQ);
			const float *gp = G32 + ((size_t) e * 7 + k) * NQ3 + q12 * NQ;
			const float *gm = G32 + ((size_t) e * 7 + 6) * NQ3 + q12 * NQ;
			const float *w = wz + kLtFz[k] * NX * NX * NQ;
			const bool addm = k == 2;
			float g[NQ], h[NQ];
#pragma unroll
			for (int q3 = 0; q3 < NQ; q3++) {
				g[q3] = gp[q3];
				h[q3] = addm ? gm[q3] : 0.0f;
			}
#pragma unroll
			for (int cc = 0; cc < ROWS; cc++) {
				float s = 0.0f;
#pragma unroll
				for (int q3 = 0; q3 < NQ; q3++) s = fmaf(g[q3], w[cc * NQ + q3], s);
				if (addm) {
#pragma unroll
					for (int q3 = 0; q3 < NQ; q3++) s = fmaf(h[q3], wz[cc * NQ + q3], s);
				}
				const float hi = tc::to_tf32(s);
				const float lo = tc::to_tf32(s - hi);
				const uint32_t o = tc::kmaj_off32(e * ROWS + cc, kq, TM);
				*reinterpret_cast<float *>(aop_hi + o) = hi;
				*reinterpret_cast<float *>(aop_lo + o) = lo;
			}
		}
		if constexpr (KD > L::KREAL) {
			constexpr int PAD = KD - L::KREAL;     // K padding: zero (the B operand is zero there too)
			for (int i = tid; i < TM * PAD; i += NT) {
				const uint32_t o = tc::kmaj_off32(i / PAD, L::KREAL + i % PAD, TM);
				*reinterpret_cast<float *>(aop_hi + o) = 0.0f;
				*reinterpret_cast<float *>(aop_lo + o) = 0.0f;
			}
		}
		// ---- stages 2+3 on the tensor cores: 3xTF32, small terms first
		tc::fence_async_smem();
		tc::fence_before_sync();
		__syncthreads();
		if (tid == 0) {
			tc::fence_after_sync();
			constexpr uint32_t idesc = tc::instr_desc(TM, NB, tc::kTF32);
			constexpr uint32_t lbo_a = (TM / 8) * 128, lbo_b = (NB / 8) * 128;
#pragma unroll
			for (int pass = 0; pass < 3; pass++) {
				const unsigned char *pa = pass == 0 ? aop_lo : aop_hi;
				const unsigned char *pb = pass == 1 ? bop_lo : bop_hi;
#pragma unroll
				for (int st = 0; st < KD / 8; st++) {
					const uint64_t da = tc::smem_desc(pa + st * 2 * lbo_a, lbo_a, 128);
					const uint64_t db = tc::smem_desc(pb + st * 2 * lbo_b, lbo_b, 128);
					tc::mma_tf32(tmem, da, db, idesc, pass > 0 || st > 0);
				}
			}
			tc::mma_commit(&bar_mma);
		}
		bool ok = mbar_wait_bounded(&bar_mma, phase, args.status, args.wait_limit);
		if (!ok) mbar_wait_bounded(&bar_mma, phase, nullptr, 1u << 26);   // no MMA left in flight
		phase ^= 1u;
		if (!__syncthreads_and(ok ? 1 : 0)) break;
		tc::fence_after_sync();
		// ---- epilogue: TMEM row (e, c, c') -> A[(a,b,c)][(a',b',c')] (FP64, shared memory)
		{
			constexpr int NCH = NB / 16, CH0 = (NCH + 1) / 2;
			const int quarter = warp & 3, half = warp >> 2;
			const int r = quarter * 32 + lane, e = r / ROWS, cc = r % ROWS, c = cc / NX, cp = cc % NX;
			const bool live = e < ne;
			for (int ch = half ? CH0 : 0; ch < (half ? NCH : CH0); ch++) {
				float v[16];
				tc::tmem_ld16(tmem + ((uint32_t) (quarter * 32) << 16) + (uint32_t) (ch * 16), v);
#pragma unroll
				for (int j = 0; j < 16; j++) {
					const int n = ch * 16 + j;
					if (live && n < L::NREAL) {
						const int bp = n % NX, b = (n / NX) % NX, ap = (n / (NX * NX)) % NX, a = n / (NX * NX * NX);
						Afp[(size_t) e * NL2 + ((a * NX + b) * NX + c) * NL + (ap * NX + bp) * NX + cp] = (double) v[j];
					}
				}
			}
		}
		tc::fence_before_sync();
		__syncthreads();
		// ---- scatter into the CSC matrix (colour-exclusive posted adds) and the load vector
		if (args.Ax) {
			for (int p = tid; p < EBT * NL2; p += NT) {
				const int e = p / NL2, pp = p % NL2, b = pp / NL, a = pp % NL;
				const int m = s_m[e];
				if (e >= ne || a >= m || b >= m) continue;
				const double *Eb = EL + e * L::E_SIZE;
				const int *ei = reinterpret_cast<const int *>(Eb + L::E_I);
				const int64_t *cs = reinterpret_cast<const int64_t *>(Eb + L::E_CS);
				const int sa = ei[NL + a], sb = ei[NL + b];
				const double *A = Afp + (size_t) e * NL2;
				const double val = Eb[L::E_C + a] * Eb[L::E_C + b] * (A[sa * NL + sb] + A[sb * NL + sa]);
				const int64_t t = cs[b] + (int64_t) args.el_off[(k0 + e) * NL2 + b * NL + a];
				if (t < cs[NL + b]) posted_add(args.Ax + t, val);
				else if (cs[NL + b] > cs[b]) atomicOr(args.status, kErrBounds);   // empty: column not owned
			}
		}
		// ---- Dirichlet lifting in FP64, matrix-free, for the elements that have
		// lifting functions (only with the matrix: src/discretization.cc:296-317):
		// g = sum_j c_j phi_j; (K g)_i = sum_q grad phi_i . G grad g + M phi_i g,
		// with G and M the full symmetric factors (2 x the halved diagonal terms);
		// F_i -= (K g)_i
		if (do_rhs && args.Ax) {
			double *lw = reinterpret_cast<double *>(G32);      // 4 x NQ3: G grad g, M g (G32 is free now)
			for (int e = 0; e < ne; e++) {
				const int m = s_m[e], nlift = s_l[e];
				if (nlift == 0) continue;
				double *Eb = EL + e * L::E_SIZE;
				const int *ei = reinterpret_cast<const int *>(Eb + L::E_I);
				for (int q = tid; q < NQ3; q += NT) {
					const int q1 = q / (NQ * NQ), q2 = (q / NQ) % NQ, q3 = q % NQ;
					double g = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
					for (int j = m; j < m + nlift; j++) {
						const int sj = ei[NL + j], aj = sj / (NX * NX), bj = (sj / NX) % NX, cj = sj % NX;
						const double c = Eb[L::E_C + j];
						const double vx = tab[S::OVX + aj * NQ + q1], dx = tab[S::ODX + aj * NQ + q1];
						const double vy = tab[S::OVY + bj * NQ + q2], dy = tab[S::ODY + bj * NQ + q2];
						const double vz = tab[S::OVZ + cj * NQ + q3], dz = tab[S::ODZ + cj * NQ + q3];
						g += c * vx * vy * vz;
						gx += c * dx * vy * vz;
						gy += c * vx * dy * vz;
						gz += c * vx * vy * dz;
					}
					const double w = tab[S::OWX + q1] * tab[S::OWY + q2] * tab[S::OWZ + q3];
					double t[8];
					sf_point_terms(Eb + L::E_M, tab[S::OQX + q1], tab[S::OQY + q2], tab[S::OQZ + q3], w, s_cg[e], args.lf,
					               args.lf_value, t);
					lw[q] = 2.0 * t[0] * gx + t[3] * gy + t[4] * gz;
					lw[NQ3 + q] = t[3] * gx + 2.0 * t[1] * gy + t[5] * gz;
					lw[2 * NQ3 + q] = t[4] * gx + t[5] * gy + 2.0 * t[2] * gz;
					lw[3 * NQ3 + q] = args.mass ? 2.0 * t[6] * g : 0.0;
				}
				__syncthreads();
				for (int a = tid; a < m; a += NT) {
					const int sa = ei[NL + a], ai = sa / (NX * NX), bi = (sa / NX) % NX, ci = sa % NX;
					double y = 0.0;
					for (int q = 0; q < NQ3; q++) {
						const int q1 = q / (NQ * NQ), q2 = (q / NQ) % NQ, q3 = q % NQ;
						const double vx = tab[S::OVX + ai * NQ + q1], dx = tab[S::ODX + ai * NQ + q1];
						const double vy = tab[S::OVY + bi * NQ + q2], dy = tab[S::ODY + bi * NQ + q2];
						const double vz = tab[S::OVZ + ci * NQ + q3], dz = tab[S::ODZ + ci * NQ + q3];
						y += dx * vy * vz * lw[q] + vx * dy * vz * lw[NQ3 + q] + vx * vy * dz * lw[2 * NQ3 + q] +
						     vx * vy * vz * lw[3 * NQ3 + q];
					}
					Eb[L::E_F + sa] -= y;
				}
				__syncthreads();
			}
		}
		if (do_rhs) {
			for (int i = tid; i < EBT * NL; i += NT) {
				const int e = i / NL, a = i % NL;
				if (e >= ne || a >= s_m[e]) continue;
				const double *Eb = EL + e * L::E_SIZE;
				const int *ei = reinterpret_cast<const int *>(Eb + L::E_I);
				const int sa = ei[NL + a];
				posted_add(args.rhs + ei[a], Eb[L::E_F + sa] * Eb[L::E_C + a]);
			}
		}
		__syncthreads();
	}
	__syncthreads();
	tc::fence_after_sync();
	if (warp == 0) tc::tmem_dealloc(tmem, L::ACC);
}

} // namespace h3dg
