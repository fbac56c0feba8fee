// FP64 assembly for high orders on the FP64 tensor cores (DMMA,
// mma.sync.m16n8k8.f64): the element matrix as two back-to-back GEMMs per
// (test z index c, trial z index c'), exact FP64 arithmetic.
//
// Same mathematics as k_assemble_fp64_ho (src/integrals/h1.h:115-177 per pair,
// restated as sum factorisation).  For a pair (c, c'):
//   stage 1 (FP64 FMA): T1_kk[q1][q2] = sum_q3 G_g(kk) E_z^alpha[c][q3] E_z^beta[c'][q3]
//     for the 9 gradient products kk (+ mass into kk = 2), written straight
//     into the B-fragment layout of stage 2;
//   stage 2 (DMMA): V^T[bb][nu] = sum_kappa W[bb][kappa] T1[kappa][nu],
//     bb = (b, b') the y indices, kappa = (y flag, q2), nu = (x class f, q1):
//     W[bb][(fy, q2)] = E_y^(fy>>1)[b][q2] E_y^(fy&1)[b'][q2] is the same for
//     every element: its fragments are formed once per CTA;
//   stage 3 (DMMA): K[(a,b,c)][(a',b',c')] = sum_nu V^T[bb][nu] P[nu][(a', a)],
//     P[(f, q1)][(a', a)] = E_x^(f>>1)[a][q1] E_x^(f&1)[a'][q1], a fixed table.
//     The stage-2 accumulators are the stage-3 A fragments as they stand: the
//     k order of stage 3 pairs the two nu columns a thread holds (2t, 2t+1)
//     into its two k slots (t, t+4), and P is stored in that order.
// Work items: whole elements, and from args.split_from on half elements
// (trial z indices c' below / from (NX + 1) / 2, the load vector with the
// first half), so that the last round of a colour launch spreads over twice
// as many SMs.
// Pairs run trial z index c' outermost: the 81 CSC columns (a', b', c') of a
// c' receive all their rows within NX consecutive pairs, so the sectors a CTA
// writes stay in L2 until they are complete (about 0.5 MB per CTA at p = 8).
// Padding (bb and (a', a) to whole tiles, kappa and nu to multiples of 8)
// multiplies zeros; the (f, fy) pairs no product uses are zero tiles of T1
// and their MMAs are skipped at compile time.
// Scatter: every result goes to Ax through a per-plan stream in the kernel's
// output order (k_build_offd): row offset in the column, a skip marker, and
// a first-touch flag (the first colour that reaches a slot stores instead of
// adding, so Ax needs no zero-fill).  The stream is validated against the
// column lengths when it is built.  Colour-exclusive, stream-ordered posts:
// bitwise reproducible run to run.
// Dirichlet lifting and the load vector: matrix-free FP64 (ho_rhs), as in the
// other high-order kernels.
#pragma once

#include "asm_fp64_ho.cuh"
#include "asm_ho_tc.cuh"

namespace h3dg {

__device__ __forceinline__ void dmma16x8x8(double (&d)[4], double a0, double a1, double a2, double a3, double b0, double b1) {
	asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
	             : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
	             : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// y flag and x class of the 9 stage-1 products (as in k_assemble_fp64_ho)
__host__ __device__ constexpr int dm_fy(int kk) { return kk == 1 ? 3 : kk == 3 || kk == 8 ? 1 : kk == 4 || kk == 7 ? 2 : 0; }
__host__ __device__ constexpr int dm_cls(int kk) { return kk == 0 ? 3 : kk == 3 || kk == 5 ? 2 : kk == 4 || kk == 6 ? 1 : 0; }
// product of (x class f, y flag fy), or -1
__host__ __device__ constexpr int dm_kk(int f, int fy) {
	for (int kk = 0; kk < 9; kk++)
		if (dm_cls(kk) == f && dm_fy(kk) == fy) return kk;
	return -1;
}

// PHV: (c, c') pairs per iteration, 0 = as many as make 12 warps; fewer
// pairs shrink the CTA (threads and fragment buffers) so that two fit per SM
template <int P, int NQ, int PHV = 0>
struct DmShape {
	using H = HoShape<P, P, P, NQ, NQ, NQ>;
	static constexpr int NX = P + 1, NL = H::NL, NQ3 = H::NQ;
	static constexpr int NB = NX * NX;                       // (b, b') and (a', a)
	static constexpr int MT = (NB + 15) / 16;                // stage-2/3 M tiles (bb)
	static constexpr int NT3 = (NB + 7) / 8;                 // stage-3 N tiles ((a', a))
	static constexpr int KK = 4 * NQ;                        // kappa and nu extent
	static constexpr int KS = (KK + 7) / 8;                  // k steps / n tiles over them
	static constexpr int PH = PHV > 0 ? PHV : MT >= 12 ? 1 : 12 / MT;   // (c, c') pairs per iteration
	static constexpr int NW = MT * PH, NT = 32 * NW;
	static constexpr int MINB = PHV > 0 ? 2 : 1;             // CTAs per SM the registers must allow
	static constexpr int PAIRS = NX * NX, ITERS = (PAIRS + PH - 1) / PH;
	static constexpr int B2SZ = KS * KS * 64;                // one pair's stage-2 B fragments (doubles)
	static constexpr int PSZ = KS * NT3 * 64;                // stage-3 B fragments (P)
	static constexpr int EPE = PAIRS * MT * NT3 * 128;       // scatter stream entries per element
	static constexpr int BUF = 2 * PH * B2SZ;                // double-buffered
	static constexpr int UNION = ((BUF > H::MF ? BUF : H::MF) + 15) / 16 * 16;   // keeps P 16-byte aligned
	// shared memory (doubles)
	static constexpr int S_TAB = 0;
	static constexpr int S_G = S_TAB + H::TABP;
	static constexpr int S_U = S_G + 8 * NQ3;
	static constexpr int S_P = S_U + UNION;
	static constexpr int AWSZ = MT * KS * 128;               // stage-2 A fragments (W), per M tile
	static constexpr int S_AW = S_P + PSZ;
	static constexpr int S_X = S_AW + AWSZ;
	static constexpr int S_M = S_X + 24;
	static constexpr int S_C = S_M + 24;
	static constexpr int S_CS = S_C + NL;
	static constexpr int S_CE = S_CS + NL;
	static constexpr int S_D = S_CE + NL;
	static constexpr int SMEM_DOUBLES = S_D + (NL + 1) / 2 + 2;
	static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
	static_assert(SMEM_BYTES <= 227 * 1024, "DMMA kernel shared memory");
	// stage-2 tile (k step ks, n tile j) holds no product: skipped
	__host__ __device__ static constexpr bool zero_tile(int ks, int j) {
		for (int kq = ks * 8; kq < ks * 8 + 8; kq++)
			for (int nu = j * 8; nu < j * 8 + 8; nu++)
				if (kq < KK && nu < KK && dm_kk(nu / NQ, kq / NQ) >= 0) return false;
		return true;
	}
};

// Position (in doubles) of stage-2 B element (kappa, nu) inside one pair's buffer:
// b0 = B[k = t][n = g], b1 = B[k = t + 4][n = g] of tile (kappa / 8, nu / 8), lane g * 4 + t
template <class S>
__device__ __forceinline__ int dm_b2_pos(int kappa, int nu) {
	const int ks = kappa >> 3, tt = kappa & 7, j = nu >> 3, g = nu & 7;
	return ((ks * S::KS + j) * 32 + g * 4 + (tt & 3)) * 2 + (tt >> 2);
}

// Decode of one stream entry (element-local): pair, M tile, N tile, lane, register
// -> test function i and trial function j (-1 for padding)
template <class S>
__host__ __device__ __forceinline__ void dm_entry(int pair, int mt, int nt, int lane, int r, int &i, int &j) {
	constexpr int NX = S::NX, NB = S::NB;
	const int g = lane >> 2, t = lane & 3;
	const int bb = mt * 16 + g + 8 * (r >> 1), aa = nt * 8 + 2 * t + (r & 1);
	if (bb >= NB || aa >= NB) {
		i = j = -1;
		return;
	}
	const int c2 = pair / NX, c = pair % NX;
	const int b = bb / NX, b2 = bb % NX, a2 = aa / NX, a = aa % NX;
	i = (a * NX + b) * NX + c;
	j = (a2 * NX + b2) * NX + c2;
}

template <int P, int NQ, int PHV>
__global__ void __launch_bounds__(DmShape<P, NQ, PHV>::NT, DmShape<P, NQ, PHV>::MINB) k_assemble_fp64_dm(KArgsHO args, int64_t kbeg, int64_t kend) {
	using S = DmShape<P, NQ, PHV>;
	using H = typename S::H;
	constexpr int NX = S::NX, NQ3 = S::NQ3, NT = S::NT, MT = S::MT, NT3 = S::NT3, KS = S::KS, KK = S::KK;
	constexpr int PH = S::PH, NB = S::NB;
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	__shared__ int s_nlift;
	const double *tab = sm + S::S_TAB;
	double *G = sm + S::S_G, *U = sm + S::S_U, *Pf = sm + S::S_P;
	double *X = sm + S::S_X, *Mo = sm + S::S_M, *cc = sm + S::S_C;
	int64_t *cs = reinterpret_cast<int64_t *>(sm + S::S_CS), *ce = reinterpret_cast<int64_t *>(sm + S::S_CE);
	int *cd = reinterpret_cast<int *>(sm + S::S_D);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int g = lane >> 2, t = lane & 3;
	if (!stage_tables(sm + S::S_TAB, args.tables, args.table_bytes, &bar, args.status)) return;
	const double *Vx = tab + H::OVX, *Dx = tab + H::ODX, *Vy = tab + H::OVY, *Dy = tab + H::ODY;
	const double *Vz = tab + H::OVZ, *Dz = tab + H::ODZ;
	const bool do_rhs = args.rhs && args.lf;

	// ---- per CTA: stage-3 B fragments P (k order: slot t <-> nu = 8j + 2t, slot t + 4 <-> 8j + 2t + 1)
	for (int e = tid; e < S::PSZ; e += NT) {
		const int half = e & 1, ln = (e >> 1) & 31, tile = e >> 6;
		const int j = tile / NT3, nt = tile % NT3;
		const int aa = nt * 8 + (ln >> 2), nu = 8 * j + 2 * (ln & 3) + half;
		double v = 0.0;
		if (aa < NB && nu < KK) {
			const int f = nu / NQ, q1 = nu % NQ, a2 = aa / NX, a = aa % NX;
			v = ((f >> 1) ? Dx : Vx)[a * NQ + q1] * ((f & 1) ? Dx : Vx)[a2 * NQ + q1];
		}
		Pf[e] = v;
	}
	// ---- per CTA: stage-2 A fragments W, [M tile][k step][lane][4]
	double *Aw = sm + S::S_AW;
	for (int e = tid; e < S::AWSZ; e += NT) {
		const int r = e & 3, ln = (e >> 2) & 31, tile = e >> 7;
		const int mt_ = tile / KS, ks = tile % KS;
		const int bb = mt_ * 16 + (ln >> 2) + 8 * (r & 1), kq = ks * 8 + (ln & 3) + 4 * (r >> 1);
		double v = 0.0;
		if (bb < NB && kq < KK) {
			const int fy = kq / NQ, q2 = kq % NQ, b = bb / NX, b2 = bb % NX;
			v = ((fy >> 1) ? Dy : Vy)[b * NQ + q2] * ((fy & 1) ? Dy : Vy)[b2 * NQ + q2];
		}
		Aw[e] = v;
	}
	const int mt = warp % MT, ph = warp / MT;
	const double *aw = Aw + (mt * KS * 32 + lane) * 4;
	// scatter: test / trial y parts of this warp's rows bb = mt 16 + g (+ 8)
	int rb[2], cb[2];
#pragma unroll
	for (int h = 0; h < 2; h++) {
		const int bb = mt * 16 + g + 8 * h;
		rb[h] = (bb / NX) * NX;
		cb[h] = (bb % NX) * NX;
	}
	__syncthreads();

	// stage 1 for the pairs of iteration it into buffer set (it & 1): thread
	// group (pair slot, product) walks the (q1, q2) points
	constexpr int GROUPS = PH * 9, TPG = NT / GROUPS;
	const int grp = tid / TPG, gl = tid % TPG;
	int p0 = 0, p1 = S::PAIRS, iters = S::ITERS;     // pair range of the current work item
	auto stage1 = [&](int it) {
		if (grp >= GROUPS) return;
		const int p_slot = grp / 9, kk = grp % 9;
		const int pair = p0 + it * PH + p_slot;
		if (pair >= p1) return;
		const int c2 = pair / NX, c = pair % NX;
		const int fz = kHoFz[kk];
		const double *ea = ((fz >> 1) ? Dz : Vz) + c * NQ, *eb = ((fz & 1) ? Dz : Vz) + c2 * NQ;
		double ez[NQ], em[NQ];
		const bool addm = kk == 2 && args.mass;
#pragma unroll
		for (int q3 = 0; q3 < NQ; q3++) {
			ez[q3] = ea[q3] * eb[q3];
			em[q3] = addm ? Vz[c * NQ + q3] * Vz[c2 * NQ + q3] : 0.0;
		}
		const double *gp = G + kHoG[kk] * NQ3, *gm = G + 6 * NQ3;
		double *buf = U + ((it & 1) * PH + p_slot) * S::B2SZ;
		const int fy = dm_fy(kk), f = dm_cls(kk);
		for (int q12 = gl; q12 < NQ * NQ; q12 += TPG) {
			const int q1 = q12 / NQ, q2 = q12 % NQ;
			double s = 0.0;
#pragma unroll
			for (int q3 = 0; q3 < NQ; q3++) s += gp[q12 * NQ + q3] * ez[q3];
			if (addm) {
#pragma unroll
				for (int q3 = 0; q3 < NQ; q3++) s += gm[q12 * NQ + q3] * em[q3];
			}
			buf[dm_b2_pos<S>(fy * NQ + q2, f * NQ + q1)] = s;
		}
	};

	const int64_t nwhole = args.split_from - kbeg, items = nwhole + 2 * (kend - args.split_from);
	for (int64_t item = blockIdx.x; item < items; item += gridDim.x) {
		int half = -1;
		int64_t k = kbeg + item;
		if (item >= nwhole) {
			k = args.split_from + (item - nwhole) / 2;
			half = (int) ((item - nwhole) & 1);
		}
		constexpr int C2H = (NX + 1) / 2;
		p0 = half == 1 ? C2H * NX : 0;
		p1 = half == 0 ? C2H * NX : S::PAIRS;
		iters = (p1 - p0 + PH - 1) / PH;
		const double cgrad = ho_element_setup<H, NT>(args, k, X, Mo, cc, cd, cs, ce, &s_nlift);
		ho_geometry<H, NT>(args, tab, Mo, cgrad, G);
		if (do_rhs && half <= 0) ho_rhs<H, NT>(args, tab, G, U, cd, cc, cd, cc, s_nlift > 0 && args.Ax);
		if (!args.Ax) continue;
		// the fragment buffers share the work area with ho_rhs: clear them (positions
		// no product writes stay zero for the whole element)
		for (int e = tid; e < S::BUF; e += NT) U[e] = 0.0;
		__syncthreads();
		stage1(0);
		__syncthreads();
		const uint16_t *offd = args.offd + k * (int64_t) S::EPE;
		for (int it = 0; it < iters; it++) {
			// stage 1 of the next pairs: warps of even pair slots before their MMAs,
			// odd ones after, so that the DMMA pipe always has work queued
			if (!(ph & 1) && it + 1 < iters) stage1(it + 1);
			const int pair = p0 + it * PH + ph;
			if (pair < p1) {
				const double *buf = U + ((it & 1) * PH + ph) * S::B2SZ;
				// ---- stage 2: V^T (bb x nu) for this warp's M tile
				double v[KS][4];
#pragma unroll
				for (int j = 0; j < KS; j++)
#pragma unroll
					for (int r = 0; r < 4; r++) v[j][r] = 0.0;
#pragma unroll
				for (int ks = 0; ks < KS; ks++) {
					const double2 a01 = *reinterpret_cast<const double2 *>(aw + ks * 128);
					const double2 a23 = *reinterpret_cast<const double2 *>(aw + ks * 128 + 2);
#pragma unroll
					for (int j = 0; j < KS; j++) {
						if (S::zero_tile(ks, j)) continue;
						const double2 b = *reinterpret_cast<const double2 *>(buf + ((ks * KS + j) * 32 + lane) * 2);
						dmma16x8x8(v[j], a01.x, a01.y, a23.x, a23.y, b.x, b.y);
					}
				}
				// ---- stage 3, NG N tiles of (a', a) per group (independent accumulators),
				// software-pipelined: the MMAs of the next group are issued before the
				// scatter of the current one; the stream words are loaded with the MMAs.
				// Three tiles per group up to p = 6 (p = 5: 2.12 -> 1.95 ms on 16^3),
				// two above (three: p = 7 11.4 -> 11.6 ms, p = 8 unchanged)
				constexpr int NG = NX <= 7 ? 3 : 2;
				const int c2 = pair / NX, c = pair % NX;
				const uint16_t *od = offd + ((int64_t) (pair * MT + mt) * NT3) * 128 + lane * 4;
				auto mma_group = [&](int n0, double (&d)[NG][4], uint2 (&ow)[NG]) {
#pragma unroll
					for (int q = 0; q < NG; q++) {
						ow[q] = n0 + q < NT3 ? __ldcs(reinterpret_cast<const uint2 *>(od + (n0 + q) * 128)) : make_uint2(~0u, ~0u);
#pragma unroll
						for (int r = 0; r < 4; r++) d[q][r] = 0.0;
					}
#pragma unroll
					for (int j = 0; j < KS; j++)
#pragma unroll
						for (int q = 0; q < NG; q++)
							if (n0 + q < NT3) {
								const double2 b = *reinterpret_cast<const double2 *>(Pf + ((j * NT3 + n0 + q) * 32 + lane) * 2);
								dmma16x8x8(d[q], v[j][0], v[j][2], v[j][1], v[j][3], b.x, b.y);
							}
				};
				auto scatter_group = [&](int n0, const double (&d)[NG][4], const uint2 (&ow)[NG]) {
#pragma unroll
					for (int q = 0; q < NG; q++)
#pragma unroll
						for (int e = 0; e < 2; e++) {
							const int aa = (n0 + q) * 8 + 2 * t + e;
							const int ra = (aa % NX) * NX * NX + c, ca = (aa / NX) * NX * NX + c2;
#pragma unroll
							for (int h = 0; h < 2; h++) {
								const uint32_t w = h ? ow[q].y : ow[q].x;
								const uint32_t o = e ? w >> 16 : w & 0xFFFF;
								if (o == kOffSkip) continue;
								const int i = ra + rb[h], j = ca + cb[h];
								double *dst = args.Ax + cs[j] + (o & kOffMask);
								const double val = cc[i] * cc[j] * d[q][2 * h + e];
								if (o & kOffStore) posted_store(dst, val);
								else posted_add(dst, val);
							}
						}
				};
				double dA[NG][4], dB[NG][4];
				uint2 oA[NG], oB[NG];
				mma_group(0, dA, oA);
#pragma unroll 1
				for (int n0 = 0; n0 < NT3; n0 += 2 * NG) {
					if (n0 + NG < NT3) mma_group(n0 + NG, dB, oB);
					scatter_group(n0, dA, oA);
					if (n0 + 2 * NG < NT3) mma_group(n0 + 2 * NG, dA, oA);
					if (n0 + NG < NT3) scatter_group(n0 + NG, dB, oB);
				}
			}
			// the other half of the warps builds its share of the next pairs' stage 1 now
			if (ph & 1 && it + 1 < iters) stage1(it + 1);
			__syncthreads();
		}
	}
}

// Scatter stream of the DMMA kernel from the canonical position map: entry
// (element, pair, M tile, N tile, lane, register) -> row offset in column j,
// kOffSkip where (i, j) is padding or not a matrix entry, kOffStore on the
// first contribution (in launch order) to each Ax slot.  Positions are
// checked against their column here, once.
template <int P, int NQ>
__global__ void k_build_offd(const uint16_t *offc, const int32_t *cdof, const int64_t *Ap, int64_t kbeg, int64_t kend,
                             uint16_t *offd, int *status, uint8_t *touched, unsigned long long *stores) {
	using S = DmShape<P, NQ>;
	constexpr int NL = S::NL, MT = S::MT, NT3 = S::NT3;
	const int64_t total = (kend - kbeg) * (int64_t) S::EPE;
	unsigned long long nst = 0;
	for (int64_t e0 = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; e0 < total; e0 += (int64_t) gridDim.x * blockDim.x) {
		const int64_t e = kbeg * (int64_t) S::EPE + e0;
		const int64_t k = e / S::EPE;
		int rem = (int) (e % S::EPE);
		const int r = rem & 3, lane = (rem >> 2) & 31;
		rem >>= 7;
		const int nt = rem % NT3;
		rem /= NT3;
		const int mt = rem % MT, pair = rem / MT;
		int i, j;
		dm_entry<S>(pair, mt, nt, lane, r, i, j);
		uint16_t v = kOffSkip;
		if (i >= 0) {
			const int dj = cdof[k * NL + j];
			if (cdof[k * NL + i] >= 0 && dj >= 0) {
				v = offc[(k * NL + i) * NL + j];
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
		offd[e] = v;
	}
	if (stores && nst) atomicAdd(stores, nst);
}

} // namespace h3dg
