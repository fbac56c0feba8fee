// FP64 assembly with the reference's stock quadrature (uniform orders p <= 3).
//
// The stock forms int_grad_u_grad_v and int_u_v (src/integrals/h1.h:115-177)
// integrate every pair (u, v) with its own rule: order(u) + order(v) + (1,1,1)
// per direction (the inverse map's order of a hexahedron, src/refmap.cc:140),
// capped at 24, where the 1D order of Lobatto function k is max(k, 1)
// (src/shapeset/lobatto.cc:23) and a rule of order o has o / 2 + 1 Gauss
// points.  int_F_v uses the maximal order 24: 13 points per direction.
//
// At p <= 3 every pair rule has 2 .. p+1 points per direction, so all of them
// are sub-blocks of one combined tensor grid whose 1D point list is the
// concatenation of those rules (T = 2 + .. + (p+1) points per direction).
// Per element the geometric factors are evaluated once on that grid (FP64,
// as RefMap::calc_inv_ref_map, src/refmap.cc:177-231) and on the 13^3 grid
// of the load vector; then one thread per canonical pair (i <= j) sums
//     K_ij = sum_q G(q) grad phi_i . grad phi_j (+ M phi_i phi_j)
// over the pair's own sub-block (the full symmetric form).  The scatter, the
// Dirichlet lifting and the load vector are those of k_assemble_fp64:
// colour-exclusive, stream-ordered posted adds, bitwise reproducible.
#pragma once

#include "asm_fp64.cuh"

namespace h3dg {

template <int P>
struct StockShape {
	static constexpr int NX = P + 1, NL = NX * NX * NX;
	static constexpr int T = (P + 1) * (P + 2) / 2 - 1;      // combined points per direction
	static constexpr int T3 = T * T * T;
	static constexpr int R = 13, R3 = R * R * R;             // int_F_v: order 24
	// 1D tables blob: combined points / weights / values / derivatives, then the 13-point rule
	static constexpr int OQC = 0, OWC = T, OVC = 2 * T, ODC = OVC + NX * T;
	static constexpr int OQ13 = ODC + NX * T, OW13 = OQ13 + R, OV13 = OW13 + R;
	static constexpr int TAB = OV13 + NX * R, TABP = (TAB + 1) & ~1;
	// shared memory (doubles)
	static constexpr int S_TAB = 0;
	static constexpr int S_G = S_TAB + TABP;                 // 7 x T3 term weights
	static constexpr int S_R = S_G + 7 * T3;                 // R3 source weights (w det f)
	static constexpr int S_K = S_R + R3;                     // NL x NL element matrix (canonical)
	static constexpr int S_F = S_K + NL * NL;                // NL load vector (canonical)
	static constexpr int S_X = S_F + NL, S_M = S_X + 24, S_C = S_M + 24;
	static constexpr int S_I = S_C + NL;                     // ints: dof NL, shape NL
	static constexpr int S_CS = S_I + NL;                    // int64 column starts, ends
	static constexpr int SMEM_DOUBLES = S_CS + 2 * NL;
	static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};

// Gauss points of the pair rule of 1D Lobatto indices (k, k'), and where they
// start in the combined point list
__device__ __forceinline__ int stock_npts(int k, int kp) {
	const int o = (k < 2 ? 1 : k) + (kp < 2 ? 1 : kp) + 1;
	return (o > 24 ? 24 : o) / 2 + 1;
}
__device__ __forceinline__ int stock_start(int n) { return n * (n - 1) / 2 - 1; }

template <int P, int NT>
__global__ void __launch_bounds__(NT) k_assemble_stock(KArgs args, int64_t kbeg, int64_t kend) {
	using S = StockShape<P>;
	constexpr int NX = S::NX, NL = S::NL, T = S::T, T3 = S::T3, R = S::R, R3 = S::R3;
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	__shared__ int s_m, s_l;
	__shared__ double s_cg;
	double *tab = sm + S::S_TAB, *G = sm + S::S_G, *Rw = sm + S::S_R, *K = sm + S::S_K, *F = sm + S::S_F;
	double *X = sm + S::S_X, *Mo = sm + S::S_M, *cf = sm + S::S_C;
	int *ei = reinterpret_cast<int *>(sm + S::S_I);
	int64_t *cs = reinterpret_cast<int64_t *>(sm + S::S_CS);
	const int tid = threadIdx.x;
	if (!stage_tables(tab, args.tables, args.table_bytes, &bar, args.status, args.wait_limit)) return;
	const double *Qc = tab + S::OQC, *Wc = tab + S::OWC, *Vc = tab + S::OVC, *Dc = tab + S::ODC;
	const double *Q13 = tab + S::OQ13, *W13 = tab + S::OW13, *V13 = tab + S::OV13;
	const bool do_rhs = args.rhs && args.lf;

	for (int64_t k = kbeg + blockIdx.x; k < kend; k += gridDim.x) {
		// ---- element data
		if (tid == 0) {
			s_m = args.el_cnt[2 * k];
			s_l = args.el_cnt[2 * k + 1];
			s_cg = args.ecoef ? args.ecoef[args.el_id[k]] : 1.0;
		}
		if (tid < 24) X[tid] = args.xyz[3 * (int64_t) args.el_vtx[8 * k + tid / 3] + tid % 3];
		for (int j = tid; j < NL; j += NT) {
			const int dof = args.el_dof[k * NL + j];
			cf[j] = args.el_coef[k * NL + j];
			ei[j] = dof;
			ei[NL + j] = args.el_s[k * NL + j];
			cs[j] = dof >= 0 ? args.Ap[dof] : 0;
			cs[NL + j] = dof >= 0 ? args.Ap[dof + 1] : 0;
		}
		__syncthreads();
		// ---- trilinear map as monomials (as sf_monomials)
		if (tid < 24) {
			const int mo = tid / 3, r = tid % 3;
			const int usex = mo == 1 || mo == 4 || mo == 5 || mo == 7;
			const int usey = mo == 2 || mo == 4 || mo == 6 || mo == 7;
			const int usez = mo == 3 || mo == 5 || mo == 6 || mo == 7;
			double c = 0.0;
#pragma unroll
			for (int v = 0; v < 8; v++) {
				const int bx = ((v + 1) >> 1) & 1, by = (v >> 1) & 1, bz = v >> 2;
				const int neg = (usex && !bx) ^ (usey && !by) ^ (usez && !bz);
				c += neg ? -X[3 * v + r] : X[3 * v + r];
			}
			Mo[tid] = 0.125 * c;
		}
		__syncthreads();
		// ---- geometry: term weights on the combined grid, source weights on the 13^3 grid
		for (int i = tid; i < T3 + (do_rhs ? R3 : 0); i += NT) {
			double t[8];
			if (i < T3) {
				const int ix = i / (T * T), iy = (i / T) % T, iz = i % T;
				sf_point_terms(Mo, Qc[ix], Qc[iy], Qc[iz], Wc[ix] * Wc[iy] * Wc[iz], s_cg, 0, 0.0, t);
#pragma unroll
				for (int r = 0; r < 7; r++) G[r * T3 + i] = t[r];
			}
			else {
				const int q = i - T3, q1 = q / (R * R), q2 = (q / R) % R, q3 = q % R;
				sf_point_terms(Mo, Q13[q1], Q13[q2], Q13[q3], W13[q1] * W13[q2] * W13[q3], s_cg, args.lf, args.lf_value, t);
				Rw[q] = t[7];
			}
		}
		__syncthreads();
		// ---- element matrix, one canonical pair (i <= j) per thread, each on its own rule
		for (int p = tid; p < NL * NL; p += NT) {
			const int si = p / NL, sj = p % NL;
			if (si > sj) continue;
			const int a = si / (NX * NX), b = (si / NX) % NX, c = si % NX;
			const int a2 = sj / (NX * NX), b2 = (sj / NX) % NX, c2 = sj % NX;
			const int nx = stock_npts(a, a2), ny = stock_npts(b, b2), nz = stock_npts(c, c2);
			const int x0 = stock_start(nx), y0 = stock_start(ny), z0 = stock_start(nz);
			double s = 0.0;
			for (int ix = x0; ix < x0 + nx; ix++) {
				const double vxa = Vc[a * T + ix], dxa = Dc[a * T + ix], vxb = Vc[a2 * T + ix], dxb = Dc[a2 * T + ix];
				for (int iy = y0; iy < y0 + ny; iy++) {
					const double vya = Vc[b * T + iy], dya = Dc[b * T + iy], vyb = Vc[b2 * T + iy], dyb = Dc[b2 * T + iy];
					for (int iz = z0; iz < z0 + nz; iz++) {
						const double vza = Vc[c * T + iz], dza = Dc[c * T + iz], vzb = Vc[c2 * T + iz], dzb = Dc[c2 * T + iz];
						const int q = (ix * T + iy) * T + iz;
						const double gxi = dxa * vya * vza, gyi = vxa * dya * vza, gzi = vxa * vya * dza, vi = vxa * vya * vza;
						const double gxj = dxb * vyb * vzb, gyj = vxb * dyb * vzb, gzj = vxb * vyb * dzb, vj = vxb * vyb * vzb;
						s += 2.0 * (G[q] * gxi * gxj + G[T3 + q] * gyi * gyj + G[2 * T3 + q] * gzi * gzj) +
						     G[3 * T3 + q] * (gxi * gyj + gyi * gxj) + G[4 * T3 + q] * (gxi * gzj + gzi * gxj) +
						     G[5 * T3 + q] * (gyi * gzj + gzi * gyj) + (args.mass ? 2.0 * G[6 * T3 + q] * vi * vj : 0.0);
					}
				}
			}
			K[si * NL + sj] = s;
			K[sj * NL + si] = s;
		}
		// ---- load vector on the 13-point rule, by sum factorisation: thread (a, b)
		if (do_rhs)
			for (int ab = tid; ab < NX * NX; ab += NT) {
				const int a = ab / NX, b = ab % NX;
				double fc[NX];
#pragma unroll
				for (int c = 0; c < NX; c++) fc[c] = 0.0;
				for (int q1 = 0; q1 < R; q1++) {
					double s1[NX];
#pragma unroll
					for (int c = 0; c < NX; c++) s1[c] = 0.0;
					for (int q2 = 0; q2 < R; q2++) {
						const double vy = V13[b * R + q2];
						for (int q3 = 0; q3 < R; q3++) {
							const double w = Rw[(q1 * R + q2) * R + q3] * vy;
#pragma unroll
							for (int c = 0; c < NX; c++) s1[c] += w * V13[c * R + q3];
						}
					}
					const double vx = V13[a * R + q1];
#pragma unroll
					for (int c = 0; c < NX; c++) fc[c] += vx * s1[c];
				}
#pragma unroll
				for (int c = 0; c < NX; c++) F[ab * NX + c] = fc[c];
			}
		__syncthreads();
		// ---- scatter (colour-exclusive posted adds) and load vector with lifting
		const int m = s_m;
		if (args.Ax)
			for (int p = tid; p < NL * NL; p += NT) {
				const int b = p / NL, a = p % NL;
				if (a >= m || b >= m) continue;
				const double val = cf[a] * cf[b] * K[ei[NL + a] * NL + ei[NL + b]];
				const int64_t t = cs[b] + (int64_t) args.el_off[(k * NL + b) * NL + a];
				if (t < cs[NL + b]) posted_add(args.Ax + t, val);
				else if (cs[NL + b] > cs[b]) atomicOr(args.status, kErrBounds);   // empty: column not owned
			}
		if (do_rhs)
			for (int a = tid; a < m; a += NT) {
				const int sa = ei[NL + a];
				const double ca = cf[a];
				double lr = 0.0;
				for (int j = m; j < m + (args.Ax ? s_l : 0); j++)      // lifting only with the matrix (src/discretization.cc:296-317)
					lr -= ca * cf[j] * K[sa * NL + ei[NL + j]];
				lr += F[sa] * ca;
				posted_add(args.rhs + ei[a], lr);
			}
		__syncthreads();
	}
}

} // namespace h3dg
