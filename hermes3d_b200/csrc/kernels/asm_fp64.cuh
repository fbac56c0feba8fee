// FP64 element-matrix + deterministic scatter, one element per CTA pass.
//
// Replaces the per-pair form calls of Discretization::assemble
// (src/discretization.cc:290-325) with int_grad_u_grad_v / int_u_v / int_F_v
// (src/integrals/h1.h:115-177), and the binary-search insert of
// UMFPackMatrix::update (src/linsolver/umfpack.cc:80-152).
//
// Element matrix.  With G_q = w_q det J_q J_q^-1 J_q^-T (times the element
// coefficient) the grad-grad matrix in the canonical tensor basis
// phi_abc = L_a(xi) L_b(eta) L_c(zeta) is
//     K_ij = sum_q sum_rs G_q[r][s] d_r phi_i(q) d_s phi_j(q).
// It is formed as K = A + A^T with
//     A = sum_r (G_rr/2) B_r^T B_r + sum_{r<s} G_rs B_r^T B_s  (+ (M/2) V^T V)
// and every one of the 7 terms is contracted by sum factorisation over the
// three quadrature directions (q3, then q2, then q1), because each factor
// d_r phi_i(q) is a product of 1D table entries.  Work per element is
// O(nq p^6) instead of the O(nq^3 p^6) of the dense per-pair loops.
//
// Scatter.  Entry (a, b) of the element's assembly list goes to
// Ax[Ap[dof_b] + off[b][a]] (CSC: column = trial DOF).  Elements of one
// colour share no DOF, so the read-modify-write needs no atomics and the
// summation order of every entry (colour order) is fixed: bitwise
// reproducible.  Dirichlet lifting follows src/discretization.cc:316-317,
// RHS follows :329-338 (lifting only enters the RHS when a linear form is
// set, as in the reference).
#pragma once

#include "common.cuh"

namespace h3dg {

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ>
struct SfShape {
	static constexpr int NX = PX + 1, NY = PY + 1, NZ = PZ + 1;
	static constexpr int NL = NX * NY * NZ;
	static constexpr int NQ = NQX * NQY * NQZ;
	// 1D tables blob: Vx Dx Vy Dy Vz Dz (k-major, q fastest) then q/w per direction
	static constexpr int OVX = 0, ODX = OVX + NX * NQX, OVY = ODX + NX * NQX, ODY = OVY + NY * NQY;
	static constexpr int OVZ = ODY + NY * NQY, ODZ = OVZ + NZ * NQZ;
	static constexpr int OQX = ODZ + NZ * NQZ, OWX = OQX + NQX, OQY = OWX + NQX, OWY = OQY + NQY;
	static constexpr int OQZ = OWY + NQY, OWZ = OQZ + NQZ;
	static constexpr int TAB = OWZ + NQZ;
	static constexpr int TABP = (TAB + 1) & ~1;
	// products W^f[k][k'][q] = E^(f>>1)[k][q] E^(f&1)[k'][q], E^0 = V, E^1 = D
	static constexpr int WX = 4 * NX * NX * NQX, WY = 4 * NY * NY * NQY, WZ = 4 * NZ * NZ * NQZ;
	static constexpr int T1N = NQX * NQY * NZ * NZ;
	static constexpr int T2N = NQX * NY * NY * NZ * NZ;
	// shared memory in doubles
	static constexpr int S_TAB = 0;
	static constexpr int S_W = S_TAB + TABP;
	static constexpr int S_G = S_W + WX + WY + WZ;          // 8 x NQ
	static constexpr int S_T1 = S_G + 8 * NQ;
	static constexpr int S_T2 = S_T1 + T1N;
	static constexpr int S_A = S_T2 + T2N;                  // NL x NL
	static constexpr int S_F = S_A + NL * NL;
	static constexpr int S_X = S_F + NL;                    // 24
	static constexpr int S_C = S_X + 24;                    // NL coefs
	static constexpr int S_I = S_C + NL;                    // ints: dof NL, s NL
	static constexpr int SMEM_DOUBLES = S_I + NL;           // 2 NL ints = NL doubles
	static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};

// flags of the 7 terms: per direction, f = 2*alpha + beta (alpha: test side
// differentiated, beta: trial side differentiated)
__device__ __constant__ int kTermFlags[7][3] = {
	{ 3, 0, 0 }, { 0, 3, 0 }, { 0, 0, 3 },   // xx yy zz
	{ 2, 1, 0 }, { 2, 0, 1 }, { 0, 2, 1 },   // xy xz yz
	{ 0, 0, 0 }                               // mass
};

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int NT>
__global__ void __launch_bounds__(NT) k_assemble_fp64(KArgs args, int64_t kbeg, int64_t kend) {
	using S = SfShape<PX, PY, PZ, NQX, NQY, NQZ>;
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NL = S::NL, NQ = S::NQ;
	constexpr int NACC = (NL * NL + NT - 1) / NT;
	extern __shared__ __align__(16) double sm[];
	__shared__ uint64_t bar;
	double *tab = sm + S::S_TAB;
	double *Wx = sm + S::S_W, *Wy = Wx + S::WX, *Wz = Wy + S::WY;
	double *G = sm + S::S_G;
	double *T1 = sm + S::S_T1, *T2 = sm + S::S_T2;
	double *A = sm + S::S_A, *F = sm + S::S_F, *X = sm + S::S_X, *ec = sm + S::S_C;
	int *edof = reinterpret_cast<int *>(sm + S::S_I);
	int *es = edof + NL;
	const int tid = threadIdx.x;

	if (!stage_tables(tab, args.tables, args.table_bytes, &bar, args.status)) return;

	// 1D product tables, once per CTA
	for (int i = tid; i < S::WX; i += NT) {
		int q = i % NQX, kk = (i / NQX) % NX, k = (i / (NQX * NX)) % NX, f = i / (NQX * NX * NX);
		double e0 = (f >> 1) ? tab[S::ODX + k * NQX + q] : tab[S::OVX + k * NQX + q];
		double e1 = (f & 1) ? tab[S::ODX + kk * NQX + q] : tab[S::OVX + kk * NQX + q];
		Wx[i] = e0 * e1;
	}
	for (int i = tid; i < S::WY; i += NT) {
		int q = i % NQY, kk = (i / NQY) % NY, k = (i / (NQY * NY)) % NY, f = i / (NQY * NY * NY);
		double e0 = (f >> 1) ? tab[S::ODY + k * NQY + q] : tab[S::OVY + k * NQY + q];
		double e1 = (f & 1) ? tab[S::ODY + kk * NQY + q] : tab[S::OVY + kk * NQY + q];
		Wy[i] = e0 * e1;
	}
	for (int i = tid; i < S::WZ; i += NT) {
		int q = i % NQZ, kk = (i / NQZ) % NZ, k = (i / (NQZ * NZ)) % NZ, f = i / (NQZ * NZ * NZ);
		double e0 = (f >> 1) ? tab[S::ODZ + k * NQZ + q] : tab[S::OVZ + k * NQZ + q];
		double e1 = (f & 1) ? tab[S::ODZ + kk * NQZ + q] : tab[S::OVZ + kk * NQZ + q];
		Wz[i] = e0 * e1;
	}
	__syncthreads();

	const int nterms = args.mass ? 7 : 6;
	for (int64_t k = kbeg + blockIdx.x; k < kend; k += gridDim.x) {
		// ---- element data
		if (tid < 24) X[tid] = args.xyz[3 * (int64_t) args.el_vtx[8 * k + tid / 3] + tid % 3];
		for (int i = tid; i < NL; i += NT) {
			ec[i] = args.el_coef[k * NL + i];
			edof[i] = args.el_dof[k * NL + i];
			es[i] = args.el_s[k * NL + i];
		}
		const int mcnt = args.el_cnt[2 * k], lcnt = args.el_cnt[2 * k + 1];
		const double cgrad = args.ecoef ? args.ecoef[args.el_id[k]] : 1.0;
		__syncthreads();

		// ---- geometry at the quadrature points -> term weights
		for (int q = tid; q < NQ; q += NT) {
			const int q1 = q / (NQY * NQZ), q2 = (q / NQZ) % NQY, q3 = q % NQZ;
			const double vx[2] = { tab[S::OVX + q1], tab[S::OVX + NQX + q1] };
			const double dx[2] = { tab[S::ODX + q1], tab[S::ODX + NQX + q1] };
			const double vy[2] = { tab[S::OVY + q2], tab[S::OVY + NQY + q2] };
			const double dy[2] = { tab[S::ODY + q2], tab[S::ODY + NQY + q2] };
			const double vz[2] = { tab[S::OVZ + q3], tab[S::OVZ + NQZ + q3] };
			const double dz[2] = { tab[S::ODZ + q3], tab[S::ODZ + NQZ + q3] };
			double m[3][3], det, irm[3][3], xp[3];
			refmap_point(X, vx, dx, vy, dy, vz, dz, m, det, irm, xp);
			const double wd = tab[S::OWX + q1] * tab[S::OWY + q2] * tab[S::OWZ + q3] * det;
			double g[3][3];
#pragma unroll
			for (int c = 0; c < 3; c++)
#pragma unroll
				for (int d = c; d < 3; d++) g[c][d] = irm[0][c] * irm[0][d] + irm[1][c] * irm[1][d] + irm[2][c] * irm[2][d];
			const double s = wd * cgrad;
			G[0 * NQ + q] = 0.5 * s * g[0][0];
			G[1 * NQ + q] = 0.5 * s * g[1][1];
			G[2 * NQ + q] = 0.5 * s * g[2][2];
			G[3 * NQ + q] = s * g[0][1];
			G[4 * NQ + q] = s * g[0][2];
			G[5 * NQ + q] = s * g[1][2];
			G[6 * NQ + q] = 0.5 * wd;
			G[7 * NQ + q] = wd * source_value(args.lf, args.lf_value, xp);
		}
		__syncthreads();

		double acc[NACC];
#pragma unroll
		for (int r = 0; r < NACC; r++) acc[r] = 0.0;

		for (int t = 0; t < nterms; t++) {
			const int fx = kTermFlags[t][0], fy = kTermFlags[t][1], fz = kTermFlags[t][2];
			const double *Gt = G + t * NQ;
			const double *wx = Wx + fx * NX * NX * NQX;
			const double *wy = Wy + fy * NY * NY * NQY;
			const double *wz = Wz + fz * NZ * NZ * NQZ;
			// stage 1: T1[q1][q2][c][c'] = sum_q3 G[q1][q2][q3] Wz[c][c'][q3]
			for (int i = tid; i < S::T1N; i += NT) {
				const int cc = i % (NZ * NZ), q12 = i / (NZ * NZ);
				const double *gp = Gt + q12 * NQZ, *wp = wz + cc * NQZ;
				double s = 0.0;
#pragma unroll
				for (int q3 = 0; q3 < NQZ; q3++) s += gp[q3] * wp[q3];
				T1[i] = s;
			}
			__syncthreads();
			// stage 2: T2[q1][b][b'][c][c'] = sum_q2 Wy[b][b'][q2] T1[q1][q2][c][c']
			for (int i = tid; i < S::T2N; i += NT) {
				const int cc = i % (NZ * NZ), bb = (i / (NZ * NZ)) % (NY * NY), q1 = i / (NZ * NZ * NY * NY);
				const double *wp = wy + bb * NQY, *tp = T1 + q1 * NQY * NZ * NZ + cc;
				double s = 0.0;
#pragma unroll
				for (int q2 = 0; q2 < NQY; q2++) s += wp[q2] * tp[q2 * NZ * NZ];
				T2[i] = s;
			}
			__syncthreads();
			// stage 3: A[(a,b,c)][(a',b',c')] += sum_q1 Wx[a][a'][q1] T2[q1][b][b'][c][c']
#pragma unroll
			for (int r = 0; r < NACC; r++) {
				const int idx = tid + r * NT;
				if (NL * NL % NT == 0 || idx < NL * NL) {
					const int i = idx / NL, j = idx % NL;
					const int a = i / (NY * NZ), b = (i / NZ) % NY, c = i % NZ;
					const int a2 = j / (NY * NZ), b2 = (j / NZ) % NY, c2 = j % NZ;
					const double *wp = wx + (a * NX + a2) * NQX;
					const double *tp = T2 + ((b * NY + b2) * NZ + c) * NZ + c2;
					double s = acc[r];
#pragma unroll
					for (int q1 = 0; q1 < NQX; q1++) s += wp[q1] * tp[q1 * NY * NY * NZ * NZ];
					acc[r] = s;
				}
			}
			__syncthreads();
		}
#pragma unroll
		for (int r = 0; r < NACC; r++) {
			const int idx = tid + r * NT;
			if (NL * NL % NT == 0 || idx < NL * NL) A[idx] = acc[r];
		}
		// element load vector F_i = sum_q (w det f)(q) phi_i(q)
		if (args.rhs && args.lf) {
			for (int i = tid; i < NL; i += NT) {
				const int a = i / (NY * NZ), b = (i / NZ) % NY, c = i % NZ;
				double s = 0.0;
				for (int q = 0; q < NQ; q++) {
					const int q1 = q / (NQY * NQZ), q2 = (q / NQZ) % NQY, q3 = q % NQZ;
					s += G[7 * NQ + q] * tab[S::OVX + a * NQX + q1] * tab[S::OVY + b * NQY + q2] * tab[S::OVZ + c * NQZ + q3];
				}
				F[i] = s;
			}
		}
		__syncthreads();

		// ---- scatter into the CSC matrix (exclusive within a colour)
		if (args.Ax) {
			const uint16_t *off = args.el_off + k * NL * NL;
			for (int p = tid; p < mcnt * mcnt; p += NT) {
				const int b = p / mcnt, a = p % mcnt;
				const int sa = es[a], sb = es[b];
				const double v = ec[a] * ec[b] * (A[sa * NL + sb] + A[sb * NL + sa]);
				const int64_t c0 = args.Ap[edof[b]], pos = c0 + off[b * NL + a];
				if (pos < args.Ap[edof[b] + 1]) args.Ax[pos] += v;
				else atomicOr(args.status, kErrBounds);
			}
		}
		if (args.rhs && args.lf) {
			for (int a = tid; a < mcnt; a += NT) {
				const int sa = es[a];
				double lr = 0.0;
				for (int j = mcnt; j < mcnt + lcnt; j++) {
					const int sj = es[j];
					lr -= ec[a] * ec[j] * (A[sa * NL + sj] + A[sj * NL + sa]);
				}
				lr += F[sa] * ec[a];
				args.rhs[edof[a]] += lr;
			}
		}
		__syncthreads();
	}
}

} // namespace h3dg
