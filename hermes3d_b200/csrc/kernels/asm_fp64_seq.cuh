// FP64 element-matrix + deterministic scatter, terms contracted one after
// another (the variant for orders whose all-terms work area does not fit in
// shared memory), EB elements per CTA pass.
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
// A CTA works on EB elements at once: every stage is one flat loop over
// (element, item), so each block barrier is paid once per batch.
//
// Scatter.  Entry (a, b) of the element's assembly list goes to
// Ax[Ap[dof_b] + off[b][a]] (CSC: column = trial DOF).  Elements of one
// colour share no DOF, so the read-modify-write needs no atomics and the
// summation order of every entry (colour order) is fixed: bitwise
// reproducible.  Each thread issues the loads of a chunk of targets before
// any store.  Dirichlet lifting follows src/discretization.cc:316-317, the
// RHS :329-338 (lifting only enters the RHS when a linear form is set, as
// in the reference).
#pragma once

#include "asm_fp64.cuh"

namespace h3dg {

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int EB>
struct SfShapeSeq {
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
	// per-element work area: [G (8 NQ) | T1 | T2] during the terms, reused for A (NL^2) after
	static constexpr int WORK = (8 * NQ + T1N + T2N) > NL * NL ? (8 * NQ + T1N + T2N) : NL * NL;
	static constexpr int E_G = 0, E_T1 = 8 * NQ, E_T2 = E_T1 + T1N, E_A = 0;
	static constexpr int E_F = WORK;            // NL
	static constexpr int E_X = E_F + NL;        // 24
	static constexpr int E_C = E_X + 24;        // NL coefficients
	static constexpr int E_CS = E_C + NL;       // NL column starts (int64)
	static constexpr int E_CE = E_CS + NL;      // NL column ends (int64)
	static constexpr int E_I = E_CE + NL;       // ints: dof NL, s NL (NL doubles)
	static constexpr int E_SIZE = (E_I + NL + 1) & ~1;
	static constexpr int S_TAB = 0;
	static constexpr int S_W = S_TAB + TABP;
	static constexpr int S_E = S_W + WX + WY + WZ;
	static constexpr int SMEM_DOUBLES = S_E + EB * E_SIZE;
	static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};


template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int NT, int EB>
__global__ void __launch_bounds__(NT) k_assemble_fp64_seq(KArgs args, int64_t kbeg, int64_t kend) {
	using S = SfShapeSeq<PX, PY, PZ, NQX, NQY, NQZ, EB>;
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NL = S::NL, NQ = S::NQ;
	constexpr int NL2 = NL * NL;
	constexpr int NACC = (EB * NL2 + NT - 1) / NT;
	constexpr int CH = 8;   // scatter chunk: loads in flight per thread
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	__shared__ int s_m[EB], s_l[EB];
	__shared__ double s_cg[EB];
	double *tab = sm + S::S_TAB;
	double *Wx = sm + S::S_W, *Wy = Wx + S::WX, *Wz = Wy + S::WY;
	double *E0 = sm + S::S_E;
	const int tid = threadIdx.x;

	if (!stage_tables(tab, args.tables, args.table_bytes, &bar, args.status, args.wait_limit)) return;

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
	const bool do_rhs = args.rhs && args.lf;
	const int64_t nbatch = (kend - kbeg + EB - 1) / EB;
	for (int64_t bt = blockIdx.x; bt < nbatch; bt += gridDim.x) {
		const int64_t k0 = kbeg + bt * EB;
		const int ne = (int) (kend - k0 < EB ? kend - k0 : EB);

		// ---- element data
		if (tid < EB) {
			const bool live = tid < ne;
			s_m[tid] = live ? args.el_cnt[2 * (k0 + tid)] : 0;
			s_l[tid] = live ? args.el_cnt[2 * (k0 + tid) + 1] : 0;
			s_cg[tid] = live && args.ecoef ? args.ecoef[args.el_id[k0 + tid]] : 1.0;
		}
		for (int i = tid; i < EB * 24; i += NT) {
			const int e = i / 24, r = i % 24;
			E0[e * S::E_SIZE + S::E_X + r] = e < ne ? args.xyz[3 * (int64_t) args.el_vtx[8 * (k0 + e) + r / 3] + r % 3] : 0.0;
		}
		for (int i = tid; i < EB * NL; i += NT) {
			const int e = i / NL, j = i % NL;
			double *Eb = E0 + e * S::E_SIZE;
			int *ei = reinterpret_cast<int *>(Eb + S::E_I);
			const int64_t g = (k0 + e) * NL + j;
			const int dof = e < ne ? args.el_dof[g] : -1;
			Eb[S::E_C + j] = e < ne ? args.el_coef[g] : 0.0;
			ei[j] = dof;
			ei[NL + j] = e < ne ? args.el_s[g] : 0;
			int64_t *cs = reinterpret_cast<int64_t *>(Eb + S::E_CS);
			cs[j] = dof >= 0 ? args.Ap[dof] : 0;
			cs[NL + j] = dof >= 0 ? args.Ap[dof + 1] : 0;
		}
		__syncthreads();

		// ---- geometry at the quadrature points -> term weights
		for (int i = tid; i < EB * NQ; i += NT) {
			const int e = i / NQ, q = i % NQ;
			double *Eb = E0 + e * S::E_SIZE;
			double *G = Eb + S::E_G;
			const int q1 = q / (NQY * NQZ), q2 = (q / NQZ) % NQY, q3 = q % NQZ;
			const double vx[2] = { tab[S::OVX + q1], tab[S::OVX + NQX + q1] };
			const double dx[2] = { tab[S::ODX + q1], tab[S::ODX + NQX + q1] };
			const double vy[2] = { tab[S::OVY + q2], tab[S::OVY + NQY + q2] };
			const double dy[2] = { tab[S::ODY + q2], tab[S::ODY + NQY + q2] };
			const double vz[2] = { tab[S::OVZ + q3], tab[S::OVZ + NQZ + q3] };
			const double dz[2] = { tab[S::ODZ + q3], tab[S::ODZ + NQZ + q3] };
			double m[3][3], det, irm[3][3], xp[3];
			refmap_point(Eb + S::E_X, vx, dx, vy, dy, vz, dz, m, det, irm, xp);
			const double wd = tab[S::OWX + q1] * tab[S::OWY + q2] * tab[S::OWZ + q3] * det;
			double g[3][3];
#pragma unroll
			for (int c = 0; c < 3; c++)
#pragma unroll
				for (int d = c; d < 3; d++) g[c][d] = irm[0][c] * irm[0][d] + irm[1][c] * irm[1][d] + irm[2][c] * irm[2][d];
			const double s = wd * s_cg[e];
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

		// element load vectors F_i = sum_q (w det f)(q) phi_i(q)
		if (do_rhs) {
			for (int i = tid; i < EB * NL; i += NT) {
				const int e = i / NL, j = i % NL;
				double *Eb = E0 + e * S::E_SIZE;
				const double *src = Eb + S::E_G + 7 * NQ;
				const int a = j / (NY * NZ), b = (j / NZ) % NY, c = j % NZ;
				double s = 0.0;
				for (int q1 = 0; q1 < NQX; q1++) {
					double s1 = 0.0;
					for (int q2 = 0; q2 < NQY; q2++) {
						double s2 = 0.0;
#pragma unroll
						for (int q3 = 0; q3 < NQZ; q3++) s2 += src[(q1 * NQY + q2) * NQZ + q3] * tab[S::OVZ + c * NQZ + q3];
						s1 += s2 * tab[S::OVY + b * NQY + q2];
					}
					s += s1 * tab[S::OVX + a * NQX + q1];
				}
				Eb[S::E_F + j] = s;
			}
		}

		double acc[NACC];
#pragma unroll
		for (int r = 0; r < NACC; r++) acc[r] = 0.0;

		for (int t = 0; t < nterms; t++) {
			const int fx = kTermFlags[t][0], fy = kTermFlags[t][1], fz = kTermFlags[t][2];
			const double *wx = Wx + fx * NX * NX * NQX;
			const double *wy = Wy + fy * NY * NY * NQY;
			const double *wz = Wz + fz * NZ * NZ * NQZ;
			// stage 1: T1[q1][q2][c][c'] = sum_q3 G[q1][q2][q3] Wz[c][c'][q3]
			for (int i = tid; i < EB * S::T1N; i += NT) {
				const int e = i / S::T1N, ii = i % S::T1N;
				double *Eb = E0 + e * S::E_SIZE;
				const int cc = ii % (NZ * NZ), q12 = ii / (NZ * NZ);
				const double *gp = Eb + S::E_G + t * NQ + q12 * NQZ, *wp = wz + cc * NQZ;
				double s = 0.0;
#pragma unroll
				for (int q3 = 0; q3 < NQZ; q3++) s += gp[q3] * wp[q3];
				Eb[S::E_T1 + ii] = s;
			}
			__syncthreads();
			// stage 2: T2[q1][b][b'][c][c'] = sum_q2 Wy[b][b'][q2] T1[q1][q2][c][c']
			for (int i = tid; i < EB * S::T2N; i += NT) {
				const int e = i / S::T2N, ii = i % S::T2N;
				double *Eb = E0 + e * S::E_SIZE;
				const int cc = ii % (NZ * NZ), bb = (ii / (NZ * NZ)) % (NY * NY), q1 = ii / (NZ * NZ * NY * NY);
				const double *wp = wy + bb * NQY, *tp = Eb + S::E_T1 + q1 * NQY * NZ * NZ + cc;
				double s = 0.0;
#pragma unroll
				for (int q2 = 0; q2 < NQY; q2++) s += wp[q2] * tp[q2 * NZ * NZ];
				Eb[S::E_T2 + ii] = s;
			}
			__syncthreads();
			// stage 3: A[(a,b,c)][(a',b',c')] += sum_q1 Wx[a][a'][q1] T2[q1][b][b'][c][c']
#pragma unroll
			for (int r = 0; r < NACC; r++) {
				const int idx = tid + r * NT;
				if ((EB * NL2) % NT == 0 || idx < EB * NL2) {
					const int e = idx / NL2, ij = idx % NL2;
					const int i = ij / NL, j = ij % NL;
					const int a = i / (NY * NZ), b = (i / NZ) % NY, c = i % NZ;
					const int a2 = j / (NY * NZ), b2 = (j / NZ) % NY, c2 = j % NZ;
					const double *wp = wx + (a * NX + a2) * NQX;
					const double *tp = E0 + e * S::E_SIZE + S::E_T2 + ((b * NY + b2) * NZ + c) * NZ + c2;
					double s = acc[r];
#pragma unroll
					for (int q1 = 0; q1 < NQX; q1++) s += wp[q1] * tp[q1 * NY * NY * NZ * NZ];
					acc[r] = s;
				}
			}
			__syncthreads();
		}
		// A overwrites the G/T1/T2 work area (F already computed)
#pragma unroll
		for (int r = 0; r < NACC; r++) {
			const int idx = tid + r * NT;
			if ((EB * NL2) % NT == 0 || idx < EB * NL2) {
				const int e = idx / NL2, ij = idx % NL2;
				E0[e * S::E_SIZE + S::E_A + ij] = acc[r];
			}
		}
		__syncthreads();

		// ---- scatter into the CSC matrix (exclusive within a colour)
		if (args.Ax) {
			double *__restrict__ Ax = args.Ax;
			for (int base = 0; base < EB * NL2; base += NT * CH) {
				int64_t pos[CH];
				double val[CH], old[CH];
#pragma unroll
				for (int r = 0; r < CH; r++) {
					const int p = base + tid + r * NT;
					pos[r] = -1;
					val[r] = 0.0;
					if (p < EB * NL2) {
						const int e = p / NL2, pp = p % NL2;
						const int m = s_m[e];
						if (pp < m * m) {
							const double *Eb = E0 + e * S::E_SIZE;
							const int *ei = reinterpret_cast<const int *>(Eb + S::E_I);
							const int64_t *cs = reinterpret_cast<const int64_t *>(Eb + S::E_CS);
							const int b = pp / m, a = pp % m;
							const int sa = ei[NL + a], sb = ei[NL + b];
							const double *A = Eb + S::E_A;
							val[r] = Eb[S::E_C + a] * Eb[S::E_C + b] * (A[sa * NL + sb] + A[sb * NL + sa]);
							const int64_t t = cs[b] + args.el_off[(k0 + e) * NL2 + b * NL + a];
							if (t < cs[NL + b]) pos[r] = t;
							else if (cs[NL + b] > cs[b]) atomicOr(args.status, kErrBounds);   // empty: column not owned
						}
					}
				}
#pragma unroll
				for (int r = 0; r < CH; r++) old[r] = pos[r] >= 0 ? Ax[pos[r]] : 0.0;
#pragma unroll
				for (int r = 0; r < CH; r++)
					if (pos[r] >= 0) Ax[pos[r]] = old[r] + val[r];
			}
		}
		if (do_rhs) {
			for (int i = tid; i < EB * NL; i += NT) {
				const int e = i / NL, a = i % NL;
				if (a >= s_m[e]) continue;
				const double *Eb = E0 + e * S::E_SIZE;
				const int *ei = reinterpret_cast<const int *>(Eb + S::E_I);
				const double *A = Eb + S::E_A;
				const int sa = ei[NL + a];
				const double ca = Eb[S::E_C + a];
				double lr = 0.0;
				for (int j = s_m[e]; j < s_m[e] + (args.Ax ? s_l[e] : 0); j++) {      // lifting only with the matrix (src/discretization.cc:296-317)
					const int sj = ei[NL + j];
					lr -= ca * Eb[S::E_C + j] * (A[sa * NL + sj] + A[sj * NL + sa]);
				}
				lr += Eb[S::E_F + sa] * ca;
				args.rhs[ei[a]] += lr;
			}
		}
		__syncthreads();
	}
}

} // namespace h3dg
