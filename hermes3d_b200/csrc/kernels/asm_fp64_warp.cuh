// FP64 element matrix + deterministic scatter, one element per WARP.
//
// The same arithmetic as k_assemble_fp64 (every value is produced by one
// lane with the same operation sequence, so the result is bitwise identical
// to that kernel's), organised for low orders where a CTA-wide element
// leaves most of the SM waiting at block barriers: each warp of a CTA
// assembles its own elements (persistent, element g, g + G, ...) with only
// warp barriers between its phases, so a CTA of W warps keeps W independent
// elements in flight and the SM overlaps one warp's global loads and posted
// adds with the others' arithmetic.  The 1D product tables are built once
// per CTA (the only block barrier).  Stage 3: a lane owns the columns
// lane + 32 u and keeps their accumulators in registers (orders <= 2).
// Same reference correspondence as asm_fp64.cuh (src/discretization.cc:
// 290-338, src/integrals/h1.h:115-177, src/linsolver/umfpack.cc:80-152).
#pragma once

#include "asm_fp64.cuh"

namespace h3dg {

// Per-warp area: A (the element matrix, NL^2) aliases G, which is dead once
// stage 1 and the load vector have read it, so stage 3 stores each column's
// entries as soon as they are computed (no accumulators held across columns).
template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int W>
struct WarpShape : SfShape<PX, PY, PZ, NQX, NQY, NQZ, W> {
	using B = SfShape<PX, PY, PZ, NQX, NQY, NQZ, W>;
	static constexpr int E_G = 0;
	static constexpr int E_A = 0;
	static constexpr int E_T1 = 8 * B::NQ > B::NL * B::NL ? 8 * B::NQ : B::NL * B::NL;
	static constexpr int E_F = E_T1 + B::NT_TERMS * B::T1N;   // NL
	static constexpr int E_X = E_F + B::NL;      // 24
	static constexpr int E_M = E_X + 24;         // 24
	static constexpr int E_C = E_M + 24;         // NL
	static constexpr int E_CS = E_C + B::NL;     // NL int64
	static constexpr int E_CE = E_CS + B::NL;    // NL int64
	static constexpr int E_I = E_CE + B::NL;     // ints: dof NL, s NL
	static constexpr int E_SIZE = (E_I + B::NL + 1) & ~1;
	static constexpr int SMEM_DOUBLES = B::S_E + W * E_SIZE;
	static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int W, int MINB>
__global__ void __launch_bounds__(32 * W, MINB) k_assemble_fp64_warp(KArgs args, int64_t kbeg, int64_t kend) {
	constexpr int NT = 32, EB = 1;                 // per warp: 32 lanes, one element
	using S = WarpShape<PX, PY, PZ, NQX, NQY, NQZ, W>;   // W per-element areas, one per warp
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NL = S::NL, NQ = S::NQ;
	constexpr int NL2 = NL * NL;
	constexpr int COLS = S::COLS;
	constexpr int CH = 4;   // scatter chunk per lane
	constexpr int CPL = (COLS + 31) / 32;   // stage-3 columns per lane
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	__shared__ int s_mw[W], s_lw[W];
	__shared__ double s_cgw[W];
	double *tab = sm + S::S_TAB;
	double *Wx = sm + S::S_W, *Wy = Wx + S::WX, *Wz = Wy + S::WY;
	const int warp = threadIdx.x >> 5, tid = threadIdx.x & 31;
	double *E0 = sm + S::S_E + warp * S::E_SIZE;
	int *s_m = s_mw + warp, *s_l = s_lw + warp;
	double *s_cg = s_cgw + warp;

	if (!stage_tables(tab, args.tables, args.table_bytes, &bar, args.status, args.wait_limit)) return;
	constexpr int NTC = 32 * W;
	const int ctid = threadIdx.x;

	// 1D product tables, once per CTA
	for (int i = ctid; i < S::WX; i += NTC) {
		int q = i % NQX, kk = (i / NQX) % NX, k = (i / (NQX * NX)) % NX, f = i / (NQX * NX * NX);
		double e0 = (f >> 1) ? tab[S::ODX + k * NQX + q] : tab[S::OVX + k * NQX + q];
		double e1 = (f & 1) ? tab[S::ODX + kk * NQX + q] : tab[S::OVX + kk * NQX + q];
		Wx[i] = e0 * e1;
	}
	for (int i = ctid; i < S::WY; i += NTC) {
		int q = i % NQY, kk = (i / NQY) % NY, k = (i / (NQY * NY)) % NY, f = i / (NQY * NY * NY);
		double e0 = (f >> 1) ? tab[S::ODY + k * NQY + q] : tab[S::OVY + k * NQY + q];
		double e1 = (f & 1) ? tab[S::ODY + kk * NQY + q] : tab[S::OVY + kk * NQY + q];
		Wy[i] = e0 * e1;
	}
	for (int i = ctid; i < S::WZ; i += NTC) {
		int q = i % NQZ, kk = (i / NQZ) % NZ, k = (i / (NQZ * NZ)) % NZ, f = i / (NQZ * NZ * NZ);
		double e0 = (f >> 1) ? tab[S::ODZ + k * NQZ + q] : tab[S::OVZ + k * NQZ + q];
		double e1 = (f & 1) ? tab[S::ODZ + kk * NQZ + q] : tab[S::OVZ + kk * NQZ + q];
		Wz[i] = e0 * e1;
	}
	__syncthreads();

	const bool do_rhs = args.rhs && args.lf;
	// persistent warps: warp g of the grid takes elements g, g + G, ... (G = all warps)
	for (int64_t k0 = kbeg + (int64_t) blockIdx.x * W + warp; k0 < kend; k0 += (int64_t) gridDim.x * W) {
		const int ne = 1;

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
		__syncwarp();

		// ---- trilinear map as monomials: x_r = sum_m c_m[r] mono_m(xi, eta, zeta),
		// mono = 1, xi, eta, zeta, xi eta, xi zeta, eta zeta, xi eta zeta;
		// c_m = (1/8) sum_v X_v prod_{d in m} s_d(v), s_d(v) = +-1 the vertex's
		// reference coordinate (src/refdomain.cc:96-105)
		for (int i = tid; i < EB * 24; i += NT) {
			const int e = i / 24, mr = i % 24, mo = mr / 3, r = mr % 3;
			double *Eb = E0 + e * S::E_SIZE;
			const int usex = mo == 1 || mo == 4 || mo == 5 || mo == 7;
			const int usey = mo == 2 || mo == 4 || mo == 6 || mo == 7;
			const int usez = mo == 3 || mo == 5 || mo == 6 || mo == 7;
			double c = 0.0;
#pragma unroll
			for (int v = 0; v < 8; v++) {
				const int bx = ((v + 1) >> 1) & 1, by = (v >> 1) & 1, bz = v >> 2;
				const int neg = (usex && !bx) ^ (usey && !by) ^ (usez && !bz);
				const double xv = Eb[S::E_X + 3 * v + r];
				c += neg ? -xv : xv;
			}
			Eb[S::E_M + mr] = 0.125 * c;
		}
		__syncwarp();

		// ---- geometry at the quadrature points -> term weights.  Jacobian,
		// signed determinant and inverse as in RefMap::calc_inv_ref_map
		// (src/refmap.cc:177-231); G = w det J^-1 J^-T = (w / det) adj(J) adj(J)^T.
		for (int i = tid; i < EB * NQ; i += NT) {
			const int e = i / NQ, q = i % NQ;
			double *Eb = E0 + e * S::E_SIZE;
			double *G = Eb + S::E_G;
			const double *cm = Eb + S::E_M;
			const int q1 = q / (NQY * NQZ), q2 = (q / NQZ) % NQY, q3 = q % NQZ;
			const double x = tab[S::OQX + q1], y = tab[S::OQY + q2], z = tab[S::OQZ + q3];
			const double xy = x * y, xz = x * z, yz = y * z, xyz = xy * z;
			double m[3][3], xp[3];
#pragma unroll
			for (int r = 0; r < 3; r++) {
				const double c0 = cm[r], c1 = cm[3 + r], c2 = cm[6 + r], c3 = cm[9 + r];
				const double c4 = cm[12 + r], c5 = cm[15 + r], c6 = cm[18 + r], c7 = cm[21 + r];
				m[r][0] = c1 + c4 * y + c5 * z + c7 * yz;
				m[r][1] = c2 + c4 * x + c6 * z + c7 * xz;
				m[r][2] = c3 + c5 * x + c6 * y + c7 * xy;
				xp[r] = c0 + c1 * x + c2 * y + c3 * z + c4 * xy + c5 * xz + c6 * yz + c7 * xyz;
			}
			// cofactors: adj(J)[c][k] = C[k][c]; J^-1 = adj(J) / det
			const double C00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
			const double C01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
			const double C02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
			const double C10 = m[0][2] * m[2][1] - m[0][1] * m[2][2];
			const double C11 = m[0][0] * m[2][2] - m[0][2] * m[2][0];
			const double C12 = m[0][1] * m[2][0] - m[0][0] * m[2][1];
			const double C20 = m[0][1] * m[1][2] - m[0][2] * m[1][1];
			const double C21 = m[0][2] * m[1][0] - m[0][0] * m[1][2];
			const double C22 = m[0][0] * m[1][1] - m[0][1] * m[1][0];
			const double det = m[0][0] * C00 + m[0][1] * C01 + m[0][2] * C02;
			const double w = tab[S::OWX + q1] * tab[S::OWY + q2] * tab[S::OWZ + q3];
			const double wd = w * det;
			const double s = w * s_cg[e] / det;
			// (J^-1)[c][k] = C[k][c] / det  =>  G[c][d] = sum_k C[k][c] C[k][d] / det^2
			G[0 * NQ + q] = 0.5 * s * (C00 * C00 + C10 * C10 + C20 * C20);
			G[1 * NQ + q] = 0.5 * s * (C01 * C01 + C11 * C11 + C21 * C21);
			G[2 * NQ + q] = 0.5 * s * (C02 * C02 + C12 * C12 + C22 * C22);
			G[3 * NQ + q] = s * (C00 * C01 + C10 * C11 + C20 * C21);
			G[4 * NQ + q] = s * (C00 * C02 + C10 * C12 + C20 * C22);
			G[5 * NQ + q] = s * (C01 * C02 + C11 * C12 + C21 * C22);
			G[6 * NQ + q] = 0.5 * wd;
			G[7 * NQ + q] = wd * source_value(args.lf, args.lf_value, xp);
		}
		__syncwarp();

		// ---- element load vectors F_i = sum_q (w det f)(q) phi_i(q), by sum
		// factorisation: thread (e, a, b) contracts q3, then q2, then q1 for all c
		if (do_rhs) {
			for (int i = tid; i < EB * NX * NY; i += NT) {
				const int e = i / (NX * NY), ab = i % (NX * NY), a = ab / NY, b = ab % NY;
				double *Eb = E0 + e * S::E_SIZE;
				const double *src = Eb + S::E_G + 7 * NQ;
				double fc[NZ];
#pragma unroll
				for (int c = 0; c < NZ; c++) fc[c] = 0.0;
				for (int q1 = 0; q1 < NQX; q1++) {
					double s1[NZ];
#pragma unroll
					for (int c = 0; c < NZ; c++) s1[c] = 0.0;
					for (int q2 = 0; q2 < NQY; q2++) {
						const double vy = tab[S::OVY + b * NQY + q2];
#pragma unroll
						for (int q3 = 0; q3 < NQZ; q3++) {
							const double w = src[(q1 * NQY + q2) * NQZ + q3] * vy;
#pragma unroll
							for (int c = 0; c < NZ; c++) s1[c] += w * tab[S::OVZ + c * NQZ + q3];
						}
					}
					const double vx = tab[S::OVX + a * NQX + q1];
#pragma unroll
					for (int c = 0; c < NZ; c++) fc[c] += vx * s1[c];
				}
#pragma unroll
				for (int c = 0; c < NZ; c++) Eb[S::E_F + ab * NZ + c] = fc[c];
			}
		}

		// ---- stage 1: item (e, k, q1, q2) produces T1_k[q1][q2][*][*]
		//   k: 0 xx, 1 yy, 2 zz (+ mass), 3 xy, 4 xz, 5 yz
		for (int i = tid; i < EB * 6 * NQX * NQY; i += NT) {
			const int e = i / (6 * NQX * NQY), r = i % (6 * NQX * NQY);
			const int kk = r / (NQX * NQY), q12 = r % (NQX * NQY);
			double *Eb = E0 + e * S::E_SIZE;
			const double *gp = Eb + S::E_G + kk * NQ + q12 * NQZ;
			const double *wz = Wz + kT1Flags[kk][2] * NZ * NZ * NQZ;
			double g[NQZ];
#pragma unroll
			for (int q3 = 0; q3 < NQZ; q3++) g[q3] = gp[q3];
			double *out = Eb + S::E_T1 + kk * S::T1N + q12 * NZ * NZ;
			if (kk == 2 && args.mass) {
				const double *gm = Eb + S::E_G + 6 * NQ + q12 * NQZ;
				const double *wz0 = Wz;
				double h[NQZ];
#pragma unroll
				for (int q3 = 0; q3 < NQZ; q3++) h[q3] = gm[q3];
#pragma unroll
				for (int cc = 0; cc < NZ * NZ; cc++) {
					double s = 0.0;
#pragma unroll
					for (int q3 = 0; q3 < NQZ; q3++) s += g[q3] * wz[cc * NQZ + q3] + h[q3] * wz0[cc * NQZ + q3];
					out[cc] = s;
				}
			}
			else {
#pragma unroll
				for (int cc = 0; cc < NZ * NZ; cc++) {
					double s = 0.0;
#pragma unroll
					for (int q3 = 0; q3 < NQZ; q3++) s += g[q3] * wz[cc * NQZ + q3];
					out[cc] = s;
				}
			}
		}
		__syncwarp();
		// ---- stages 2+3: thread owns column (e, b, b', c, c'); it accumulates
		// the stage-2 values of the 3 x-classes in registers,
		//   V_f[q1] = sum_k(class f) sum_q2 Wy_k[b][b'][q2] T1_k[q1][q2][c][c'],
		// then A[(a,b,c)][(a',b',c')] = sum_f sum_q1 Wx_f[a][a'][q1] V_f[q1].
		{
			// lane owns columns col = lane + 32 u; each column's entries go to A
			// (aliasing G, dead by now) as soon as they are computed
			const double *Eb = E0;
			double *A = E0 + S::E_A;
#pragma unroll 1
			for (int u = 0; u < CPL; u++) {
				const int col = tid + 32 * u;
				if (col >= COLS) break;
				const int bb = col / (NZ * NZ), cc = col % (NZ * NZ);
				double V[3][NQX];
#pragma unroll
				for (int f = 0; f < 3; f++)
#pragma unroll
					for (int q1 = 0; q1 < NQX; q1++) V[f][q1] = 0.0;
#pragma unroll
				for (int kk = 0; kk < 6; kk++) {
					// compile-time after unrolling, so V stays in registers
					constexpr int kFy[6] = { 0, 3, 0, 1, 0, 2 };
					constexpr int kCls[6] = { 2, 0, 0, 1, 1, 0 };
					const double *wy = Wy + kFy[kk] * NY * NY * NQY + bb * NQY;
					const double *t1 = Eb + S::E_T1 + kk * S::T1N + cc;
					const int f = kCls[kk];
					double wyr[NQY];
#pragma unroll
					for (int q2 = 0; q2 < NQY; q2++) wyr[q2] = wy[q2];
#pragma unroll
					for (int q1 = 0; q1 < NQX; q1++) {
						double s2 = V[f][q1];
#pragma unroll
						for (int q2 = 0; q2 < NQY; q2++) s2 += wyr[q2] * t1[(q1 * NQY + q2) * NZ * NZ];
						V[f][q1] = s2;
					}
				}
				const double *wx0 = Wx, *wx2 = Wx + 2 * NX * NX * NQX, *wx3 = Wx + 3 * NX * NX * NQX;
				const int b = bb / NY, b2 = bb % NY, c = cc / NZ, c2 = cc % NZ;
#pragma unroll
				for (int r = 0; r < NX * NX; r++) {
					double s3 = 0.0;
#pragma unroll
					for (int q1 = 0; q1 < NQX; q1++)
						s3 += wx0[r * NQX + q1] * V[0][q1] + wx2[r * NQX + q1] * V[1][q1] + wx3[r * NQX + q1] * V[2][q1];
					const int a = r / NX, a2 = r % NX;
					A[((a * NY + b) * NZ + c) * NL + (a2 * NY + b2) * NZ + c2] = s3;
				}
			}
		}
		__syncwarp();

		// ---- scatter into the CSC matrix (exclusive within a colour)
		if (args.Ax) {
			double *__restrict__ Ax = args.Ax;
			for (int base = 0; base < EB * NL2; base += NT * CH) {
				int64_t pos[CH];
				double val[CH];
#pragma unroll
				for (int r = 0; r < CH; r++) {
					const int p = base + tid + r * NT;
					pos[r] = -1;
					val[r] = 0.0;
					if (p < EB * NL2) {
						const int e = p / NL2, pp = p % NL2;
						const int m = s_m[e];
						const int b = pp / NL, a = pp % NL;
						if (a < m && b < m) {
							const double *Eb = E0 + e * S::E_SIZE;
							const int *ei = reinterpret_cast<const int *>(Eb + S::E_I);
							const int64_t *cs = reinterpret_cast<const int64_t *>(Eb + S::E_CS);
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
				for (int r = 0; r < CH; r++)
					if (pos[r] >= 0) posted_add(Ax + pos[r], val[r]);
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
				posted_add(args.rhs + ei[a], lr);
			}
		}
		__syncwarp();
	}
}

} // namespace h3dg
