// Adjoint of the coefficient-weighted assembly.
//
// For L_k = lambda_k^T K(a_k) u_k - lambda_k^T f(a_k) with
//   K(a) = sum_e a_e K_e (+ mass),  a_e = exp(g_e),
//   f(a) = F - sum_e a_e K_e^{(D)} (Dirichlet lifting, src/discretization.cc:316-317),
// the gradient with respect to the per-element log-coefficient is
//   dL_k / dg_{k,e} = a_{k,e} * S_{k,e},   S_{k,e} = lambda_e^T K_e^{(1)} (u_e + d_e),
// where K_e^{(1)} is the unit-coefficient grad-grad element matrix, lambda_e
// and u_e are the element restrictions (assembly-list coefficients applied)
// and d_e the lifting coefficients.  S is evaluated matrix-free:
//   S = sum_q grad(l_h)^T G_q grad(w_h),  G_q = w_q det J^-1 J^-T,
// with grad(l_h), grad(w_h) interpolated to the Gauss points by sum
// factorisation.  The geometry is computed once per element and shared by
// all fields; S is reduced in a fixed order (deterministic).
#pragma once

#include "common.cuh"

namespace h3dg {

struct AdjArgs {
	const double *xyz;
	const int32_t *el_vtx;     // assembly order
	const int32_t *el_id;
	// either the assembly-list tables (el_s/el_dof/el_coef + counts) ...
	const int32_t *el_cnt;
	const uint16_t *el_s;
	const int32_t *el_dof;
	const double *el_coef;
	// ... or the canonical tables (high orders)
	const int32_t *cdof;
	const double *ccoef;
	const double *tables;
	int table_bytes;
	int nfields;
	int lift;                  // 1: include the Dirichlet lifting d_e (the RHS carries it only with a linear form)
	int64_t ne, ndof;
	const double *logcoef;     // nfields x ne (element-id order), or nullptr (a = 1)
	const double *u;           // nfields x ndof
	const double *lam;         // nfields x ndof
	double *S;                 // nfields x ne (element-id order), may be nullptr
	double *grad;              // nfields x ne, may be nullptr
	int *status;
};

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ>
struct AdjShape {
	static constexpr int NX = PX + 1, NY = PY + 1, NZ = PZ + 1;
	static constexpr int NL = NX * NY * NZ;
	static constexpr int NQ = NQX * NQY * NQZ;
	static constexpr int OVX = 0, ODX = OVX + NX * NQX, OVY = ODX + NX * NQX, ODY = OVY + NY * NQY;
	static constexpr int OVZ = ODY + NY * NQY, ODZ = OVZ + NZ * NQZ;
	static constexpr int OQX = ODZ + NZ * NQZ, OWX = OQX + NQX, OQY = OWX + NQX, OWY = OQY + NQY;
	static constexpr int OQZ = OWY + NQY, OWZ = OQZ + NQZ;
	static constexpr int TAB = OWZ + NQZ;
	static constexpr int TABP = (TAB + 1) & ~1;
	static constexpr int S_G = TABP;                       // 6 NQ
	static constexpr int S_C = S_G + 6 * NQ;               // 2 NL: coefficients l_e, w_e
	static constexpr int S_Q = S_C + 2 * NL;               // 2 x 2 NX NY NQZ
	static constexpr int S_P = S_Q + 4 * NX * NY * NQZ;    // 2 x 3 NX NQY NQZ
	static constexpr int S_X = S_P + 6 * NX * NQY * NQZ;   // 24
	static constexpr int S_M = S_X + 24;                   // 24
	static constexpr int S_R = S_M + 24;                   // reduction scratch (32)
	static constexpr int SMEM_DOUBLES = S_R + 32;
	static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int NT>
__global__ void __launch_bounds__(NT) k_adjoint(AdjArgs args) {
	using S = AdjShape<PX, PY, PZ, NQX, NQY, NQZ>;
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NL = S::NL, NQ = S::NQ;
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	const double *tab = sm;
	double *G = sm + S::S_G, *cf = sm + S::S_C, *Qw = sm + S::S_Q, *Pw = sm + S::S_P;
	double *X = sm + S::S_X, *Mo = sm + S::S_M, *red = sm + S::S_R;
	const int tid = threadIdx.x;
	if (!stage_tables(sm, args.tables, args.table_bytes, &bar, args.status)) return;
	const double *Vx = tab + S::OVX, *Dx = tab + S::ODX, *Vy = tab + S::OVY, *Dy = tab + S::ODY;
	const double *Vz = tab + S::OVZ, *Dz = tab + S::ODZ;
	const bool canon = args.cdof != nullptr;

	for (int64_t k = blockIdx.x; k < args.ne; k += gridDim.x) {
		if (tid < 24) X[tid] = args.xyz[3 * (int64_t) args.el_vtx[8 * k + tid / 3] + tid % 3];
		__syncthreads();
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
		// unit-coefficient G (full, symmetric: xx yy zz xy xz yz)
		for (int q = tid; q < NQ; q += NT) {
			const int q1 = q / (NQY * NQZ), q2 = (q / NQZ) % NQY, q3 = q % NQZ;
			const double x = tab[S::OQX + q1], y = tab[S::OQY + q2], z = tab[S::OQZ + q3];
			const double xy = x * y, xz = x * z, yz = y * z;
			double m[3][3];
#pragma unroll
			for (int r = 0; r < 3; r++) {
				const double c1 = Mo[3 + r], c2 = Mo[6 + r], c3 = Mo[9 + r];
				const double c4 = Mo[12 + r], c5 = Mo[15 + r], c6 = Mo[18 + r], c7 = Mo[21 + r];
				m[r][0] = c1 + c4 * y + c5 * z + c7 * yz;
				m[r][1] = c2 + c4 * x + c6 * z + c7 * xz;
				m[r][2] = c3 + c5 * x + c6 * y + c7 * xy;
			}
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
			const double s = tab[S::OWX + q1] * tab[S::OWY + q2] * tab[S::OWZ + q3] / det;
			G[0 * NQ + q] = s * (C00 * C00 + C10 * C10 + C20 * C20);
			G[1 * NQ + q] = s * (C01 * C01 + C11 * C11 + C21 * C21);
			G[2 * NQ + q] = s * (C02 * C02 + C12 * C12 + C22 * C22);
			G[3 * NQ + q] = s * (C00 * C01 + C10 * C11 + C20 * C21);
			G[4 * NQ + q] = s * (C00 * C02 + C10 * C12 + C20 * C22);
			G[5 * NQ + q] = s * (C01 * C02 + C11 * C12 + C21 * C22);
		}
		const int64_t eid = args.el_id[k];
		for (int f = 0; f < args.nfields; f++) {
			const double *u = args.u + (int64_t) f * args.ndof, *lam = args.lam + (int64_t) f * args.ndof;
			// canonical restrictions: cf[0..NL) = l_e, cf[NL..2NL) = w_e = u_e + d_e
			for (int i = tid; i < 2 * NL; i += NT) cf[i] = 0.0;
			__syncthreads();
			if (canon) {
				for (int i = tid; i < NL; i += NT) {
					const int d = args.cdof[k * NL + i];
					const double c = args.ccoef[k * NL + i];
					cf[i] = d >= 0 ? c * lam[d] : 0.0;
					cf[NL + i] = d >= 0 ? c * u[d] : (args.lift ? c : 0.0);
				}
			}
			else {
				const int m = args.el_cnt[2 * k], l = args.el_cnt[2 * k + 1];
				for (int a = tid; a < m + l; a += NT) {
					const int s = args.el_s[k * NL + a];
					const int d = args.el_dof[k * NL + a];
					const double c = args.el_coef[k * NL + a];
					cf[s] = a < m ? c * lam[d] : 0.0;
					cf[NL + s] = a < m ? c * u[d] : (args.lift ? c : 0.0);
				}
			}
			__syncthreads();
			// interpolate both: Q[v][0]=sum_c x V_z, Q[v][1]=sum_c x D_z  (v = l, w)
			for (int i = tid; i < 2 * NX * NY * NQZ; i += NT) {
				const int v = i / (NX * NY * NQZ), r = i % (NX * NY * NQZ);
				const int ab = r / NQZ, q3 = r % NQZ;
				const double *x = cf + v * NL + ab * NZ;
				double s0 = 0.0, s1 = 0.0;
#pragma unroll
				for (int c = 0; c < NZ; c++) {
					s0 += x[c] * Vz[c * NQZ + q3];
					s1 += x[c] * Dz[c * NQZ + q3];
				}
				Qw[(2 * v) * NX * NY * NQZ + r] = s0;
				Qw[(2 * v + 1) * NX * NY * NQZ + r] = s1;
			}
			__syncthreads();
			// P[v][0]=sum_b Q0 V_y, P[v][1]=sum_b Q0 D_y, P[v][2]=sum_b Q1 V_y
			for (int i = tid; i < 2 * NX * NQY * NQZ; i += NT) {
				const int v = i / (NX * NQY * NQZ), r = i % (NX * NQY * NQZ);
				const int a = r / (NQY * NQZ), q2 = (r / NQZ) % NQY, q3 = r % NQZ;
				const double *q0 = Qw + (2 * v) * NX * NY * NQZ, *q1p = Qw + (2 * v + 1) * NX * NY * NQZ;
				double s00 = 0.0, s10 = 0.0, s01 = 0.0;
#pragma unroll
				for (int b = 0; b < NY; b++) {
					const double a0 = q0[(a * NY + b) * NQZ + q3], a1 = q1p[(a * NY + b) * NQZ + q3];
					s00 += a0 * Vy[b * NQY + q2];
					s10 += a0 * Dy[b * NQY + q2];
					s01 += a1 * Vy[b * NQY + q2];
				}
				Pw[(3 * v) * NX * NQY * NQZ + r] = s00;
				Pw[(3 * v + 1) * NX * NQY * NQZ + r] = s10;
				Pw[(3 * v + 2) * NX * NQY * NQZ + r] = s01;
			}
			__syncthreads();
			// per point: grads of l and w, contract with G
			double acc = 0.0;
			for (int q = tid; q < NQ; q += NT) {
				const int q1 = q / (NQY * NQZ), q23 = q % (NQY * NQZ);
				double gl[3] = { 0.0, 0.0, 0.0 }, gw[3] = { 0.0, 0.0, 0.0 };
#pragma unroll
				for (int a = 0; a < NX; a++) {
					const double vx = Vx[a * NQX + q1], dx = Dx[a * NQX + q1];
					const int o = a * NQY * NQZ + q23;
					gl[0] += Pw[o] * dx;
					gl[1] += Pw[NX * NQY * NQZ + o] * vx;
					gl[2] += Pw[2 * NX * NQY * NQZ + o] * vx;
					gw[0] += Pw[3 * NX * NQY * NQZ + o] * dx;
					gw[1] += Pw[4 * NX * NQY * NQZ + o] * vx;
					gw[2] += Pw[5 * NX * NQY * NQZ + o] * vx;
				}
				const double gxx = G[q], gyy = G[NQ + q], gzz = G[2 * NQ + q];
				const double gxy = G[3 * NQ + q], gxz = G[4 * NQ + q], gyz = G[5 * NQ + q];
				acc += gl[0] * (gxx * gw[0] + gxy * gw[1] + gxz * gw[2]) + gl[1] * (gxy * gw[0] + gyy * gw[1] + gyz * gw[2]) +
				       gl[2] * (gxz * gw[0] + gyz * gw[1] + gzz * gw[2]);
			}
			// fixed-order block reduction
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
			if ((tid & 31) == 0) red[tid >> 5] = acc;
			__syncthreads();
			if (tid == 0) {
				double s = 0.0;
				for (int w = 0; w < NT / 32; w++) s += red[w];
				const int64_t o = (int64_t) f * args.ne + eid;
				if (args.S) args.S[o] = s;
				if (args.grad) args.grad[o] = (args.logcoef ? exp(args.logcoef[o]) : 1.0) * s;
			}
			__syncthreads();
		}
	}
}

// Mixed orders and hanging nodes: the same sensitivities with per-element
// orders and rules (runtime loops bounded by PM / QM).  Ordinary elements
// take their canonical restrictions from the plan's canonical tables;
// constrained elements from the constraint weights: column u of the element
// (a global DOF, or the Dirichlet lifting, last) contributes w x[u] to the
// canonical function s of each of its (s, w) pairs.  One thread accumulates
// the columns and their entries in order, so the sums are deterministic.  Sensitivities of element ids with no active element (refined
// parents) are left to the caller (zero-filled by the host).
struct AdjMixedArgs {
	const double *xyz;
	const int32_t *el_vtx, *el_id, *el_desc;   // ordinary elements (assembly order)
	const int64_t *el_base;
	const int32_t *cdof;
	const double *ccoef;
	int64_t ne;
	const int32_t *ce_vtx, *ce_id, *ce_desc;   // constrained elements
	const int64_t *ce_ubase, *ce_wptr;
	const int32_t *ce_udof;
	const uint16_t *ce_ws;
	const double *ce_ww;
	int64_t nce;
	const double *tables;
	int table_bytes;
	int nfields;
	int lift;
	int64_t ne_ids, ndof;
	const double *logcoef, *u, *lam;
	double *S, *grad;
	int *status;
};

template <int PM, int QM>
struct AdjMixedShape {
	static constexpr int NM = PM + 1, NLM = NM * NM * NM, Q3 = QM * QM * QM;
	static constexpr int R_G = 0;                          // 6 x nq
	static constexpr int R_C = R_G + 6 * Q3;               // 2 x nl
	static constexpr int R_Q = R_C + 2 * NLM;              // 4 x NX NY nqz
	static constexpr int R_P = R_Q + 4 * NM * NM * QM;     // 6 x NX nqy nqz
	static constexpr int R_X = R_P + 6 * NM * QM * QM;
	static constexpr int R_M = R_X + 24;
	static constexpr int R_R = R_M + 24;
	static constexpr int END = R_R + 32;
	static size_t smem_bytes(int table_bytes) { return (size_t) ((table_bytes + 15) / 16) * 16 + sizeof(double) * END; }
};

template <int PM, int QM, int NT>
__global__ void __launch_bounds__(NT) k_adjoint_mixed(AdjMixedArgs args) {
	using S = AdjMixedShape<PM, QM>;
	constexpr int NM = S::NM;
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	const int tid = threadIdx.x, lane = tid & 31;
	if (!stage_tables(sm, args.tables, args.table_bytes, &bar, args.status)) return;
	const double *tab = sm;
	double *R = sm + ((args.table_bytes + 15) / 16) * 2;
	double *G = R + S::R_G, *cf = R + S::R_C, *Qw = R + S::R_Q, *Pw = R + S::R_P;
	double *X = R + S::R_X, *Mo = R + S::R_M, *red = R + S::R_R;

	for (int64_t item = blockIdx.x; item < args.ne + args.nce; item += gridDim.x) {
		const bool ce = item >= args.ne;
		const int64_t k = ce ? item - args.ne : item;
		const int32_t *dsc = (ce ? args.ce_desc : args.el_desc) + k * 12;
		const int32_t *vtx = (ce ? args.ce_vtx : args.el_vtx) + 8 * k;
		const int64_t eid = ce ? args.ce_id[k] : args.el_id[k];
		const int nqx = dsc[3], nqy = dsc[4], nqz = dsc[5];
		const int NX = dsc[0] + 1, NY = dsc[1] + 1, NZ = dsc[2] + 1, NL = NX * NY * NZ, NQ = nqx * nqy * nqz;
		const double *Vx = tab + dsc[6], *Dx = Vx + NX * nqx, *Qx = Dx + NX * nqx, *Wx = Qx + nqx;
		const double *Vy = tab + dsc[7], *Dy = Vy + NY * nqy, *Qy = Dy + NY * nqy, *Wy = Qy + nqy;
		const double *Vz = tab + dsc[8], *Dz = Vz + NZ * nqz, *Qz = Dz + NZ * nqz, *Wz = Qz + nqz;
		if (tid < 24) X[tid] = args.xyz[3 * (int64_t) vtx[tid / 3] + tid % 3];
		__syncthreads();
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
		// unit-coefficient G (xx yy zz xy xz yz) at the element's rule
		for (int q = tid; q < NQ; q += NT) {
			const int q1 = q / (nqy * nqz), q2 = (q / nqz) % nqy, q3 = q % nqz;
			const double x = Qx[q1], y = Qy[q2], z = Qz[q3];
			const double xy = x * y, xz = x * z, yz = y * z;
			double m[3][3];
#pragma unroll
			for (int r = 0; r < 3; r++) {
				const double c1 = Mo[3 + r], c2 = Mo[6 + r], c3 = Mo[9 + r];
				const double c4 = Mo[12 + r], c5 = Mo[15 + r], c6 = Mo[18 + r], c7 = Mo[21 + r];
				m[r][0] = c1 + c4 * y + c5 * z + c7 * yz;
				m[r][1] = c2 + c4 * x + c6 * z + c7 * xz;
				m[r][2] = c3 + c5 * x + c6 * y + c7 * xy;
			}
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
			const double s = Wx[q1] * Wy[q2] * Wz[q3] / det;
			G[0 * NQ + q] = s * (C00 * C00 + C10 * C10 + C20 * C20);
			G[1 * NQ + q] = s * (C01 * C01 + C11 * C11 + C21 * C21);
			G[2 * NQ + q] = s * (C02 * C02 + C12 * C12 + C22 * C22);
			G[3 * NQ + q] = s * (C00 * C01 + C10 * C11 + C20 * C21);
			G[4 * NQ + q] = s * (C00 * C02 + C10 * C12 + C20 * C22);
			G[5 * NQ + q] = s * (C01 * C02 + C11 * C12 + C21 * C22);
		}
		for (int f = 0; f < args.nfields; f++) {
			const double *u = args.u + (int64_t) f * args.ndof, *lam = args.lam + (int64_t) f * args.ndof;
			// canonical restrictions: cf[0..NL) = l_e, cf[NL..2NL) = w_e = u_e + d_e
			for (int i = tid; i < 2 * NL; i += NT) cf[i] = 0.0;
			__syncthreads();
			if (!ce) {
				const int64_t b = args.el_base[k];
				for (int i = tid; i < NL; i += NT) {
					const int d = args.cdof[b + i];
					const double c = args.ccoef[b + i];
					cf[i] = d >= 0 ? c * lam[d] : 0.0;
					cf[NL + i] = d >= 0 ? c * u[d] : (args.lift ? c : 0.0);
				}
			}
			else if (tid == 0) {
				// one thread, entries in order: the lifting column sums several Dirichlet
				// functions and may list a canonical function more than once
				for (int64_t col = args.ce_ubase[k]; col < args.ce_ubase[k + 1]; col++) {
					const int dv = args.ce_udof[col];
					const double xl = dv >= 0 ? lam[dv] : 0.0, xw = dv >= 0 ? u[dv] : (args.lift ? 1.0 : 0.0);
					for (int64_t e = args.ce_wptr[col]; e < args.ce_wptr[col + 1]; e++) {
						const int s = args.ce_ws[e];
						const double w = args.ce_ww[e];
						cf[s] += w * xl;
						cf[NL + s] += w * xw;
					}
				}
			}
			__syncthreads();
			// interpolate both: Q[v][0] = sum_c x V_z, Q[v][1] = sum_c x D_z
			const int QS = NX * NY * nqz, PS = NX * nqy * nqz;
			for (int i = tid; i < 2 * QS; i += NT) {
				const int v = i / QS, r = i % QS;
				const int ab = r / nqz, q3 = r % nqz;
				const double *x = cf + v * NL + ab * NZ;
				double s0 = 0.0, s1 = 0.0;
				for (int c = 0; c < NZ; c++) {
					s0 += x[c] * Vz[c * nqz + q3];
					s1 += x[c] * Dz[c * nqz + q3];
				}
				Qw[(2 * v) * QS + r] = s0;
				Qw[(2 * v + 1) * QS + r] = s1;
			}
			__syncthreads();
			for (int i = tid; i < 2 * PS; i += NT) {
				const int v = i / PS, r = i % PS;
				const int a = r / (nqy * nqz), q2 = (r / nqz) % nqy, q3 = r % nqz;
				const double *q0 = Qw + (2 * v) * QS, *q1p = Qw + (2 * v + 1) * QS;
				double s00 = 0.0, s10 = 0.0, s01 = 0.0;
				for (int b = 0; b < NY; b++) {
					const double a0 = q0[(a * NY + b) * nqz + q3], a1 = q1p[(a * NY + b) * nqz + q3];
					s00 += a0 * Vy[b * nqy + q2];
					s10 += a0 * Dy[b * nqy + q2];
					s01 += a1 * Vy[b * nqy + q2];
				}
				Pw[(3 * v) * PS + r] = s00;
				Pw[(3 * v + 1) * PS + r] = s10;
				Pw[(3 * v + 2) * PS + r] = s01;
			}
			__syncthreads();
			double acc = 0.0;
			for (int q = tid; q < NQ; q += NT) {
				const int q1 = q / (nqy * nqz), q23 = q % (nqy * nqz);
				double gl[3] = { 0.0, 0.0, 0.0 }, gw[3] = { 0.0, 0.0, 0.0 };
				for (int a = 0; a < NX; a++) {
					const double vx = Vx[a * nqx + q1], dx = Dx[a * nqx + q1];
					const int o = a * nqy * nqz + q23;
					gl[0] += Pw[o] * dx;
					gl[1] += Pw[PS + o] * vx;
					gl[2] += Pw[2 * PS + o] * vx;
					gw[0] += Pw[3 * PS + o] * dx;
					gw[1] += Pw[4 * PS + o] * vx;
					gw[2] += Pw[5 * PS + o] * vx;
				}
				const double gxx = G[q], gyy = G[NQ + q], gzz = G[2 * NQ + q];
				const double gxy = G[3 * NQ + q], gxz = G[4 * NQ + q], gyz = G[5 * NQ + q];
				acc += gl[0] * (gxx * gw[0] + gxy * gw[1] + gxz * gw[2]) + gl[1] * (gxy * gw[0] + gyy * gw[1] + gyz * gw[2]) +
				       gl[2] * (gxz * gw[0] + gyz * gw[1] + gzz * gw[2]);
			}
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
			if (lane == 0) red[tid >> 5] = acc;
			__syncthreads();
			if (tid == 0) {
				double s = 0.0;
				for (int w = 0; w < NT / 32; w++) s += red[w];
				const int64_t o = (int64_t) f * args.ne_ids + eid;
				if (args.S) args.S[o] = s;
				if (args.grad) args.grad[o] = (args.logcoef ? exp(args.logcoef[o]) : 1.0) * s;
			}
			__syncthreads();
		}
		(void) NM;
	}
}

} // namespace h3dg
