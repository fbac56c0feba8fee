// Kernel (a): per-element reference-map geometry at the volume Gauss points
// (RefMap::calc_inv_ref_map and calc_phys_x/y/z, src/refmap.cc:177-316).
//
// A block takes whole elements (as many as fit 256 points, at least one):
// their 8 vertex coordinates are gathered once into shared memory and turned
// into the 24 monomial coefficients of the trilinear map, then one thread per
// point evaluates the Jacobian, its signed determinant, the transposed
// inverse (the layout of RefMap::calc_inv_ref_map) and the physical point:
// 104 bytes out per point.  HBM-write bound.  Output index = (element id -
// 1) * nq + q, q = (q1*nqy + q2)*nqz + q3: an element's points are
// contiguous, so the block stages its 9- and 3-double records in shared
// memory and writes them back as contiguous runs.
#pragma once

#include "common.cuh"

namespace h3dg {

struct GeomArgs {
	const double *xyz;
	const int32_t *el_vtx;   // assembly order
	const int32_t *el_id;
	const double *qx, *qy, *qz;   // device 1D rules (points)
	int nqx, nqy, nqz;
	int64_t ne;
	double *jac, *irm, *xphys;
};

constexpr int kGeomThreads = 256;
constexpr int kGeomMaxElems = 32;     // elements per block (nq >= 8 at 256 threads)

__global__ void __launch_bounds__(kGeomThreads) k_geometry(GeomArgs g) {
	__shared__ double s_irm[kGeomThreads * 9], s_xp[kGeomThreads * 3];
	__shared__ int64_t s_o[kGeomThreads];
	__shared__ double s_x[kGeomMaxElems * 24], s_mo[kGeomMaxElems * 24];
	const int nq = g.nqx * g.nqy * g.nqz, nqyz = g.nqy * g.nqz;
	const int epb = nq >= kGeomThreads ? 1 : min(kGeomThreads / nq, kGeomMaxElems);
	const int tid = threadIdx.x;
	const int64_t k0 = (int64_t) blockIdx.x * epb;
	const int ne = (int) min((int64_t) epb, g.ne - k0);
	// vertex coordinates, then the monomial coefficients c_m = (1/8) sum_v X_v prod_{d in m} s_d(v)
	for (int i = tid; i < ne * 24; i += kGeomThreads) {
		const int e = i / 24, r = i % 24;
		s_x[i] = g.xyz[3 * (int64_t) g.el_vtx[8 * (k0 + e) + r / 3] + r % 3];
	}
	__syncthreads();
	for (int i = tid; i < ne * 24; i += kGeomThreads) {
		const int e = i / 24, mr = i % 24, mo = mr / 3, r = mr % 3;
		const int usex = mo == 1 || mo == 4 || mo == 5 || mo == 7;
		const int usey = mo == 2 || mo == 4 || mo == 6 || mo == 7;
		const int usez = mo == 3 || mo == 5 || mo == 6 || mo == 7;
		double c = 0.0;
#pragma unroll
		for (int v = 0; v < 8; v++) {
			const int bx = ((v + 1) >> 1) & 1, by = (v >> 1) & 1, bz = v >> 2;
			const int neg = (usex && !bx) ^ (usey && !by) ^ (usez && !bz);
			const double xv = s_x[e * 24 + 3 * v + r];
			c += neg ? -xv : xv;
		}
		s_mo[i] = 0.125 * c;
	}
	__syncthreads();
	const int npts = ne * nq;
	for (int i0 = 0; i0 < npts; i0 += kGeomThreads) {
		const int i = i0 + tid;
		s_o[tid] = -1;
		if (i < npts) {
			const int e = i / nq, q = i - e * nq;
			const int q1 = q / nqyz, q2 = (q - q1 * nqyz) / g.nqz, q3 = q - q1 * nqyz - q2 * g.nqz;
			const double x = g.qx[q1], y = g.qy[q2], z = g.qz[q3];
			const double xy = x * y, xz = x * z, yz = y * z, xyz = xy * z;
			const double *cm = s_mo + e * 24;
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
			// signed determinant (rule of Sarrus) and transposed inverse, as refmap_point
			const double det = m[0][0] * m[1][1] * m[2][2] + m[0][1] * m[1][2] * m[2][0] + m[0][2] * m[1][0] * m[2][1] -
			                   m[2][0] * m[1][1] * m[0][2] - m[2][1] * m[1][2] * m[0][0] - m[2][2] * m[1][0] * m[0][1];
			const double ij = 1.0 / det;
			double *d = s_irm + 9 * tid;
			d[0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * ij;
			d[1] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * ij;
			d[2] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * ij;
			d[3] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * ij;
			d[4] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * ij;
			d[5] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * ij;
			d[6] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * ij;
			d[7] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * ij;
			d[8] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * ij;
#pragma unroll
			for (int r = 0; r < 3; r++) s_xp[3 * tid + r] = xp[r];
			const int64_t o = (int64_t) g.el_id[k0 + e] * nq + q;
			s_o[tid] = o;
			if (g.jac) g.jac[o] = det;
		}
		__syncthreads();
		// consecutive j of one element's run go to consecutive addresses
		if (g.irm)
			for (int j = tid; j < kGeomThreads * 9; j += kGeomThreads) {
				const int64_t o = s_o[j / 9];
				if (o >= 0) g.irm[9 * o + j % 9] = s_irm[j];
			}
		if (g.xphys)
			for (int j = tid; j < kGeomThreads * 3; j += kGeomThreads) {
				const int64_t o = s_o[j / 3];
				if (o >= 0) g.xphys[3 * o + j % 3] = s_xp[j];
			}
		__syncthreads();
	}
}

} // namespace h3dg
