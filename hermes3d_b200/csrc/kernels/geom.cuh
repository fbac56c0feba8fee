// Kernel (a): per-element reference-map geometry at the volume Gauss points
// (RefMap::calc_inv_ref_map and calc_phys_x/y/z, src/refmap.cc:177-316).
//
// One thread per (element, point).  Reads the 8 vertex coordinates of its
// element (gathered through the connectivity) and writes the signed
// determinant, the transposed inverse Jacobian (9) and the physical point
// (3): 104 bytes out per point, 96 + 32 bytes in per element.  HBM-write
// bound.  Output index = (element id - 1) * nq + q, q = (q1*nqy + q2)*nqz + q3:
// an element's points are contiguous, so the block stages its 9- and
// 3-double records in shared memory and writes them back as contiguous runs
// (a direct store of one record field per thread would touch a separate
// 32-byte sector per lane).
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

__global__ void __launch_bounds__(kGeomThreads) k_geometry(GeomArgs g) {
	__shared__ double s_irm[kGeomThreads * 9], s_xp[kGeomThreads * 3];
	__shared__ int64_t s_o[kGeomThreads];
	const int nq = g.nqx * g.nqy * g.nqz;
	const int tid = threadIdx.x;
	const int64_t t = (int64_t) blockIdx.x * kGeomThreads + tid;
	s_o[tid] = -1;
	if (t < g.ne * nq) {
		const int64_t k = t / nq;
		const int q = (int) (t % nq);
		const int q1 = q / (g.nqy * g.nqz), q2 = (q / g.nqz) % g.nqy, q3 = q % g.nqz;
		double X[24];
		const int32_t *vv = g.el_vtx + 8 * k;
#pragma unroll
		for (int v = 0; v < 8; v++) {
			const double *p = g.xyz + 3 * (int64_t) vv[v];
			X[3 * v] = p[0];
			X[3 * v + 1] = p[1];
			X[3 * v + 2] = p[2];
		}
		const double x = g.qx[q1], y = g.qy[q2], z = g.qz[q3];
		const double vx[2] = { (1.0 - x) * 0.5, (1.0 + x) * 0.5 }, dd[2] = { -0.5, 0.5 };
		const double vy[2] = { (1.0 - y) * 0.5, (1.0 + y) * 0.5 };
		const double vz[2] = { (1.0 - z) * 0.5, (1.0 + z) * 0.5 };
		double m[3][3], det, irm[3][3], xp[3];
		refmap_point(X, vx, dd, vy, dd, vz, dd, m, det, irm, xp);
		const int64_t o = (int64_t) g.el_id[k] * nq + q;
		s_o[tid] = o;
		if (g.jac) g.jac[o] = det;
#pragma unroll
		for (int r = 0; r < 3; r++)
#pragma unroll
			for (int c = 0; c < 3; c++) s_irm[9 * tid + 3 * r + c] = irm[r][c];
#pragma unroll
		for (int r = 0; r < 3; r++) s_xp[3 * tid + r] = xp[r];
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
}

} // namespace h3dg
