// Device helpers shared by the assembly kernels: bulk (TMA) copies into
// shared memory completed on an mbarrier, bounded waits, kernel arguments.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace h3dg {

// polls of a bounded mbarrier wait before it gives up (seconds at the B200's clock)
constexpr unsigned kWaitPolls = 1u << 24;

// error bits written to the plan's device status word
constexpr int kErrTimeout = 1;
constexpr int kErrBounds = 2;    // a scatter target fell outside its (non-empty) CSC column (store skipped);
                                 // an empty column belongs to another part of a partitioned plan: skipped silently

// Everything a fused assembly kernel reads, as device pointers.
struct KArgs {
	const double *xyz;        // vertices, nv x 3
	const int32_t *el_vtx;    // assembly order, ne x 8
	const int32_t *el_cnt;    // ne x 2 (matrix entries, lifting entries)
	const uint16_t *el_s;     // ne x nl canonical index
	const int32_t *el_dof;    // ne x nl
	const double *el_coef;    // ne x nl
	const uint16_t *el_off;   // ne x nl x nl, [b][a]: row position of dof_a in column dof_b
	const int32_t *el_id;     // ne: element id - 1
	const double *ecoef;      // per element id: grad-grad coefficient, or nullptr
	const int64_t *Ap;        // ndof + 1
	const double *tables;     // 1D tables blob (see table_layout)
	int table_bytes;
	int mass;                 // add int_u_v
	int lf;                   // linear form kind (H3DG_LF_*)
	double lf_value;
	double *Ax;               // nnz (may be nullptr)
	double *rhs;              // ndof (may be nullptr)
	int *status;              // device status word
	unsigned wait_limit;      // polls of the bounded waits (kWaitPolls; 0 only from the test hook)
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(ok)
		: "r"(smem_u32(bar)), "r"(parity)
		: "memory");
	return ok != 0;
}

// 1D bulk copy global -> shared (TMA engine, non-tensor form).  Both
// addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
	asm volatile(
		"cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
		"l"(src), "r"(bytes), "r"(smem_u32(bar))
		: "memory");
}

// Wait on phase `parity` of an mbarrier for at most `limit` polls.  Returns
// false (and records kErrTimeout) if the phase did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *status, uint32_t limit = kWaitPolls) {
	for (uint32_t it = 0; it < limit; it++)
		if (mbar_try_wait(bar, parity)) return true;
	if (status) atomicOr(status, kErrTimeout);
	return false;
}

// Stage the 1D tables blob into shared memory with one bulk copy (thread 0
// issues, everybody waits).  Returns false on timeout; the caller must then
// leave after a bounded second wait so no copy is left in flight.
__device__ __forceinline__ bool stage_tables(double *dst, const double *src, int bytes, uint64_t *bar, int *status,
                                             uint32_t limit = kWaitPolls) {
	if (threadIdx.x == 0) {
		mbar_init(bar, 1);
		fence_mbar_init();
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		mbar_arrive_expect_tx(bar, (uint32_t) bytes);
		bulk_g2s(dst, src, (uint32_t) bytes, bar);
	}
	bool ok = mbar_wait_bounded(bar, 0, status, limit);
	if (!ok) mbar_wait_bounded(bar, 0, nullptr, 1u << 26);
	// every thread returns the same verdict, so an early exit is block-uniform
	return __syncthreads_and(ok ? 1 : 0) != 0;
}

// Reference-map geometry at one quadrature point from the 8 vertex
// coordinates X[v][r] and the 1D vertex-function values / derivatives at the
// point's three coordinates (index 0 = l0, 1 = l1).  Follows
// RefMap::calc_inv_ref_map (src/refmap.cc:177-231): m[r][c] = dx_r/dxi_c,
// signed determinant by the rule of Sarrus, irm = transposed inverse.
__device__ __forceinline__ void refmap_point(const double *X, const double vx[2], const double dx[2], const double vy[2],
                                             const double dy[2], const double vz[2], const double dz[2], double m[3][3],
                                             double &det, double irm[3][3], double xp[3]) {
	// RefHex vertex order: (x,y,z) bits of vertex v: x = ((v+1)>>1)&1, y = (v>>1)&1, z = v>>2
	for (int r = 0; r < 3; r++) {
		m[r][0] = m[r][1] = m[r][2] = 0.0;
		xp[r] = 0.0;
	}
#pragma unroll
	for (int v = 0; v < 8; v++) {
		const int bx = ((v + 1) >> 1) & 1, by = (v >> 1) & 1, bz = v >> 2;
		const double nx = dx[bx] * vy[by] * vz[bz];
		const double ny = vx[bx] * dy[by] * vz[bz];
		const double nz = vx[bx] * vy[by] * dz[bz];
		const double n0 = vx[bx] * vy[by] * vz[bz];
#pragma unroll
		for (int r = 0; r < 3; r++) {
			const double c = X[3 * v + r];
			m[r][0] += c * nx;
			m[r][1] += c * ny;
			m[r][2] += c * nz;
			xp[r] += c * n0;
		}
	}
	det = m[0][0] * m[1][1] * m[2][2] + m[0][1] * m[1][2] * m[2][0] + m[0][2] * m[1][0] * m[2][1] -
	      m[2][0] * m[1][1] * m[0][2] - m[2][1] * m[1][2] * m[0][0] - m[2][2] * m[1][0] * m[0][1];
	const double ij = 1.0 / det;
	irm[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * ij;
	irm[1][0] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * ij;
	irm[2][0] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * ij;
	irm[0][1] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * ij;
	irm[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * ij;
	irm[2][1] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * ij;
	irm[0][2] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * ij;
	irm[1][2] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * ij;
	irm[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * ij;
}

// Posted add to global memory (no value returned, so the issuing thread does
// not wait for it).  Used for the colour-exclusive scatter: within one
// launch every target address receives at most one add, and launches are
// ordered on the stream, so the summation order of each entry is the colour
// order whatever the scheduling -- the result is bitwise reproducible.
__device__ __forceinline__ void posted_add(double *addr, double v) {
	asm volatile("red.global.add.f64 [%0], %1;" ::"l"(addr), "d"(v) : "memory");
}

// Plain store of an entry's first contribution (same ordering constraints
// for the compiler as posted_add)
__device__ __forceinline__ void posted_store(double *addr, double v) {
	asm volatile("st.global.f64 [%0], %1;" ::"l"(addr), "d"(v) : "memory");
}

__device__ __forceinline__ double source_value(int lf, double value, const double xp[3]) {
	if (lf == 1) return value;
	if (lf == 2) return sinpi(xp[0]) * sinpi(xp[1]) * sinpi(xp[2]);   // sin(pi x) sin(pi y) sin(pi z)
	return 0.0;
}

} // namespace h3dg
