// Kernel variant table (see kernel_tables.h).
#include "kernel_tables.h"
#include "kernels/asm_ho_tc.cuh"

namespace h3dg_tables {

template <int P, int NQ, int MINB = 1>
static HoSpec ho_tc_spec() {
	return HoSpec { P, NQ, &h3dg::k_assemble_ho_tc<P, P, P, NQ, NQ, NQ, MINB>, 256,
	                h3dg::HoTcShape<P, P, P, NQ, NQ, NQ>::SMEM_BYTES, false };
}

std::vector<HoSpec> &ho_tc_table() {
	static std::vector<HoSpec> t = {
		ho_tc_spec<1, 3, 2>(), ho_tc_spec<2, 4, 2>(), ho_tc_spec<3, 5, 2>(), ho_tc_spec<4, 6, 2>(), ho_tc_spec<5, 6>(), ho_tc_spec<5, 7>(), ho_tc_spec<6, 7>(),
		ho_tc_spec<6, 8>(), ho_tc_spec<7, 8>(), ho_tc_spec<7, 9>(), ho_tc_spec<8, 9>(), ho_tc_spec<8, 10>(),
	};
	return t;
}

cudaError_t build_offt(const uint16_t *offc, const int32_t *cdof, const int64_t *Ap, int64_t ne, int px, int nq,
                       uint16_t **offt, size_t *count, int *status, cudaStream_t st) {
	(void) nq;
	const int nx = px + 1, nb = (nx * nx + 15) / 16 * 16;
	const size_t n = (size_t) ne * nx * (size_t) (nx * nx * nx) * nb;
	cudaError_t e = cudaMalloc((void **) offt, sizeof(uint16_t) * n);
	if (e != cudaSuccess) return e;
	*count = n;
	h3dg::k_build_offt<<<148 * 8, 256, 0, st>>>(offc, cdof, Ap, ne, nx, nx, nx, nb, *offt, status);
	return cudaGetLastError();
}

} // namespace h3dg_tables
