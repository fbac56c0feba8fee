// Kernel variant table (see kernel_tables.h).
#include "kernel_tables.h"
#include "kernels/asm_ho_tc.cuh"

namespace h3dg_tables {

template <int P, int NQ>
static HoSpec ho_tc_spec() {
	return HoSpec { P, NQ, &h3dg::k_assemble_ho_tc<P, P, P, NQ, NQ, NQ>, 256,
	                h3dg::HoTcShape<P, P, P, NQ, NQ, NQ>::SMEM_BYTES, false };
}

std::vector<HoSpec> &ho_tc_table() {
	static std::vector<HoSpec> t = {
		ho_tc_spec<2, 4>(), ho_tc_spec<3, 5>(), ho_tc_spec<5, 6>(), ho_tc_spec<5, 7>(), ho_tc_spec<6, 7>(),
		ho_tc_spec<6, 8>(), ho_tc_spec<7, 8>(), ho_tc_spec<7, 9>(), ho_tc_spec<8, 9>(), ho_tc_spec<8, 10>(),
	};
	return t;
}

} // namespace h3dg_tables
