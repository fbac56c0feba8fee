// Kernel variant table (see kernel_tables.h).
#include "kernel_tables.h"

namespace h3dg_tables {

template <int P, int NQ, int NT>
static HoSpec ho_spec() {
	return HoSpec { P, NQ, &h3dg::k_assemble_fp64_ho<P, P, P, NQ, NQ, NQ, NT>, NT,
	                h3dg::HoShape<P, P, P, NQ, NQ, NQ>::SMEM_BYTES, false };
}

std::vector<HoSpec> &ho_table() {
	static std::vector<HoSpec> t = {
		ho_spec<1, 3, 128>(), ho_spec<2, 4, 128>(), ho_spec<3, 5, 256>(), ho_spec<4, 6, 256>(),
		ho_spec<5, 6, 256>(), ho_spec<5, 7, 256>(), ho_spec<6, 7, 256>(), ho_spec<6, 8, 256>(),
		ho_spec<7, 8, 256>(), ho_spec<7, 9, 256>(), ho_spec<8, 9, 256>(), ho_spec<8, 10, 256>(),
		ho_spec<8, 10, 384>(),
	};
	return t;
}

} // namespace h3dg_tables
