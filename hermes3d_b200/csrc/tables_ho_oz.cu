// Kernel variant table (see kernel_tables.h).
#include "kernel_tables.h"
#include "kernels/asm_ho_oz.cuh"

namespace h3dg_tables {

template <int P, int NQ, int MINB = 1>
static HoSpec ho_oz_spec() {
	return HoSpec { P, NQ, &h3dg::k_assemble_ho_oz<P, P, P, NQ, NQ, NQ, MINB>, 256,
	                h3dg::HoOzShape<P, P, P, NQ, NQ, NQ>::SMEM_BYTES, false };
}

std::vector<HoSpec> &ho_oz_table() {
	static std::vector<HoSpec> t = {
		ho_oz_spec<1, 3, 2>(), ho_oz_spec<2, 4, 2>(), ho_oz_spec<3, 5, 2>(), ho_oz_spec<4, 6, 2>(), ho_oz_spec<5, 6>(), ho_oz_spec<5, 7>(), ho_oz_spec<6, 7>(),
		ho_oz_spec<6, 8>(), ho_oz_spec<7, 8>(), ho_oz_spec<7, 9>(), ho_oz_spec<8, 9>(), ho_oz_spec<8, 10>(),
	};
	return t;
}

} // namespace h3dg_tables
