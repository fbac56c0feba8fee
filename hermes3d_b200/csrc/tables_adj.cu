// Kernel variant table (see kernel_tables.h).
#include "kernel_tables.h"

namespace h3dg_tables {

template <int P, int NQ>
static AdjSpec adj_spec() {
	return AdjSpec { P, NQ, &h3dg::k_adjoint<P, P, P, NQ, NQ, NQ, 128>, h3dg::AdjShape<P, P, P, NQ, NQ, NQ>::SMEM_BYTES, false };
}

std::vector<AdjSpec> &adj_table() {
	static std::vector<AdjSpec> t = {
		adj_spec<1, 2>(), adj_spec<1, 3>(), adj_spec<2, 3>(), adj_spec<2, 4>(), adj_spec<3, 4>(), adj_spec<3, 5>(),
		adj_spec<4, 5>(), adj_spec<4, 6>(), adj_spec<5, 6>(), adj_spec<5, 7>(), adj_spec<6, 7>(), adj_spec<6, 8>(),
		adj_spec<8, 10>(),
	};
	return t;
}

} // namespace h3dg_tables
