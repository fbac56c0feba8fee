// C-ABI implementation: handles, device plan, kernel dispatch.
#include "../../include/h3dg.h"
#include "host/h3dg_host.h"
#include "host/lobatto.h"
#include "kernel_tables.h"
#include "kernels/tc_selftest.cuh"
#include "kernels/geom.cuh"
#include "kernels/cg.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

struct h3dg_mesh {
	h3dg::Mesh m;
};

struct h3dg_space {
	h3dg_mesh *mesh = nullptr;
	h3dg::Space s;
};

namespace {

thread_local std::string g_err;

h3dg_status fail(h3dg_status s, const std::string &msg) {
	g_err = msg;
	return s;
}

#define H3DG_CUDA_TRY(call)                                                                              \
	do {                                                                                                 \
		cudaError_t e_ = (call);                                                                         \
		if (e_ != cudaSuccess) return fail(H3DG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
	} while (0)

template <class T>
struct DBuf {
	T *p = nullptr;
	size_t n = 0;
	~DBuf() { release(); }
	void release() {
		if (p) cudaFree(p);
		p = nullptr;
		n = 0;
	}
	cudaError_t alloc(size_t count) {
		release();
		n = count;
		if (count == 0) return cudaSuccess;
		return cudaMalloc((void **) &p, sizeof(T) * count);
	}
	cudaError_t upload(const std::vector<T> &v) {
		cudaError_t e = alloc(v.size());
		if (e != cudaSuccess || v.empty()) return e;
		return cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
	}
};

} // namespace

struct h3dg_disc {
	int device = 0;
	h3dg_space *space = nullptr;
	h3dg_space *test_space = nullptr;  // test space of a system block (nullptr: the trial space)
	int bf = 0;
	std::vector<double> ecoef;       // per element id
	int lf = H3DG_LF_NONE;
	double lf_value = 0.0;
	int qmode = H3DG_QUAD_FIXED, qn = 0;
	DBuf<double> cg_work;            // conjugate-gradient vectors and partial sums
	// evaluation plan (norms), built at the first norms call after create_pattern
	bool have_eval = false;
	int64_t ev_ne = 0;
	int ev_nlmax = 0, ev_amax = 0, ev_bmax = 0;
	DBuf<int32_t> ev_desc, ev_vtx, ev_edof;
	DBuf<int64_t> ev_gptr, ev_eptr;
	DBuf<uint16_t> ev_gs;
	DBuf<double> ev_ecoef, ev_tables, ev_partial, ev_out;
	// surface forms (natural boundary faces)
	int sbf = 0, slf = 0;
	double sg[h3dg::kSurfMarkers] = {};
	DBuf<int32_t> sf_desc, sf_vtx, sf_dof;
	DBuf<int64_t> sf_base, sf_obase;
	DBuf<double> sf_coef, sf_tables;
	DBuf<int16_t> sf_ab;
	DBuf<uint16_t> sf_off;
	bool have_plan = false;
	bool on_device = false;
	int nparts = 1, part = 0;  // z-slab partition of the next plan (1: whole mesh)
	int prec_hint = H3DG_PREC_FP64;   // precision the next plan is built for
	unsigned prepared = 0;     // bit p: an assembly with precision p completed on the current plan
	int debug_once = 0;        // test hook for the next assembly (H3DG_DEBUG_*)
	h3dg::PlanScope scope;     // element subset and owned DOFs of the current plan's part
	int variant = -1;          // autotuned kernel variant (index into the kernel table)
	float variant_ms = 0.0f;
	h3dg::Plan plan;
	int32_t last_launches = 0;
	int32_t last_kind = H3DG_KERNEL_OTHER;   // kernel family of the last volume assembly

	// device plan
	DBuf<double> xyz, coef, tables, qx, qy, qz, Ax, rhs;
	DBuf<int64_t> Ap;
	DBuf<int32_t> Ai, el_vtx, el_cnt, el_dof, el_id;
	DBuf<uint16_t> el_s, el_off, el_offc;
	DBuf<uint16_t> el_offt;    // tensor-core scatter stream (built at the first split-precision assembly)
	bool offt_store_all = false;   // its first-touch stores cover every Ax slot
	DBuf<uint16_t> el_offd;    // FP64 tensor-core scatter stream (built at the first FP64 high-order assembly)
	bool offd_store_all = false;
	DBuf<double> ho_scratch;   // per-CTA global work area of the FP64-accurate split kernel
	DBuf<int32_t> el_cdof, el_tcdof;
	DBuf<double> el_ccoef, el_tccoef;
	DBuf<double> el_coef;
	DBuf<int> status;
	// segmented scatter: plan tables, the item schedule of the current launch
	// shape, counters and the element-matrix ring
	DBuf<int32_t> seg_kof, seg_col, seg_pe, seg_items, seg_p1n, seg_p2n;
	DBuf<int64_t> seg_cptr;
	DBuf<uint16_t> seg_plm, seg_off;
	DBuf<unsigned> seg_ctr;
	DBuf<double> seg_ring;
	int seg_ctas = 0, seg_per_item = 0, seg_nitems = 0, seg_ring_win = 0;
	bool seg_all_dofs = false;  // every DOF has a column (no RHS zero-fill needed)
	int table_bytes = 0;
	// kernel-only timing records
	std::vector<cudaEvent_t> tev;
	int tcap = 0, tn = 0;
	// mixed-order path: plan tables, work counters, tuned variants, and the
	// CUDA graph of one whole assembly (memsets + every launch), cached for
	// the output pointers it was captured with
	DBuf<int32_t> el_desc;
	DBuf<int64_t> el_base, el_obase;
	DBuf<uint16_t> el_offm;
	DBuf<unsigned> mx_counters;
	// elements with constrained nodes: W columns, slot map, per-CTA scratch
	DBuf<int32_t> ce_desc, ce_vtx, ce_id, ce_udof, ce_order;
	DBuf<int64_t> ce_ubase, ce_wptr, ce_obase, ce_ebase;
	DBuf<uint16_t> ce_ws, ce_off;
	DBuf<double> ce_ww, ce_scratch, ce_out;
	int64_t ce_stride = 0;
	int ce_per_sm[h3dg::Plan::kCedClasses] = { 1, 1, 1 };
	int mx_variant[h3dg::Plan::kClasses] = { -1, -1, -1 };
	cudaGraphExec_t mx_exec = nullptr;
	double *mx_ax = nullptr, *mx_rhs = nullptr;
	const double *mx_coef = nullptr;   // coefficient array the graph was captured with
	int32_t mx_launches = 0;
	cudaStream_t mx_s[3] = { nullptr, nullptr, nullptr };
	cudaEvent_t mx_ev[5] = { nullptr, nullptr, nullptr, nullptr, nullptr };
	void reset_mixed() {
		if (mx_exec) cudaGraphExecDestroy(mx_exec);
		mx_exec = nullptr;
		mx_ax = mx_rhs = nullptr;
		for (int c = 0; c < h3dg::Plan::kClasses; c++) mx_variant[c] = -1;
	}
	~h3dg_disc() {
		for (auto e : tev) cudaEventDestroy(e);
		reset_mixed();
		for (auto s : mx_s)
			if (s) cudaStreamDestroy(s);
		for (auto e : mx_ev)
			if (e) cudaEventDestroy(e);
	}
};

extern "C" {

int h3dg_version(void) { return 1; }

const char *h3dg_status_string(h3dg_status s) {
	switch (s) {
		case H3DG_OK: return "ok";
		case H3DG_ERR_INVALID_ARG: return "invalid argument";
		case H3DG_ERR_CUDA: return "CUDA error";
		case H3DG_ERR_OUT_OF_MEMORY: return "out of memory";
		case H3DG_ERR_UNSUPPORTED_FORM: return "unsupported form";
		case H3DG_ERR_MESH: return "mesh error";
		case H3DG_ERR_STATE: return "call out of order";
		case H3DG_ERR_TIMEOUT: return "device wait timed out";
		case H3DG_ERR_TOO_LARGE: return "size limit exceeded";
		default: return "unknown status";
	}
}

const char *h3dg_last_error(void) { return g_err.c_str(); }

// ---------------------------------------------------------------- mesh

h3dg_status h3dg_mesh_create(h3dg_mesh **mesh) {
	if (!mesh) return fail(H3DG_ERR_INVALID_ARG, "mesh: null output pointer");
	*mesh = new (std::nothrow) h3dg_mesh();
	return *mesh ? H3DG_OK : fail(H3DG_ERR_OUT_OF_MEMORY, "mesh: allocation failed");
}

h3dg_status h3dg_mesh_destroy(h3dg_mesh *mesh) {
	delete mesh;
	return H3DG_OK;
}

h3dg_status h3dg_mesh_add_vertices(h3dg_mesh *mesh, const double *xyz, int64_t n) {
	if (!mesh || (n > 0 && !xyz) || n < 0) return fail(H3DG_ERR_INVALID_ARG, "add_vertices: bad arguments");
	if (mesh->m.finalized) return fail(H3DG_ERR_STATE, "add_vertices: mesh already finalized");
	mesh->m.xyz.insert(mesh->m.xyz.end(), xyz, xyz + 3 * n);
	return H3DG_OK;
}

h3dg_status h3dg_mesh_add_hexes(h3dg_mesh *mesh, const int64_t *vtx, int64_t n) {
	if (!mesh || (n > 0 && !vtx) || n < 0) return fail(H3DG_ERR_INVALID_ARG, "add_hexes: bad arguments");
	if (mesh->m.finalized) return fail(H3DG_ERR_STATE, "add_hexes: mesh already finalized");
	for (int64_t i = 0; i < 8 * n; i++) mesh->m.hex.push_back(vtx[i] - 1);
	return H3DG_OK;
}

h3dg_status h3dg_mesh_add_quad_boundaries(h3dg_mesh *mesh, const int64_t *vtx, const int32_t *marker, int64_t n) {
	if (!mesh || (n > 0 && (!vtx || !marker)) || n < 0) return fail(H3DG_ERR_INVALID_ARG, "add_quad_boundaries: bad arguments");
	if (mesh->m.finalized) return fail(H3DG_ERR_STATE, "add_quad_boundaries: mesh already finalized");
	for (int64_t i = 0; i < n; i++) {
		mesh->m.bquad.push_back({ vtx[4 * i] - 1, vtx[4 * i + 1] - 1, vtx[4 * i + 2] - 1, vtx[4 * i + 3] - 1 });
		mesh->m.bmarker.push_back(marker[i]);
	}
	return H3DG_OK;
}

h3dg_status h3dg_mesh_finalize(h3dg_mesh *mesh) {
	if (!mesh) return fail(H3DG_ERR_INVALID_ARG, "finalize: null mesh");
	std::string err;
	if (mesh->m.finalize(err) != 0) return fail(H3DG_ERR_MESH, err);
	return H3DG_OK;
}

h3dg_status h3dg_mesh_refine_element(h3dg_mesh *mesh, int64_t elem_id, int reft) {
	if (!mesh) return fail(H3DG_ERR_INVALID_ARG, "refine_element: null mesh");
	if (!mesh->m.finalized) return fail(H3DG_ERR_STATE, "refine_element: mesh not finalized");
	if (reft != 7) return fail(H3DG_ERR_MESH, "refine_element: only REFT_HEX_XYZ (7) is supported");
	if (elem_id < 1 || elem_id > mesh->m.ne()) return fail(H3DG_ERR_INVALID_ARG, "refine_element: element id out of range");
	std::string err;
	if (mesh->m.refine_xyz(elem_id - 1, err) != 0) return fail(H3DG_ERR_MESH, err);
	return H3DG_OK;
}

h3dg_status h3dg_mesh_refine_elements(h3dg_mesh *mesh, const int64_t *elem_ids, int64_t n, int reft) {
	if (!mesh || (n > 0 && !elem_ids) || n < 0) return fail(H3DG_ERR_INVALID_ARG, "refine_elements: bad arguments");
	if (!mesh->m.finalized) return fail(H3DG_ERR_STATE, "refine_elements: mesh not finalized");
	if (reft != 7) return fail(H3DG_ERR_MESH, "refine_elements: only REFT_HEX_XYZ (7) is supported");
	std::string err;
	for (int64_t i = 0; i < n; i++) {
		if (elem_ids[i] < 1 || elem_ids[i] > mesh->m.ne()) err = "refine_elements: element id out of range";
		else if (mesh->m.refine_xyz(elem_ids[i] - 1, err, false) != 0) {}
		if (!err.empty()) {
			std::string e2;
			mesh->m.finalize(e2);
			return fail(H3DG_ERR_MESH, err);
		}
	}
	if (mesh->m.finalize(err) != 0) return fail(H3DG_ERR_MESH, err);
	return H3DG_OK;
}

h3dg_status h3dg_mesh_get_arrays(const h3dg_mesh *mesh, double *xyz, int64_t *hex, int64_t *parent) {
	if (!mesh) return fail(H3DG_ERR_INVALID_ARG, "get_arrays: null mesh");
	const h3dg::Mesh &m = mesh->m;
	if (xyz) std::copy(m.xyz.begin(), m.xyz.end(), xyz);
	if (hex)
		for (size_t i = 0; i < m.hex.size(); i++) hex[i] = m.hex[i] + 1;
	if (parent)
		for (int64_t e = 0; e < m.ne(); e++) parent[e] = m.parent.empty() ? 0 : m.parent[e] + 1;
	return H3DG_OK;
}

h3dg_status h3dg_mesh_counts(const h3dg_mesh *mesh, int64_t *nv, int64_t *ne, int64_t *nfacets, int64_t *nedges) {
	if (!mesh) return fail(H3DG_ERR_INVALID_ARG, "counts: null mesh");
	if (nv) *nv = mesh->m.nv();
	if (ne) *ne = mesh->m.ne();
	if (nfacets) *nfacets = mesh->m.nfacets;
	if (nedges) *nedges = mesh->m.nedges;
	return H3DG_OK;
}

// ---------------------------------------------------------------- space

h3dg_status h3dg_space_create(h3dg_mesh *mesh, h3dg_space **space) {
	if (!mesh || !space) return fail(H3DG_ERR_INVALID_ARG, "space_create: bad arguments");
	if (!mesh->m.finalized) return fail(H3DG_ERR_STATE, "space_create: mesh not finalized");
	h3dg_space *s = new (std::nothrow) h3dg_space();
	if (!s) return fail(H3DG_ERR_OUT_OF_MEMORY, "space_create: allocation failed");
	s->mesh = mesh;
	s->s.mesh = &mesh->m;
	*space = s;
	return H3DG_OK;
}

h3dg_status h3dg_space_destroy(h3dg_space *space) {
	delete space;
	return H3DG_OK;
}

h3dg_status h3dg_space_set_bc_types(h3dg_space *space, h3dg_bc_type_fn fn, void *ctx) {
	if (!space) return fail(H3DG_ERR_INVALID_ARG, "set_bc_types: null space");
	space->s.bc_type_fn = fn;
	space->s.bc_type_ctx = ctx;
	return H3DG_OK;
}

h3dg_status h3dg_space_set_bc_values(h3dg_space *space, h3dg_bc_value_fn fn, void *ctx) {
	if (!space) return fail(H3DG_ERR_INVALID_ARG, "set_bc_values: null space");
	space->s.bc_value_fn = fn;
	space->s.bc_value_ctx = ctx;
	return H3DG_OK;
}

h3dg_status h3dg_space_set_uniform_order(h3dg_space *space, int px, int py, int pz) {
	if (!space) return fail(H3DG_ERR_INVALID_ARG, "set_uniform_order: null space");
	if (px < 1 || py < 1 || pz < 1 || px > h3dg::kMaxOrder || py > h3dg::kMaxOrder || pz > h3dg::kMaxOrder)
		return fail(H3DG_ERR_INVALID_ARG, "set_uniform_order: order out of range 1..10");
	int64_t ne = space->s.mesh->ne();
	space->s.order.resize(3 * ne);
	for (int64_t e = 0; e < ne; e++) {
		space->s.order[3 * e] = px;
		space->s.order[3 * e + 1] = py;
		space->s.order[3 * e + 2] = pz;
	}
	space->s.assigned = false;
	return H3DG_OK;
}

h3dg_status h3dg_space_set_element_orders(h3dg_space *space, const int32_t *orders, int64_t ne) {
	if (!space || !orders || ne != space->s.mesh->ne()) return fail(H3DG_ERR_INVALID_ARG, "set_element_orders: bad arguments");
	for (int64_t i = 0; i < 3 * ne; i++)
		if (orders[i] < 1 || orders[i] > h3dg::kMaxOrder) return fail(H3DG_ERR_INVALID_ARG, "set_element_orders: order out of range 1..10");
	space->s.order.assign(orders, orders + 3 * ne);
	space->s.assigned = false;
	return H3DG_OK;
}

h3dg_status h3dg_space_assign_dofs(h3dg_space *space, int first_dof, int stride, int64_t *ndof) {
	if (!space || stride < 1 || first_dof < 0) return fail(H3DG_ERR_INVALID_ARG, "assign_dofs: bad arguments");
	std::string err;
	if (space->s.assign_dofs(first_dof, stride, err) != 0) return fail(H3DG_ERR_STATE, "assign_dofs: " + err);
	if (ndof) *ndof = space->s.ndof();
	return H3DG_OK;
}

h3dg_status h3dg_space_get_element_assembly_list(const h3dg_space *space, int64_t elem_id, int64_t *idx, int32_t *dof,
                                                 double *coef, int32_t cap, int32_t *cnt) {
	if (!space || !space->s.assigned) return fail(H3DG_ERR_STATE, "get_element_assembly_list: assign_dofs() first");
	if (elem_id < 1 || elem_id > space->s.mesh->ne()) return fail(H3DG_ERR_INVALID_ARG, "get_element_assembly_list: element id out of range");
	std::vector<h3dg::AsmEntry> al;
	space->s.element_assembly_list(elem_id - 1, al);
	if (cnt) *cnt = (int32_t) al.size();
	for (int32_t i = 0; i < cap && i < (int32_t) al.size(); i++) {
		if (idx) idx[i] = al[i].idx;
		if (dof) dof[i] = al[i].dof;
		if (coef) coef[i] = al[i].coef;
	}
	return H3DG_OK;
}

// ---------------------------------------------------------------- discretization

h3dg_status h3dg_disc_create(h3dg_disc **disc, int device) {
	if (!disc) return fail(H3DG_ERR_INVALID_ARG, "disc_create: null output pointer");
	h3dg_disc *d = new (std::nothrow) h3dg_disc();
	if (!d) return fail(H3DG_ERR_OUT_OF_MEMORY, "disc_create: allocation failed");
	d->device = device;
	*disc = d;
	return H3DG_OK;
}

h3dg_status h3dg_disc_destroy(h3dg_disc *disc) {
	if (!disc) return H3DG_OK;
	cudaSetDevice(disc->device);
	delete disc;
	return H3DG_OK;
}

h3dg_status h3dg_disc_set_space(h3dg_disc *disc, h3dg_space *space) {
	if (!disc || !space) return fail(H3DG_ERR_INVALID_ARG, "set_space: bad arguments");
	disc->space = space;
	disc->have_plan = false;
	return H3DG_OK;
}

h3dg_status h3dg_disc_set_test_space(h3dg_disc *disc, h3dg_space *test) {
	if (!disc) return fail(H3DG_ERR_INVALID_ARG, "set_test_space: bad arguments");
	disc->test_space = test;
	disc->have_plan = false;
	return H3DG_OK;
}

h3dg_status h3dg_disc_set_bilinear_form(h3dg_disc *disc, int form, const double *elem_coef, int64_t ne) {
	if (!disc) return fail(H3DG_ERR_INVALID_ARG, "set_bilinear_form: null disc");
	if (form != H3DG_BF_GRAD_GRAD && form != H3DG_BF_GRAD_GRAD_MASS)
		return fail(H3DG_ERR_UNSUPPORTED_FORM, "set_bilinear_form: only int_grad_u_grad_v and int_grad_u_grad_v + int_u_v run on the device");
	disc->bf = form;
	if (elem_coef) {
		if (!disc->space || ne != disc->space->s.mesh->ne()) return fail(H3DG_ERR_INVALID_ARG, "set_bilinear_form: coefficient count != elements");
		disc->ecoef.assign(elem_coef, elem_coef + ne);
	}
	else disc->ecoef.clear();
	disc->have_plan = false;
	return H3DG_OK;
}

h3dg_status h3dg_disc_set_linear_form(h3dg_disc *disc, int form, double value) {
	if (!disc) return fail(H3DG_ERR_INVALID_ARG, "set_linear_form: null disc");
	if (form != H3DG_LF_NONE && form != H3DG_LF_CONST && form != H3DG_LF_SIN)
		return fail(H3DG_ERR_UNSUPPORTED_FORM, "set_linear_form: unknown linear form");
	disc->lf = form;
	disc->lf_value = value;
	return H3DG_OK;
}

h3dg_status h3dg_disc_set_surface_forms(h3dg_disc *disc, int bilinear, int linear, const double *g, int ng) {
	if (!disc) return fail(H3DG_ERR_INVALID_ARG, "set_surface_forms: null disc");
	if ((bilinear != H3DG_SBF_NONE && bilinear != H3DG_SBF_U_V) || (linear != H3DG_SLF_NONE && linear != H3DG_SLF_G_V))
		return fail(H3DG_ERR_UNSUPPORTED_FORM, "set_surface_forms: unknown surface form");
	if (ng < 0 || ng > h3dg::kSurfMarkers || (ng > 0 && !g))
		return fail(H3DG_ERR_INVALID_ARG, "set_surface_forms: g needs 0..16 values (markers 0..15)");
	disc->sbf = bilinear;
	disc->slf = linear;
	for (int m = 0; m < h3dg::kSurfMarkers; m++) disc->sg[m] = m < ng ? g[m] : 0.0;
	return H3DG_OK;
}

h3dg_status h3dg_disc_set_quadrature(h3dg_disc *disc, int mode, int n) {
	if (!disc || (mode != H3DG_QUAD_FIXED && mode != H3DG_QUAD_P_PLUS && mode != H3DG_QUAD_STOCK) || n < 0 ||
	    n > h3dg::kMaxQuadPoints)
		return fail(H3DG_ERR_INVALID_ARG, "set_quadrature: bad arguments");
	disc->qmode = mode;
	disc->qn = n;
	disc->have_plan = false;
	return H3DG_OK;
}

static void build_table_blob(const h3dg::Plan &P, std::vector<double> &blob) {
	// layout of SfShape: Vx Dx Vy Dy Vz Dz, then qx wx qy wy qz wz; padded to 16 bytes
	blob.clear();
	auto put_dir = [&](int p, const std::vector<double> &q) {
		for (int k = 0; k <= p; k++)
			for (size_t i = 0; i < q.size(); i++) blob.push_back(h3dg::lobatto_value(k, q[i]));
		for (int k = 0; k <= p; k++)
			for (size_t i = 0; i < q.size(); i++) blob.push_back(h3dg::lobatto_deriv(k, q[i]));
	};
	put_dir(P.px, P.qx);
	put_dir(P.py, P.qy);
	put_dir(P.pz, P.qz);
	blob.insert(blob.end(), P.qx.begin(), P.qx.end());
	blob.insert(blob.end(), P.wx.begin(), P.wx.end());
	blob.insert(blob.end(), P.qy.begin(), P.qy.end());
	blob.insert(blob.end(), P.wy.begin(), P.wy.end());
	blob.insert(blob.end(), P.qz.begin(), P.qz.end());
	blob.insert(blob.end(), P.wz.begin(), P.wz.end());
	if (blob.size() % 2) blob.push_back(0.0);
}

// 1D tables of the stock rule (layout of StockShape): the rules of 2 .. p+1
// points concatenated (points, weights, Lobatto values and derivatives at
// them), then the 13-point rule of the load vector (points, weights, values)
static void build_stock_blob(int p, std::vector<double> &blob) {
	blob.clear();
	std::vector<double> qc, wc, q, w;
	for (int n = 2; n <= p + 1; n++) {
		h3dg::gauss_legendre(n, q, w);
		qc.insert(qc.end(), q.begin(), q.end());
		wc.insert(wc.end(), w.begin(), w.end());
	}
	blob.insert(blob.end(), qc.begin(), qc.end());
	blob.insert(blob.end(), wc.begin(), wc.end());
	for (int k = 0; k <= p; k++)
		for (double x : qc) blob.push_back(h3dg::lobatto_value(k, x));
	for (int k = 0; k <= p; k++)
		for (double x : qc) blob.push_back(h3dg::lobatto_deriv(k, x));
	h3dg::gauss_legendre(13, q, w);
	blob.insert(blob.end(), q.begin(), q.end());
	blob.insert(blob.end(), w.begin(), w.end());
	for (int k = 0; k <= p; k++)
		for (double x : q) blob.push_back(h3dg::lobatto_value(k, x));
	if (blob.size() % 2) blob.push_back(0.0);
}

h3dg_status h3dg_disc_create_pattern(h3dg_disc *disc, int64_t *ndof, int64_t *nnz) {
	if (!disc || !disc->space) return fail(H3DG_ERR_STATE, "create_pattern: set_space() first");
	if (!disc->space->s.assigned) return fail(H3DG_ERR_STATE, "create_pattern: assign_dofs() first");
	if (!disc->bf) return fail(H3DG_ERR_STATE, "create_pattern: set_bilinear_form() first");
	const h3dg::Space &sp = disc->space->s;
	int nq[3];
	for (int d = 0; d < 3; d++)
		nq[d] = disc->qmode == H3DG_QUAD_FIXED ? disc->qn : disc->qmode == H3DG_QUAD_STOCK ? 2 : sp.order[d] + disc->qn;
	std::string err;
	// orders >= 5: the element matrix does not fit in shared memory; the
	// high-order kernel works on canonical tables
	int pmax = 0;
	for (size_t i = 0; i < sp.order.size(); i++) pmax = std::max(pmax, sp.order[i]);
	// H3DG_FORCE_HIGH_ORDER=1 routes every order through the high-order kernel
	// (used by the parity tests to check that kernel on the low-order fixtures)
	const char *force = std::getenv("H3DG_FORCE_HIGH_ORDER");
	// at p = 4 the tensor-core kernels (FP64 DMMA, or 3xTF32 when intended) are
	// faster than the low-order FP64 kernel: uniform p = 4 with a rule the FP64
	// tensor-core kernel is instantiated for takes the high-order path
	bool dm4 = false;
	if (pmax == 4 && disc->qmode != H3DG_QUAD_STOCK && nq[0] == nq[1] && nq[1] == nq[2])
		for (auto &k : h3dg_tables::dm_table())
			if (k.p == 4 && k.nq == nq[0]) dm4 = true;
	const int canon_from = disc->prec_hint == H3DG_PREC_TF32X3 || dm4 ? 4 : 5;
	const bool canon = pmax >= canon_from || (force && force[0] == '1');
	// elements of different order triples: the mixed-order (batched) path;
	// H3DG_FORCE_MIXED=1 routes uniform spaces there too (parity tests)
	bool mixed = false;
	for (int64_t e = 1; e < (int64_t) sp.order.size() / 3 && !mixed; e++)
		for (int d = 0; d < 3; d++)
			if (sp.order[3 * e + d] != sp.order[d]) mixed = true;
	const char *force_mixed = std::getenv("H3DG_FORCE_MIXED");
	if (force_mixed && force_mixed[0] == '1') mixed = true;
	// refined meshes (hanging nodes) always take the batched path
	if (sp.mesh->nrefined) mixed = true;
	disc->reset_mixed();
	const h3dg::PlanScope *scope = nullptr;
	disc->scope = h3dg::PlanScope();
	if (disc->nparts > 1) {
		if (h3dg::make_partition_scope(sp, disc->nparts, disc->part, disc->scope, err) != 0)
			return fail(H3DG_ERR_INVALID_ARG, "create_pattern: " + err);
		scope = &disc->scope;
	}
	const h3dg::Space *tsp = disc->test_space && disc->test_space != disc->space ? &disc->test_space->s : nullptr;
	if (tsp) {
		// a block of a system with two different spaces: canonical FP64 plan at the
		// larger order, rows from the test space, columns from the trial space
		bool tmixed = false;
		for (int64_t e = 1; e < (int64_t) tsp->order.size() / 3 && !tmixed; e++)
			for (int d = 0; d < 3; d++)
				if (tsp->order[3 * e + d] != tsp->order[d]) tmixed = true;
		if (!tsp->assigned) return fail(H3DG_ERR_STATE, "create_pattern: assign_dofs() on the test space first");
		if (tsp->mesh != sp.mesh || mixed || tmixed || sp.mesh->nrefined || disc->nparts > 1 || disc->sbf || disc->slf ||
		    disc->qmode == H3DG_QUAD_STOCK)
			return fail(H3DG_ERR_INVALID_ARG, "create_pattern: a block with two spaces needs one mesh, uniform orders in "
			                                  "each space, no refinement, partition, surface forms or stock rule");
		for (int d = 0; d < 3; d++)
			if (disc->qmode == H3DG_QUAD_P_PLUS) nq[d] = std::max(sp.order[d], tsp->order[d]) + disc->qn;
		disc->reset_mixed();
		disc->scope = h3dg::PlanScope();
		if (h3dg::build_plan(sp, nq[0], nq[1], nq[2], disc->plan, err, true, nullptr, tsp) != 0)
			return fail(H3DG_ERR_INVALID_ARG, "create_pattern: " + err);
		const h3dg::Plan &P2 = disc->plan;
		disc->on_device = false;
		disc->have_plan = true;
		disc->prepared = 0;
		disc->have_eval = false;
		disc->variant = -1;
		if (ndof) *ndof = P2.ndof;
		if (nnz) *nnz = P2.nnz;
		return H3DG_OK;
	}
	if (disc->qmode == H3DG_QUAD_STOCK) {
		// the stock rule: uniform orders 1..3, whole elements (no hanging nodes), volume forms
		if (mixed || canon || sp.order[0] != sp.order[1] || sp.order[0] != sp.order[2] || pmax > 3 || disc->sbf ||
		    disc->slf)
			return fail(H3DG_ERR_INVALID_ARG, "create_pattern: the stock quadrature needs one order 1..3 in every "
			                                  "direction, no refinement and no surface forms");
	}
	if (mixed) {
		if (h3dg::build_plan_mixed(sp, disc->qmode == H3DG_QUAD_P_PLUS, disc->qn, disc->plan, err, scope) != 0)
			return fail(H3DG_ERR_INVALID_ARG, "create_pattern: " + err);
	}
	else if (h3dg::build_plan(sp, nq[0], nq[1], nq[2], disc->plan, err, canon, scope) != 0)
		return fail(H3DG_ERR_INVALID_ARG, "create_pattern: " + err);
	if ((disc->sbf || disc->slf) &&
	    h3dg::build_surface_plan(sp, disc->qmode == H3DG_QUAD_P_PLUS, disc->qn, disc->plan, err) != 0)
		return fail(H3DG_ERR_INVALID_ARG, "create_pattern: " + err);
	const h3dg::Plan &P = disc->plan;
	disc->on_device = false;
	disc->have_plan = true;
	disc->prepared = 0;
	disc->have_eval = false;
	disc->variant = -1;
	if (ndof) *ndof = P.ndof;
	if (nnz) *nnz = P.nnz;
	return H3DG_OK;
}

// Device copy of the plan, made on the first device call (create() itself
// is host work, as in the reference).
static h3dg_status noalloc_scratch(double **out);

static h3dg_status ensure_device(h3dg_disc *disc) {
	if (disc->on_device) return H3DG_OK;
	const h3dg::Space &sp = disc->space->s;
	const h3dg::Plan &P = disc->plan;
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	H3DG_CUDA_TRY(disc->xyz.upload(sp.mesh->xyz));
	H3DG_CUDA_TRY(disc->Ap.upload(P.Ap));
	H3DG_CUDA_TRY(disc->Ai.upload(P.Ai));
	H3DG_CUDA_TRY(disc->el_vtx.upload(P.el_vtx));
	H3DG_CUDA_TRY(disc->el_cnt.upload(P.el_cnt));
	H3DG_CUDA_TRY(disc->el_id.upload(P.el_id));
	if (P.mixed) {
		H3DG_CUDA_TRY(disc->el_desc.upload(P.el_desc));
		H3DG_CUDA_TRY(disc->el_base.upload(P.el_base));
		H3DG_CUDA_TRY(disc->el_obase.upload(P.el_obase));
		H3DG_CUDA_TRY(disc->el_cdof.upload(P.el_cdof));
		H3DG_CUDA_TRY(disc->el_ccoef.upload(P.el_ccoef));
		H3DG_CUDA_TRY(disc->el_offm.upload(P.el_offm));
		H3DG_CUDA_TRY(disc->mx_counters.alloc((size_t) P.ncolors * (h3dg::Plan::kClasses + h3dg::Plan::kCedClasses)));
		if (P.nce > 0) {
			H3DG_CUDA_TRY(disc->ce_desc.upload(P.ce_desc));
			H3DG_CUDA_TRY(disc->ce_vtx.upload(P.ce_vtx));
			H3DG_CUDA_TRY(disc->ce_id.upload(P.ce_id));
			H3DG_CUDA_TRY(disc->ce_udof.upload(P.ce_udof));
			H3DG_CUDA_TRY(disc->ce_ubase.upload(P.ce_ubase));
			H3DG_CUDA_TRY(disc->ce_wptr.upload(P.ce_wptr));
			H3DG_CUDA_TRY(disc->ce_obase.upload(P.ce_obase));
			H3DG_CUDA_TRY(disc->ce_ws.upload(P.ce_ws));
			H3DG_CUDA_TRY(disc->ce_off.upload(P.ce_off));
			H3DG_CUDA_TRY(disc->ce_ww.upload(P.ce_ww));
			H3DG_CUDA_TRY(disc->ce_order.upload(P.ce_order));
			H3DG_CUDA_TRY(disc->ce_ebase.upload(P.ce_ebase));
			H3DG_CUDA_TRY(disc->ce_out.alloc((size_t) P.ce_ebase.back()));
			// per-CTA scratch (element matrix + load vector) for every resident CTA
			int nsm = 148;
			cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
			const int table_bytes = (int) (P.mixed_tables.size() * sizeof(double));
			int64_t blocks = 0;
			for (int cls = 0; cls < h3dg::Plan::kCedClasses; cls++) {
				h3dg_tables::CedSpec &k = h3dg_tables::ced_table()[cls];
				const size_t smem = k.smem(table_bytes);
				if (!k.configured || k.configured_smem < smem) {
					H3DG_CUDA_TRY(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
					k.configured = true;
					k.configured_smem = smem;
				}
				int per_sm = 1;
				cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.threads, smem);
				disc->ce_per_sm[cls] = per_sm < 1 ? 1 : per_sm;
				blocks = std::max<int64_t>(blocks, (int64_t) nsm * disc->ce_per_sm[cls]);
			}
			disc->ce_stride = (P.ce_scratch + 1) / 2 * 2;
			H3DG_CUDA_TRY(disc->ce_scratch.alloc((size_t) (disc->ce_stride * blocks)));
		}
		disc->el_offc.release();
		disc->el_offt.release();
		disc->offt_store_all = false;
		disc->el_offd.release();
		disc->offd_store_all = false;
	}
	else if (P.canon) {
		H3DG_CUDA_TRY(disc->el_cdof.upload(P.el_cdof));
		H3DG_CUDA_TRY(disc->el_ccoef.upload(P.el_ccoef));
		if (P.two_space) {
			H3DG_CUDA_TRY(disc->el_tcdof.upload(P.el_tcdof));
			H3DG_CUDA_TRY(disc->el_tccoef.upload(P.el_tccoef));
		}
		H3DG_CUDA_TRY(disc->el_offc.upload(P.el_offc));
		disc->el_offt.release();
		disc->offt_store_all = false;
		disc->el_offd.release();
		disc->offd_store_all = false;
	}
	else {
		H3DG_CUDA_TRY(disc->el_s.upload(P.el_s));
		H3DG_CUDA_TRY(disc->el_dof.upload(P.el_dof));
		H3DG_CUDA_TRY(disc->el_coef.upload(P.el_coef));
		H3DG_CUDA_TRY(disc->el_off.upload(P.el_off));
		if (P.seg) {
			H3DG_CUDA_TRY(disc->seg_kof.upload(P.seg_kof));
			H3DG_CUDA_TRY(disc->seg_col.upload(P.seg_col));
			H3DG_CUDA_TRY(disc->seg_cptr.upload(P.seg_cptr));
			H3DG_CUDA_TRY(disc->seg_pe.upload(P.seg_pe));
			H3DG_CUDA_TRY(disc->seg_plm.upload(P.seg_plm));
			H3DG_CUDA_TRY(disc->seg_off.upload(P.seg_off));
			disc->seg_all_dofs = (int64_t) P.seg_col.size() == P.ndof;
		}
		disc->seg_ctas = 0;
	}
	if (P.nsf > 0) {
		H3DG_CUDA_TRY(disc->sf_desc.upload(P.sf_desc));
		H3DG_CUDA_TRY(disc->sf_vtx.upload(P.sf_vtx));
		H3DG_CUDA_TRY(disc->sf_dof.upload(P.sf_dof));
		H3DG_CUDA_TRY(disc->sf_base.upload(P.sf_base));
		H3DG_CUDA_TRY(disc->sf_obase.upload(P.sf_obase));
		H3DG_CUDA_TRY(disc->sf_coef.upload(P.sf_coef));
		H3DG_CUDA_TRY(disc->sf_tables.upload(P.sf_tables));
		H3DG_CUDA_TRY(disc->sf_ab.upload(P.sf_ab));
		H3DG_CUDA_TRY(disc->sf_off.upload(P.sf_off));
	}
	std::vector<double> blob;
	if (P.mixed) blob = P.mixed_tables;
	else if (disc->qmode == H3DG_QUAD_STOCK) build_stock_blob(P.px, blob);
	else build_table_blob(P, blob);
	disc->table_bytes = (int) (blob.size() * sizeof(double));
	H3DG_CUDA_TRY(disc->tables.upload(blob));
	H3DG_CUDA_TRY(disc->qx.upload(P.qx));
	H3DG_CUDA_TRY(disc->qy.upload(P.qy));
	H3DG_CUDA_TRY(disc->qz.upload(P.qz));
	if (!disc->ecoef.empty()) H3DG_CUDA_TRY(disc->coef.upload(disc->ecoef));
	else disc->coef.release();
	H3DG_CUDA_TRY(disc->status.alloc(1));
	H3DG_CUDA_TRY(cudaMemset(disc->status.p, 0, sizeof(int)));
	// the module holding the no-allocation staging array is loaded on first
	// use (lazy loading), which allocates it: do that here, in an allocating call
	{
		double *scratch = nullptr;
		h3dg_status s0 = noalloc_scratch(&scratch);
		if (s0 != H3DG_OK) return s0;
	}
	disc->on_device = true;
	return H3DG_OK;
}

h3dg_status h3dg_disc_set_precision(h3dg_disc *disc, int precision) {
	if (!disc || (precision != H3DG_PREC_FP64 && precision != H3DG_PREC_TF32X3 && precision != H3DG_PREC_OZAKI))
		return fail(H3DG_ERR_INVALID_ARG, "set_precision: unknown precision");
	disc->prec_hint = precision;
	disc->have_plan = false;
	return H3DG_OK;
}

h3dg_status h3dg_disc_set_partition(h3dg_disc *disc, int nparts, int part) {
	if (!disc || nparts < 1 || part < 0 || part >= nparts) return fail(H3DG_ERR_INVALID_ARG, "set_partition: need 0 <= part < nparts");
	disc->nparts = nparts;
	disc->part = part;
	disc->have_plan = false;
	return H3DG_OK;
}

h3dg_status h3dg_disc_get_partition(const h3dg_disc *disc, uint8_t *owned, int64_t *nslab, int64_t *nhalo, int64_t *nowned) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "get_partition: create_pattern() first");
	const int64_t nd = disc->plan.ndof;
	const bool whole = disc->nparts <= 1;
	if (owned) {
		if (whole) std::memset(owned, 1, (size_t) nd);
		else
			for (int64_t d = 0; d < nd; d++) owned[d] = (uint8_t) disc->scope.owned[d];
	}
	if (nslab) *nslab = whole ? disc->plan.ne : disc->scope.nslab;
	if (nhalo) *nhalo = whole ? 0 : disc->scope.nhalo;
	if (nowned) *nowned = whole ? nd : disc->scope.nowned;
	return H3DG_OK;
}

h3dg_status h3dg_disc_get_partition_elements(const h3dg_disc *disc, uint8_t *in_part, int64_t ne) {
	if (!disc || !disc->have_plan || !in_part) return fail(H3DG_ERR_STATE, "get_partition_elements: create_pattern() first");
	if (ne != disc->space->s.mesh->ne()) return fail(H3DG_ERR_INVALID_ARG, "get_partition_elements: ne must be the mesh's element count");
	if (disc->nparts <= 1) {
		std::memset(in_part, 1, (size_t) ne);
		return H3DG_OK;
	}
	std::memset(in_part, 0, (size_t) ne);
	for (int64_t e : disc->scope.elems) in_part[e] = 1;
	return H3DG_OK;
}

h3dg_status h3dg_disc_get_pattern(const h3dg_disc *disc, int64_t *Ap, int32_t *Ai) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "get_pattern: create_pattern() first");
	if (Ap) std::memcpy(Ap, disc->plan.Ap.data(), sizeof(int64_t) * disc->plan.Ap.size());
	if (Ai) std::memcpy(Ai, disc->plan.Ai.data(), sizeof(int32_t) * disc->plan.Ai.size());
	return H3DG_OK;
}

} // extern "C"

using namespace h3dg_tables;

extern "C" {

// The high-order kernel of a precision for the current plan, its resident
// CTAs per SM and the doubles of the per-CTA work area it needs (FP64-accurate
// split only; 0 otherwise).
static h3dg_status ho_select(h3dg_disc *disc, int precision, HoSpec **out, int *per_sm_out, size_t *scratch_need) {
	const h3dg::Plan &P = disc->plan;
	std::vector<HoSpec> &table = precision == H3DG_PREC_TF32X3 ? ho_tc_table()
	                             : precision == H3DG_PREC_OZAKI ? ho_oz_table() : ho_table();
	HoSpec *k = nullptr;
	for (size_t i = 0; i < table.size(); i++)
		if (table[i].p == P.px && table[i].nq == P.nqx) k = &table[i];
	if (!k) return fail(H3DG_ERR_INVALID_ARG, "assemble: no high-order kernel instantiated for this order / rule / precision");
	if (!k->configured) {
		H3DG_CUDA_TRY(cudaFuncSetAttribute(k->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) k->smem));
		k->configured = true;
	}
	int nsm = 148, per_sm = 1;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k->fn, k->threads, k->smem);
	if (per_sm < 1) per_sm = 1;
	*out = k;
	*per_sm_out = per_sm;
	// G of every resident CTA: 8 x points doubles each (L2-resident)
	*scratch_need = precision == H3DG_PREC_OZAKI ? (size_t) nsm * per_sm * 8 * (size_t) P.nqx * P.nqy * P.nqz : 0;
	return H3DG_OK;
}

// The FP64 tensor-core kernel for the current plan, or nullptr (two-space
// blocks, orders / rules without an instance, or H3DG_HO_FP64_FMA=1, which
// keeps the FMA kernel: tests compare the two)
static DmSpec *dm_select(h3dg_disc *disc, int precision) {
	const h3dg::Plan &P = disc->plan;
	if (precision != H3DG_PREC_FP64 || P.two_space) return nullptr;
	const char *fma = std::getenv("H3DG_HO_FP64_FMA");
	if (fma && fma[0] == '1') return nullptr;
	const char *var = std::getenv("H3DG_DM_VARIANT");
	int want = var ? std::atoi(var) : 0, seen = 0;
	DmSpec *first = nullptr;
	for (auto &k : dm_table())
		if (k.p == P.px && k.nq == P.nqx) {
			if (!first) first = &k;
			if (seen++ == want) return &k;
		}
	return first;
}

static h3dg_status assemble_dm(h3dg_disc *disc, DmSpec &k, double *d_Ax, double *d_rhs, cudaStream_t st) {
	const h3dg::Plan &P = disc->plan;
	if (!k.configured) {
		H3DG_CUDA_TRY(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) k.smem));
		k.configured = true;
	}
	if (d_Ax && !disc->el_offd.p && P.ne > 0) {
		// built once per plan and validated against the column lengths
		size_t cnt = 0;
		unsigned long long stores = 0;
		H3DG_CUDA_TRY(build_offd(k, disc->el_offc.p, disc->el_cdof.p, disc->Ap.p, P.ne, P.color_ptr.data(), P.ncolors, P.nnz,
		                         &disc->el_offd.p, &cnt, &stores, disc->status.p, st));
		disc->el_offd.n = cnt;
		disc->offd_store_all = (int64_t) stores == P.nnz;
		int hs = 0;
		H3DG_CUDA_TRY(cudaMemcpyAsync(&hs, disc->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
		H3DG_CUDA_TRY(cudaStreamSynchronize(st));
		if (hs & h3dg::kErrBounds) {
			disc->el_offd.release();
			disc->offd_store_all = false;
			cudaMemsetAsync(disc->status.p, 0, sizeof(int), st);
			return fail(H3DG_ERR_STATE, "assemble: a scatter position falls outside its column (plan corrupt)");
		}
	}
	h3dg::KArgsHO a = {};
	a.xyz = disc->xyz.p;
	a.el_vtx = disc->el_vtx.p;
	a.el_id = disc->el_id.p;
	a.ecoef = disc->coef.p;
	a.cdof = disc->el_cdof.p;
	a.ccoef = disc->el_ccoef.p;
	a.offc = disc->el_offc.p;
	a.offd = disc->el_offd.p;
	a.Ap = disc->Ap.p;
	a.tables = disc->tables.p;
	a.table_bytes = disc->table_bytes;
	a.mass = disc->bf == H3DG_BF_GRAD_GRAD_MASS;
	a.lf = disc->lf;
	a.lf_value = disc->lf_value;
	a.Ax = d_Ax;
	a.rhs = disc->lf ? d_rhs : nullptr;
	a.status = disc->status.p;
	// first-touch stores cover every slot: no zero-fill of Ax
	if (d_Ax && !disc->offd_store_all) H3DG_CUDA_TRY(cudaMemsetAsync(d_Ax, 0, sizeof(double) * P.nnz, st));
	if (d_rhs) H3DG_CUDA_TRY(cudaMemsetAsync(d_rhs, 0, sizeof(double) * P.nrhs(), st));
	int nsm = 148, per_sm = 1;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.threads, k.smem);
	if (per_sm < 1) per_sm = 1;
	const bool rec = disc->tn < disc->tcap;
	if (rec) H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn], st));
	int32_t launches = 0;
	for (int c = 0; c < P.ncolors; c++) {
		int64_t kb = P.color_ptr[c], ke = P.color_ptr[c + 1];
		if (ke <= kb) continue;
		// a last round that would leave more than half the CTA slots idle runs as half elements
		const int64_t slots = (int64_t) nsm * per_sm, n = ke - kb, rem = n % slots;
		a.split_from = rem > 0 && 2 * rem <= slots ? ke - rem : ke;
		const int64_t items = (a.split_from - kb) + 2 * (ke - a.split_from);
		int64_t grid = std::min<int64_t>(items, (int64_t) nsm * per_sm);
		k.fn<<<(unsigned) grid, k.threads, k.smem, st>>>(a, kb, ke);
		launches++;
	}
	H3DG_CUDA_TRY(cudaGetLastError());
	if (rec) {
		H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn + 1], st));
		disc->tn++;
	}
	disc->last_launches = launches;
	disc->last_kind = H3DG_KERNEL_HO_FP64_DMMA;
	return H3DG_OK;
}

static h3dg_status assemble_ho(h3dg_disc *disc, int precision, double *d_Ax, double *d_rhs, cudaStream_t st) {
	const h3dg::Plan &P = disc->plan;
	if (DmSpec *dm = dm_select(disc, precision)) return assemble_dm(disc, *dm, d_Ax, d_rhs, st);
	HoSpec *kp = nullptr;
	int per_sm = 1;
	size_t scratch_need = 0;
	{
		h3dg_status s0 = ho_select(disc, precision, &kp, &per_sm, &scratch_need);
		if (s0 != H3DG_OK) return s0;
	}
	h3dg::KArgsHO a;
	a.xyz = disc->xyz.p;
	a.el_vtx = disc->el_vtx.p;
	a.el_id = disc->el_id.p;
	a.ecoef = disc->coef.p;
	a.cdof = disc->el_cdof.p;
	a.ccoef = disc->el_ccoef.p;
	a.tcdof = P.two_space ? disc->el_tcdof.p : nullptr;
	a.tccoef = P.two_space ? disc->el_tccoef.p : nullptr;
	a.offc = disc->el_offc.p;
	if ((precision == H3DG_PREC_TF32X3 || precision == H3DG_PREC_OZAKI) && d_Ax && !disc->el_offt.p && P.ne > 0) {
		// built once per plan; the build validates every position against its
		// column, so the split kernel posts without a per-entry bounds test
		size_t cnt = 0;
		unsigned long long stores = 0;
		H3DG_CUDA_TRY(build_offt(disc->el_offc.p, disc->el_cdof.p, disc->Ap.p, P.ne, P.px, P.nqx, P.color_ptr.data(),
		                         P.ncolors, P.nnz, &disc->el_offt.p, &cnt, &stores, disc->status.p, st));
		disc->el_offt.n = cnt;
		// every slot first-touched by a store: the split kernels need no zero-fill of Ax
		disc->offt_store_all = (int64_t) stores == P.nnz;
		int hs = 0;
		H3DG_CUDA_TRY(cudaMemcpyAsync(&hs, disc->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
		H3DG_CUDA_TRY(cudaStreamSynchronize(st));
		if (hs & h3dg::kErrBounds) {
			disc->el_offt.release();
			disc->offt_store_all = false;
			cudaMemsetAsync(disc->status.p, 0, sizeof(int), st);
			return fail(H3DG_ERR_STATE, "assemble: a scatter position falls outside its column (plan corrupt)");
		}
	}
	a.offt = disc->el_offt.p;
	a.offd = nullptr;
	a.split_from = 0;
	a.Ap = disc->Ap.p;
	a.tables = disc->tables.p;
	a.table_bytes = disc->table_bytes;
	a.mass = disc->bf == H3DG_BF_GRAD_GRAD_MASS;
	a.lf = disc->lf;
	a.lf_value = disc->lf_value;
	a.Ax = d_Ax;
	a.rhs = disc->lf ? d_rhs : nullptr;
	a.status = disc->status.p;
	// the 3xTF32 epilogue stores each slot's first contribution (no zero-fill needed)
	if (d_Ax && !(precision == H3DG_PREC_TF32X3 && disc->offt_store_all))
		H3DG_CUDA_TRY(cudaMemsetAsync(d_Ax, 0, sizeof(double) * P.nnz, st));
	if (d_rhs) H3DG_CUDA_TRY(cudaMemsetAsync(d_rhs, 0, sizeof(double) * P.nrhs(), st));
	int nsm = 148;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	HoSpec &k = *kp;
	a.gscratch = nullptr;
	if (precision == H3DG_PREC_OZAKI) {
		if (disc->ho_scratch.n < scratch_need) H3DG_CUDA_TRY(disc->ho_scratch.alloc(scratch_need));
		a.gscratch = disc->ho_scratch.p;
	}
	const bool rec = disc->tn < disc->tcap;
	if (rec) H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn], st));
	int32_t launches = 0;
	for (int c = 0; c < P.ncolors; c++) {
		int64_t kb = P.color_ptr[c], ke = P.color_ptr[c + 1];
		if (ke <= kb) continue;
		int64_t grid = std::min<int64_t>(ke - kb, (int64_t) nsm * per_sm);
		k.fn<<<(unsigned) grid, k.threads, k.smem, st>>>(a, kb, ke);
		launches++;
	}
	H3DG_CUDA_TRY(cudaGetLastError());
	if (rec) {
		H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn + 1], st));
		disc->tn++;
	}
	disc->last_launches = launches;
	disc->last_kind = precision == H3DG_PREC_TF32X3 ? H3DG_KERNEL_HO_TF32X3
	                  : precision == H3DG_PREC_OZAKI ? H3DG_KERNEL_HO_OZAKI : H3DG_KERNEL_HO_FP64_FMA;
	return H3DG_OK;
}

// set while h3dg_disc_assemble_host_noalloc runs: the mixed path then
// launches directly instead of instantiating a graph
static thread_local bool t_mixed_direct = false;

// Mixed orders: per colour, one launch per kernel class; the classes of a
// colour touch disjoint entries and run as parallel branches, colours are
// joined in order.  The whole assembly is captured once into a CUDA graph
// (per output pointers) and replayed.
static h3dg_status assemble_mixed(h3dg_disc *disc, double *d_Ax, double *d_rhs, cudaStream_t st) {
	const h3dg::Plan &P = disc->plan;
	constexpr int NC = h3dg::Plan::kClasses;
	h3dg::KArgsMixed a;
	a.xyz = disc->xyz.p;
	a.el_vtx = disc->el_vtx.p;
	a.el_id = disc->el_id.p;
	a.ecoef = disc->coef.p;
	a.el_desc = disc->el_desc.p;
	a.el_base = disc->el_base.p;
	a.el_obase = disc->el_obase.p;
	a.cdof = disc->el_cdof.p;
	a.ccoef = disc->el_ccoef.p;
	a.offm = disc->el_offm.p;
	a.Ap = disc->Ap.p;
	a.tables = disc->tables.p;
	a.table_bytes = disc->table_bytes;
	a.mass = disc->bf == H3DG_BF_GRAD_GRAD_MASS;
	a.lf = disc->lf;
	a.lf_value = disc->lf_value;
	a.Ax = d_Ax;
	a.rhs = disc->lf ? d_rhs : nullptr;
	a.status = disc->status.p;
	a.counters = disc->mx_counters.p;
	int nsm = 148;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	auto prepare = [&](MixSpec &k, int &per_sm) -> h3dg_status {
		const size_t smem = k.smem(disc->table_bytes);
		if (!k.configured || k.configured_smem < smem) {
			H3DG_CUDA_TRY(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
			k.configured = true;
			k.configured_smem = smem;
		}
		per_sm = 1;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.threads, smem);
		if (per_sm < 1) per_sm = 1;
		return H3DG_OK;
	};
	auto launch = [&](MixSpec &k, int per_sm, int c, int cls, cudaStream_t s) -> bool {
		const int li = c * NC + cls;
		const int64_t kb = P.launch_ptr[li], ke = P.launch_ptr[li + 1];
		if (ke <= kb) return false;
		const int64_t grid = std::min<int64_t>(ke - kb, (int64_t) nsm * per_sm);
		k.fn<<<(unsigned) grid, k.threads, k.smem(disc->table_bytes), s>>>(a, kb, ke, li);
		return true;
	};
	constexpr int NCE = h3dg::Plan::kCedClasses;
	const size_t ncnt = sizeof(unsigned) * (size_t) P.ncolors * (NC + NCE);
	// constrained elements: one kernel per class, scratch for every resident CTA
	h3dg::KArgsCed ca;
	int ce_per_sm[NCE] = { 1, 1, 1 };
	if (P.nce > 0) {
		ca.xyz = disc->xyz.p;
		ca.el_vtx = disc->ce_vtx.p;
		ca.el_id = disc->ce_id.p;
		ca.ecoef = disc->coef.p;
		ca.el_desc = disc->ce_desc.p;
		ca.ubase = disc->ce_ubase.p;
		ca.udof = disc->ce_udof.p;
		ca.wptr = disc->ce_wptr.p;
		ca.ws = disc->ce_ws.p;
		ca.ww = disc->ce_ww.p;
		ca.obase = disc->ce_obase.p;
		ca.off = disc->ce_off.p;
		ca.Ap = disc->Ap.p;
		ca.tables = disc->tables.p;
		ca.table_bytes = disc->table_bytes;
		ca.mass = a.mass;
		ca.lf = a.lf;
		ca.lf_value = a.lf_value;
		ca.Ax = d_Ax;
		ca.rhs = a.rhs;
		ca.status = disc->status.p;
		ca.counters = disc->mx_counters.p + (size_t) P.ncolors * NC;
		ca.scratch = disc->ce_scratch.p;
		ca.scratch_stride = disc->ce_stride;
		ca.order = disc->ce_order.p;
		ca.ebase = disc->ce_ebase.p;
		ca.out = disc->ce_out.p;
		for (int cls = 0; cls < NCE; cls++) ce_per_sm[cls] = disc->ce_per_sm[cls];
	}
	// constrained elements: every element's entries in one launch per class
	// (no colouring, it writes only its own output slice), then per colour a
	// scatter of those entries after all colours of the other elements
	auto launch_ced_compute = [&](int cls, cudaStream_t s) -> bool {
		const int64_t kb = P.ce_class_ptr[cls], ke = P.ce_class_ptr[cls + 1];
		if (ke <= kb) return false;
		CedSpec &k = ced_table()[cls];
		const int64_t grid = std::min<int64_t>(ke - kb, (int64_t) nsm * ce_per_sm[cls]);
		k.fn<<<(unsigned) grid, k.threads, k.smem(disc->table_bytes), s>>>(ca, kb, ke, cls);
		return true;
	};
	auto launch_ced_scatter = [&](int c, cudaStream_t s) -> bool {
		const int64_t kb = P.ce_color_ptr[c], ke = P.ce_color_ptr[c + 1];
		if (ke <= kb) return false;
		const int64_t grid = std::min<int64_t>(ke - kb, (int64_t) nsm * 8);
		ced_scatter_fn()<<<(unsigned) grid, kCedScatterThreads, 0, s>>>(ca, kb, ke);
		return true;
	};
	// variants: time each class's launches once per plan, keep the fastest
	if (disc->mx_variant[0] < 0) {
		cudaEvent_t e0, e1;
		H3DG_CUDA_TRY(cudaEventCreate(&e0));
		H3DG_CUDA_TRY(cudaEventCreate(&e1));
		for (int cls = 0; cls < NC; cls++) {
			float best = 1e30f;
			int besti = -1;
			for (size_t vi = 0; vi < mix_table().size(); vi++) {
				MixSpec &k = mix_table()[vi];
				if (k.cls != cls) continue;
				int per_sm;
				if (prepare(k, per_sm) != H3DG_OK) return H3DG_ERR_CUDA;
				if (besti < 0) besti = (int) vi;
				float tot = 0.0f;
				for (int rep = 0; rep < 2; rep++) {
					H3DG_CUDA_TRY(cudaMemsetAsync(disc->mx_counters.p, 0, ncnt, st));
					H3DG_CUDA_TRY(cudaEventRecord(e0, st));
					for (int c = 0; c < P.ncolors; c++) launch(k, per_sm, c, cls, st);
					H3DG_CUDA_TRY(cudaEventRecord(e1, st));
					H3DG_CUDA_TRY(cudaEventSynchronize(e1));
					float ms = 0.0f;
					H3DG_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
					if (rep) tot += ms;
				}
				if (tot < best) { best = tot; besti = (int) vi; }
			}
			disc->mx_variant[cls] = besti;
		}
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		H3DG_CUDA_TRY(cudaGetLastError());
	}
	int per_sm[NC];
	for (int cls = 0; cls < NC; cls++)
		if (prepare(mix_table()[disc->mx_variant[cls]], per_sm[cls]) != H3DG_OK) return H3DG_ERR_CUDA;
	// the whole assembly, on s0 with the classes 1, 2 of each colour forked to s1, s2
	auto enqueue = [&](cudaStream_t s0, cudaStream_t s1, cudaStream_t s2, bool fork) -> h3dg_status {
		int32_t n = 0;
		if (d_Ax) H3DG_CUDA_TRY(cudaMemsetAsync(d_Ax, 0, sizeof(double) * P.nnz, s0));
		if (d_rhs) H3DG_CUDA_TRY(cudaMemsetAsync(d_rhs, 0, sizeof(double) * P.ndof, s0));
		H3DG_CUDA_TRY(cudaMemsetAsync(disc->mx_counters.p, 0, ncnt, s0));
		cudaStream_t s3 = fork ? disc->mx_s[2] : s0;
		if (P.nce > 0) {
			if (fork) {
				H3DG_CUDA_TRY(cudaEventRecord(disc->mx_ev[3], s0));
				H3DG_CUDA_TRY(cudaStreamWaitEvent(s3, disc->mx_ev[3], 0));
			}
			for (int cls = 0; cls < NCE; cls++)
				if (launch_ced_compute(cls, s3)) n++;
			if (fork) H3DG_CUDA_TRY(cudaEventRecord(disc->mx_ev[4], s3));
		}
		for (int c = 0; c < P.ncolors; c++) {
			if (fork) {
				H3DG_CUDA_TRY(cudaEventRecord(disc->mx_ev[0], s0));
				H3DG_CUDA_TRY(cudaStreamWaitEvent(s1, disc->mx_ev[0], 0));
				H3DG_CUDA_TRY(cudaStreamWaitEvent(s2, disc->mx_ev[0], 0));
			}
			cudaStream_t ss[NC] = { s0, s1, s2 };
			for (int cls = 0; cls < NC; cls++)
				if (launch(mix_table()[disc->mx_variant[cls]], per_sm[cls], c, cls, ss[cls])) n++;

			if (fork) {
				H3DG_CUDA_TRY(cudaEventRecord(disc->mx_ev[1], s1));
				H3DG_CUDA_TRY(cudaEventRecord(disc->mx_ev[2], s2));
				H3DG_CUDA_TRY(cudaStreamWaitEvent(s0, disc->mx_ev[1], 0));
				H3DG_CUDA_TRY(cudaStreamWaitEvent(s0, disc->mx_ev[2], 0));
			}
		}
		if (P.nce > 0) {
			if (fork) H3DG_CUDA_TRY(cudaStreamWaitEvent(s0, disc->mx_ev[4], 0));
			for (int c = 0; c < P.ncolors; c++)
				if (launch_ced_scatter(c, s0)) n++;
		}
		H3DG_CUDA_TRY(cudaGetLastError());
		disc->mx_launches = n;
		return H3DG_OK;
	};
	const bool rec = disc->tn < disc->tcap;
	if (t_mixed_direct) {
		if (rec) H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn], st));
		h3dg_status s = enqueue(st, st, st, false);
		if (s != H3DG_OK) return s;
	}
	else {
		if (!disc->mx_exec || disc->mx_ax != d_Ax || disc->mx_rhs != d_rhs || disc->mx_coef != disc->coef.p) {
			if (disc->mx_exec) cudaGraphExecDestroy(disc->mx_exec);
			disc->mx_exec = nullptr;
			for (auto &s : disc->mx_s)
				if (!s) H3DG_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
			for (auto &e : disc->mx_ev)
				if (!e) H3DG_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
			cudaStream_t cap;
			H3DG_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
			cudaGraph_t g = nullptr;
			H3DG_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
			h3dg_status s = enqueue(cap, disc->mx_s[0], disc->mx_s[1], true);
			cudaError_t e = cudaStreamEndCapture(cap, &g);
			cudaStreamDestroy(cap);
			if (s != H3DG_OK) {
				if (g) cudaGraphDestroy(g);
				return s;
			}
			if (e != cudaSuccess) return fail(H3DG_ERR_CUDA, std::string("assemble: graph capture: ") + cudaGetErrorString(e));
			e = cudaGraphInstantiate(&disc->mx_exec, g, 0);
			cudaGraphDestroy(g);
			if (e != cudaSuccess) {
				disc->mx_exec = nullptr;
				return fail(H3DG_ERR_CUDA, std::string("assemble: graph instantiate: ") + cudaGetErrorString(e));
			}
			disc->mx_ax = d_Ax;
			disc->mx_rhs = d_rhs;
			disc->mx_coef = disc->coef.p;
		}
		if (rec) H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn], st));
		H3DG_CUDA_TRY(cudaGraphLaunch(disc->mx_exec, st));
	}
	if (rec) {
		H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn + 1], st));
		disc->tn++;
	}
	disc->last_launches = disc->mx_launches;
	return H3DG_OK;
}

static h3dg_status assemble_volume(h3dg_disc *disc, int precision, double *d_Ax, double *d_rhs, void *stream);

// surface forms, after the volume assembly on the same stream, face colours in order
static h3dg_status assemble_surface(h3dg_disc *disc, double *d_Ax, double *d_rhs, cudaStream_t st) {
	const h3dg::Plan &P = disc->plan;
	if (P.nsf == 0 || !d_Ax || !(disc->sbf || disc->slf)) return H3DG_OK;
	h3dg::KArgsSurf a;
	a.xyz = disc->xyz.p;
	a.desc = disc->sf_desc.p;
	a.vtx = disc->sf_vtx.p;
	a.base = disc->sf_base.p;
	a.obase = disc->sf_obase.p;
	a.dof = disc->sf_dof.p;
	a.coef = disc->sf_coef.p;
	a.ab = disc->sf_ab.p;
	a.off = disc->sf_off.p;
	a.Ap = disc->Ap.p;
	a.tables = disc->sf_tables.p;
	a.bf = disc->sbf;
	a.lf = disc->slf;
	for (int m = 0; m < h3dg::kSurfMarkers; m++) a.g[m] = disc->sg[m];
	a.Ax = d_Ax;
	a.rhs = d_rhs;
	a.status = disc->status.p;
	int nqmax = 0;
	for (int64_t k = 0; k < P.nsf; k++) nqmax = std::max(nqmax, P.sf_desc[k * h3dg::Plan::kSfDescInts + 4] * P.sf_desc[k * h3dg::Plan::kSfDescInts + 5]);
	const size_t smem = sizeof(double) * (size_t) nqmax * (P.sf_max_n + 1);
	SurfFn fn = surf_fn();
	if (smem > 48 * 1024) H3DG_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
	int nsm = 148;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	int32_t n = 0;
	for (size_t c = 0; c + 1 < P.sf_color_ptr.size(); c++) {
		const int64_t kb = P.sf_color_ptr[c], ke = P.sf_color_ptr[c + 1];
		if (ke <= kb) continue;
		const int64_t grid = std::min<int64_t>(ke - kb, (int64_t) nsm * 4);
		fn<<<(unsigned) grid, kSurfThreads, smem, st>>>(a, kb, ke);
		n++;
	}
	H3DG_CUDA_TRY(cudaGetLastError());
	disc->last_launches += n;
	return H3DG_OK;
}

h3dg_status h3dg_disc_solve_cg(h3dg_disc *disc, const double *d_Ax, const double *d_rhs, double *d_x, double rtol,
                               int maxit, int *iters, double *relres, void *stream) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "solve_cg: create_pattern() first");
	if (!d_Ax || !d_rhs || !d_x || !(rtol > 0.0) || maxit < 1) return fail(H3DG_ERR_INVALID_ARG, "solve_cg: bad arguments");
	if (disc->nparts > 1) return fail(H3DG_ERR_STATE, "solve_cg: the matrix of one part is not the whole operator");
	{ h3dg_status s0 = ensure_device(disc); if (s0 != H3DG_OK) return s0; }
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	cudaStream_t st = (cudaStream_t) stream;
	const int64_t n = disc->plan.ndof;
	const size_t need = 5 * (size_t) n + h3dg::kCgBlocks + 8;
	if (disc->cg_work.n < need) H3DG_CUDA_TRY(disc->cg_work.alloc(need));
	double *r = disc->cg_work.p, *z = r + n, *p = z + n, *q = p + n, *dinv = q + n;
	double *partial = dinv + n, *scal = partial + h3dg::kCgBlocks;
	const int64_t *Ap = disc->Ap.p;
	const int32_t *Ai = disc->Ai.p;
	const unsigned g = 148 * 8;
	auto dot = [&](const double *a, const double *b, double &out) -> h3dg_status {
		h3dg::k_cg_dot_partial<<<h3dg::kCgBlocks, h3dg::kCgThreads, 0, st>>>(a, b, n, partial);
		h3dg::k_cg_dot_final<<<1, h3dg::kCgThreads, 0, st>>>(partial, h3dg::kCgBlocks, scal);
		H3DG_CUDA_TRY(cudaMemcpyAsync(&out, scal, sizeof(double), cudaMemcpyDeviceToHost, st));
		H3DG_CUDA_TRY(cudaStreamSynchronize(st));
		return H3DG_OK;
	};
	h3dg::k_cg_invdiag<<<g, h3dg::kCgThreads, 0, st>>>(Ap, Ai, d_Ax, dinv, n);
	h3dg::k_cg_spmv<<<g, h3dg::kCgThreads, 0, st>>>(Ap, Ai, d_Ax, d_x, q, n);
	h3dg::k_cg_init<<<g, h3dg::kCgThreads, 0, st>>>(d_rhs, q, dinv, r, z, p, n);
	H3DG_CUDA_TRY(cudaGetLastError());
	double bb = 0.0, rz = 0.0, rr = 0.0;
	if (dot(d_rhs, d_rhs, bb) != H3DG_OK || dot(r, z, rz) != H3DG_OK || dot(r, r, rr) != H3DG_OK) return H3DG_ERR_CUDA;
	const double bnorm = std::sqrt(bb);
	int it = 0;
	while (it < maxit && std::sqrt(rr) > rtol * bnorm) {
		h3dg::k_cg_spmv<<<g, h3dg::kCgThreads, 0, st>>>(Ap, Ai, d_Ax, p, q, n);
		double pq = 0.0;
		if (dot(p, q, pq) != H3DG_OK) return H3DG_ERR_CUDA;
		if (!(pq > 0.0)) break;                           // not positive definite on this direction
		const double alpha = rz / pq;
		h3dg::k_cg_update_xr<<<g, h3dg::kCgThreads, 0, st>>>(d_x, r, z, p, q, dinv, alpha, n);
		double rz1 = 0.0;
		if (dot(r, z, rz1) != H3DG_OK || dot(r, r, rr) != H3DG_OK) return H3DG_ERR_CUDA;
		h3dg::k_cg_update_p<<<g, h3dg::kCgThreads, 0, st>>>(p, z, rz1 / rz, n);
		rz = rz1;
		it++;
	}
	H3DG_CUDA_TRY(cudaGetLastError());
	H3DG_CUDA_TRY(cudaStreamSynchronize(st));
	if (iters) *iters = it;
	if (relres) *relres = bnorm > 0.0 ? std::sqrt(rr) / bnorm : 0.0;
	return H3DG_OK;
}

h3dg_status h3dg_disc_norms(h3dg_disc *disc, const double *d_sol, int exact, double *out, void *stream) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "norms: create_pattern() first");
	if (!d_sol || !out || exact < H3DG_EXACT_ZERO || exact > H3DG_EXACT_SIN) return fail(H3DG_ERR_INVALID_ARG, "norms: bad arguments");
	{ h3dg_status s0 = ensure_device(disc); if (s0 != H3DG_OK) return s0; }
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	cudaStream_t st = (cudaStream_t) stream;
	if (!disc->have_eval) {
		h3dg::EvalPlan E;
		std::string err;
		if (h3dg::build_eval_plan(disc->space->s, disc->qmode == H3DG_QUAD_P_PLUS, disc->qn, E, err) != 0)
			return fail(H3DG_ERR_INVALID_ARG, "norms: " + err);
		H3DG_CUDA_TRY(disc->ev_desc.upload(E.desc));
		H3DG_CUDA_TRY(disc->ev_vtx.upload(E.vtx));
		H3DG_CUDA_TRY(disc->ev_edof.upload(E.edof));
		H3DG_CUDA_TRY(disc->ev_gptr.upload(E.gptr));
		H3DG_CUDA_TRY(disc->ev_eptr.upload(E.eptr));
		H3DG_CUDA_TRY(disc->ev_gs.upload(E.gs));
		H3DG_CUDA_TRY(disc->ev_ecoef.upload(E.ecoef));
		H3DG_CUDA_TRY(disc->ev_tables.upload(E.tables));
		H3DG_CUDA_TRY(disc->ev_partial.alloc((size_t) std::max<int64_t>(1, 4 * E.ne)));
		H3DG_CUDA_TRY(disc->ev_out.alloc(4));
		disc->ev_ne = E.ne;
		disc->ev_nlmax = E.nlmax;
		disc->ev_amax = E.amax;
		disc->ev_bmax = E.bmax;
		disc->have_eval = true;
	}
	h3dg::KArgsNorm a;
	a.xyz = disc->xyz.p;
	a.el_vtx = disc->ev_vtx.p;
	a.el_desc = disc->ev_desc.p;
	a.gptr = disc->ev_gptr.p;
	a.eptr = disc->ev_eptr.p;
	a.gs = disc->ev_gs.p;
	a.edof = disc->ev_edof.p;
	a.ecoef = disc->ev_ecoef.p;
	a.tables = disc->ev_tables.p;
	a.sol = d_sol;
	a.exact = exact;
	a.partial = disc->ev_partial.p;
	const size_t smem = sizeof(double) * ((size_t) disc->ev_nlmax + disc->ev_amax + disc->ev_bmax + 4 * kNormThreads);
	NormFn fn = norm_fn();
	if (smem > 48 * 1024) H3DG_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
	int nsm = 148;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	if (disc->ev_ne > 0) {
		const int64_t grid = std::min<int64_t>(disc->ev_ne, (int64_t) nsm * 4);
		fn<<<(unsigned) grid, kNormThreads, smem, st>>>(a, disc->ev_ne, disc->ev_nlmax, disc->ev_amax, disc->ev_bmax);
		norm_reduce_fn()<<<1, kNormThreads, 0, st>>>(disc->ev_partial.p, disc->ev_ne, disc->ev_out.p);
		H3DG_CUDA_TRY(cudaGetLastError());
	}
	double v[4] = { 0.0, 0.0, 0.0, 0.0 };
	if (disc->ev_ne > 0) {
		H3DG_CUDA_TRY(cudaMemcpyAsync(v, disc->ev_out.p, sizeof(v), cudaMemcpyDeviceToHost, st));
		H3DG_CUDA_TRY(cudaStreamSynchronize(st));
	}
	// calc_error / calc_norm: the square root only above 1e-14 (src/norm.cc:58,79)
	for (int j = 0; j < 4; j++) out[j] = v[j] > 10e-15 ? std::sqrt(v[j]) : v[j];
	return H3DG_OK;
}

h3dg_status h3dg_disc_assemble(h3dg_disc *disc, int precision, double *d_Ax, double *d_rhs, void *stream) {
	h3dg_status s = assemble_volume(disc, precision, d_Ax, d_rhs, stream);
	if (s != H3DG_OK) return s;
	s = assemble_surface(disc, d_Ax, d_rhs, (cudaStream_t) stream);
	// the plan's lazily made device state for this precision now exists
	// (h3dg_disc_assemble_host_noalloc requires it)
	if (s == H3DG_OK) disc->prepared |= 1u << precision;
	return s;
}

// Low-order uniform plans: the colour-sweep kernels for (p, rule) and, where
// the plan carries the segmented-scatter tables, the segmented kernels
// (numbered from kSegVariant).  H3DG_SCATTER=colour or =segmented keeps one
// family (tests compare the two bit for bit).
static constexpr int kSegVariant = 1000;

static std::vector<int> lo_candidates(const h3dg_disc *disc) {
	const h3dg::Plan &P = disc->plan;
	const char *only = std::getenv("H3DG_SCATTER");
	const bool colour = !only || std::strcmp(only, "segmented") != 0;
	const bool seg = P.seg && (!only || std::strcmp(only, "colour") != 0);
	std::vector<int> c;
	if (colour)
		for (size_t i = 0; i < kernel_table().size(); i++)
			if (kernel_table()[i].p == P.px && kernel_table()[i].nq == P.nqx) c.push_back((int) i);
	if (seg)
		for (size_t i = 0; i < seg_table().size(); i++)
			if (seg_table()[i].p == P.px && seg_table()[i].nq == P.nqx) c.push_back(kSegVariant + (int) i);
	return c;
}

static int seg_colcap(const h3dg::Plan &P) { return (std::min(P.seg_maxcol, 2048) + 1) & ~1; }

// Item schedule (ticket order) and ring of a segmented launch with as many
// CTAs as fit on the device.  The column items of ready window v follow the
// element items of window v + lag, lag ~ the elements one round of all CTAs
// takes, so their elements are done by the time they are taken; the ring
// holds span + lag + 2 windows, so an element item overwrites only slots
// whose column items precede it in ticket order (it waits for them).
static h3dg_status seg_prepare(h3dg_disc *disc, SegSpec &k, int nsm) {
	const h3dg::Plan &P = disc->plan;
	const int colcap = seg_colcap(P);
	const size_t smem = k.smem(colcap);
	if (!k.configured || k.configured_smem < smem) {
		H3DG_CUDA_TRY(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
		k.configured = true;
		k.configured_smem = smem;
	}
	int per_sm = 1;
	H3DG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.threads, smem));
	const int ctas = nsm * std::max(per_sm, 1);
	if (disc->seg_ctas == ctas && disc->seg_per_item == k.per_item && disc->seg_items.p && !std::getenv("H3DG_SEG_LAG") &&
	    !std::getenv("H3DG_SEG_RING"))
		return H3DG_OK;
	const int W = P.seg_window, nwin = P.seg_nwin;
	// H3DG_SEG_LAG: the lag in rounds of all CTAs (default 2)
	const double rounds = std::getenv("H3DG_SEG_LAG") ? std::atof(std::getenv("H3DG_SEG_LAG")) : 2.0;
	const int lag = (int) std::min<int64_t>(nwin, (int64_t) std::ceil(rounds * ctas * k.per_item / W) + 2);
	std::vector<int32_t> items, p1n(nwin, 0), p2n(nwin, 0);
	auto columns = [&](int v) {
		for (int64_t b = P.seg_p2ptr[v]; b < P.seg_p2ptr[v + 1]; b++) {
			items.insert(items.end(), &P.seg_p2[4 * b], &P.seg_p2[4 * b] + 4);
			p2n[v]++;
		}
	};
	for (int w = 0; w < nwin; w++) {
		const int64_t e1 = std::min<int64_t>((int64_t) (w + 1) * W, P.ne);
		for (int64_t e = (int64_t) w * W; e < e1; e += k.per_item) {
			items.insert(items.end(), { w, -1, (int32_t) e, (int32_t) std::min<int64_t>(e + k.per_item, e1) });
			p1n[w]++;
		}
		if (w - lag >= 0) columns(w - lag);
	}
	for (int v = std::max(0, nwin - lag); v < nwin; v++) columns(v);
	// ring: beyond span + lag, the windows the tickets in flight cover (about
	// two per CTA), so an element item rarely finds the column items that last
	// read its slots still running.  H3DG_SEG_RING: extra windows (profiling)
	const int per_win = (int) std::max<int64_t>(1, (int64_t) items.size() / 4 / nwin);
	const int front = (2 * ctas + per_win - 1) / per_win;
	const int extra = std::getenv("H3DG_SEG_RING") ? std::atoi(std::getenv("H3DG_SEG_RING")) : front + 2;
	const int ring_win = (int) std::min<int64_t>(nwin, (int64_t) P.seg_span + lag + std::max(2, extra));
	const int cw = (P.nl + 2) & ~1;
	const size_t ring = (size_t) ring_win * W * P.nl * cw;
	H3DG_CUDA_TRY(disc->seg_items.upload(items));
	H3DG_CUDA_TRY(disc->seg_p1n.upload(p1n));
	H3DG_CUDA_TRY(disc->seg_p2n.upload(p2n));
	if (disc->seg_ctr.n != (size_t) (2 + 2 * nwin + 4)) H3DG_CUDA_TRY(disc->seg_ctr.alloc(2 + 2 * nwin + 4));
	if (disc->seg_ring.n < ring) H3DG_CUDA_TRY(disc->seg_ring.alloc(ring));
	disc->seg_ctas = ctas;
	disc->seg_per_item = k.per_item;
	disc->seg_nitems = (int) (items.size() / 4);
	disc->seg_ring_win = ring_win;
	return H3DG_OK;
}

static h3dg_status seg_launch(h3dg_disc *disc, SegSpec &k, const h3dg::KArgs &a, double *d_Ax, double *d_rhs, cudaStream_t st) {
	const h3dg::Plan &P = disc->plan;
	if (!d_Ax && !(d_rhs && disc->lf)) {
		if (d_rhs) H3DG_CUDA_TRY(cudaMemsetAsync(d_rhs, 0, sizeof(double) * P.ndof, st));
		return H3DG_OK;
	}
	// DOFs without a column of this plan (another part's, or no linear form): zero
	if (d_rhs && (!disc->lf || !disc->seg_all_dofs)) H3DG_CUDA_TRY(cudaMemsetAsync(d_rhs, 0, sizeof(double) * P.ndof, st));
	H3DG_CUDA_TRY(cudaMemsetAsync(disc->seg_ctr.p, 0, sizeof(unsigned) * disc->seg_ctr.n, st));
	h3dg::SegArgs g;
	g.kof = disc->seg_kof.p;
	g.items = disc->seg_items.p;
	g.nitems = disc->seg_nitems;
	g.col = disc->seg_col.p;
	g.cptr = disc->seg_cptr.p;
	g.pe = disc->seg_pe.p;
	g.plm = disc->seg_plm.p;
	g.off = disc->seg_off.p;
	g.p1n = disc->seg_p1n.p;
	g.p2n = disc->seg_p2n.p;
	g.ctr = disc->seg_ctr.p;
	g.nwin = P.seg_nwin;
	g.ring_win = disc->seg_ring_win;
	g.span = P.seg_span;
	g.ring_slots = disc->seg_ring_win * P.seg_window;
	g.ring = disc->seg_ring.p;
	g.colcap = seg_colcap(P);
	k.fn<<<(unsigned) disc->seg_ctas, k.threads, k.smem(g.colcap), st>>>(a, g);
	H3DG_CUDA_TRY(cudaGetLastError());
	return H3DG_OK;
}

// KArgs of the low-order kernels for the current plan and outputs
static h3dg::KArgs lo_args(h3dg_disc *disc, double *d_Ax, double *d_rhs) {
	h3dg::KArgs a;
	a.xyz = disc->xyz.p;
	a.el_vtx = disc->el_vtx.p;
	a.el_cnt = disc->el_cnt.p;
	a.el_s = disc->el_s.p;
	a.el_dof = disc->el_dof.p;
	a.el_coef = disc->el_coef.p;
	a.el_off = disc->el_off.p;
	a.el_id = disc->el_id.p;
	a.ecoef = disc->coef.p;
	a.Ap = disc->Ap.p;
	a.tables = disc->tables.p;
	a.table_bytes = disc->table_bytes;
	a.mass = disc->bf == H3DG_BF_GRAD_GRAD_MASS;
	a.lf = disc->lf;
	a.lf_value = disc->lf_value;
	a.Ax = d_Ax;
	a.rhs = disc->lf ? d_rhs : nullptr;
	a.status = disc->status.p;
	a.wait_limit = h3dg::kWaitPolls;
	return a;
}

// One launch per colour of kernel k (split precision at low orders: one CTA
// per SM; otherwise as many as fit), outputs zeroed first.
static h3dg_status assemble_colours(h3dg_disc *disc, KernelSpec &k, double *d_Ax, double *d_rhs, cudaStream_t st,
                                    bool one_per_sm) {
	const h3dg::Plan &P = disc->plan;
	{
		h3dg_status s0 = ensure_device(disc);
		if (s0 != H3DG_OK) return s0;
	}
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	if (!k.configured) {
		H3DG_CUDA_TRY(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) k.smem));
		k.configured = true;
	}
	h3dg::KArgs a = lo_args(disc, d_Ax, d_rhs);
	if (disc->debug_once == H3DG_DEBUG_WAIT_GIVES_UP) a.wait_limit = 0;
	disc->debug_once = 0;
	int nsm = 148, per_sm = 1;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	if (!one_per_sm) {
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.threads, k.smem);
		per_sm = std::max(per_sm, 1);
	}
	const bool rec = disc->tn < disc->tcap;
	if (rec) H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn], st));
	if (d_Ax) H3DG_CUDA_TRY(cudaMemsetAsync(d_Ax, 0, sizeof(double) * P.nnz, st));
	if (d_rhs) H3DG_CUDA_TRY(cudaMemsetAsync(d_rhs, 0, sizeof(double) * P.ndof, st));
	int32_t n = 0;
	for (int c = 0; c < P.ncolors; c++) {
		const int64_t kb = P.color_ptr[c], ke = P.color_ptr[c + 1];
		if (ke <= kb) continue;
		const int64_t nb = (ke - kb + k.eb - 1) / k.eb;
		k.fn<<<(unsigned) std::min<int64_t>(nb, (int64_t) nsm * per_sm), k.threads, k.smem, st>>>(a, kb, ke);
		n++;
	}
	H3DG_CUDA_TRY(cudaGetLastError());
	if (rec) {
		H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn + 1], st));
		disc->tn++;
	}
	disc->last_launches = n;
	return H3DG_OK;
}

static h3dg_status assemble_volume(h3dg_disc *disc, int precision, double *d_Ax, double *d_rhs, void *stream) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "assemble: create_pattern() first");
	disc->last_kind = H3DG_KERNEL_OTHER;
	if (precision != H3DG_PREC_FP64 && precision != H3DG_PREC_TF32X3 && precision != H3DG_PREC_OZAKI)
		return fail(H3DG_ERR_INVALID_ARG, "assemble: unknown precision");
	const h3dg::Plan &P = disc->plan;
	if (P.mixed) {
		h3dg_status s0 = ensure_device(disc);
		if (s0 != H3DG_OK) return s0;
		H3DG_CUDA_TRY(cudaSetDevice(disc->device));
		return assemble_mixed(disc, d_Ax, d_rhs, (cudaStream_t) stream);
	}
	if (P.px != P.py || P.px != P.pz || P.nqx != P.nqy || P.nqx != P.nqz)
		return fail(H3DG_ERR_INVALID_ARG, "assemble: anisotropic orders need the batched path");
	if (P.canon) {
		h3dg_status s0 = ensure_device(disc);
		if (s0 != H3DG_OK) return s0;
		H3DG_CUDA_TRY(cudaSetDevice(disc->device));
		// a two-space block is assembled in FP64 (the split kernels take one space)
		return assemble_ho(disc, P.two_space ? H3DG_PREC_FP64 : precision, d_Ax, d_rhs, (cudaStream_t) stream);
	}
	// the reference's stock quadrature: FP64 per-pair rules
	if (disc->qmode == H3DG_QUAD_STOCK) {
		KernelSpec *ks = nullptr;
		for (auto &k : stock_table())
			if (k.p == P.px) ks = &k;
		if (!ks) return fail(H3DG_ERR_INVALID_ARG, "assemble: no stock-quadrature kernel for this order");
		return assemble_colours(disc, *ks, d_Ax, d_rhs, (cudaStream_t) stream, false);
	}
	// split precision at low orders: the batched tensor-core kernel, where one
	// is instantiated for (p, rule); otherwise FP64 (the split kernels of the
	// high-order path need create() with the precision hint)
	if (precision == H3DG_PREC_TF32X3) {
		KernelSpec *lt = nullptr;
		for (auto &k : lo_tc_table())
			if (k.p == P.px && k.nq == P.nqx) lt = &k;
		if (lt) return assemble_colours(disc, *lt, d_Ax, d_rhs, (cudaStream_t) stream, true);
	}
	// candidates: colour-sweep kernels (index into kernel_table) and, where
	// the plan has its tables, segmented-scatter kernels (kSegVariant + index
	// into seg_table); all give the same bits
	const std::vector<int> cands = lo_candidates(disc);
	if (cands.empty()) return fail(H3DG_ERR_INVALID_ARG, "assemble: no FP64 kernel instantiated for this order / rule");
	{
		h3dg_status s0 = ensure_device(disc);
		if (s0 != H3DG_OK) return s0;
	}
	if (!disc->xyz.p || !disc->el_vtx.p || !disc->el_off.p || !disc->Ap.p || !disc->tables.p || !disc->status.p || !disc->el_s.p)
		return fail(H3DG_ERR_STATE, "assemble: device plan missing");
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	cudaStream_t st = (cudaStream_t) stream;
	h3dg::KArgs a = lo_args(disc, d_Ax, d_rhs);
	int nsm = 148;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	// one assembly with candidate ci; returns launches, or -1 on a CUDA error
	auto run = [&](int ci) -> int32_t {
		if (ci >= kSegVariant) {
			SegSpec &k = seg_table()[ci - kSegVariant];
			if (seg_prepare(disc, k, nsm) != H3DG_OK) return -1;
			return seg_launch(disc, k, a, d_Ax, d_rhs, st) == H3DG_OK ? 1 : -1;
		}
		KernelSpec &k = kernel_table()[ci];
		if (d_Ax && cudaMemsetAsync(d_Ax, 0, sizeof(double) * P.nnz, st) != cudaSuccess) return -1;
		if (d_rhs && cudaMemsetAsync(d_rhs, 0, sizeof(double) * P.ndof, st) != cudaSuccess) return -1;
		if (!k.configured) {
			if (cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) k.smem) != cudaSuccess) return -1;
			k.configured = true;
		}
		int per_sm = 1;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.threads, k.smem);
		if (per_sm < 1) per_sm = 1;
		int32_t n = 0;
		for (int c = 0; c < P.ncolors; c++) {
			int64_t kb = P.color_ptr[c], ke = P.color_ptr[c + 1];
			if (ke <= kb) continue;
			int64_t nb = (ke - kb + k.eb - 1) / k.eb;
			int64_t grid = std::min<int64_t>(nb, (int64_t) nsm * per_sm);
			k.fn<<<(unsigned) grid, k.threads, k.smem, st>>>(a, kb, ke);
			n++;
		}
		return cudaGetLastError() == cudaSuccess ? n : -1;
	};
	// autotune once per plan: time one assembly with every candidate
	// H3DG_FP64_VARIANT=i pins candidate i (profiling runs) and skips the timing pass
	if (disc->variant < 0 && std::getenv("H3DG_FP64_VARIANT")) {
		int v = std::atoi(std::getenv("H3DG_FP64_VARIANT"));
		disc->variant = cands[(size_t) std::max(0, std::min(v, (int) cands.size() - 1))];
	}
	if (disc->variant < 0 && cands.size() > 1) {
		cudaEvent_t e0, e1;
		H3DG_CUDA_TRY(cudaEventCreate(&e0));
		H3DG_CUDA_TRY(cudaEventCreate(&e1));
		float best = 1e30f;
		int besti = cands[0];
		for (int ci : cands) {
			if (run(ci) < 0) continue;
			H3DG_CUDA_TRY(cudaEventRecord(e0, st));
			for (int r = 0; r < 2; r++) run(ci);
			H3DG_CUDA_TRY(cudaEventRecord(e1, st));
			H3DG_CUDA_TRY(cudaEventSynchronize(e1));
			float ms = 0;
			H3DG_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
			if (ms < best) { best = ms; besti = ci; }
		}
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		disc->variant = besti;
		disc->variant_ms = best / 2;
	}
	const int ci = disc->variant >= 0 ? disc->variant : cands[0];
	// test hook: the table-staging wait of this assembly gives up at once
	if (disc->debug_once == H3DG_DEBUG_WAIT_GIVES_UP) a.wait_limit = 0;
	disc->debug_once = 0;
	const bool rec = disc->tn < disc->tcap;
	if (rec) H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn], st));
	const int32_t launches = run(ci);
	if (launches < 0) {
		cudaError_t e = cudaGetLastError();
		return fail(H3DG_ERR_CUDA, std::string("assemble: launch failed: ") + cudaGetErrorString(e));
	}
	if (rec) {
		H3DG_CUDA_TRY(cudaEventRecord(disc->tev[2 * disc->tn + 1], st));
		disc->tn++;
	}
	disc->last_launches = launches;
	return H3DG_OK;
}

// Adjoint of a mixed-order plan (hanging nodes included): one runtime-order
// kernel over the ordinary and the constrained elements; sensitivities of
// element ids without an active element (refined parents) are zero.
static h3dg_status adjoint_mixed(h3dg_disc *disc, int nfields, const double *d_logcoef, const double *d_u,
                                 const double *d_lambda, double *d_S, double *d_grad, void *stream) {
	constexpr int PM = 8, QM = 10, NT = 256;
	const h3dg::Plan &P = disc->plan;
	auto fits = [&](const std::vector<int32_t> &desc, int64_t n) {
		for (int64_t k = 0; k < n; k++)
			for (int d = 0; d < 3; d++)
				if (desc[k * 12 + d] > PM || desc[k * 12 + 3 + d] > QM) return false;
		return true;
	};
	if (!fits(P.el_desc, P.ne) || !fits(P.ce_desc, P.nce))
		return fail(H3DG_ERR_INVALID_ARG, "adjoint: mixed-order plans up to order 8 and 10 points per direction");
	{
		h3dg_status s0 = ensure_device(disc);
		if (s0 != H3DG_OK) return s0;
	}
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	h3dg::AdjMixedArgs a = {};
	a.xyz = disc->xyz.p;
	a.el_vtx = disc->el_vtx.p;
	a.el_id = disc->el_id.p;
	a.el_desc = disc->el_desc.p;
	a.el_base = disc->el_base.p;
	a.cdof = disc->el_cdof.p;
	a.ccoef = disc->el_ccoef.p;
	a.ne = P.ne;
	if (P.nce > 0) {
		a.ce_vtx = disc->ce_vtx.p;
		a.ce_id = disc->ce_id.p;
		a.ce_desc = disc->ce_desc.p;
		a.ce_ubase = disc->ce_ubase.p;
		a.ce_wptr = disc->ce_wptr.p;
		a.ce_udof = disc->ce_udof.p;
		a.ce_ws = disc->ce_ws.p;
		a.ce_ww = disc->ce_ww.p;
	}
	a.nce = P.nce;
	a.tables = disc->tables.p;
	a.table_bytes = disc->table_bytes;
	a.nfields = nfields;
	a.lift = disc->lf != H3DG_LF_NONE;
	a.ne_ids = P.ne_ids;
	a.ndof = P.ndof;
	a.logcoef = d_logcoef;
	a.u = d_u;
	a.lam = d_lambda;
	a.S = d_S;
	a.grad = d_grad;
	a.status = disc->status.p;
	auto fn = &h3dg::k_adjoint_mixed<PM, QM, NT>;
	const size_t smem = h3dg::AdjMixedShape<PM, QM>::smem_bytes(disc->table_bytes);
	H3DG_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
	cudaStream_t st = (cudaStream_t) stream;
	const size_t bytes = sizeof(double) * (size_t) nfields * (size_t) P.ne_ids;
	if (d_S) H3DG_CUDA_TRY(cudaMemsetAsync(d_S, 0, bytes, st));
	if (d_grad) H3DG_CUDA_TRY(cudaMemsetAsync(d_grad, 0, bytes, st));
	int nsm = 148, per_sm = 1;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NT, smem);
	if (per_sm < 1) per_sm = 1;
	const int64_t items = P.ne + P.nce;
	if (items > 0) {
		fn<<<(unsigned) std::min<int64_t>(items, (int64_t) nsm * per_sm), NT, smem, st>>>(a);
		H3DG_CUDA_TRY(cudaGetLastError());
	}
	disc->last_launches = items > 0 ? 1 : 0;
	return H3DG_OK;
}

h3dg_status h3dg_disc_adjoint(h3dg_disc *disc, int nfields, const double *d_logcoef, const double *d_u,
                              const double *d_lambda, double *d_S, double *d_grad, void *stream) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "adjoint: create_pattern() first");
	if (nfields < 1 || !d_u || !d_lambda) return fail(H3DG_ERR_INVALID_ARG, "adjoint: bad arguments");
	const h3dg::Plan &P = disc->plan;
	if (P.mixed) return adjoint_mixed(disc, nfields, d_logcoef, d_u, d_lambda, d_S, d_grad, stream);
	if (P.px != P.py || P.px != P.pz || P.nqx != P.nqy || P.nqx != P.nqz)
		return fail(H3DG_ERR_INVALID_ARG, "adjoint: anisotropic orders need the batched path");
	AdjSpec *k = nullptr;
	for (auto &a : adj_table())
		if (a.p == P.px && a.nq == P.nqx) k = &a;
	if (!k) return fail(H3DG_ERR_INVALID_ARG, "adjoint: no kernel instantiated for this order / rule");
	{
		h3dg_status s0 = ensure_device(disc);
		if (s0 != H3DG_OK) return s0;
	}
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	h3dg::AdjArgs a;
	a.xyz = disc->xyz.p;
	a.el_vtx = disc->el_vtx.p;
	a.el_id = disc->el_id.p;
	a.el_cnt = disc->el_cnt.p;
	a.el_s = P.canon ? nullptr : disc->el_s.p;
	a.el_dof = P.canon ? nullptr : disc->el_dof.p;
	a.el_coef = P.canon ? nullptr : disc->el_coef.p;
	a.cdof = P.canon ? disc->el_cdof.p : nullptr;
	a.ccoef = P.canon ? disc->el_ccoef.p : nullptr;
	a.tables = disc->tables.p;
	a.table_bytes = disc->table_bytes;
	a.nfields = nfields;
	a.lift = disc->lf != H3DG_LF_NONE;
	a.ne = P.ne;
	a.ndof = P.ndof;
	a.logcoef = d_logcoef;
	a.u = d_u;
	a.lam = d_lambda;
	a.S = d_S;
	a.grad = d_grad;
	a.status = disc->status.p;
	if (!k->configured) {
		H3DG_CUDA_TRY(cudaFuncSetAttribute(k->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) k->smem));
		k->configured = true;
	}
	int nsm = 148, per_sm = 1;
	cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, disc->device);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k->fn, 128, k->smem);
	if (per_sm < 1) per_sm = 1;
	int64_t grid = std::min<int64_t>(P.ne, (int64_t) nsm * per_sm);
	k->fn<<<(unsigned) grid, 128, k->smem, (cudaStream_t) stream>>>(a);
	H3DG_CUDA_TRY(cudaGetLastError());
	disc->last_launches = 1;
	return H3DG_OK;
}

h3dg_status h3dg_tc_selftest(int kind, const float *d_A, const float *d_B, float *d_C, int device) {
	if (kind != 1 && kind != 2 && kind != 8) return fail(H3DG_ERR_INVALID_ARG, "tc_selftest: kind must be 1 (bf16), 2 (tf32) or 8 (int8)");
	H3DG_CUDA_TRY(cudaSetDevice(device));
	int *st = nullptr;
	H3DG_CUDA_TRY(cudaMalloc(&st, sizeof(int)));
	H3DG_CUDA_TRY(cudaMemset(st, 0, sizeof(int)));
	if (kind == 2) h3dg::k_tc_selftest<h3dg::tc::kTF32><<<1, 128>>>(d_A, d_B, d_C, st);
	else if (kind == 1) h3dg::k_tc_selftest<h3dg::tc::kBF16><<<1, 128>>>(d_A, d_B, d_C, st);
	else h3dg::k_tc_selftest<h3dg::tc::kI8><<<1, 128>>>(d_A, d_B, d_C, st);
	cudaError_t e = cudaDeviceSynchronize();
	int hs = 0;
	if (e == cudaSuccess) e = cudaMemcpy(&hs, st, sizeof(int), cudaMemcpyDeviceToHost);
	cudaFree(st);
	if (e != cudaSuccess) return fail(H3DG_ERR_CUDA, std::string("tc_selftest: ") + cudaGetErrorString(e));
	if (hs) return fail(H3DG_ERR_TIMEOUT, "tc_selftest: MMA completion wait gave up");
	return H3DG_OK;
}

h3dg_status h3dg_disc_get_tuning(const h3dg_disc *disc, int32_t *threads, int32_t *elems_per_cta, float *ms) {
	if (!disc) return fail(H3DG_ERR_INVALID_ARG, "get_tuning: null disc");
	int t = -1, eb = -1;
	if (disc->variant >= kSegVariant) {
		t = seg_table()[disc->variant - kSegVariant].threads;
		eb = seg_table()[disc->variant - kSegVariant].eb;
	}
	else if (disc->variant >= 0) {
		t = kernel_table()[disc->variant].threads;
		eb = kernel_table()[disc->variant].eb;
	}
	if (threads) *threads = t;
	if (elems_per_cta) *elems_per_cta = eb;
	if (ms) *ms = disc->variant_ms;
	return H3DG_OK;
}

h3dg_status h3dg_disc_seg_stats(const h3dg_disc *disc, int64_t *out) {
	if (!disc || !out) return fail(H3DG_ERR_INVALID_ARG, "seg_stats: bad arguments");
	for (int i = 0; i < 8; i++) out[i] = 0;
	if (!disc->seg_ctr.p) return H3DG_OK;
	unsigned w[4];
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	H3DG_CUDA_TRY(cudaMemcpy(w, disc->seg_ctr.p + disc->seg_ctr.n - 4, sizeof(w), cudaMemcpyDeviceToHost));
	for (int i = 0; i < 4; i++) out[i] = w[i];
	out[4] = disc->seg_nitems;
	out[5] = disc->seg_ring_win;
	out[6] = disc->seg_ctas;
	out[7] = disc->plan.seg_span;
	return H3DG_OK;
}

h3dg_status h3dg_disc_tuned_scatter(const h3dg_disc *disc, int32_t *segmented) {
	if (!disc || !segmented) return fail(H3DG_ERR_INVALID_ARG, "tuned_scatter: bad arguments");
	*segmented = disc->variant < 0 ? -1 : disc->variant >= kSegVariant ? 1 : 0;
	return H3DG_OK;
}

h3dg_status h3dg_disc_enable_kernel_timing(h3dg_disc *disc, int32_t n) {
	if (!disc || n < 0) return fail(H3DG_ERR_INVALID_ARG, "enable_kernel_timing: bad arguments");
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	for (auto e : disc->tev) cudaEventDestroy(e);
	disc->tev.assign(2 * (size_t) n, nullptr);
	for (auto &e : disc->tev) H3DG_CUDA_TRY(cudaEventCreate(&e));
	disc->tcap = n;
	disc->tn = 0;
	return H3DG_OK;
}

h3dg_status h3dg_disc_kernel_times(h3dg_disc *disc, float *ms, int32_t cap, int32_t *n) {
	if (!disc || !n) return fail(H3DG_ERR_INVALID_ARG, "kernel_times: bad arguments");
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	int k = 0;
	for (; k < disc->tn && k < cap; k++) {
		H3DG_CUDA_TRY(cudaEventSynchronize(disc->tev[2 * k + 1]));
		H3DG_CUDA_TRY(cudaEventElapsedTime(&ms[k], disc->tev[2 * k], disc->tev[2 * k + 1]));
	}
	*n = k;
	disc->tn = 0;
	return H3DG_OK;
}

h3dg_status h3dg_disc_assemble_host(h3dg_disc *disc, int precision, double *Ax, double *rhs) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "assemble_host: create_pattern() first");
	const h3dg::Plan &P = disc->plan;
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	if (Ax && disc->Ax.n != (size_t) P.nnz) H3DG_CUDA_TRY(disc->Ax.alloc(P.nnz));
	if (rhs && disc->rhs.n != (size_t) P.nrhs()) H3DG_CUDA_TRY(disc->rhs.alloc(P.nrhs()));
	h3dg_status s = h3dg_disc_assemble(disc, precision, Ax ? disc->Ax.p : nullptr, rhs ? disc->rhs.p : nullptr, nullptr);
	if (s != H3DG_OK) return s;
	if (Ax) H3DG_CUDA_TRY(cudaMemcpy(Ax, disc->Ax.p, sizeof(double) * P.nnz, cudaMemcpyDeviceToHost));
	if (rhs) H3DG_CUDA_TRY(cudaMemcpy(rhs, disc->rhs.p, sizeof(double) * P.nrhs(), cudaMemcpyDeviceToHost));
	int st = 0;
	H3DG_CUDA_TRY(cudaMemcpy(&st, disc->status.p, sizeof(int), cudaMemcpyDeviceToHost));
	if (st) {
		cudaMemset(disc->status.p, 0, sizeof(int));
		if (st & h3dg::kErrBounds) return fail(H3DG_ERR_STATE, "assemble_host: a scatter target fell outside its column (plan corrupt)");
		return fail(H3DG_ERR_TIMEOUT, "assemble_host: a device wait gave up");
	}
	return H3DG_OK;
}

} // extern "C"

// Staging array of h3dg_disc_assemble_host_noalloc (16 MiB on every device
// that loads the library, held until exit; no allocation at call time).
static __device__ __align__(256) double g_noalloc_scratch[H3DG_NOALLOC_SCRATCH_DOUBLES];

// Device address of the staging array on the current device.  The host-side
// name g_noalloc_scratch is only a stand-in: a kernel must be given this
// address.  It is looked up on every call -- once the module is loaded the
// lookup allocates nothing -- so an address never outlives a context that a
// cudaDeviceReset destroyed.
static h3dg_status noalloc_scratch(double **out) {
	double *p = nullptr;
	cudaError_t e = cudaGetSymbolAddress((void **) &p, g_noalloc_scratch);
	if (e != cudaSuccess || !p)
		return fail(H3DG_ERR_CUDA, std::string("assemble_host_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
	*out = p;
	return H3DG_OK;
}

extern "C" {

h3dg_status h3dg_disc_assemble_host_noalloc(h3dg_disc *disc, int precision, double *Ax, double *rhs) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "assemble_host_noalloc: create_pattern() first");
	if (precision != H3DG_PREC_FP64 && precision != H3DG_PREC_TF32X3 && precision != H3DG_PREC_OZAKI)
		return fail(H3DG_ERR_INVALID_ARG, "assemble_host_noalloc: unknown precision");
	const h3dg::Plan &P = disc->plan;
	const size_t rhs_off = ((size_t) P.nnz + 31) / 32 * 32;          // 256-byte boundary
	const size_t need = (rhs ? rhs_off + (size_t) P.nrhs() : (size_t) P.nnz);
	if (need > (size_t) H3DG_NOALLOC_SCRATCH_DOUBLES)
		return fail(H3DG_ERR_TOO_LARGE, "assemble_host_noalloc: nnz + ndof = " + std::to_string(need) +
		                                    " doubles exceed the fixed staging array of " +
		                                    std::to_string((size_t) H3DG_NOALLOC_SCRATCH_DOUBLES) +
		                                    " (16 MiB); use h3dg_disc_assemble_host");
	// everything h3dg_disc_assemble would allocate lazily must already exist:
	// an allocating assembly with this precision completed on this plan
	if (!disc->on_device || !disc->status.p || !(disc->prepared & (1u << precision)))
		return fail(H3DG_ERR_STATE, "assemble_host_noalloc: make one allocating assembly call with this precision on "
		                            "this plan first (h3dg_disc_assemble or h3dg_disc_assemble_host)");
	if (P.canon && (precision == H3DG_PREC_TF32X3 || precision == H3DG_PREC_OZAKI) && Ax && !disc->el_offt.p && P.ne > 0)
		return fail(H3DG_ERR_STATE, "assemble_host_noalloc: split-precision scatter stream not built; make one allocating "
		                            "split-precision assembly call with the matrix first");
	if (P.canon && Ax && P.ne > 0 && dm_select(disc, precision) && !disc->el_offd.p)
		return fail(H3DG_ERR_STATE, "assemble_host_noalloc: FP64 tensor-core scatter stream not built; make one allocating "
		                            "FP64 assembly call with the matrix first");
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	if (P.canon && precision == H3DG_PREC_OZAKI && P.ne > 0) {
		// the work area assemble_ho would (re)allocate: present and large enough
		HoSpec *k = nullptr;
		int per_sm = 1;
		size_t scratch_need = 0;
		h3dg_status s0 = ho_select(disc, precision, &k, &per_sm, &scratch_need);
		if (s0 != H3DG_OK) return s0;
		if (disc->ho_scratch.n < scratch_need)
			return fail(H3DG_ERR_STATE, "assemble_host_noalloc: split-precision work area smaller than this plan needs; "
			                            "make one allocating assembly call with this precision first");
	}
	if (P.mixed && disc->mx_variant[0] < 0)
		return fail(H3DG_ERR_STATE, "assemble_host_noalloc: kernel variants not tuned yet; make one allocating assembly "
		                            "call first");
	if (!P.mixed && !P.canon && disc->variant < 0) {
		if (lo_candidates(disc).size() > 1)
			return fail(H3DG_ERR_STATE, "assemble_host_noalloc: kernel variant not tuned yet; make one allocating assembly "
			                            "call first");
	}
	double *scratch = nullptr;
	h3dg_status s0 = noalloc_scratch(&scratch);
	if (s0 != H3DG_OK) return s0;
	double *d_Ax = Ax ? scratch : nullptr;
	double *d_rhs = rhs ? scratch + rhs_off : nullptr;
	t_mixed_direct = true;
	h3dg_status s = h3dg_disc_assemble(disc, precision, d_Ax, d_rhs, nullptr);   // zeroes its outputs first
	t_mixed_direct = false;
	if (s != H3DG_OK) return s;
	if (Ax) H3DG_CUDA_TRY(cudaMemcpy(Ax, d_Ax, sizeof(double) * P.nnz, cudaMemcpyDeviceToHost));
	if (rhs) H3DG_CUDA_TRY(cudaMemcpy(rhs, d_rhs, sizeof(double) * P.nrhs(), cudaMemcpyDeviceToHost));
	int st = 0;
	H3DG_CUDA_TRY(cudaMemcpy(&st, disc->status.p, sizeof(int), cudaMemcpyDeviceToHost));
	if (st) {
		cudaMemset(disc->status.p, 0, sizeof(int));
		if (st & h3dg::kErrBounds) return fail(H3DG_ERR_STATE, "assemble_host_noalloc: a scatter target fell outside its column (plan corrupt)");
		return fail(H3DG_ERR_TIMEOUT, "assemble_host_noalloc: a device wait gave up");
	}
	return H3DG_OK;
}

h3dg_status h3dg_disc_update_vertices(h3dg_disc *disc, const double *xyz, int64_t nv) {
	if (!disc || !disc->have_plan || !xyz || nv != disc->space->s.mesh->nv())
		return fail(H3DG_ERR_INVALID_ARG, "update_vertices: bad arguments or no plan");
	{ h3dg_status s0 = ensure_device(disc); if (s0 != H3DG_OK) return s0; }
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	H3DG_CUDA_TRY(cudaMemcpy(disc->xyz.p, xyz, sizeof(double) * 3 * nv, cudaMemcpyHostToDevice));
	return H3DG_OK;
}

h3dg_status h3dg_disc_update_coefficients(h3dg_disc *disc, const double *elem_coef, int64_t ne) {
	if (!disc || !disc->have_plan || !elem_coef || ne != disc->plan.ne_ids)
		return fail(H3DG_ERR_INVALID_ARG, "update_coefficients: bad arguments or no plan");
	{ h3dg_status s0 = ensure_device(disc); if (s0 != H3DG_OK) return s0; }
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	if (disc->coef.n != (size_t) ne) H3DG_CUDA_TRY(disc->coef.alloc(ne));
	H3DG_CUDA_TRY(cudaMemcpy(disc->coef.p, elem_coef, sizeof(double) * ne, cudaMemcpyHostToDevice));
	disc->ecoef.assign(elem_coef, elem_coef + ne);
	return H3DG_OK;
}

h3dg_status h3dg_disc_update_coefficients_device(h3dg_disc *disc, const double *d_elem_coef, int64_t ne, void *stream) {
	if (!disc || !disc->have_plan || !d_elem_coef || ne != disc->plan.ne_ids)
		return fail(H3DG_ERR_INVALID_ARG, "update_coefficients_device: bad arguments or no plan");
	{ h3dg_status s0 = ensure_device(disc); if (s0 != H3DG_OK) return s0; }
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	if (disc->coef.n != (size_t) ne) H3DG_CUDA_TRY(disc->coef.alloc(ne));
	H3DG_CUDA_TRY(cudaMemcpyAsync(disc->coef.p, d_elem_coef, sizeof(double) * ne, cudaMemcpyDeviceToDevice, (cudaStream_t) stream));
	return H3DG_OK;
}

h3dg_status h3dg_disc_debug_inject(h3dg_disc *disc, int what) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "debug_inject: create_pattern() first");
	const h3dg::Plan &P = disc->plan;
	if (what == H3DG_DEBUG_WAIT_GIVES_UP) {
		disc->debug_once = what;
		return H3DG_OK;
	}
	if (what != H3DG_DEBUG_CORRUPT_POSITION) return fail(H3DG_ERR_INVALID_ARG, "debug_inject: unknown hook");
	if (P.mixed || P.canon) return fail(H3DG_ERR_INVALID_ARG, "debug_inject: position hook needs a low-order plan");
	{ h3dg_status s0 = ensure_device(disc); if (s0 != H3DG_OK) return s0; }
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	// entry (a = 0, b = 0) of the first element with a matrix entry, in the
	// colour sweeps' map and in the segmented scatter's pair of that column
	for (int64_t k = 0; k < P.ne; k++)
		if (P.el_cnt[2 * k] > 0) {
			const uint16_t bad = 0xFFFF;
			H3DG_CUDA_TRY(cudaMemcpy(disc->el_off.p + (size_t) k * P.nl * P.nl, &bad, sizeof(bad), cudaMemcpyHostToDevice));
			if (P.seg) {
				const int32_t d = P.el_dof[(size_t) k * P.nl];
				int32_t e = -1;
				for (int64_t i = 0; i < P.ne && e < 0; i++)
					if (P.seg_kof[i] == k) e = (int32_t) i;
				for (size_t j = 0; j < P.seg_col.size(); j++)
					if (P.seg_col[j] == d)
						for (int64_t t = P.seg_cptr[j]; t < P.seg_cptr[j + 1]; t++)
							if (P.seg_pe[t] == e && (P.seg_plm[t] & 0xff) == 0)
								H3DG_CUDA_TRY(cudaMemcpy(disc->seg_off.p + (size_t) t * P.nl, &bad, sizeof(bad), cudaMemcpyHostToDevice));
			}
			return H3DG_OK;
		}
	return fail(H3DG_ERR_INVALID_ARG, "debug_inject: the plan has no matrix entry");
}

h3dg_status h3dg_disc_last_launch_count(const h3dg_disc *disc, int32_t *count) {
	if (!disc || !count) return fail(H3DG_ERR_INVALID_ARG, "last_launch_count: bad arguments");
	*count = disc->last_launches;
	return H3DG_OK;
}

h3dg_status h3dg_disc_last_kernel(const h3dg_disc *disc, int32_t *kind) {
	if (!disc || !kind) return fail(H3DG_ERR_INVALID_ARG, "last_kernel: bad arguments");
	*kind = disc->last_kind;
	return H3DG_OK;
}

h3dg_status h3dg_disc_geometry(h3dg_disc *disc, double *d_jac, double *d_irm, double *d_xyz, void *stream) {
	if (!disc || !disc->have_plan) return fail(H3DG_ERR_STATE, "geometry: create_pattern() first");
	const h3dg::Plan &P = disc->plan;
	if (P.mixed) return fail(H3DG_ERR_INVALID_ARG, "geometry: one rule per plan needed (mixed-order plan)");
	{ h3dg_status s0 = ensure_device(disc); if (s0 != H3DG_OK) return s0; }
	H3DG_CUDA_TRY(cudaSetDevice(disc->device));
	h3dg::GeomArgs g;
	g.xyz = disc->xyz.p;
	g.el_vtx = disc->el_vtx.p;
	g.el_id = disc->el_id.p;
	g.qx = disc->qx.p;
	g.qy = disc->qy.p;
	g.qz = disc->qz.p;
	g.nqx = P.nqx;
	g.nqy = P.nqy;
	g.nqz = P.nqz;
	g.ne = P.ne;
	g.jac = d_jac;
	g.irm = d_irm;
	g.xphys = d_xyz;
	const int nq = P.nqx * P.nqy * P.nqz;
	if (P.ne == 0 || nq == 0) return H3DG_OK;
	// whole elements per block, as the kernel takes them
	const int epb = nq >= h3dg::kGeomThreads ? 1 : std::min(h3dg::kGeomThreads / nq, h3dg::kGeomMaxElems);
	h3dg::k_geometry<<<(unsigned) ((P.ne + epb - 1) / epb), h3dg::kGeomThreads, 0, (cudaStream_t) stream>>>(g);
	H3DG_CUDA_TRY(cudaGetLastError());
	disc->last_launches = 1;
	return H3DG_OK;
}

} // extern "C"
