// Host-side mesh topology, H1 Lobatto DOF numbering, Dirichlet lifting,
// assembly lists and the CSC pattern / per-element tables.
#include "h3dg_host.h"
#include "lobatto.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <unordered_map>

namespace h3dg {

// RefHex (src/refdomain.cc:96-130)
const int kHexEdgeVtx[12][2] = { { 0, 1 }, { 1, 2 }, { 3, 2 }, { 0, 3 }, { 0, 4 }, { 1, 5 },
                                 { 2, 6 }, { 3, 7 }, { 4, 5 }, { 5, 6 }, { 7, 6 }, { 4, 7 } };
const int kHexFaceVtx[6][4] = { { 0, 3, 7, 4 }, { 1, 2, 6, 5 }, { 0, 1, 5, 4 },
                                { 3, 2, 6, 7 }, { 0, 1, 2, 3 }, { 4, 5, 6, 7 } };
const int kHexFaceEdges[6][4] = { { 3, 7, 11, 4 }, { 1, 6, 9, 5 }, { 0, 5, 8, 4 },
                                  { 2, 6, 10, 7 }, { 0, 1, 2, 3 }, { 8, 9, 10, 11 } };
// Lobatto vertex functions l_x(xi) l_y(eta) l_z(zeta) (h1lobattohex.cc:68-73)
const int kVertexXYZ[8][3] = { { 0, 0, 0 }, { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 },
                               { 0, 0, 1 }, { 1, 0, 1 }, { 1, 1, 1 }, { 0, 1, 1 } };
// reference-domain vertex coordinates (refdomain.cc:96-105)
static const double kRefVtx[8][3] = { { -1, -1, -1 }, { 1, -1, -1 }, { 1, 1, -1 }, { -1, 1, -1 },
                                      { -1, -1, 1 }, { 1, -1, 1 }, { 1, 1, 1 }, { -1, 1, 1 } };

// edge function tensor patterns: (x,y,z) with 'K' marking the running index
// (h1lobattohex.cc:320-353)
static const int kEdgePat[12][3] = { { -1, 0, 0 }, { 1, -1, 0 }, { -1, 1, 0 }, { 0, -1, 0 },
                                     { 0, 0, -1 }, { 1, 0, -1 }, { 1, 1, -1 }, { 0, 1, -1 },
                                     { -1, 0, 1 }, { 1, -1, 1 }, { -1, 1, 1 }, { 0, -1, 1 } };
// face function patterns (h1lobattohex.cc:355-403): fixed coordinate value and
// the two running directions (first = i (horizontal), second = j (vertical))
static const int kFaceFixedDir[6] = { 0, 0, 1, 1, 2, 2 };
static const int kFaceFixedVal[6] = { 0, 1, 0, 1, 0, 1 };
static const int kFaceDirs[6][2] = { { 1, 2 }, { 1, 2 }, { 0, 2 }, { 0, 2 }, { 0, 1 }, { 0, 1 } };
static const int kEdgeDir[12] = { 0, 1, 0, 1, 2, 2, 2, 2, 0, 1, 0, 1 };   // order.h get_edge_order

// ---------------------------------------------------------------- index decoding
// decompose() (h1lobattohex.cc:75-130) expressed as canonical tensor indices
// plus a sign: an orientation flip of direction d evaluates L_k(-x), which is
// (-1)^k L_k(x) for the k >= 2 functions it is applied to.
Canon decode_index(int64_t idx) {
	int type = (int) ((idx >> 19) & 3);
	int ori = (int) ((idx >> 12) & 7);
	int ind[3] = { (int) ((idx >> 8) & 15), (int) ((idx >> 4) & 15), (int) (idx & 15) };
	int flip[3] = { 0, 0, 0 };
	(void) type;
	int n01 = (ind[0] < 2) + (ind[1] < 2) + (ind[2] < 2);
	if (n01 == 2) {
		for (int d = 0; d < 3; d++)
			if (ind[d] >= 2) flip[d] = ori & 1;       // edge: the running direction
	}
	else if (n01 == 1) {
		int d1 = -1, d2 = -1;                         // the two face directions, ascending
		for (int d = 0; d < 3; d++)
			if (ind[d] >= 2) { if (d1 < 0) d1 = d; else d2 = d; }
		if (ori % 2 == 1) flip[d1] = 1;
		if (ori % 4 >= 2) flip[d2] = 1;
		if (ori >= 4) {
			std::swap(ind[d1], ind[d2]);
			std::swap(flip[d1], flip[d2]);
		}
	}
	int sign = 1;
	for (int d = 0; d < 3; d++)
		if (flip[d] && (ind[d] & 1)) sign = -sign;
	return Canon { ind[0], ind[1], ind[2], sign };
}

static double shape_value(int64_t idx, double x, double y, double z) {
	Canon c = decode_index(idx);
	return c.sign * lobatto_value(c.a, x) * lobatto_value(c.b, y) * lobatto_value(c.c, z);
}

// ---------------------------------------------------------------- mesh
namespace {
struct Key4Hash {
	size_t operator()(const std::array<int64_t, 4> &k) const {
		uint64_t h = 1469598103934665603ull;
		for (int i = 0; i < 4; i++) { h ^= (uint64_t) k[i] + 0x9e3779b97f4a7c15ull; h *= 1099511628211ull; h ^= h >> 29; }
		return (size_t) h;
	}
};
struct Key2Hash {
	size_t operator()(const std::pair<int64_t, int64_t> &k) const {
		uint64_t h = (uint64_t) k.first * 0x9e3779b97f4a7c15ull ^ ((uint64_t) k.second + 0x632be59bd9b4e019ull);
		h ^= h >> 31;
		return (size_t) (h * 0xbf58476d1ce4e5b9ull);
	}
};
}

// Mesh::add_hex / add_quad_boundary / ugh (src/mesh.cc:975-1102) and the
// loader's outer-face check (src/loader/mesh3d.cc:272-282).  Facet and edge
// ids are handed out in creation order, which is the order the reference's
// FOR_ALL_FACETS / FOR_ALL_EDGES loops visit them.
int Mesh::finalize(std::string &err) {
	int64_t n = ne(), nvert = nv();
	for (int64_t i = 0; i < 8 * n; i++)
		if (hex[i] < 0 || hex[i] >= nvert) { err = "Invalid vertex index was found in the section defining hexes."; return -1; }
	std::unordered_map<std::array<int64_t, 4>, int64_t, Key4Hash> fmap;
	std::unordered_map<std::pair<int64_t, int64_t>, int64_t, Key2Hash> emap;
	fmap.reserve(4 * n);
	emap.reserve(4 * n);
	elem_face.assign(6 * n, -1);
	elem_edge.assign(12 * n, -1);
	facet_left.clear(); facet_left_face.clear(); facet_right.clear();
	for (int64_t e = 0; e < n; e++) {
		const int64_t *v = &hex[8 * e];
		// Mesh::ref_edges: edges in local order
		for (int ie = 0; ie < 12; ie++) {
			int64_t a = v[kHexEdgeVtx[ie][0]], b = v[kHexEdgeVtx[ie][1]];
			std::pair<int64_t, int64_t> k(std::min(a, b), std::max(a, b));
			auto it = emap.find(k);
			if (it == emap.end()) it = emap.emplace(k, (int64_t) emap.size()).first;
			elem_edge[12 * e + ie] = it->second;
		}
		for (int f = 0; f < 6; f++) {
			std::array<int64_t, 4> k = { v[kHexFaceVtx[f][0]], v[kHexFaceVtx[f][1]], v[kHexFaceVtx[f][2]], v[kHexFaceVtx[f][3]] };
			std::sort(k.begin(), k.end());
			auto it = fmap.find(k);
			if (it == fmap.end()) {
				int64_t id = (int64_t) facet_left.size();
				fmap.emplace(k, id);
				facet_left.push_back(e);
				facet_left_face.push_back(f);
				facet_right.push_back(-1);
				elem_face[6 * e + f] = id;
			}
			else {
				if (facet_right[it->second] >= 0) { err = "A face is shared by more than two hexahedra."; return -1; }
				facet_right[it->second] = e;
				elem_face[6 * e + f] = it->second;
			}
		}
	}
	nfacets = (int64_t) facet_left.size();
	nedges = (int64_t) emap.size();
	facet_outer.assign(nfacets, 0);
	facet_marker.assign(nfacets, MARKER_UNDEFINED);
	for (size_t b = 0; b < bquad.size(); b++) {
		std::array<int64_t, 4> k = bquad[b];
		std::sort(k.begin(), k.end());
		auto it = fmap.find(k);
		if (it == fmap.end()) continue;   // add_quad_boundary returns NULL for an unknown face
		if (facet_right[it->second] >= 0) { err = "A boundary quad names an interior face."; return -1; }
		facet_outer[it->second] = 1;
		facet_marker[it->second] = bmarker[b];
	}
	for (int64_t f = 0; f < nfacets; f++)
		if (!facet_outer[f] && facet_right[f] < 0) { err = "Not all outer faces have defined boundary condition."; return -1; }
	edge_bnd.assign(nedges, 0);
	for (int64_t f = 0; f < nfacets; f++)
		if (facet_outer[f]) {
			int64_t e = facet_left[f];
			int lf = (int) facet_left_face[f];
			for (int k = 0; k < 4; k++) edge_bnd[elem_edge[12 * e + kHexFaceEdges[lf][k]]] = 1;
		}
	finalized = true;
	return 0;
}

// Hex::get_edge_orientation (src/mesh.cc:274-284)
int Mesh::edge_orientation(int64_t e, int iedge) const {
	const int64_t *v = &hex[8 * e];
	return v[kHexEdgeVtx[iedge][0]] < v[kHexEdgeVtx[iedge][1]] ? 0 : 1;
}

// Hex::get_face_orientation (src/mesh.cc:286-308), including its search for
// the minimum vertex id that starts from 1000: on faces whose four (1-based)
// vertex ids are all >= 1000, local vertex 0 is taken as the minimum.
int Mesh::face_orientation(int64_t e, int iface) const {
	const int64_t *vv = &hex[8 * e];
	uint64_t v[4];
	for (int i = 0; i < 4; i++) v[i] = (uint64_t) vv[kHexFaceVtx[iface][i]] + 1;
	uint64_t minval = 1000;
	int mn = 0;
	for (int i = 0; i < 4; i++)
		if (v[i] < minval) { minval = v[i]; mn = i; }
	if (mn == 0) return (v[1] < v[3]) ? 0 : 4;
	if (mn == 1) return (v[0] < v[2]) ? 1 : 6;
	if (mn == 2) return (v[3] < v[1]) ? 3 : 7;
	return (v[2] < v[0]) ? 2 : 5;
}

// ---------------------------------------------------------------- space

static int edge_order_of(const int *o, int iedge) { return o[kEdgeDir[iedge]]; }

static void face_order_of(const int *o, int iface, int &h, int &v) {
	h = o[kFaceDirs[iface][0]];
	v = o[kFaceDirs[iface][1]];
}

static void edge_indices(int iedge, int ori, int order, std::vector<int64_t> &out) {
	out.clear();
	for (int i = 2; i <= order; i++) {
		int t[3];
		for (int d = 0; d < 3; d++) t[d] = kEdgePat[iedge][d] < 0 ? i : kEdgePat[iedge][d];
		out.push_back(encode_index(SHFN_EDGE, iedge, t[0], t[1], t[2], ori));
	}
}

static void face_indices(int iface, int ori, int h, int v, std::vector<int64_t> &out) {
	out.clear();
	for (int i = 2; i <= h; i++)
		for (int j = 2; j <= v; j++) {
			int t[3];
			t[kFaceFixedDir[iface]] = kFaceFixedVal[iface];
			t[kFaceDirs[iface][0]] = i;
			t[kFaceDirs[iface][1]] = j;
			out.push_back(encode_index(SHFN_FACE, iface, t[0], t[1], t[2], ori));
		}
}

static void bubble_indices(const int *o, std::vector<int64_t> &out) {
	out.clear();
	for (int i = 2; i <= o[0]; i++)
		for (int j = 2; j <= o[1]; j++)
			for (int k = 2; k <= o[2]; k++) out.push_back(encode_index(SHFN_BUBBLE, 0, i, j, k, 0));
}

static inline int64_t vertex_index(int iv) {
	return encode_index(SHFN_VERTEX, 0, kVertexXYZ[iv][0], kVertexXYZ[iv][1], kVertexXYZ[iv][2], 0);
}

// trilinear reference map x(xi) (src/refmap.cc:265-316)
static void phys_point(const Mesh &m, int64_t e, double x, double y, double z, double out[3]) {
	out[0] = out[1] = out[2] = 0.0;
	for (int v = 0; v < 8; v++) {
		double N = lobatto_value(kVertexXYZ[v][0], x) * lobatto_value(kVertexXYZ[v][1], y) * lobatto_value(kVertexXYZ[v][2], z);
		const double *X = &m.xyz[3 * m.hex[8 * e + v]];
		for (int r = 0; r < 3; r++) out[r] += X[r] * N;
	}
}

// Cholesky solve of a symmetric positive-definite system (upper triangle given)
static void chol_solve(std::vector<double> &a, int n, std::vector<double> &b) {
	std::vector<double> p(n);
	for (int i = 0; i < n; i++)
		for (int j = i; j < n; j++) {
			double sum = a[i * n + j];
			for (int k = i - 1; k >= 0; k--) sum -= a[i * n + k] * a[j * n + k];
			if (i == j) p[i] = std::sqrt(sum);
			else a[j * n + i] = sum / p[i];
		}
	for (int i = 0; i < n; i++) {
		double sum = b[i];
		for (int k = i - 1; k >= 0; k--) sum -= a[i * n + k] * b[k];
		b[i] = sum / p[i];
	}
	for (int i = n - 1; i >= 0; i--) {
		double sum = b[i];
		for (int k = i + 1; k < n; k++) sum -= a[k * n + i] * b[k];
		b[i] = sum / p[i];
	}
}

// H1Space::calc_edge_boundary_projection (src/space/h1.cc:161-258): L2
// projection, in the reference coordinate of the edge, of g minus the linear
// vertex interpolant onto the edge functions.  The right-hand side uses the
// 13-point rule (the maximal edge order, 24); the mass matrix is computed
// exactly (same rule), as the reference's per-pair rule also is.
void Space::lift_edge(int64_t e, int iedge) {
	int64_t eid = mesh->elem_edge[12 * e + iedge];
	EData &en = ed[eid];
	if (en.bc != BC_ESSENTIAL || en.has_proj) return;
	int nf = en.n;
	if (nf <= 0) return;
	std::vector<int64_t> idx;
	edge_indices(iedge, mesh->edge_orientation(e, iedge), en.order, idx);
	std::vector<double> q, w;
	gauss_legendre(kMaxQuadPoints, q, w);
	int v0 = kHexEdgeVtx[iedge][0], v1 = kHexEdgeVtx[iedge][1];
	double c0 = vd[mesh->hex[8 * e + v0]].proj, c1 = vd[mesh->hex[8 * e + v1]].proj;
	std::vector<double> M(nf * nf, 0.0), rhs(nf, 0.0);
	for (int k = 0; k < kMaxQuadPoints; k++) {
		double t = (q[k] + 1.0) * 0.5, s = 1.0 - t;
		double pt[3];
		for (int d = 0; d < 3; d++) pt[d] = kRefVtx[v0][d] * s + kRefVtx[v1][d] * t;
		double X[3];
		phys_point(*mesh, e, pt[0], pt[1], pt[2], X);
		double g = bc_value_fn ? bc_value_fn(en.marker, X[0], X[1], X[2], bc_value_ctx) : 0.0;
		g -= c0 * shape_value(vertex_index(v0), pt[0], pt[1], pt[2]) + c1 * shape_value(vertex_index(v1), pt[0], pt[1], pt[2]);
		std::vector<double> phi(nf);
		for (int i = 0; i < nf; i++) phi[i] = shape_value(idx[i], pt[0], pt[1], pt[2]);
		for (int i = 0; i < nf; i++) {
			for (int j = i; j < nf; j++) M[i * nf + j] += w[k] * phi[i] * phi[j];
			rhs[i] += w[k] * phi[i] * g;
		}
	}
	chol_solve(M, nf, rhs);
	en.proj = rhs;
	en.has_proj = true;
}

// H1Space::calc_face_boundary_projection (src/space/h1.cc:260-394)
void Space::lift_face(int64_t e, int iface) {
	int64_t fid = mesh->elem_face[6 * e + iface];
	FData &fn = fd[fid];
	if (fn.bc != BC_ESSENTIAL || fn.has_proj) return;
	int nf = fn.n;
	if (nf <= 0) return;
	// vertex and edge functions of the face with their lifting coefficients
	std::vector<int64_t> bidx;
	std::vector<double> bcoef;
	for (int k = 0; k < 4; k++) {
		int lv = kHexFaceVtx[iface][k];
		bidx.push_back(vertex_index(lv));
		bcoef.push_back(vd[mesh->hex[8 * e + lv]].proj);
	}
	std::vector<int64_t> tmp;
	for (int k = 0; k < 4; k++) {
		int le = kHexFaceEdges[iface][k];
		const EData &en = ed[mesh->elem_edge[12 * e + le]];
		if (en.n > 0) {
			edge_indices(le, mesh->edge_orientation(e, le), en.order, tmp);
			for (int i = 0; i < en.n; i++) {
				bidx.push_back(tmp[i]);
				bcoef.push_back(en.has_proj ? en.proj[i] : 0.0);
			}
		}
	}
	std::vector<int64_t> idx;
	face_indices(iface, mesh->face_orientation(e, iface), fn.ox, fn.oy, idx);
	std::vector<double> q, w;
	gauss_legendre(kMaxQuadPoints, q, w);
	std::vector<double> M(nf * nf, 0.0), rhs(nf, 0.0), phi(nf);
	int fdir = kFaceFixedDir[iface], d1 = kFaceDirs[iface][0], d2 = kFaceDirs[iface][1];
	for (int k = 0; k < kMaxQuadPoints; k++)
		for (int l = 0; l < kMaxQuadPoints; l++) {
			double pt[3];
			pt[fdir] = kFaceFixedVal[iface] ? 1.0 : -1.0;
			pt[d1] = q[k];
			pt[d2] = q[l];
			double wt = w[k] * w[l];
			double X[3];
			phys_point(*mesh, e, pt[0], pt[1], pt[2], X);
			double g = bc_value_fn ? bc_value_fn(fn.marker, X[0], X[1], X[2], bc_value_ctx) : 0.0;
			for (size_t b = 0; b < bidx.size(); b++) g -= bcoef[b] * shape_value(bidx[b], pt[0], pt[1], pt[2]);
			for (int i = 0; i < nf; i++) phi[i] = shape_value(idx[i], pt[0], pt[1], pt[2]);
			for (int i = 0; i < nf; i++) {
				for (int j = i; j < nf; j++) M[i * nf + j] += wt * phi[i] * phi[j];
				rhs[i] += wt * phi[i] * g;
			}
		}
	chol_solve(M, nf, rhs);
	fn.proj = rhs;
	fn.has_proj = true;
}

static void set_bc_info(int &bc, int &marker, int newbc, int newmarker) {
	// Space::set_bc_info (src/space.cc:464-470)
	if (newbc == BC_ESSENTIAL || (newbc == BC_NATURAL && bc == BC_NONE)) {
		bc = newbc;
		marker = newmarker;
	}
}

// Space::assign_dofs (src/space.cc:1991-2028) for meshes without hanging
// nodes: enforce_minimum_rule, set_bc_information, H1Space::assign_dofs_internal
// and update_constraints (boundary projections).
int Space::assign_dofs(int first, int strd, std::string &err) {
	if (!mesh || !mesh->finalized) { err = "mesh not finalized"; return -1; }
	int64_t ne = mesh->ne();
	if ((int64_t) order.size() != 3 * ne) { err = "element orders not set"; return -1; }
	for (int64_t i = 0; i < 3 * ne; i++)
		if (order[i] < 1 || order[i] > kMaxOrder) { err = "element order out of range 1..10"; return -1; }
	first_dof = next_dof = first;
	stride = strd;
	vd.assign(mesh->nv(), VData());
	ed.assign(mesh->nedges, EData());
	fd.assign(mesh->nfacets, FData());
	bd.assign(ne, BData());

	// enforce_minimum_rule (src/space.cc:172-239)
	for (int64_t e = 0; e < ne; e++) {
		const int *o = &order[3 * e];
		for (int f = 0; f < 6; f++) {
			FData &fn = fd[mesh->elem_face[6 * e + f]];
			int h, v;
			face_order_of(o, f, h, v);
			if (mesh->face_orientation(e, f) >= 4) std::swap(h, v);
			if (fn.ox < 0) { fn.ox = h; fn.oy = v; }
			else { fn.ox = std::min(fn.ox, h); fn.oy = std::min(fn.oy, v); }
		}
		for (int ie = 0; ie < 12; ie++) {
			EData &en = ed[mesh->elem_edge[12 * e + ie]];
			int eo = edge_order_of(o, ie);
			if (en.order < 0 || eo < en.order) en.order = eo;
		}
	}

	// set_bc_information (src/space.cc:472-502)
	for (int64_t f = 0; f < mesh->nfacets; f++) {
		if (!mesh->facet_outer[f]) continue;
		int marker = mesh->facet_marker[f];
		int bc = bc_type_fn ? bc_type_fn(marker, bc_type_ctx) : BC_ESSENTIAL;
		fd[f].bc = bc;
		if (fd[f].marker == MARKER_UNDEFINED) fd[f].marker = marker;
		int64_t e = mesh->facet_left[f];
		int lf = (int) mesh->facet_left_face[f];
		for (int k = 0; k < 4; k++) {
			VData &v = vd[mesh->hex[8 * e + kHexFaceVtx[lf][k]]];
			set_bc_info(v.bc, v.marker, bc, marker);
		}
		for (int k = 0; k < 4; k++) {
			int64_t eid = mesh->elem_edge[12 * e + kHexFaceEdges[lf][k]];
			if (mesh->edge_bnd[eid]) set_bc_info(ed[eid].bc, ed[eid].marker, bc, marker);
		}
	}

	// H1Space::assign_dofs_internal (src/space/h1.cc:75-126)
	std::vector<char> seen(mesh->nv(), 0);
	for (int64_t e = 0; e < ne; e++)
		for (int iv = 0; iv < 8; iv++) {
			int64_t v = mesh->hex[8 * e + iv];
			if (seen[v]) continue;
			seen[v] = 1;
			if (vd[v].bc == BC_ESSENTIAL) vd[v].dof = DIRICHLET_DOF;
			else { vd[v].dof = next_dof; next_dof += stride; }
		}
	std::vector<char> eseen(mesh->nedges, 0);
	for (int64_t e = 0; e < ne; e++)
		for (int ie = 0; ie < 12; ie++) {
			int64_t id = mesh->elem_edge[12 * e + ie];
			if (eseen[id]) continue;
			eseen[id] = 1;
			EData &en = ed[id];
			int n = en.order - 1;
			if (en.bc == BC_ESSENTIAL) en.dof = DIRICHLET_DOF;
			else { en.dof = next_dof; next_dof += n * stride; }
			en.n = n;
		}
	std::vector<char> fseen(mesh->nfacets, 0);
	for (int64_t e = 0; e < ne; e++)
		for (int f = 0; f < 6; f++) {
			int64_t id = mesh->elem_face[6 * e + f];
			if (fseen[id]) continue;
			fseen[id] = 1;
			FData &fn = fd[id];
			int n = (fn.ox - 1) * (fn.oy - 1);
			if (fn.bc == BC_ESSENTIAL) fn.dof = DIRICHLET_DOF;
			else { fn.dof = next_dof; next_dof += n * stride; }
			fn.n = n;
		}
	for (int64_t e = 0; e < ne; e++) {
		const int *o = &order[3 * e];
		int n = (o[0] - 1) * (o[1] - 1) * (o[2] - 1);
		bd[e].n = n;
		bd[e].dof = next_dof;
		next_dof += n * stride;
	}

	// update_constraints (src/space.cc:2030-2066): vertex projections first,
	// then edge and face projections element by element (uc_element, :1943-1987)
	for (int64_t e = 0; e < ne; e++)
		for (int f = 0; f < 6; f++) {
			if (!mesh->facet_outer[mesh->elem_face[6 * e + f]]) continue;
			for (int k = 0; k < 4; k++) {
				int64_t vid = mesh->hex[8 * e + kHexFaceVtx[f][k]];
				VData &v = vd[vid];
				if (v.bc == BC_ESSENTIAL) {
					const double *X = &mesh->xyz[3 * vid];
					v.proj = bc_value_fn ? bc_value_fn(v.marker, X[0], X[1], X[2], bc_value_ctx) : 0.0;
				}
			}
		}
	for (int64_t e = 0; e < ne; e++) {
		for (int ie = 0; ie < 12; ie++) lift_edge(e, ie);
		for (int f = 0; f < 6; f++)
			if (mesh->facet_outer[mesh->elem_face[6 * e + f]]) lift_face(e, f);
	}
	assigned = true;
	return 0;
}

static inline void al_add(std::vector<AsmEntry> &al, int64_t idx, int dof, double coef) {
	if (coef == 0.0) return;                      // AsmList::add (src/asmlist.h:57-65)
	al.push_back(AsmEntry { idx, dof, coef });
}

// H1Space::get_element_assembly_list (src/space/h1.cc:130-137) with the
// vertex / edge / face / bubble lists of src/space.cc:296-450.
void Space::element_assembly_list(int64_t e, std::vector<AsmEntry> &al) const {
	al.clear();
	for (int iv = 0; iv < 8; iv++) {
		const VData &v = vd[mesh->hex[8 * e + iv]];
		al_add(al, vertex_index(iv), v.dof, v.dof >= 0 ? 1.0 : v.proj);
	}
	std::vector<int64_t> idx;
	for (int ie = 0; ie < 12; ie++) {
		const EData &en = ed[mesh->elem_edge[12 * e + ie]];
		if (en.n <= 0) continue;
		edge_indices(ie, mesh->edge_orientation(e, ie), en.order, idx);
		if (en.dof >= 0) {
			for (int j = 0; j < en.n; j++) al_add(al, idx[j], en.dof + j * stride, 1.0);
		}
		else if (en.has_proj) {
			for (int j = 0; j < en.n; j++) al_add(al, idx[j], DIRICHLET_DOF, en.proj[j]);
		}
	}
	for (int f = 0; f < 6; f++) {
		const FData &fn = fd[mesh->elem_face[6 * e + f]];
		if (fn.n <= 0) continue;
		face_indices(f, mesh->face_orientation(e, f), fn.ox, fn.oy, idx);
		if (fn.dof >= 0) {
			for (int j = 0; j < fn.n; j++) al_add(al, idx[j], fn.dof + j * stride, 1.0);
		}
		else if (fn.has_proj) {
			for (int j = 0; j < fn.n; j++) al_add(al, idx[j], DIRICHLET_DOF, fn.proj[j]);
		}
	}
	if (bd[e].n > 0) {
		bubble_indices(&order[3 * e], idx);
		for (int j = 0; j < bd[e].n; j++) al_add(al, idx[j], bd[e].dof + j * stride, 1.0);
	}
}

// ---------------------------------------------------------------- plan

template <class F>
static void parallel_for(int64_t n, F f) {
	unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
	if (n < 4096 || nt == 1) { f(0, n); return; }
	std::vector<std::thread> th;
	int64_t chunk = (n + nt - 1) / nt;
	for (unsigned t = 0; t < nt; t++) {
		int64_t lo = t * chunk, hi = std::min(n, lo + chunk);
		if (lo >= hi) break;
		th.emplace_back([=, &f]() { f(lo, hi); });
	}
	for (auto &t : th) t.join();
}

// z-slab partition (multi-GPU sharding, no communication on the data path).
// Slabs: the elements ordered by centroid (z, then y, then x, then index),
// cut into nparts contiguous ranges of equal count.  Owner of a DOF: the
// part of the lowest-numbered element whose assembly list holds it as a
// matrix entry.  Halo: elements outside the slab that hold an owned DOF.
int make_partition_scope(const Space &sp, int nparts, int part, PlanScope &S, std::string &err) {
	if (!sp.assigned) { err = "assign_dofs() has not been called"; return -1; }
	if (nparts < 1 || part < 0 || part >= nparts) { err = "partition: need 0 <= part < nparts"; return -1; }
	const Mesh &m = *sp.mesh;
	const int64_t ne = m.ne(), nd = sp.ndof();
	std::vector<std::array<double, 3>> cen(ne);
	for (int64_t e = 0; e < ne; e++) {
		double c[3] = { 0, 0, 0 };
		for (int v = 0; v < 8; v++)
			for (int r = 0; r < 3; r++) c[r] += m.xyz[3 * m.hex[8 * e + v] + r];
		cen[e] = { c[0] / 8, c[1] / 8, c[2] / 8 };
	}
	std::vector<int64_t> ord(ne);
	for (int64_t e = 0; e < ne; e++) ord[e] = e;
	std::sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) {
		if (cen[a][2] != cen[b][2]) return cen[a][2] < cen[b][2];
		if (cen[a][1] != cen[b][1]) return cen[a][1] < cen[b][1];
		if (cen[a][0] != cen[b][0]) return cen[a][0] < cen[b][0];
		return a < b;
	});
	std::vector<int> epart(ne);
	for (int64_t r = 0; r < ne; r++) epart[ord[r]] = (int) ((r * nparts) / std::max<int64_t>(ne, 1));
	std::vector<int64_t> first(nd, -1);
	std::vector<std::vector<int32_t>> edofs(ne);
	parallel_for(ne, [&](int64_t lo, int64_t hi) {
		std::vector<AsmEntry> al;
		for (int64_t e = lo; e < hi; e++) {
			sp.element_assembly_list(e, al);
			for (auto &a : al)
				if (a.dof >= 0) edofs[e].push_back(a.dof);
		}
	});
	for (int64_t e = 0; e < ne; e++)
		for (int32_t d : edofs[e])
			if (first[d] < 0) first[d] = e;
	S = PlanScope();
	S.owned.assign(nd, 0);
	for (int64_t d = 0; d < nd; d++)
		if (first[d] >= 0 && epart[first[d]] == part) {
			S.owned[d] = 1;
			S.nowned++;
		}
	for (int64_t e = 0; e < ne; e++) {
		bool take = epart[e] == part;
		if (take) S.nslab++;
		else {
			for (int32_t d : edofs[e])
				if (S.owned[d]) { take = true; break; }
			if (take) S.nhalo++;
		}
		if (take) S.elems.push_back(e);
	}
	return 0;
}

// Discretization::create (src/discretization.cc:164-230) + SparseMatrix
// pre_add_ij / sort_and_store_indices (src/matrix.cc:156-189) +
// UMFPackMatrix::alloc (src/linsolver/umfpack.cc:46-71): per column (trial
// DOF), the sorted, de-duplicated rows (test DOFs) of every element that
// holds both.  Built here column by column from the DOF -> element adjacency
// instead of page lists.  Also produces the per-element tables, the
// row-position map used by the scatter and an element colouring.

int build_plan(const Space &sp, int nqx, int nqy, int nqz, Plan &P, std::string &err, bool canon,
               const PlanScope *scope) {
	if (!sp.assigned) { err = "assign_dofs() has not been called"; return -1; }
	const Mesh &m = *sp.mesh;
	const int64_t ne = scope ? (int64_t) scope->elems.size() : m.ne();
	auto G = [&](int64_t e) -> int64_t { return scope ? scope->elems[e] : e; };   // plan element -> mesh element
	P = Plan();
	P.ne = ne;
	P.ndof = sp.ndof();
	P.px = sp.order[0]; P.py = sp.order[1]; P.pz = sp.order[2];
	for (int64_t e = 0; e < ne; e++)
		if (sp.order[3 * G(e)] != P.px || sp.order[3 * G(e) + 1] != P.py || sp.order[3 * G(e) + 2] != P.pz) {
			err = "plan requires one element order triple; bucket mixed orders first";
			return -1;
		}
	P.nl = (P.px + 1) * (P.py + 1) * (P.pz + 1);
	if (nqx < 1 || nqy < 1 || nqz < 1 || nqx > kMaxQuadPoints || nqy > kMaxQuadPoints || nqz > kMaxQuadPoints) {
		err = "Gauss points per direction must be in 1..13";
		return -1;
	}
	P.nqx = nqx; P.nqy = nqy; P.nqz = nqz;
	gauss_legendre(nqx, P.qx, P.wx);
	gauss_legendre(nqy, P.qy, P.wy);
	gauss_legendre(nqz, P.qz, P.wz);
	const int nl = P.nl;

	// element tables in element-id order first
	std::vector<int32_t> cnt(2 * ne), dofs((size_t) ne * nl, -1);
	std::vector<uint16_t> ss((size_t) ne * nl, 0);
	std::vector<double> cf((size_t) ne * nl, 0.0);
	std::string perr;
	std::vector<int> bad(ne, 0);
	parallel_for(ne, [&](int64_t lo, int64_t hi) {
		std::vector<AsmEntry> al;
		for (int64_t e = lo; e < hi; e++) {
			sp.element_assembly_list(G(e), al);
			int mcount = 0, lcount = 0;
			for (auto &a : al) (a.dof >= 0 ? mcount : lcount)++;
			if (mcount + lcount > nl) { bad[e] = 1; continue; }
			int im = 0, il = mcount;
			for (auto &a : al) {
				Canon c = decode_index(a.idx);
				int s = (c.a * (P.py + 1) + c.b) * (P.pz + 1) + c.c;
				int k = a.dof >= 0 ? im++ : il++;
				ss[(size_t) e * nl + k] = (uint16_t) s;
				dofs[(size_t) e * nl + k] = a.dof >= 0 ? a.dof : DIRICHLET_DOF;
				cf[(size_t) e * nl + k] = c.sign * a.coef;
			}
			// a DOF may appear once per element (no hanging-node constraints)
			for (int i = 0; i < mcount && !bad[e]; i++)
				for (int j = i + 1; j < mcount; j++)
					if (dofs[(size_t) e * nl + i] == dofs[(size_t) e * nl + j]) { bad[e] = 2; break; }
			cnt[2 * e] = mcount;
			cnt[2 * e + 1] = lcount;
		}
	});
	for (int64_t e = 0; e < ne; e++)
		if (bad[e]) { err = bad[e] == 1 ? "assembly list longer than the element basis" : "a DOF repeats in one assembly list (constrained space)"; return -1; }

	// DOF -> elements adjacency (CSR)
	int64_t nd = P.ndof;
	std::vector<int64_t> dptr(nd + 1, 0);
	for (int64_t e = 0; e < ne; e++)
		for (int k = 0; k < cnt[2 * e]; k++) dptr[dofs[(size_t) e * nl + k] + 1]++;
	for (int64_t d = 0; d < nd; d++) dptr[d + 1] += dptr[d];
	std::vector<int32_t> dadj(dptr[nd]);
	{
		std::vector<int64_t> fill(dptr.begin(), dptr.end() - 1);
		for (int64_t e = 0; e < ne; e++)
			for (int k = 0; k < cnt[2 * e]; k++) dadj[fill[dofs[(size_t) e * nl + k]]++] = (int32_t) e;
	}

	// column lengths, then columns
	std::vector<int64_t> collen(nd, 0);
	auto column = [&](int64_t d, std::vector<int32_t> &buf) {
		buf.clear();
		if (scope && !scope->owned[d]) return;                     // another part's column
		for (int64_t k = dptr[d]; k < dptr[d + 1]; k++) {
			int64_t e = dadj[k];
			for (int j = 0; j < cnt[2 * e]; j++) buf.push_back(dofs[(size_t) e * nl + j]);
		}
		std::sort(buf.begin(), buf.end());
		buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
	};
	parallel_for(nd, [&](int64_t lo, int64_t hi) {
		std::vector<int32_t> buf;
		for (int64_t d = lo; d < hi; d++) { column(d, buf); collen[d] = (int64_t) buf.size(); }
	});
	P.Ap.assign(nd + 1, 0);
	for (int64_t d = 0; d < nd; d++) P.Ap[d + 1] = P.Ap[d] + collen[d];
	P.nnz = P.Ap[nd];
	P.Ai.resize(P.nnz);
	int64_t maxcol = 0;
	for (int64_t d = 0; d < nd; d++) maxcol = std::max(maxcol, collen[d]);
	if (maxcol > 65535) { err = "a column holds more than 65535 rows"; return -1; }
	parallel_for(nd, [&](int64_t lo, int64_t hi) {
		std::vector<int32_t> buf;
		for (int64_t d = lo; d < hi; d++) {
			column(d, buf);
			std::copy(buf.begin(), buf.end(), P.Ai.begin() + P.Ap[d]);
		}
	});

	// greedy colouring in element order: colour = smallest not used by an
	// earlier element sharing a DOF
	std::vector<int> color(ne, -1);
	int ncol = 0;
	{
		std::vector<int64_t> stamp(64, -1);
		for (int64_t e = 0; e < ne; e++) {
			for (int k = 0; k < cnt[2 * e]; k++) {
				int d = dofs[(size_t) e * nl + k];
				for (int64_t t = dptr[d]; t < dptr[d + 1]; t++) {
					int64_t o = dadj[t];
					if (o < e && color[o] >= 0) {
						if (color[o] >= (int) stamp.size()) stamp.resize(color[o] + 1, -1);
						stamp[color[o]] = e;
					}
				}
			}
			int c = 0;
			while (c < (int) stamp.size() && stamp[c] == e) c++;
			color[e] = c;
			ncol = std::max(ncol, c + 1);
			if (c + 1 > (int) stamp.size()) stamp.resize(c + 1, -1);
		}
	}
	P.ncolors = ncol;
	std::vector<int64_t> order_(ne);
	{
		std::vector<int64_t> cc(ncol + 1, 0);
		for (int64_t e = 0; e < ne; e++) cc[color[e] + 1]++;
		for (int c = 0; c < ncol; c++) cc[c + 1] += cc[c];
		P.color_ptr = cc;
		std::vector<int64_t> fill(cc.begin(), cc.end() - 1);
		for (int64_t e = 0; e < ne; e++) order_[fill[color[e]]++] = e;
	}

	P.canon = canon;
	if (canon) {
		// canonical tables: every canonical index must occur at most once per element
		for (int64_t e = 0; e < ne; e++) {
			std::vector<char> seen(nl, 0);
			for (int k = 0; k < cnt[2 * e] + cnt[2 * e + 1]; k++) {
				int sidx = ss[(size_t) e * nl + k];
				if (seen[sidx]) { err = "a canonical function repeats in one assembly list"; return -1; }
				seen[sidx] = 1;
			}
		}
		P.el_vtx.resize(8 * ne);
		P.el_id.resize(ne);
		P.el_cdof.assign((size_t) ne * nl, -1);
		P.el_ccoef.assign((size_t) ne * nl, 0.0);
		P.el_offc.assign((size_t) ne * nl * nl, 0);
		P.el_cnt.resize(2 * ne);
		parallel_for(ne, [&](int64_t lo, int64_t hi) {
			for (int64_t k = lo; k < hi; k++) {
				int64_t e = order_[k];
				P.el_id[k] = (int32_t) G(e);
				for (int v = 0; v < 8; v++) P.el_vtx[8 * k + v] = (int32_t) m.hex[8 * G(e) + v];
				P.el_cnt[2 * k] = cnt[2 * e];
				P.el_cnt[2 * k + 1] = cnt[2 * e + 1];
				for (int t = 0; t < cnt[2 * e] + cnt[2 * e + 1]; t++) {
					int sidx = ss[(size_t) e * nl + t];
					P.el_cdof[(size_t) k * nl + sidx] = dofs[(size_t) e * nl + t];
					P.el_ccoef[(size_t) k * nl + sidx] = cf[(size_t) e * nl + t];
				}
				int mc = cnt[2 * e];
				for (int b = 0; b < mc; b++) {
					int col = dofs[(size_t) e * nl + b], sj = ss[(size_t) e * nl + b];
					const int32_t *c0 = &P.Ai[P.Ap[col]], *c1 = &P.Ai[P.Ap[col + 1]];
					for (int a = 0; a < mc; a++) {
						int row = dofs[(size_t) e * nl + a], si = ss[(size_t) e * nl + a];
						const int32_t *pos = std::lower_bound(c0, c1, row);
						P.el_offc[((size_t) k * nl + si) * nl + sj] = (uint16_t) (pos - c0);
					}
				}
			}
		});
		return 0;
	}

	// tables in assembly (colour-major) order
	P.el_vtx.resize(8 * ne);
	P.el_cnt.resize(2 * ne);
	P.el_s.resize((size_t) ne * nl);
	P.el_dof.resize((size_t) ne * nl);
	P.el_coef.resize((size_t) ne * nl);
	P.el_id.resize(ne);
	P.el_off.assign((size_t) ne * nl * nl, 0);
	parallel_for(ne, [&](int64_t lo, int64_t hi) {
		for (int64_t k = lo; k < hi; k++) {
			int64_t e = order_[k];
			P.el_id[k] = (int32_t) G(e);
			for (int v = 0; v < 8; v++) P.el_vtx[8 * k + v] = (int32_t) m.hex[8 * G(e) + v];
			P.el_cnt[2 * k] = cnt[2 * e];
			P.el_cnt[2 * k + 1] = cnt[2 * e + 1];
			std::copy(&ss[(size_t) e * nl], &ss[(size_t) e * nl] + nl, &P.el_s[(size_t) k * nl]);
			std::copy(&dofs[(size_t) e * nl], &dofs[(size_t) e * nl] + nl, &P.el_dof[(size_t) k * nl]);
			std::copy(&cf[(size_t) e * nl], &cf[(size_t) e * nl] + nl, &P.el_coef[(size_t) k * nl]);
			int mc = cnt[2 * e];
			for (int b = 0; b < mc; b++) {
				int col = dofs[(size_t) e * nl + b];
				const int32_t *c0 = &P.Ai[P.Ap[col]], *c1 = &P.Ai[P.Ap[col + 1]];
				for (int a = 0; a < mc; a++) {
					int row = dofs[(size_t) e * nl + a];
					const int32_t *pos = std::lower_bound(c0, c1, row);
					P.el_off[((size_t) k * nl + b) * nl + a] = (uint16_t) (pos - c0);
				}
			}
		}
	});
	return 0;
}

// Mixed orders.  Same pattern rule as build_plan (the CSC pattern does not
// depend on how the elements are grouped); the per-element tables are
// variable-length, indexed by prefix bases.
int build_plan_mixed(const Space &sp, bool p_plus, int qn, Plan &P, std::string &err, const PlanScope *scope) {
	if (!sp.assigned) { err = "assign_dofs() has not been called"; return -1; }
	const Mesh &m = *sp.mesh;
	const int64_t ne = scope ? (int64_t) scope->elems.size() : m.ne();
	auto G = [&](int64_t e) -> int64_t { return scope ? scope->elems[e] : e; };   // plan element -> mesh element
	P = Plan();
	P.ne = ne;
	P.ndof = sp.ndof();
	P.mixed = true;
	P.canon = true;
	P.px = P.py = P.pz = -1;
	P.nqx = P.nqy = P.nqz = -1;

	// orders, rules, table sets, kernel class
	std::vector<int64_t> eb(ne + 1, 0);
	std::vector<std::array<int, 11>> desc(ne);
	std::vector<std::pair<int, int>> set_key;
	std::vector<int> set_off;
	auto table_set = [&](int p, int nq) -> int {
		for (size_t t = 0; t < set_key.size(); t++)
			if (set_key[t].first == p && set_key[t].second == nq) return set_off[t];
		int off = (int) P.mixed_tables.size();
		std::vector<double> q, w;
		gauss_legendre(nq, q, w);
		for (int k = 0; k <= p; k++)
			for (int i = 0; i < nq; i++) P.mixed_tables.push_back(lobatto_value(k, q[i]));
		for (int k = 0; k <= p; k++)
			for (int i = 0; i < nq; i++) P.mixed_tables.push_back(lobatto_deriv(k, q[i]));
		P.mixed_tables.insert(P.mixed_tables.end(), q.begin(), q.end());
		P.mixed_tables.insert(P.mixed_tables.end(), w.begin(), w.end());
		if (P.mixed_tables.size() % 2) P.mixed_tables.push_back(0.0);
		set_key.push_back({ p, nq });
		set_off.push_back(off);
		return off;
	};
	for (int64_t e = 0; e < ne; e++) {
		auto &d = desc[e];
		int nl = 1, pmax = 0, qmax = 0;
		for (int r = 0; r < 3; r++) {
			const int p = sp.order[3 * G(e) + r];
			const int nq = p_plus ? p + qn : qn;
			if (p < 1 || p > 10) { err = "element order out of range"; return -1; }
			if (nq < 1 || nq > kMaxQuadPoints) { err = "Gauss points per direction must be in 1..13"; return -1; }
			d[r] = p;
			d[3 + r] = nq;
			d[6 + r] = table_set(p, nq);
			nl *= p + 1;
			pmax = std::max(pmax, p);
			qmax = std::max(qmax, nq);
		}
		d[9] = nl;
		int cls = -1;
		for (int c = 0; c < Plan::kClasses && cls < 0; c++)
			if (pmax <= Plan::kClassP[c] && qmax <= Plan::kClassQ[c]) cls = c;
		if (cls < 0) { err = "mixed-order kernels cover orders <= 6 and <= 8 points per direction"; return -1; }
		d[10] = cls;
		eb[e + 1] = eb[e] + nl;
		P.max_nl = std::max(P.max_nl, nl);
	}

	// assembly lists
	std::vector<int32_t> cnt(2 * ne), dofs(eb[ne], -1);
	std::vector<uint16_t> ss(eb[ne], 0);
	std::vector<double> cf(eb[ne], 0.0);
	std::vector<int> bad(ne, 0);
	parallel_for(ne, [&](int64_t lo, int64_t hi) {
		std::vector<AsmEntry> al;
		std::vector<char> seen;
		for (int64_t e = lo; e < hi; e++) {
			const int nl = desc[e][9], py = desc[e][1], pz = desc[e][2];
			sp.element_assembly_list(G(e), al);
			int mcount = 0, lcount = 0;
			for (auto &a : al) (a.dof >= 0 ? mcount : lcount)++;
			if (mcount + lcount > nl) { bad[e] = 1; continue; }
			int im = 0, il = mcount;
			seen.assign(nl, 0);
			for (auto &a : al) {
				Canon c = decode_index(a.idx);
				int sidx = (c.a * (py + 1) + c.b) * (pz + 1) + c.c;
				if (sidx < 0 || sidx >= nl || seen[sidx]) { bad[e] = 3; break; }
				seen[sidx] = 1;
				int k = a.dof >= 0 ? im++ : il++;
				ss[eb[e] + k] = (uint16_t) sidx;
				dofs[eb[e] + k] = a.dof >= 0 ? a.dof : DIRICHLET_DOF;
				cf[eb[e] + k] = c.sign * a.coef;
			}
			cnt[2 * e] = mcount;
			cnt[2 * e + 1] = lcount;
		}
	});
	for (int64_t e = 0; e < ne; e++)
		if (bad[e]) {
			err = bad[e] == 1 ? "assembly list longer than the element basis" : "a canonical function repeats in one assembly list (constrained space)";
			return -1;
		}

	// DOF -> elements adjacency, CSC pattern (as build_plan)
	const int64_t nd = P.ndof;
	std::vector<int64_t> dptr(nd + 1, 0);
	for (int64_t e = 0; e < ne; e++)
		for (int k = 0; k < cnt[2 * e]; k++) dptr[dofs[eb[e] + k] + 1]++;
	for (int64_t d = 0; d < nd; d++) dptr[d + 1] += dptr[d];
	std::vector<int32_t> dadj(dptr[nd]);
	{
		std::vector<int64_t> fill(dptr.begin(), dptr.end() - 1);
		for (int64_t e = 0; e < ne; e++)
			for (int k = 0; k < cnt[2 * e]; k++) dadj[fill[dofs[eb[e] + k]]++] = (int32_t) e;
	}
	std::vector<int64_t> collen(nd, 0);
	auto column = [&](int64_t d, std::vector<int32_t> &buf) {
		buf.clear();
		if (scope && !scope->owned[d]) return;                     // another part's column
		for (int64_t k = dptr[d]; k < dptr[d + 1]; k++) {
			int64_t e = dadj[k];
			for (int j = 0; j < cnt[2 * e]; j++) buf.push_back(dofs[eb[e] + j]);
		}
		std::sort(buf.begin(), buf.end());
		buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
	};
	parallel_for(nd, [&](int64_t lo, int64_t hi) {
		std::vector<int32_t> buf;
		for (int64_t d = lo; d < hi; d++) { column(d, buf); collen[d] = (int64_t) buf.size(); }
	});
	P.Ap.assign(nd + 1, 0);
	for (int64_t d = 0; d < nd; d++) P.Ap[d + 1] = P.Ap[d] + collen[d];
	P.nnz = P.Ap[nd];
	P.Ai.resize(P.nnz);
	int64_t maxcol = 0;
	for (int64_t d = 0; d < nd; d++) maxcol = std::max(maxcol, collen[d]);
	if (maxcol > 65535) { err = "a column holds more than 65535 rows"; return -1; }
	parallel_for(nd, [&](int64_t lo, int64_t hi) {
		std::vector<int32_t> buf;
		for (int64_t d = lo; d < hi; d++) {
			column(d, buf);
			std::copy(buf.begin(), buf.end(), P.Ai.begin() + P.Ap[d]);
		}
	});

	// greedy colouring in element order
	std::vector<int> color(ne, -1);
	int ncol = 0;
	{
		std::vector<int64_t> stamp(64, -1);
		for (int64_t e = 0; e < ne; e++) {
			for (int k = 0; k < cnt[2 * e]; k++) {
				int d = dofs[eb[e] + k];
				for (int64_t t = dptr[d]; t < dptr[d + 1]; t++) {
					int64_t o = dadj[t];
					if (o < e && color[o] >= 0) {
						if (color[o] >= (int) stamp.size()) stamp.resize(color[o] + 1, -1);
						stamp[color[o]] = e;
					}
				}
			}
			int c = 0;
			while (c < (int) stamp.size() && stamp[c] == e) c++;
			color[e] = c;
			ncol = std::max(ncol, c + 1);
			if (c + 1 > (int) stamp.size()) stamp.resize(c + 1, -1);
		}
	}
	P.ncolors = ncol;

	// order: colour, class, decreasing work (nl^2 * points), element id
	std::vector<int64_t> order_(ne);
	for (int64_t e = 0; e < ne; e++) order_[e] = e;
	auto work = [&](int64_t e) { return (int64_t) desc[e][9] * desc[e][9] * desc[e][3]; };
	std::sort(order_.begin(), order_.end(), [&](int64_t x, int64_t y) {
		if (color[x] != color[y]) return color[x] < color[y];
		if (desc[x][10] != desc[y][10]) return desc[x][10] < desc[y][10];
		int64_t wx = work(x), wy = work(y);
		if (wx != wy) return wx > wy;
		return x < y;
	});
	P.launch_ptr.assign((size_t) ncol * Plan::kClasses + 1, 0);
	for (int64_t e = 0; e < ne; e++) P.launch_ptr[(size_t) color[e] * Plan::kClasses + desc[e][10] + 1]++;
	for (size_t i = 0; i + 1 < P.launch_ptr.size(); i++) P.launch_ptr[i + 1] += P.launch_ptr[i];
	P.color_ptr.assign(ncol + 1, 0);
	for (int c = 0; c <= ncol; c++) P.color_ptr[c] = P.launch_ptr[(size_t) c * Plan::kClasses];

	// per-element tables in assembly order
	P.el_base.assign(ne + 1, 0);
	P.el_obase.assign(ne + 1, 0);
	for (int64_t k = 0; k < ne; k++) {
		const int nl = desc[order_[k]][9];
		P.el_base[k + 1] = P.el_base[k] + nl;
		P.el_obase[k + 1] = P.el_obase[k] + (int64_t) nl * nl;
	}
	P.el_vtx.resize(8 * ne);
	P.el_id.resize(ne);
	P.el_cnt.resize(2 * ne);
	P.el_desc.assign((size_t) ne * Plan::kDescInts, 0);
	P.el_cdof.assign(P.el_base[ne], -1);
	P.el_ccoef.assign(P.el_base[ne], 0.0);
	P.el_offm.assign(P.el_obase[ne], 0);
	parallel_for(ne, [&](int64_t lo, int64_t hi) {
		for (int64_t k = lo; k < hi; k++) {
			const int64_t e = order_[k];
			const int nl = desc[e][9];
			P.el_id[k] = (int32_t) G(e);
			for (int v = 0; v < 8; v++) P.el_vtx[8 * k + v] = (int32_t) m.hex[8 * G(e) + v];
			for (int t = 0; t < 11; t++) P.el_desc[(size_t) k * Plan::kDescInts + t] = desc[e][t];
			P.el_cnt[2 * k] = cnt[2 * e];
			P.el_cnt[2 * k + 1] = cnt[2 * e + 1];
			const int64_t cb = P.el_base[k], ob = P.el_obase[k];
			for (int t = 0; t < cnt[2 * e] + cnt[2 * e + 1]; t++) {
				const int sidx = ss[eb[e] + t];
				P.el_cdof[cb + sidx] = dofs[eb[e] + t];
				P.el_ccoef[cb + sidx] = cf[eb[e] + t];
			}
			const int mc = cnt[2 * e];
			for (int b = 0; b < mc; b++) {
				const int col = dofs[eb[e] + b], sj = ss[eb[e] + b];
				const int32_t *c0 = &P.Ai[P.Ap[col]], *c1 = &P.Ai[P.Ap[col + 1]];
				for (int a = 0; a < mc; a++) {
					const int row = dofs[eb[e] + a], si = ss[eb[e] + a];
					const int32_t *pos = std::lower_bound(c0, c1, row);
					P.el_offm[ob + (int64_t) sj * nl + si] = (uint16_t) (pos - c0);
				}
			}
		}
	});
	return 0;
}

} // namespace h3dg
