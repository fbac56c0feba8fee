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
// FOR_ALL_FACETS / FOR_ALL_EDGES loops visit them.  With refined elements
// the facets of all elements (active or not) are kept: a parent's face and
// the quarter faces of its children are distinct facets, as in the
// reference's facet tree (refine_quad_facet, src/mesh.cc:1843-2018).
int Mesh::finalize(std::string &err) {
	int64_t n = ne(), nvert = nv();
	for (int64_t i = 0; i < 8 * n; i++)
		if (hex[i] < 0 || hex[i] >= nvert) { err = "Invalid vertex index was found in the section defining hexes."; return -1; }
	const bool tree = nrefined > 0;
	std::unordered_map<std::array<int64_t, 4>, int64_t, Key4Hash> fmap;
	std::unordered_map<std::pair<int64_t, int64_t>, int64_t, Key2Hash> emap;
	fmap.reserve(4 * n);
	emap.reserve(4 * n);
	elem_face.assign(6 * n, -1);
	elem_edge.assign(12 * n, -1);
	facet_left.clear(); facet_left_face.clear(); facet_right.clear();
	edge_vtx.clear();
	for (int64_t e = 0; e < n; e++) {
		const int64_t *v = &hex[8 * e];
		// Mesh::ref_edges: edges in local order
		for (int ie = 0; ie < 12; ie++) {
			int64_t a = v[kHexEdgeVtx[ie][0]], b = v[kHexEdgeVtx[ie][1]];
			std::pair<int64_t, int64_t> k(std::min(a, b), std::max(a, b));
			auto it = emap.find(k);
			if (it == emap.end()) {
				it = emap.emplace(k, (int64_t) emap.size()).first;
				edge_vtx.push_back(k);
			}
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
	facet_ced.assign(nfacets, 0);
	for (size_t b = 0; b < bquad.size(); b++) {
		std::array<int64_t, 4> k = bquad[b];
		std::sort(k.begin(), k.end());
		auto it = fmap.find(k);
		if (it == fmap.end()) continue;   // add_quad_boundary returns NULL for an unknown face
		if (facet_right[it->second] >= 0) { err = "A boundary quad names an interior face."; return -1; }
		facet_outer[it->second] = 1;
		facet_marker[it->second] = bmarker[b];
	}
	if (tree) {
		// a child's face with no second element lies on its parent's face:
		// outer (with the parent's marker) if that face is, else it is a quarter
		// of a face whose other side is an active, unrefined element
		for (int64_t f = 0; f < nfacets; f++) {
			if (facet_right[f] >= 0 || facet_outer[f]) continue;
			const int64_t e = facet_left[f], P = parent[e];
			if (P < 0) continue;
			const int lf = (int) facet_left_face[f];
			int i = 0;
			while (i < 8 && sons[8 * P + i] != e) i++;
			bool on_parent_face = false;
			for (int k = 0; k < 4; k++) on_parent_face |= kHexFaceVtx[lf][k] == i;
			if (!on_parent_face) { err = "refinement: inner child face without a neighbour"; return -1; }
			const int64_t pf = elem_face[6 * P + lf];
			if (facet_outer[pf]) {
				facet_outer[f] = 1;
				facet_marker[f] = facet_marker[pf];
			}
			else facet_ced[f] = 1;
		}
	}
	for (int64_t f = 0; f < nfacets; f++)
		if (!facet_outer[f] && facet_right[f] < 0 && !facet_ced[f]) { err = "Not all outer faces have defined boundary condition."; return -1; }
	edge_bnd.assign(nedges, 0);
	for (int64_t f = 0; f < nfacets; f++)
		if (facet_outer[f]) {
			int64_t e = facet_left[f];
			int lf = (int) facet_left_face[f];
			for (int k = 0; k < 4; k++) edge_bnd[elem_edge[12 * e + kHexFaceEdges[lf][k]]] = 1;
		}
	// hanging nodes (Space::fc_element / fc_face, src/space.cc:598-736): every
	// face of an inactive element whose neighbour across it is active
	vertex_ced.assign(nvert, 0);
	edge_ced.assign(nedges, 0);
	interfaces.clear();
	if (tree) {
		for (int64_t P = 0; P < n; P++) {
			if (sons[8 * P] < 0) continue;
			for (int f = 0; f < 6; f++) {
				const int64_t pf = elem_face[6 * P + f];
				if (facet_outer[pf]) continue;
				const int64_t N = facet_left[pf] == P ? facet_right[pf] : facet_left[pf];
				if (N < 0 || !active(N)) continue;
				const int Nf = facet_left[pf] == N ? (int) facet_left_face[pf] : -1;
				int fN = Nf;
				if (fN < 0)
					for (int g = 0; g < 6; g++)
						if (elem_face[6 * N + g] == pf) fN = g;
				interfaces.push_back(Interface { P, f, N, fN });
				for (int k = 0; k < 4; k++) {
					const int i = kHexFaceVtx[f][k];
					const int64_t c = sons[8 * P + i];
					facet_ced[elem_face[6 * c + f]] = 1;
					for (int q = 0; q < 4; q++) {
						const int lv = kHexFaceVtx[f][q];
						if (lv != i) vertex_ced[hex[8 * c + lv]] = 1;
						edge_ced[elem_edge[12 * c + kHexFaceEdges[f][q]]] = 1;
					}
				}
			}
		}
	}
	finalized = true;
	return 0;
}

// Mesh::refine_element with REFT_HEX_XYZ (src/mesh.cc:1262-1323, refine_hex_8
// :1555-1633): the 12 edge midpoints, the 6 face midpoints (registered for
// both diagonals) and the centre are looked up or created in that order
// (get_midpoint / set_midpoint, :2064-2101, the vertex at (a + b) / 2), and the
// 8 children keep the parent's orientation.  Child i holds the parent's
// corner i; its vertex j is the point halfway between the parent's corners i
// and j in the reference domain (corner, edge midpoint, face midpoint or
// centre).  Only base elements are refined (one level).
int Mesh::refine_xyz(int64_t e, std::string &err, bool refinalize) {
	if (!finalized && nrefined == 0) { err = "refine: mesh not finalized"; return -1; }
	if (e < 0 || e >= ne()) { err = "refine: element id out of range"; return -1; }
	if (parent.empty()) {
		parent.assign(ne(), -1);
		sons.assign(8 * ne(), -1);
	}
	if (sons[8 * e] >= 0) { err = "refine: element is not active"; return -1; }
	if (parent[e] >= 0) { err = "refine: only base elements can be refined (one refinement level)"; return -1; }
	int64_t vtx[8];
	for (int k = 0; k < 8; k++) vtx[k] = hex[8 * e + k];
	auto key = [](int64_t a, int64_t b) { return std::make_pair(std::min(a, b), std::max(a, b)); };
	auto get_mid = [&](int64_t a, int64_t b) -> int64_t {
		auto it = midpoints.find(key(a, b));
		if (it != midpoints.end()) return it->second;
		const int64_t id = nv();
		for (int r = 0; r < 3; r++) xyz.push_back((xyz[3 * a + r] + xyz[3 * b + r]) / 2.0);
		midpoints[key(a, b)] = id;
		return id;
	};
	int64_t emp[12], fmp[6];
	for (int ie = 0; ie < 12; ie++) emp[ie] = get_mid(vtx[kHexEdgeVtx[ie][0]], vtx[kHexEdgeVtx[ie][1]]);
	for (int f = 0; f < 6; f++) {
		fmp[f] = get_mid(emp[kHexFaceEdges[f][0]], emp[kHexFaceEdges[f][2]]);
		midpoints[key(emp[kHexFaceEdges[f][1]], emp[kHexFaceEdges[f][3]])] = fmp[f];
	}
	const int64_t ctr = get_mid(fmp[0], fmp[1]);
	midpoints[key(fmp[2], fmp[3])] = ctr;
	midpoints[key(fmp[4], fmp[5])] = ctr;
	for (int i = 0; i < 8; i++) {
		const int64_t c = ne();
		for (int j = 0; j < 8; j++) {
			int diff = 0, same_dir = -1;
			for (int d = 0; d < 3; d++) {
				if (kRefVtx[i][d] != kRefVtx[j][d]) diff++;
				else same_dir = d;
			}
			int64_t v = vtx[i];
			if (diff == 1) {
				for (int ie = 0; ie < 12; ie++)
					if ((kHexEdgeVtx[ie][0] == i && kHexEdgeVtx[ie][1] == j) || (kHexEdgeVtx[ie][0] == j && kHexEdgeVtx[ie][1] == i)) v = emp[ie];
			}
			else if (diff == 2) v = fmp[2 * same_dir + (kRefVtx[i][same_dir] > 0 ? 1 : 0)];
			else if (diff == 3) v = ctr;
			hex.push_back(v);
		}
		parent.push_back(e);
		for (int k = 0; k < 8; k++) sons.push_back(-1);
		sons[8 * e + i] = c;
	}
	nrefined++;
	finalized = false;
	return refinalize ? finalize(err) : 0;
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

// Cholesky solve of a symmetric positive-definite system (upper triangle
// given): the decomposition and substitutions of Numerical Recipes (Press et
// al., 2nd ed., section 2.9, choldc / cholsl), the published algorithm the
// reference uses (src/matrix.cc:105-130), in the same loop order so that the
// projection coefficients agree to rounding.  Returns -1 on a pivot that is
// not positive (where the reference's choldc exits) and -2 on a non-finite
// solution (boundary values that are not finite).
static int chol_solve(std::vector<double> &a, int n, std::vector<double> &b) {
	std::vector<double> p(n);
	for (int i = 0; i < n; i++)
		for (int j = i; j < n; j++) {
			double sum = a[i * n + j];
			for (int k = i - 1; k >= 0; k--) sum -= a[i * n + k] * a[j * n + k];
			if (i == j) {
				if (!(sum > 0.0)) return -1;
				p[i] = std::sqrt(sum);
			}
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
	for (int i = 0; i < n; i++)
		if (!std::isfinite(b[i])) return -2;
	return 0;
}

// H1Space::calc_edge_boundary_projection (src/space/h1.cc:161-258): L2
// projection, in the reference coordinate of the edge, of g minus the linear
// vertex interpolant onto the edge functions.  The right-hand side uses the
// 13-point rule (the maximal edge order, 24); the mass matrix is computed
// exactly (same rule), as the reference's per-pair rule also is.
int Space::lift_edge(int64_t e, int iedge) {
	int64_t eid = mesh->elem_edge[12 * e + iedge];
	EData &en = ed[eid];
	if (en.bc != BC_ESSENTIAL || en.has_proj) return 0;
	int nf = en.n;
	if (nf <= 0) return 0;
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
	const int rc = chol_solve(M, nf, rhs);
	if (rc != 0) return rc;
	en.proj = rhs;
	en.has_proj = true;
	return 0;
}

// H1Space::calc_face_boundary_projection (src/space/h1.cc:260-394)
int Space::lift_face(int64_t e, int iface) {
	int64_t fid = mesh->elem_face[6 * e + iface];
	FData &fn = fd[fid];
	if (fn.bc != BC_ESSENTIAL || fn.has_proj) return 0;
	int nf = fn.n;
	if (nf <= 0) return 0;
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
		const int64_t eid = mesh->elem_edge[12 * e + le];
		const EData &en = ed[eid];
		if (en.ced) {
			// a constrained edge contributes the restriction of the constraining
			// edge's lifting (src/space/h1.cc:311-322)
			auto it = econs.find(eid);
			if (it == econs.end()) continue;
			const CedEdge &ce = it->second;
			const bool flip = mesh->hex[8 * e + kHexEdgeVtx[le][0]] > mesh->hex[8 * e + kHexEdgeVtx[le][1]];
			for (size_t j = 0; j < ce.dof.size(); j++) {
				if (ce.dof[j] >= 0) continue;
				for (int mm = 2; mm <= ce.order; mm++) {
					int t[3];
					for (int d = 0; d < 3; d++) t[d] = kEdgePat[le][d] < 0 ? mm : kEdgePat[le][d];
					bidx.push_back(encode_index(SHFN_EDGE, le, t[0], t[1], t[2], 0));
					bcoef.push_back(((flip && (mm & 1)) ? -1.0 : 1.0) * ce.c[j * (ce.order - 1) + mm - 2]);
				}
			}
			continue;
		}
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
	const int rc = chol_solve(M, nf, rhs);
	if (rc != 0) return rc;
	fn.proj = rhs;
	fn.has_proj = true;
	return 0;
}

static void set_bc_info(int &bc, int &marker, int newbc, int newmarker) {
	// Space::set_bc_info (src/space.cc:464-470)
	if (newbc == BC_ESSENTIAL || (newbc == BC_NATURAL && bc == BC_NONE)) {
		bc = newbc;
		marker = newmarker;
	}
}

// Space::assign_dofs (src/space.cc:1991-2028): find constraints (the mesh's
// hanging-node flags), enforce_minimum_rule, set_bc_information,
// H1Space::assign_dofs_internal and update_constraints (boundary projections,
// then the constraints of the hanging nodes).  Only active elements carry
// DOFs; constrained nodes get none.
int Space::assign_dofs(int first, int strd, std::string &err) {
	if (!mesh || !mesh->finalized) { err = "mesh not finalized"; return -1; }
	int64_t ne = mesh->ne();
	if ((int64_t) order.size() != 3 * ne) { err = "element orders not set"; return -1; }
	for (int64_t i = 0; i < 3 * ne; i++)
		if (mesh->active(i / 3) && (order[i] < 1 || order[i] > kMaxOrder)) { err = "element order out of range 1..10"; return -1; }
	first_dof = next_dof = first;
	stride = strd;
	vd.assign(mesh->nv(), VData());
	ed.assign(mesh->nedges, EData());
	fd.assign(mesh->nfacets, FData());
	bd.assign(ne, BData());
	vcons.clear();
	econs.clear();
	fcons.clear();
	if (mesh->nrefined) {
		for (int64_t v = 0; v < mesh->nv(); v++) vd[v].ced = mesh->vertex_ced[v];
		for (int64_t i = 0; i < mesh->nedges; i++) ed[i].ced = mesh->edge_ced[i];
		for (int64_t f = 0; f < mesh->nfacets; f++) fd[f].ced = mesh->facet_ced[f];
	}

	// enforce_minimum_rule (src/space.cc:172-239)
	for (int64_t e = 0; e < ne; e++) {
		if (!mesh->active(e)) continue;
		const int *o = &order[3 * e];
		for (int f = 0; f < 6; f++) {
			FData &fn = fd[mesh->elem_face[6 * e + f]];
			if (fn.ced) continue;
			int h, v;
			face_order_of(o, f, h, v);
			if (mesh->face_orientation(e, f) >= 4) std::swap(h, v);
			if (fn.ox < 0) { fn.ox = h; fn.oy = v; }
			else { fn.ox = std::min(fn.ox, h); fn.oy = std::min(fn.oy, v); }
		}
		for (int ie = 0; ie < 12; ie++) {
			EData &en = ed[mesh->elem_edge[12 * e + ie]];
			if (en.ced) continue;
			int eo = edge_order_of(o, ie);
			if (en.order < 0 || eo < en.order) en.order = eo;
		}
	}

	// set_bc_information (src/space.cc:472-502): every outer facet, those of
	// refined elements included
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
	for (int64_t e = 0; e < ne; e++) {
		if (!mesh->active(e)) continue;
		for (int iv = 0; iv < 8; iv++) {
			int64_t v = mesh->hex[8 * e + iv];
			if (seen[v] || vd[v].ced) continue;
			seen[v] = 1;
			if (vd[v].bc == BC_ESSENTIAL) vd[v].dof = DIRICHLET_DOF;
			else { vd[v].dof = next_dof; next_dof += stride; }
		}
	}
	std::vector<char> eseen(mesh->nedges, 0);
	for (int64_t e = 0; e < ne; e++) {
		if (!mesh->active(e)) continue;
		for (int ie = 0; ie < 12; ie++) {
			int64_t id = mesh->elem_edge[12 * e + ie];
			if (eseen[id] || ed[id].ced) continue;
			eseen[id] = 1;
			EData &en = ed[id];
			int n = en.order - 1;
			if (en.bc == BC_ESSENTIAL) en.dof = DIRICHLET_DOF;
			else { en.dof = next_dof; next_dof += n * stride; }
			en.n = n;
		}
	}
	std::vector<char> fseen(mesh->nfacets, 0);
	for (int64_t e = 0; e < ne; e++) {
		if (!mesh->active(e)) continue;
		for (int f = 0; f < 6; f++) {
			int64_t id = mesh->elem_face[6 * e + f];
			if (fseen[id] || fd[id].ced) continue;
			fseen[id] = 1;
			FData &fn = fd[id];
			int n = (fn.ox - 1) * (fn.oy - 1);
			if (fn.bc == BC_ESSENTIAL) fn.dof = DIRICHLET_DOF;
			else { fn.dof = next_dof; next_dof += n * stride; }
			fn.n = n;
		}
	}
	for (int64_t e = 0; e < ne; e++) {
		if (!mesh->active(e)) continue;
		const int *o = &order[3 * e];
		int n = (o[0] - 1) * (o[1] - 1) * (o[2] - 1);
		bd[e].n = n;
		bd[e].dof = next_dof;
		next_dof += n * stride;
	}

	// update_constraints (src/space.cc:2030-2066): vertex projections on the
	// outer faces of active elements, then edge and face projections element
	// by element over all elements (uc_element, :1943-1987)
	for (int64_t e = 0; e < ne; e++) {
		if (!mesh->active(e)) continue;
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
	}
	// element id order; the constraints of the hanging nodes (computed by
	// uc_element of the refined base element) come after every base element
	// and before the children, whose boundary projections use them
	// a projection that fails (pivot not positive, or boundary values that are
	// not finite) is an error, as choldc's EXIT is in the reference
	auto lift_element = [&](int64_t e) -> int {
		for (int ie = 0; ie < 12; ie++) {
			const int rc = lift_edge(e, ie);
			if (rc) {
				err = std::string("boundary projection of an edge of element ") + std::to_string(e + 1) +
				      (rc == -1 ? ": projection matrix not positive definite" : ": Dirichlet values not finite");
				return -1;
			}
		}
		if (!mesh->active(e)) return 0;
		for (int f = 0; f < 6; f++)
			if (mesh->facet_outer[mesh->elem_face[6 * e + f]]) {
				const int rc = lift_face(e, f);
				if (rc) {
					err = std::string("boundary projection of a face of element ") + std::to_string(e + 1) +
					      (rc == -1 ? ": projection matrix not positive definite" : ": Dirichlet values not finite");
					return -1;
				}
			}
		return 0;
	};
	for (int64_t e = 0; e < ne; e++)
		if ((!mesh->nrefined || mesh->parent[e] < 0) && lift_element(e) != 0) return -1;
	if (!mesh->interfaces.empty() && build_constraints(err) != 0) return -1;
	if (mesh->nrefined)
		for (int64_t e = 0; e < ne; e++)
			if (mesh->parent[e] >= 0 && lift_element(e) != 0) return -1;
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
	if (element_constrained(e)) { constrained_assembly_list(e, al); return; }
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

// ---------------------------------------------------------------- hanging nodes
//
// The reference expresses a constrained function as a combination of the
// element's own edge / face functions whose coefficients it finds by
// collocation at Chebyshev points (calc_constrained_*_combination,
// src/shapeset/h1lobattohex.cc:428-719) and attaches it to the DOFs of the
// constraining nodes through base lists (src/space.cc:739-1941).  That
// combination is the restriction of the constraining global function to the
// constrained node: a polynomial of the same degree, so the expansion in the
// node's Lobatto functions is exact and unique.  Here it is computed directly:
// a global function's trace on the big face is a product l_a(x1) l_b(x2) in
// the big element's face coordinates; restricted to a half interval each
// factor is expanded as f(u) = f(-1) l_0(u) + f(1) l_1(u) + sum_m R_m l_m(u),
// R_m = int f'(u) l_m'(u) du (the l_m', m >= 2, are orthonormal on [-1, 1]).
// Vertex coefficients are function values at the hanging vertex
// (calc_vertex_*_ced), edge coefficients the R_m of the varying factor times
// the value of the fixed one (calc_edge_edge_ced, calc_mid_edge_edge_ced,
// calc_edge_face_ced), face coefficients products of R_m (calc_face_face_ced).

// bubble coefficients R_2..R_k of u -> l_k(mid + half u)
static void restrict_bubbles(int k, double mid, double half, double *R) {
	std::vector<double> q, w;
	gauss_legendre(std::max(2, k), q, w);
	for (int m = 2; m <= k; m++) {
		double s = 0.0;
		for (size_t i = 0; i < q.size(); i++) s += w[i] * half * lobatto_deriv(k, mid + half * q[i]) * lobatto_deriv(m, q[i]);
		R[m - 2] = s;
	}
}

bool Space::element_constrained(int64_t e) const {
	if (!mesh->nrefined || !mesh->active(e)) return false;
	for (int iv = 0; iv < 8; iv++)
		if (vd[mesh->hex[8 * e + iv]].ced) return true;
	for (int ie = 0; ie < 12; ie++)
		if (ed[mesh->elem_edge[12 * e + ie]].ced) return true;
	for (int f = 0; f < 6; f++)
		if (fd[mesh->elem_face[6 * e + f]].ced) return true;
	return false;
}

// Space::update_constraints -> uc_element / uc_face (src/space.cc:1574-1987)
// for one refinement level: every constrained node lies on a quarter of an
// interface face (the face of an active element whose other side is
// refined); its constraint is computed once, from the first such face.
int Space::build_constraints(std::string &err) {
	const Mesh &m = *mesh;
	std::vector<AsmEntry> al;
	for (const Mesh::Interface &I : m.interfaces) {
		const int64_t N = I.big, P = I.small_parent;
		const int fN = I.big_face, dN = kFaceFixedDir[fN], vN = kFaceFixedVal[fN];
		const int d1N = kFaceDirs[fN][0], d2N = kFaceDirs[fN][1];
		// traces of the big element's global functions on the interface face
		struct Trace { int dof; double coef; int a1, a2; };
		std::vector<Trace> tr;
		element_assembly_list(N, al);
		for (const AsmEntry &x : al) {
			const Canon c = decode_index(x.idx);
			const int ind[3] = { c.a, c.b, c.c };
			if (ind[dN] != vN) continue;
			tr.push_back(Trace { x.dof, c.sign * x.coef, ind[d1N], ind[d2N] });
		}
		// positions of the 9 points of the refined face in the big face's coordinates
		std::unordered_map<int64_t, std::array<double, 2>> pos;
		int64_t corner[4];
		for (int k = 0; k < 4; k++) {
			const int lv = kHexFaceVtx[fN][k];
			corner[k] = m.hex[8 * N + lv];
			pos[corner[k]] = { kRefVtx[lv][d1N], kRefVtx[lv][d2N] };
		}
		auto mid = [&](int64_t a, int64_t b) -> int64_t {
			auto it = m.midpoints.find(std::make_pair(std::min(a, b), std::max(a, b)));
			return it == m.midpoints.end() ? -1 : it->second;
		};
		int64_t emp[4];
		for (int k = 0; k < 4; k++) {
			const int64_t a = corner[k], b = corner[(k + 1) % 4];
			emp[k] = mid(a, b);
			if (emp[k] < 0) { err = "constraints: missing edge midpoint"; return -1; }
			pos[emp[k]] = { 0.5 * (pos[a][0] + pos[b][0]), 0.5 * (pos[a][1] + pos[b][1]) };
		}
		const int64_t fmp = mid(emp[0], emp[2]);
		if (fmp < 0) { err = "constraints: missing face midpoint"; return -1; }
		pos[fmp] = { 0.0, 0.0 };
		auto value = [&](const Trace &t, double x1, double x2) { return t.coef * lobatto_value(t.a1, x1) * lobatto_value(t.a2, x2); };

		for (int k = 0; k < 4; k++) {
			const int i = kHexFaceVtx[I.face][k];
			const int64_t c = m.sons[8 * P + i];
			// hanging vertices: values of the global functions
			for (int q = 0; q < 4; q++) {
				const int64_t vid = m.hex[8 * c + kHexFaceVtx[I.face][q]];
				if (!vd[vid].ced || vcons.count(vid)) continue;
				auto it = pos.find(vid);
				if (it == pos.end()) { err = "constraints: vertex off the interface"; return -1; }
				CedVertex cv;
				for (const Trace &t : tr) {
					const double v = value(t, it->second[0], it->second[1]);
					if (v == 0.0) continue;
					cv.dof.push_back(t.dof);
					cv.val.push_back(v);
				}
				vcons[vid] = cv;
			}
			// constrained edges: bubble part of the restriction, parametrised
			// from the lower to the higher vertex id
			for (int q = 0; q < 4; q++) {
				const int64_t eid = m.elem_edge[12 * c + kHexFaceEdges[I.face][q]];
				if (!ed[eid].ced || econs.count(eid)) continue;
				const auto &A = pos.at(m.edge_vtx[eid].first), &B = pos.at(m.edge_vtx[eid].second);
				const int r = A[0] != B[0] ? 0 : 1;                  // varying face coordinate
				const double emid = 0.5 * (A[r] + B[r]), ehalf = 0.5 * (B[r] - A[r]), fixed = A[1 - r];
				CedEdge ce;
				for (const Trace &t : tr) ce.order = std::max(ce.order, r == 0 ? t.a1 : t.a2);
				const int nb = ce.order - 1;
				std::vector<double> R(std::max(nb, 1));
				for (const Trace &t : tr) {
					const int kv = r == 0 ? t.a1 : t.a2, kf = r == 0 ? t.a2 : t.a1;
					if (kv < 2) continue;
					const double fv = t.coef * lobatto_value(kf, fixed);
					if (fv == 0.0) continue;
					restrict_bubbles(kv, emid, ehalf, R.data());
					ce.dof.push_back(t.dof);
					for (int mm = 2; mm <= ce.order; mm++) ce.c.push_back(mm <= kv ? fv * R[mm - 2] : 0.0);
				}
				econs[eid] = ce;
			}
			// the quarter face: products of bubble parts; axes from the lowest
			// vertex id (h towards its lower-id neighbour, v towards the other)
			const int64_t qf = m.elem_face[6 * c + I.face];
			if (fd[qf].ced && !fcons.count(qf)) {
				int64_t qv[4];
				for (int q = 0; q < 4; q++) qv[q] = m.hex[8 * c + kHexFaceVtx[I.face][q]];
				int o = 0;
				for (int q = 1; q < 4; q++)
					if (qv[q] < qv[o]) o = q;
				int64_t vh = qv[(o + 1) % 4], vv = qv[(o + 3) % 4];
				if (vv < vh) std::swap(vh, vv);
				const auto &O = pos.at(qv[o]), &H = pos.at(vh), &V = pos.at(vv);
				const int rh = O[0] != H[0] ? 0 : 1;                 // face coordinate along h
				const double hmid = 0.5 * (O[rh] + H[rh]), hhalf = 0.5 * (H[rh] - O[rh]);
				const double vmid = 0.5 * (O[1 - rh] + V[1 - rh]), vhalf = 0.5 * (V[1 - rh] - O[1 - rh]);
				CedFace cf;
				for (const Trace &t : tr) {
					cf.oh = std::max(cf.oh, rh == 0 ? t.a1 : t.a2);
					cf.ov = std::max(cf.ov, rh == 0 ? t.a2 : t.a1);
				}
				std::vector<double> Rh(std::max(cf.oh - 1, 1)), Rv(std::max(cf.ov - 1, 1));
				for (const Trace &t : tr) {
					const int kh = rh == 0 ? t.a1 : t.a2, kv = rh == 0 ? t.a2 : t.a1;
					if (kh < 2 || kv < 2) continue;
					restrict_bubbles(kh, hmid, hhalf, Rh.data());
					restrict_bubbles(kv, vmid, vhalf, Rv.data());
					cf.dof.push_back(t.dof);
					for (int a = 2; a <= cf.oh; a++)
						for (int b = 2; b <= cf.ov; b++) cf.c.push_back(a <= kh && b <= kv ? t.coef * Rh[a - 2] * Rv[b - 2] : 0.0);
				}
				fcons[qf] = cf;
			}
		}
	}
	return 0;
}

// assembly list of an element with constrained nodes (expanded form): the
// unconstrained nodes as in element_assembly_list, each constrained node's
// functions tied to the global functions of its constraint
void Space::constrained_assembly_list(int64_t e, std::vector<AsmEntry> &al) const {
	const Mesh &m = *mesh;
	al.clear();
	auto canon = [](int type, int ef, const int t[3]) { return encode_index(type, ef, t[0], t[1], t[2], 0); };
	for (int iv = 0; iv < 8; iv++) {
		const int64_t vid = m.hex[8 * e + iv];
		const VData &v = vd[vid];
		if (!v.ced) { al_add(al, vertex_index(iv), v.dof, v.dof >= 0 ? 1.0 : v.proj); continue; }
		const CedVertex &cv = vcons.at(vid);
		for (size_t k = 0; k < cv.dof.size(); k++) al_add(al, vertex_index(iv), cv.dof[k], cv.val[k]);
	}
	std::vector<int64_t> idx;
	for (int ie = 0; ie < 12; ie++) {
		const int64_t eid = m.elem_edge[12 * e + ie];
		const EData &en = ed[eid];
		if (!en.ced) {
			if (en.n <= 0) continue;
			edge_indices(ie, m.edge_orientation(e, ie), en.order, idx);
			if (en.dof >= 0) {
				for (int j = 0; j < en.n; j++) al_add(al, idx[j], en.dof + j * stride, 1.0);
			}
			else if (en.has_proj) {
				for (int j = 0; j < en.n; j++) al_add(al, idx[j], DIRICHLET_DOF, en.proj[j]);
			}
			continue;
		}
		const CedEdge &ce = econs.at(eid);
		const bool flip = m.hex[8 * e + kHexEdgeVtx[ie][0]] > m.hex[8 * e + kHexEdgeVtx[ie][1]];
		const int nb = ce.order - 1;
		for (size_t k = 0; k < ce.dof.size(); k++)
			for (int mm = 2; mm <= ce.order; mm++) {
				int t[3];
				for (int d = 0; d < 3; d++) t[d] = kEdgePat[ie][d] < 0 ? mm : kEdgePat[ie][d];
				const double sg = (flip && (mm & 1)) ? -1.0 : 1.0;
				al_add(al, canon(SHFN_EDGE, ie, t), ce.dof[k], sg * ce.c[k * nb + mm - 2]);
			}
	}
	for (int f = 0; f < 6; f++) {
		const int64_t fid = m.elem_face[6 * e + f];
		const FData &fn = fd[fid];
		if (!fn.ced) {
			if (fn.n <= 0) continue;
			face_indices(f, m.face_orientation(e, f), fn.ox, fn.oy, idx);
			if (fn.dof >= 0) {
				for (int j = 0; j < fn.n; j++) al_add(al, idx[j], fn.dof + j * stride, 1.0);
			}
			else if (fn.has_proj) {
				for (int j = 0; j < fn.n; j++) al_add(al, idx[j], DIRICHLET_DOF, fn.proj[j]);
			}
			continue;
		}
		const CedFace &cf = fcons.at(fid);
		// local position of the face's axis vertices
		int64_t qv[4];
		int lvq[4];
		for (int q = 0; q < 4; q++) { lvq[q] = kHexFaceVtx[f][q]; qv[q] = m.hex[8 * e + lvq[q]]; }
		int o = 0;
		for (int q = 1; q < 4; q++)
			if (qv[q] < qv[o]) o = q;
		int ih = (o + 1) % 4, iv = (o + 3) % 4;
		if (qv[iv] < qv[ih]) std::swap(ih, iv);
		int dh = -1, dv = -1;
		double sh = 1.0, sv = 1.0;
		for (int d = 0; d < 3; d++) {
			if (kRefVtx[lvq[o]][d] != kRefVtx[lvq[ih]][d]) { dh = d; sh = kRefVtx[lvq[ih]][d] > kRefVtx[lvq[o]][d] ? 1.0 : -1.0; }
			if (kRefVtx[lvq[o]][d] != kRefVtx[lvq[iv]][d]) { dv = d; sv = kRefVtx[lvq[iv]][d] > kRefVtx[lvq[o]][d] ? 1.0 : -1.0; }
		}
		const int nv_ = cf.ov - 1, nper = (cf.oh - 1) * nv_;
		for (size_t k = 0; k < cf.dof.size(); k++)
			for (int a = 2; a <= cf.oh; a++)
				for (int b = 2; b <= cf.ov; b++) {
					int t[3];
					t[kFaceFixedDir[f]] = kFaceFixedVal[f];
					t[dh] = a;
					t[dv] = b;
					const double sg = ((sh < 0 && (a & 1)) ? -1.0 : 1.0) * ((sv < 0 && (b & 1)) ? -1.0 : 1.0);
					al_add(al, canon(SHFN_FACE, f, t), cf.dof[k], sg * cf.c[k * nper + (a - 2) * nv_ + (b - 2)]);
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
// Slabs: the active elements (refined parents are not assembled) ordered by
// centroid (z, then y, then x, then index), cut into nparts contiguous ranges
// of equal count.  Owner of a DOF: the part of the lowest-numbered active
// element whose assembly list holds it as a matrix entry (constrained
// elements list the DOFs of their constraining functions).  Halo: elements
// outside the slab that hold an owned DOF.
int make_partition_scope(const Space &sp, int nparts, int part, PlanScope &S, std::string &err) {
	if (!sp.assigned) { err = "assign_dofs() has not been called"; return -1; }
	if (nparts < 1 || part < 0 || part >= nparts) { err = "partition: need 0 <= part < nparts"; return -1; }
	const Mesh &m = *sp.mesh;
	const int64_t ne = m.ne(), nd = sp.ndof();
	// active elements only (a refined mesh's parents are not assembled)
	std::vector<int64_t> ord;
	for (int64_t e = 0; e < ne; e++)
		if (m.active(e)) ord.push_back(e);
	const int64_t na = (int64_t) ord.size();
	std::vector<std::array<double, 3>> cen(ne);
	for (int64_t e : ord) {
		double c[3] = { 0, 0, 0 };
		for (int v = 0; v < 8; v++)
			for (int r = 0; r < 3; r++) c[r] += m.xyz[3 * m.hex[8 * e + v] + r];
		cen[e] = { c[0] / 8, c[1] / 8, c[2] / 8 };
	}
	std::sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) {
		if (cen[a][2] != cen[b][2]) return cen[a][2] < cen[b][2];
		if (cen[a][1] != cen[b][1]) return cen[a][1] < cen[b][1];
		if (cen[a][0] != cen[b][0]) return cen[a][0] < cen[b][0];
		return a < b;
	});
	std::vector<int> epart(ne, -1);
	for (int64_t r = 0; r < na; r++) epart[ord[r]] = (int) ((r * nparts) / std::max<int64_t>(na, 1));
	std::vector<int64_t> first(nd, -1);
	std::vector<std::vector<int32_t>> edofs(ne);
	parallel_for(ne, [&](int64_t lo, int64_t hi) {
		std::vector<AsmEntry> al;
		for (int64_t e = lo; e < hi; e++) {
			if (epart[e] < 0) continue;
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
		if (epart[e] < 0) continue;                             // refined parent
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
               const PlanScope *scope, const Space *test) {
	if (!sp.assigned || (test && !test->assigned)) { err = "assign_dofs() has not been called"; return -1; }
	const Mesh &m = *sp.mesh;
	const int64_t ne = scope ? (int64_t) scope->elems.size() : m.ne();
	auto G = [&](int64_t e) -> int64_t { return scope ? scope->elems[e] : e; };   // plan element -> mesh element
	if (m.nrefined) { err = "refined meshes take the batched path"; return -1; }
	const Space &ts = test ? *test : sp;
	const bool two = &ts != &sp;
	if (two && (ts.mesh != sp.mesh || scope)) { err = "the test and trial spaces of a block share one mesh (no partition)"; return -1; }
	if (two) canon = true;
	P = Plan();
	P.ne = ne;
	P.ne_ids = m.ne();
	P.ndof = sp.ndof();
	P.two_space = two;
	P.nrow = ts.ndof();
	for (const Space *S : { &sp, &ts })
		for (int64_t e = 0; e < ne; e++)
			if (S->order[3 * G(e)] != S->order[0] || S->order[3 * G(e) + 1] != S->order[1] || S->order[3 * G(e) + 2] != S->order[2]) {
				err = "plan requires one element order triple; bucket mixed orders first";
				return -1;
			}
	P.px = std::max(sp.order[0], ts.order[0]);
	P.py = std::max(sp.order[1], ts.order[1]);
	P.pz = std::max(sp.order[2], ts.order[2]);
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

	// element tables in element-id order first: per element the assembly
	// list's matrix entries, then its lifting entries; DOFs counted from the
	// space's first DOF; canonical indices in the plan's (largest) basis
	auto extract = [&](const Space &S, std::vector<int32_t> &cnt, std::vector<int32_t> &dofs, std::vector<uint16_t> &ss,
	                   std::vector<double> &cf) -> int {
		cnt.assign(2 * ne, 0);
		dofs.assign((size_t) ne * nl, -1);
		ss.assign((size_t) ne * nl, 0);
		cf.assign((size_t) ne * nl, 0.0);
		std::vector<int> bad(ne, 0);
		parallel_for(ne, [&](int64_t lo, int64_t hi) {
			std::vector<AsmEntry> al;
			for (int64_t e = lo; e < hi; e++) {
				S.element_assembly_list(G(e), al);
				int mcount = 0, lcount = 0;
				for (auto &a : al) (a.dof >= 0 ? mcount : lcount)++;
				if (mcount + lcount > nl) { bad[e] = 1; continue; }
				int im = 0, il = mcount;
				for (auto &a : al) {
					Canon c = decode_index(a.idx);
					int sidx = (c.a * (P.py + 1) + c.b) * (P.pz + 1) + c.c;
					int k = a.dof >= 0 ? im++ : il++;
					ss[(size_t) e * nl + k] = (uint16_t) sidx;
					dofs[(size_t) e * nl + k] = a.dof >= 0 ? a.dof - S.first_dof : DIRICHLET_DOF;
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
		return 0;
	};
	std::vector<int32_t> cnt, dofs, tcnt_v, tdofs_v;
	std::vector<uint16_t> ss, tss_v;
	std::vector<double> cf, tcf_v;
	if (extract(sp, cnt, dofs, ss, cf) != 0) return -1;
	if (two && extract(ts, tcnt_v, tdofs_v, tss_v, tcf_v) != 0) return -1;
	// the test side: the test space's tables, or the trial space's
	const std::vector<int32_t> &tcnt = two ? tcnt_v : cnt, &tdofs = two ? tdofs_v : dofs;
	const std::vector<uint16_t> &tss = two ? tss_v : ss;
	const std::vector<double> &tcf = two ? tcf_v : cf;

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
			for (int j = 0; j < tcnt[2 * e]; j++) buf.push_back(tdofs[(size_t) e * nl + j]);   // rows: test DOFs
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

	// test DOF -> elements adjacency of a two-space plan (the RHS and the rows
	// of a column are test DOFs: elements sharing one must not share a colour)
	std::vector<int64_t> tptr;
	std::vector<int32_t> tadj;
	if (two) {
		const int64_t nt = P.nrow;
		tptr.assign(nt + 1, 0);
		for (int64_t e = 0; e < ne; e++)
			for (int k = 0; k < tcnt[2 * e]; k++) tptr[tdofs[(size_t) e * nl + k] + 1]++;
		for (int64_t d = 0; d < nt; d++) tptr[d + 1] += tptr[d];
		tadj.resize(tptr[nt]);
		std::vector<int64_t> fill(tptr.begin(), tptr.end() - 1);
		for (int64_t e = 0; e < ne; e++)
			for (int k = 0; k < tcnt[2 * e]; k++) tadj[fill[tdofs[(size_t) e * nl + k]]++] = (int32_t) e;
	}

	// greedy colouring in element order: colour = smallest not used by an
	// earlier element sharing a DOF
	std::vector<int> color(ne, -1);
	int ncol = 0;
	{
		std::vector<int64_t> stamp(64, -1);
		auto mark = [&](int64_t e, const std::vector<int64_t> &ptr, const std::vector<int32_t> &adj, int d) {
			for (int64_t t = ptr[d]; t < ptr[d + 1]; t++) {
				int64_t o = adj[t];
				if (o < e && color[o] >= 0) {
					if (color[o] >= (int) stamp.size()) stamp.resize(color[o] + 1, -1);
					stamp[color[o]] = e;
				}
			}
		};
		for (int64_t e = 0; e < ne; e++) {
			for (int k = 0; k < cnt[2 * e]; k++) mark(e, dptr, dadj, dofs[(size_t) e * nl + k]);
			if (two)
				for (int k = 0; k < tcnt[2 * e]; k++) mark(e, tptr, tadj, tdofs[(size_t) e * nl + k]);
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
		for (int side = 0; side < (two ? 2 : 1); side++) {
			const std::vector<int32_t> &cn = side ? tcnt : cnt;
			const std::vector<uint16_t> &sx = side ? tss : ss;
			for (int64_t e = 0; e < ne; e++) {
				std::vector<char> seen(nl, 0);
				for (int k = 0; k < cn[2 * e] + cn[2 * e + 1]; k++) {
					int sidx = sx[(size_t) e * nl + k];
					if (seen[sidx]) { err = "a canonical function repeats in one assembly list"; return -1; }
					seen[sidx] = 1;
				}
			}
		}
		P.el_vtx.resize(8 * ne);
		P.el_id.resize(ne);
		P.el_cdof.assign((size_t) ne * nl, -1);
		P.el_ccoef.assign((size_t) ne * nl, 0.0);
		if (two) {
			P.el_tcdof.assign((size_t) ne * nl, -1);
			P.el_tccoef.assign((size_t) ne * nl, 0.0);
		}
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
				if (two)
					for (int t = 0; t < tcnt[2 * e] + tcnt[2 * e + 1]; t++) {
						int sidx = tss[(size_t) e * nl + t];
						P.el_tcdof[(size_t) k * nl + sidx] = tdofs[(size_t) e * nl + t];
						P.el_tccoef[(size_t) k * nl + sidx] = tcf[(size_t) e * nl + t];
					}
				int mc = cnt[2 * e], tmc = tcnt[2 * e];
				for (int b = 0; b < mc; b++) {
					int col = dofs[(size_t) e * nl + b], sj = ss[(size_t) e * nl + b];
					const int32_t *c0 = &P.Ai[P.Ap[col]], *c1 = &P.Ai[P.Ap[col + 1]];
					for (int a = 0; a < tmc; a++) {
						int row = tdofs[(size_t) e * nl + a], si = tss[(size_t) e * nl + a];
						const int32_t *pos = std::lower_bound(c0, c1, row);
						P.el_offc[((size_t) k * nl + si) * nl + sj] = (uint16_t) (pos - c0);
					}
				}
			}
		});
		return 0;
	}

	// tables in assembly (colour-major) order
	P.seg_kof.resize(ne);
	for (int64_t k = 0; k < ne; k++) P.seg_kof[order_[k]] = (int32_t) k;
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
	if (P.px <= kSegMaxOrder && P.py <= kSegMaxOrder && P.pz <= kSegMaxOrder) build_seg_tables(P, kSegWindow);
	return 0;
}

// Tables of the segmented scatter (see Plan::seg).  Needs the colour-major
// element tables and seg_kof.
void build_seg_tables(Plan &P, int window) {
	const int64_t ne = P.ne, nd = P.ndof;
	const int nl = P.nl;
	P.seg = true;
	P.seg_window = window;
	P.seg_nwin = (int) ((ne + window - 1) / window);
	std::vector<int64_t> elem_of_k(ne);
	for (int64_t e = 0; e < ne; e++) elem_of_k[P.seg_kof[e]] = e;
	// pairs of every column in assembly order (k ascending)
	std::vector<int64_t> nptr(nd + 1, 0);
	for (int64_t k = 0; k < ne; k++)
		for (int b = 0; b < P.el_cnt[2 * k]; b++) nptr[P.el_dof[(size_t) k * nl + b] + 1]++;
	for (int64_t d = 0; d < nd; d++) nptr[d + 1] += nptr[d];
	const int64_t npairs = nptr[nd];
	std::vector<int64_t> pk(npairs);
	std::vector<uint8_t> plb(npairs);
	{
		std::vector<int64_t> fill(nptr.begin(), nptr.end() - 1);
		for (int64_t k = 0; k < ne; k++)
			for (int b = 0; b < P.el_cnt[2 * k]; b++) {
				const int64_t t = fill[P.el_dof[(size_t) k * nl + b]]++;
				pk[t] = k;
				plb[t] = (uint8_t) b;
			}
	}
	// first and ready window of every column; processing order by ready window
	std::vector<int32_t> first(nd, 0), ready(nd, -1);
	int span = 0;
	for (int64_t d = 0; d < nd; d++) {
		if (nptr[d + 1] == nptr[d]) continue;
		int64_t lo = ne, hi = -1;
		for (int64_t t = nptr[d]; t < nptr[d + 1]; t++) {
			const int64_t e = elem_of_k[pk[t]];
			lo = std::min(lo, e);
			hi = std::max(hi, e);
		}
		first[d] = (int32_t) (lo / window);
		ready[d] = (int32_t) (hi / window);
		span = std::max(span, ready[d] - first[d]);
	}
	P.seg_span = span;
	int maxcol = 0;
	for (int64_t d = 0; d < nd; d++) maxcol = std::max<int64_t>(maxcol, P.Ap[d + 1] - P.Ap[d]);
	P.seg_maxcol = maxcol;
	std::vector<int64_t> wptr(P.seg_nwin + 1, 0);
	for (int64_t d = 0; d < nd; d++)
		if (ready[d] >= 0) wptr[ready[d] + 1]++;
	for (int w = 0; w < P.seg_nwin; w++) wptr[w + 1] += wptr[w];
	const int64_t ncol = wptr[P.seg_nwin];
	P.seg_col.resize(ncol);
	{
		std::vector<int64_t> fill(wptr.begin(), wptr.end() - 1);
		for (int64_t d = 0; d < nd; d++)
			if (ready[d] >= 0) P.seg_col[fill[ready[d]]++] = (int32_t) d;
	}
	P.seg_cptr.assign(ncol + 1, 0);
	for (int64_t j = 0; j < ncol; j++) P.seg_cptr[j + 1] = P.seg_cptr[j] + (nptr[P.seg_col[j] + 1] - nptr[P.seg_col[j]]);
	P.seg_pe.resize(npairs);
	P.seg_plm.resize(npairs);
	// row positions, padded at the end so a 16-byte-rounded bulk copy of the
	// last batch stays inside the array
	P.seg_off.assign((size_t) npairs * nl + 16, 0);
	parallel_for(ncol, [&](int64_t lo, int64_t hi) {
		for (int64_t j = lo; j < hi; j++) {
			const int64_t d = P.seg_col[j];
			for (int64_t u = 0; u < nptr[d + 1] - nptr[d]; u++) {
				const int64_t s = nptr[d] + u, t = P.seg_cptr[j] + u;
				const int64_t k = pk[s];
				const int lb = plb[s], m = P.el_cnt[2 * k];
				P.seg_pe[t] = (int32_t) elem_of_k[k];
				P.seg_plm[t] = (uint16_t) (lb | (m << 8));
				std::copy(&P.el_off[((size_t) k * nl + lb) * nl], &P.el_off[((size_t) k * nl + lb) * nl] + m,
				          &P.seg_off[(size_t) t * nl]);
			}
		}
	});
	// column batches: consecutive columns of one ready window, at most
	// kSegBatchCols columns and seg_batch_pairs(nl) pairs
	P.seg_p2.clear();
	P.seg_p2ptr.assign(P.seg_nwin + 1, 0);
	for (int w = 0; w < P.seg_nwin; w++) {
		int64_t j = wptr[w];
		while (j < wptr[w + 1]) {
			int64_t j1 = j + 1;
			int lo = first[P.seg_col[j]];
			while (j1 < wptr[w + 1] && j1 - j < kSegBatchCols &&
			       P.seg_cptr[j1 + 1] - P.seg_cptr[j] <= seg_batch_pairs(nl)) {
				lo = std::min(lo, first[P.seg_col[j1]]);
				j1++;
			}
			P.seg_p2.insert(P.seg_p2.end(), { w, lo, (int32_t) j, (int32_t) j1 });
			j = j1;
		}
		P.seg_p2ptr[w + 1] = (int64_t) P.seg_p2.size() / 4;
	}
	// a column whose pairs exceed one batch's staging area: colour sweeps only
	for (int64_t j = 0; j < ncol; j++)
		if (P.seg_cptr[j + 1] - P.seg_cptr[j] > seg_batch_pairs(nl)) {
			P.seg = false;
			break;
		}
	if (!P.seg) {
		P.seg_col.clear(); P.seg_cptr.clear(); P.seg_pe.clear(); P.seg_plm.clear(); P.seg_off.clear();
		P.seg_p2.clear(); P.seg_p2ptr.clear();
	}
}

// Mixed orders.  Same pattern rule as build_plan (the CSC pattern does not
// depend on how the elements are grouped); the per-element tables are
// variable-length, indexed by prefix bases.
int build_plan_mixed(const Space &sp, bool p_plus, int qn, Plan &P, std::string &err, const PlanScope *scope) {
	if (!sp.assigned) { err = "assign_dofs() has not been called"; return -1; }
	const Mesh &m = *sp.mesh;
	std::vector<int64_t> act;                                  // plan element -> mesh element
	if (scope) act = scope->elems;
	else
		for (int64_t e = 0; e < m.ne(); e++)
			if (m.active(e)) act.push_back(e);
	const int64_t ne = (int64_t) act.size();
	auto G = [&](int64_t e) -> int64_t { return act[e]; };
	P = Plan();
	P.ndof = sp.ndof();
	P.ne_ids = m.ne();
	P.mixed = true;
	P.canon = true;
	P.px = P.py = P.pz = -1;
	P.nqx = P.nqy = P.nqz = -1;

	// table sets (p, nq) shared by all elements
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

	// assembly lists; constrained elements in expanded form, grouped by DOF
	struct CedTmp { int p[3]; std::vector<int32_t> udof; std::vector<std::vector<std::pair<int, double>>> col; };
	std::vector<char> isced(ne, 0);
	std::vector<CedTmp> ctmp(ne);
	std::vector<std::vector<AsmEntry>> als(ne);
	parallel_for(ne, [&](int64_t lo, int64_t hi) {
		for (int64_t e = lo; e < hi; e++) {
			isced[e] = sp.element_constrained(G(e));
			sp.element_assembly_list(G(e), als[e]);
		}
	});
	std::vector<std::array<int, 11>> desc(ne);
	std::vector<int64_t> eb(ne + 1, 0);
	for (int64_t e = 0; e < ne; e++) {
		auto &d = desc[e];
		int pe[3];
		for (int r = 0; r < 3; r++) pe[r] = sp.order[3 * G(e) + r];
		if (isced[e])
			for (const AsmEntry &x : als[e]) {
				const Canon c = decode_index(x.idx);
				pe[0] = std::max(pe[0], c.a);
				pe[1] = std::max(pe[1], c.b);
				pe[2] = std::max(pe[2], c.c);
			}
		int nl = 1, pmax = 0, qmax = 0;
		for (int r = 0; r < 3; r++) {
			const int p = sp.order[3 * G(e) + r];
			const int nq = p_plus ? p + qn : qn;
			if (p < 1 || p > 10) { err = "element order out of range"; return -1; }
			if (nq < 1 || nq > kMaxQuadPoints) { err = "Gauss points per direction must be in 1..13"; return -1; }
			d[r] = pe[r];
			d[3 + r] = nq;
			d[6 + r] = table_set(pe[r], nq);
			nl *= pe[r] + 1;
			pmax = std::max(pmax, pe[r]);
			qmax = std::max(qmax, nq);
		}
		d[9] = nl;
		int cls = -1;
		if (!isced[e]) {
			for (int c = 0; c < Plan::kClasses && cls < 0; c++)
				if (pmax <= Plan::kClassP[c] && qmax <= Plan::kClassQ[c]) cls = c;
			if (cls < 0) { err = "mixed-order kernels cover orders <= 6 and <= 8 points per direction"; return -1; }
			P.max_nl = std::max(P.max_nl, nl);
		}
		else {
			for (int c = 0; c < Plan::kCedClasses && cls < 0; c++)
				if (pmax <= Plan::kCedClassP[c] && qmax <= Plan::kCedClassQ[c]) cls = c;
			if (cls < 0) { err = "constrained elements: orders <= 8 and <= 10 points per direction"; return -1; }
			P.ce_max_nl = std::max(P.ce_max_nl, nl);
		}
		d[10] = cls;
		eb[e + 1] = eb[e] + std::max<int64_t>(nl, (int64_t) als[e].size());
	}

	std::vector<int32_t> cnt(2 * ne), dofs(eb[ne], -1);
	std::vector<uint16_t> ss(eb[ne], 0);
	std::vector<double> cf(eb[ne], 0.0);
	std::vector<int> bad(ne, 0);
	parallel_for(ne, [&](int64_t lo, int64_t hi) {
		std::vector<char> seen;
		for (int64_t e = lo; e < hi; e++) {
			const int nl = desc[e][9], py = desc[e][1], pz = desc[e][2];
			const std::vector<AsmEntry> &al = als[e];
			if (isced[e]) {
				CedTmp &t = ctmp[e];
				std::unordered_map<int, int> col_of;
				std::vector<std::pair<int, double>> lift;
				for (const AsmEntry &x : al) {
					const Canon c = decode_index(x.idx);
					const int sidx = (c.a * (py + 1) + c.b) * (pz + 1) + c.c;
					if (sidx < 0 || sidx >= nl) { bad[e] = 3; break; }
					const double w = c.sign * x.coef;
					if (x.dof < 0) { lift.push_back({ sidx, w }); continue; }
					auto it = col_of.find(x.dof);
					if (it == col_of.end()) {
						it = col_of.emplace(x.dof, (int) t.udof.size()).first;
						t.udof.push_back(x.dof);
						t.col.emplace_back();
					}
					t.col[it->second].push_back({ sidx, w });
				}
				if (!lift.empty()) {
					t.udof.push_back(DIRICHLET_DOF);
					t.col.push_back(lift);
				}
				const int nu = (int) t.udof.size() - (lift.empty() ? 0 : 1);
				cnt[2 * e] = nu;
				cnt[2 * e + 1] = 0;
				for (int k = 0; k < nu; k++) dofs[eb[e] + k] = t.udof[k];
				continue;
			}
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

	// order: colour, class, decreasing work (nl^2 * points), element id;
	// unconstrained and constrained elements in separate lists
	std::vector<int64_t> order_, corder;
	for (int64_t e = 0; e < ne; e++) (isced[e] ? corder : order_).push_back(e);
	auto work = [&](int64_t e) { return (int64_t) desc[e][9] * desc[e][9] * desc[e][3]; };
	auto cmp = [&](int64_t x, int64_t y) {
		if (color[x] != color[y]) return color[x] < color[y];
		if (desc[x][10] != desc[y][10]) return desc[x][10] < desc[y][10];
		int64_t wx = work(x), wy = work(y);
		if (wx != wy) return wx > wy;
		return x < y;
	};
	std::sort(order_.begin(), order_.end(), cmp);
	std::sort(corder.begin(), corder.end(), cmp);
	const int64_t nn = (int64_t) order_.size(), nc = (int64_t) corder.size();
	P.ne = nn;
	P.nce = nc;
	P.launch_ptr.assign((size_t) ncol * Plan::kClasses + 1, 0);
	for (int64_t e : order_) P.launch_ptr[(size_t) color[e] * Plan::kClasses + desc[e][10] + 1]++;
	for (size_t i = 0; i + 1 < P.launch_ptr.size(); i++) P.launch_ptr[i + 1] += P.launch_ptr[i];
	P.color_ptr.assign(ncol + 1, 0);
	for (int c = 0; c <= ncol; c++) P.color_ptr[c] = P.launch_ptr[(size_t) c * Plan::kClasses];
	P.ce_launch_ptr.assign((size_t) ncol * Plan::kCedClasses + 1, 0);
	for (int64_t e : corder) P.ce_launch_ptr[(size_t) color[e] * Plan::kCedClasses + desc[e][10] + 1]++;
	for (size_t i = 0; i + 1 < P.ce_launch_ptr.size(); i++) P.ce_launch_ptr[i + 1] += P.ce_launch_ptr[i];

	// per-element tables in assembly order
	P.el_base.assign(nn + 1, 0);
	P.el_obase.assign(nn + 1, 0);
	for (int64_t k = 0; k < nn; k++) {
		const int nl = desc[order_[k]][9];
		P.el_base[k + 1] = P.el_base[k] + nl;
		P.el_obase[k + 1] = P.el_obase[k] + (int64_t) nl * nl;
	}
	P.el_vtx.resize(8 * nn);
	P.el_id.resize(nn);
	P.el_cnt.resize(2 * nn);
	P.el_desc.assign((size_t) nn * Plan::kDescInts, 0);
	P.el_cdof.assign(P.el_base[nn], -1);
	P.el_ccoef.assign(P.el_base[nn], 0.0);
	P.el_offm.assign(P.el_obase[nn], 0);
	parallel_for(nn, [&](int64_t lo, int64_t hi) {
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

	// constrained elements
	P.ce_desc.assign((size_t) nc * Plan::kDescInts, 0);
	P.ce_vtx.resize(8 * nc);
	P.ce_id.resize(nc);
	P.ce_ubase.assign(nc + 1, 0);
	P.ce_obase.assign(nc + 1, 0);
	P.ce_wptr.assign(1, 0);
	for (int64_t k = 0; k < nc; k++) {
		const int64_t e = corder[k];
		const CedTmp &t = ctmp[e];
		P.ce_id[k] = (int32_t) G(e);
		for (int v = 0; v < 8; v++) P.ce_vtx[8 * k + v] = (int32_t) m.hex[8 * G(e) + v];
		for (int q = 0; q < 11; q++) P.ce_desc[(size_t) k * Plan::kDescInts + q] = desc[e][q];
		P.ce_ubase[k + 1] = P.ce_ubase[k] + (int64_t) t.udof.size();
		const int64_t nlk = desc[e][9];
		P.ce_scratch = std::max<int64_t>(P.ce_scratch, nlk * nlk + nlk + (int64_t) t.udof.size() * nlk);
		const int64_t nu = cnt[2 * e];
		P.ce_obase[k + 1] = P.ce_obase[k] + nu * nu;
		for (size_t u = 0; u < t.udof.size(); u++) {
			P.ce_udof.push_back(t.udof[u]);
			for (const auto &sw : t.col[u]) {
				P.ce_ws.push_back((uint16_t) sw.first);
				P.ce_ww.push_back(sw.second);
			}
			P.ce_wptr.push_back((int64_t) P.ce_ws.size());
		}
	}
	P.ce_color_ptr.assign(ncol + 1, 0);
	for (int c = 0; c <= ncol; c++) P.ce_color_ptr[c] = P.ce_launch_ptr[(size_t) c * Plan::kCedClasses];
	P.ce_ebase.assign(nc + 1, 0);
	for (int64_t k = 0; k < nc; k++) {
		const int64_t nu = cnt[2 * corder[k]];
		P.ce_ebase[k + 1] = P.ce_ebase[k] + nu * nu + nu;
	}
	P.ce_order.resize(nc);
	for (int64_t k = 0; k < nc; k++) P.ce_order[k] = (int32_t) k;
	std::sort(P.ce_order.begin(), P.ce_order.end(), [&](int32_t x, int32_t y) {
		const int64_t ex = corder[x], ey = corder[y];
		if (desc[ex][10] != desc[ey][10]) return desc[ex][10] < desc[ey][10];
		const int64_t wx = work(ex), wy = work(ey);
		if (wx != wy) return wx > wy;
		return x < y;
	});
	P.ce_class_ptr.assign(Plan::kCedClasses + 1, 0);
	for (int64_t k = 0; k < nc; k++) P.ce_class_ptr[desc[corder[k]][10] + 1]++;
	for (int c = 0; c < Plan::kCedClasses; c++) P.ce_class_ptr[c + 1] += P.ce_class_ptr[c];
	P.ce_off.assign(P.ce_obase[nc], 0);
	parallel_for(nc, [&](int64_t lo, int64_t hi) {
		for (int64_t k = lo; k < hi; k++) {
			const CedTmp &t = ctmp[corder[k]];
			const int64_t nu = P.ce_obase[k + 1] - P.ce_obase[k] == 0 ? 0 : cnt[2 * corder[k]];
			for (int64_t v = 0; v < nu; v++) {
				const int col = t.udof[v];
				const int32_t *c0 = &P.Ai[P.Ap[col]], *c1 = &P.Ai[P.Ap[col + 1]];
				for (int64_t u = 0; u < nu; u++) {
					const int32_t *pos = std::lower_bound(c0, c1, t.udof[u]);
					P.ce_off[P.ce_obase[k] + v * nu + u] = (uint16_t) (pos - c0);
				}
			}
		}
	});
	return 0;
}

// ---------------------------------------------------------------- evaluation plan

int build_eval_plan(const Space &sp, bool p_plus, int qn, EvalPlan &E, std::string &err) {
	if (!sp.assigned) { err = "assign_dofs() has not been called"; return -1; }
	const Mesh &m = *sp.mesh;
	E = EvalPlan();
	E.gptr.assign(1, 0);
	E.eptr.assign(1, 0);
	std::vector<std::pair<int, int>> set_key;
	std::vector<int> set_off;
	auto table_set = [&](int p, int nq) -> int {
		for (size_t t = 0; t < set_key.size(); t++)
			if (set_key[t].first == p && set_key[t].second == nq) return set_off[t];
		int off = (int) E.tables.size();
		std::vector<double> q, w;
		gauss_legendre(nq, q, w);
		for (int k = 0; k <= p; k++)
			for (int i = 0; i < nq; i++) E.tables.push_back(lobatto_value(k, q[i]));
		for (int k = 0; k <= p; k++)
			for (int i = 0; i < nq; i++) E.tables.push_back(lobatto_deriv(k, q[i]));
		E.tables.insert(E.tables.end(), q.begin(), q.end());
		E.tables.insert(E.tables.end(), w.begin(), w.end());
		set_key.push_back({ p, nq });
		set_off.push_back(off);
		return off;
	};
	std::vector<AsmEntry> al;
	for (int64_t e = 0; e < m.ne(); e++) {
		if (!m.active(e)) continue;
		sp.element_assembly_list(e, al);
		int pe[3];
		for (int r = 0; r < 3; r++) pe[r] = sp.order[3 * e + r];
		struct Ent { int s; int dof; double c; size_t ord; };
		std::vector<Ent> ents;
		std::vector<Canon> cs;
		for (const AsmEntry &x : al) {
			const Canon c = decode_index(x.idx);
			pe[0] = std::max(pe[0], c.a);
			pe[1] = std::max(pe[1], c.b);
			pe[2] = std::max(pe[2], c.c);
			cs.push_back(c);
		}
		int32_t d[12] = { 0 };
		int nl = 1;
		for (int r = 0; r < 3; r++) {
			const int p = sp.order[3 * e + r];
			const int nq = p_plus ? p + qn : qn;
			if (nq < 1 || nq > kMaxQuadPoints || pe[r] > kMaxOrder) { err = "evaluation: order or rule out of range"; return -1; }
			d[r] = pe[r];
			d[3 + r] = nq;
			d[6 + r] = table_set(pe[r], nq);
			nl *= pe[r] + 1;
		}
		d[9] = nl;
		for (size_t i = 0; i < al.size(); i++) {
			const Canon &c = cs[i];
			const int s = (c.a * (pe[1] + 1) + c.b) * (pe[2] + 1) + c.c;
			ents.push_back(Ent { s, al[i].dof, c.sign * al[i].coef, i });
		}
		std::stable_sort(ents.begin(), ents.end(), [](const Ent &x, const Ent &y) { return x.s < y.s; });
		for (size_t i = 0; i < ents.size(); i++) {
			if (i == 0 || ents[i].s != ents[i - 1].s) {
				E.gs.push_back((uint16_t) ents[i].s);
				if (i > 0) E.eptr.push_back((int64_t) E.edof.size());
			}
			E.edof.push_back(ents[i].dof);
			E.ecoef.push_back(ents[i].c);
		}
		if (!ents.empty()) E.eptr.push_back((int64_t) E.edof.size());
		E.gptr.push_back((int64_t) E.gs.size());
		E.desc.insert(E.desc.end(), d, d + 12);
		for (int v = 0; v < 8; v++) E.vtx.push_back((int32_t) m.hex[8 * e + v]);
		E.nlmax = std::max(E.nlmax, nl);
		E.amax = std::max(E.amax, 2 * (pe[0] + 1) * (pe[1] + 1) * d[5]);
		E.bmax = std::max(E.bmax, 3 * (pe[0] + 1) * d[4] * d[5]);
		E.ne++;
	}
	if (E.tables.empty()) E.tables.push_back(0.0);
	return 0;
}

// ---------------------------------------------------------------- surface forms

// Discretization::assemble's surface loop (src/discretization.cc:345-412):
// every outer face of an active element whose marker's BC type is natural,
// with the boundary assembly list (H1Space::get_boundary_assembly_list,
// src/space/h1.cc:139-147: the face's vertex, edge and face functions, i.e.
// the functions whose trace on the face is not zero).
int build_surface_plan(const Space &sp, bool p_plus, int qn, Plan &P, std::string &err) {
	const Mesh &m = *sp.mesh;
	if (m.nrefined) { err = "surface forms on refined meshes are not supported"; return -1; }
	P.nsf = 0;
	P.sf_max_n = 0;
	P.sf_desc.clear(); P.sf_vtx.clear(); P.sf_base.assign(1, 0); P.sf_dof.clear(); P.sf_coef.clear(); P.sf_ab.clear();
	P.sf_obase.assign(1, 0); P.sf_off.clear(); P.sf_color_ptr.clear(); P.sf_tables.clear();
	std::vector<std::pair<int, int>> set_key;
	std::vector<int> set_off;
	auto table_set = [&](int p, int nq) -> int {
		for (size_t t = 0; t < set_key.size(); t++)
			if (set_key[t].first == p && set_key[t].second == nq) return set_off[t];
		int off = (int) P.sf_tables.size();
		std::vector<double> q, w;
		gauss_legendre(nq, q, w);
		P.sf_tables.insert(P.sf_tables.end(), q.begin(), q.end());
		P.sf_tables.insert(P.sf_tables.end(), w.begin(), w.end());
		for (int k = 0; k <= p; k++)
			for (int i = 0; i < nq; i++) P.sf_tables.push_back(lobatto_value(k, q[i]));
		set_key.push_back({ p, nq });
		set_off.push_back(off);
		return off;
	};
	std::vector<AsmEntry> al;
	std::vector<std::vector<int32_t>> face_dofs;
	for (int64_t e = 0; e < m.ne(); e++) {
		if (!m.active(e)) continue;
		for (int f = 0; f < 6; f++) {
			const int64_t fid = m.elem_face[6 * e + f];
			if (!m.facet_outer[fid]) continue;
			const int marker = m.facet_marker[fid];
			const int bc = sp.bc_type_fn ? sp.bc_type_fn(marker, sp.bc_type_ctx) : BC_ESSENTIAL;
			if (bc != BC_NATURAL) continue;
			sp.element_assembly_list(e, al);
			const int dn = kFaceFixedDir[f], side = kFaceFixedVal[f];
			const int d1 = kFaceDirs[f][0], d2 = kFaceDirs[f][1];
			std::vector<int32_t> fd_;
			int n = 0;
			for (const AsmEntry &x : al) {
				const Canon c = decode_index(x.idx);
				const int ind[3] = { c.a, c.b, c.c };
				if (ind[dn] != side) continue;
				P.sf_dof.push_back(x.dof);
				P.sf_coef.push_back(c.sign * x.coef);
				P.sf_ab.push_back((int16_t) ind[d1]);
				P.sf_ab.push_back((int16_t) ind[d2]);
				if (x.dof >= 0) fd_.push_back(x.dof);
				n++;
			}
			const int p1 = sp.order[3 * e + d1], p2 = sp.order[3 * e + d2];
			const int nq1 = p_plus ? p1 + qn : qn, nq2 = p_plus ? p2 + qn : qn;
			if (nq1 < 1 || nq1 > kMaxQuadPoints || nq2 < 1 || nq2 > kMaxQuadPoints) { err = "surface rule out of range"; return -1; }
			int32_t d[Plan::kSfDescInts] = { (int32_t) e, f, marker, n, nq1, nq2, table_set(p1, nq1), table_set(p2, nq2) };
			P.sf_desc.insert(P.sf_desc.end(), d, d + Plan::kSfDescInts);
			for (int v = 0; v < 8; v++) P.sf_vtx.push_back((int32_t) m.hex[8 * e + v]);
			P.sf_base.push_back((int64_t) P.sf_dof.size());
			P.sf_obase.push_back(P.sf_obase.back() + (int64_t) n * n);
			P.sf_max_n = std::max(P.sf_max_n, n);
			face_dofs.push_back(fd_);
			P.nsf++;
		}
	}
	// offsets into the volume pattern
	P.sf_off.assign(P.sf_obase.back(), 0);
	for (int64_t k = 0; k < P.nsf; k++) {
		const int64_t b = P.sf_base[k], n = P.sf_base[k + 1] - b, ob = P.sf_obase[k];
		for (int64_t j = 0; j < n; j++) {
			const int dj = P.sf_dof[b + j];
			if (dj < 0) continue;
			const int32_t *c0 = &P.Ai[P.Ap[dj]], *c1 = &P.Ai[P.Ap[dj + 1]];
			for (int64_t i = 0; i < n; i++) {
				const int di = P.sf_dof[b + i];
				if (di < 0) continue;
				const int32_t *pos = std::lower_bound(c0, c1, di);
				if (pos == c1 || *pos != di) { err = "surface entry outside the volume pattern"; return -1; }
				P.sf_off[ob + j * n + i] = (uint16_t) (pos - c0);
			}
		}
	}
	// greedy colouring of the faces by shared DOFs, faces reordered by colour
	std::unordered_map<int32_t, std::vector<int64_t>> dof_faces;
	std::vector<int> col(P.nsf, -1);
	int ncol = 0;
	for (int64_t k = 0; k < P.nsf; k++) {
		std::vector<char> used(ncol + 1, 0);
		for (int32_t d : face_dofs[k]) {
			auto it = dof_faces.find(d);
			if (it == dof_faces.end()) continue;
			for (int64_t o : it->second) used[col[o]] = 1;
		}
		int c = 0;
		while (used[c]) c++;
		col[k] = c;
		ncol = std::max(ncol, c + 1);
		for (int32_t d : face_dofs[k]) dof_faces[d].push_back(k);
	}
	std::vector<int64_t> ord(P.nsf);
	for (int64_t k = 0; k < P.nsf; k++) ord[k] = k;
	std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return col[a] < col[b]; });
	Plan Q;
	Q.sf_base.assign(1, 0);
	Q.sf_obase.assign(1, 0);
	for (int64_t k : ord) {
		const int64_t b = P.sf_base[k], n = P.sf_base[k + 1] - b, ob = P.sf_obase[k];
		Q.sf_desc.insert(Q.sf_desc.end(), &P.sf_desc[k * Plan::kSfDescInts], &P.sf_desc[(k + 1) * Plan::kSfDescInts]);
		Q.sf_vtx.insert(Q.sf_vtx.end(), &P.sf_vtx[8 * k], &P.sf_vtx[8 * k + 8]);
		Q.sf_dof.insert(Q.sf_dof.end(), P.sf_dof.begin() + b, P.sf_dof.begin() + b + n);
		Q.sf_coef.insert(Q.sf_coef.end(), P.sf_coef.begin() + b, P.sf_coef.begin() + b + n);
		Q.sf_ab.insert(Q.sf_ab.end(), P.sf_ab.begin() + 2 * b, P.sf_ab.begin() + 2 * (b + n));
		Q.sf_off.insert(Q.sf_off.end(), P.sf_off.begin() + ob, P.sf_off.begin() + ob + n * n);
		Q.sf_base.push_back((int64_t) Q.sf_dof.size());
		Q.sf_obase.push_back((int64_t) Q.sf_off.size());
	}
	P.sf_desc.swap(Q.sf_desc); P.sf_vtx.swap(Q.sf_vtx); P.sf_dof.swap(Q.sf_dof); P.sf_coef.swap(Q.sf_coef);
	P.sf_ab.swap(Q.sf_ab); P.sf_off.swap(Q.sf_off); P.sf_base.swap(Q.sf_base); P.sf_obase.swap(Q.sf_obase);
	P.sf_color_ptr.assign(ncol + 1, 0);
	for (int64_t k = 0; k < P.nsf; k++) P.sf_color_ptr[col[k] + 1]++;
	for (int c = 0; c < ncol; c++) P.sf_color_ptr[c + 1] += P.sf_color_ptr[c];
	if (P.sf_tables.empty()) P.sf_tables.push_back(0.0);
	return 0;
}

} // namespace h3dg
