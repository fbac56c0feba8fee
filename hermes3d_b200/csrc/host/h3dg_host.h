// Host-side mesh, H1 Lobatto space and assembly plan.
//
// This is the part of the assembly path that runs once per mesh/space on
// the CPU: topology, orientations, DOF numbering, Dirichlet lifting
// coefficients, assembly lists, the CSC sparsity pattern and the per-element
// tables the GPU kernels consume.  The numbering rules reproduce the
// reference's bit for bit (checked against the reference itself by the
// parity tests); each routine cites the reference code it follows.
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace h3dg {

// ---------------------------------------------------------------- reference tables
// RefHex (src/refdomain.cc:96-130)
extern const int kHexEdgeVtx[12][2];
extern const int kHexFaceVtx[6][4];
extern const int kHexFaceEdges[6][4];
extern const int kVertexXYZ[8][3];   // Lobatto vertex indices (h1lobattohex.cc:68-73)

enum BcType { BC_ESSENTIAL = 0, BC_NATURAL = 1, BC_NONE = 2 };   // src/space.h:44-48
constexpr int DIRICHLET_DOF = -1;                                  // src/common.h:187
constexpr int MARKER_UNDEFINED = -1;

enum ShfnType { SHFN_VERTEX = 0, SHFN_EDGE = 1, SHFN_FACE = 2, SHFN_BUBBLE = 3 };

// h1_hex_index_t bit layout (src/shapeset/h1lobattohex.cc:36-65)
inline int64_t encode_index(int type, int ef, int x, int y, int z, int ori) {
	return ((int64_t) type << 19) | ((int64_t) ef << 15) | ((int64_t) ori << 12) | (x << 8) | (y << 4) | z;
}

// Decoded form of a shape index: tensor indices (a,b,c) of the canonical
// basis L_a(xi) L_b(eta) L_c(zeta) and the sign that orientation flips
// introduce (decompose(), h1lobattohex.cc:98-130; L_k(-x) = (-1)^k L_k(x)).
struct Canon {
	int a, b, c;
	int sign;
};
Canon decode_index(int64_t idx);

// ---------------------------------------------------------------- mesh
struct Mesh {
	// input (vertex and element ids are 1-based in the reference; stored 0-based here)
	std::vector<double> xyz;                 // nv x 3
	std::vector<int64_t> hex;                // ne x 8 (0-based vertex index, RefHex order)
	std::vector<std::array<int64_t, 4>> bquad;
	std::vector<int> bmarker;

	// derived by finalize()
	int64_t nfacets = 0, nedges = 0;
	std::vector<int64_t> elem_face;          // ne x 6 -> facet id (creation order)
	std::vector<int64_t> elem_edge;          // ne x 12 -> edge id
	std::vector<int64_t> facet_left, facet_left_face, facet_right;  // right = -1 if none
	std::vector<int> facet_outer;            // 1 if boundary facet
	std::vector<int> facet_marker;           // boundary marker (outer facets)
	std::vector<int> edge_bnd;
	bool finalized = false;

	// refinement tree (Mesh::refine_element with REFT_HEX_XYZ, src/mesh.cc:1262-1633):
	// children get the next element ids, new vertices the next vertex ids
	std::vector<int64_t> parent;             // ne: parent element, -1 for a base element
	std::vector<int64_t> sons;               // ne x 8: child elements (-1: none, element active)
	std::map<std::pair<int64_t, int64_t>, int64_t> midpoints;   // vertex pair (ascending) -> midpoint vertex
	int64_t nrefined = 0;

	// derived by finalize() when elements are refined: hanging nodes
	// (Space::fc_element, src/space.cc:598-736).  A face of an inactive element
	// whose neighbour across it is active is a constraining face: the nodes its
	// refinement created (edge midpoints, face midpoint, half edges, mid edges,
	// quarter faces) are constrained.
	std::vector<char> vertex_ced, edge_ced, facet_ced;
	struct Interface { int64_t small_parent; int face; int64_t big; int big_face; };
	std::vector<Interface> interfaces;
	std::vector<std::pair<int64_t, int64_t>> edge_vtx;   // nedges: the two vertices (ascending)

	int64_t nv() const { return (int64_t) xyz.size() / 3; }
	int64_t ne() const { return (int64_t) hex.size() / 8; }
	bool active(int64_t e) const { return sons.empty() || sons[8 * e] < 0; }

	int finalize(std::string &err);
	int refine_xyz(int64_t e, std::string &err, bool refinalize = true);
	int edge_orientation(int64_t e, int iedge) const;
	int face_orientation(int64_t e, int iface) const;
};

// ---------------------------------------------------------------- space
typedef int (*BcTypeFn)(int marker, void *ctx);
typedef double (*BcValueFn)(int marker, double x, double y, double z, void *ctx);

struct AsmEntry {
	int64_t idx;     // reference shape index (h1_hex_index_t encoding)
	int dof;         // global DOF, or DIRICHLET_DOF
	double coef;     // 1.0, or the Dirichlet lifting coefficient
};

// Restriction of global basis functions to a constrained node, in the node's
// own parametrisation (edge: from its lower to its higher vertex id; face: see
// ced_face_axes).  Entry k holds a global function (DOF, or DIRICHLET_DOF with
// the lifting value folded in) and the coefficients of the node's functions.
struct CedVertex { std::vector<int> dof; std::vector<double> val; };
struct CedEdge { int order = 1; std::vector<int> dof; std::vector<double> c; };              // c: n x (order - 1), m = 2..order
struct CedFace { int oh = 1, ov = 1; std::vector<int> dof; std::vector<double> c; };         // c: n x (oh - 1)(ov - 1)

struct Space {
	const Mesh *mesh = nullptr;
	std::vector<int> order;                  // ne x 3 element orders
	BcTypeFn bc_type_fn = nullptr;
	void *bc_type_ctx = nullptr;
	BcValueFn bc_value_fn = nullptr;
	void *bc_value_ctx = nullptr;

	// node data (src/space.h:110-300)
	struct VData { int bc = BC_NONE, marker = MARKER_UNDEFINED, dof = -2; double proj = 0.0; bool ced = false; };
	struct EData { int bc = BC_NONE, marker = MARKER_UNDEFINED, order = -1, dof = -2, n = -1; std::vector<double> proj; bool has_proj = false; bool ced = false; };
	struct FData { int bc = BC_NONE, marker = MARKER_UNDEFINED, ox = -1, oy = -1, dof = -2, n = -1; std::vector<double> proj; bool has_proj = false; bool ced = false; };
	struct BData { int dof = -2, n = -1; };
	std::vector<VData> vd;
	std::vector<EData> ed;
	std::vector<FData> fd;
	std::vector<BData> bd;
	int first_dof = 0, next_dof = 0, stride = 1;
	bool assigned = false;
	// constraints of the hanging nodes (empty without refinement)
	std::map<int64_t, CedVertex> vcons;
	std::map<int64_t, CedEdge> econs;
	std::map<int64_t, CedFace> fcons;

	int ndof() const { return (next_dof - first_dof) / stride; }
	bool constrained() const { return !vcons.empty() || !econs.empty() || !fcons.empty(); }
	int assign_dofs(int first, int stride, std::string &err);
	// For an element with constrained nodes the list is in expanded form: one
	// entry per (canonical function, global function), idx = the canonical
	// function with orientation 0, coef = the restriction coefficient (sign
	// included).  A constrained function of the reference's list
	// (src/space.cc:296-450, negative CED indices) is the sum of its entries.
	void element_assembly_list(int64_t e, std::vector<AsmEntry> &al) const;
	bool element_constrained(int64_t e) const;

private:
	int lift_edge(int64_t e, int iedge);     // 0, or -1 / -2 when the projection fails
	int lift_face(int64_t e, int iface);
	int build_constraints(std::string &err);
	void constrained_assembly_list(int64_t e, std::vector<AsmEntry> &al) const;
};

// ---------------------------------------------------------------- assembly plan
// Everything the device kernels need for one (space, quadrature) pair.
struct Plan {
	int64_t ne = 0, ndof = 0, nnz = 0;
	int px = 0, py = 0, pz = 0;              // uniform element order of this plan
	int nl = 0;                              // (px+1)(py+1)(pz+1)
	int nqx = 0, nqy = 0, nqz = 0;           // Gauss points per direction

	// CSC pattern, == Discretization::create + UMFPackMatrix::alloc
	std::vector<int64_t> Ap;                 // ndof + 1
	std::vector<int32_t> Ai;                 // nnz

	// per element (assembly order), padded to nl entries
	std::vector<int32_t> el_vtx;             // ne x 8
	std::vector<int32_t> el_cnt;             // ne x 2: matrix entries m, lifting entries l
	std::vector<uint16_t> el_s;              // ne x nl canonical index (a*(py+1)+b)*(pz+1)+c
	std::vector<int32_t> el_dof;             // ne x nl
	std::vector<double> el_coef;             // ne x nl (orientation sign x AsmList coef)
	std::vector<uint16_t> el_off;            // ne x nl x nl: row position of dof_a in column dof_b
	std::vector<int32_t> el_id;              // reference element id - 1 of each assembly slot

	// canonical form (high orders): indexed by the canonical function, not the
	// AsmList entry; requires each canonical function to occur at most once
	bool canon = false;
	std::vector<int32_t> el_cdof;            // ne x nl: DOF or -1
	std::vector<double> el_ccoef;            // ne x nl: sign x coefficient (lifting value when DOF = -1), 0 absent
	// a block of a system whose test space differs from the trial space
	// (src/discretization.cc:290-325 with spaces m != n): the test space's
	// canonical tables; the CSC columns are trial DOFs, the rows test DOFs
	bool two_space = false;
	int64_t nrow = 0;                        // test DOFs of a two-space plan
	int64_t nrhs() const { return two_space ? nrow : ndof; }   // RHS length (rows)
	std::vector<int32_t> el_tcdof;           // ne x nl: test DOF or -1
	std::vector<double> el_tccoef;           // ne x nl: test coefficient (0 absent)
	std::vector<uint16_t> el_offc;           // ne x nl x nl: [i][j] row position of cdof_i in column cdof_j

	// element colouring: no two elements of a colour share a DOF
	int ncolors = 0;
	std::vector<int64_t> color_ptr;          // ncolors + 1 (ranges in assembly order)

	// Segmented scatter (uniform low orders).  The element matrices are
	// computed in element order (plan element index, ascending mesh id) into
	// a ring of slots in global memory; every CSC column is then summed from
	// the matrices of its elements, in assembly order (colour, then element:
	// the order in which the colour sweeps add), and written once.  Elements
	// are grouped in windows of seg_window; a column is "ready" in the window
	// of its last element and is processed after that window.  Pairs (column,
	// element) carry the element's local index of the column's DOF and the
	// row positions of the element's DOFs inside the column.
	bool seg = false;
	int seg_window = 0;                      // elements per window
	int seg_nwin = 0;                        // windows
	int seg_span = 0;                        // max over columns: ready window - first window
	int seg_maxcol = 0;                      // longest column (rows)
	std::vector<int32_t> seg_kof;            // ne: plan element -> assembly index k
	std::vector<int32_t> seg_col;            // columns in processing order: DOF
	std::vector<int64_t> seg_cptr;           // columns + 1: pair ranges
	std::vector<int32_t> seg_pe;             // per pair: plan element
	std::vector<uint16_t> seg_plm;           // per pair: local index of the DOF | matrix entries << 8
	std::vector<uint16_t> seg_off;           // per pair x nl: row position of the element's row a (a < m)
	std::vector<int32_t> seg_p2;             // column batches, 4 ints each: ready window, first window, begin, end
	std::vector<int64_t> seg_p2ptr;          // seg_nwin + 1: column batches per ready window

	// 1D tables (b): per direction, V[k][q] and D[k][q] (k <= p, q < nq) and rule
	std::vector<double> qx, wx, qy, wy, qz, wz;

	// mixed orders (batched path): every element has its own order triple and
	// rule.  Canonical tables with per-element bases; el_offm is [j][i]
	// (column-major: for one trial function j the rows i are contiguous).
	bool mixed = false;
	static constexpr int kClasses = 3;       // kernel classes by (max order, max points)
	static constexpr int kClassP[kClasses] = { 2, 4, 6 };
	static constexpr int kClassQ[kClasses] = { 4, 6, 8 };
	static constexpr int kDescInts = 12;     // px py pz nqx nqy nqz ox oy oz nl class -
	std::vector<int32_t> el_desc;            // ne x kDescInts (assembly order); o*: offsets (doubles) of the
	                                         // direction's table set in mixed_tables
	std::vector<int64_t> el_base;            // ne + 1: element k's nl entries of el_cdof / el_ccoef start here
	std::vector<int64_t> el_obase;           // ne + 1: element k's nl * nl entries of el_offm start here
	std::vector<uint16_t> el_offm;           // [j][i] row position of cdof_i in column cdof_j
	std::vector<double> mixed_tables;        // per (p, nq) set: V[(p+1) nq], D[(p+1) nq], q[nq], w[nq]
	std::vector<int64_t> launch_ptr;         // ncolors * kClasses + 1: (colour, class) ranges, assembly order
	int max_nl = 0;
	int64_t ne_ids = 0;                      // element ids of the mesh (coefficient arrays are indexed by them)

	// elements with constrained nodes (hanging nodes): the element matrix is
	// computed in the element's canonical basis, with the orders raised to
	// those of the constraining functions, and mapped onto the global
	// functions by W: column u of element k lists (canonical function, weight)
	// pairs; a global DOF has one column, the Dirichlet lifting one more (DOF -1,
	// always last).  K_uv = sum_a sum_b w_a w_b K[s_b][s_a].
	static constexpr int kCedClasses = 3;
	static constexpr int kCedClassP[kCedClasses] = { 4, 6, 8 };
	static constexpr int kCedClassQ[kCedClasses] = { 6, 8, 10 };
	int64_t nce = 0;
	int ce_max_nl = 0;
	int64_t ce_scratch = 0;                  // doubles of per-CTA scratch: max nl^2 + nl + columns x nl
	std::vector<int32_t> ce_desc;            // nce x kDescInts (as el_desc, orders raised)
	std::vector<int32_t> ce_vtx, ce_id;      // nce x 8, nce
	std::vector<int64_t> ce_ubase;           // nce + 1: the element's columns
	std::vector<int32_t> ce_udof;            // per column: DOF or -1
	std::vector<int64_t> ce_wptr;            // columns + 1
	std::vector<uint16_t> ce_ws;             // canonical function
	std::vector<double> ce_ww;               // weight
	std::vector<int64_t> ce_obase;           // nce + 1
	std::vector<uint16_t> ce_off;            // per element [v][u] (DOF columns): row position of DOF u in column DOF v
	std::vector<int64_t> ce_launch_ptr;      // ncolors * kCedClasses + 1
	std::vector<int64_t> ce_color_ptr;       // ncolors + 1: the colour's elements (scatter launches)
	std::vector<int32_t> ce_order;           // compute order: by class, then decreasing work
	std::vector<int64_t> ce_class_ptr;       // kCedClasses + 1: ranges of ce_order
	std::vector<int64_t> ce_ebase;           // nce + 1: output slice (nu x nu entries, then nu rhs values)

	// surface forms on the outer faces of active elements whose marker is
	// natural (src/discretization.cc:345-412): per face the trace functions of
	// the element's assembly list (canonical index on the face's normal equal
	// to the face's side), the element's rule on the face's two directions
	static constexpr int kSfDescInts = 8;    // element (mesh index), face, marker, n, nq1, nq2, t1, t2
	int64_t nsf = 0;
	int sf_max_n = 0;
	std::vector<int32_t> sf_desc;            // nsf x kSfDescInts; t1, t2: offsets of the direction tables
	std::vector<int32_t> sf_vtx;             // nsf x 8
	std::vector<int64_t> sf_base;            // nsf + 1: trace functions
	std::vector<int32_t> sf_dof;             // DOF or -1
	std::vector<double> sf_coef;             // sign x assembly-list coefficient
	std::vector<int16_t> sf_ab;              // 2 per trace function: Lobatto index along the two face directions
	std::vector<int64_t> sf_obase;           // nsf + 1
	std::vector<uint16_t> sf_off;            // [j][i]: row position of dof_i in column dof_j (both >= 0)
	std::vector<int64_t> sf_color_ptr;       // colours of faces (no two faces of a colour share a DOF)
	std::vector<double> sf_tables;           // per (order, points) set: q[nq], w[nq], V[(p+1) nq]
};

// Evaluation plan of a finite-element function on the active elements (norms,
// src/norm.cc:33-180): per element its orders and rule (p_d + qn or qn points,
// orders raised where constraints need it), and its expanded assembly list
// grouped by canonical function (groups ascending, entries in list order).
struct EvalPlan {
	int64_t ne = 0;
	int nlmax = 0, amax = 0, bmax = 0;       // largest C, A and B work arrays (doubles)
	std::vector<int32_t> desc;               // ne x 12 (as Plan::el_desc)
	std::vector<int32_t> vtx;                // ne x 8
	std::vector<int64_t> gptr, eptr;         // ne + 1, groups + 1
	std::vector<uint16_t> gs;
	std::vector<int32_t> edof;
	std::vector<double> ecoef;
	std::vector<double> tables;              // per set: V, D, q, w (as Plan::mixed_tables)
};
int build_eval_plan(const Space &sp, bool p_plus, int qn, EvalPlan &E, std::string &err);

// surface-form plan of the outer faces whose marker is natural (needs the
// volume plan's pattern); nq per direction p_d + qn (p_plus) or qn
int build_surface_plan(const Space &sp, bool p_plus, int qn, Plan &P, std::string &err);

// One part of a z-slab partition of the mesh (multi-GPU sharding without
// communication): the part's slab of elements plus the one-element halo that
// touches its DOFs, and the DOFs it owns.  A DOF belongs to the part whose
// slab holds the lowest-numbered element with that DOF in its assembly list.
// A plan built with a scope holds the full CSC columns of the owned DOFs
// (global row and column numbering) and empty columns elsewhere, so every
// owned column equals the one of the whole-mesh plan.
struct PlanScope {
	std::vector<int64_t> elems;              // element indices (0-based, ascending): slab + halo
	std::vector<char> owned;                 // ndof: 1 where this part owns the DOF (CSC column)
	int64_t nslab = 0, nhalo = 0, nowned = 0;
};
int make_partition_scope(const Space &sp, int nparts, int part, PlanScope &scope, std::string &err);

// segmented scatter: orders it is built for, elements per window, and the
// bounds of one column batch (columns, pairs: the staging area of a batch)
constexpr int kSegMaxOrder = 3;
constexpr int kSegWindow = 256;
constexpr int kSegBatchCols = 32;
constexpr int seg_batch_pairs(int nl) { return nl <= 27 ? 128 : 64; }
void build_seg_tables(Plan &plan, int window);

// test: the test space of a system block (nullptr: the trial space); a
// two-space plan is canonical, at the larger of the two (uniform) orders.
// DOFs are numbered from each space's first DOF (the plan's own numbering).
int build_plan(const Space &sp, int nqx, int nqy, int nqz, Plan &plan, std::string &err, bool canon = false,
               const PlanScope *scope = nullptr, const Space *test = nullptr);

// Mixed orders: per element p_d + qn points per direction (p_plus) or qn
// (fixed).  Elements are grouped by colour, then by kernel class, and within
// a (colour, class) range ordered by decreasing work.
int build_plan_mixed(const Space &sp, bool p_plus, int qn, Plan &plan, std::string &err, const PlanScope *scope = nullptr);

} // namespace h3dg
