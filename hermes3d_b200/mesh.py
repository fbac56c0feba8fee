"""Hexahedral meshes: the reference's Mesh building calls, the mesh3d text
format of Mesh3DReader, and seeded structured unit-cube generators.

Vertex and element ids are 1-based, as in the reference (src/mesh.cc:915-1000).
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from . import _capi as capi


class Mesh:
    """Mirror of ``Mesh`` (src/mesh.h:522-698) for hexahedra.

    Build with add_vertex / add_hex / add_quad_boundary (or the array forms)
    and call ``ugh()`` once, as the reference's loader does.
    """

    def __init__(self):
        self._xyz = []
        self._hex = []
        self._bq = []
        self._bm = []
        self.handle = None
        self.xyz = None
        self.hexes = None
        self.bquads = None
        self.bmarkers = None
        self.parent = None
        self.refinements = []
        self._base = None

    # --- reference-style incremental calls
    def add_vertex(self, x, y, z):
        self._xyz.append((float(x), float(y), float(z)))
        return len(self._xyz)

    def add_hex(self, vtcs):
        self._hex.append(tuple(int(v) for v in vtcs))
        return len(self._hex)

    def add_quad_boundary(self, vtcs, marker):
        self._bq.append(tuple(int(v) for v in vtcs))
        self._bm.append(int(marker))

    # --- array forms
    def set_arrays(self, xyz, hexes, bquads, bmarkers):
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self.hexes = np.ascontiguousarray(hexes, dtype=np.int64).reshape(-1, 8)
        self.bquads = np.ascontiguousarray(bquads, dtype=np.int64).reshape(-1, 4)
        self.bmarkers = np.ascontiguousarray(bmarkers, dtype=np.int32).reshape(-1)
        return self

    def ugh(self):
        """Finalise topology (Mesh::ugh) and check every outer face has a boundary."""
        if self.xyz is None:
            self.set_arrays(np.array(self._xyz, dtype=np.float64).reshape(-1, 3),
                            np.array(self._hex, dtype=np.int64).reshape(-1, 8),
                            np.array(self._bq, dtype=np.int64).reshape(-1, 4),
                            np.array(self._bm, dtype=np.int32))
        h = C.c_void_p()
        capi.call("h3dg_mesh_create", C.byref(h))
        self.handle = h
        capi.call("h3dg_mesh_add_vertices", h, capi.ptr(self.xyz, C.c_double), len(self.xyz))
        capi.call("h3dg_mesh_add_hexes", h, capi.ptr(self.hexes, C.c_int64), len(self.hexes))
        capi.call("h3dg_mesh_add_quad_boundaries", h, capi.ptr(self.bquads, C.c_int64),
                  capi.ptr(self.bmarkers, C.c_int32), len(self.bquads))
        capi.call("h3dg_mesh_finalize", h)
        self._base = (self.xyz, self.hexes)
        self.parent = np.zeros(len(self.hexes), np.int64)
        return self

    finalize = ugh

    REFT_HEX_XYZ = 7

    def refine_element(self, elem_id, refinement=REFT_HEX_XYZ):
        """Mesh::refine_element (src/mesh.cc:1262-1279), REFT_HEX_XYZ of an active base
        element; children get the next element ids, new vertices the next vertex ids."""
        if self.handle is None:
            self.ugh()
        capi.call("h3dg_mesh_refine_element", self.handle, int(elem_id), int(refinement))
        self.refinements.append((int(elem_id), int(refinement)))
        self._read_back()
        return True

    def refine_elements(self, elem_ids, refinement=REFT_HEX_XYZ):
        """refine_element for each id in order, rebuilding the topology once."""
        if self.handle is None:
            self.ugh()
        ids = np.ascontiguousarray(elem_ids, dtype=np.int64)
        capi.call("h3dg_mesh_refine_elements", self.handle, capi.ptr(ids, C.c_int64), len(ids), int(refinement))
        self.refinements += [(int(e), int(refinement)) for e in ids]
        self._read_back()
        return True

    def _read_back(self):
        nv, ne, _, _ = self.counts()
        xyz = np.zeros((nv, 3), np.float64)
        hexes = np.zeros((ne, 8), np.int64)
        parent = np.zeros(ne, np.int64)
        capi.call("h3dg_mesh_get_arrays", self.handle, capi.ptr(xyz, C.c_double), capi.ptr(hexes, C.c_int64),
                  capi.ptr(parent, C.c_int64))
        self.xyz, self.hexes, self.parent = xyz, hexes, parent

    @property
    def num_active_elements(self):
        return int(self.active.sum())

    @property
    def active(self):
        """Boolean mask over element ids 1..ne (index id - 1): not refined."""
        act = np.ones(len(self.hexes), bool)
        if self.parent is not None:
            act[self.parent[self.parent > 0] - 1] = False
        return act

    @property
    def num_elements(self):
        return len(self.hexes)

    @property
    def num_vertices(self):
        return len(self.xyz)

    def counts(self):
        v = [C.c_int64() for _ in range(4)]
        capi.call("h3dg_mesh_counts", self.handle, *[C.byref(x) for x in v])
        return tuple(x.value for x in v)

    def __del__(self):
        if getattr(self, "handle", None) and capi._lib is not None:
            capi.lib().h3dg_mesh_destroy(self.handle)
            self.handle = None

    # --- file formats
    def save_bin(self, path):
        """Binary mesh file read by the oracle driver ("H3DMESH1"): the base mesh
        (refinements are passed to the driver separately)."""
        xyz, hexes = self._base if self._base is not None else (self.xyz, self.hexes)
        with open(path, "wb") as f:
            f.write(b"H3DMESH1")
            f.write(struct.pack("<q", len(xyz)))
            f.write(xyz.tobytes())
            f.write(struct.pack("<q", len(hexes)))
            f.write(hexes.tobytes())
            bq = np.concatenate([self.bquads, self.bmarkers.astype(np.int64)[:, None]], axis=1)
            f.write(struct.pack("<q", len(bq)))
            f.write(np.ascontiguousarray(bq).tobytes())


def load_mesh3d(path):
    """Read the reference's mesh3d text format (src/loader/mesh3d.cc:103-290): hexes and
    quad boundaries only."""
    rows = []
    with open(path) as f:
        for line in f:
            s = line.split("#", 1)[0].strip() if line.lstrip().startswith("#") else line.strip()
            if s:
                rows.append(s)
    it = iter(rows)
    nv = int(next(it))
    xyz = [tuple(float(t) for t in next(it).split()[:3]) for _ in range(nv)]
    ntet = int(next(it))
    for _ in range(ntet):
        next(it)
    nhex = int(next(it))
    hexes = [tuple(int(t) for t in next(it).split()[:8]) for _ in range(nhex)]
    npr = int(next(it))
    for _ in range(npr):
        next(it)
    ntri = int(next(it))
    for _ in range(ntri):
        next(it)
    nq = int(next(it))
    bq, bm = [], []
    for _ in range(nq):
        t = [int(x) for x in next(it).split()]
        bq.append(t[:4])
        bm.append(t[4])
    for h in hexes:
        if any(v < 1 or v > nv for v in h):
            raise ValueError("Invalid vertex index was found in the section defining hexes.")
    m = Mesh()
    return m.set_arrays(np.array(xyz), np.array(hexes), np.array(bq).reshape(-1, 4), np.array(bm))


def unit_cube(n, jitter=0.0, seed=0, nx=None, ny=None, nz=None):
    """Structured hexahedral mesh of [0,1]^3 with n^3 elements (or nx*ny*nz).

    Vertices are numbered lexicographically (x fastest), elements likewise,
    each with the RefHex vertex order (src/refdomain.cc:96-105).  With
    ``jitter`` > 0 every interior vertex coordinate is moved by an i.i.d.
    uniform offset in [-jitter*h, jitter*h] drawn from ``numpy.random.default_rng(seed)``
    (non-affine trilinear maps).  Boundary faces get markers 1..6
    (x=0, x=1, y=0, y=1, z=0, z=1).
    """
    nx = nx or n
    ny = ny or n
    nz = nz or n
    gx = np.linspace(0.0, 1.0, nx + 1)
    gy = np.linspace(0.0, 1.0, ny + 1)
    gz = np.linspace(0.0, 1.0, nz + 1)
    Z, Y, X = np.meshgrid(gz, gy, gx, indexing="ij")
    xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    if jitter:
        h = np.array([1.0 / nx, 1.0 / ny, 1.0 / nz])
        rng = np.random.default_rng(seed)
        d = rng.uniform(-1.0, 1.0, size=xyz.shape) * (jitter * h)
        K, J, I = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
        interior = ((I > 0) & (I < nx) & (J > 0) & (J < ny) & (K > 0) & (K < nz)).ravel()
        xyz[interior] += d[interior]

    def vid(i, j, k):
        return 1 + i + (nx + 1) * (j + (ny + 1) * k)

    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    hexes = np.stack([vid(i, j, k), vid(i + 1, j, k), vid(i + 1, j + 1, k), vid(i, j + 1, k),
                      vid(i, j, k + 1), vid(i + 1, j, k + 1), vid(i + 1, j + 1, k + 1), vid(i, j + 1, k + 1)], axis=1)
    bq, bm = [], []
    b, a = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
    a, b = a.ravel(), b.ravel()
    for x0, mk in ((0, 1), (nx, 2)):
        bq.append(np.stack([vid(x0, a, b), vid(x0, a + 1, b), vid(x0, a + 1, b + 1), vid(x0, a, b + 1)], 1))
        bm.append(np.full(len(a), mk))
    b, a = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    a, b = a.ravel(), b.ravel()
    for y0, mk in ((0, 3), (ny, 4)):
        bq.append(np.stack([vid(a, y0, b), vid(a + 1, y0, b), vid(a + 1, y0, b + 1), vid(a, y0, b + 1)], 1))
        bm.append(np.full(len(a), mk))
    b, a = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    a, b = a.ravel(), b.ravel()
    for z0, mk in ((0, 5), (nz, 6)):
        bq.append(np.stack([vid(a, b, z0), vid(a + 1, b, z0), vid(a + 1, b + 1, z0), vid(a, b + 1, z0)], 1))
        bm.append(np.full(len(a), mk))
    return Mesh().set_arrays(xyz, hexes, np.concatenate(bq), np.concatenate(bm))


def permute_vertices(mesh, seed=0, rotate=True):
    """Relabel vertex ids at random (and rotate each hex's local numbering by a
    random symmetry of the cube) so that edges and faces get every orientation.
    Returns a new (un-finalised) Mesh with the same geometry."""
    rng = np.random.default_rng(seed)
    nv = mesh.num_vertices
    perm = rng.permutation(nv)                  # new index of old vertex i
    inv = np.empty(nv, dtype=np.int64)
    inv[perm] = np.arange(nv)
    xyz = mesh.xyz[inv]
    hexes = perm[mesh.hexes - 1] + 1
    if rotate:
        syms = _cube_symmetries()
        choice = rng.integers(0, len(syms), size=len(hexes))
        hexes = np.stack([hexes[e][syms[c]] for e, c in enumerate(choice)])
    bq = perm[mesh.bquads - 1] + 1
    return Mesh().set_arrays(xyz, hexes, bq, mesh.bmarkers.copy())


def _cube_symmetries():
    """The 24 rotations of the reference hexahedron as vertex permutations."""
    ref = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                    [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]])
    out = []
    import itertools
    for p in itertools.permutations(range(3)):
        for s in itertools.product((1, -1), repeat=3):
            R = np.zeros((3, 3))
            for r in range(3):
                R[r, p[r]] = s[r]
            if np.linalg.det(R) < 0:
                continue
            img = ref @ R.T
            out.append([int(np.where((ref == v).all(1))[0][0]) for v in img])
    return out
