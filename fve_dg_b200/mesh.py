"""Flat tetrahedral meshes in the DGMesh layout (include/Mesh/MeshGenerator.h:46-57) and the
periodic box generator. A `Mesh` is what ExplicitConvection consumes, the way the reference's
ExplicitConvection::eval consumes a ComputingMesh (src/Mesh/ComputingMesh.cpp:268-298)."""
import ctypes

import numpy as np

from . import _lib as L

BC = {"Dirichlet": 0, "Neumann": 1, "Robin": 2, "Pseudo3DX": 3, "Pseudo3DY": 4, "Pseudo3DZ": 5,
      "Inflow": 6, "Outflow": 7, "Wall": 8, "WallTD": 9, "WallTN": 10, "WallTR": 11}


class Mesh:
    """Raw topology (form (b) of dg_mesh_desc), optionally with reference-held geometry (form (a))."""

    def __init__(self, points, cells, faces, face_cells, face_nodes1=None, periodic=None, bc=None,
                 cell_faces=None, cell_cells=None, geometry=None, nghost=0):
        self.points = L.as_f64(points).reshape(-1, 3)
        self.cells = L.as_i64(cells).reshape(-1, 4)
        self.faces = L.as_i64(faces).reshape(-1, 3)
        self.face_cells = L.as_i64(face_cells).reshape(-1, 2)
        self.face_nodes1 = None if face_nodes1 is None else L.as_i64(face_nodes1).reshape(-1, 3)
        self.periodic = None if periodic is None else L.as_u8(periodic)
        self.bc = None if bc is None else L.as_u8(bc)
        self.cell_faces = None if cell_faces is None else L.as_i64(cell_faces).reshape(-1, 4)
        self.cell_cells = None if cell_cells is None else L.as_i64(cell_cells).reshape(-1, 4)
        self.geometry = geometry  # dict(natural, normal, area, invjac, detj) or None
        self.nghost = int(nghost)  # the last nghost cells are ghost copies (dg_mesh_desc.nghost)

    @property
    def ncell(self):
        return self.cells.shape[0]

    @property
    def nface(self):
        return self.faces.shape[0]

    def desc(self):
        d = L.MeshDesc()
        d.ncell = self.ncell
        d.nface = self.nface
        d.face_cells = L.iptr(self.face_cells)
        d.face_bc = L.u8ptr(self.bc)
        if self.geometry is not None:
            g = self.geometry
            self._keep = [L.as_f64(g[k]) for k in ("natural", "normal", "area", "invjac", "detj")]
            d.face_natural, d.face_normal, d.face_area, d.cell_invjac, d.cell_detj = map(L.dptr, self._keep)
        d.npts = self.points.shape[0]
        d.points = L.dptr(self.points)
        d.cell_nodes = L.iptr(self.cells)
        d.face_nodes = L.iptr(self.faces)
        d.face_nodes1 = L.iptr(self.face_nodes1)
        d.face_periodic = L.u8ptr(self.periodic)
        d.nghost = self.nghost
        return d

    def compute_geometry(self):
        """Geometry with the reference's arithmetic (ComputingMesh.cpp:27-171), from topology."""
        nf, nc = self.nface, self.ncell
        out = dict(normal=np.zeros((nf, 3)), area=np.zeros(nf), natural=np.zeros((nf, 2, 3, 3)),
                   invjac=np.zeros((nc, 9)), detj=np.zeros(nc), centroid=np.zeros((nc, 3)))
        d = self.desc()
        L.check(L.lib().dg_mesh_geometry(ctypes.byref(d), L.dptr(out["normal"]), L.dptr(out["area"]),
                                         L.dptr(out["natural"]), L.dptr(out["invjac"]), L.dptr(out["detj"]),
                                         L.dptr(out["centroid"])), "dg_mesh_geometry")
        return out

    def face_perms(self):
        perm = np.zeros((self.nface, 2), dtype=np.int8)
        d = self.desc()
        L.check(L.lib().dg_face_perms(ctypes.byref(d), perm.ctypes.data_as(L.c_int8_p)), "dg_face_perms")
        return perm

    def cell_centroids(self):
        return self.points[self.cells].mean(axis=1)


def box_mesh(n, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), jitter=0.0, seed=20261203,
             periodic=(1, 1, 1), bc="Pseudo3DZ"):
    """n^3 cubes x 6 Kuhn tetrahedra on [lo, hi]^3; see dg_box_mesh_create in include/dg_gpu.h."""
    lib = L.lib()
    lo_a = (ctypes.c_double * 3)(*lo)
    hi_a = (ctypes.c_double * 3)(*hi)
    per = (ctypes.c_int * 3)(*[int(p) for p in periodic])
    err = ctypes.c_int(0)
    bcv = BC[bc] if isinstance(bc, str) else int(bc)
    h = lib.dg_box_mesh_create(int(n), lo_a, hi_a, float(jitter), int(seed), per, bcv, ctypes.byref(err))
    if not h:
        raise L.DGError(err.value, "dg_box_mesh_create")
    try:
        d = L.MeshDesc()
        cf = L.c_int64_p()
        cc = L.c_int64_p()
        L.check(lib.dg_box_mesh_view(h, ctypes.byref(d), ctypes.byref(cf), ctypes.byref(cc)), "dg_box_mesh_view")
        nc, nf, npn = d.ncell, d.nface, d.npts

        def arr(p, n_, dt):
            return np.ctypeslib.as_array(p, shape=(n_,)).astype(dt, copy=True)

        m = Mesh(points=arr(d.points, 3 * npn, np.float64), cells=arr(d.cell_nodes, 4 * nc, np.int64),
                 faces=arr(d.face_nodes, 3 * nf, np.int64), face_cells=arr(d.face_cells, 2 * nf, np.int64),
                 face_nodes1=arr(d.face_nodes1, 3 * nf, np.int64), periodic=arr(d.face_periodic, nf, np.uint8),
                 bc=arr(d.face_bc, nf, np.uint8), cell_faces=arr(cf, 4 * nc, np.int64),
                 cell_cells=arr(cc, 4 * nc, np.int64))
    finally:
        lib.dg_box_mesh_destroy(h)
    m.n = int(n)
    m.lo = tuple(float(x) for x in lo)
    m.hi = tuple(float(x) for x in hi)
    return m
