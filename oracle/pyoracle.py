"""Test infrastructure (oracle): ctypes bindings of the two CPU checkers.

  Oracle  -- oracle/liboracle.so, the plain-C restatement (dg_oracle.c)
  RefLib  -- oracle/_ref/libfvedg_ref.so, the reference's own ExplicitConvection compiled from
             source with ref_harness.cpp (absent when the reference was not available at build)

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs import this.
Meshes are passed as plain numpy arrays in the DGMesh layout.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfvedg_ref.so")

dp = ctypes.POINTER(ctypes.c_double)
i64p = ctypes.POINTER(ctypes.c_int64)
u64p = ctypes.POINTER(ctypes.c_uint64)
u8p = ctypes.POINTER(ctypes.c_uint8)

FLUX = {"LF": 0, "Roe": 1}


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(dp)


def nb_of(order):
    return (order + 1) * (order + 2) * (order + 3) // 6


class _OrcMesh(ctypes.Structure):
    _fields_ = [("npts", ctypes.c_int64), ("pts", dp), ("ncell", ctypes.c_int64), ("cells", i64p),
                ("nface", ctypes.c_int64), ("faces", i64p), ("face_cells", i64p), ("face_nodes1", i64p),
                ("periodic", u8p), ("bc", u8p)]


class Oracle:
    """C restatement of ExplicitConvection::eval + SSP-RK3 (single-threaded)."""

    def __init__(self, points, cells, faces, face_cells, face_nodes1=None, periodic=None, bc=None):
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle)")
        self.L = ctypes.CDLL(ORACLE_SO)
        self._arrs = [np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3),
                      np.ascontiguousarray(cells, dtype=np.int64).reshape(-1, 4),
                      np.ascontiguousarray(faces, dtype=np.int64).reshape(-1, 3),
                      np.ascontiguousarray(face_cells, dtype=np.int64).reshape(-1, 2)]
        fn1 = self._arrs[2] if face_nodes1 is None else np.ascontiguousarray(face_nodes1, dtype=np.int64).reshape(-1, 3)
        per = None if periodic is None else np.ascontiguousarray(periodic, dtype=np.uint8)
        bcs = None if bc is None else np.ascontiguousarray(bc, dtype=np.uint8)
        self._arrs += [fn1, per, bcs]
        p, c, f, fc = self._arrs[:4]
        self.m = _OrcMesh(p.shape[0], p.ctypes.data_as(dp), c.shape[0], c.ctypes.data_as(i64p), f.shape[0],
                          f.ctypes.data_as(i64p), fc.ctypes.data_as(i64p), fn1.ctypes.data_as(i64p),
                          None if per is None else per.ctypes.data_as(u8p),
                          None if bcs is None else bcs.ctypes.data_as(u8p))
        self.ncell, self.nface = c.shape[0], f.shape[0]
        mp = ctypes.POINTER(_OrcMesh)
        L = self.L
        L.orc_residual.argtypes = [mp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   dp, dp, ctypes.c_double, dp, ctypes.c_int]
        L.orc_mass.argtypes = [mp, ctypes.c_int, ctypes.c_int, dp]
        L.orc_ssprk3.argtypes = [mp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp,
                                 ctypes.c_double, ctypes.c_int, ctypes.c_double, dp]
        L.orc_geometry.argtypes = [mp, dp, dp, dp, dp, dp, dp]
        L.orc_conservation.argtypes = [mp, ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp]
        L.orc_basis.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]

    @classmethod
    def from_mesh(cls, m):
        return cls(m.points, m.cells, m.faces, m.face_cells, m.face_nodes1, m.periodic, m.bc)

    def residual(self, U, order, qv, qf, gamma=1.4, flux="LF", t=0.0, dirichlet=None, part=0):
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.zeros_like(U)
        dd = None if dirichlet is None else np.ascontiguousarray(dirichlet, dtype=np.float64)
        rc = self.L.orc_residual(ctypes.byref(self.m), order, gamma, FLUX[flux], qv, qf, U.ctypes.data_as(dp),
                                 R.ctypes.data_as(dp), t, _d(dd), part)
        if rc != 0:
            raise RuntimeError(f"orc_residual failed: {rc}")
        return R

    def mass(self, order, qv):
        b = np.zeros((self.ncell, 5 * nb_of(order)))
        self.L.orc_mass(ctypes.byref(self.m), order, qv, b.ctypes.data_as(dp))
        return b

    def ssprk3(self, U, order, qv, qf, dt, nsteps, gamma=1.4, flux="LF", t0=0.0, dirichlet=None):
        U = np.array(U, dtype=np.float64, copy=True)
        b = self.mass(order, qv)
        dd = None if dirichlet is None else np.ascontiguousarray(dirichlet, dtype=np.float64)
        rc = self.L.orc_ssprk3(ctypes.byref(self.m), order, gamma, FLUX[flux], qv, qf, U.ctypes.data_as(dp),
                               b.ctypes.data_as(dp), dt, nsteps, t0, _d(dd))
        if rc != 0:
            raise RuntimeError(f"orc_ssprk3 failed: {rc}")
        return U

    def geometry(self):
        nf, nc = self.nface, self.ncell
        out = dict(normal=np.zeros((nf, 3)), area=np.zeros(nf), natural=np.zeros((nf, 2, 3, 3)),
                   invjac=np.zeros((nc, 9)), detj=np.zeros(nc), centroid=np.zeros((nc, 3)))
        self.L.orc_geometry(ctypes.byref(self.m), *[out[k].ctypes.data_as(dp) for k in
                                                    ("normal", "area", "natural", "invjac", "detj", "centroid")])
        return out

    def conservation(self, U, order, qv, gamma=1.4):
        out = np.zeros(6)
        U = np.ascontiguousarray(U, dtype=np.float64)
        self.L.orc_conservation(ctypes.byref(self.m), order, qv, gamma, U.ctypes.data_as(dp), out.ctypes.data_as(dp))
        return out

    def basis(self, order, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        nb = nb_of(order)
        phi = np.zeros((xyz.shape[0], nb))
        grad = np.zeros((xyz.shape[0], nb, 3))
        self.L.orc_basis(order, xyz.shape[0], xyz.ctypes.data_as(dp), phi.ctypes.data_as(dp), grad.ctypes.data_as(dp))
        return phi, grad


def ref_available():
    return os.path.exists(REF_SO)


class RefLib:
    """The reference's own operator (ComputingMesh(DGMesh) + ExplicitConvection<...>)."""

    def __init__(self):
        if not os.path.exists(REF_SO):
            raise RuntimeError("oracle/_ref/libfvedg_ref.so is not built (make -C oracle ref)")
        L = ctypes.CDLL(REF_SO)
        L.fveref_mesh_create.restype = ctypes.c_void_p
        L.fveref_mesh_create.argtypes = [ctypes.c_uint64, dp, ctypes.c_uint64, u64p, u64p, u64p, ctypes.c_uint64,
                                         u64p, u64p, u8p, u64p, u64p]
        L.fveref_mesh_destroy.argtypes = [ctypes.c_void_p]
        L.fveref_mesh_export.argtypes = [ctypes.c_void_p, dp, dp, dp, u64p, dp, dp, dp]
        L.fveref_eval.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp,
                                  ctypes.c_double, ctypes.c_int]
        L.fveref_ssprk3.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_double]
        L.fveref_mass.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
        L.fveref_diffusion.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_double]
        L.fveref_limit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_int]
        L.fveref_quad_tet.argtypes = [ctypes.c_int, dp, dp]
        L.fveref_quad_tri.argtypes = [ctypes.c_int, dp, dp]
        L.fveref_basis.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
        L.fveref_block_bytes.restype = ctypes.c_size_t
        L.fveref_block_bytes.argtypes = [ctypes.c_int]
        L.fveref_set_dirichlet.argtypes = [dp]
        L.fveref_set_threads.argtypes = [ctypes.c_int]
        L.fveref_box_create.restype = ctypes.c_void_p
        L.fveref_box_create.argtypes = [ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_uint64,
                                        ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.fveref_orthhex_create.restype = ctypes.c_void_p
        L.fveref_orthhex_create.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int]
        L.fveref_mesh_sizes.argtypes = [ctypes.c_void_p, u64p]
        L.fveref_mesh_topology.argtypes = [ctypes.c_void_p, dp, u64p, u64p, u64p, u64p, u64p, u64p, u8p, u8p]
        L.fveref_project.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp, dp]
        self.L = L

    def set_threads(self, n):
        self.L.fveref_set_threads(int(n))

    def threads(self):
        return int(self.L.fveref_get_threads())

    def phy_cpu(self):
        return int(self.L.fveref_phy_cpu())

    def quad(self, kind, rid):
        f = self.L.fveref_quad_tet if kind == 0 else self.L.fveref_quad_tri
        n = f(rid, None, None)
        pts = np.zeros((n, 3 if kind == 0 else 2))
        w = np.zeros(n)
        f(rid, pts.ctypes.data_as(dp), w.ctypes.data_as(dp))
        return pts, w

    def basis(self, order, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        nb = nb_of(order)
        phi = np.zeros((xyz.shape[0], nb))
        grad = np.zeros((xyz.shape[0], nb, 3))
        self.L.fveref_basis(order, xyz.shape[0], xyz.ctypes.data_as(dp), phi.ctypes.data_as(dp), grad.ctypes.data_as(dp))
        return phi, grad

    def block_bytes(self, order):
        return int(self.L.fveref_block_bytes(order))

    def set_dirichlet(self, params10):
        self.L.fveref_set_dirichlet(np.ascontiguousarray(params10, dtype=np.float64).ctypes.data_as(dp))

    def mesh(self, points, cells, faces, face_cells, cell_faces, cell_cells, face_nodes1=None, periodic=None, bc=None):
        return RefMesh(self, points, cells, faces, face_cells, cell_faces, cell_cells, face_nodes1, periodic, bc)

    def box(self, n, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), jitter=0.0, seed=20261203, periodic=(1, 1, 1), bc=5):
        """The periodic Kuhn box made by the oracle itself (ref_harness.cpp build_box), as a reference
        ComputingMesh; same mesh as the product's box_mesh with the same arguments."""
        lo_a, hi_a = np.array(lo, dtype=np.float64), np.array(hi, dtype=np.float64)
        per = (ctypes.c_int * 3)(*[int(p) for p in periodic])
        h = self.L.fveref_box_create(int(n), lo_a.ctypes.data_as(dp), hi_a.ctypes.data_as(dp), float(jitter),
                                     int(seed), per, int(bc))
        if not h:
            raise RuntimeError("fveref_box_create failed")
        return RefMesh.from_handle(self, h)

    def orthhex(self, n, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), bc_z=5, bc_side=0):
        """The reference's own mesh route OrthHexMesh -> split_hex6_scan -> ComputingMesh(GeneralMesh)
        (ref_harness.cpp build_orthhex): n^3 hexahedra, boundary faces with |n_z| > 0.5 typed bc_z, the
        others bc_side."""
        lo_a, hi_a = np.array(lo, dtype=np.float64), np.array(hi, dtype=np.float64)
        h = self.L.fveref_orthhex_create(int(n), lo_a.ctypes.data_as(dp), hi_a.ctypes.data_as(dp), int(bc_z),
                                         int(bc_side))
        if not h:
            raise RuntimeError("fveref_orthhex_create failed")
        return RefMesh.from_handle(self, h)


class RefMesh:
    def __init__(self, ref, points, cells, faces, face_cells, cell_faces, cell_cells, face_nodes1, periodic, bc):
        self.ref = ref
        U64 = np.uint64
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        c = np.ascontiguousarray(cells, dtype=np.int64).astype(U64).reshape(-1, 4)
        f = np.ascontiguousarray(faces, dtype=np.int64).astype(U64).reshape(-1, 3)
        fc = np.ascontiguousarray(face_cells, dtype=np.int64).reshape(-1, 2).copy()
        per = np.zeros(f.shape[0], dtype=np.uint8) if periodic is None else np.ascontiguousarray(periodic, dtype=np.uint8)
        pcell = np.full(f.shape[0], np.iinfo(np.uint64).max, dtype=U64)
        pnodes = f.copy() if face_nodes1 is None else np.ascontiguousarray(face_nodes1, dtype=np.int64).astype(U64).reshape(-1, 3)
        mask = per.astype(bool)
        pcell[mask] = fc[mask, 1].astype(U64)
        fcu = fc.astype(U64)  # -1 becomes uInt(-1)
        cf = np.ascontiguousarray(cell_faces, dtype=np.int64).astype(U64).reshape(-1, 4)
        cc = np.ascontiguousarray(cell_cells, dtype=np.int64).astype(U64).reshape(-1, 4)
        bcs = None if bc is None else np.ascontiguousarray(bc, dtype=np.uint8)
        self._keep = [pts, c, f, fcu, cf, cc, pcell, pnodes, bcs]
        self.ncell, self.nface = c.shape[0], f.shape[0]
        self.h = ref.L.fveref_mesh_create(pts.shape[0], pts.ctypes.data_as(dp), c.shape[0], c.ctypes.data_as(u64p),
                                          cf.ctypes.data_as(u64p), cc.ctypes.data_as(u64p), f.shape[0],
                                          f.ctypes.data_as(u64p), fcu.ctypes.data_as(u64p),
                                          None if bcs is None else bcs.ctypes.data_as(u8p),
                                          pcell.ctypes.data_as(u64p), pnodes.ctypes.data_as(u64p))

    @classmethod
    def from_mesh(cls, ref, m):
        return cls(ref, m.points, m.cells, m.faces, m.face_cells, m.cell_faces, m.cell_cells, m.face_nodes1,
                   m.periodic, m.bc)

    @classmethod
    def from_handle(cls, ref, h):
        """A mesh the harness built itself; its flat topology is exported into numpy arrays (int64, -1 for
        a missing neighbour) with the attribute names of the product's Mesh."""
        self = cls.__new__(cls)
        self.ref, self.h, self._keep = ref, h, []
        sz = np.zeros(3, dtype=np.uint64)
        if ref.L.fveref_mesh_sizes(h, sz.ctypes.data_as(u64p)) != 0:
            raise RuntimeError("fveref_mesh_sizes failed")
        npts, nc, nf = (int(v) for v in sz)
        self.ncell, self.nface = nc, nf
        U64 = np.uint64
        pts = np.zeros((npts, 3))
        cells, cf, cc = (np.zeros((nc, 4), dtype=U64) for _ in range(3))
        faces, fn1 = np.zeros((nf, 3), dtype=U64), np.zeros((nf, 3), dtype=U64)
        fc = np.zeros((nf, 2), dtype=U64)
        per, bc = np.zeros(nf, dtype=np.uint8), np.zeros(nf, dtype=np.uint8)
        ref.L.fveref_mesh_topology(h, pts.ctypes.data_as(dp), *[a.ctypes.data_as(u64p) for a in (cells, cf, cc, faces,
                                                                                                  fc, fn1)],
                                   per.ctypes.data_as(u8p), bc.ctypes.data_as(u8p))
        self.points = pts
        self.cells, self.cell_faces, self.cell_cells = (a.astype(np.int64) for a in (cells, cf, cc))
        self.faces, self.face_cells, self.face_nodes1 = (a.astype(np.int64) for a in (faces, fc, fn1))
        self.periodic, self.bc = per, bc
        return self

    PROBLEMS = {"vortex": 0, "density_wave": 1, "taylor_green": 2}

    def project(self, order, problem, params):
        """Initial coefficients by the reference's DGBasisEvaluator<P>::func2coef, per cell (ref_harness.cpp
        run_project): problem 'vortex' params (cx,cy,cz, ax,ay,az, beta, gamma, ux,uy,uz, period or 0),
        'density_wave' (A, kx,ky,kz, ux,uy,uz, p, gamma), 'taylor_green' (Mach, gamma)."""
        U = np.zeros((self.ncell, 5 * nb_of(order)))
        prm = np.ascontiguousarray(params, dtype=np.float64)
        rc = self.ref.L.fveref_project(self.h, order, self.PROBLEMS[problem], prm.ctypes.data_as(dp),
                                       U.ctypes.data_as(dp))
        if rc != 0:
            raise RuntimeError(f"fveref_project rc={rc}")
        return U

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.L.fveref_mesh_destroy(self.h)
            self.h = None

    def export(self):
        nf, nc = self.nface, self.ncell
        out = dict(normal=np.zeros((nf, 3)), area=np.zeros(nf), natural=np.zeros((nf, 2, 3, 3)),
                   face_cells=np.zeros((nf, 2), dtype=np.uint64), invjac=np.zeros((nc, 9)), detj=np.zeros(nc),
                   centroid=np.zeros((nc, 3)))
        self.ref.L.fveref_mesh_export(self.h, out["normal"].ctypes.data_as(dp), out["area"].ctypes.data_as(dp),
                                      out["natural"].ctypes.data_as(dp), out["face_cells"].ctypes.data_as(u64p),
                                      out["invjac"].ctypes.data_as(dp), out["detj"].ctypes.data_as(dp),
                                      out["centroid"].ctypes.data_as(dp))
        fc = out["face_cells"].astype(np.int64)  # uInt(-1) -> -1
        out["face_cells"] = fc
        return out

    def eval(self, U, order, qv, qf, gamma_id=0, t=0.0, part=0):
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.zeros_like(U)
        rc = self.ref.L.fveref_eval(self.h, order, gamma_id, qv, qf, U.ctypes.data_as(dp), R.ctypes.data_as(dp), t, part)
        if rc != 0:
            raise RuntimeError(f"fveref_eval: no instantiation for P{order} rules ({qv},{qf}) rc={rc}")
        return R

    def mass(self, order, qv):
        b = np.zeros((self.ncell, 5 * nb_of(order)))
        rc = self.ref.L.fveref_mass(self.h, order, qv, b.ctypes.data_as(dp))
        if rc != 0:
            raise RuntimeError(f"fveref_mass rc={rc}")
        return b

    def diffusion(self, U, order, qv, qf, t=0.0):
        """ExplicitDiffusion<P, QC, QF>::eval(mesh, U, t)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.zeros_like(U)
        rc = self.ref.L.fveref_diffusion(self.h, order, qv, qf, U.ctypes.data_as(dp), R.ctypes.data_as(dp), t)
        if rc != 0:
            raise RuntimeError(f"fveref_diffusion rc={rc}")
        return R

    def limit(self, U, Uprev, order, qv, gamma=1.4, only_avg=False):
        """PositiveLimiter<P, QC, only_avg>: constructMinMax(U, Uprev) then apply(U, Uprev)."""
        U = np.array(U, dtype=np.float64, copy=True)
        Uprev = np.ascontiguousarray(Uprev, dtype=np.float64)
        rc = self.ref.L.fveref_limit(self.h, order, qv, U.ctypes.data_as(dp), Uprev.ctypes.data_as(dp), gamma,
                                     int(only_avg))
        if rc != 0:
            raise RuntimeError(f"fveref_limit rc={rc}")
        return U

    def ssprk3(self, U, mass, order, qv, qf, dt, nsteps, gamma_id=0, t0=0.0):
        U = np.array(U, dtype=np.float64, copy=True)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        rc = self.ref.L.fveref_ssprk3(self.h, order, gamma_id, qv, qf, U.ctypes.data_as(dp), mass.ctypes.data_as(dp),
                                      dt, nsteps, t0)
        if rc != 0:
            raise RuntimeError(f"fveref_ssprk3 rc={rc}")
        return U
