"""CPU: pin the oracle (and the product's host tables/geometry) against the reference.

Fixtures under tests/golden/ are outputs of the reference's own ExplicitConvection::eval and
ComputingMesh (tests/golden/make_golden.py). When oracle/_ref is built, the same checks also run
live against the reference on fresh meshes."""
import glob
import os

import numpy as np
import pytest

from conftest import CASES, rel_l2
from fve_dg_b200 import Mesh, box_mesh, problems
from oracle.pyoracle import Oracle, RefLib, RefMesh, ref_available

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def mesh_from(z):
    return Mesh(z["mesh_points"], z["mesh_cells"], z["mesh_faces"], z["mesh_face_cells"], z["mesh_face_nodes1"],
                z["mesh_periodic"], z["mesh_bc"], z["mesh_cell_faces"], z["mesh_cell_cells"])


def cases_of(z):
    out = []
    for k in z:
        if k.startswith("U_P"):
            P, qv, qf = k[3:].split("_")
            out.append((int(P), int(qv), int(qf)))
    return out


def test_fixtures_present():
    assert len(FILES) >= 3


@pytest.mark.parametrize("path", FILES, ids=os.path.basename)
def test_oracle_residual_matches_golden(path):
    z = load(path)
    m = mesh_from(z)
    o = Oracle.from_mesh(m)
    for (P, qv, qf) in cases_of(z):
        R = o.residual(z[f"U_P{P}_{qv}_{qf}"], P, qv, qf, dirichlet=z.get("dirichlet"))
        assert rel_l2(R, z[f"R_P{P}_{qv}_{qf}"]) < 1e-12, (P, qv, qf)


@pytest.mark.parametrize("path", FILES, ids=os.path.basename)
def test_geometry_matches_golden(path):
    """Connectivity, face maps and orientation bit-exact; normals/areas/J^-T to a few ulp."""
    z = load(path)
    m = mesh_from(z)
    for g in (m.compute_geometry(), Oracle.from_mesh(m).geometry()):
        assert np.array_equal(g["natural"], z["geo_natural"])
        assert np.array_equal(z["geo_face_cells"], m.face_cells)
        assert np.all((g["normal"] * z["geo_normal"]).sum(axis=1) > 0.999)  # same orientation
        assert np.abs(g["normal"] - z["geo_normal"]).max() <= 4 * np.finfo(float).eps
        assert np.abs(g["area"] - z["geo_area"]).max() <= 4 * np.finfo(float).eps * z["geo_area"].max()
        assert np.abs(g["detj"] - z["geo_detj"]).max() <= 4 * np.finfo(float).eps * z["geo_detj"].max()
        assert np.abs(g["invjac"] - z["geo_invjac"]).max() <= 8 * np.finfo(float).eps * np.abs(z["geo_invjac"]).max()


def test_box_mesh_is_reproducible():
    """The generator (seeded mt19937_64 jitter) reproduces the fixture meshes exactly."""
    specs = {"periodic_n2.npz": dict(n=2, jitter=0.1, seed=11),
             "dirichlet_n2.npz": dict(n=2, jitter=0.1, seed=12, periodic=(0, 0, 0), bc="Dirichlet"),
             "pseudo3dz_n2.npz": dict(n=2, jitter=0.1, seed=13, periodic=(1, 1, 0), bc="Pseudo3DZ")}
    for name, kw in specs.items():
        z = load(os.path.join(GOLDEN, name))
        m = box_mesh(**kw)
        for k in ("points", "cells", "faces", "face_cells", "face_nodes1", "periodic", "bc", "cell_faces",
                  "cell_cells"):
            assert np.array_equal(getattr(m, k).reshape(z["mesh_" + k].shape), z["mesh_" + k]), (name, k)


def test_basis_matches_golden():
    z = load(os.path.join(GOLDEN, "periodic_n2.npz"))
    pts = z["basisq_pts"]
    m = mesh_from(z)
    o = Oracle.from_mesh(m)
    for P in (1, 2, 3, 4):
        for phi, grad in (problems.basis(P, pts), o.basis(P, pts)):
            scale = np.abs(z[f"basisq_P{P}_phi"]).max()
            assert np.abs(phi - z[f"basisq_P{P}_phi"]).max() <= 1e-14 * scale
            gs = np.abs(z[f"basisq_P{P}_grad"]).max()
            assert np.abs(grad - z[f"basisq_P{P}_grad"]).max() <= 1e-14 * gs


def test_basis_is_orthogonal():
    """The reference basis is orthogonal on the reference tet (diagonal mass)."""
    pts, w = problems.quad_rule(0, 6)  # degree 9: exact for P4 products
    phi, _ = problems.basis(4, pts)
    M = (phi * w[:, None]).T @ phi
    off = M - np.diag(np.diag(M))
    assert np.abs(off).max() < 1e-14 * np.abs(np.diag(M)).max()


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
@pytest.mark.parametrize("P,qv,qf", CASES)
def test_oracle_matches_reference_live(P, qv, qf):
    m = box_mesh(3, jitter=0.1, seed=100 + P)
    U = problems.project(m, P, problems.taylor_green())
    U = U + 1e-2 * np.random.default_rng(P).standard_normal(U.shape)
    rm = RefMesh.from_mesh(RefLib(), m)
    o = Oracle.from_mesh(m)
    assert rel_l2(o.residual(U, P, qv, qf), rm.eval(U, P, qv, qf)) < 1e-12
    for part in (1, 2):
        assert rel_l2(o.residual(U, P, qv, qf, part=part), rm.eval(U, P, qv, qf, part=part)) < 1e-12


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
def test_oracle_rk_and_mass_match_reference_live():
    m = box_mesh(2, jitter=0.1, seed=7)
    P, qv, qf = 2, 1, 2
    U = problems.project(m, P, problems.isentropic_vortex(center=(0.5, 0.5, 0.5), beta=1.0))
    rm = RefMesh.from_mesh(RefLib(), m)
    o = Oracle.from_mesh(m)
    b_ref = rm.mass(P, qv)
    assert rel_l2(o.mass(P, qv), b_ref) < 1e-14
    Ur = rm.ssprk3(U, b_ref, P, qv, qf, 1e-3, 2)
    Uo = o.ssprk3(U, P, qv, qf, 1e-3, 2)
    assert rel_l2(Uo, Ur) < 1e-13


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
def test_reference_padded_block_size():
    """LongVector pads each block to 32 bytes (DenseMatrix alignas(32)): P1..P4 strides."""
    ref = RefLib()
    assert [ref.block_bytes(P) for P in (1, 2, 3, 4)] == [160, 416, 800, 1408]
    assert [ref.block_bytes(P) for P in (0, 5)] == [64, 2240]


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
def test_quadrature_tables_are_the_references_bit_for_bit():
    """Every rule of quad_tables.inc, the P5 Auto rules (Degree11Points94, Degree13Points36)
    included, equals the reference's own points and weights exactly."""
    ref = RefLib()
    for kind, nrules in ((0, 8), (1, 5)):
        for rid in range(nrules):
            p_ref, w_ref = ref.quad(kind, rid)
            p, w = problems.quad_rule(kind, rid)
            assert np.array_equal(p, p_ref) and np.array_equal(w, w_ref), (kind, rid)
    assert problems.auto_rules(0) == (2, 2) and problems.auto_rules(5) == (7, 4)


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
@pytest.mark.parametrize("P", [0, 5])
def test_orders_0_and_5_match_reference_live(P):
    """P0 (finite volume) and P5, the other orders ExplicitConvection.cpp:5-16 instantiates, with
    the reference's Auto rules: basis values and gradients, and the oracle's residual against the
    reference's eval."""
    qv, qf = problems.auto_rules(P)
    m = box_mesh(3, jitter=0.1, seed=200 + P)
    ref = RefLib()
    pts, _ = problems.quad_rule(0, qv)
    phi_r, grad_r = ref.basis(P, pts)
    phi, grad = problems.basis(P, pts)
    assert np.abs(phi - phi_r).max() <= 1e-13 * np.abs(phi_r).max()
    assert np.abs(grad - grad_r).max() <= 1e-13 * max(np.abs(grad_r).max(), 1.0)
    U = problems.project(m, P, problems.taylor_green())
    U = U + 1e-2 * np.random.default_rng(P).standard_normal(U.shape)
    rm = RefMesh.from_mesh(ref, m)
    o = Oracle.from_mesh(m)
    assert rel_l2(o.residual(U, P, qv, qf), rm.eval(U, P, qv, qf)) < 1e-12
    b = rm.mass(P, qv)
    assert rel_l2(o.mass(P, qv), b) < 1e-14
    U0 = problems.project(m, P, problems.density_wave())
    assert rel_l2(o.ssprk3(U0, P, qv, qf, 1e-3, 2), rm.ssprk3(U0, b, P, qv, qf, 1e-3, 2)) < 1e-13
