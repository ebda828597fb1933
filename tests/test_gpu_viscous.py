"""GPU: the explicit viscous operator against the reference's own ExplicitDiffusion<P, QC, QF>::eval
(include/DG/DG_Schemes/ExplicitDiffusion.h:133-626), compiled from source into oracle/_ref."""
import numpy as np
import pytest

from conftest import CASES, rel_l2
from fve_dg_b200 import ExplicitConvection, box_mesh, problems
from oracle.pyoracle import RefLib, RefMesh, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference library not built")]

TOL = 1e-12  # relative L2, the FP64 parity bar


def state(m, P, seed, amp=1e-2):
    U = problems.project(m, P, problems.density_wave(A=0.3))
    return U + amp * np.random.default_rng(seed).standard_normal(U.shape) * np.abs(U).max()


@pytest.fixture(scope="module")
def mesh3():
    return box_mesh(3, jitter=0.1, seed=5)


@pytest.mark.parametrize("P,qv,qf", CASES)
def test_viscous_matches_reference(mesh3, P, qv, qf):
    U = state(mesh3, P, 40 + P)
    Rr = RefMesh.from_mesh(RefLib(), mesh3).diffusion(U, P, qv, qf)
    conv = ExplicitConvection(mesh3, order=P, quad_vol=qv, quad_face=qf)
    R = conv.viscous_eval(U)
    assert np.abs(Rr).max() > 0
    assert rel_l2(R, Rr) < TOL, rel_l2(R, Rr)


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_viscous_boundary_faces(P):
    """Non-periodic box: Dirichlet on all sides, then Pseudo3DZ, then a type that contributes nothing."""
    from test_gpu_parity import face_points_physical
    qv, qf = problems.auto_rules(P)
    prm = np.array([1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 0.5, 0.25, 1.0, 1.4])
    for bc in ("Dirichlet", "Pseudo3DZ", "Wall"):
        m = box_mesh(2, jitter=0.1, seed=3, periodic=(0, 0, 0), bc=bc)
        U = state(m, P, 50 + P, amp=1e-3)
        conv = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf)
        if bc == "Dirichlet":
            X = face_points_physical(m, qf)
            conv.set_dirichlet(problems.density_wave(A=prm[1], vel=tuple(prm[5:8]))(X))
        ref = RefLib()
        ref.set_dirichlet(prm)
        Rr = RefMesh.from_mesh(ref, m).diffusion(U, P, qv, qf)
        assert rel_l2(conv.viscous_eval(U), Rr) < TOL, bc


def test_viscous_properties(mesh3):
    P, qv, qf = 3, 3, 3
    conv = ExplicitConvection(mesh3, order=P, quad_vol=qv, quad_face=qf)
    U = state(mesh3, P, 7)
    R1 = conv.viscous_eval(U)
    assert np.allclose(conv.viscous_eval(U, mu=2.5), 2.5 * R1, rtol=1e-13, atol=1e-13 * np.abs(R1).max())
    # uniform flow: no gradients and no jumps, so no viscous residual
    C = np.zeros_like(U)
    C[:, :5] = [1.2, 0.3, -0.2, 0.1, 3.0]
    assert np.abs(conv.viscous_eval(C)).max() < 1e-12
    # the mass equation carries no viscous term
    assert np.abs(R1[:, 0::5]).max() == 0.0
