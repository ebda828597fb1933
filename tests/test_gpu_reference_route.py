"""GPU: the CUDA path on the reference's own mesh route, and configuration 1 exactly as stated.

- OrthHexMesh -> split_hex6_scan -> rebuild_cell_topology -> ComputingMesh(const GeneralMesh&)
  (include/Mesh/OrthHexMesh.h:7-106, src/Mesh/GeneralMesh.cpp:4-129, src/Mesh/ComputingMesh.cpp:205-263),
  the route the reference's drivers take (examples/Vortex/123/Vortex.cpp:101-106): node orders from
  unordered_set iteration, the split's own face numbering, Pseudo3DZ on the z faces and Dirichlet on
  the side faces. The product is given this mesh as raw topology (geometry computed by the library)
  and as the reference's geometry (form (a)); residuals and parts against ExplicitConvection::eval,
  P1..P4, and SSP-RK3 steps against the reference's LongVector loop.
- Configuration 1: periodic [0,10]^3 as 8^3x6 = 3,072 tets, isentropic vortex (strength 5, z axis
  through (5,5,5), free stream rho 1, u (1,1,0), p 1), P1, Degree2Points4 / Degree3Points6, LF,
  SSP-RK3 at CFL 0.3 for 20 FP64 steps, each step against the reference's own loop.
"""
import numpy as np
import pytest

from conftest import rel_l2
from fve_dg_b200 import ExplicitConvection, Mesh, box_mesh, problems
from oracle.pyoracle import Oracle, RefLib, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference library not built")]

TOL = 1e-12
DW = np.array([1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 0.5, 0.25, 1.0, 1.4])  # the harness's Dirichlet density wave


def face_points_physical(m, qf):
    pts, _ = problems.quad_rule(1, qf)
    P = m.points[m.faces]
    lam = np.stack([1 - pts[:, 0] - pts[:, 1], pts[:, 0], pts[:, 1]], axis=1)
    return np.einsum("ga,fad->fgd", lam, P)


def route_meshes(rm):
    """The reference mesh as raw topology (form (b)) and with the reference's geometry (form (a))."""
    mb = Mesh(rm.points, rm.cells, rm.faces, rm.face_cells, bc=rm.bc)
    g = rm.export()
    ma = Mesh(rm.points, rm.cells, rm.faces, rm.face_cells, bc=rm.bc,
              geometry=dict(natural=g["natural"], normal=g["normal"], area=g["area"], invjac=g["invjac"],
                            detj=g["detj"]))
    return mb, ma


@pytest.mark.parametrize("P,qv,qf", [(1, 0, 1), (2, 1, 2), (3, 3, 3), (4, 5, 3), (3, 4, 3)])
@pytest.mark.parametrize("flux", ["LF", "Roe"])
def test_residual_on_reference_mesh_route(P, qv, qf, flux):
    ref = RefLib()
    ref.set_dirichlet(DW)
    rm = ref.orthhex(3, hi=(1.0, 1.0, 0.5), bc_z=5, bc_side=0)
    U = rm.project(P, "density_wave", [0.2, 1.0, 1.0, 1.0, 1.0, 0.5, 0.25, 1.0, 1.4])
    U = U + 1e-3 * np.random.default_rng(P).standard_normal(U.shape) * np.abs(U).max()
    parts = [rm.eval(U, P, qv, qf, part=k) for k in range(4)] if flux == "LF" else None
    for m in route_meshes(rm):
        conv = ExplicitConvection(m, order=P, flux=flux, quad_vol=qv, quad_face=qf)
        X = face_points_physical(m, qf)
        conv.set_dirichlet(problems.density_wave(A=DW[1], vel=tuple(DW[5:8]))(X))
        if flux == "LF":
            assert rel_l2(conv.eval(U), parts[0]) < TOL
            assert rel_l2(conv.eval_cells(U), parts[1]) < TOL
            assert rel_l2(conv.eval_internals(U), parts[2]) < TOL
            assert rel_l2(conv.eval_boundarys(U), parts[3]) < TOL
        else:  # the reference has no Roe solver: against the C restatement on the same mesh
            Ro = Oracle(rm.points, rm.cells, rm.faces, rm.face_cells, bc=rm.bc).residual(
                U, P, qv, qf, flux="Roe", dirichlet=DW)
            assert rel_l2(conv.eval(U), Ro) < TOL
        conv.close()


@pytest.mark.parametrize("P,qv,qf", [(1, 0, 1), (2, 1, 2), (3, 3, 3)])
def test_ssprk3_on_reference_mesh_route(P, qv, qf):
    ref = RefLib()
    rm = ref.orthhex(3, hi=(1.0, 1.0, 0.5), bc_z=5, bc_side=5)  # Pseudo3DZ everywhere: no time-dependent data
    U0 = rm.project(P, "density_wave", [0.2, 1.0, 1.0, 1.0, 1.0, 0.5, 0.25, 1.0, 1.4])
    b = rm.mass(P, qv)
    dt, n = 1e-3, 4
    Ur = rm.ssprk3(U0, b, P, qv, qf, dt, n)
    for m in route_meshes(rm):
        conv = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf)
        conv.set_state(U0)
        conv.ssprk3(dt, n)
        assert rel_l2(conv.get_state(), Ur) < TOL
        assert rel_l2(conv.get_state() - U0, Ur - U0) < 1e-10
        conv.close()


def test_config1_vortex_p1_twenty_steps():
    P, qv, qf, L, n = 1, 0, 1, 10.0, 8
    ref = RefLib()
    rm = ref.box(n, hi=(L,) * 3)  # the oracle's own copy of the periodic mesh
    m = box_mesh(n, hi=(L,) * 3)
    assert m.ncell == 3072
    U0 = problems.project(m, P, problems.isentropic_vortex())
    Ur = rm.project(P, "vortex", [5, 5, 5, 0, 0, 1, 5.0, 1.4, 1, 1, 0, 0.0])
    assert rel_l2(U0, Ur) < 1e-14
    conv = ExplicitConvection(m, order=P, flux="LF", quad_vol=qv, quad_face=qf)
    conv.set_state(U0)
    dt = problems.cfl_dt(0.3, L / n, P, conv.max_wave_speed())
    b = rm.mass(P, qv)
    Ug_prev, Ur_prev = U0, U0
    worst = 0.0
    for step in range(20):
        conv.ssprk3(dt, 1)
        Ug = conv.get_state()
        Ur = rm.ssprk3(Ur_prev, b, P, qv, qf, dt, 1, t0=step * dt)
        e = rel_l2(Ug, Ur)
        worst = max(worst, e)
        assert e < TOL, (step, e)
        assert rel_l2(Ug - Ug_prev, Ur - Ur_prev) < 1e-10, step  # the step's increment itself
        Ug_prev, Ur_prev = Ug, Ur
    conv.close()
