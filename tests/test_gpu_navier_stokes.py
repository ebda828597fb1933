"""GPU: compressible Navier-Stokes stepping (dg_config.mu > 0): every SSP-RK3 stage adds the viscous
residual, L = (R_visc - R_conv) / b, as the reference's viscous driver steps
(tests/test_diffusion.cpp:381-382). Checked against the same loop on the CPU built from the oracle's
convective residual and the reference's own ExplicitDiffusion (compiled into oracle/_ref)."""
import numpy as np
import pytest

from conftest import rel_l2
from fve_dg_b200 import ExplicitConvection, box_mesh, problems
from oracle.pyoracle import Oracle, RefLib, RefMesh, ref_available

pytestmark = pytest.mark.gpu


def cpu_ns_ssprk3(m, U0, P, qv, qf, dt, nsteps):
    """Shu-Osher SSP-RK3 with L = (ExplicitDiffusion::eval - convection residual) / mass on the CPU;
    the reference fixes mu = Pr = 1."""
    o, rm = Oracle.from_mesh(m), RefMesh.from_mesh(RefLib(), m)
    b = o.mass(P, qv)

    def L(U):
        return (rm.diffusion(U, P, qv, qf) - o.residual(U, P, qv, qf)) / b

    U = U0.copy()
    for _ in range(nsteps):
        U1 = U + dt * L(U)
        U2 = 0.75 * U + 0.25 * (U1 + dt * L(U1))
        U = U / 3.0 + 2.0 / 3.0 * (U2 + dt * L(U2))
    return U


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
@pytest.mark.parametrize("P,qv,qf,walls", [(1, 0, 1, False), (2, 1, 2, False), (3, 3, 3, False), (2, 1, 2, True)])
def test_navier_stokes_stepping_matches_reference_loop(P, qv, qf, walls):
    """walls: Pseudo3DZ boundary faces in z (their viscous and convective terms), else periodic."""
    m = (box_mesh(4, jitter=0.1, seed=33, periodic=(1, 1, 0), bc="Pseudo3DZ") if walls
         else box_mesh(4, jitter=0.1, seed=31))
    U0 = problems.project(m, P, problems.density_wave(A=0.2, vel=(1.0, 0.5, 0.25)))
    dt, nsteps = 2e-5, 3
    want = cpu_ns_ssprk3(m, U0, P, qv, qf, dt, nsteps)
    conv = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, mu=1.0, prandtl=1.0)
    conv.set_state(U0)
    conv.ssprk3(dt, nsteps, graph=True)
    got = conv.get_state()
    euler = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf)
    euler.set_state(U0)
    euler.ssprk3(dt, nsteps)
    assert rel_l2(euler.get_state() - U0, want - U0) > 1e-3  # the viscous terms matter here
    assert rel_l2(got - U0, want - U0) < 1e-10, rel_l2(got - U0, want - U0)
    plain = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, mu=1.0, prandtl=1.0)
    plain.set_state(U0)
    plain.ssprk3(dt, nsteps)
    assert np.array_equal(plain.get_state(), got)  # graph replay = plain steps


@pytest.mark.parametrize("schedule", ["two-launch", "persistent"])
def test_navier_stokes_mixed_form_tracks_fp64(schedule):
    m = box_mesh(6, jitter=0.1, seed=32)
    P = 3
    U0 = problems.project(m, P, problems.density_wave(A=0.2, vel=(1.0, 0.5, 0.25)))
    dt, nsteps = 1e-5, 4
    ref = ExplicitConvection(m, order=P, mu=0.5, prandtl=0.72)
    ref.set_state(U0)
    ref.ssprk3(dt, nsteps)
    mixed = ExplicitConvection(m, order=P, mu=0.5, prandtl=0.72, precision="mixed", schedule=schedule)
    mixed.set_state(U0)
    mixed.ssprk3(dt, nsteps, graph=True)
    d64, dmx = ref.get_state() - U0, mixed.get_state() - U0
    assert rel_l2(dmx, d64) < 1e-4, rel_l2(dmx, d64)


def test_viscosity_is_validated():
    m = box_mesh(2)
    for kw in (dict(mu=-1.0), dict(mu=1.0, prandtl=0.0), dict(mu=float("nan"))):
        with pytest.raises(Exception):
            ExplicitConvection(m, order=2, **kw)
