"""GPU: the persistent work-queue schedule, ensembles of uneven meshes and the autotuner."""
import numpy as np
import pytest

from conftest import rel_l2
from fve_dg_b200 import Ensemble, ExplicitConvection, box_mesh, problems

pytestmark = pytest.mark.gpu


def vortex_mesh_state(n, P, seed):
    rng = np.random.default_rng(seed)
    m = box_mesh(n, hi=(10.0, 10.0, 10.0))
    axis = rng.normal(size=3)
    U = problems.project(m, P, problems.isentropic_vortex(center=rng.uniform(0, 10, 3), axis=axis,
                                                          beta=rng.uniform(1, 5), period=10.0))
    return m, U


@pytest.mark.parametrize("P,qv,qf", [(2, 1, 2), (3, 3, 3)])
def test_persistent_matches_two_launch(P, qv, qf):
    m, U = vortex_mesh_state(4, P, 1)
    a = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision="mixed")
    b = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision="mixed", schedule="persistent")
    for c in (a, b):
        c.set_state(U)
        c.ssprk3(1e-3, 3)
    assert np.array_equal(a.get_state(), b.get_state())  # same per-group work, any order
    b.set_state(U)
    b.ssprk3(1e-3, 3, graph=True)
    assert np.array_equal(a.get_state(), b.get_state())


def test_ensemble_matches_separate_solves():
    P, qv, qf = 2, 1, 2
    sizes = [3, 5, 4]
    parts = [vortex_mesh_state(n, P, 10 + i) for i, n in enumerate(sizes)]
    dts = np.array([1e-3, 2e-3, 1.5e-3])
    for prec, sched in (("mixed", "persistent"), ("mixed", "two-launch"), ("fp64", "two-launch")):
        ens = Ensemble([m for m, _ in parts], order=P, quad_vol=qv, quad_face=qf, precision=prec, schedule=sched)
        ens.set_state(np.concatenate([U for _, U in parts]))
        ens.ssprk3(dts, 4, graph=True)
        got = ens.split(ens.get_state())
        for i, (m, U) in enumerate(parts):
            one = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision=prec, schedule=sched)
            one.set_state(U)
            one.ssprk3(dts[i], 4)
            assert np.array_equal(got[i], one.get_state()), (prec, sched, i)


def test_ensemble_mixed_close_to_fp64():
    P = 2
    parts = [vortex_mesh_state(n, P, 20 + n) for n in (3, 6)]
    st = np.concatenate([U for _, U in parts])
    out = {}
    for prec, sched in (("mixed", "persistent"), ("fp64", "two-launch")):
        ens = Ensemble([m for m, _ in parts], order=P, quad_vol=1, quad_face=2, precision=prec, schedule=sched)
        ens.set_state(st)
        ens.ssprk3([2e-3, 1e-3], 10)
        out[prec] = ens.get_state()
    assert rel_l2(out["mixed"], out["fp64"]) < 1e-6


def test_autotune_records_and_restores():
    m, U = vortex_mesh_state(6, 3, 3)
    c = ExplicitConvection(m, order=3, quad_vol=3, quad_face=3, precision="mixed", schedule="persistent")
    c.set_state(U)
    rep = c.autotune(1e-3)
    assert np.array_equal(c.get_state(), U)
    assert len(rep["candidates"]) >= 4 and "chosen" in rep
    assert rep["chosen"]["ms_per_step"] == min(x["ms_per_step"] for x in rep["candidates"])
    c.ssprk3(1e-3, 2)  # the chosen tiles run
    assert c.check_state() == 0


@pytest.mark.parametrize("extra", [dict(mu=0.05, prandtl=0.72), dict(mu=0.05, prandtl=0.72, limiter="positive")])
def test_ensemble_navier_stokes_matches_separate_solves(extra):
    """Navier-Stokes stepping (and the limiter) in an ensemble: each instance, with its own dt,
    steps exactly as it does alone."""
    P, qv, qf = 2, 1, 2
    sizes = [3, 4]
    parts = [vortex_mesh_state(n, P, 20 + i) for i, n in enumerate(sizes)]
    dts = np.array([1e-3, 1.5e-3])
    for prec, sched in (("mixed", "two-launch"), ("fp64", "two-launch"), ("mixed", "persistent")):
        ens = Ensemble([m for m, _ in parts], order=P, quad_vol=qv, quad_face=qf, precision=prec, schedule=sched,
                       **extra)
        ens.set_state(np.concatenate([U for _, U in parts]))
        ens.ssprk3(dts, 3, graph=True)
        got = ens.split(ens.get_state())
        for i, (m, U) in enumerate(parts):
            one = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision=prec, schedule=sched, **extra)
            one.set_state(U)
            one.ssprk3(dts[i], 3)
            assert np.all(np.isfinite(got[i]))
            assert np.array_equal(got[i], one.get_state()), (prec, sched, i)


def test_bounded_wait_expires_and_context_stays_usable():
    """Failure detection of the persistent schedule without a GPU fault: a wait whose completion
    count can never be reached (dg_watchdog_selftest raises face region 0's required count by one)
    gives up after a few thousand polls; the kernel returns, the host reads DG_E_WATCHDOG, and the
    same context then steps exactly like one that never saw the expired wait."""
    import ctypes
    from fve_dg_b200 import _lib as L
    P, qv, qf = 2, 1, 2
    m, U = vortex_mesh_state(4, P, 3)
    a = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision="mixed", schedule="persistent")
    b = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision="mixed", schedule="persistent")
    a.set_state(U)
    assert L.lib().dg_watchdog_selftest(a._ctx, ctypes.c_int64(4096)) == L.DG_E_WATCHDOG
    assert L.lib().dg_watchdog_selftest(a._ctx, ctypes.c_int64(0)) == L.DG_E_ARG
    b.set_state(U)
    for c in (a, b):
        c.ssprk3(1e-3, 3)
    assert np.array_equal(a.get_state(), b.get_state())
    a.ssprk3(1e-3, 2, graph=True)  # graph replay on the same context after the expired wait
    b.ssprk3(1e-3, 2, graph=True)
    assert np.array_equal(a.get_state(), b.get_state())
    two = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision="mixed")
    two.set_state(U)
    assert L.lib().dg_watchdog_selftest(two._ctx, ctypes.c_int64(4096)) == L.DG_E_ARG  # two-launch form: no waits
