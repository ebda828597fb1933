"""GPU: one mesh split into parts with ghost elements (fve_dg_b200/partition.py), each part its own
context, stepped one SSP-RK3 stage at a time (dg_ssprk3_stage) with the ghost rows of every stage
input filled from their owners by the library's gather and scatter kernels (dg_halo_pack,
dg_halo_unpack) in between. The owned states must equal the
whole-mesh context's. (Parts run as separate contexts on one GPU, one after another; the NCCL
exchange between processes is the same plan, checked on CPU over gloo.)"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2
from fve_dg_b200 import ExplicitConvection, box_mesh, problems
from fve_dg_b200 import _lib as L
from fve_dg_b200.partition import emulated_ranks, step_emulated

pytestmark = pytest.mark.gpu


def run_parts(m, U0, nparts, dt, nsteps, **kw):
    ranks = emulated_ranks(m, nparts, **kw)
    for r in ranks:
        r.set_state(U0)
    step_emulated(ranks, dt, nsteps)
    got = np.empty_like(U0)
    for r in ranks:
        got[r.lm.owned] = r.get_owned()
    return got


def run_whole(m, U0, dt, nsteps, **kw):
    conv = ExplicitConvection(m, **kw)
    conv.set_state(U0)
    conv.ssprk3(dt, nsteps)
    return conv.get_state()


CASES = [
    # (mesh kwargs, nparts, convection kwargs, tolerance)
    (dict(periodic=(1, 1, 1)), 2, dict(order=3), 0.0),
    (dict(periodic=(1, 1, 1)), 3, dict(order=2, flux="Roe"), 0.0),
    (dict(periodic=(1, 1, 0), bc="Pseudo3DZ"), 4, dict(order=3), 0.0),
    (dict(periodic=(1, 1, 1)), 2, dict(order=3, precision="mixed"), 1e-13),
    (dict(periodic=(1, 1, 1)), 3, dict(order=3, precision="mixed", schedule="persistent"), 1e-13),
    (dict(periodic=(1, 1, 0), bc="Pseudo3DZ"), 2, dict(order=4, precision="mixed"), 1e-13),
    # Navier-Stokes: the viscous residual of each stage reads the exchanged ghost rows; a ghost's
    # penalty length comes from its vertices (equal to the whole mesh's to rounding)
    (dict(periodic=(1, 1, 0), bc="Pseudo3DZ"), 3, dict(order=2, mu=0.001, prandtl=0.72), 1e-12),
    (dict(periodic=(1, 1, 1)), 2, dict(order=3, mu=3e-4, prandtl=0.72, precision="mixed"), 1e-12),
]


@pytest.mark.parametrize("mk,nparts,kw,tol", CASES)
def test_parts_equal_whole_mesh(mk, nparts, kw, tol):
    m = box_mesh(6, jitter=0.1, seed=21, **mk)
    U0 = problems.project(m, kw["order"], problems.density_wave(A=0.3, vel=(1.0, 0.5, 0.25)))
    dt, nsteps = 2e-3, 4
    want = run_whole(m, U0, dt, nsteps, **kw)
    got = run_parts(m, U0, nparts, dt, nsteps, **kw)
    assert np.abs(want - U0).max() > 1e-4  # the state moved
    assert rel_l2(got, want) <= tol, rel_l2(got, want)


@pytest.mark.parametrize("precision,tol", [("fp64", 0.0), ("mixed", 1e-13)])
def test_owned_residual_equals_whole_mesh(precision, tol):
    from fve_dg_b200.partition import LocalMesh, partition_elements
    m = box_mesh(6, jitter=0.1, seed=22)
    U = problems.project(m, 3, problems.density_wave(A=0.3, vel=(1.0, 0.5, 0.25)))
    want = ExplicitConvection(m, order=3, precision=precision).eval(U)
    part = partition_elements(m, 3)
    for r in range(3):
        lm = LocalMesh(m, part, r)
        got = ExplicitConvection(lm.mesh, order=3, precision=precision).eval(U[lm.l2g])[: lm.n_owned]
        assert rel_l2(got, want[lm.owned]) <= tol


@pytest.mark.parametrize("kw", [dict(order=3, precision="mixed"), dict(order=2, precision="mixed", mu=0.001,
                                                                     prandtl=0.72, limiter="positive"),
                                dict(order=2), dict(order=3, precision="mixed", schedule="persistent")])
def test_phased_stages_equal_whole_mesh(kw):
    """Each stage in two phases around the exchange (dg_ssprk3_stage_phase): the faces between owned
    elements before the ghost rows arrive, the rest after."""
    m = box_mesh(6, jitter=0.1, seed=24, periodic=(1, 1, 0), bc="Pseudo3DZ")
    U0 = problems.project(m, kw["order"], problems.density_wave(A=0.3, vel=(1.0, 0.5, 0.25)))
    dt, nsteps = 2e-3, 3
    want = run_whole(m, U0, dt, nsteps, **kw)
    ranks = emulated_ranks(m, 3, **kw)
    for r in ranks:
        r.set_state(U0)
    step_emulated(ranks, dt, nsteps, phased=True)
    got = np.empty_like(U0)
    for r in ranks:
        got[r.lm.owned] = r.get_owned()
    tol = 0.0 if kw.get("precision", "fp64") == "fp64" else 1e-12
    assert rel_l2(got, want) <= tol, rel_l2(got, want)
    # the overlapped form (exchange on a second stream, ordered by events) gives the same states
    ranks2 = emulated_ranks(m, 3, **kw)
    for r in ranks2:
        r.set_state(U0)
    import torch
    for _ in range(nsteps):
        for st in range(3):
            torch.cuda.synchronize()
            for r in ranks2:
                r.overlapped_stage(dt, st)
    torch.cuda.synchronize()
    for r in ranks2:
        r.wait()
    got2 = np.empty_like(U0)
    for r in ranks2:
        got2[r.lm.owned] = r.get_owned()
    assert np.array_equal(got2, got)


def test_parts_with_limiter_equal_whole_mesh():
    m = box_mesh(6, jitter=0.1, seed=11)
    P = 2
    U0 = problems.project(m, P, problems.density_wave(A=0.8, vel=(2.0, 1.0, 0.5), p=0.01))
    kw = dict(order=P, quad_vol=1, quad_face=2, limiter="positive")
    dt = 1e-3
    want = run_whole(m, U0, dt, 3, **kw)
    plain = run_whole(m, U0, dt, 3, order=P, quad_vol=1, quad_face=2)
    assert np.abs(want - plain).max() > 1e-8  # the limiter acted
    got = run_parts(m, U0, 3, dt, 3, **kw)
    assert rel_l2(got, want) == 0.0, rel_l2(got, want)


def test_stage_entry_points_validate():
    m = box_mesh(3)
    conv = ExplicitConvection(m, order=2)
    lib = L.lib()
    assert lib.dg_state_device(conv._ctx, 3) is None
    assert lib.dg_ssprk3_stage(conv._ctx, 1e-3, 0) == -7  # no state yet
    conv.set_state(np.zeros(conv.shape) + np.tile([1.0, 0, 0, 0, 2.5] + [0.0] * (conv.shape[1] - 5), 1))
    assert lib.dg_ssprk3_stage(conv._ctx, 1e-3, 3) == -1
    assert lib.dg_ssprk3_stage(conv._ctx, -1.0, 0) == -1
    assert lib.dg_refresh_split(conv._ctx, 0, None, 5, None) == -1
    assert lib.dg_refresh_split(conv._ctx, 0, None, 0, None) == 0
    for which in range(3):
        assert lib.dg_state_device(conv._ctx, which)
    assert lib.dg_ssprk3_stage(conv._ctx, 1e-3, 0) == 0
    assert lib.dg_ssprk3(conv._ctx, 0.0, 0) == 0


@pytest.mark.parametrize("P", [2, 3])
def test_owned_viscous_and_limiter_equal_whole_mesh(P):
    """The viscous operator and the standalone limiter on a part with ghost elements give the
    whole mesh's owned rows: ghosts need only their faces to owned elements."""
    from fve_dg_b200.partition import LocalMesh, partition_elements
    m = box_mesh(6, jitter=0.1, seed=23, periodic=(1, 1, 0), bc="Pseudo3DZ")
    U = problems.project(m, P, problems.density_wave(A=0.6, vel=(1.0, 0.5, 0.25), p=0.05))
    rng = np.random.default_rng(P)
    Ur = U + 0.05 * rng.standard_normal(U.shape) * (np.arange(U.shape[1]) >= 5) * np.abs(U[:, :5]).max()
    whole = ExplicitConvection(m, order=P)
    V = whole.viscous_eval(U, mu=0.01, prandtl=0.72)
    Lw = whole.limit(Ur, U)
    part = partition_elements(m, 3)
    for r in range(3):
        lm = LocalMesh(m, part, r)
        conv = ExplicitConvection(lm.mesh, order=P)
        Vl = conv.viscous_eval(U[lm.l2g], mu=0.01, prandtl=0.72)[: lm.n_owned]
        assert rel_l2(Vl, V[lm.owned]) <= 1e-14, rel_l2(Vl, V[lm.owned])
        Ll = conv.limit(Ur[lm.l2g], U[lm.l2g])[: lm.n_owned]
        assert rel_l2(Ll, Lw[lm.owned]) == 0.0
