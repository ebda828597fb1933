"""GPU: the positivity-preserving limiter (PositiveLimiter.h:12-261) against the reference's own
limiter, compiled from source into oracle/_ref, and the limiter inside the SSP-RK3 loop."""
import numpy as np
import pytest

from conftest import rel_l2
from fve_dg_b200 import ExplicitConvection, box_mesh, problems
from oracle.pyoracle import RefLib, RefMesh, ref_available

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2, the FP64 parity bar
# (order, volume rule): the configurations' rules and the reference's Auto rules
LIM_CASES = [(1, 0), (1, 2), (2, 1), (2, 2), (3, 3), (3, 4), (4, 5), (4, 6)]


def rough_states(m, P, seed, A, noise):
    """A previous state (density wave of amplitude A) and a current one with noisy high modes."""
    rng = np.random.default_rng(seed)
    Uprev = problems.project(m, P, problems.density_wave(A=A))
    hi = np.arange(Uprev.shape[1]) >= 5
    U = Uprev + noise * rng.standard_normal(Uprev.shape) * hi * np.abs(Uprev[:, :5]).max()
    U[:, :5] += 0.01 * rng.standard_normal((U.shape[0], 5))
    return U, Uprev


def point_states(U, P, qv):
    """Conserved states at the volume rule's points, (ncell, npts, 5)."""
    pts, _ = problems.quad_rule(0, qv)
    phi, _ = problems.basis(P, pts)
    return np.einsum("gb,ebk->egk", phi, U.reshape(U.shape[0], -1, 5))


def admissible(U, P, qv, gamma=1.4):
    """Density > 0 and pressure >= -1e-12 |E| at every volume point (the limiter's bisection stops at
    the crossing p = 0, so a limited point may sit at p = 0 to round-off)."""
    S = point_states(U, P, qv)
    rho = S[..., 0]
    p = (gamma - 1.0) * (S[..., 4] - 0.5 * (S[..., 1] ** 2 + S[..., 2] ** 2 + S[..., 3] ** 2) / np.where(rho > 0, rho, 1))
    return bool(np.all(rho > 0) and np.all(p >= -1e-12 * np.abs(S[..., 4])))


@pytest.fixture(scope="module")
def mesh3():
    return box_mesh(3, jitter=0.1, seed=5)


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
@pytest.mark.parametrize("P,qv", LIM_CASES)
@pytest.mark.parametrize("only_avg", [False, True])
def test_limiter_matches_reference(mesh3, P, qv, only_avg):
    rm = RefMesh.from_mesh(RefLib(), mesh3)
    conv = ExplicitConvection(mesh3, order=P, quad_vol=qv)
    for A, noise, seed in ((0.2, 0.05, 1), (0.97, 0.3, 2)):  # mild; near vacuum (density and pressure steps)
        U, Uprev = rough_states(mesh3, P, 100 * P + seed, A, noise)
        got = conv.limit(U, Uprev, only_neighbor_avg=only_avg)
        want = rm.limit(U, Uprev, P, qv, 1.4, only_avg)
        assert np.abs(want - U).max() > 1e-3            # the limiter acted
        assert np.array_equal(got[:, :5], U[:, :5])     # element means untouched
        assert rel_l2(got, want) < TOL, (A, rel_l2(got, want))


def test_limiter_makes_points_admissible(mesh3):
    P, qv = 3, 3
    U, Uprev = rough_states(mesh3, P, 7, 0.97, 0.5)
    conv = ExplicitConvection(mesh3, order=P, quad_vol=qv)
    assert not admissible(U, P, qv)
    assert admissible(conv.limit(U, Uprev), P, qv)


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
def test_limited_stepping_matches_reference_loop():
    """SSP-RK3 with the limiter after every stage (bounds from the stage input) on the GPU against
    the same loop on the CPU: the oracle's residual and the reference's own PositiveLimiter."""
    from oracle.pyoracle import Oracle
    m = box_mesh(6, jitter=0.1, seed=11)
    P, qv, qf = 2, 1, 2
    U0 = problems.project(m, P, problems.density_wave(A=0.8, vel=(2.0, 1.0, 0.5), p=0.01))
    c = U0[:, :5]
    u = c[:, 1:4] / c[:, :1]
    pres = 0.4 * (c[:, 4] - 0.5 * c[:, 0] * (u ** 2).sum(1))
    lam = (np.sqrt((u ** 2).sum(1)) + np.sqrt(1.4 * pres / c[:, 0])).max()
    dt, nsteps = problems.cfl_dt(0.3, 1.0 / 6, P, lam), 3
    o, rm = Oracle.from_mesh(m), RefMesh.from_mesh(RefLib(), m)
    b = o.mass(P, qv)

    def L(U):
        return -o.residual(U, P, qv, qf) / b

    def lim(cur, prev):
        return rm.limit(cur, prev, P, qv, 1.4, False)

    U, acted = U0.copy(), 0.0
    for _ in range(nsteps):
        U1 = lim(U + dt * L(U), U)
        U2 = lim(0.75 * U + 0.25 * (U1 + dt * L(U1)), U1)
        U3 = U / 3 + 2.0 / 3 * (U2 + dt * L(U2))
        Un = lim(U3, U2)
        acted = max(acted, np.abs(Un - U3).max())
        U = Un
    assert acted > 1e-6  # the limiter changed the solution
    conv = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, limiter="positive")
    conv.set_state(U0)
    c0 = conv.conservation()
    conv.ssprk3(dt, nsteps, graph=True)
    got = conv.get_state()
    assert rel_l2(got, U) < 1e-9
    c1 = conv.conservation()
    assert abs(c1[0] - c0[0]) <= 1e-12 * abs(c0[0]) and abs(c1[4] - c0[4]) <= 1e-12 * abs(c0[4])
    plain = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, limiter="positive")
    plain.set_state(U0)
    plain.ssprk3(dt, nsteps)
    assert np.array_equal(plain.get_state(), got)  # graph replay = plain steps
    mixed = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, limiter="positive", precision="mixed")
    mixed.set_state(U0)
    mixed.ssprk3(dt, nsteps, graph=True)
    assert rel_l2(mixed.get_state(), got) < 1e-5


def test_limiter_option_is_validated():
    m = box_mesh(2)
    with pytest.raises(Exception):
        ExplicitConvection(m, order=2, quad_vol=1, limiter=7)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_limiter_bounds_follow_the_state(precision):
    """The limiter's bounds for a stage come from the previous stage's limited output; a state set
    from outside recomputes them. Graph replays after a new set_state, and stage-by-stage stepping,
    give exactly what plain stepping gives."""
    from fve_dg_b200 import _lib as L
    m = box_mesh(6, jitter=0.1, seed=11)
    P = 2
    U0 = problems.project(m, P, problems.density_wave(A=0.8, vel=(2.0, 1.0, 0.5), p=0.01))
    U1 = problems.project(m, P, problems.density_wave(A=0.6, vel=(-1.0, 0.5, 1.5), p=0.02))
    lam = 0.0
    for U in (U0, U1):
        c = U[:, :5]
        u = c[:, 1:4] / c[:, :1]
        pres = 0.4 * (c[:, 4] - 0.5 * c[:, 0] * (u ** 2).sum(1))
        lam = max(lam, (np.sqrt((u ** 2).sum(1)) + np.sqrt(1.4 * pres / c[:, 0])).max())
    dt = problems.cfl_dt(0.3, 1.0 / 6, P, lam)
    kw = dict(order=P, quad_vol=1, quad_face=2, limiter="positive", precision=precision)
    ref = {}
    for name, U in (("a", U0), ("b", U1)):
        c = ExplicitConvection(m, **kw)
        c.set_state(U)
        c.ssprk3(dt, 3)
        ref[name] = c.get_state()
        assert np.all(np.isfinite(ref[name])) and np.abs(ref[name] - U).max() > 1e-6
    conv = ExplicitConvection(m, **kw)
    for name, U in (("a", U0), ("b", U1), ("a", U0)):
        conv.set_state(U)
        conv.ssprk3(dt, 3, graph=True)
        assert np.array_equal(conv.get_state(), ref[name]), name
    conv.set_state(U1)
    for _ in range(3):
        for st in range(3):
            assert L.lib().dg_ssprk3_stage(conv._ctx, dt, st) == 0
    conv.ssprk3(dt, 0)
    assert np.array_equal(conv.get_state(), ref["b"])
