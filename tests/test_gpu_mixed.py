"""GPU: the mixed-precision form (BF16 hi/lo tensor-core contractions, FP32 flux, FP64 RK state)
against the FP64 form and the oracle."""
import numpy as np
import pytest

from conftest import CASES, rel_l2
from fve_dg_b200 import ExplicitConvection, box_mesh, problems
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu

# Residual tolerance of the mixed form, relative L2 against the FP64 residual. Each contraction
# carries about 16 bits on the deviations from the element/face means and the flux is FP32.
RES_TOL = 1e-4
# State tolerance after time stepping (density and energy, relative L2 against FP64).
STATE_TOL = 1e-6


@pytest.mark.parametrize("P,qv,qf", CASES)
def test_mixed_residual_close_to_fp64(P, qv, qf):
    m = box_mesh(3, jitter=0.1, seed=5)
    U = problems.project(m, P, problems.density_wave())
    U += 1e-3 * np.random.default_rng(P).standard_normal(U.shape)
    R64 = Oracle.from_mesh(m).residual(U, P, qv, qf)
    mixed = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision="mixed")
    assert rel_l2(mixed.eval(U), R64) < RES_TOL


@pytest.mark.parametrize("flux", ["LF", "Roe"])
def test_mixed_taylor_green_state_error(flux):
    """Low-Mach flow (p0 ~ 71): the mean-subtracted contractions keep the state within 1e-6."""
    n, P, qv, qf = 8, 3, 3, 3
    L = 2 * np.pi
    m = box_mesh(n, hi=(L, L, L))
    U0 = problems.project(m, P, problems.taylor_green())
    f64 = ExplicitConvection(m, order=P, flux=flux, quad_vol=qv, quad_face=qf)
    mix = ExplicitConvection(m, order=P, flux=flux, quad_vol=qv, quad_face=qf, precision="mixed")
    f64.set_state(U0)
    mix.set_state(U0)
    dt = problems.cfl_dt(0.3, L / n, P, f64.max_wave_speed())
    f64.ssprk3(dt, 50)
    mix.ssprk3(dt, 50)
    err = problems.l2_errors(m, P, mix.get_state(), Uref=f64.get_state())
    assert err[0] < STATE_TOL and err[4] < STATE_TOL, err


def test_mixed_conserves_exactly():
    """Single-valued face fluxes and exactly negated lifts: sums are conserved to round-off."""
    m = box_mesh(4, jitter=0.1, seed=2)
    P = 2
    U0 = problems.project(m, P, problems.density_wave())
    mix = ExplicitConvection(m, order=P, precision="mixed")
    mix.set_state(U0)
    c0 = mix.conservation()
    mix.ssprk3(2e-3, 10)
    c1 = mix.conservation()
    assert np.all(np.abs(c1[:5] - c0[:5]) <= 1e-12 * np.maximum(1.0, np.abs(c0[:5])))


def test_mixed_graph_matches_stream():
    m = box_mesh(4, jitter=0.1, seed=4)
    P = 3
    U0 = problems.project(m, P, problems.density_wave())
    mix = ExplicitConvection(m, order=P, quad_vol=3, quad_face=3, precision="mixed")
    mix.set_state(U0)
    mix.ssprk3(1e-3, 3)
    a = mix.get_state()
    mix.set_state(U0)
    mix.ssprk3(1e-3, 3, graph=True)
    assert np.array_equal(a, mix.get_state())


@pytest.mark.parametrize("P,qv,qf", [(1, 0, 1), (2, 1, 2), (3, 3, 3)])
def test_staged_element_kernel_is_bit_identical(P, qv, qf):
    """The element kernel whose group rows arrive by TMA bulk copies (one or two CTAs per SM) does the
    same arithmetic in the same order as the one that loads them phase by phase."""
    m = box_mesh(4, jitter=0.1, seed=7)
    U0 = problems.project(m, P, problems.density_wave())
    U0 += 1e-3 * np.random.default_rng(P).standard_normal(U0.shape)
    got = []
    for shape in ((0, 1), (1, 1), (1, 2)):
        c = ExplicitConvection(m, order=P, flux="Roe", quad_vol=qv, quad_face=qf, precision="mixed")
        c.set_element_shape(*shape)
        R = c.eval(U0)
        c.set_state(U0)
        c.ssprk3(1e-3, 2)
        c.ssprk3(1e-3, 2, graph=True)
        got.append((R, c.get_state()))
        c.close()
    for R, S in got[1:]:
        assert np.array_equal(R, got[0][0])
        assert np.array_equal(S, got[0][1])


def test_two_launch_autotune_records_element_shapes():
    m = box_mesh(6, hi=(2 * np.pi,) * 3)
    U = problems.project(m, 3, problems.taylor_green())
    c = ExplicitConvection(m, order=3, flux="Roe", quad_vol=3, quad_face=3, precision="mixed")
    c.set_state(U)
    rep = c.autotune(1e-3)
    assert np.array_equal(c.get_state(), U)
    assert rep["schedule"] == "two-launch" and len(rep["candidates"]) == 3
    assert rep["chosen"]["ms_per_step"] == min(x["ms_per_step"] for x in rep["candidates"])
    c.ssprk3(1e-3, 2)
    assert c.check_state() == 0
    c.close()
    p4 = ExplicitConvection(box_mesh(2), order=4, quad_vol=5, quad_face=3, precision="mixed")
    with pytest.raises(RuntimeError):
        p4.set_element_shape(1, 1)  # P4 state rows are not whole 16-byte units
    p4.close()
