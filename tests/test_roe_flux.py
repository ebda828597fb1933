"""The Roe flux, which the reference declares but never defines (tests/test_flux/RiemannSolvers.h:21-27),
pinned to the published Roe scheme through a second, independent construction.

The oracle (oracle/dg_oracle.c flux_roe) builds the dissipation from the wave strengths and right
eigenvectors of the 3D Euler equations, and the GPU kernels match the oracle's residual to 1e-12
(tests/test_gpu_parity.py). Here the same flux is built another way, from the Roe matrix itself:
  A~ = dF.n/dU evaluated at the Roe averages (u~, H~) of the two states (Roe's property
       F(UR).n - F(UL).n = A~ (UR - UL) holds exactly for this matrix);
  |A~| from its spectral projectors, |A~| = f(l1) P1 + |q| Pq + f(l5) P5 with l1,5 = q -+ c~ and
       Harten's fix f(l) = (l^2 + d^2) / (2 d) for |l| < d, d = 0.1 c~;
  F^ = (F(UL).n + F(UR).n) / 2 - |A~| (UR - UL) / 2.
Plus the flux's defining properties: consistency F^(U, U, n) = F(U).n and conservation
F^(UL, UR, n) = -F^(UR, UL, -n)."""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SO = os.path.join(ROOT, "oracle", "liboracle.so")
GAMMA = 1.4


def oracle_flux(kind, UL, UR, n, gamma=GAMMA):
    L = ctypes.CDLL(SO)
    dp = ctypes.POINTER(ctypes.c_double)
    L.orc_numerical_flux.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_double, dp]
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (UL, UR, n)]
    F = np.zeros(5)
    assert L.orc_numerical_flux(kind, *(x.ctypes.data_as(dp) for x in a), gamma, F.ctypes.data_as(dp)) == 0
    return F


def conserved(rho, u, p, gamma=GAMMA):
    return np.array([rho, *(rho * u), p / (gamma - 1) + 0.5 * rho * u @ u])


def physical_flux_n(U, n, gamma=GAMMA):
    rho, m, E = U[0], U[1:4], U[4]
    u = m / rho
    p = (gamma - 1) * (E - 0.5 * rho * u @ u)
    un = u @ n
    return np.array([rho * un, *(m * un + p * n), (E + p) * un])


def roe_matrix_flux(UL, UR, n, gamma=GAMMA):
    """F^ from the Roe matrix and its spectral projectors (see the module docstring)."""
    def prim(U):
        rho = U[0]
        u = U[1:4] / rho
        p = (gamma - 1) * (U[4] - 0.5 * rho * u @ u)
        return rho, u, (U[4] + p) / rho
    rL, uL, HL = prim(UL)
    rR, uR, HR = prim(UR)
    sL, sR = np.sqrt(rL), np.sqrt(rR)
    u = (sL * uL + sR * uR) / (sL + sR)
    H = (sL * HL + sR * HR) / (sL + sR)
    g = gamma - 1
    k = 0.5 * u @ u
    q = u @ n
    c = np.sqrt(g * (H - k))
    A = np.zeros((5, 5))
    A[0, 1:4] = n
    for i in range(3):
        A[1 + i, 0] = g * k * n[i] - u[i] * q
        for j in range(3):
            A[1 + i, 1 + j] = u[i] * n[j] - g * n[i] * u[j] + (q if i == j else 0.0)
        A[1 + i, 4] = g * n[i]
    A[4, 0] = (g * k - H) * q
    A[4, 1:4] = H * n - g * u * q
    A[4, 4] = gamma * q
    l1, l5 = q - c, q + c
    I5 = np.eye(5)
    P1 = (A - q * I5) @ (A - l5 * I5) / ((l1 - q) * (l1 - l5))
    P5 = (A - q * I5) @ (A - l1 * I5) / ((l5 - q) * (l5 - l1))
    Pq = I5 - P1 - P5
    d = 0.1 * c

    def fix(lam):
        return (lam * lam + d * d) / (2 * d) if abs(lam) < d else abs(lam)
    absA = fix(l1) * P1 + abs(q) * Pq + fix(l5) * P5
    dU = UR - UL
    return 0.5 * (physical_flux_n(UL, n) + physical_flux_n(UR, n)) - 0.5 * absA @ dU, A


def random_pairs(seed, count, sonic=False):
    rng = np.random.default_rng(seed)
    for _ in range(count):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        rho = rng.uniform(0.5, 2.0, 2)
        p = rng.uniform(0.5, 2.0, 2)
        u = rng.uniform(-1.0, 1.0, (2, 3))
        if sonic:  # normal velocity near the sound speed: Harten's fix is active on one wave
            c = np.sqrt(GAMMA * p[0] / rho[0])
            u[0] += (c - u[0] @ n) * n
            u[1] = u[0] + 0.05 * rng.uniform(-1, 1, 3)
            rho[1], p[1] = rho[0] * (1 + 0.02 * rng.uniform(-1, 1)), p[0] * (1 + 0.02 * rng.uniform(-1, 1))
        yield conserved(rho[0], u[0], p[0]), conserved(rho[1], u[1], p[1]), n


@pytest.mark.skipif(not os.path.exists(SO), reason="oracle not built")
@pytest.mark.parametrize("sonic", [False, True])
def test_roe_flux_equals_roe_matrix_construction(sonic):
    checked = 0
    for UL, UR, n in random_pairs(7 + sonic, 200, sonic):
        want, A = roe_matrix_flux(UL, UR, n)
        # Roe's property of the matrix used for the comparison
        dF = physical_flux_n(UR, n) - physical_flux_n(UL, n)
        assert np.allclose(A @ (UR - UL), dF, rtol=0, atol=1e-12 * max(1.0, np.abs(dF).max()))
        got = oracle_flux(1, UL, UR, n)
        assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max()), (got, want)
        checked += 1
    assert checked == 200


@pytest.mark.skipif(not os.path.exists(SO), reason="oracle not built")
@pytest.mark.parametrize("kind", [0, 1])
def test_numerical_flux_is_consistent_and_conservative(kind):
    for UL, UR, n in random_pairs(11, 100):
        FU = oracle_flux(kind, UL, UL, n)
        want = physical_flux_n(UL, n)
        assert np.abs(FU - want).max() <= 1e-13 * max(1.0, np.abs(want).max())
        F1 = oracle_flux(kind, UL, UR, n)
        F2 = oracle_flux(kind, UR, UL, -n)
        assert np.abs(F1 + F2).max() <= 1e-13 * max(1.0, np.abs(F1).max())
