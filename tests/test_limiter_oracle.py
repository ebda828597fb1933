"""CPU: the reference's own positivity limiter (oracle/_ref, PositiveLimiter.h:12-261) behaves as the
GPU tests assume: element means untouched, the density and pressure made admissible at the volume
points, and both bound modes act on rough states."""
import numpy as np
import pytest

from fve_dg_b200 import box_mesh, problems
from oracle.pyoracle import RefLib, RefMesh, ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="reference library not built")


@pytest.mark.parametrize("P,qv", [(1, 0), (2, 1), (3, 3), (4, 5)])
def test_reference_limiter_properties(P, qv):
    m = box_mesh(2, jitter=0.1, seed=4)
    rng = np.random.default_rng(P)
    Uprev = problems.project(m, P, problems.density_wave(A=0.97))
    U = Uprev + 0.4 * rng.standard_normal(Uprev.shape) * (np.arange(Uprev.shape[1]) >= 5) * np.abs(Uprev).max()
    rm = RefMesh.from_mesh(RefLib(), m)
    pts, _ = problems.quad_rule(0, qv)
    phi, _ = problems.basis(P, pts)
    for only_avg in (False, True):
        L = rm.limit(U, Uprev, P, qv, 1.4, only_avg)
        assert np.array_equal(L[:, :5], U[:, :5])
        assert np.abs(L - U).max() > 1e-3
        S = np.einsum("gb,ebk->egk", phi, L.reshape(L.shape[0], -1, 5))
        rho = S[..., 0]
        p = 0.4 * (S[..., 4] - 0.5 * (S[..., 1] ** 2 + S[..., 2] ** 2 + S[..., 3] ** 2) / rho)
        assert np.all(rho > 0) and np.all(p >= -1e-12 * np.abs(S[..., 4]))
