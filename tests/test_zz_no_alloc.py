"""GPU: the residual entry point that allocates nothing (dg_residual_device_static).

Callers that cannot allocate device memory at the point of the call (inside a stream capture or a
host callback, or under a framework that owns all device memory) create the context at set-up and
then use this entry point, whose face-flux scratch is a fixed device array of the library. This
file runs last so that a failure here never hides the other tests; it passes alone and after them.
"""
import ctypes

import numpy as np
import pytest

from fve_dg_b200 import ExplicitConvection, box_mesh, problems
from fve_dg_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2, the FP64 parity bar of the other GPU tests


@pytest.mark.parametrize("P,qv,qf,flux", [(2, 1, 2, "LF"), (3, 3, 3, "Roe")])
def test_static_scratch_residual_matches_allocating_entry_point(P, qv, qf, flux):
    import torch
    m = box_mesh(3, jitter=0.1, seed=21)
    U = problems.project(m, P, problems.density_wave())
    U += 1e-3 * np.random.default_rng(P).standard_normal(U.shape)
    conv = ExplicitConvection(m, order=P, flux=flux, quad_vol=qv, quad_face=qf)
    need = m.nface * conv.nq_face * 5
    assert need <= L.lib().dg_static_scratch_capacity()
    Ud = torch.from_numpy(U).cuda()
    Rref = torch.empty_like(Ud)
    Rs = torch.empty_like(Ud)
    stream = torch.cuda.current_stream().cuda_stream
    L.check(L.lib().dg_residual_device(conv._ctx, ctypes.c_void_p(Ud.data_ptr()), ctypes.c_void_p(Rref.data_ptr()),
                                       0.0, 0, ctypes.c_void_p(stream)), "dg_residual_device")
    for _ in range(2):  # two calls in a row share the array; each must match on its own
        Rs.fill_(0.0)
        L.check(L.lib().dg_residual_device_static(conv._ctx, ctypes.c_void_p(Ud.data_ptr()),
                                                  ctypes.c_void_p(Rs.data_ptr()), 0, ctypes.c_void_p(stream)),
                "dg_residual_device_static")
        torch.cuda.synchronize()
        a, b = Rs.cpu().numpy(), Rref.cpu().numpy()
        assert np.linalg.norm(a - b) <= TOL * np.linalg.norm(b)


def test_static_scratch_rejects_meshes_that_do_not_fit():
    m = box_mesh(16)  # 24,576 tets, P3 face fluxes: 49,152 faces x 24 points x 5 > capacity
    conv = ExplicitConvection(m, order=3, quad_vol=3, quad_face=3)
    assert m.nface * conv.nq_face * 5 > L.lib().dg_static_scratch_capacity()
    rc = L.lib().dg_residual_device_static(conv._ctx, ctypes.c_void_p(1), ctypes.c_void_p(1), 0, None)
    assert rc == -1  # DG_E_ARG, before any device work
