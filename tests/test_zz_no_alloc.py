"""GPU: the residual entry point that allocates nothing (dg_residual_device_static).

Some callers cannot call cudaMalloc once they are running: frameworks whose pool allocator took all
device memory at start-up, and time-critical loops in which cudaMalloc/cudaFree could synchronise
the device. They create the context during set-up and then use this entry point, whose face-flux
scratch is a fixed device array of the library. This file runs last so that a failure here never
hides the other tests; it passes alone and after them.
"""
import ctypes

import numpy as np
import pytest

from fve_dg_b200 import ExplicitConvection, box_mesh, problems
from fve_dg_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2, the FP64 parity bar of the other GPU tests


def _call(fn, ctx, U, R, stream, *extra):
    return fn(ctx, ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(R.data_ptr()), *extra, ctypes.c_void_p(stream))


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
    lib = L.lib()
    L.check(_call(lib.dg_residual_device, conv._ctx, Ud, Rref, stream, ctypes.c_double(0.0), 0), "dg_residual_device")
    torch.cuda.synchronize()
    b = Rref.cpu().numpy()
    free0 = None
    for i in range(3):  # calls in a row share the array; each must match on its own
        Rs.fill_(0.0)
        L.check(_call(lib.dg_residual_device_static, conv._ctx, Ud, Rs, stream, 0), "dg_residual_device_static")
        torch.cuda.synchronize()
        if i == 0:  # the first call on the device looks the array up; later calls must take no memory
            free0 = torch.cuda.mem_get_info()[0]
        a = Rs.cpu().numpy()
        assert np.linalg.norm(a - b) <= TOL * np.linalg.norm(b)
    assert torch.cuda.mem_get_info()[0] == free0, "a call of the static entry point took device memory"
    conv.close()


def test_static_scratch_on_a_mixed_context_returns_the_fp64_residual():
    import torch
    P, qv, qf = 3, 3, 3
    m = box_mesh(3, jitter=0.1, seed=22)
    U = problems.project(m, P, problems.taylor_green())
    U += 1e-3 * np.random.default_rng(5).standard_normal(U.shape)
    mixed = ExplicitConvection(m, order=P, flux="Roe", quad_vol=qv, quad_face=qf, precision="mixed")
    fp64 = ExplicitConvection(m, order=P, flux="Roe", quad_vol=qv, quad_face=qf, precision="fp64")
    Ud = torch.from_numpy(U).cuda()
    Rref, Rs = torch.empty_like(Ud), torch.empty_like(Ud)
    stream = torch.cuda.current_stream().cuda_stream
    lib = L.lib()
    L.check(_call(lib.dg_residual_device, fp64._ctx, Ud, Rref, stream, ctypes.c_double(0.0), 0), "dg_residual_device")
    for _ in range(2):
        Rs.fill_(0.0)
        L.check(_call(lib.dg_residual_device_static, mixed._ctx, Ud, Rs, stream, 0), "dg_residual_device_static")
        torch.cuda.synchronize()
        a, b = Rs.cpu().numpy(), Rref.cpu().numpy()
        assert np.linalg.norm(a - b) <= TOL * np.linalg.norm(b)
    mixed.close()
    fp64.close()


def test_static_scratch_rejects_meshes_that_do_not_fit():
    m = box_mesh(16)  # 24,576 tets, P3 face fluxes: 49,152 faces x 24 points x 5 > capacity
    conv = ExplicitConvection(m, order=3, quad_vol=3, quad_face=3)
    assert m.nface * conv.nq_face * 5 > L.lib().dg_static_scratch_capacity()
    rc = L.lib().dg_residual_device_static(conv._ctx, ctypes.c_void_p(1), ctypes.c_void_p(1), 0, None)
    assert rc == -1  # DG_E_ARG, before any device work
    conv.close()
