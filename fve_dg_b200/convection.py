"""Host-side mirror of the reference's ExplicitConvection<Order, Flux, QuadC, QuadF>
(include/DG/DG_Schemes/ExplicitConvection.h:9-45) over the B200 kernels.

    conv = ExplicitConvection(mesh, order=3, flux="LF", quad_vol=-1, quad_face=-1, gamma=1.4)
    R = conv.eval(U, t)          # ExplicitConvection::eval, ExplicitConvection.cpp:136-141
    R = conv.eval_cells(U, t)    # :144-198
    R = conv.eval_internals(U, t)# :201-272
    R = conv.eval_boundarys(U, t)# :21-128

U and R are float64 arrays of shape (ncell, 5*Nb) in the reference's coefficient layout
coef[e][5*b + k]. Like the reference, eval is stateless with respect to U and returns a new array.
Beyond the reference interface the object also owns a device-resident state for the SSP-RK3 loop
(set_state / ssprk3 / get_state), the diagonal mass of the drivers, and conservation sums.
"""
import ctypes
import os

import numpy as np

from . import _lib as L

FLUX = {"LF": 0, "Roe": 1}
PRECISION = {"fp64": 0, "mixed": 1}
SCHEDULE = {"two-launch": 0, "persistent": 1}
LIMITER = {None: 0, "none": 0, "positive": 1, "positive-avg": 2}


class ExplicitConvection:
    def __init__(self, mesh, order=3, flux="LF", quad_vol=-1, quad_face=-1, gamma=1.4,
                 precision="fp64", device=0, schedule="two-launch", limiter=None, mu=0.0, prandtl=1.0,
                 _ensemble=None):
        """mu > 0 steps the compressible Navier-Stokes equations: every SSP-RK3 stage adds the viscous
        residual (viscous_eval with mu and prandtl) as the reference's viscous driver does."""
        self.mesh = mesh
        self.order = int(order)
        self.flux = flux
        self.gamma = float(gamma)
        self.precision = precision
        self.schedule = schedule
        cfg = L.Config(order=self.order, flux=FLUX[flux] if isinstance(flux, str) else int(flux),
                       quad_vol=int(quad_vol), quad_face=int(quad_face), gamma=self.gamma,
                       precision=PRECISION[precision] if isinstance(precision, str) else int(precision),
                       device=int(device), schedule=SCHEDULE[schedule] if isinstance(schedule, str) else int(schedule),
                       limiter=LIMITER[limiter] if limiter is None or isinstance(limiter, str) else int(limiter),
                       mu=float(mu), prandtl=float(prandtl))
        self.mu, self.prandtl = float(mu), float(prandtl)
        err = ctypes.c_int(0)
        if _ensemble is None:
            self._desc = mesh.desc()
            self._ctx = L.lib().dg_create(ctypes.byref(self._desc), ctypes.byref(cfg), ctypes.byref(err))
        else:
            self._descs = (L.MeshDesc * len(_ensemble))(*[m.desc() for m in _ensemble])
            self._ctx = L.lib().dg_create_ensemble(self._descs, len(_ensemble), ctypes.byref(cfg), ctypes.byref(err))
        if not self._ctx:
            raise L.DGError(err.value, "dg_create")
        nb, nqv, nqf, qv, qf = (ctypes.c_int() for _ in range(5))
        L.check(L.lib().dg_info(self._ctx, ctypes.byref(nb), ctypes.byref(nqv), ctypes.byref(nqf),
                                ctypes.byref(qv), ctypes.byref(qf)), "dg_info")
        self.num_basis, self.nq_vol, self.nq_face = nb.value, nqv.value, nqf.value
        self.quad_vol, self.quad_face = qv.value, qf.value

    def close(self):
        if getattr(self, "_ctx", None):
            L.lib().dg_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ncell(self):
        return self.mesh.ncell

    @property
    def shape(self):
        return (self.ncell, 5 * self.num_basis)

    def limit(self, U, Uprev, only_neighbor_avg=False):
        """PositiveLimiter::constructMinMax(U, Uprev) then apply(U, Uprev) on the GPU: bounds from
        Uprev, the limited U returned (element means unchanged)."""
        U = np.array(U, dtype=np.float64, copy=True)
        Uprev = np.ascontiguousarray(Uprev, dtype=np.float64)
        L.check(L.lib().dg_limit(self._ctx, L.dptr(U), L.dptr(Uprev), 0, int(bool(only_neighbor_avg))), "dg_limit")
        return U

    def viscous_eval(self, U, mu=1.0, prandtl=1.0):
        """ExplicitDiffusion::eval on the GPU (FP64): the viscous residual of U with viscosity mu and
        Prandtl number prandtl (the reference fixes both to 1)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.empty_like(U)
        L.check(L.lib().dg_viscous_residual(self._ctx, L.dptr(U), L.dptr(R), 0, float(mu), float(prandtl)),
                "dg_viscous_residual")
        return R

    def save_checkpoint(self, path, t=0.0, step=0):
        """Binary checkpoint of the device state with the time and step (dg_save_checkpoint)."""
        L.check(L.lib().dg_save_checkpoint(self._ctx, os.fsencode(path), float(t), int(step)), "dg_save_checkpoint")

    def load_checkpoint(self, path):
        """Restore a checkpoint written for the same mesh, order and volume rule; returns (t, step)."""
        t, step = ctypes.c_double(0.0), ctypes.c_int64(0)
        L.check(L.lib().dg_load_checkpoint(self._ctx, os.fsencode(path), ctypes.byref(t), ctypes.byref(step)),
                "dg_load_checkpoint")
        return t.value, step.value

    def autotune(self, dt):
        """Time the mixed form's candidates on the current state (which is restored) and keep the
        fastest: the tile queue of the persistent schedule, or the element kernel's shape of the
        two-launch schedule. Returns the JSON record of all candidates and the choice."""
        buf = ctypes.create_string_buffer(1 << 14)
        L.check(L.lib().dg_autotune(self._ctx, float(dt), buf, len(buf)), "dg_autotune")
        import json
        return json.loads(buf.value.decode())

    def set_element_shape(self, staged, ctas_per_sm=1):
        """Pin the two-launch element kernel's shape (a choice dg_autotune records)."""
        L.check(L.lib().dg_set_element_shape(self._ctx, int(bool(staged)), int(ctas_per_sm)), "dg_set_element_shape")

    def _state(self, U):
        U = L.as_f64(U)
        if U.shape != self.shape:
            U = U.reshape(self.shape)
        return U

    def _eval(self, U, t, part):
        U = self._state(U)
        R = np.empty(self.shape)
        L.check(L.lib().dg_residual(self._ctx, L.dptr(U), L.dptr(R), 0, float(t), part), "dg_residual")
        return R

    def eval(self, U, t=0.0):
        return self._eval(U, t, 0)

    def eval_cells(self, U, t=0.0):
        return self._eval(U, t, 1)

    def eval_internals(self, U, t=0.0):
        return self._eval(U, t, 2)

    def eval_boundarys(self, U, t=0.0):
        return self._eval(U, t, 3)

    def eval_device(self, U_ptr, R_ptr, t=0.0, part=0, stream=0):
        """Residual on device buffers (raw pointers, packed layout) enqueued on a CUDA stream."""
        L.check(L.lib().dg_residual_device(self._ctx, ctypes.c_void_p(U_ptr), ctypes.c_void_p(R_ptr),
                                           float(t), part, ctypes.c_void_p(stream)), "dg_residual_device")

    def mass(self):
        b = np.empty(self.shape)
        L.check(L.lib().dg_mass(self._ctx, L.dptr(b), 0), "dg_mass")
        return b

    def set_dirichlet(self, UD):
        UD = L.as_f64(UD).reshape(self.mesh.nface, self.nq_face, 5)
        L.check(L.lib().dg_set_dirichlet(self._ctx, L.dptr(UD)), "dg_set_dirichlet")

    def set_state(self, U):
        U = self._state(U)
        L.check(L.lib().dg_set_state(self._ctx, L.dptr(U), 0), "dg_set_state")

    def get_state(self):
        U = np.empty(self.shape)
        L.check(L.lib().dg_get_state(self._ctx, L.dptr(U), 0), "dg_get_state")
        return U

    def ssprk3(self, dt, nsteps=1, graph=False):
        f = L.lib().dg_ssprk3_graph if graph else L.lib().dg_ssprk3
        L.check(f(self._ctx, float(dt), int(nsteps)), "dg_ssprk3")

    def ssprk3_timed(self, dt, nsteps, nclass=5):
        """Step with CUDA events around every launch; returns {class: (total_ms, launches)}."""
        out = np.zeros(2 * nclass)
        L.check(L.lib().dg_ssprk3_timed(self._ctx, float(dt), int(nsteps), L.dptr(out), nclass), "dg_ssprk3_timed")
        return {k: (out[2 * k], int(out[2 * k + 1])) for k in range(nclass) if out[2 * k + 1] > 0}

    @property
    def stream(self):
        """Raw cudaStream_t of the context (wrap with torch.cuda.ExternalStream to time on it)."""
        return L.lib().dg_stream(self._ctx)

    def conservation(self):
        out = np.zeros(6)
        L.check(L.lib().dg_conservation(self._ctx, L.dptr(out)), "dg_conservation")
        return out

    def max_wave_speed(self):
        lam = ctypes.c_double(0.0)
        L.check(L.lib().dg_max_wave_speed(self._ctx, ctypes.byref(lam)), "dg_max_wave_speed")
        return lam.value

    def check_state(self):
        """Number of volume points with NaN/Inf, rho <= 0 or p <= 0 (0 when the state is physical)."""
        bad = ctypes.c_int64(0)
        rc = L.lib().dg_check_state(self._ctx, ctypes.byref(bad))
        if rc not in (L.DG_OK, -5):
            L.check(rc, "dg_check_state")
        return bad.value


class Ensemble(ExplicitConvection):
    """Independent solves on several meshes (of different sizes) in one context: the instances are
    laid end to end as one disconnected mesh, so each RK stage of all instances is one set of
    launches. State arrays are the instances' states concatenated in order."""

    def __init__(self, meshes, **kw):
        self.meshes = list(meshes)
        offs = np.cumsum([0] + [m.ncell for m in self.meshes])
        self._offsets = offs
        super().__init__(_Union(int(offs[-1])), _ensemble=self.meshes, **kw)
        got = np.zeros(len(self.meshes) + 1, dtype=np.int64)
        n = L.lib().dg_ensemble_offsets(self._ctx, L.iptr(got))
        assert n == len(self.meshes) and np.array_equal(got, offs)

    @property
    def offsets(self):
        return self._offsets

    def split(self, U):
        return [U[self._offsets[i]:self._offsets[i + 1]] for i in range(len(self.meshes))]

    def ssprk3(self, dt, nsteps=1, graph=False):
        dt = L.as_f64(np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(self.meshes),)))
        L.check(L.lib().dg_ssprk3_ensemble(self._ctx, L.dptr(dt), int(nsteps), int(bool(graph))), "dg_ssprk3_ensemble")


class _Union:
    def __init__(self, ncell):
        self.ncell = ncell


def launch_count():
    return int(L.lib().dg_launch_count())
