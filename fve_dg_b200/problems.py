"""Problem setups for the explicit Euler path: initial states, L2 projection onto the modal basis,
CFL time step and error norms. The reference keeps these in its example drivers
(examples/*/problem.h, DGBasisEvaluator::func2coef in include/DG/DG_Basis/DG_Basis_Evaluator.h:33-59,
examples/Vortex/tools.h:35-68); the 3D problems below are new and stated in code:

  * isentropic vortex: free stream rho=1, u=(1,1,0), p=1, gamma=1.4; a vortex of strength beta
    around the line through `center` along unit `axis`: with d_perp the offset from the axis and
    r^2 = |d_perp|^2, du = beta/(2 pi) exp((1-r^2)/2) (axis x d_perp),
    T = 1 - (gamma-1) beta^2/(8 gamma pi^2) exp(1-r^2), rho = T^(1/(gamma-1)), p = rho^gamma.
  * density wave: rho = 1 + A sin(2 pi k.(x - u t)), u = (1, 0.5, 0.25), p = 1 (exact solution
    for all t on a periodic box).
  * Taylor-Green vortex: rho = 1, u = (sin x cos y cos z, -cos x sin y cos z, 0),
    p = p0 + (cos 2x + cos 2y)(cos 2z + 2)/16, p0 = 1/(gamma Ma^2) so that Ma = U0/c0 = 0.1.
"""
import ctypes

import numpy as np

from . import _lib as L


def quad_rule(kind, rule_id):
    n = L.lib().dg_quad_rule(kind, rule_id, None, None)
    if n <= 0:
        raise L.DGError(n, "dg_quad_rule")
    pts = np.zeros((n, 3 if kind == 0 else 2))
    w = np.zeros(n)
    L.lib().dg_quad_rule(kind, rule_id, L.dptr(pts), L.dptr(w))
    return pts, w


def auto_rules(order):
    qv, qf = ctypes.c_int(), ctypes.c_int()
    L.check(L.lib().dg_auto_rules(order, ctypes.byref(qv), ctypes.byref(qf)), "dg_auto_rules")
    return qv.value, qf.value


def num_basis(order):
    return (order + 1) * (order + 2) * (order + 3) // 6


def basis(order, xyz):
    xyz = L.as_f64(xyz).reshape(-1, 3)
    nb = num_basis(order)
    phi = np.zeros((xyz.shape[0], nb))
    grad = np.zeros((xyz.shape[0], nb, 3))
    L.check(L.lib().dg_basis(order, xyz.shape[0], L.dptr(xyz), L.dptr(phi), L.dptr(grad)), "dg_basis")
    return phi, grad


def physical_points(mesh, ref_pts):
    """x = p0 (1 - xi1 - xi2 - xi3) + p1 xi1 + p2 xi2 + p3 xi3 for every cell and reference point:
    shape (ncell, npts, 3) (CompTetrahedron::transform_to_physical, ComputingMesh.cpp:136-142)."""
    P = mesh.points[mesh.cells]  # (nc, 4, 3)
    lam = np.concatenate([1.0 - ref_pts.sum(axis=1, keepdims=True), ref_pts], axis=1)  # (nq, 4)
    return np.einsum("qa,cad->cqd", lam, P)


def project(mesh, order, func, rule=None):
    """L2 projection c_k = sum_g f(x_g) phi_k w_g / sum_g phi_k^2 w_g per cell (func2coef,
    DG_Basis_Evaluator.h:33-59; by default with the reference's Auto tet rule for the order).
    func maps (..., 3) points to (..., 5) conserved states. Returns (ncell, 5*Nb)."""
    if rule is None:
        rule = auto_rules(order)[0]
    pts, w = quad_rule(0, rule)
    phi, _ = basis(order, pts)
    X = physical_points(mesh, pts)
    F = func(X)  # (nc, nq, 5)
    ld = np.longdouble  # the reference sums in long double (Scalar128)
    phi, w = phi.astype(ld), w.astype(ld)
    diag = (phi * phi * w[:, None]).sum(axis=0)  # (nb,)
    coef = np.einsum("cqk,qb,q->cbk", F.astype(ld), phi, w) / diag[None, :, None]
    return np.ascontiguousarray(coef.astype(np.float64).reshape(mesh.ncell, -1))


def conserved(rho, u, v, w, p, gamma):
    return np.stack([rho, rho * u, rho * v, rho * w, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)], axis=-1)


def isentropic_vortex(center=(5.0, 5.0, 5.0), axis=(0.0, 0.0, 1.0), beta=5.0, gamma=1.4,
                      uinf=(1.0, 1.0, 0.0), t=0.0, period=None):
    c = np.asarray(center, dtype=float)
    a = np.asarray(axis, dtype=float)
    a = a / np.linalg.norm(a)
    ui = np.asarray(uinf, dtype=float)

    def f(X):
        d = X - (c + ui * t)
        if period is not None:
            d = d - period * np.round(d / period)
        dpar = (d @ a)[..., None] * a
        dp = d - dpar
        r2 = (dp * dp).sum(axis=-1)
        swirl = np.cross(a, dp)
        amp = beta / (2 * np.pi) * np.exp(0.5 * (1.0 - r2))
        vel = ui + amp[..., None] * swirl
        T = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * np.pi ** 2) * np.exp(1.0 - r2)
        rho = T ** (1.0 / (gamma - 1.0))
        p = rho ** gamma
        return conserved(rho, vel[..., 0], vel[..., 1], vel[..., 2], p, gamma)

    return f


def density_wave(A=0.2, k=(1.0, 1.0, 1.0), vel=(1.0, 0.5, 0.25), p=1.0, gamma=1.4, t=0.0):
    k = np.asarray(k, dtype=float)
    u = np.asarray(vel, dtype=float)

    def f(X):
        rho = 1.0 + A * np.sin(2 * np.pi * ((X - u * t) @ k))
        one = np.ones_like(rho)
        return conserved(rho, u[0] * one, u[1] * one, u[2] * one, p * one, gamma)

    return f


def taylor_green(mach=0.1, gamma=1.4):
    p0 = 1.0 / (gamma * mach * mach)

    def f(X):
        x, y, z = X[..., 0], X[..., 1], X[..., 2]
        u = np.sin(x) * np.cos(y) * np.cos(z)
        v = -np.cos(x) * np.sin(y) * np.cos(z)
        w = np.zeros_like(x)
        p = p0 + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0
        return conserved(np.ones_like(x), u, v, w, p, gamma)

    return f


def cfl_dt(cfl, edge, order, lam_max):
    """dt = CFL h / ((2P + 1) lambda_max) with the reference drivers' length scale
    h = edge / sqrt(3) / 3 for a box of cubes of side `edge` cut into tetrahedra
    (examples/TaylerGreenVortex/TGBatch.cpp:358-383)."""
    h = edge / np.sqrt(3.0) / 3.0
    return cfl * h / ((2 * order + 1) * lam_max)


def l2_errors(mesh, order, U, Uref=None, exact=None, rule=None, momentum_norm=False):
    """Relative L2 error per conserved variable at volume quadrature points
    (examples/Vortex/tools.h:35-68): ||U - Uref|| / ||Uref||, against a coefficient array Uref
    or an exact-solution function `exact`. With momentum_norm, the three momentum components are
    divided by the norm of the whole momentum field, ||rho u|| = sqrt(sum_i ||rho u_i||^2), instead of
    their own norms: a component that is nearly zero everywhere (rho w of a Taylor-Green vortex starts
    at 0) then gets an error on the flow's own scale rather than a ratio of two tiny numbers."""
    if rule is None:
        rule = auto_rules(order)[0]
    pts, w = quad_rule(0, rule)
    phi, _ = basis(order, pts)
    nb = num_basis(order)
    geo = mesh.compute_geometry()
    dj = geo["detj"]
    Uq = np.einsum("qb,cbk->cqk", phi, U.reshape(-1, nb, 5))
    if Uref is not None:
        Rq = np.einsum("qb,cbk->cqk", phi, Uref.reshape(-1, nb, 5))
    else:
        Rq = exact(physical_points(mesh, pts))
    wq = w[None, :, None] * dj[:, None, None]
    num = np.sqrt((wq * (Uq - Rq) ** 2).sum(axis=(0, 1)))
    den = np.sqrt((wq * Rq ** 2).sum(axis=(0, 1)))
    if momentum_norm:
        den[1:4] = np.sqrt((den[1:4] ** 2).sum())
    return num / np.maximum(den, 1e-300)
