"""Solution I/O: the reference's text solution format, and a binary checkpoint/restart.

Text format, as examples/Eular1D/Sod1D/Riemann1D.cpp:249-286 writes it and
examples/Vortex/tools.h:72-129 reads it: one line per (cell, volume quadrature point), cells in
order and the points of each cell in rule order; on each line the physical point ``x y z`` and then,
for the conserved variables rho, rho u, rho v, rho w, rho E in turn, the computed value and the exact
one (``Uh_k Us_k``); every number with 16 significant digits (``std::setprecision(16)``, i.e.
``%.16g``), separated by two spaces. Files are named ``<dir>/solution/T_<step>_N_<mesh size>.txt``
(src/base/FilesystemManager.cpp:14-17). Reading projects the point values back onto the modal basis
with the rule's weights, c_k = sum_g v_g phi_k(x_g) w_g / sum_g phi_k(x_g)^2 w_g (tools.h:96-129).

The binary checkpoint (``ExplicitConvection.save_checkpoint`` / ``load_checkpoint``) is written by
the library (``dg_save_checkpoint`` / ``dg_load_checkpoint`` in include/dg_gpu.h).
"""
import os

import numpy as np

from . import problems


def solution_file_name(base_dir, time_step, mesh_size):
    return os.path.join(base_dir, "solution", f"T_{int(time_step)}_N_{int(mesh_size)}.txt")


def physical_points(mesh, quad_vol):
    """Physical positions of the volume rule's points in every cell, (ncell, nq, 3), computed as
    CompTetrahedron::transform_to_physical (src/Mesh/ComputingMesh.cpp:136-142)."""
    pts, _ = problems.quad_rule(0, quad_vol)
    P = mesh.points[mesh.cells][:, None]  # (ncell, 1, 4, 3)
    x0, x1, x2 = (pts[None, :, i, None] for i in range(3))
    return P[..., 0, :] * (1 - x0 - x1 - x2) + P[..., 1, :] * x0 + P[..., 2, :] * x1 + P[..., 3, :] * x2


def point_values(U, order, quad_vol):
    """Conserved states at the volume rule's points, (ncell, nq, 5)."""
    pts, _ = problems.quad_rule(0, quad_vol)
    phi, _ = problems.basis(order, pts)
    return np.einsum("gb,ebk->egk", phi, np.asarray(U, dtype=np.float64).reshape(len(U), -1, 5))


def write_solution(path, mesh, U, order, quad_vol, exact=None):
    """Write the state U (ncell, 5 Nb) in the reference's text format; `exact` maps (..., 3) points
    to (..., 5) states for the Us columns (zeros when None)."""
    X = physical_points(mesh, quad_vol)
    Uh = point_values(U, order, quad_vol)
    Us = np.zeros_like(Uh) if exact is None else np.asarray(exact(X), dtype=np.float64).reshape(Uh.shape)
    cols = np.empty(X.shape[:2] + (13,))
    cols[..., :3] = X
    cols[..., 3::2] = Uh
    cols[..., 4::2] = Us
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    np.savetxt(path, cols.reshape(-1, 13), fmt="%.16g", delimiter="  ")


def read_solution(path, mesh, order, quad_vol):
    """Read a solution file of the reference's text format back into coefficients (ncell, 5 Nb) by
    the projection of tools.h:96-129. Returns (coefficients, exact point values)."""
    pts, w = problems.quad_rule(0, quad_vol)
    phi, _ = problems.basis(order, pts)
    nq = len(w)
    data = np.loadtxt(path, ndmin=2)
    if data.shape != (mesh.ncell * nq, 13):
        raise ValueError(f"{path}: expected {mesh.ncell * nq} lines of 13 numbers, found {data.shape}")
    Uh = data[:, 3::2].reshape(mesh.ncell, nq, 5)
    Us = data[:, 4::2].reshape(mesh.ncell, nq, 5)
    norm = (phi * phi * w[:, None]).sum(axis=0)                   # sum_g phi_k^2 w_g
    coef = np.einsum("egk,gb,g->ebk", Uh, phi, w) / norm[None, :, None]
    return coef.reshape(mesh.ncell, -1), Us
