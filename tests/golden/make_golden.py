"""Generate the golden fixtures in this directory from the reference itself.

The reference has no golden vectors or known-answer tests of its own for this path (its tests/
directory holds print-only programs), so the fixtures are outputs of the reference's own
ExplicitConvection::eval and ComputingMesh, compiled from source into oracle/_ref/libfvedg_ref.so
by `make -C oracle ref`. Run from the repository root:

    python tests/golden/make_golden.py

Each fixture stores the flat mesh, the input coefficients U and the reference's residual R, plus
the reference's geometry and basis values, so the CPU tests can check the oracle (and the GPU
tests the kernels) without the reference being present.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from fve_dg_b200 import box_mesh, problems  # noqa: E402
from oracle.pyoracle import RefLib, RefMesh  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
# (order, tet rule, tri rule): the configurations' rules and the reference's Auto rules
CASES = [(1, 0, 1), (1, 2, 2), (2, 1, 2), (2, 2, 3), (3, 3, 3), (3, 4, 3), (4, 5, 3), (4, 6, 3)]
DIRICHLET = np.array([1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 0.5, 0.25, 1.0, 1.4])


def mesh_arrays(m):
    return dict(points=m.points, cells=m.cells, faces=m.faces, face_cells=m.face_cells,
                face_nodes1=m.face_nodes1, periodic=m.periodic, bc=m.bc, cell_faces=m.cell_faces,
                cell_cells=m.cell_cells)


def make(name, m, cases, seed, dirichlet=None, basis_tables=False):
    ref = RefLib()
    if dirichlet is not None:
        ref.set_dirichlet(dirichlet)
    rm = RefMesh.from_mesh(ref, m)
    g = rm.export()
    out = {f"mesh_{k}": v for k, v in mesh_arrays(m).items()}
    out.update({f"geo_{k}": v for k, v in g.items()})
    rng = np.random.default_rng(seed)
    for (P, qv, qf) in cases:
        U = problems.project(m, P, problems.density_wave())
        # inputs rounded to float32-representable values: exact in float64, smaller on disk
        U = (U + 1e-2 * rng.standard_normal(U.shape)).astype(np.float32).astype(np.float64)
        R = rm.eval(U, P, qv, qf)
        out[f"U_P{P}_{qv}_{qf}"] = U
        out[f"R_P{P}_{qv}_{qf}"] = R
    if basis_tables:  # basis values of every order at the Degree9Points57 points
        pts, _ = ref.quad(0, 6)
        for P in (1, 2, 3, 4):
            phi, grad = ref.basis(P, pts)
            out[f"basisq_P{P}_phi"] = phi
            out[f"basisq_P{P}_grad"] = grad
        out["basisq_pts"] = pts
    if dirichlet is not None:
        out["dirichlet"] = dirichlet
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def main():
    make("periodic_n2.npz", box_mesh(2, jitter=0.1, seed=11), CASES, seed=1, basis_tables=True)
    make("dirichlet_n2.npz", box_mesh(2, jitter=0.1, seed=12, periodic=(0, 0, 0), bc="Dirichlet"),
         [(1, 0, 1), (2, 1, 2), (3, 3, 3)], seed=2, dirichlet=DIRICHLET)
    make("pseudo3dz_n2.npz", box_mesh(2, jitter=0.1, seed=13, periodic=(1, 1, 0), bc="Pseudo3DZ"),
         [(2, 1, 2), (4, 5, 3)], seed=3)


if __name__ == "__main__":
    main()
