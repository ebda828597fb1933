"""CPU: meshes and initial data made by the oracle alone, against the product's.

- The oracle's own periodic Kuhn box (ref_harness.cpp build_box, an independent restatement) is the
  product's box_mesh array for array, so the reference's CPU timings run on the same mesh without
  loading the product.
- The product's L2 projection (problems.project) against the reference's own
  DGBasisEvaluator<P>::func2coef (include/DG/DG_Basis/DG_Basis_Evaluator.h:33-59).
- The reference's own mesh route, OrthHexMesh -> split_hex6_scan -> rebuild_cell_topology ->
  ComputingMesh(const GeneralMesh&) (include/Mesh/OrthHexMesh.h:7-106, src/Mesh/GeneralMesh.cpp:4-129,
  src/Mesh/ComputingMesh.cpp:205-263): its node orders (unordered_set iteration) and face numbering
  given to the product as raw topology give the reference's connectivity and face maps bit for bit.
- bench.py's reference arm never loads the product's library.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, rel_l2
from fve_dg_b200 import Mesh, box_mesh, problems
from oracle.pyoracle import RefLib, ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="reference library not built")

KEYS = ("points", "cells", "faces", "face_cells", "face_nodes1", "periodic", "bc", "cell_faces", "cell_cells")


@pytest.mark.parametrize("kw", [dict(n=3, jitter=0.1), dict(n=4, hi=(2 * np.pi,) * 3),
                                dict(n=5, hi=(10.0,) * 3, jitter=0.07, seed=9),
                                dict(n=3, jitter=0.1, periodic=(1, 1, 0), bc=5),
                                dict(n=2, jitter=0.1, periodic=(0, 0, 0), bc=0)])
def test_oracle_box_is_the_product_box(kw):
    ref = RefLib()
    rm = ref.box(**kw)
    m = box_mesh(**kw)
    for k in KEYS:
        a, b = getattr(rm, k), getattr(m, k)
        assert a.shape == b.shape and np.array_equal(a, b.astype(a.dtype)), k


PROBLEMS = {
    "taylor_green": (problems.taylor_green(), [0.1, 1.4], 2 * np.pi, 0.0),
    "density_wave": (problems.density_wave(), [0.2, 1.0, 1.0, 1.0, 1.0, 0.5, 0.25, 1.0, 1.4], 1.0, 0.1),
    "vortex": (problems.isentropic_vortex(period=10.0), [5, 5, 5, 0, 0, 1, 5, 1.4, 1, 1, 0, 10.0], 10.0, 0.0),
}


@pytest.mark.parametrize("name", sorted(PROBLEMS))
@pytest.mark.parametrize("P", [0, 1, 2, 3, 4, 5])
def test_projection_matches_reference_func2coef(name, P):
    func, prm, L, jit = PROBLEMS[name]
    ref = RefLib()
    rm = ref.box(3, hi=(L,) * 3, jitter=jit)
    m = box_mesh(3, hi=(L,) * 3, jitter=jit)
    Ur = rm.project(P, name, prm)
    Up = problems.project(m, P, func)
    assert rel_l2(Up, Ur) < 1e-14


def orthhex_product_mesh(rm):
    return Mesh(rm.points, rm.cells, rm.faces, rm.face_cells, bc=rm.bc)


@pytest.mark.parametrize("n", [2, 3, 5])
def test_reference_mesh_route_connectivity_and_face_maps(n):
    ref = RefLib()
    rm = ref.orthhex(n, hi=(1.0, 2.0, 0.5), bc_z=5, bc_side=0)
    assert rm.ncell == 6 * n ** 3
    g_ref = rm.export()
    assert np.array_equal(g_ref["face_cells"], rm.face_cells)
    m = orthhex_product_mesh(rm)
    g = m.compute_geometry()
    assert np.array_equal(g["natural"], g_ref["natural"])  # face maps of both sides, bit for bit
    assert np.all((g["normal"] * g_ref["normal"]).sum(axis=1) > 0.999)  # orientation out of cells[0]
    eps = np.finfo(float).eps
    assert np.abs(g["normal"] - g_ref["normal"]).max() <= 4 * eps
    assert np.abs(g["area"] - g_ref["area"]).max() <= 4 * eps * g_ref["area"].max()
    assert np.abs(g["detj"] - g_ref["detj"]).max() <= 4 * eps * g_ref["detj"].max()
    assert np.abs(g["invjac"] - g_ref["invjac"]).max() <= 8 * eps * np.abs(g_ref["invjac"]).max()
    # the node orders come from the reference's unordered_set iteration: no cell lists its nodes in
    # ascending order (the Kuhn generator's cells mostly do), and the face maps cover most of the 24
    assert not (np.diff(rm.cells, axis=1) > 0).all(axis=1).any()
    perm = m.face_perms()
    assert np.unique(perm[:, 0]).size >= 12


def test_reference_arm_loads_only_oracle_libraries():
    code = (
        "import sys, json; sys.path.insert(0, %r); sys.argv = ['bench.py', '--impl', 'reference', '--config', "
        "'vortex', '--steps', '1', '--warmup', '3']\n"
        "import runpy\n"
        "runpy.run_path(%r, run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libfvedg_b200' not in maps, 'product library loaded'\n"
        "assert 'libfvedg_ref' in maps\n"
        "assert 'fve_dg_b200' not in ' '.join(sys.modules), 'product package imported'\n"
        "print('ARM-OK')\n" % (ROOT, os.path.join(ROOT, "bench.py")))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ARM-OK" in r.stdout
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][0]
    import json
    d = json.loads(line)
    assert d["impl"] == "reference" and d["value"] > 0 and d["config"]["tets"] == 3072
