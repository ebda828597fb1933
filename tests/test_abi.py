"""CPU: the C-ABI libraries load and export every symbol their headers declare; host-only entry
points (mesh, geometry, face maps, tables) work without a GPU and reject malformed input."""
import ctypes
import os
import re

import numpy as np
import pytest

from fve_dg_b200 import Mesh, box_mesh
from fve_dg_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header, prefix):
    txt = open(os.path.join(ROOT, header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(" + prefix + r"[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_entry_point_is_exported():
    names = declared("include/dg_gpu.h", "dg_")
    assert len(names) >= 30
    lib = ctypes.CDLL(L.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(L.exported_symbols()) <= set(names)


def test_oracle_libraries_export_their_api():
    from oracle import pyoracle
    o = ctypes.CDLL(pyoracle.ORACLE_SO)
    for n in declared("oracle/dg_oracle.h", "orc_"):
        assert hasattr(o, n), n
    if pyoracle.ref_available():
        r = ctypes.CDLL(pyoracle.REF_SO)
        for n in ("fveref_mesh_create", "fveref_eval", "fveref_ssprk3", "fveref_mass", "fveref_basis",
                  "fveref_quad_tet", "fveref_quad_tri", "fveref_mesh_export"):
            assert hasattr(r, n), n


def test_status_strings_and_capacity():
    lib = L.lib()
    for code in range(0, -9, -1):
        assert lib.dg_status_string(code)
    assert lib.dg_static_scratch_capacity() == 4 << 20


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_box_mesh_invariants(n):
    m = box_mesh(n, jitter=0.1, seed=n)
    assert m.ncell == 6 * n ** 3
    assert m.nface == 12 * n ** 3            # periodic: every face shared by two cells
    assert np.all(m.face_cells[:, 1] >= 0)
    fc = m.face_cells
    deg = np.bincount(fc.ravel(), minlength=m.ncell)
    assert np.all(deg == 4)
    # neighbour symmetry of cell_cells
    cc = m.cell_cells
    for c in range(m.ncell):
        for nb in cc[c]:
            assert c in cc[nb]
    # periodic faces pair translated node sets
    per = m.periodic.astype(bool)
    assert per.sum() == 6 * n * n
    # jitter touches interior vertices only
    g = box_mesh(n)
    nv = n + 1
    ijk = np.stack(np.meshgrid(np.arange(nv), np.arange(nv), np.arange(nv), indexing="ij"), -1).reshape(-1, 3)[:, ::-1]
    on_boundary = np.any((ijk == 0) | (ijk == n), axis=1)
    assert np.array_equal(m.points[on_boundary], g.points[on_boundary])


def test_non_periodic_box_boundary_faces():
    n = 3
    m = box_mesh(n, periodic=(1, 0, 1), bc="Dirichlet")
    bnd = m.face_cells[:, 1] < 0
    assert bnd.sum() == 2 * 2 * n * n          # two y-planes of 2 n^2 triangles
    assert np.all(m.bc[bnd] == 0)


def test_face_maps_and_geometry_are_consistent():
    m = box_mesh(2, jitter=0.1, seed=4)
    perm = m.face_perms()
    assert perm.min() >= 0 and perm.max() < 24
    g = m.compute_geometry()
    assert np.allclose(np.linalg.norm(g["normal"], axis=1), 1.0, atol=1e-14)
    assert np.all(g["area"] > 0) and np.all(g["detj"] > 0)
    # the normal points from cells[0] to cells[1] for interior, non-periodic faces
    cen = g["centroid"]
    inner = m.periodic == 0
    d = cen[m.face_cells[inner, 1]] - cen[m.face_cells[inner, 0]]
    assert np.all((g["normal"][inner] * d).sum(axis=1) > 0)
    # total volume of the unit box
    assert np.isclose(g["detj"].sum() / 6.0, 1.0, rtol=1e-12)


def test_malformed_meshes_are_rejected():
    m = box_mesh(2)
    bad = Mesh(m.points, m.cells, m.faces, m.face_cells.copy(), m.face_nodes1, m.periodic, m.bc)
    bad.face_cells[0, 0] = m.ncell + 5           # index out of range
    with pytest.raises(L.DGError) as e:
        bad.face_perms()
    assert e.value.code == -2
    bad = Mesh(m.points, m.cells, m.faces, m.face_cells.copy(), m.face_nodes1, m.periodic, m.bc)
    bad.face_cells[0, 1] = bad.face_cells[1, 1]  # a cell with five faces, another with three
    with pytest.raises(L.DGError):
        bad.face_perms()
    bad = Mesh(m.points, m.cells, m.faces.copy(), m.face_cells, m.face_nodes1, m.periodic, m.bc)
    bad.faces[0] = [0, 0, 1]                     # face nodes not a face of its cell
    with pytest.raises(L.DGError):
        bad.face_perms()
    g = m.compute_geometry()
    nat = g["natural"].copy()
    nat[0, 0, 0] = [0.5, 0.0, 0.0]               # not a vertex of the reference tet
    geo = dict(natural=nat, normal=g["normal"], area=g["area"], invjac=g["invjac"], detj=g["detj"])
    bad = Mesh(m.points, m.cells, m.faces, m.face_cells, m.face_nodes1, m.periodic, m.bc, geometry=geo)
    with pytest.raises(L.DGError):
        bad.face_perms()


def test_c_header_compiles_as_c_and_links():
    """include/dg_gpu.h is plain C: a C program that includes it and takes the address of every
    entry point compiles with gcc (C11) and links against the library, as an FFI consumer would."""
    import re
    import shutil
    import subprocess
    import tempfile
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "dg_gpu.h")).read()
    names = sorted(set(re.findall(r"\b(dg_[a-z0-9_]+)\s*\(", header)))
    body = "\n".join(f"    p[n++] = (void*)&{nm};" for nm in names)
    src = f'#include "dg_gpu.h"\n#include <stdio.h>\nint main(void) {{\n    void* p[{len(names) + 1}]; int n = 0;\n{body}\n    printf("%d %p\\n", n, p[0]);\n    return 0;\n}}\n'
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "abi.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "abi")
        lib = os.path.join(root, "fve_dg_b200")
        r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(root, "include"), c, "-o", exe,
                            "-L", lib, "-lfvedg_b200", "-Wl,-rpath," + lib], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    assert len(names) >= 30
