"""Build step: regenerate quad_tables.inc, the quadrature rules the DG path integrates with.

The rules must be the reference's own, bit for bit, or the residual cannot match it. This script
reads them out of the reference's quadrature headers through oracle/_ref/libfvedg_ref.so (the
reference compiled from source by `make -C oracle ref`) and writes every double as a C99 hex
float, so the committed file carries the exact bits. Provenance of each rule:

  tet (reference points/weights from include/GaussQuadrature/QuadTetHighOrder.h, generated by
  scripts/codegen/QuadTet.py from data/QuadData/NME_6313_cubature_tetra_p*_n*.dat, weights / 6;
  Degree5Points15 from include/GaussQuadrature/QuadTetLowerOrder.h:1):
    0 Degree2Points4   1 Degree4Points11  2 Degree5Points15  3 Degree6Points23
    4 Degree7Points31  5 Degree8Points44  6 Degree9Points57  7 Degree11Points94 (the P5 Auto rule)
  tri (include/GaussQuadrature/QuadTriLowerOrder.h:1-69 and QuadTriHighOrder.h:1-24, the latter
  from data/QuadData/rotationalsymmetry.txt, weights / 2):
    0 Degree3Points4   1 Degree3Points6   2 Degree4Points7 (exact to degree 5)
    3 Degree10Points24 (rotationally symmetric only; exact to about 1e-10)
    4 Degree13Points36 (QuadTriHighOrder.h, the P5 Auto rule)

Run from the repository root after building the reference library:
    python fve_dg_b200/csrc/gen_quad_tables.py
"""
import ctypes
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
TET = ["Degree2Points4", "Degree4Points11", "Degree5Points15", "Degree6Points23",
       "Degree7Points31", "Degree8Points44", "Degree9Points57", "Degree11Points94"]
TRI = ["Degree3Points4", "Degree3Points6", "Degree4Points7", "Degree10Points24", "Degree13Points36"]
TET_DEG = [2, 4, 5, 6, 7, 8, 9, 11]
TRI_DEG = [3, 3, 5, 10, 13]


def main():
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libfvedg_ref.so"))
    P = ctypes.POINTER(ctypes.c_double)
    out = ["/* Generated by gen_quad_tables.py from the reference's quadrature tables. Do not edit.",
           " * Layout per rule: npts rows of (x, y, z, w) for tets and (x, y, w) for triangles. */",
           "#ifndef FVEDG_QUAD_TABLES_INC", "#define FVEDG_QUAD_TABLES_INC", ""]
    tet_n, tri_n = [], []
    for i, name in enumerate(TET):
        n = lib.fveref_quad_tet(i, None, None)
        pts = (ctypes.c_double * (3 * n))()
        w = (ctypes.c_double * n)()
        lib.fveref_quad_tet(i, pts, w)
        tet_n.append(n)
        out.append(f"/* tet {i}: {name}, degree {TET_DEG[i]} */")
        out.append(f"static const double fvedg_tet_rule{i}[{4 * n}] = {{")
        for g in range(n):
            vals = [pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], w[g]]
            out.append("  " + ", ".join(float(v).hex() for v in vals) + ",")
        out.append("};")
    for i, name in enumerate(TRI):
        n = lib.fveref_quad_tri(i, None, None)
        pts = (ctypes.c_double * (2 * n))()
        w = (ctypes.c_double * n)()
        lib.fveref_quad_tri(i, pts, w)
        tri_n.append(n)
        out.append(f"/* tri {i}: {name}, degree {TRI_DEG[i]} */")
        out.append(f"static const double fvedg_tri_rule{i}[{3 * n}] = {{")
        for g in range(n):
            vals = [pts[2 * g], pts[2 * g + 1], w[g]]
            out.append("  " + ", ".join(float(v).hex() for v in vals) + ",")
        out.append("};")
    out.append(f"#define FVEDG_NUM_TET_RULES {len(TET)}")
    out.append(f"#define FVEDG_NUM_TRI_RULES {len(TRI)}")
    out.append("static const int fvedg_tet_npts[FVEDG_NUM_TET_RULES] = {" + ", ".join(map(str, tet_n)) + "};")
    out.append("static const int fvedg_tri_npts[FVEDG_NUM_TRI_RULES] = {" + ", ".join(map(str, tri_n)) + "};")
    out.append("static const int fvedg_tet_degree[FVEDG_NUM_TET_RULES] = {" + ", ".join(map(str, TET_DEG)) + "};")
    out.append("static const int fvedg_tri_degree[FVEDG_NUM_TRI_RULES] = {" + ", ".join(map(str, TRI_DEG)) + "};")
    out.append("static const double* const fvedg_tet_rules[FVEDG_NUM_TET_RULES] = {" +
               ", ".join(f"fvedg_tet_rule{i}" for i in range(len(TET))) + "};")
    out.append("static const double* const fvedg_tri_rules[FVEDG_NUM_TRI_RULES] = {" +
               ", ".join(f"fvedg_tri_rule{i}" for i in range(len(TRI))) + "};")
    out.append("#endif")
    path = os.path.join(HERE, "quad_tables.inc")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
    print("wrote", path, "tet", tet_n, "tri", tri_n, file=sys.stderr)


if __name__ == "__main__":
    main()
