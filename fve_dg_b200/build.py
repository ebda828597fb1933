"""Build the native library in-tree: fve_dg_b200/libfvedg_b200.so (host C++ + sm_100a CUDA).

Host sources are compiled with g++ (-O3 -mfma; geometry from raw topology then agrees with the
reference's to a few ulp, connectivity and face maps bit for bit); CUDA sources with nvcc for
sm_100a only. The oracle
(oracle/liboracle.so) and, when the reference sources are present, oracle/_ref/libfvedg_ref.so
are built by oracle/Makefile; `build_all()` drives both.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libfvedg_b200.so")
OBJ = os.path.join(PKG, "_build")
HOST_SRCS = ["host_mesh.cpp", "host_tables.cpp", "host_partition.cpp"]
CUDA_SRCS = ["dg_api.cu"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _run(cmd):
    print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose_ptxas=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".inc"))]
    headers.append(os.path.join(ROOT, "include", "dg_gpu.h"))
    objs = []
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    for src in HOST_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + headers):
            _run([CXX, "-std=c++17", "-O3", "-mavx2", "-mfma", "-ffp-contract=fast", "-fPIC", "-Wall"] + inc + ["-c", s, "-o", o])
        objs.append(o)
    nvcc = _nvcc()
    for src in CUDA_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", CXX] + GENCODE + inc
            if verbose_ptxas:
                cmd.append("-Xptxas=-v")
            _run(cmd + ["-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([nvcc, "-shared", "-ccbin", CXX] + GENCODE + ["-o", LIB] + objs + ["-lcudart"])
    return LIB


def build_oracle(with_ref=None):
    """Build oracle/liboracle.so, and oracle/_ref/libfvedg_ref.so when the reference is present."""
    ref_dir = os.environ.get("FVEDG_REFERENCE", "/root/reference")
    if with_ref is None:
        with_ref = os.path.isdir(os.path.join(ref_dir, "src", "DG"))
    target = "ref" if with_ref else "all"
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), target, "REF=" + ref_dir, "-j8"])


def build_all(force=False):
    build(force=force)
    build_oracle()


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
