"""CPU: the bench's roofline bookkeeping. Every kernel class the bench can time (both forms, both
schedules, the limiter, the viscous residual of Navier-Stokes stepping) has an algorithmic byte
count, and the roofline object carries the contract's keys whichever class dominates."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("P,nqf", [(1, 6), (2, 7), (3, 24), (4, 24)])
def test_every_kernel_class_has_bytes(P, nqf):
    b = load_bench()
    ncell, nface = 6 * 16 ** 3, 12 * 16 ** 3
    for names in b.KNAMES.values():
        for name in names.values():
            assert b.kernel_bytes(name, P, ncell, nface, nqf) > 0, name
    with pytest.raises(ValueError):
        b.kernel_bytes("no_such_kernel", P, ncell, nface, nqf)


@pytest.mark.parametrize("key", [("fp64", "two-launch"), ("mixed", "two-launch"), ("mixed", "persistent")])
def test_roofline_for_each_dominant_class(key):
    b = load_bench()
    P, ncell, nface, nqf, nb = 3, 6 * 16 ** 3, 12 * 16 ** 3, 24, 20
    classes = list(b.KNAMES[key])
    for dom in classes:  # each class in turn takes the most time
        kt = {k: ((10.0 if k == dom else 1.0) * 3, 3) for k in classes}
        r = b.make_roofline(kt, key[0], key[1], P, ncell, nface, nqf, nb, "tgv")
        for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
            assert k in r, k
        assert r["kernel"] == b.KNAMES[key][dom]
        assert r["achieved"] > 0 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
