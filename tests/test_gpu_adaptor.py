"""GPU: the C++ drop-in ExplicitConvectionGPU (include/ExplicitConvectionGPU.h), compiled against
the reference's headers, against the reference's own ExplicitConvection on the same ComputingMesh
(Dirichlet and Pseudo3DZ boundaries, P1..P4, eval and its three parts)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "adaptor_check")


@pytest.mark.skipif(not os.path.exists(BIN), reason="adaptor_check is built only where the reference sources are")
def test_cpp_drop_in_matches_reference():
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")
    assert r.stdout.count("rel L2") == 2 * 5 * 4
