"""GPU: the C++ drop-ins, compiled against the reference's headers, against the reference's own
classes on the same ComputingMesh (Kuhn boxes with Dirichlet and Pseudo3DZ boundaries, and the
reference's own OrthHexMesh -> split_hex6_scan -> ComputingMesh(GeneralMesh) box with both):
- ExplicitConvectionGPU (include/ExplicitConvectionGPU.h) against ExplicitConvection: P1..P4 with
  the configurations' rules, P0, P3 and P5 with the Auto rules; eval and its three parts;
- ExplicitDiffusionGPU (include/ExplicitDiffusionGPU.h) against ExplicitDiffusion: P1..P3;
- PositiveLimiterGPU (include/PositiveLimiterGPU.h) against PositiveLimiter: P2, P3, both bound
  modes, on states the limiter changes."""
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
    assert r.stdout.count(" part ") == 3 * 7 * 4
    assert r.stdout.count(" diffusion ") == 3 * 3
    assert r.stdout.count(" limiter ") == 3 * 3
    assert r.stdout.count("orthhex-split6 ") == 7 * 4 + 3 + 3
