"""CPU: the reference's text solution format (Riemann1D.cpp:249-286 writes it, Vortex/tools.h:72-129
reads it) - layout, number format and the write/read round trip."""
import numpy as np
import pytest

from fve_dg_b200 import box_mesh, io, problems


@pytest.mark.parametrize("P,qv", [(1, 0), (2, 1), (3, 3), (4, 5)])
def test_text_round_trip(tmp_path, P, qv):
    m = box_mesh(2, jitter=0.1, seed=2)
    f = problems.density_wave()
    U = problems.project(m, P, f, rule=qv)
    path = io.solution_file_name(str(tmp_path), 7, 2)
    assert path.endswith("solution/T_7_N_2.txt")
    io.write_solution(path, m, U, P, qv, exact=f)
    V, Us = io.read_solution(path, m, P, qv)
    # 16 significant digits per number, and the rule integrates phi_j phi_k exactly: the coefficients
    # come back to round-off
    assert np.abs(V - U).max() <= 1e-13 * np.abs(U).max()
    X = io.physical_points(m, qv)
    assert np.allclose(Us, f(X), rtol=1e-15, atol=1e-15)


def test_text_layout(tmp_path):
    m = box_mesh(1)
    P, qv = 1, 0
    U = problems.project(m, P, problems.density_wave(), rule=qv)
    path = str(tmp_path / "s.txt")
    io.write_solution(path, m, U, P, qv)
    lines = open(path).read().splitlines()
    assert len(lines) == m.ncell * 4                       # Degree2Points4: 4 points per cell
    fields = lines[0].split("  ")
    assert len(fields) == 13                               # x y z, then (Uh, Us) for 5 variables
    x = io.physical_points(m, qv)[0, 0]
    assert fields[:3] == ["%.16g" % v for v in x]
    assert fields[4] == "0"                                # no exact solution given
