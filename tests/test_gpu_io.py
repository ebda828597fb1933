"""GPU: binary checkpoint / restart of the device state (dg_save_checkpoint / dg_load_checkpoint)."""
import numpy as np
import pytest

from fve_dg_b200 import ExplicitConvection, box_mesh, problems
from fve_dg_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_checkpoint_round_trip_and_restart(tmp_path, precision):
    m = box_mesh(3, jitter=0.1, seed=6)
    P, qv, qf = 2, 1, 2
    U0 = problems.project(m, P, problems.density_wave())
    a = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision=precision)
    a.set_state(U0)
    a.ssprk3(1e-3, 4)
    path = str(tmp_path / "ck.bin")
    a.save_checkpoint(path, t=4e-3, step=4)
    b = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision=precision)
    t, step = b.load_checkpoint(path)
    assert (t, step) == (4e-3, 4)
    assert np.array_equal(a.get_state(), b.get_state())
    # a restart continues exactly as the uninterrupted run
    a.ssprk3(1e-3, 3)
    b.ssprk3(1e-3, 3)
    assert np.array_equal(a.get_state(), b.get_state())


def test_checkpoint_rejects_corruption_and_mismatch(tmp_path):
    m = box_mesh(3, jitter=0.1, seed=6)
    a = ExplicitConvection(m, order=2, quad_vol=1, quad_face=2)
    a.set_state(problems.project(m, 2, problems.density_wave()))
    path = tmp_path / "ck.bin"
    a.save_checkpoint(str(path))
    raw = bytearray(path.read_bytes())
    raw[200] ^= 1  # one flipped bit in the state
    bad = tmp_path / "bad.bin"
    bad.write_bytes(bytes(raw))
    with pytest.raises(L.DGError) as e:
        a.load_checkpoint(str(bad))
    assert e.value.code == -8
    other = ExplicitConvection(box_mesh(2), order=2, quad_vol=1, quad_face=2)
    with pytest.raises(L.DGError) as e:
        other.load_checkpoint(str(path))
    assert e.value.code == -2
    with pytest.raises(L.DGError) as e:
        a.load_checkpoint(str(tmp_path / "missing.bin"))
    assert e.value.code == -8
