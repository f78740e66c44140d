"""Field state as .npy through a context: save, load into another context
(the load counts as the init), identical continuation; a file of another
shape is refused and leaves the field alone."""
import numpy as np
import pytest

import life_simulation_b200 as lb
from life_simulation_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def test_save_load_state_continues_identically(tmp_path):
    params, w, h, init = wl.workload("single_256")
    a = lb.LeniaModule(params, w, h)
    a.reset(4)
    for f in range(3):
        a.encode(f, 1)
    path = str(tmp_path / "state.npy")
    a.save_state(path)
    assert np.array_equal(np.load(path), a.field())
    b = lb.LeniaModule(params, w, h)
    b.reset(4)
    b.load_state(path)
    assert np.array_equal(b.field(), a.field())
    for f in range(3, 6):
        a.encode(f, 1)
        b.encode(f, 1)
    assert np.array_equal(a.field(), b.field())
    before = b.field()
    np.save(tmp_path / "wrong.npy", np.zeros((h, w + 2), np.float32))
    with pytest.raises(lb.LeniaError, match="shape mismatch"):
        b.load_state(str(tmp_path / "wrong.npy"))
    assert np.array_equal(b.field(), before)
    a.close()
    b.close()
