"""Launch shapes and the autotuner (sphgpu_set_launch / sphgpu_autotune): the
threads per block of the neighbour passes change no result, bit for bit, and
the autotuner keeps, per pass, the fastest of the shapes it timed (the default
of 128 unless another is more than 3% faster), and applies
a cached choice without timing again."""
import os
import tempfile

import numpy as np
import pytest

import scenes
import sphgpu
from checkers import STATE_FIELDS

pytestmark = pytest.mark.gpu


def _engine(sc):
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    return eng


@pytest.mark.parametrize("factory", [lambda: scenes.dam_break_2d(dx=0.02, steps=100),
                                     lambda: scenes.soil_column_3d(dx=0.05, steps=100)])
def test_launch_shape_changes_no_result(factory):
    outs = []
    for tb in ([128] * 10, [32, 64, 96, 32, 64, 96, 32, 64, 96, 32]):
        eng = _engine(factory())
        eng.set_launch(tb)
        assert list(eng.launch()) == tb
        eng.step(12)
        outs.append({k: eng.get_field(k) for k in STATE_FIELDS})
        eng.close()
    for k in STATE_FIELDS:
        a, b = outs[0][k], outs[1][k]
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert same.all(), k


def test_autotune_picks_the_fastest_and_caches_it():
    cache = os.path.join(tempfile.mkdtemp(), "tune.txt")
    eng = _engine(scenes.soil_column_3d(dx=0.02, steps=100))
    table = eng.autotune(steps=2, cache_path=cache)
    chosen = eng.launch()
    cand = np.array([32, 64, 96, 128])
    assert (table > 0).all()
    for q in range(table.shape[1]):
        best = int(np.argmin(table[:3, q]))
        want = cand[best] if table[best, q] < 0.97 * table[3, q] else 128
        assert chosen[q] == want, q
    print("autotune ms per pass (rows 32/64/96/128):\n", np.round(table, 4), "\nchosen", chosen)
    assert os.path.exists(cache)
    eng.close()
    again = _engine(scenes.soil_column_3d(dx=0.02, steps=100))
    t2 = again.autotune(steps=2, cache_path=cache)
    assert (t2 == 0).all()
    assert np.array_equal(again.launch(), chosen)
    again.close()


def test_set_launch_rejects_other_sizes():
    eng = _engine(scenes.dam_break_2d(dx=0.04, steps=10))
    for bad in ([16] * 10, [160] * 10, [100] * 10):
        with pytest.raises(sphgpu.SPHError):
            eng.set_launch(bad)
    eng.close()
