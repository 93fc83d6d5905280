"""Batches of independent cases: one graph launch steps every case, with
results bit for bit equal to stepping each case on its own."""
import numpy as np
import pytest

import fribois2d_b200 as fb
from fribois2d_b200 import case as cases

pytestmark = pytest.mark.gpu


def _cases():
    a = cases.tiny_cylinder()
    b = cases.tiny_cylinder(n3m=64, n2m=40, nlm=48, dt=4e-3)
    b.name = "tiny_cylinder_b"
    b.params.visc = 1.0 / 150.0
    c = cases.tiny_rectangle()
    return [a, b, c]


def _open(c, root):
    s = fb.Solver(c.write(str(root / c.name)))
    q2 = s.get("q2")
    q2[1:c.n3m + 1] += c.v_perturbation()
    s.set("q2", q2)
    return s


def test_batch_equals_separate_runs(tmp_path):
    cs = _cases()
    alone = [_open(c, tmp_path / "alone") for c in cs]
    for s in alone:
        s.advance(0, 7)
    together = [_open(c, tmp_path / "batch") for c in cs]
    batch = fb.Batch(together)
    batch.advance(3)
    batch.advance(4)
    assert batch.last_ms() > 0.0
    for s1, s2 in zip(alone, together):
        for f in ("q2", "q3", "pr"):
            assert np.array_equal(s1.get(f), s2.get(f)), f
        assert np.array_equal(s1.last_history(), s2.last_history())
    batch.close()
    for s in alone + together:
        s.close()


def test_batch_rejects_variable_dt(tmp_path):
    c = cases.tiny_cylinder()
    c.params.idtv = False
    s = fb.Solver(c.write(str(tmp_path / c.name)))
    with pytest.raises(fb.FBError) as e:
        fb.Batch([s])
    assert e.value.code == fb.FB_ERR_UNSUPPORTED
    s.close()
