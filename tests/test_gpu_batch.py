"""Batches of independent cases: one graph launch steps every case.  The
graph mode holds every case's own captured step; the grouped mode launches
each stage once over every group of cases of one launch geometry (grouped
INT8 tensor-core transforms, or batched DGEMMs in the FP64 comparison form).
Both are checked against stepping each case on its own."""
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


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_batch_graph_equals_separate_runs(tmp_path):
    cs = _cases()
    alone = [_open(c, tmp_path / "alone") for c in cs]
    for s in alone:
        s.advance(0, 7)
    together = [_open(c, tmp_path / "batch") for c in cs]
    batch = fb.Batch(together, mode=fb.BATCH_GRAPH)
    assert batch.info()["groups"] == 0 and batch.info()["singles"] == len(cs)
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


def _grouped_cases():
    """Two cases on one grid with different Re (one group, transforms as
    batched cuBLAS DGEMMs), a second grid, a rectangle, two cases of the
    first grid in the precision form (a group of grouped 3xTF32 transforms)
    and two more with the INT8 FP64 transforms (the default form)."""
    a = cases.tiny_cylinder()
    b = cases.tiny_cylinder()
    b.name = "tiny_cylinder_re150"
    b.params.visc = 1.0 / 150.0
    c = cases.tiny_cylinder(n3m=64, n2m=40, nlm=48, dt=4e-3)
    d = cases.tiny_rectangle()
    e = cases.tiny_cylinder()
    e.name = "tiny_cylinder_tf32"
    f = cases.tiny_cylinder()
    f.name = "tiny_cylinder_tf32_re120"
    f.params.visc = 1.0 / 120.0
    g = cases.tiny_cylinder()
    g.name = "tiny_cylinder_int8"
    h = cases.tiny_cylinder()
    h.name = "tiny_cylinder_int8_re130"
    h.params.visc = 1.0 / 130.0
    return [a, b, c, d, e, f, g, h], {4, 5}, {6, 7}


def test_batch_grouped_matches_separate_runs(tmp_path):
    cs, precision, int8 = _grouped_cases()
    alone, together = [], []
    for i, c in enumerate(cs):
        s1 = _open(c, tmp_path / "alone")
        s2 = _open(c, tmp_path / "grouped")
        if i in precision:
            s1.set_poisson(fb.POISSON_TF32X3)
            s2.set_poisson(fb.POISSON_TF32X3)
        if i in int8:
            s1.set_poisson(fb.POISSON_INT8X8)
            s2.set_poisson(fb.POISSON_INT8X8)
        if i in (0, 1):
            s1.set_poisson(fb.POISSON_FP64)
            s2.set_poisson(fb.POISSON_FP64)
        alone.append(s1)
        together.append(s2)
    for s in alone:
        s.autotune()
        s.advance(0, 6)
    batch = fb.Batch(together)  # advanced 6 steps below
    info = batch.info()
    print("grouped batch:", info)
    assert info["groups"] >= 3 and info["launches"] > 0 and info["singles"] == 0
    steps = 6
    batch.advance(2)
    batch.advance(steps - 2)
    worst = {False: 0.0, True: 0.0}
    for i, (s1, s2) in enumerate(zip(alone, together)):
        for f in ("q2", "q3", "pr"):
            e = rel(s2.get(f), s1.get(f))
            worst[i in precision] = max(worst[i in precision], e)
            # the grouped reductions (pressure mean) sum in another order; in
            # the precision form such last-bit differences can move a TF32
            # rounding, so its bound is the form's own tolerance against the
            # FP64 path, 1e-9 per step
            assert e <= (1e-9 * steps if i in precision else 1e-12), (i, f, e)
        h1, h2 = s1.last_history(), s2.last_history()
        assert h2[8] == h1[8] and h2[30] == h1[30]          # clock, fluid solves
        np.testing.assert_allclose(h2[:21], h1[:21], rtol=1e-10, atol=1e-14)
    print("grouped vs alone, worst field difference (FP64, precision form):", worst[False], worst[True])
    batch.close()
    for s in alone + together:
        s.close()


def test_batch_grouped_one_launch_per_stage(tmp_path):
    """A group's launches per step do not grow with its size."""
    counts = []
    for n in (1, 4):
        ss = []
        for i in range(n):
            c = cases.tiny_cylinder()
            c.name = f"tiny_cylinder_{n}_{i}"
            c.params.visc = 1.0 / (100.0 + 10.0 * i)
            ss.append(_open(c, tmp_path / f"n{n}"))
        b = fb.Batch(ss)
        b.advance(2)
        counts.append(b.info())
        b.close()
        for s in ss:
            s.close()
    assert counts[0]["groups"] == 1 and counts[1]["groups"] == 1 and counts[1]["singles"] == 0
    assert counts[1]["launches"] == counts[0]["launches"]
