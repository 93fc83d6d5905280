"""Checkpoint/restart and end-of-step diagnostics on the device path."""
import numpy as np
import pytest

import fribois2d_b200 as fb
from fribois2d_b200 import HIST_NAMES
from fribois2d_b200 import case as cases
from fribois2d_b200 import io as fio

pytestmark = pytest.mark.gpu


def _solver(c, path):
    s = fb.Solver(path)
    q2 = s.get("q2")
    q2[1:c.n3m + 1] += c.v_perturbation()
    s.set("q2", q2)
    return s


def test_restart_continues_bit_for_bit(tmp_path):
    c = cases.tiny_rectangle()
    path = c.write(str(tmp_path / c.name))
    a = _solver(c, path)
    a.advance(0, 10)
    a.write_restart(str(tmp_path / "restart"))
    ha = a.advance(10, 6)
    fa = {f: a.get(f) for f in ("q2", "q3", "pr")}
    a.close()
    b = fb.Solver(path)
    b.read_restart(str(tmp_path / "restart"))
    hb = b.advance(10, 6)
    for f in ("q2", "q3", "pr"):
        assert np.array_equal(b.get(f), fa[f]), f
    assert np.array_equal(ha, hb)
    b.close()
    text = (tmp_path / "restart" / "master_rigid.dat").read_text().splitlines()
    assert len(text) == 5 and float(text[0]) == pytest.approx(ha[0, HIST_NAMES.index("time")])


def test_restart_rejects_a_different_grid(tmp_path):
    c = cases.tiny_rectangle()
    a = _solver(c, c.write(str(tmp_path / "a")))
    a.advance(0, 2)
    a.write_restart(str(tmp_path / "restart"))
    a.close()
    d = cases.tiny_cylinder()
    b = fb.Solver(d.write(str(tmp_path / "b")))
    with pytest.raises(fb.FBError):
        b.read_restart(str(tmp_path / "restart"))
    b.close()


def test_report_diagnostics_match_the_fields(tmp_path):
    c = cases.tiny_cylinder()
    s = _solver(c, c.write(str(tmp_path / c.name)))
    s.set_report(True)
    h = s.advance(0, 3)
    q2, q3 = s.get("q2"), s.get("q3")
    rc, zz = s.get("rc"), s.get("zz")
    u2, u3 = s.get("udx2m"), s.get("udx3m")
    n2m, n3m = c.n2m, c.n3m
    # 0-based views: field[k, j-1]; rc[j-1] = rc(j)
    v2 = q2[1:n3m + 1, :n2m]
    v3 = q3[1:n3m + 1, :n2m]
    v2p = q2[1:n3m + 1, 1:n2m + 1]
    v3p = q3[2:n3m + 2, :n2m]
    row = h[-1]
    col = {n: HIST_NAMES.index(n) for n in HIST_NAMES}
    assert row[col["vmax2"]] == np.max(np.abs(v2)) and row[col["vmax3"]] == np.max(np.abs(v3))
    assert row[col["vmin2"]] == np.min(v2) and row[col["vmin3"]] == np.min(v3)
    div = (v2p - v2) * u2[None, :n2m] + (v3p - v3) * u3[:n3m, None]
    assert row[col["dmax"]] == pytest.approx(np.max(np.abs(div)), rel=1e-12, abs=1e-300)
    vol = np.outer(zz[1:n3m + 1] - zz[:n3m], rc[1:n2m + 1] - rc[:n2m])
    ek = 0.5 * np.sum(((v2 + v2p) * 0.5) ** 2 * vol + ((v3 + v3p) * 0.5) ** 2 * vol) / (c.params.rext2 * c.params.alx3)
    assert row[col["ektot"]] == pytest.approx(ek, rel=1e-12)
    cfl = np.max(np.abs((v2 + v2p) * 0.5 * u2[None, :n2m]) + np.abs((v3 + v3p) * 0.5 * u3[:n3m, None]))
    assert row[col["cflm_end"]] == pytest.approx(cfl * c.params.dt, rel=1e-14)
    assert row[col["dt"]] == c.params.dt
    s.set_report(False)
    h2 = s.advance(3, 1)
    assert h2[0, col["dmax"]] == 0.0
    r = fio.Reporter(str(tmp_path / "out"))
    r.write(h, 0)
    lines = (tmp_path / "out" / "fluid_rep.out").read_text().splitlines()
    assert len(lines) == 3 and float(lines[2][25:41]) == pytest.approx(c.params.dt, rel=1e-8)
    s.close()


def test_marker_round_trip_through_the_host(tmp_path):
    """fb_set_markers returns before its device copies finish (staged in pinned
    memory) and fb_get_markers reads all four arrays with one wait: a host
    that keeps its own marker state, stepping per call, gets exactly the
    stepping of the device-side state, and the caller's buffers may be reused
    at once."""
    c = cases.tiny_cylinder()
    path = c.write(str(tmp_path / c.name))
    a, b = _solver(c, path), _solver(c, path)
    a.advance(0, 5)
    b.advance(0, 5)
    names = ("lmcc", "lmvel", "lmacc", "lmnor")
    for ns in range(5, 15):
        got = b.get_markers()
        for g, n in zip(got, names):
            np.testing.assert_array_equal(g.reshape(-1), b.get(n).reshape(-1))
        bufs = [g.copy() for g in got]
        b.set_markers(*bufs)
        for buf in bufs:
            buf[:] = np.nan   # reused at once: the staged copy is what the device receives
        a.fluid_tsch(ns)
        a.rigid(ns)
        b.fluid_tsch(ns)
        b.rigid(ns)
    for f in ("q2", "q3", "pr"):
        np.testing.assert_array_equal(a.get(f), b.get(f))
    for g, n in zip(b.get_markers(), names):
        np.testing.assert_array_equal(g.reshape(-1), a.get(n).reshape(-1))
    a.close()
    b.close()


def test_step_markers_equals_the_four_calls(tmp_path):
    """fb_step_markers (markers in, fluid step, rigid update, markers out, one
    wait) leaves the same state, markers and forcecomp rows, bit for bit, as
    fb_set_markers + fb_fluid_tsch + fb_rigid + fb_get_markers."""
    import ctypes
    c = cases.tiny_cylinder()
    path = c.write(str(tmp_path / c.name))
    a, b = _solver(c, path), _solver(c, path)
    a.advance(0, 3)
    b.advance(0, 3)
    L = fb.lib()
    dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))   # noqa: E731
    names = ("lmcc", "lmvel", "lmacc", "lmnor")
    ma = [np.zeros(2 * c.nlm) for _ in names]
    assert L.fb_get_markers(a.ctx, *[dp(m) for m in ma]) == 0   # the device layout, as the host keeps it
    mb = [m.copy() for m in ma]
    fa, fb_ = np.zeros(8), np.zeros(8)
    for ns in range(3, 12):
        assert L.fb_set_markers(a.ctx, *[dp(m) for m in ma]) == 0
        assert L.fb_fluid_tsch(a.ctx, ns) == 0
        assert L.fb_rigid(a.ctx, ns, dp(fa)) == 0
        assert L.fb_get_markers(a.ctx, *[dp(m) for m in ma]) == 0
        assert L.fb_step_markers(b.ctx, ns, *[dp(m) for m in mb], dp(fb_)) == 0
        np.testing.assert_array_equal(fa, fb_)
        for x, y in zip(ma, mb):
            np.testing.assert_array_equal(x, y)
    for f in ("q2", "q3", "pr"):
        np.testing.assert_array_equal(a.get(f), b.get(f))
    np.testing.assert_array_equal(a.last_history(), b.last_history())
    a.close()
    b.close()
