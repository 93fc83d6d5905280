"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances: stages whose device arithmetic follows the reference's
operation order (compiled without FMA contraction) must match bit for bit;
line solves use precomputed reciprocal pivots and a warp-parallel
recurrence, so they match to round-off (1e-13 relative); the Poisson
potential is compared through the quantities that depend on it (the
projected velocity and the mean-free pressure), because the reference
leaves its Neumann null mode undetermined.  Full steps: 1e-10 relative per
step on the fields; lift and displacement histories: 1e-8 relative to the
history's range (the bar the hot path is built to).
"""
import os

import numpy as np
import pytest

import fribois2d_b200 as fb
from fribois2d_b200 import case as cases
from paritylib import Pair, rel

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
SMALL = [cases.tiny_cylinder, cases.tiny_rectangle]


def _sub(a, k0, k1, j0, j1):
    return a[k0:k1 + 1, j0 - 1:j1]


@pytest.mark.parametrize("maker", SMALL)
def test_stage_by_stage(maker, tmp_path):
    """Each reference subroutine on identical inputs (state re-synced from
    the oracle before every stage)."""
    p = Pair(maker(), str(tmp_path))
    o, s = p.o, p.s
    n2m, n3m = p.n2m, p.n3m
    for ns in range(2):
        assert o.step(ns) == 0
    p.sync_to_gpu()
    ns = 2
    dt = o.scalars()["dt"]
    for n in (1, 2, 3):
        o.set_substep(ns, n)
        s.set_substep(ns, n)
        if n == 1:
            o.stage("cfl")
            assert s.stage("cfl") == 0
            assert rel(s.scalars()["cflm"], o.scalars()["cflm"] * dt) <= 1e-15
        o.stage("boucdq")
        assert s.stage("boucdq", n) == 0
        for b in ("dqb2n", "dq2x2o", "dq3x2o"):
            np.testing.assert_array_equal(s.get(b), p.ob(b))
        assert rel(s.get("dqb3n"), p.ob("dqb3n")) <= 1e-14  # mass-flux sum order
        for x in ("hdnl2", "hdnl3", "invtr2", "invtr3"):
            o.stage(x, n)
        assert s.stage("nl_rhs", n) == 0
        for f, k0, j0 in (("rhs2", 1, 2), ("ru2", 1, 2), ("rhs3", 2, 1), ("ru3", 2, 1)):
            np.testing.assert_array_equal(_sub(s.get(f), k0, n3m, j0, n2m), _sub(p.of(f), k0, n3m, j0, n2m),
                                          err_msg=f"{f} substep {n}")
        p.sync_to_gpu()
        if n == 1:
            o.stage("lgrdistribution")
            assert s.stage("lgrdistribution", n) == 0
            np.testing.assert_array_equal(s.geti("lmind"), o.ia("lmind"))
        o.stage("forcing", n)
        assert s.stage("forcing", n) == 0
        rhs2 = p.of("rhs2") + p.of("fey") * dt
        rhs3 = p.of("rhs3") + p.of("fez") * dt
        np.testing.assert_array_equal(_sub(s.get("rhs2"), 1, n3m, 2, n2m), _sub(rhs2, 1, n3m, 2, n2m))
        np.testing.assert_array_equal(_sub(s.get("rhs3"), 2, n3m, 1, n2m), _sub(rhs3, 2, n3m, 1, n2m))
        if n == 1:
            np.testing.assert_array_equal(s.get("phi"), o.a("phi"))
            np.testing.assert_array_equal(s.get("cl"), o.a("cl"))
            np.testing.assert_array_equal(s.geti("eulins"), o.ia("eulins"))
        r2, r3 = p.of("rhs2").copy(), p.of("rhs3").copy()
        r2[1:n3m + 1, 1:n2m] = rhs2[1:n3m + 1, 1:n2m]
        r3[2:n3m + 1, 0:n2m] = rhs3[2:n3m + 1, 0:n2m]
        s.set("rhs2", r2)
        s.set("rhs3", r3)
        o.stage("helsolve", n)
        assert s.stage("helsolve", n) == 0
        assert rel(s.get("q2"), p.of("q2")) <= 1e-13
        assert rel(s.get("q3"), p.of("q3")) <= 1e-13
        p.sync_to_gpu()
        o.stage("divg", n)
        assert s.stage("divg", n) == 0
        np.testing.assert_array_equal(_sub(s.get("dph"), 1, n3m, 1, n2m), _sub(p.of("dph"), 1, n3m, 1, n2m))
        o.stage("phcalc", n)
        assert s.stage("phcalc", n) == 0
        # projection with each side's own potential
        o.stage("updvp", n)
        o.stage("prcalc", n)
        assert s.stage("updvp", n) == 0
        assert rel(s.get("q2"), p.of("q2")) <= 1e-11
        assert rel(s.get("q3"), p.of("q3")) <= 1e-11
        o.stage("pr_submean", n)
        o.stage("boucqt", n)
        assert s.stage("pr_submean", n) == 0
        assert rel(_sub(s.get("pr"), 1, n3m, 1, n2m), _sub(p.of("pr"), 1, n3m, 1, n2m)) <= 1e-10
        p.sync_to_gpu()
    o.stage("checkbcs")
    o.stage("loads")
    assert s.stage("loads") == 0
    for a in ("press", "tau", "bcerrv", "bcerrw"):
        np.testing.assert_array_equal(s.get(a), o.a(a), err_msg=a)
    o.stage("rigid")
    assert s.stage("rigid") == 0
    assert rel(s.get("rigid"), o.a("rigid")) <= 1e-14
    assert rel(s.get("forces")[1:], o.a("forces")[1:]) <= 1e-13
    for a in ("lmcc", "lmvel", "lmacc", "lmnor", "vert"):
        assert rel(s.get(a), o.a(a)) <= 1e-14, a


@pytest.mark.parametrize("maker", SMALL)
def test_full_steps(maker, tmp_path):
    """fluid_tsch + rigid through the C ABI against the oracle, step by step."""
    p = Pair(maker(), str(tmp_path))
    n2m, n3m = p.n2m, p.n3m
    for ns in range(12):
        assert p.o.step(ns) == 0
        p.s.fluid_tsch(ns)
        p.s.rigid(ns)
        for f in ("q2", "q3"):
            assert rel(_sub(p.s.get(f), 1, n3m, 1, n2m), _sub(p.of(f), 1, n3m, 1, n2m)) <= 1e-10, (f, ns)
        assert rel(_sub(p.s.get("pr"), 1, n3m, 1, n2m), _sub(p.of("pr"), 1, n3m, 1, n2m)) <= 1e-10
        assert rel(p.s.get("forces")[1:4], p.o.a("forces")[1:4]) <= 1e-10
        assert rel(p.s.get("rigid"), p.o.a("rigid")) <= 1e-12


@pytest.mark.parametrize("maker,col", [(cases.tiny_cylinder, ("Fy", "py")),
                                       (cases.tiny_rectangle, ("M", "pa"))])
def test_lift_and_displacement_history(maker, col, tmp_path):
    """300 steps through the graph-replayed fb_advance: the lift (or moment)
    and displacement (or pitch) histories within 1e-8 of the oracle's."""
    c = maker()
    p = Pair(c, str(tmp_path))
    steps = 300
    hist = p.s.advance(0, steps)
    names = fb.HIST_NAMES
    ref_force, ref_disp = [], []
    for ns in range(steps):
        assert p.o.step(ns) == 0
        f = p.o.a("forces")
        r = p.o.a("rigid")
        ref_force.append(f[{"Fy": 1, "M": 3}[col[0]]])
        ref_disp.append(r[9 + {"py": 0, "pa": 2}[col[1]]])
    gf = hist[:, names.index(col[0])]
    gd = hist[:, names.index(col[1])]
    ref_force, ref_disp = np.array(ref_force), np.array(ref_disp)
    assert np.max(np.abs(gf - ref_force)) <= 1e-8 * np.max(np.abs(ref_force))
    span = max(np.ptp(ref_disp), 1e-300)
    assert np.max(np.abs(gd - ref_disp)) <= 1e-8 * span
    assert np.max(np.abs(gd - ref_disp)) <= 1e-12 * max(1.0, np.max(np.abs(ref_disp)))


@pytest.mark.parametrize("maker", SMALL)
def test_golden_trajectory(maker, tmp_path):
    """Against the committed oracle trajectory (LAPACK eigen data there, the
    device's own eigen-decomposition here)."""
    c = maker()
    z = np.load(os.path.join(GOLD, f"traj_{c.name}.npz"))
    path = c.write(str(tmp_path / c.name))
    s = fb.Solver(path)
    q2 = s.get("q2")
    q2[1:c.n3m + 1] += c.v_perturbation()
    s.set("q2", q2)
    steps = int(z["steps"][0])
    hist = s.advance(0, steps)
    assert rel(hist[:, 1:4], z["forces"][:, 1:4]) <= 1e-9
    assert rel(hist[:, 9:18], z["rigid"][:, 9:18]) <= 1e-12
    assert rel(s.get("q3")[1:c.n3m + 1, :c.n2m], z["q3"][1:c.n3m + 1, :c.n2m]) <= 1e-10


def test_advance_is_bitwise_equal_to_stepwise(tmp_path):
    """The captured CUDA graph replays exactly the stepwise C-ABI calls."""
    c = cases.tiny_cylinder()
    path = c.write(str(tmp_path / c.name))
    a, b = fb.Solver(path), fb.Solver(path)
    h = a.advance(0, 25)
    rows = []
    for ns in range(25):
        b.fluid_tsch(ns)
        rows.append(b.rigid(ns))
    for f in ("q2", "q3", "pr"):
        np.testing.assert_array_equal(a.get(f), b.get(f))
    np.testing.assert_array_equal(h[:, :8], np.array(rows))
    assert h[-1, 8] == pytest.approx(25 * c.params.dt, rel=1e-12)


def test_dense_markers_spread_in_marker_order(tmp_path):
    """400 markers on the small cylinder (radius 0.5, h = 1/8): about 16 per
    grid spacing, so more support boxes start in some cells than one entry
    of the spreading table holds and those cells continue at the next
    level.  The forcing stage still adds every cell's contributions in
    marker order (bit for bit with the oracle), and full steps follow the
    oracle to 1e-10."""
    p = Pair(cases.tiny_cylinder(nlm=400), str(tmp_path))
    o, s = p.o, p.s
    n2m, n3m = p.n2m, p.n3m
    for ns in range(2):
        assert o.step(ns) == 0
    p.sync_to_gpu()
    dt = o.scalars()["dt"]
    o.set_substep(2, 1)
    s.set_substep(2, 1)
    o.stage("cfl")
    assert s.stage("cfl") == 0
    o.stage("boucdq")
    assert s.stage("boucdq", 1) == 0
    for x in ("hdnl2", "hdnl3", "invtr2", "invtr3"):   # q2f, q3f: what the forcing interpolates
        o.stage(x, 1)
    assert s.stage("nl_rhs", 1) == 0
    p.sync_to_gpu()
    o.stage("lgrdistribution")
    assert s.stage("lgrdistribution", 1) == 0
    o.stage("forcing", 1)
    assert s.stage("forcing", 1) == 0
    rhs2 = p.of("rhs2") + p.of("fey") * dt
    rhs3 = p.of("rhs3") + p.of("fez") * dt
    np.testing.assert_array_equal(_sub(s.get("rhs2"), 1, n3m, 2, n2m), _sub(rhs2, 1, n3m, 2, n2m))
    np.testing.assert_array_equal(_sub(s.get("rhs3"), 2, n3m, 1, n2m), _sub(rhs3, 2, n3m, 1, n2m))
    for ns in range(2, 6):
        p.sync_to_gpu()
        assert o.step(ns) == 0
        s.fluid_tsch(ns)
        s.rigid(ns)
        for f in ("q2", "q3"):
            assert rel(_sub(s.get(f), 1, n3m, 1, n2m), _sub(p.of(f), 1, n3m, 1, n2m)) <= 1e-10, (f, ns)
        assert rel(s.get("forces")[1:4], o.a("forces")[1:4]) <= 1e-10, ns
    s.close()


def test_marker_outside_domain_is_reported_not_faulted(tmp_path):
    """A marker pushed outside the grid on the host is caught by the device
    kernels' bounds checks (lgrdistribution.F90:217-221) and reported."""
    c = cases.tiny_cylinder()
    s = fb.Solver(c.write(str(tmp_path / c.name)))
    lm = s.get("lmcc")
    lm[0] = -1.0
    s.set("lmcc", lm)
    with pytest.raises(fb.FBError) as e:
        s.fluid_tsch(0)
    assert e.value.code == fb.FB_ERR_MARKER_OUT


def test_cfl_overflow_is_reported(tmp_path):
    """fluid_tsch.F90:49-54: a velocity field above cfllim stops the step."""
    c = cases.tiny_cylinder()
    s = fb.Solver(c.write(str(tmp_path / c.name)))
    q3 = s.get("q3")
    q3[:] = 1.0e4
    s.set("q3", q3)
    with pytest.raises(fb.FBError) as e:
        s.fluid_tsch(0)
    assert e.value.code == fb.FB_ERR_CFL


def test_nan_velocity_is_reported(tmp_path):
    """A NaN velocity is a CFL failure, not a finite CFL number: the max
    reduction keeps it (as +inf) instead of dropping it."""
    c = cases.tiny_cylinder()
    s = fb.Solver(c.write(str(tmp_path / c.name)))
    q2 = s.get("q2")
    q2[5, 3] = np.nan
    s.set("q2", q2)
    with pytest.raises(fb.FBError) as e:
        s.fluid_tsch(0)
    assert e.value.code == fb.FB_ERR_CFL


@pytest.mark.parametrize("nsst", [3, 1])
def test_variable_dt_matches_oracle(nsst, tmp_path):
    """idtv = .false. (fluid_tsch.F90:34-48): dt = cflmax / cflm from the
    second step on, capped by dtmax; the device rebuilds its Helmholtz
    factors for every new dt.  RK3 and Adams-Bashforth (whose coefficients
    use dt/dt_o)."""
    c = cases.tiny_cylinder()
    c.params.idtv = False
    c.params.cflmax = 0.25
    c.params.dtmax = 0.02
    c.params.nsst = nsst
    p = Pair(c, str(tmp_path))
    n2m, n3m = p.n2m, p.n3m
    dts = []
    for ns in range(8):
        assert p.o.step(ns) == 0
        h = p.s.advance(ns, 1)
        dts.append(h[0, fb.HIST_NAMES.index("dt")])
        assert dts[-1] == pytest.approx(p.o.scalars()["dt"], rel=1e-13)
        for f in ("q2", "q3"):
            assert rel(_sub(p.s.get(f), 1, n3m, 1, n2m), _sub(p.of(f), 1, n3m, 1, n2m)) <= 1e-10, (f, ns)
        assert rel(p.s.get("rigid"), p.o.a("rigid")) <= 1e-12
    assert dts[0] == c.params.dt and len(set(dts[1:])) > 1   # dt really varies


def _windows(s):
    import ctypes
    dims = (ctypes.c_int32 * 8)()
    assert fb.lib().fb_get_dims(s.ctx, dims) == 0
    return dims[7] & 0xff, dims[7] >> 8


@pytest.mark.parametrize("maker", [cases.tiny_rectangle, cases.viv_cylinder_384x256])
def test_windowed_helsolve_matches_line_scans(maker, tmp_path, monkeypatch):
    """The truncated-window helsolve agrees with the full line scans to
    round-off over several steps (both are exact LU substitutions up to the
    2^-56 truncation of the window)."""
    c = maker()
    path = c.write(str(tmp_path / c.name))
    pert = c.v_perturbation()
    out = []
    for mode in ("", "scan"):
        if mode:
            monkeypatch.setenv("FRIBOIS2D_HELSOLVE", mode)
        s = fb.Solver(path)
        wy, wz = _windows(s)
        assert (wy > 0 and wz > 0) if not mode else (wy == 0 and wz == 0)
        q2 = s.get("q2")
        q2[1:c.n3m + 1] += pert
        s.set("q2", q2)
        h = s.advance(0, 5)
        out.append((s.get("q2"), s.get("q3"), s.get("pr"), h))
        s.close()
    (a2, a3, ap, ah), (b2, b3, bp, bh) = out
    assert rel(a2, b2) <= 1e-13 and rel(a3, b3) <= 1e-13 and rel(ap, bp) <= 1e-11
    assert rel(ah[:, 1:4], bh[:, 1:4]) <= 1e-11
