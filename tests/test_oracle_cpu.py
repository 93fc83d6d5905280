"""CPU tests of the oracle (test infrastructure) against LAPACK and the golden
fixtures, and of its physical invariants.  No GPU needed."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from fribois2d_b200 import case as cases

GOLD = os.path.join(os.path.dirname(__file__), "golden")
P = ctypes.POINTER


def _dp(a):
    return a.ctypes.data_as(P(ctypes.c_double))


def test_dgttrf_dgtts2_restatement_matches_lapack():
    """fbo_dgttrf/fbo_dgtts2 restate LAPACK 3.8 DGTTRF/DGTTRS (called by
    src/solve_fluid.F90:93-97 and src/phcalc_outflow.F90:48-52)."""
    z = np.load(os.path.join(GOLD, "lapack_gtt.npz"))
    lib = oracle.lib()
    pivoted = 0
    for i in range(int(z["count"][0])):
        lo, di, up, b = (z[f"s{i}_{k}"].copy() for k in ("lo", "di", "up", "b"))
        n = len(di)
        du2 = np.zeros(max(n - 2, 1))
        ipiv = np.zeros(n, dtype=np.int32)
        info = lib.fbo_dgttrf(n, _dp(lo), _dp(di), _dp(up), _dp(du2), ipiv.ctypes.data_as(P(ctypes.c_int)))
        assert info == int(z[f"s{i}_info"][0])
        np.testing.assert_array_equal(ipiv, z[f"s{i}_ipiv"])
        pivoted += int(np.any(ipiv != np.arange(1, n + 1)))
        # factors: identical operations, so equal up to LAPACK's own build flags
        np.testing.assert_allclose(lo, z[f"s{i}_dl"], rtol=1e-14, atol=0)
        np.testing.assert_allclose(di, z[f"s{i}_d"], rtol=1e-14, atol=0)
        np.testing.assert_allclose(up, z[f"s{i}_du"], rtol=1e-14, atol=0)
        np.testing.assert_allclose(du2[:max(n - 2, 0)], z[f"s{i}_du2"][:max(n - 2, 0)], rtol=1e-14, atol=0)
        lib.fbo_dgtts2(n, _dp(lo), _dp(di), _dp(up), _dp(du2), ipiv.ctypes.data_as(P(ctypes.c_int)), _dp(b))
        np.testing.assert_allclose(b, z[f"s{i}_x"], rtol=1e-12, atol=1e-14)
    assert pivoted >= 2, "the fixture must exercise row interchanges"


def test_phini_matches_lapack_fixture():
    """oracle.phini calls DGEEV/DGESV like src/phini.F90:52-92."""
    z = np.load(os.path.join(GOLD, "phini_tiny.npz"))
    wr, zmm, zmmt = oracle.phini(z["amphk"], z["acphk"], z["apphk"])
    np.testing.assert_allclose(np.sort(wr), np.sort(z["wr"]), rtol=0, atol=1e-12)
    np.testing.assert_allclose(zmm @ zmmt, np.eye(len(wr)), atol=1e-12)
    np.testing.assert_allclose(zmm, z["zmm"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("maker", [cases.tiny_cylinder, cases.tiny_rectangle])
def test_oracle_trajectory_matches_fixture(maker, tmp_path):
    """Regression pin of the oracle: the committed trajectory is reproduced."""
    c = maker()
    z = np.load(os.path.join(GOLD, f"traj_{c.name}.npz"))
    path = c.write(str(tmp_path / c.name))
    o = oracle.Oracle(oracle.parse_deck(path), eigen=(z["eig_wr"], z["eig_zmm"], z["eig_zmmt"]), threads=1)
    o.add_v_perturbation(c.v_perturbation())
    for ns in range(int(z["steps"][0])):
        assert o.step(ns) == 0
        np.testing.assert_array_equal(o.a("forces"), z["forces"][ns])
        np.testing.assert_array_equal(o.a("rigid"), z["rigid"][ns])
    np.testing.assert_array_equal(o.field("q2", 0, o.n3), z["q2"])
    np.testing.assert_array_equal(o.field("pr", 0, o.n3), z["pr"])


def test_oracle_thread_count_does_not_change_results(tmp_path):
    c = cases.tiny_rectangle()
    path = c.write(str(tmp_path / c.name))
    d = oracle.parse_deck(path)
    out = []
    for th in (1, 4):
        o = oracle.Oracle(d, threads=th)
        for ns in range(3):
            assert o.step(ns) == 0
        out.append(o.field("q3", 0, o.n3).copy())
    np.testing.assert_array_equal(out[0], out[1])


def test_projection_makes_field_divergence_free(tmp_path):
    """After phcalc + updvp the discrete divergence vanishes (the invariant
    ttime.F90:36-50 checks against resid)."""
    c = cases.tiny_cylinder()
    path = c.write(str(tmp_path / c.name))
    o = oracle.Oracle(oracle.parse_deck(path), threads=1)
    o.add_v_perturbation(c.v_perturbation())
    for ns in range(3):
        assert o.step(ns) == 0
    q2, q3 = o.field("q2", 0, o.n3), o.field("q3", 0, o.n3)
    udx2m, udx3m = o.a("udx2m"), o.a("udx3m")
    n2m, n3m = o.n2m, o.n3m
    div = ((q2[1:n3m + 1, 1:n2m + 1] - q2[1:n3m + 1, 0:n2m]) * udx2m[1:n2m + 1][None, :]
           + (q3[2:n3m + 2, 0:n2m] - q3[1:n3m + 1, 0:n2m]) * udx3m[1:n3m + 1][:, None])
    assert np.max(np.abs(div)) < 1e-9


def test_mls_partition_of_unity(tmp_path):
    """MLSint.F90:157-163: each marker's transfer weights sum to one."""
    c = cases.tiny_rectangle()
    path = c.write(str(tmp_path / c.name))
    o = oracle.Oracle(oracle.parse_deck(path), threads=1)
    assert o.step(0) == 0
    phi = o.a("phi").reshape(o.nlm, 2, 9)
    np.testing.assert_allclose(phi.sum(axis=2), 1.0, atol=1e-10)


def test_marker_outside_domain_is_reported(tmp_path):
    """lgrdistribution.F90:217-221 stops the run; the oracle returns the code."""
    c = cases.tiny_cylinder()
    path = c.write(str(tmp_path / c.name))
    o = oracle.Oracle(oracle.parse_deck(path), threads=1)
    o.a("lmcc")[0] = -1.0
    assert o.fluid_tsch(0) == 3
