"""CPU tests of the product's host side (no GPU): deck parsing, grid metrics
and coefficients, the eigen set-up that replaces DGEEV+DGESV, the marker
set-up, and the exported C ABI."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import oracle
import fribois2d_b200 as fb
from fribois2d_b200 import case as cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fribois2d.h")
DECKS = os.path.join(ROOT, "tests", "golden", "decks")


@pytest.fixture(scope="module", autouse=True)
def _built():
    from fribois2d_b200 import build
    build.build()


def test_library_exports_every_declared_symbol():
    names = re.findall(r"^\s*(?:int|const char \*)\s*(fb_\w+)\s*\(", open(HEADER).read(), re.M)
    assert len(names) >= 20
    out = subprocess.check_output(["nm", "-D", "--defined-only", fb.LIB_PATH], text=True)
    exported = set(re.findall(r" T (fb_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = fb.lib()
    for n in names:
        assert hasattr(lib, n)
    assert "sm_100a" in fb.version()


def test_fortran_module_binds_every_entry_point():
    """include/fribois2d.f90 (no Fortran compiler here, so checked as text):
    one bind(C) interface per header function and the header's constants
    with the same values."""
    hdr = open(HEADER).read()
    f90 = open(os.path.join(ROOT, "include", "fribois2d.f90")).read()
    names = re.findall(r"^\s*(?:int|const char \*)\s*(fb_\w+)\s*\(", hdr, re.M)
    bound = re.findall(r'bind\(C, name="(fb_\w+)"\)', f90)
    assert sorted(names) == sorted(bound)
    consts = dict(re.findall(r"^#define (FB_\w+) (-?\d+)", hdr, re.M))
    fvals = dict((k, v) for k, v in re.findall(r"(FB_\w+) = (-?\d+)", f90))
    assert set(fvals) == set(consts)
    for k, v in consts.items():
        assert fvals[k] == v, k


def test_int8_product_bound_is_enforced_before_any_device_work():
    """The INT8 digit product keeps its weight classes in int32: K is bounded
    by 2^31 / (S * 127^2) and larger K is refused without touching the GPU."""
    from oracle import i8x8
    src = open(os.path.join(ROOT, "fribois2d_b200", "csrc", "tc_gemm.h")).read()
    kmax = int(re.search(r"kI8MaxK = (\d+);", src).group(1))
    assert int(re.search(r"kI8S = (\d+);", src).group(1)) == i8x8.S
    assert kmax * i8x8.S * 127 * 127 < 2 ** 31
    a = np.zeros(4 * (kmax + 1))
    c = np.zeros(16)
    import ctypes
    f = fb.lib().fb_gemm_i8x8
    p = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert f(0, 4, 4, kmax + 1, p(a), p(a), p(c)) == fb.FB_ERR_UNSUPPORTED


@pytest.mark.parametrize("maker", [cases.tiny_cylinder, cases.tiny_rectangle, cases.viv_cylinder_384x256])
def test_host_setup_bit_identical_to_oracle(maker, tmp_path):
    c = maker()
    path = c.write(str(tmp_path / c.name))
    h = fb.HostSetup(path)
    d = oracle.parse_deck(path)
    o = oracle.Oracle(d, eigen=(np.zeros(c.n3m), np.eye(c.n3m), np.eye(c.n3m)))
    assert (h.n2, h.n3, h.nlm, h.nsst) == (d["n2"], d["n3"], d["nlm"], d["nsst"])
    for name in ("rc", "rm", "zz", "zm", "udx2c", "udx2m", "udx3c", "udx3m", "amphj", "acphj",
                 "apphj", "amphk", "acphk", "apphk"):
        a = h.array(name)
        np.testing.assert_array_equal(a, o.a(name)[1:len(a) + 1], err_msg=name)
    for name in ("lmcc", "lmvel", "lmacc", "lmnor", "lmA", "vert", "rigid"):
        np.testing.assert_array_equal(h.array(name), o.a(name), err_msg=name)


def test_eigen_setup_reproduces_lapack_poisson_operator(tmp_path):
    """The symmetric-tridiagonal eigen-decomposition (host.cpp) replaces
    phini's DGEEV + DGESV: same spectrum, Z diag(wr) Z^-1 equals the operator."""
    c = cases.viv_cylinder_384x256()
    path = c.write(str(tmp_path / c.name))
    h = fb.HostSetup(path)
    d = oracle.parse_deck(path)
    o = oracle.Oracle(d, eigen=(np.zeros(c.n3m), np.eye(c.n3m), np.eye(c.n3m)))
    wr_l, zmm_l, zmmt_l = oracle.phini(o.a("amphk"), o.a("acphk"), o.a("apphk"))
    wr, zmm, zmmt = h.array("wr"), h.array("zmm"), h.array("zmmt")
    scale = np.max(np.abs(wr_l))
    np.testing.assert_allclose(np.sort(wr), np.sort(wr_l), rtol=0, atol=1e-13 * scale)
    n = c.n3m
    B = np.zeros((n, n))
    ak, ck, pk = o.a("amphk"), o.a("acphk"), o.a("apphk")
    for k in range(1, n + 1):
        B[k - 1, k - 1] = ck[k]
        if k < n:
            B[k - 1, k] = pk[k]
        if k > 1:
            B[k - 1, k - 2] = ak[k]
    np.testing.assert_allclose(zmm @ np.diag(wr) @ zmmt, B, rtol=0, atol=2e-13 * scale)
    np.testing.assert_allclose(zmm @ zmmt, np.eye(n), rtol=0, atol=1e-12)
    # the null (Neumann) mode is present once
    assert np.sum(np.abs(wr) < 1e-10 * scale) == 1


def test_eigen_tridiag_on_uniform_neumann_operator():
    """Known answer: the uniform Neumann second difference has eigenvalues
    -4 sin^2(pi m / (2 n)), m = 0..n-1."""
    n = 64
    am = np.r_[0.0, np.ones(n - 1)]
    ap = np.r_[np.ones(n - 1), 0.0]
    ac = -(am + ap)
    wr, zmm, zmmt = fb.eigen_tridiag(am, ac, ap)
    exact = -4.0 * np.sin(np.pi * np.arange(n) / (2 * n)) ** 2
    np.testing.assert_allclose(np.sort(wr), np.sort(exact), atol=1e-13)


@pytest.mark.parametrize("deck,nlm", [("OscCyl1DOF", 377), ("GallRect1DOF", 798)])
def test_reference_decks_parse_identically(deck, nlm, tmp_path):
    """The reference's own input decks: both parsers agree, markers are
    counted as newlines - 1 (utils_proc.F90:529-535)."""
    src = os.path.join(DECKS, deck)
    dst = str(tmp_path / "input_FSI")
    shutil.copytree(src, dst)
    d = oracle.parse_deck(dst)
    assert d["nlm"] == nlm
    h = fb.HostSetup(dst)
    assert (h.n2, h.n3, h.nlm) == (d["n2"], d["n3"], nlm)
    np.testing.assert_array_equal(h.array("rc"), d["ycoord"])
    np.testing.assert_array_equal(h.array("zz"), d["zcoord"])
    o = oracle.Oracle(d, eigen=(np.zeros(d["n3"] - 1), np.eye(d["n3"] - 1), np.eye(d["n3"] - 1)))
    for name in ("lmcc", "lmnor", "lmA", "vert", "rigid"):
        np.testing.assert_array_equal(h.array(name), o.a(name), err_msg=name)


def test_malformed_deck_is_rejected(tmp_path):
    c = cases.tiny_cylinder()
    path = c.write(str(tmp_path / c.name))
    with open(os.path.join(path, "fluid_par.in")) as f:
        lines = f.read().split("\n")
    lines[3] = "abc, def # broken grid size"
    with open(os.path.join(path, "fluid_par.in"), "w") as f:
        f.write("\n".join(lines))
    with pytest.raises(fb.FBError) as e:
        fb.HostSetup(path)
    assert e.value.code == fb.FB_ERR_INPUT


def test_missing_file_is_rejected(tmp_path):
    c = cases.tiny_cylinder()
    path = c.write(str(tmp_path / c.name))
    os.remove(os.path.join(path, "zcoord.dat"))
    with pytest.raises(fb.FBError) as e:
        fb.HostSetup(path)
    assert e.value.code == fb.FB_ERR_INPUT
