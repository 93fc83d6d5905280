"""GPU test of fb_cfl_noalloc, the entry point for callers that cannot let
the library allocate device memory (their arrays belong to another runtime
or to an arena with a hard budget).  It must agree with the CFL stage of a
regular context on the same velocity field, call after call."""
import ctypes

import numpy as np
import pytest

import fribois2d_b200 as fb
from fribois2d_b200 import case as cases

pytestmark = pytest.mark.gpu


def test_cfl_noalloc_matches_context(tmp_path):
    import torch

    c = cases.tiny_cylinder()
    s = fb.Solver(c.write(str(tmp_path / c.name)))
    q2 = s.get("q2")
    q2[1:c.n3m + 1] += c.v_perturbation()
    s.set("q2", q2)
    s.advance(0, 3, history=False)          # a developed, non-uniform field
    s.set_substep(3, 1)
    assert s.stage("cfl") == 0
    ref = s.scalars()
    # the caller's own device arrays (dense rows: pitch = n2)
    dev = torch.device("cuda", 0)
    t = {name: torch.from_numpy(np.ascontiguousarray(s.get(name))).to(dev)
         for name in ("q2", "q3", "rc", "zz", "udx2m", "udx3m")}
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    lib = fb.lib()
    f = lib.fb_cfl_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                  ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    udx2m = t["udx2m"][:c.n2m].contiguous()
    udx3m = t["udx3m"][:c.n3m].contiguous()
    p = c.params
    for call in range(2):
        out.zero_()
        torch.cuda.synchronize()
        st = f(t["q2"].data_ptr(), t["q3"].data_ptr(), p.n2, p.n2, p.n3, t["rc"].data_ptr(),
               t["zz"].data_ptr(), udx2m.data_ptr(), udx3m.data_ptr(), p.dt, p.rext2, p.alx3,
               out.data_ptr(), None)
        assert st == 0, st
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[0] == pytest.approx(ref["cflm"], rel=1e-13, abs=0), call
        assert got[1] == pytest.approx(ref["q3avg"], rel=1e-13, abs=0), call
    # a NaN velocity is not hidden by the max reduction: the CFL number is +inf
    t["q2"][5, 3] = float("nan")
    st = f(t["q2"].data_ptr(), t["q3"].data_ptr(), p.n2, p.n2, p.n3, t["rc"].data_ptr(),
           t["zz"].data_ptr(), udx2m.data_ptr(), udx3m.data_ptr(), p.dt, p.rext2, p.alx3,
           out.data_ptr(), None)
    assert st == 0, st
    torch.cuda.synchronize()
    assert out.cpu().numpy()[0] == float("inf")


def test_cfl_noalloc_rejects_grids_beyond_its_scratch():
    lib = fb.lib()
    f = lib.fb_cfl_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                  ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    n3 = 8192 + 2
    assert f(dummy, dummy, 8, 8, n3, dummy, dummy, dummy, dummy, 1e-3, 1.0, 1.0, dummy, None) == fb.FB_ERR_UNSUPPORTED
