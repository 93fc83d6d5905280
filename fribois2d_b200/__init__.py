"""B200-native FRiBoIS2D fluid time step.

The product is the native library ``libfribois2d.so`` (CUDA, sm_100a) behind
the C ABI in ``include/fribois2d.h``.  This module is a thin ctypes binding
that mirrors the reference's driver-level interface (src/main.F90:51-97):

* ``Solver(input_dir)``      -- read_genin + fluid_pre + read_rigid + rigid_pre
* ``Solver.fluid_tsch(ns)``  -- fluid_tsch(ns, 'a')  (src/fluid_tsch.F90:4)
* ``Solver.rigid(ns)``       -- rigid(ns, 'a', 0)    (src/rigid.F90:4), time += dt
* ``Solver.advance(ns0, n)`` -- n iterations of the main loop body, CUDA graph

Errors are raised as :class:`FBError` carrying the library's status code,
where the reference would call stopcase/MPI_ABORT.  There is no CPU
fallback: if the native library cannot be loaded, import-time use fails.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfribois2d.so")

FB_OK = 0
STATUS = {0: "FB_OK", 1: "FB_ERR_CFL", 2: "FB_ERR_MLS", 3: "FB_ERR_MARKER_OUT",
          4: "FB_ERR_INPUT", 5: "FB_ERR_CUDA", 6: "FB_ERR_STATE", 7: "FB_ERR_UNSUPPORTED",
          8: "FB_ERR_NUMERIC", 9: "FB_ERR_TIMEOUT"}
FB_ERR_CFL, FB_ERR_MLS, FB_ERR_MARKER_OUT, FB_ERR_INPUT = 1, 2, 3, 4
FB_ERR_CUDA, FB_ERR_STATE, FB_ERR_UNSUPPORTED, FB_ERR_NUMERIC, FB_ERR_TIMEOUT = 5, 6, 7, 8, 9
POISSON_FP64, POISSON_TF32X3, POISSON_INT8X8 = 0, 1, 2
COUPLING_LOOSE, COUPLING_STRONG, COUPLING_LEARNED = 0, 1, 2
BATCH_GROUPED, BATCH_GRAPH = 0, 1

# array ids (include/fribois2d.h)
IDS = dict(q2=0, q3=1, pr=2, dph=3, rhs2=7, rhs3=8, ru2=9, ru3=10, qb2s=20, qb2n=21, dqb2s=22,
           dqb2n=23, qb3s=24, qb3n=25, dqb3s=26, dqb3n=27, dq2x2o=28, dq3x2o=29, rc=40, rm=41,
           zz=42, zm=43, udx2c=48, udx2m=49, udx3c=50, udx3m=51, amphj=64, acphj=65, apphj=66,
           amphk=67, acphk=68, apphk=69, wr=80, zmm=81, zmmt=82, lmcc=90, lmvel=91, lmacc=92,
           lmnor=93, lmA=94, vert=95, phi=96, cl=97, press=98, tau=99, bcerrv=100, bcerrw=101,
           rigid=110, scalars=111, forces=112, hmn=113)
IIDS = dict(lmind=0, eulins=1)
FIELDS = ("q2", "q3", "pr", "dph", "rhs2", "rhs3", "ru2", "ru3")
BOUNDARY = ("qb2s", "qb2n", "dqb2s", "dqb2n", "qb3s", "qb3n", "dqb3s", "dqb3n", "dq2x2o", "dq3x2o")
STAGES = dict(cfl=0, boucdq=1, nl_rhs=2, lgrdistribution=6, forcing=7, helsolve=8, divg=9,
              phcalc=10, updvp=11, pr_submean=13, checkbcs=15, loads=16, rigid=17,
              gemm_fwd=100, poisson_tri=101, gemm_bwd=102, tf32x3_gemm=103, i8_split=104,
              i8x8_gemm=105)
HIST_COLS = 31
HIST_NAMES = ("time", "Fy", "Fz", "M", "Fyp", "Fzp", "Fyv", "Fzv", "time_end", "py", "pz", "pa",
              "vy", "vz", "va", "ay", "az", "aa", "nbcv", "nbcw", "cflm", "dt",
              "cflm_end", "dmax", "ektot", "vorti", "vmax2", "vmax3", "vmin2", "vmin3", "solves")
SCALAR_NAMES = ("time", "dt", "dt_o", "beta", "al", "ga", "ro", "cflm", "q3avg", "nbcv", "nbcw",
                "ddmin", "pravg")


class FBError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        super().__init__(f"{where}: {STATUS.get(code, code)} ({_status_string(code)})")


_LIB = None


def _status_string(code: int) -> str:
    try:
        return lib().fb_status_string(code).decode()
    except Exception:  # pragma: no cover - library missing
        return "?"


def lib() -> ctypes.CDLL:
    """Load the native library (never a fallback: raises if it is missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"native library missing: {LIB_PATH} (run python -m fribois2d_b200.build)")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp, dp, ip, i64 = ctypes.c_void_p, P(ctypes.c_double), P(ctypes.c_int32), ctypes.c_int64
    sig = {
        "fb_create": ([ctypes.c_char_p, ctypes.c_int, P(vp)], ctypes.c_int),
        "fb_destroy": ([vp], ctypes.c_int),
        "fb_fluid_tsch": ([vp, ctypes.c_int], ctypes.c_int),
        "fb_rigid": ([vp, ctypes.c_int, dp], ctypes.c_int),
        "fb_advance": ([vp, ctypes.c_int, ctypes.c_int, dp], ctypes.c_int),
        "fb_get_loads": ([vp, dp, dp], ctypes.c_int),
        "fb_set_markers": ([vp, dp, dp, dp, dp], ctypes.c_int),
        "fb_get_markers": ([vp, dp, dp, dp, dp], ctypes.c_int),
        "fb_step_markers": ([vp, ctypes.c_int, dp, dp, dp, dp, dp], ctypes.c_int),
        "fb_get_dims": ([vp, ip], ctypes.c_int),
        "fb_get_array": ([vp, ctypes.c_int, dp, i64], ctypes.c_int),
        "fb_set_array": ([vp, ctypes.c_int, dp, i64], ctypes.c_int),
        "fb_get_iarray": ([vp, ctypes.c_int, ip, i64], ctypes.c_int),
        "fb_synchronize": ([vp], ctypes.c_int),
        "fb_set_substep": ([vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "fb_stage": ([vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "fb_last_advance_ms": ([vp, dp], ctypes.c_int),
        "fb_time_stage": ([vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp], ctypes.c_int),
        "fb_kernel_count": ([vp, ip], ctypes.c_int),
        "fb_host_create": ([ctypes.c_char_p, P(vp)], ctypes.c_int),
        "fb_host_destroy": ([vp], ctypes.c_int),
        "fb_host_dims": ([vp, ip], ctypes.c_int),
        "fb_host_array": ([vp, ctypes.c_int, dp, i64], ctypes.c_int),
        "fb_eigen_tridiag": ([ctypes.c_int, dp, dp, dp, dp, dp, dp], ctypes.c_int),
        "fb_set_poisson": ([vp, ctypes.c_int], ctypes.c_int),
        "fb_set_refinement": ([vp, ctypes.c_int], ctypes.c_int),
        "fb_set_report": ([vp, ctypes.c_int], ctypes.c_int),
        "fb_set_coupling": ([vp, ctypes.c_int, ctypes.c_double, ctypes.c_int], ctypes.c_int),
        "fb_set_predictor": ([vp, vp, P(ctypes.c_float)], ctypes.c_int),
        "fb_coupling_stats": ([vp, dp], ctypes.c_int),
        "fb_coupling_samples": ([vp, P(ctypes.c_float), P(ctypes.c_float), ctypes.c_int, ip], ctypes.c_int),
        "fb_mlp_create": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, P(vp)], ctypes.c_int),
        "fb_mlp_destroy": ([vp], ctypes.c_int),
        "fb_mlp_params": ([vp, ip], ctypes.c_int),
        "fb_mlp_get": ([vp, P(ctypes.c_float)], ctypes.c_int),
        "fb_mlp_set": ([vp, P(ctypes.c_float)], ctypes.c_int),
        "fb_mlp_predict": ([vp, P(ctypes.c_float), ctypes.c_int, P(ctypes.c_float)], ctypes.c_int),
        "fb_mlp_grad": ([vp, P(ctypes.c_float), P(ctypes.c_float), ctypes.c_int, P(ctypes.c_float),
                         P(ctypes.c_float)], ctypes.c_int),
        "fb_mlp_train": ([vp, P(ctypes.c_float), P(ctypes.c_float), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_float, ctypes.c_uint64, P(ctypes.c_float)], ctypes.c_int),
        "fb_batch_create": ([P(vp), ctypes.c_int, P(vp)], ctypes.c_int),
        "fb_batch_create_mode": ([P(vp), ctypes.c_int, ctypes.c_int, P(vp)], ctypes.c_int),
        "fb_batch_info": ([vp, P(ctypes.c_int32)], ctypes.c_int),
        "fb_batch_advance": ([vp, ctypes.c_int], ctypes.c_int),
        "fb_batch_last_ms": ([vp, dp], ctypes.c_int),
        "fb_batch_destroy": ([vp], ctypes.c_int),
        "fb_last_history": ([vp, dp], ctypes.c_int),
        "fb_write_restart": ([vp, ctypes.c_char_p], ctypes.c_int),
        "fb_read_restart": ([vp, ctypes.c_char_p], ctypes.c_int),
        "fb_gemm_i8x8": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp], ctypes.c_int),
        "fb_gemm_tf32x3": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp],
                           ctypes.c_int),
        "fb_autotune": ([vp, ip], ctypes.c_int),
        "fb_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "fb_version": ([], ctypes.c_char_p),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _LIB = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(code: int, where: str) -> None:
    if code != FB_OK:
        raise FBError(code, where)


class HostSetup:
    """Host-only set-up of a case (parsing, metrics, eigen data); no GPU."""

    def __init__(self, input_dir: str):
        self._lib = lib()
        h = ctypes.c_void_p()
        _check(self._lib.fb_host_create(input_dir.encode(), ctypes.byref(h)), "fb_host_create")
        self.h = h
        dims = (ctypes.c_int32 * 8)()
        _check(self._lib.fb_host_dims(self.h, dims), "fb_host_dims")
        self.n2, self.n3, self.nlm, self.nsst, self.idtv, self.ibact, self.wfun, self.forst = list(dims)
        self.n2m, self.n3m = self.n2 - 1, self.n3 - 1

    def __del__(self):
        if getattr(self, "h", None):
            self._lib.fb_host_destroy(self.h)
            self.h = None

    def array(self, name: str) -> np.ndarray:
        n = {"rc": self.n2, "rm": self.n2, "udx2c": self.n2, "udx2m": self.n2, "amphj": self.n2,
             "acphj": self.n2, "apphj": self.n2, "zz": self.n3, "zm": self.n3, "udx3c": self.n3,
             "udx3m": self.n3, "amphk": self.n3, "acphk": self.n3, "apphk": self.n3,
             "wr": self.n3m, "zmm": self.n3m ** 2, "zmmt": self.n3m ** 2, "lmcc": 2 * self.nlm,
             "lmvel": 2 * self.nlm, "lmacc": 2 * self.nlm, "lmnor": 2 * self.nlm,
             "lmA": self.nlm, "vert": 2 * (self.nlm + 1), "rigid": 18}[name]
        out = np.zeros(n, dtype=np.float64)
        _check(self._lib.fb_host_array(self.h, IDS[name], _dp(out), n), f"fb_host_array({name})")
        if name in ("zmm", "zmmt"):
            return out.reshape(self.n3m, self.n3m, order="F")
        return out


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class MLP:
    """The learned coupling predictor's perceptron (n_in -> 64 -> 64 -> n_out,
    tanh, FP32), trained and evaluated by the library's own CUDA kernels."""

    def __init__(self, n_in: int = 27, n_out: int = 2, seed: int = 0, device: int = 0):
        self._lib = lib()
        self.n_in, self.n_out = n_in, n_out
        self.m = ctypes.c_void_p()
        _check(self._lib.fb_mlp_create(int(device), n_in, n_out, int(seed), ctypes.byref(self.m)), "fb_mlp_create")
        n = ctypes.c_int()
        _check(self._lib.fb_mlp_params(self.m, ctypes.byref(n)), "fb_mlp_params")
        self.n_params = n.value

    def params(self) -> np.ndarray:
        p = np.zeros(self.n_params, dtype=np.float32)
        _check(self._lib.fb_mlp_get(self.m, _fp(p)), "fb_mlp_get")
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(self._lib.fb_mlp_set(self.m, _fp(p)), "fb_mlp_set")

    def predict(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], self.n_out), dtype=np.float32)
        _check(self._lib.fb_mlp_predict(self.m, _fp(x), x.shape[0], _fp(y)), "fb_mlp_predict")
        return y

    def grad(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = ctypes.c_float()
        _check(self._lib.fb_mlp_grad(self.m, _fp(x), _fp(t), x.shape[0], _fp(g), ctypes.byref(loss)),
               "fb_mlp_grad")
        return g, loss.value

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int, batch: int = 256, lr: float = 1e-3,
              seed: int = 0) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = ctypes.c_float()
        _check(self._lib.fb_mlp_train(self.m, _fp(x), _fp(t), x.shape[0], int(epochs), int(batch), float(lr),
                                      int(seed), ctypes.byref(loss)), "fb_mlp_train")
        return loss.value

    def close(self) -> None:
        if self.m:
            self._lib.fb_mlp_destroy(self.m)
            self.m = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent cases (Solver objects on one device, fixed dt, RK3) advanced
    together by one CUDA graph launch per step (fb_batch_*).  mode
    BATCH_GROUPED (default): one launch per stage over every group of cases of
    one launch geometry; BATCH_GRAPH: every case's own captured step on its
    own graph branch (bitwise equal to stepping it alone)."""

    def __init__(self, solvers, mode: int = BATCH_GROUPED):
        self.solvers = list(solvers)
        self._lib = lib()
        arr = (ctypes.c_void_p * len(self.solvers))(*[s.ctx.value for s in self.solvers])
        self.b = ctypes.c_void_p()
        _check(self._lib.fb_batch_create_mode(arr, len(self.solvers), int(mode), ctypes.byref(self.b)),
               "fb_batch_create_mode")

    def info(self) -> dict:
        """groups, cases on their own branch, own kernel launches per step."""
        out = (ctypes.c_int32 * 3)()
        _check(self._lib.fb_batch_info(self.b, out), "fb_batch_info")
        return {"groups": out[0], "singles": out[1], "launches": out[2]}

    def advance(self, nsteps: int) -> None:
        _check(self._lib.fb_batch_advance(self.b, int(nsteps)), "fb_batch_advance")

    def last_ms(self) -> float:
        ms = ctypes.c_double()
        _check(self._lib.fb_batch_last_ms(self.b, ctypes.byref(ms)), "fb_batch_last_ms")
        return ms.value

    def close(self) -> None:
        if self.b:
            self._lib.fb_batch_destroy(self.b)
            self.b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gemm_i8x8(A: np.ndarray, B: np.ndarray, device: int = 0) -> np.ndarray:
    """C = A @ B.T to FP64 accuracy on the INT8 tensor cores (8 digit slices)."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    M, K = A.shape
    N = B.shape[0]
    C = np.zeros((M, N), dtype=np.float64, order="F")
    _check(lib().fb_gemm_i8x8(int(device), M, N, K, _dp(A), _dp(B), _dp(C)), "fb_gemm_i8x8")
    return C


def gemm_tf32x3(A: np.ndarray, B: np.ndarray, device: int = 0, bn: int = 128) -> np.ndarray:
    """C = A @ B.T on the tensor cores in split precision (3xTF32)."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    M, K = A.shape
    N, K2 = B.shape
    if K2 != K:
        raise ValueError("inner dimensions differ")
    C = np.zeros((M, N), dtype=np.float64, order="F")
    _check(lib().fb_gemm_tf32x3(int(device), M, N, K, int(bn), _dp(A), _dp(B), _dp(C)), "fb_gemm_tf32x3")
    return C


def eigen_tridiag(am: np.ndarray, ac: np.ndarray, ap: np.ndarray):
    """Eigen-decomposition of a tridiagonal operator with positive off-diagonal
    products (the z Poisson operator of src/phini.F90:59-65)."""
    n = len(ac)
    am = np.ascontiguousarray(am, dtype=np.float64)
    ac = np.ascontiguousarray(ac, dtype=np.float64)
    ap = np.ascontiguousarray(ap, dtype=np.float64)
    wr = np.zeros(n)
    zmm = np.zeros(n * n)
    zmmt = np.zeros(n * n)
    _check(lib().fb_eigen_tridiag(n, _dp(am), _dp(ac), _dp(ap), _dp(wr), _dp(zmm), _dp(zmmt)),
           "fb_eigen_tridiag")
    return wr, zmm.reshape(n, n, order="F"), zmmt.reshape(n, n, order="F")


class Solver:
    """One FRiBoIS2D case on one GPU (the drop-in for src/main.F90's loop)."""

    def __init__(self, input_dir: str, device: int = 0):
        self._lib = lib()
        c = ctypes.c_void_p()
        _check(self._lib.fb_create(input_dir.encode(), int(device), ctypes.byref(c)), "fb_create")
        self.ctx = c
        dims = (ctypes.c_int32 * 8)()
        _check(self._lib.fb_get_dims(self.ctx, dims), "fb_get_dims")
        self.n2, self.n3, self.nlm, self.nsst, self.pitch, self.ldh = list(dims)[:6]
        self.n2m, self.n3m = self.n2 - 1, self.n3 - 1

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self._lib.fb_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- reference entry points
    def fluid_tsch(self, ns: int) -> None:
        _check(self._lib.fb_fluid_tsch(self.ctx, int(ns)), "fb_fluid_tsch")

    def rigid(self, ns: int) -> np.ndarray:
        row = np.zeros(8)
        _check(self._lib.fb_rigid(self.ctx, int(ns), _dp(row)), "fb_rigid")
        return row

    def advance(self, ns0: int, nsteps: int, history: bool = True) -> Optional[np.ndarray]:
        hist = np.zeros((nsteps, HIST_COLS)) if history else None
        ptr = _dp(hist) if history else ctypes.POINTER(ctypes.c_double)()
        _check(self._lib.fb_advance(self.ctx, int(ns0), int(nsteps), ptr), "fb_advance")
        return hist

    def last_advance_ms(self) -> float:
        ms = ctypes.c_double()
        _check(self._lib.fb_last_advance_ms(self.ctx, ctypes.byref(ms)), "fb_last_advance_ms")
        return ms.value

    def time_stage(self, name: str, n: int = 1, reps: int = 20) -> float:
        """Average device ms of one launch of a stage (overwrites the state)."""
        ms = ctypes.c_double()
        _check(self._lib.fb_time_stage(self.ctx, STAGES[name], int(n), int(reps), ctypes.byref(ms)),
               f"fb_time_stage({name})")
        return ms.value

    def kernel_count(self) -> int:
        v = ctypes.c_int32()
        _check(self._lib.fb_kernel_count(self.ctx, ctypes.byref(v)), "fb_kernel_count")
        return v.value

    def get_loads(self):
        p = np.zeros(self.nlm)
        t = np.zeros(2 * self.nlm)
        _check(self._lib.fb_get_loads(self.ctx, _dp(p), _dp(t)), "fb_get_loads")
        return p, t.reshape(self.nlm, 2)

    def set_markers(self, lmcc=None, lmvel=None, lmacc=None, lmnor=None) -> None:
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
                for a in (lmcc, lmvel, lmacc, lmnor)]
        ptrs = [ctypes.POINTER(ctypes.c_double)() if a is None else _dp(a) for a in arrs]
        _check(self._lib.fb_set_markers(self.ctx, *ptrs), "fb_set_markers")

    def get_markers(self):
        """lmcc, lmvel, lmacc, lmnor, each (nlm, 2), read with one wait."""
        out = [np.empty(2 * self.nlm) for _ in range(4)]
        _check(self._lib.fb_get_markers(self.ctx, *[_dp(a) for a in out]), "fb_get_markers")
        return [a.reshape(self.nlm, 2) for a in out]

    # ---- stages (one reference subroutine each)
    def set_substep(self, ns: int, n: int) -> None:
        _check(self._lib.fb_set_substep(self.ctx, int(ns), int(n)), "fb_set_substep")

    def stage(self, name: str, n: int = 1) -> int:
        return self._lib.fb_stage(self.ctx, STAGES[name], int(n))

    # ---- state
    def _count(self, name: str) -> int:
        if name in FIELDS:
            return (self.n3 + 1) * self.n2
        if name in BOUNDARY or name in ("rc", "rm", "udx2c", "udx2m", "amphj", "acphj", "apphj"):
            return self.n2
        if name in ("zz", "zm", "udx3c", "udx3m", "amphk", "acphk", "apphk"):
            return self.n3
        return {"wr": self.n3m, "zmm": self.n3m ** 2, "zmmt": self.n3m ** 2,
                "lmcc": 2 * self.nlm, "lmvel": 2 * self.nlm, "lmacc": 2 * self.nlm,
                "lmnor": 2 * self.nlm, "lmA": self.nlm, "vert": 2 * (self.nlm + 1),
                "phi": 18 * self.nlm, "cl": 2 * self.nlm, "press": self.nlm, "tau": 2 * self.nlm,
                "bcerrv": self.nlm, "bcerrw": self.nlm, "rigid": 18, "scalars": 13,
                "forces": 8, "hmn": self.n3m * self.ldh}[name]

    def get(self, name: str) -> np.ndarray:
        """Copy of a device array; fields come back as ``(n3+1, n2)``: row k, column j-1."""
        n = self._count(name)
        out = np.zeros(n)
        _check(self._lib.fb_get_array(self.ctx, IDS[name], _dp(out), n), f"fb_get_array({name})")
        if name in FIELDS:
            return out.reshape(self.n3 + 1, self.n2)
        if name in ("zmm", "zmmt"):
            return out.reshape(self.n3m, self.n3m, order="F")
        return out

    def set(self, name: str, value: np.ndarray) -> None:
        a = np.ascontiguousarray(value, dtype=np.float64).reshape(-1)
        n = self._count(name)
        if a.size != n:
            raise ValueError(f"{name}: expected {n} values, got {a.size}")
        _check(self._lib.fb_set_array(self.ctx, IDS[name], _dp(a), n), f"fb_set_array({name})")

    def geti(self, name: str) -> np.ndarray:
        n = {"lmind": 4 * self.nlm, "eulins": 36 * self.nlm}[name]
        out = np.zeros(n, dtype=np.int32)
        _check(self._lib.fb_get_iarray(self.ctx, IIDS[name], out.ctypes.data_as(
            ctypes.POINTER(ctypes.c_int32)), n), f"fb_get_iarray({name})")
        return out

    def scalars(self) -> dict:
        s = self.get("scalars")
        return {k: float(s[i]) for i, k in enumerate(SCALAR_NAMES)}

    def set_poisson(self, mode: int) -> None:
        """POISSON_INT8X8 (the default: FP64-accurate transforms on the INT8
        tensor cores), POISSON_FP64 (the transforms as cuBLAS DGEMMs, the
        comparison arm) or POISSON_TF32X3 (3xTF32 tensor-core transforms plus
        FP64 refinement sweeps)."""
        _check(self._lib.fb_set_poisson(self.ctx, int(mode)), "fb_set_poisson")

    def set_refinement(self, sweeps: int) -> None:
        """FP64 refinement sweeps of the precision form (1..4, default 2)."""
        _check(self._lib.fb_set_refinement(self.ctx, int(sweeps)), "fb_set_refinement")

    def autotune(self):
        """Tile shapes for this grid size, timed on this context: returns
        (helsolve tile height, tensor-core GEMM tile width)."""
        ch = (ctypes.c_int32 * 2)()
        _check(self._lib.fb_autotune(self.ctx, ch), "fb_autotune")
        return int(ch[0]), int(ch[1])

    def set_coupling(self, mode: int, tol: float = 1e-8, max_iter: int = 50) -> None:
        """COUPLING_LOOSE (the reference), COUPLING_STRONG or COUPLING_LEARNED."""
        _check(self._lib.fb_set_coupling(self.ctx, int(mode), float(tol), int(max_iter)), "fb_set_coupling")

    def set_predictor(self, mlp, norm) -> None:
        self._norm = np.ascontiguousarray(norm, dtype=np.float32)
        _check(self._lib.fb_set_predictor(self.ctx, mlp.m, _fp(self._norm)), "fb_set_predictor")
        self._mlp = mlp   # keep it alive while the context uses it

    def coupling_stats(self) -> dict:
        out = np.zeros(4)
        _check(self._lib.fb_coupling_stats(self.ctx, _dp(out)), "fb_coupling_stats")
        return {"steps": out[0], "solves": out[1], "unconverged": out[2], "initial_residual": out[3]}

    def coupling_samples(self):
        n = ctypes.c_int()
        _check(self._lib.fb_coupling_samples(self.ctx, None, None, 0, ctypes.byref(n)), "fb_coupling_samples")
        x = np.zeros((n.value, 27), dtype=np.float32)
        t = np.zeros((n.value, 2), dtype=np.float32)
        if n.value:
            _check(self._lib.fb_coupling_samples(self.ctx, _fp(x), _fp(t), n.value, ctypes.byref(n)),
                   "fb_coupling_samples")
        return x, t

    def set_report(self, on: bool = True) -> None:
        """End-of-step diagnostics of ttime.F90 into history columns 22..29."""
        _check(self._lib.fb_set_report(self.ctx, int(bool(on))), "fb_set_report")

    def last_history(self) -> np.ndarray:
        row = np.zeros(HIST_COLS)
        _check(self._lib.fb_last_history(self.ctx, _dp(row)), "fb_last_history")
        return row

    def write_restart(self, folder: str) -> None:
        os.makedirs(folder, exist_ok=True)
        _check(self._lib.fb_write_restart(self.ctx, folder.encode()), "fb_write_restart")

    def read_restart(self, folder: str) -> None:
        _check(self._lib.fb_read_restart(self.ctx, folder.encode()), "fb_read_restart")

    def synchronize(self) -> None:
        _check(self._lib.fb_synchronize(self.ctx), "fb_synchronize")

    def dims(self) -> list:
        """n2, n3, nlm, nsst, field pitch, Poisson pitch, pivoting flags,
        helsolve windows of substep 1 (y | z << 8; 0 = full line scans)."""
        d = (ctypes.c_int32 * 8)()
        _check(self._lib.fb_get_dims(self.ctx, d), "fb_get_dims")
        return list(d)


def version() -> str:
    return lib().fb_version().decode()
