"""CPU oracle for the FRiBoIS2D fluid time step -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package, always as the checker.  The product
(``fribois2d_b200``) never imports it.

Parity status: UNPINNED against the reference binary (Fortran/MPI, not
buildable here, no tests or golden vectors upstream).  What is pinned:

* ``phini`` calls LAPACK's DGEEV and DGESV through scipy with the same
  arguments as src/phini.F90:52-92;
* the C restatement of DGTTRF/DGTTRS is checked against scipy's LAPACK;
* the C oracle is cross-checked against an independent NumPy restatement
  (``oracle.npref``) that calls LAPACK's DGTTRF/DGTTRS for every line.

Parsers here restate src/utils_proc.F90 (list-directed reads) independently
of the product's C++ parser, so that the tests compare two readings of the
same deck.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, List, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libfbo.so")

# ------------------------------------------------------------------ build


def build(force: bool = False) -> str:
    """Compile fbo.c (-O3, no FP contraction, OpenMP) into libfbo.so."""
    src = os.path.join(HERE, "fbo.c")
    hdr = os.path.join(HERE, "fbo.h")
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(src), os.path.getmtime(hdr))):
        return LIB
    cmd = ["gcc", "-O3", "-std=gnu11", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           "-fPIC", "-shared", "-o", LIB + ".tmp", src, "-lm"]
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


# ------------------------------------------------------- list-directed read


class _Records:
    """Sequential Fortran records with list-directed ``read(u,*)``."""

    def __init__(self, path: str):
        with open(path, "r") as fh:
            self.lines = fh.read().split("\n")
        self.pos = 0

    def skip(self) -> None:
        self.pos += 1

    def read(self, n: int) -> List[str]:
        vals: List[str] = []
        while len(vals) < n:
            if self.pos >= len(self.lines):
                raise EOFError("end of file during list-directed read")
            line = self.lines[self.pos]
            self.pos += 1
            stop = False
            for tok in line.replace(",", " ").split():
                if tok.startswith("/"):
                    stop = True
                    break
                vals.append(tok)
                if len(vals) == n:
                    break
            if stop and len(vals) < n:
                raise ValueError("slash before all values were read")
        return vals


def _real(t: str) -> float:
    return float(t.replace("d", "e").replace("D", "e"))


def _logical(t: str) -> bool:
    t = t.lstrip(".").upper()
    if t.startswith("T"):
        return True
    if t.startswith("F"):
        return False
    raise ValueError(f"not a logical: {t}")


def parse_deck(path: str) -> Dict:
    """Read an ``input_FSI`` directory the way the reference does.

    global_par.in  src/utils_proc.F90:59-83
    fluid_par.in   src/utils_proc.F90:142-170
    rigid_par.in   src/utils_proc.F90:18-36
    y/zcoord.dat   src/cordin.F90:255-266
    lmdata.in      src/utils_proc.F90:529-548 (markers = newlines - 1)
    """
    d: Dict = {}
    r = _Records(os.path.join(path, "global_par.in"))
    r.skip()
    d["dt"] = _real(r.read(1)[0])
    d["idtv"] = _logical(r.read(1)[0])
    d["dtmax"] = _real(r.read(1)[0])
    d["cflmax"] = _real(r.read(1)[0])
    d["cfllim"] = _real(r.read(1)[0])
    d["outfol"] = r.read(1)[0]
    d["irest"] = _logical(r.read(1)[0])
    d["trestart"] = _real(r.read(1)[0])
    r.skip(); r.skip(); r.skip()
    d["ibact"] = _logical(r.read(1)[0])
    r.skip(); r.skip(); r.skip()
    d["kprobe"] = _real(r.read(1)[0])
    d["prlgr"] = _logical(r.read(1)[0])
    d["tprtag"] = _real(r.read(1)[0])
    d["forst"] = int(r.read(1)[0])
    d["radiusSD"] = _real(r.read(1)[0])
    d["wfun"] = int(r.read(1)[0])

    r = _Records(os.path.join(path, "fluid_par.in"))
    r.skip()
    d["alx3"] = _real(r.read(1)[0])
    d["rext2"] = _real(r.read(1)[0])
    n3, n2 = r.read(2)
    d["n3"], d["n2"] = int(n3), int(n2)
    d["istr3"] = int(r.read(1)[0])
    r.read(5)
    r.read(2)
    d["istr2"] = int(r.read(1)[0])
    r.read(5)
    r.read(2)
    r.skip(); r.skip(); r.skip()
    d["nsst"] = int(r.read(1)[0])
    d["nwrit"] = _logical(r.read(1)[0])
    d["tframef"] = _real(r.read(1)[0])
    d["resid"] = _real(r.read(1)[0])
    d["cou"] = _real(r.read(1)[0])
    r.skip(); r.skip(); r.skip()
    d["visc"] = _real(r.read(1)[0])
    d["inslws"] = _logical(r.read(1)[0])
    d["inslwn"] = _logical(r.read(1)[0])
    d["q3uw"] = _real(r.read(1)[0])
    d["q3lw"] = _real(r.read(1)[0])

    r = _Records(os.path.join(path, "rigid_par.in"))
    r.skip()
    d["cbody"] = _logical(r.read(1)[0])
    d["cmposi"] = tuple(_real(t) for t in r.read(2))
    d["cmroti"] = _real(r.read(1)[0])
    # the dummy argument is a scalar: only the first value is read
    d["ipert"] = (_real(r.read(1)[0]), 0.0, 0.0)
    d["rbgravF"] = tuple(_real(t) for t in r.read(2))
    d["rbden"] = _real(r.read(1)[0])
    d["rba"] = tuple(_real(t) for t in r.read(2))
    d["rbmcon"] = tuple(int(t) for t in r.read(3))
    d["kk"] = tuple(_real(t) for t in r.read(3))
    d["kk3"] = tuple(_real(t) for t in r.read(3))
    d["cc"] = tuple(_real(t) for t in r.read(3))
    d["rtcoup"] = _logical(r.read(1)[0])
    d["rrr"] = _real(r.read(1)[0])

    if d["istr2"] != 100 or d["istr3"] != 100:
        raise ValueError("only grids read from ycoord.dat/zcoord.dat (istr = 100) are supported")
    r = _Records(os.path.join(path, "ycoord.dat"))
    d["ycoord"] = np.array([_real(r.read(1)[0]) for _ in range(d["n2"])], dtype=np.float64)
    r = _Records(os.path.join(path, "zcoord.dat"))
    d["zcoord"] = np.array([_real(r.read(1)[0]) for _ in range(d["n3"])], dtype=np.float64)

    nlm = 0
    vert = np.zeros((0, 2))
    if d["ibact"]:
        with open(os.path.join(path, "lmdata.in"), "rb") as fh:
            nlm = fh.read().count(b"\n") - 1
        r = _Records(os.path.join(path, "lmdata.in"))
        vert = np.array([[_real(t) for t in r.read(2)] for _ in range(nlm + 1)], dtype=np.float64)
    d["nlm"] = nlm
    d["vert"] = vert
    return d


# ------------------------------------------------------------- eigen set-up


def phini(amphk: np.ndarray, acphk: np.ndarray, apphk: np.ndarray) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """src/phini.F90:4-99: DGEEV of the z operator, DGESV for its inverse.

    Inputs are 1-based arrays as returned by the oracle (index 0 unused).
    Returns ``(wr, zmm, zmmt)`` with ``zmm``/``zmmt`` ``n3m x n3m`` in
    Fortran (column-major) order.
    """
    from scipy.linalg import lapack

    n3m = len(amphk) - 3  # arrays are allocated n3 + 2
    bm = np.zeros((n3m, n3m), dtype=np.float64, order="F")
    for kc in range(1, n3m + 1):
        bm[kc - 1, kc - 1] = acphk[kc]
        if kc + 1 <= n3m:
            bm[kc - 1, kc] = apphk[kc]
        if kc - 1 >= 1:
            bm[kc - 1, kc - 2] = amphk[kc]
    wr, wi, vl, vr, info = lapack.dgeev(bm, compute_vl=0, compute_vr=1)
    if info != 0:
        raise RuntimeError("DGEEV failed")
    if np.max(np.abs(wi)) != 0.0:
        raise RuntimeError("complex eigenvalues in the z Poisson operator")
    zmm = np.asfortranarray(vr)
    lu, piv, zmmt, info = lapack.dgesv(vr.copy(order="F"), np.eye(n3m, order="F"))
    if info != 0:
        raise RuntimeError("DGESV failed")
    return np.ascontiguousarray(wr), zmm, np.asfortranarray(zmmt)


# ------------------------------------------------------------------ ctypes


class _Params(ctypes.Structure):
    _fields_ = [
        ("n2", ctypes.c_int), ("n3", ctypes.c_int), ("nsst", ctypes.c_int),
        ("idtv", ctypes.c_int), ("ibact", ctypes.c_int), ("cbody", ctypes.c_int),
        ("wfun", ctypes.c_int), ("forst", ctypes.c_int), ("inslws", ctypes.c_int),
        ("inslwn", ctypes.c_int), ("rtcoup", ctypes.c_int), ("nlm", ctypes.c_int),
        ("rbmcon", ctypes.c_int * 3),
        ("alx3", ctypes.c_double), ("rext2", ctypes.c_double), ("dt", ctypes.c_double),
        ("dtmax", ctypes.c_double), ("cflmax", ctypes.c_double), ("cfllim", ctypes.c_double),
        ("resid", ctypes.c_double), ("cou", ctypes.c_double), ("visc", ctypes.c_double),
        ("q3uw", ctypes.c_double), ("q3lw", ctypes.c_double), ("kprobe", ctypes.c_double),
        ("radiusSD", ctypes.c_double), ("rbden", ctypes.c_double),
        ("rba", ctypes.c_double * 2), ("cmposi", ctypes.c_double * 2),
        ("cmroti", ctypes.c_double), ("rbgravF", ctypes.c_double * 2),
        ("kk", ctypes.c_double * 3), ("kk3", ctypes.c_double * 3), ("cc", ctypes.c_double * 3),
        ("rrr", ctypes.c_double), ("ipert", ctypes.c_double * 3),
    ]


# ids mirrored from fbo.h
IDS = dict(q2=0, q3=1, pr=2, dph=3, q2f=4, q3f=5, rhs=6, rhs2=7, rhs3=8, ru2=9, ru3=10,
           qcap=11, fey=12, fez=13, qb2s=20, qb2n=21, dqb2s=22, dqb2n=23, qb3s=24, qb3n=25,
           dqb3s=26, dqb3n=27, dq2x2o=28, dq3x2o=29, rc=40, rm=41, zz=42, zm=43, g2rc=44,
           g2rm=45, g3rc=46, g3rm=47, udx2c=48, udx2m=49, udx3c=50, udx3m=51, am2j=52,
           ac2j=53, ap2j=54, am3j=55, ac3j=56, ap3j=57, am3ck=58, ac3ck=59, ap3ck=60,
           am3sk=61, ac3sk=62, ap3sk=63, amphj=64, acphj=65, apphj=66, amphk=67, acphk=68,
           apphk=69, wr=80, zmm=81, zmmt=82, lmcc=90, lmvel=91, lmacc=92, lmnor=93, lmA=94,
           vert=95, phi=96, cl=97, press=98, tau=99, bcerrv=100, bcerrw=101, rigid=110,
           scalars=111, forces=112)
IIDS = dict(lmind=0, eulins=1, jmv=2, jpv=3, kmv=4, kpv=5)
FIELDS = ("q2", "q3", "pr", "dph", "q2f", "q3f", "rhs", "rhs2", "rhs3", "ru2", "ru3", "qcap",
          "fey", "fez")
STAGES = dict(cfl=0, boucdq=1, hdnl2=2, hdnl3=3, invtr2=4, invtr3=5, lgrdistribution=6,
              forcing=7, helsolve=8, divg=9, phcalc=10, updvp=11, prcalc=12, pr_submean=13,
              boucqt=14, checkbcs=15, loads=16, rigid=17, solq2j=18, solq2k=19, solq3j=20,
              solq3k=21)
KG = 2  # ghost rows below k = 1


def _load():
    lib = ctypes.CDLL(build())
    P = ctypes.POINTER
    dp = P(ctypes.c_double)
    lib.fbo_create.restype = ctypes.c_void_p
    lib.fbo_create.argtypes = [P(_Params), dp, dp, dp]
    lib.fbo_destroy.argtypes = [ctypes.c_void_p]
    lib.fbo_set_eigen.argtypes = [ctypes.c_void_p, dp, dp, dp]
    lib.fbo_array.restype = dp
    lib.fbo_array.argtypes = [ctypes.c_void_p, ctypes.c_int, P(ctypes.c_long)]
    lib.fbo_iarray.restype = P(ctypes.c_int)
    lib.fbo_iarray.argtypes = [ctypes.c_void_p, ctypes.c_int, P(ctypes.c_long)]
    for f in ("fbo_fluid_tsch", "fbo_rigid", "fbo_step"):
        getattr(lib, f).argtypes = [ctypes.c_void_p, ctypes.c_int]
        getattr(lib, f).restype = ctypes.c_int
    lib.fbo_set_substep.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.fbo_stage.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.fbo_stage.restype = ctypes.c_int
    lib.fbo_status.argtypes = [ctypes.c_void_p]
    lib.fbo_status.restype = ctypes.c_int
    lib.fbo_dgttrf.argtypes = [ctypes.c_int, dp, dp, dp, dp, P(ctypes.c_int)]
    lib.fbo_dgttrf.restype = ctypes.c_int
    lib.fbo_dgtts2.argtypes = [ctypes.c_int, dp, dp, dp, dp, P(ctypes.c_int), dp]
    lib.fbo_set_threads.argtypes = [ctypes.c_int]
    lib.fbo_coupled_step.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_double, dp]
    lib.fbo_coupled_step.restype = ctypes.c_int
    lib.fbo_rigid_mode.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    lib.fbo_rigid_mode.restype = ctypes.c_int
    lib.fbo_snapshot.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.fbo_snapshot.restype = ctypes.c_int
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _load()
    return _LIB


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def params_from_deck(d: Dict) -> _Params:
    p = _Params()
    for k in ("n2", "n3", "nsst", "wfun", "forst", "nlm"):
        setattr(p, k, int(d[k]))
    for k in ("idtv", "ibact", "cbody", "inslws", "inslwn", "rtcoup"):
        setattr(p, k, int(bool(d[k])))
    for k in ("alx3", "rext2", "dt", "dtmax", "cflmax", "cfllim", "resid", "cou", "visc",
              "q3uw", "q3lw", "kprobe", "radiusSD", "rbden", "cmroti", "rrr"):
        setattr(p, k, float(d[k]))
    for k, n in (("rbmcon", 3),):
        for i in range(n):
            getattr(p, k)[i] = int(d[k][i])
    for k, n in (("rba", 2), ("cmposi", 2), ("rbgravF", 2), ("kk", 3), ("kk3", 3), ("cc", 3),
                 ("ipert", 3)):
        for i in range(n):
            getattr(p, k)[i] = float(d[k][i])
    return p


class Oracle:
    """One case on the CPU oracle.  Fields are exposed as ``(k, j)`` views
    with ``k = -2 .. n3+2`` mapped to rows ``0 .. n3+4``."""

    def __init__(self, deck: Dict, eigen=None, threads: int = 0):
        self.lib = lib()
        if threads:
            self.lib.fbo_set_threads(int(threads))
        self.deck = deck
        self.n2, self.n3 = deck["n2"], deck["n3"]
        self.n2m, self.n3m = self.n2 - 1, self.n3 - 1
        self.nlm = deck["nlm"]
        p = params_from_deck(deck)
        y = np.ascontiguousarray(deck["ycoord"], dtype=np.float64)
        z = np.ascontiguousarray(deck["zcoord"], dtype=np.float64)
        v = np.ascontiguousarray(deck["vert"], dtype=np.float64).reshape(-1)
        if v.size == 0:
            v = np.zeros(2)
        self.h = self.lib.fbo_create(ctypes.byref(p), _dptr(y), _dptr(z), _dptr(v))
        self._keep = (p, y, z, v)
        if eigen is None:
            eigen = phini(self.a("amphk"), self.a("acphk"), self.a("apphk"))
        self.set_eigen(*eigen)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.fbo_destroy(self.h)
            self.h = None

    def set_eigen(self, wr, zmm, zmmt) -> None:
        wr = np.ascontiguousarray(wr, dtype=np.float64)
        zmm = np.asfortranarray(zmm, dtype=np.float64)
        zmmt = np.asfortranarray(zmmt, dtype=np.float64)
        self.eigen = (wr, zmm, zmmt)
        self.lib.fbo_set_eigen(self.h, _dptr(wr), _dptr(zmm.reshape(-1, order="F").copy()),
                               _dptr(zmmt.reshape(-1, order="F").copy()))

    def a(self, name: str) -> np.ndarray:
        """Zero-copy view of an oracle array."""
        n = ctypes.c_long()
        ptr = self.lib.fbo_array(self.h, IDS[name], ctypes.byref(n))
        arr = np.ctypeslib.as_array(ptr, shape=(n.value,))
        if name in FIELDS:
            return arr.reshape(self.n3 + 1 + 2 * KG, self.n2)
        return arr

    def ia(self, name: str) -> np.ndarray:
        n = ctypes.c_long()
        ptr = self.lib.fbo_iarray(self.h, IIDS[name], ctypes.byref(n))
        return np.ctypeslib.as_array(ptr, shape=(n.value,))

    def field(self, name: str, k0: int = 0, k1: int = None) -> np.ndarray:
        """Rows ``k0..k1`` (inclusive, reference k numbering) of a field."""
        if k1 is None:
            k1 = self.n3
        return self.a(name)[k0 + KG:k1 + KG + 1]

    def stage(self, name: str, n: int = 1) -> int:
        return self.lib.fbo_stage(self.h, STAGES[name], n)

    def set_substep(self, ns: int, n: int) -> None:
        self.lib.fbo_set_substep(self.h, ns, n)

    def fluid_tsch(self, ns: int) -> int:
        return self.lib.fbo_fluid_tsch(self.h, ns)

    def rigid(self, ns: int) -> int:
        return self.lib.fbo_rigid(self.h, ns)

    def step(self, ns: int) -> int:
        return self.lib.fbo_step(self.h, ns)

    def scalars(self) -> Dict[str, float]:
        s = self.a("scalars")
        keys = ("time", "dt", "dt_o", "beta", "al", "ga", "ro", "cflm", "q3avg", "nbcv",
                "nbcw", "ddmin", "pravg")
        return {k: float(s[i]) for i, k in enumerate(keys)}

    def coupled_step(self, ns: int, tol: float = 1e-8, maxit: int = 50, omega0: float = 0.5,
                     guess: np.ndarray = None) -> Tuple[int, int, float]:
        """One strongly coupled step (fbo_coupled_step; the project's own
        iteration, the reference couples explicitly).  The initial guess is
        the plain predictor's -- the last two converged loads extrapolated
        linearly -- unless `guess` (Fy, Fz, M) is given; the relaxation
        starts from the last Aitken factor of an earlier step.  Returns
        (status, fluid solves, relative load residual of the guess)."""
        hist = self.__dict__.setdefault("_coupled_loads", [])
        last = self.__dict__.setdefault("_aitken", [])
        if guess is not None:
            F0 = np.asarray(guess, dtype=np.float64)
        elif len(hist) >= 2:
            F0 = 2.0 * hist[-1] - hist[-2]
        elif len(hist) == 1:
            F0 = hist[-1].copy()
        else:
            F0 = np.zeros(3)
        F0 = np.ascontiguousarray(F0, dtype=np.float64)
        q = next((i for i in range(3) if int(self.deck["rbmcon"][i]) == 0), 0)
        out = np.zeros(7)
        w0 = min(2.0, max(0.05, last[-1])) if last else omega0
        st = self.lib.fbo_coupled_step(self.h, ns, _dptr(F0), tol, maxit, q, w0, _dptr(out))
        if st == 0:
            hist.append(out[:3].copy())
            if out[6] != 0.0:
                last.append(float(out[6]))
        return st, int(out[3]), float(out[4])

    def add_v_perturbation(self, pert: np.ndarray) -> None:
        """Add a ``(n3m, n2)`` perturbation to ``q2`` rows ``k = 1..n3m``."""
        self.field("q2", 1, self.n3m)[:] += pert


def load_case(path: str, threads: int = 0) -> Oracle:
    return Oracle(parse_deck(path), threads=threads)
