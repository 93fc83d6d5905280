"""Generate the golden fixtures under tests/golden/.

The reference (Fortran/MPI) cannot be built here and ships no tests or
golden vectors, so the fixtures pin the two things that can be pinned:

* ``lapack_gtt.npz`` -- LAPACK's own DGTTRF/DGTTRS (through scipy) on the
  kinds of tridiagonal systems the reference factorises per line
  (src/solve_fluid.F90, src/phcalc_outflow.F90), including pivoting ones;
* ``phini_tiny.npz`` -- LAPACK DGEEV + DGESV on the z Poisson operator of
  the small cylinder case, exactly as src/phini.F90:52-92 calls them;
* ``traj_<case>.npz`` -- short trajectories of the CPU oracle on the two
  small cases (per-step loads and rigid-body state, final fields), used to
  catch regressions in the oracle and as a fixed target for the device;
* ``hist_<case>.npz`` -- full-length oracle histories of the benched cases
  (the 384 x 256 VIV cylinder over 2000 steps, the 1024 x 768 galloping
  rectangle over 5000 steps): the forcecomp.out and rigid-state rows of
  every step and the final q2, q3, pr sampled every 4th row and column.
  The oracle computes phini through LAPACK here, as the reference does.

Run:  python tests/golden/make_golden.py            (small fixtures)
      python tests/golden/make_golden.py --hist NAME [THREADS] (one long history)
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from fribois2d_b200 import case as cases  # noqa: E402

TRAJ_STEPS = 40


def lapack_systems(seed: int = 7):
    from scipy.linalg import lapack
    rng = np.random.default_rng(seed)
    out = {}
    specs = []
    for n in (3, 5, 17, 40, 64):
        # diagonally dominant, unit diagonal (the normalised Helmholtz rows)
        lo = rng.uniform(-0.45, 0.0, n - 1)
        up = rng.uniform(-0.45, 0.0, n - 1)
        specs.append(("dom", n, lo, np.ones(n), up))
        # weakly dominant with pivoting (the near-null Poisson mode)
        lo2 = rng.uniform(-1.5, 1.5, n - 1)
        di2 = rng.uniform(-0.3, 0.3, n)
        up2 = rng.uniform(-1.0, 1.0, n - 1)
        specs.append(("piv", n, lo2, di2, up2))
    for i, (kind, n, lo, di, up) in enumerate(specs):
        b = rng.standard_normal(n)
        dl, d, du, du2, ipiv, info = lapack.dgttrf(lo.copy(), di.copy(), up.copy())
        x, info2 = lapack.dgttrs(dl, d, du, du2, ipiv, b.copy())
        out[f"s{i}_lo"], out[f"s{i}_di"], out[f"s{i}_up"], out[f"s{i}_b"] = lo, di, up, b
        out[f"s{i}_dl"], out[f"s{i}_d"], out[f"s{i}_du"], out[f"s{i}_du2"] = dl, d, du, du2
        out[f"s{i}_ipiv"] = ipiv.astype(np.int32)  # 1-based, as LAPACK returns it
        out[f"s{i}_x"] = x
        out[f"s{i}_info"] = np.array([info, info2])
    out["count"] = np.array([len(specs)])
    return out


HIST_STEPS = {"viv_cylinder_384x256": 2000, "galloping_rectangle_1024x768": 5000}
HIST_STRIDE = 4


def long_history(name: str, threads: int = 0) -> None:
    """Oracle history of a benched case over its full step count."""
    c = cases.WORKLOADS[name]()
    root = tempfile.mkdtemp(prefix="golden_")
    path = c.write(os.path.join(root, c.name))
    o = oracle.Oracle(oracle.parse_deck(path), threads=threads)
    o.add_v_perturbation(c.v_perturbation())
    steps = HIST_STEPS[name]
    forces = np.zeros((steps, 8))
    rigid = np.zeros((steps, 18))
    for ns in range(steps):
        st = o.step(ns)
        assert st == 0, (ns, st)
        forces[ns] = o.a("forces")
        rigid[ns] = o.a("rigid")
        if ns % 250 == 0:
            print(name, ns, flush=True)
    sub = np.s_[::HIST_STRIDE, ::HIST_STRIDE]
    np.savez_compressed(
        os.path.join(HERE, f"hist_{name}.npz"), forces=forces, rigid=rigid, steps=np.array([steps]),
        stride=np.array([HIST_STRIDE]), q2=o.field("q2", 0, o.n3)[sub].copy(),
        q3=o.field("q3", 0, o.n3)[sub].copy(), pr=o.field("pr", 0, o.n3)[sub].copy())


def main() -> None:
    if len(sys.argv) in (3, 4) and sys.argv[1] == "--hist":
        long_history(sys.argv[2], threads=int(sys.argv[3]) if len(sys.argv) == 4 else 0)
        return
    np.savez_compressed(os.path.join(HERE, "lapack_gtt.npz"), **lapack_systems())
    root = tempfile.mkdtemp(prefix="golden_")
    c = cases.tiny_cylinder()
    path = c.write(os.path.join(root, c.name))
    d = oracle.parse_deck(path)
    o = oracle.Oracle(d)
    wr, zmm, zmmt = o.eigen
    np.savez_compressed(os.path.join(HERE, "phini_tiny.npz"), wr=wr, zmm=zmm, zmmt=zmmt,
                        amphk=o.a("amphk"), acphk=o.a("acphk"), apphk=o.a("apphk"))
    for mk in (cases.tiny_cylinder, cases.tiny_rectangle):
        c = mk()
        path = c.write(os.path.join(root, c.name))
        o = oracle.Oracle(oracle.parse_deck(path), threads=1)
        o.add_v_perturbation(c.v_perturbation())
        forces, rigid = [], []
        for ns in range(TRAJ_STEPS):
            st = o.step(ns)
            assert st == 0, st
            forces.append(o.a("forces").copy())
            rigid.append(o.a("rigid").copy())
        np.savez_compressed(
            os.path.join(HERE, f"traj_{c.name}.npz"), forces=np.array(forces), rigid=np.array(rigid),
            q2=o.field("q2", 0, o.n3).copy(), q3=o.field("q3", 0, o.n3).copy(),
            pr=o.field("pr", 0, o.n3).copy(), lmcc=o.a("lmcc").copy(), steps=np.array([TRAJ_STEPS]),
            eig_wr=o.eigen[0], eig_zmm=o.eigen[1], eig_zmmt=o.eigen[2])
    print("written to", HERE)


if __name__ == "__main__":
    main()
