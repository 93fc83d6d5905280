"""The learned initial guess of the strong coupling iteration.

Training data come from the solver itself: a seeded sweep of VIV cylinder
cases advanced together (one coupled batch: the fluid solves of every case
in grouped launches, the iteration on the device) with strong coupling and
the plain (extrapolating) predictor.  Every converged step yields 27
features -- for the free coordinate's displacement, velocity and load, the
second differences of the last 8 converged values divided by their root
mean square (the shape of the recent curvature), then Re, mass ratio and
reduced velocity -- and 2 targets: the corrections that the step's
displacement and load needed on top of their linear extrapolations, in units
of that root mean square, less a structured prior (the curvature
extrapolated linearly, i.e. a cubic extrapolation of the history, switched
off in windows where one value dominates).  The perceptron learns that
residual; it is trained and evaluated by the library's own CUDA kernels
(fribois2d_b200.MLP).  The coupling adds prior + residual to the linear
extrapolation of the load as its initial guess and keeps its convergence
test unchanged; without a network set, the learned mode uses the prior
alone.
"""
from __future__ import annotations

import os
import tempfile
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from . import COUPLING_LEARNED, COUPLING_STRONG, MLP, Batch, Solver
from . import case as cases


def sweep(n: int, seed: int = 0, n3m: int = 48, n2m: int = 32, h: float = 1.0 / 8, nlm: int = 40,
          dt: float = 5e-3) -> List[cases.Case]:
    """Small VIV cases: Re uniform in [60, 200], mass ratio log-uniform in
    [2, 20], reduced velocity uniform in [2, 12] (one draw per case)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        re = float(rng.uniform(60.0, 200.0))
        mr = float(np.exp(rng.uniform(np.log(2.0), np.log(20.0))))
        ur = float(rng.uniform(2.0, 12.0))
        c = cases.viv_cylinder(n3m=n3m, n2m=n2m, h=h, zwin=(-1.0, 2.0), ywin=(-1.0, 1.0), zdom=(-3.0, 9.0),
                               ydom=(-3.0, 3.0), nlm=nlm, re=re, mass_ratio=mr, u_red=ur, dt=dt,
                               name=f"viv_sweep_{seed}_{i:03d}")
        out.append(c)
    return out


def _open(c: cases.Case, root: str, device: int = 0) -> Solver:
    s = Solver(c.write(os.path.join(root, c.name)), device=device)
    q2 = s.get("q2")
    q2[1:c.n3m + 1] += c.v_perturbation()
    s.set("q2", q2)
    return s


def generate(case_list: Sequence[cases.Case], steps: int, tol: float = 1e-8, device: int = 0,
             chunk: int = 4096) -> Tuple[np.ndarray, np.ndarray, float]:
    """(features, targets, mean fluid solves per step) of strongly coupled
    runs with the plain predictor, all cases advanced as one batch."""
    root = tempfile.mkdtemp(prefix="fbsweep_")
    solvers = [_open(c, root, device) for c in case_list]
    for s in solvers:
        s.set_coupling(COUPLING_STRONG, tol)
    b = Batch(solvers)
    xs, ts = [], []
    done = 0
    while done < steps:   # the samples of every case drained before its ring fills
        k = min(chunk, steps - done)
        b.advance(k)
        for s in solvers:
            x, t = s.coupling_samples()
            xs.append(x)
            ts.append(t)
        done += k
    b.close()
    solves = nsteps = 0.0
    for s in solvers:
        st = s.coupling_stats()
        solves += st["solves"]
        nsteps += st["steps"]
        s.close()
    return np.concatenate(xs), np.concatenate(ts), solves / max(nsteps, 1.0)


def standardise(x: np.ndarray, t: np.ndarray) -> np.ndarray:
    """norm = (x mean[27], x std[27], t mean[2], t std[2]); constant
    features (std 0) keep a unit scale."""
    xm, xsd = x.mean(0), x.std(0)
    tm, tsd = t.mean(0), t.std(0)
    xsd = np.where(xsd > 0, xsd, 1.0)
    tsd = np.where(tsd > 0, tsd, 1.0)
    return np.concatenate([xm, xsd, tm, tsd]).astype(np.float32)


def apply_norm(norm: np.ndarray, x: np.ndarray, t: np.ndarray = None):
    ni = x.shape[1]
    xn = (x - norm[:ni]) / norm[ni:2 * ni]
    if t is None:
        return xn.astype(np.float32)
    no = t.shape[1]
    tn = (t - norm[2 * ni:2 * ni + no]) / norm[2 * ni + no:2 * ni + 2 * no]
    return xn.astype(np.float32), tn.astype(np.float32)


@dataclass
class Predictor:
    mlp: MLP
    norm: np.ndarray
    final_loss: float


# The network's residual, in units of the history's scale, is trained and
# applied within this bound (couple.cu clamps to the same value): on smooth
# steps the prior's residual is ~1e-3 of that scale, and beyond a few
# hundredths it is a jump of the loads that no smooth history predicts.
RESIDUAL_BOUND = 0.02


def predictable(t: np.ndarray, bound: float = RESIDUAL_BOUND) -> np.ndarray:
    """Samples whose targets (the prior's residuals, in units of the history's
    scale) are within `bound`: the steps a smooth history can predict.  The
    rest -- jumps of the loads as markers cross grid lines -- are left out of
    training, and the device clamps the network's residual to the same bound."""
    return np.all(np.abs(t) <= bound, axis=1)


def train(x: np.ndarray, t: np.ndarray, epochs: int = 300, batch: int = 128, lr: float = 2e-3, seed: int = 0,
          device: int = 0) -> Predictor:
    keep = predictable(t)
    x, t = x[keep], t[keep]
    norm = standardise(x, t)
    xn, tn = apply_norm(norm, x, t)
    m = MLP(x.shape[1], t.shape[1], seed=seed, device=device)
    loss = m.train(xn, tn, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return Predictor(m, norm, loss)


def mean_solves(c: cases.Case, steps: int, predictor=None, tol: float = 1e-8, device: int = 0,
                skip: int = 0) -> Tuple[float, np.ndarray, float]:
    """Mean fluid solves per step of a strongly coupled run over the steps
    after the first `skip`, its history rows and the mean relative load
    residual of the initial guesses (over all steps).  predictor: None (the
    plain predictor), "prior" (the learned mode's structured prior without a
    network) or a trained Predictor."""
    root = tempfile.mkdtemp(prefix="fbeval_")
    s = _open(c, root, device)
    if predictor is None:
        s.set_coupling(COUPLING_STRONG, tol)
    else:
        s.set_coupling(COUPLING_LEARNED, tol)
        if predictor != "prior":
            s.set_predictor(predictor.mlp, predictor.norm)
    h = s.advance(0, steps)
    st = s.coupling_stats()
    s.close()
    col = h[skip:, 30]
    return float(col.mean()), h, st["initial_residual"]
