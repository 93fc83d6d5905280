"""Helpers shared by the parity tests: one case on the oracle and on the GPU
with identical inputs (same deck, same eigen data, same noise)."""
from __future__ import annotations

import os
import tempfile

import numpy as np

import oracle
import fribois2d_b200 as fb
from fribois2d_b200 import case as cases

FIELDS = ("q2", "q3", "pr", "dph", "rhs2", "rhs3", "ru2", "ru3")


def rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-300)
    return float(np.max(np.abs(a - b))) / scale if a.size else 0.0


def deck_dir(c: cases.Case, root: str = None) -> str:
    root = root or tempfile.mkdtemp(prefix="fbdeck_")
    path = os.path.join(root, c.name)
    c.write(path)
    return path


class Pair:
    """The same case on the oracle and on the device."""

    def __init__(self, c: cases.Case = None, root: str = None, gpu: bool = True, threads: int = 0,
                 deck: str = None):
        """A generated case `c` (written under `root`, seeded v noise added
        to both sides) or an existing deck directory `deck` (taken as is)."""
        self.case = c
        self.dir = deck if deck else deck_dir(c, root)
        self.host = fb.HostSetup(self.dir)
        eig = (self.host.array("wr"), self.host.array("zmm"), self.host.array("zmmt"))
        self.o = oracle.Oracle(oracle.parse_deck(self.dir), eigen=eig, threads=threads)
        pert = c.v_perturbation() if c is not None else None
        if pert is not None:
            self.o.add_v_perturbation(pert)
        self.s = None
        if gpu:
            self.s = fb.Solver(self.dir)
            if pert is not None:
                q2 = self.s.get("q2")
                q2[1:c.n3m + 1] += pert
                self.s.set("q2", q2)
        self.n2, self.n3 = self.o.n2, self.o.n3
        self.n2m, self.n3m = self.n2 - 1, self.n3 - 1

    # oracle views in the device layout (rows k = 0..n3, columns j-1)
    def of(self, name: str) -> np.ndarray:
        return self.o.field(name, 0, self.n3)

    def ob(self, name: str) -> np.ndarray:
        return self.o.a(name)[1:self.n2 + 1]

    def sync_to_gpu(self) -> None:
        """Copy the oracle state into the device so a stage sees equal inputs."""
        for f in FIELDS:
            self.s.set(f, self.of(f))
        for b in fb.BOUNDARY:
            self.s.set(b, self.ob(b))
        for m in ("lmcc", "lmvel", "lmacc", "lmnor", "vert", "rigid"):
            self.s.set(m, self.o.a(m))
