"""Input decks in FRiBoIS2D's ``input_FSI`` format, and the synthetic cases.

A deck is the directory the reference reads at start-up:

* ``global_par.in``  -- parsed by ``read_genin``      (src/utils_proc.F90:45-129)
* ``fluid_par.in``   -- parsed by ``read_fluid_in``   (src/utils_proc.F90:135-222)
* ``rigid_par.in``   -- parsed by ``read_input_par_RBM`` (src/utils_proc.F90:2-39)
* ``ycoord.dat`` / ``zcoord.dat`` -- node coordinates, one per record,
  read when ``istr2 = istr3 = 100`` (src/cordin.F90:243-278)
* ``lmdata.in``      -- closed polygon, ``nlm + 1`` vertices ``y z`` per
  record (src/utils_proc.F90:519-578)

The record layout written here follows the reference's decks line for line
(positional list-directed reads: header and blank records are skipped by
position, so they must be present).

The grid generator restates the cubic stretching of the reference's
pre-processor (preproc/cubicstr.m:1-37): a uniform window of spacing ``h``
around the body and ``x(s) = B s + A s^3`` outside it, with ``B = h n`` so
that the first stretched cell continues the window spacing.  The marker
generators follow preproc/MAIN_input_OscCyl1DOF.m:93-101 (vertices on the
body outline, markers at segment midpoints are derived by the solver).
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Optional, Tuple

import numpy as np


@dataclasses.dataclass
class DeckParams:
    """Every value the three ``*_par.in`` files carry.

    Field names are the reference's variable names (src/declarations.F90).
    """

    # global_par.in
    dt: float = 1.0e-3
    idtv: bool = True          # True: fixed dt, check CFL only
    dtmax: float = 5.0e-3
    cflmax: float = 0.2
    cfllim: float = 2.0
    outfol: str = "out"
    irest: bool = False
    trestart: float = 50.0
    ibact: bool = True
    kprobe: float = 1.0
    prlgr: bool = False
    tprtag: float = 0.5
    forst: int = 1
    radiusSD: float = 1.6
    wfun: int = 1
    # fluid_par.in
    alx3: float = 40.0
    rext2: float = 60.0
    n3: int = 0
    n2: int = 0
    nsst: int = 3
    nwrit: bool = False
    tframef: float = 0.2
    resid: float = 1.0e-7
    cou: float = 0.8
    visc: float = 0.01
    inslws: bool = False
    inslwn: bool = False
    q3uw: float = 0.0
    q3lw: float = 0.0
    # rigid_par.in
    cbody: bool = True
    cmposi: Tuple[float, float] = (30.0, 15.0)
    cmroti: float = 0.0
    ipert: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rbgravF: Tuple[float, float] = (0.0, 0.0)
    rbden: float = 10.0
    rba: Tuple[float, float] = (math.pi / 4.0, math.pi / 32.0)
    rbmcon: Tuple[int, int, int] = (0, 1, 1)
    kk: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    kk3: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    cc: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rtcoup: bool = False
    rrr: float = 0.4


def _fl(v: bool) -> str:
    return ".true." if v else ".false."


def _num(v: float) -> str:
    return repr(float(v))


def write_deck(path: str, p: DeckParams, ycoord: np.ndarray, zcoord: np.ndarray,
               vert: Optional[np.ndarray]) -> None:
    """Write a complete ``input_FSI`` directory.

    ``vert`` is ``(nlm+1, 2)`` with columns ``(y, z)``; the last vertex closes
    the polygon.  ``ycoord``/``zcoord`` hold ``n2``/``n3`` node coordinates.
    """
    os.makedirs(path, exist_ok=True)
    assert len(ycoord) == p.n2 and len(zcoord) == p.n3
    g = [
        "###################### COMMON SETTINGS",
        f"{_num(p.dt)}      # time-step size                       (dt)",
        f"{_fl(p.idtv)}      # fixed time-step size                 (idtv)",
        f"{_num(p.dtmax)}      # largest time-step size for variable dt (dtmax)",
        f"{_num(p.cflmax)}      # maximum CFL for variable dt        (cflmax)",
        f"{_num(p.cfllim)}      # maximum CFL for stability          (cfllim)",
        f"{p.outfol}      # output folder filename                 (outfol)",
        f"{_fl(p.irest)}      # simulation restart                  (irest)",
        f"{_num(p.trestart)}      # restart interval                 (trestart)",
        "",
        "",
        "###################### FSI CASE",
        f"{_fl(p.ibact)}     # activate immersed boundary treatment  (ibact)",
        "",
        "",
        "###################### FORCING OPTIONS",
        f"{_num(p.kprobe)}         # scale factor for normal arrays   (kprobe)",
        f"{_fl(p.prlgr)}      # write quantities at Lagrangian markers (prlgr)",
        f"{_num(p.tprtag)}      # time interval for prlgr             (tprtag)",
        f"{int(p.forst)}           # iterative forcing steps           (forst)",
        f"{_num(p.radiusSD)}         # support domain radius         (radiusSD)",
        f"{int(p.wfun)}           # MLS weighting function           (wfun)",
        "",
        "",
    ]
    f = [
        "###################### DOMAIN AND GRID",
        f"{_num(p.alx3)}       # domain length in Z-dir              (alx3)",
        f"{_num(p.rext2)}       # domain length in Y-dir             (rext2)",
        f"{int(p.n3)}, {int(p.n2)} # grid resolution in Z, Y          (n3,n2)",
        "100           # bunching law in Z direction (read grid)    (istr3)",
        "8.0,8.0,100,90,101    # options for istr3=3 (unused)",
        "6.0,9.0     # uniform region for istr3=3 (unused)           (int3)",
        "100           # bunching law in Y direction (read grid)    (istr2)",
        "3.0,3.0,100,60,101  # options for istr2=3 (unused)",
        "2.0,4.0     # uniform region for istr2=3 (unused)           (int2)",
        "",
        "",
        "###################### SIMULATION SETTING",
        f"{int(p.nsst)}           # time-stepping scheme               (nsst)",
        f"{_fl(p.nwrit)}      # write fluid solution to file          (nwrit)",
        f"{_num(p.tframef)}      # interval for writing the solution  (tframef)",
        f"{_num(p.resid)}     # maximum local divergence              (resid)",
        f"{_num(p.cou)}         # Courant number for outflow wave eqn  (cou)",
        "",
        "",
        "###################### BOUNDARY CONDITIONS AND DIM.LESS PARAMETERS",
        f"{_num(p.visc)}        # inverse of the Reynolds number      (visc)",
        f"{_fl(p.inslws)}      # no-slip condition on the bottom wall (inslws)",
        f"{_fl(p.inslwn)}      # no-slip condition on the top wall    (inslwn)",
        f"{_num(p.q3uw)}         # Z velocity on upper wall            (q3uw)",
        f"{_num(p.q3lw)}         # Z velocity on lower wall            (q3lw)",
        "",
    ]
    r = [
        "#################################### RIGID BODY PARAMETERS",
        f"{_fl(p.cbody)}    # closed body                             (cbody)",
        f"{_num(p.cmposi[0])}, {_num(p.cmposi[1])}      # initial CM [y,z] (cmposi)",
        f"{_num(p.cmroti)}            # initial CM angle              (cmroti)",
        ",".join(_num(v) for v in p.ipert) + "  # initial velocity perturbation (ipert)",
        ",".join(_num(v) for v in p.rbgravF) + "  # gravity force components   (rbgravF)",
        f"{_num(p.rbden)}            # body relative density           (rbden)",
        ",".join(_num(v) for v in p.rba) + "  # area and moment of area       (rba)",
        ",".join(str(int(v)) for v in p.rbmcon) + "  # constraint array        (rbmcon)",
        ",".join(_num(v) for v in p.kk) + "  # stiffness (y,z,a)",
        ",".join(_num(v) for v in p.kk3) + "  # cubic stiffness (y,z,a)",
        ",".join(_num(v) for v in p.cc) + "  # damping (y,z,a)",
        f"{_fl(p.rtcoup)}           # translation-rotation coupling",
        f"{_num(p.rrr)}             # rt ratio                        (rrr)",
        "",
    ]
    for name, lines in (("global_par.in", g), ("fluid_par.in", f), ("rigid_par.in", r)):
        with open(os.path.join(path, name), "w") as fh:
            fh.write("\n".join(lines) + "\n")
    for name, arr in (("ycoord.dat", ycoord), ("zcoord.dat", zcoord)):
        with open(os.path.join(path, name), "w") as fh:
            fh.write("\n".join(f"{float(v):.17g} " for v in arr))
    if vert is not None:
        with open(os.path.join(path, "lmdata.in"), "w") as fh:
            # one record per vertex, newline-terminated: the reader counts
            # markers as newlines - 1 (src/utils_proc.F90:529-535)
            fh.write("".join(f"{float(a):.17g} \t{float(b):.17g} \t\n" for a, b in vert))


# --------------------------------------------------------------------------
# grids

def _cubic_side(length: float, n: int, h: float) -> np.ndarray:
    """Offsets of ``n+1`` nodes covering ``[0, length]`` starting at spacing h.

    ``x(s) = B s + A s^3`` with ``B = h n`` and ``A = length - B``
    (preproc/cubicstr.m:12-20).
    """
    B = h * n
    A = length - B
    if A < 0.0:
        raise ValueError("stretched region too short for its cell count")
    s = np.arange(n + 1, dtype=np.float64) / n
    x = B * s + A * s ** 3
    x[-1] = length
    return x


def stretched_axis(length: float, n_cells: int, lo: float, hi: float, h: float) -> np.ndarray:
    """Node coordinates on ``[0, length]``: uniform spacing ``h`` on ``[lo, hi]``.

    The cells left over by the window are split between the two stretched
    sides so that their outermost spacings are as close as possible.
    """
    nu = int(round((hi - lo) / h))
    if abs(nu * h - (hi - lo)) > 1e-9 * max(1.0, hi - lo):
        raise ValueError("window is not a whole number of cells")
    rest = n_cells - nu
    if rest < 2:
        raise ValueError("no cells left for the stretched regions")
    dl, dr = lo, length - hi
    best = None
    for nl in range(1, rest):
        nr = rest - nl
        if dl - h * nl < 0 or dr - h * nr < 0:
            continue
        el = h + 3.0 * (dl - h * nl) / nl
        er = h + 3.0 * (dr - h * nr) / nr
        score = max(el, er) / min(el, er)
        if best is None or score < best[0]:
            best = (score, nl, nr)
    if best is None:
        raise ValueError("cannot stretch: too many cells for the outer regions")
    _, nl, nr = best
    left = lo - _cubic_side(dl, nl, h)[::-1]
    mid = lo + h * np.arange(nu + 1, dtype=np.float64)
    right = hi + _cubic_side(dr, nr, h)
    x = np.concatenate([left[:-1], mid, right[1:]])
    x[0] = 0.0
    x[-1] = length
    assert len(x) == n_cells + 1 and np.all(np.diff(x) > 0)
    return x


def uniform_axis(length: float, n_cells: int) -> np.ndarray:
    return np.linspace(0.0, length, n_cells + 1)


# --------------------------------------------------------------------------
# bodies

def circle_vertices(yc: float, zc: float, radius: float, nlm: int) -> np.ndarray:
    """``nlm+1`` vertices ``(y, z)``, counter-clockwise in the (z, y) plane,
    last vertex repeating the first (preproc/MAIN_input_OscCyl1DOF.m:95-97)."""
    th = np.linspace(0.0, 2.0 * np.pi, nlm + 1)
    z = radius * np.cos(th) + zc
    y = radius * np.sin(th) + yc
    v = np.stack([y, z], axis=1)
    v[-1] = v[0]
    return v


def rectangle_vertices(yc: float, zc: float, len_z: float, len_y: float, nlm: int,
                       cluster: float = 0.6) -> np.ndarray:
    """Rectangle outline with markers clustered towards the corners.

    Each side gets markers in proportion to its length; along a side the
    parameter ``u`` maps to ``u - c sin(2 pi u)/(2 pi)``, which is densest at
    both ends.  Counter-clockwise in the (z, y) plane starting at the
    downstream-bottom corner, closed.
    """
    sides = [len_y, len_z, len_y, len_z]
    per = sum(sides)
    counts = [max(2, int(round(nlm * s / per))) for s in sides]
    counts[1] += nlm - sum(counts)
    z0, z1 = zc - len_z / 2, zc + len_z / 2
    y0, y1 = yc - len_y / 2, yc + len_y / 2
    corners = [(z1, y0), (z1, y1), (z0, y1), (z0, y0), (z1, y0)]
    pts = []
    for s in range(4):
        n = counts[s]
        u = np.arange(n, dtype=np.float64) / n
        t = u - cluster * np.sin(2 * np.pi * u) / (2 * np.pi)
        za, ya = corners[s]
        zb, yb = corners[s + 1]
        for tt in t:
            pts.append((ya + (yb - ya) * tt, za + (zb - za) * tt))
    pts.append(pts[0])
    v = np.array(pts, dtype=np.float64)
    assert len(v) == nlm + 1
    return v


# --------------------------------------------------------------------------
# synthetic cases

@dataclasses.dataclass
class Case:
    name: str
    params: DeckParams
    ycoord: np.ndarray
    zcoord: np.ndarray
    vert: np.ndarray
    v_noise: float = 0.0          # std of the Gaussian noise added to v
    noise_seed: int = 0
    steps: int = 1

    @property
    def n2m(self) -> int:
        return self.params.n2 - 1

    @property
    def n3m(self) -> int:
        return self.params.n3 - 1

    @property
    def cells(self) -> int:
        return self.n2m * self.n3m

    @property
    def nlm(self) -> int:
        return len(self.vert) - 1

    def write(self, path: str) -> str:
        write_deck(path, self.params, self.ycoord, self.zcoord, self.vert)
        return path

    def v_perturbation(self) -> np.ndarray:
        """Noise for v on the interior v-points, shape ``(n3m, n2)`` (k, j).

        Drawn once from ``numpy.random.default_rng(seed)`` over
        ``j = 2..n2m`` (fastest) and ``k = 1..n3m``, i.e. Fortran column
        order of ``q2(j, k)``; the wall rows ``j = 1, n2`` stay zero.
        """
        n2, n3m = self.params.n2, self.n3m
        out = np.zeros((n3m, n2), dtype=np.float64)
        if self.v_noise > 0.0:
            rng = np.random.default_rng(self.noise_seed)
            out[:, 1:n2 - 1] = self.v_noise * rng.standard_normal((n3m, n2 - 2))
        return out


def viv_cylinder(n3m: int = 384, n2m: int = 256, h: float = 1.0 / 48,
                 zwin=(-1.5, 4.5), ywin=(-2.0, 2.0), zdom=(-10.0, 30.0),
                 ydom=(-15.0, 15.0), nlm: int = 302, re: float = 100.0,
                 mass_ratio: float = 10.0, u_red: float = 5.0, dt: float = 2e-3,
                 steps: int = 2000, noise: float = 1e-3, name: str = "viv_cylinder") -> Case:
    """Elastically mounted circular cylinder (D = 1), transverse 1-DOF.

    Coordinates are shifted so that the domain starts at 0, as the reference
    requires (src/lgrdistribution.F90:32-36, src/updvp.F90:127).
    """
    L3 = zdom[1] - zdom[0]
    L2 = ydom[1] - ydom[0]
    zc, yc = -zdom[0], -ydom[0]
    z = stretched_axis(L3, n3m, zwin[0] + zc, zwin[1] + zc, h)
    y = stretched_axis(L2, n2m, ywin[0] + yc, ywin[1] + yc, h)
    area = math.pi / 4.0
    ky = mass_ratio * area * (2.0 * math.pi / u_red) ** 2
    p = DeckParams(dt=dt, idtv=True, alx3=L3, rext2=L2, n3=n3m + 1, n2=n2m + 1,
                   visc=1.0 / re, cmposi=(yc, zc), cmroti=0.0, rbden=mass_ratio,
                   rba=(area, math.pi / 32.0), rbmcon=(0, 1, 1), kk=(ky, 0.0, 0.0))
    return Case(name, p, y, z, circle_vertices(yc, zc, 0.5, nlm), v_noise=noise,
                noise_seed=0, steps=steps)


def galloping_rectangle(n3m: int = 1024, n2m: int = 768, h: float = 1.0 / 96,
                        zwin=(-2.5, 6.5), ywin=(-3.0, 3.0), zdom=(-12.0, 40.0),
                        ydom=(-20.0, 20.0), side_ratio: float = 4.0, nlm: int = 1200,
                        re: float = 200.0, inertia_ratio: float = 50.0,
                        u_red: float = 8.0, pitch_deg: float = 2.0, dt: float = 1e-3,
                        steps: int = 5000, name: str = "galloping_rectangle") -> Case:
    """Rectangle of thickness D = 1 and length ``side_ratio``, pitch-only.

    The inertia ratio is the body's moment of inertia about its centroid in
    units of rho_f D^4, ``rbden * rba(2)``; the torsional spring follows from
    the reduced velocity, ``k_a = I (2 pi / U_r)^2``.
    """
    L3 = zdom[1] - zdom[0]
    L2 = ydom[1] - ydom[0]
    zc, yc = -zdom[0], -ydom[0]
    z = stretched_axis(L3, n3m, zwin[0] + zc, zwin[1] + zc, h)
    y = stretched_axis(L2, n2m, ywin[0] + yc, ywin[1] + yc, h)
    area = side_ratio * 1.0
    jj = area * (side_ratio ** 2 + 1.0) / 12.0
    rbden = inertia_ratio / jj
    ka = inertia_ratio * (2.0 * math.pi / u_red) ** 2
    p = DeckParams(dt=dt, idtv=True, alx3=L3, rext2=L2, n3=n3m + 1, n2=n2m + 1,
                   visc=1.0 / re, cmposi=(yc, zc), cmroti=math.radians(pitch_deg),
                   rbden=rbden, rba=(area, jj), rbmcon=(1, 1, 0), kk=(0.0, 0.0, ka))
    return Case(name, p, y, z, rectangle_vertices(yc, zc, side_ratio, 1.0, nlm),
                v_noise=0.0, steps=steps)


def viv_cylinder_384x256() -> Case:
    """VIV cylinder, 384 (z) x 256 (y) cells, h = D/48, 302 markers."""
    return viv_cylinder(name="viv_cylinder_384x256")


def galloping_rectangle_1024x768() -> Case:
    """Rotational galloping rectangle, 1024 (z) x 768 (y) cells, h = D/96."""
    return galloping_rectangle(name="galloping_rectangle_1024x768")


def viv_cylinder_2048x1536() -> Case:
    """VIV cylinder, 2048 (z) x 1536 (y) cells, h = D/192, 604 markers, Re 200."""
    return viv_cylinder(n3m=2048, n2m=1536, h=1.0 / 192, zwin=(-2.0, 6.0), ywin=(-3.0, 3.0),
                        nlm=604, re=200.0, name="viv_cylinder_2048x1536")


def tiny_cylinder(n3m: int = 48, n2m: int = 32, h: float = 1.0 / 8, nlm: int = 40,
                  noise: float = 1e-3, dt: float = 5e-3) -> Case:
    """Small VIV case for fast parity tests (same physics, coarse grid)."""
    return viv_cylinder(n3m=n3m, n2m=n2m, h=h, zwin=(-1.0, 2.0), ywin=(-1.0, 1.0),
                        zdom=(-3.0, 9.0), ydom=(-3.0, 3.0), nlm=nlm, dt=dt, steps=10,
                        noise=noise, name=f"tiny_cylinder_{n3m}x{n2m}")


def tiny_rectangle(n3m: int = 64, n2m: int = 40, h: float = 1.0 / 8, nlm: int = 60,
                   dt: float = 5e-3) -> Case:
    """Small pitching rectangle (side ratio 2) for fast parity tests."""
    return galloping_rectangle(n3m=n3m, n2m=n2m, h=h, zwin=(-1.5, 2.5), ywin=(-1.0, 1.0),
                               zdom=(-4.0, 10.0), ydom=(-3.0, 3.0), side_ratio=2.0,
                               nlm=nlm, re=200.0, dt=dt, steps=10, pitch_deg=5.0,
                               name=f"tiny_rectangle_{n3m}x{n2m}")


# grid sizes (z cells, y cells) of the batched VIV workload with their
# uniform spacing: two markers per spacing on the circle, CFL ~ 0.1 at U = 1
BATCH_GRIDS = ((256, 192, 1.0 / 24), (384, 256, 1.0 / 32), (512, 384, 1.0 / 48), (768, 512, 1.0 / 64))


def viv_batch(n: int = 256, seed: int = 0, steps: int = 1000):
    """Independent VIV cylinder cases drawn by seed: grid size from
    BATCH_GRIDS, Re uniform in [60, 200], mass ratio log-uniform in [2, 20],
    reduced velocity uniform in [2, 12]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        n3m, n2m, h = BATCH_GRIDS[int(rng.integers(len(BATCH_GRIDS)))]
        re = float(rng.uniform(60.0, 200.0))
        mr = float(np.exp(rng.uniform(np.log(2.0), np.log(20.0))))
        ur = float(rng.uniform(2.0, 12.0))
        cz, cy = int(0.4 * n3m) // 10 * 10, int(0.4 * n2m) // 10 * 10   # window cells
        wz, wy = cz * h, cy * h
        z0 = -round(0.3 * cz) * h
        out.append(viv_cylinder(n3m=n3m, n2m=n2m, h=h, zwin=(z0, z0 + wz), ywin=(-0.5 * wy, 0.5 * wy),
                                nlm=int(round(2.0 * math.pi / h)), re=re, mass_ratio=mr, u_red=ur,
                                dt=0.1 * h, steps=steps, name=f"viv_batch_{i:03d}_{n3m}x{n2m}"))
    return out


WORKLOADS = {f.__name__: f for f in (viv_cylinder_384x256, galloping_rectangle_1024x768, viv_cylinder_2048x1536)}
