"""Time one stage (or kernel) of the fluid step on a named workload.

    python -m fribois2d_b200.stagetime WORKLOAD STAGE [POISSON] [REPS] [--no-tune]

WORKLOAD is one of the benchmark cases (``case.WORKLOADS``), STAGE a name of
``fribois2d_b200.STAGES`` (``helsolve``, ``i8x8_gemm``, ``poisson_tri`` ...) or
``step`` (full time steps), POISSON ``int8x8`` (default), ``fp64`` or
``tf32x3``.  The case is set up, autotuned (unless ``--no-tune``: the
library's default tiles, and no tuning launches before the stage's own) and
advanced two steps; then the
stage runs once as a warm-up and REPS times (default 2) from a captured
graph, and its mean device time is printed; with ``step``, REPS steps run
from the step's captured graph and the time per step and the kernel launches
per step are printed (the last REPS x launches of a profiler's launch list
are those steps).  Few launches precede the timed ones, which makes this the
driver for kernel captures with a profiler.
"""
from __future__ import annotations

import os
import sys
import tempfile

from . import POISSON_FP64, POISSON_INT8X8, POISSON_TF32X3, Solver
from . import case as cases

FORMS = {"int8x8": POISSON_INT8X8, "fp64": POISSON_FP64, "tf32x3": POISSON_TF32X3}


def main(argv) -> int:
    tune = "--no-tune" not in argv
    argv = [a for a in argv if a != "--no-tune"]
    if len(argv) < 2:
        print(__doc__)
        return 2
    name, stage = argv[0], argv[1]
    form = argv[2] if len(argv) > 2 else "int8x8"
    reps = int(argv[3]) if len(argv) > 3 else 2
    c = cases.WORKLOADS[name]()
    s = Solver(c.write(os.path.join(tempfile.mkdtemp(prefix="fbstage_"), c.name)))
    s.set_poisson(FORMS[form])
    tiles = s.autotune() if tune else "library defaults"
    q2 = s.get("q2")
    q2[1:c.n3m + 1] += c.v_perturbation()
    s.set("q2", q2)
    s.advance(0, 2, history=False)
    if stage == "step":
        s.advance(2, reps, history=False)
        print(f"{name} step: {s.last_advance_ms() * 1e3 / reps:.1f} us per step over {reps} steps, "
              f"{s.kernel_count()} kernel launches per step (tiles {tiles})")
    else:
        s.set_substep(2, 1)
        ms = s.time_stage(stage, 1, reps=reps)
        print(f"{name} {stage}: {ms * 1e3:.2f} us per launch (tiles {tiles})")
    s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
