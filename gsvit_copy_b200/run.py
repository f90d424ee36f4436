"""Run a GSvit parameter file on the B200 library and write GSvit's text
outputs (point logs, far-field logs):

    python -m gsvit_copy_b200.run deck.par [--outdir DIR] [--device N] [--steps N]

The keyword subset and the output formats are those of
gsvit_copy_b200.parfile.  Steps default to the deck's COMP value."""
from __future__ import annotations

import argparse
import os
import sys

from .parfile import load_par, write_outputs
from .solver import Solver


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("par")
    ap.add_argument("--outdir", default=None, help="where the logs go (default: the deck's directory)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--steps", type=int, default=None)
    a = ap.parse_args(argv)
    run = load_par(a.par)
    n = run.scene.nsteps if a.steps is None else a.steps
    with Solver(run.scene, device=a.device) as s:
        s.step(n)
        probes = s.probes() if len(run.points) else None
        series = s.nfff_series() if run.scene.nfff else None
    files = write_outputs(run, probes, series, n, a.outdir or run.base)
    for f in files:
        print(f)
    return 0


if __name__ == "__main__":
    sys.exit(main())
