"""Run a GSvit parameter file on the B200 library and write GSvit's text
outputs (point logs, far-field logs):

    python -m gsvit_copy_b200.run deck.par [--outdir DIR] [--device N] [--steps N]
                                           [--killer FILE [--check-every N]]

The keyword subset and the output formats are those of
gsvit_copy_b200.parfile.  Steps default to the deck's COMP value.  With
--killer, the run stops cleanly once FILE holds the integer 1, as GSvit's
`--killer` does (svit.c:91-107, 159-181, 260-264), and writes its outputs for
the steps done."""
from __future__ import annotations

import argparse
import os
import re
import sys

from .parfile import load_par, write_outputs
from .solver import Solver


def killer_says_stop(path) -> bool:
    """GSvit's killcheck (svit.c:91-107): the file exists and its first
    whitespace-separated token reads as the integer 1."""
    if not path or not os.path.exists(path):
        return False
    try:
        with open(path) as fh:
            text = fh.read(64)
    except OSError:
        return False
    m = re.match(r"\s*([+-]?\d+)", text)
    return bool(m) and int(m.group(1)) == 1


def run_steps(step, nsteps: int, killer=None, check_every: int = 1) -> int:
    """Advance nsteps through step(k).  With a killer file, look at it after
    every `check_every` steps (GSvit: after every step) and stop when it says 1.
    Returns the number of steps done."""
    if not killer:
        step(nsteps)
        return nsteps
    done = 0
    every = max(1, int(check_every))
    while done < nsteps:
        k = min(every, nsteps - done)
        step(k)
        done += k
        if killer_says_stop(killer):
            break
    return done


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("par")
    ap.add_argument("--outdir", default=None, help="where the logs go (default: the deck's directory)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--killer", default=None, help="external shutdown file: the run stops once it holds 1")
    ap.add_argument("--check-every", type=int, default=1, help="steps between looks at the killer file")
    a = ap.parse_args(argv)
    run = load_par(a.par)
    n = run.scene.nsteps if a.steps is None else a.steps
    with Solver(run.scene, device=a.device) as s:
        done = run_steps(s.step, n, a.killer, a.check_every)
        probes = s.probes() if len(run.points) else None
        series = s.nfff_series() if run.scene.nfff else None
    if done < n:
        print(f"GSvit forced to quit by external file after {done} steps", file=sys.stderr)
    files = write_outputs(run, probes, series, done, a.outdir or run.base)
    for f in files:
        print(f)
    return 0


if __name__ == "__main__":
    sys.exit(main())
