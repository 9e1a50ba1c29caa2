"""Device time of every kernel in the caps time step, by kernel.

Runs the bench workload (random PV of spectral peak k0 on an n^2 grid,
surgery every step, recontouring every nregmax regularisations) through the
C-ABI with the library's per-launch timer on (casl_kernel_times: a pair of
CUDA events around every launch, on the launch's own stream), and prints one
table for a block of regular steps and one for the step that recontours.
The event pairs add a few microseconds per launch, so the step time printed
here is above the bench's; use the tables for shares, the bench for speed.

    python -m hydra_b200.bench_step --n 1024 --steps 10 [--which 2]

With CASL_TRACE=1 the library also prints each recontouring's phases
(CUDA events between its stages).
"""
import argparse
import time

import torch

from hydra_b200.casl import CaslGPU
from hydra_b200.synthetic import random_pv


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--k0", type=float, default=16.0)
    ap.add_argument("--levels", type=int, default=80)
    ap.add_argument("--steps", type=int, default=10, help="regular steps in the first table")
    ap.add_argument("--nregmax", type=int, default=20)
    ap.add_argument("--which", type=int, default=1,
                    help="tabulate the step of this recontouring (1: step nregmax; each later "
                         "one nregmax - 1 steps on, the step after a recontouring regularising)")
    a = ap.parse_args(argv)
    g = CaslGPU(a.n, ncontq=a.levels, force_surgery=1, dtmax=0.05, nregmax=a.nregmax,
                npm=16_000_000, nm=1_000_000)
    g.initialise(random_pv(a.n, a.k0, 0))
    warm = 3
    g.step(warm)
    torch.cuda.synchronize()
    g.kernel_times(1)
    t = time.perf_counter()
    g.step(a.steps)
    torch.cuda.synchronize()
    ms = 1e3 * (time.perf_counter() - t) / a.steps
    print(f"# {a.steps} regular steps, {ms:.2f} ms/step with the per-launch timer on")
    print(g.kernel_times(2), end="")
    # up to the step before the chosen recontouring, then that step alone
    done = warm + a.steps
    target = a.nregmax + (a.which - 1) * (a.nregmax - 1)
    left = target - 1 - done
    if left >= 0:
        if left:
            g.step(left)
        torch.cuda.synchronize()
        g.kernel_times(2)
        g.step(1)
        torch.cuda.synchronize()
        print("# the step that recontours (surgery, recontouring, advance)")
        print(g.kernel_times(2), end="")
    g.kernel_times(0)
    g.close()


if __name__ == "__main__":
    main()
