"""One recontouring of the bench workload inside a profiler range.

Initialises the bench workload (random PV of spectral peak k0 on an n^2
grid, 80 levels), takes a few steps so that contours exist, then calls
casl_recontour once (contours plus a zero residual: the path casl_step takes
every nregmax regularisations) between cudaProfilerStart and
cudaProfilerStop, so that a profiler started with --profile-from-start off
sees exactly the recontouring's kernels.  Prints the contour and node counts
and the recontouring's wall time.

    python -m hydra_b200.bench_recontour --n 512
"""
import argparse
import time

import numpy as np
import torch

from hydra_b200.casl import CaslGPU
from hydra_b200.synthetic import random_pv


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--k0", type=float, default=16.0)
    ap.add_argument("--levels", type=int, default=80)
    ap.add_argument("--steps", type=int, default=3)
    a = ap.parse_args(argv)
    torch.cuda.init()
    g = CaslGPU(a.n, ncontq=a.levels, force_surgery=1, dtmax=0.05, npm=16_000_000, nm=1_000_000)
    g.initialise(random_pv(a.n, a.k0, 0))
    g.step(a.steps)
    g.synchronize()
    z = np.zeros((a.n, a.n))
    torch.cuda.profiler.start()
    t = time.perf_counter()
    g.recontour(z)
    g.synchronize()
    ms = 1e3 * (time.perf_counter() - t)
    torch.cuda.profiler.stop()
    nq, npt, qjump = g.counts()
    print(f"recontour {a.n}^2: {nq} contours, {npt} nodes, {ms:.2f} ms (wall)")
    g.close()


if __name__ == "__main__":
    main()
