"""Device time of the batched real-FFT passes behind each spectral entry
point (ptospc, spctop, gradient, main_invert) at one grid size.

Every transform launch is bracketed by CUDA events on the library's stream
(the host copies of the C-ABI calls fall outside them), so the numbers are
the kernels' own.  One JSON line per entry point: microseconds per launch
and achieved GB/s on the algorithmic bytes (each element read once and
written once per pass, plus the extra fields a fused load reads).

    python -m hydra_b200.bench_transforms --n 1024 --reps 20
"""
import argparse
import json

import numpy as np

from hydra_b200.casl import CaslGPU

PROF_OFF, PROF_FFT = 0, 1


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args(argv)
    n = a.n
    g = CaslGPU(n, ncontq=10, npm=1000)
    rng = np.random.default_rng(0)
    q = rng.standard_normal((n, n))
    s = g.ptospc(q)
    calls = {
        "ptospc": lambda: g.ptospc(q),
        "spctop": lambda: g.spctop(s),
        "gradient": lambda: g.gradient(s),
        "main_invert": lambda: g.main_invert(s),
    }
    for name, fn in calls.items():
        for _ in range(3):
            fn()
        g.profile(PROF_FFT)
        for _ in range(a.reps):
            fn()
        ms, launches, nbytes = g.profile_read()
        g.profile(PROF_OFF)
        print(json.dumps({"transform": name, "n": n, "launches": launches,
                          "us_per_launch": 1e3 * ms / launches,
                          "gbs": nbytes / (ms * 1e-3) / 1e9}))
    g.close()


if __name__ == "__main__":
    main()
