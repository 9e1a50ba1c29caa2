"""Per-kernel device times of the closure network's tensor-core kernels.

Runs the network's forward and backward passes (casl_net_forward /
casl_net_backward) on an n x n input with every launch of the library timed
by a pair of CUDA events (casl_kernel_times), and reports for each
convolution kernel its mean time and its tensor-core rate: executed FLOPs
(2 * n^2 * 25 * CIN * COUT with the padded channel counts the MMAs run) per
second, against the measured dense BF16 peak.

  python -m hydra_b200.bench_closure [--n 512] [--reps 20]
"""
from __future__ import annotations

import argparse
import json
import os
import re

import numpy as np

from .casl import NET_IN, NET_OUT, CaslNet

# padded channel counts of each convolution, from the kernel's name: the
# forward and input-gradient kernels k_conv5<CIN, COUT, R, MODE> and the
# weight gradients k_conv5_wgrad<CIN, COUT, R> (CIN the layer input, COUT
# its output; an input gradient runs with the layer's COUT as its CIN)
_NAME = re.compile(r"(k_conv5(?:_wgrad)?)<(\d+), (\d+), \d+(?:, (\d+))?>")


def peak_tflops():
    try:
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        with open(os.path.join(root, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def run(n=512, reps=20, device=0):
    net = CaslNet(n, device=device)
    rng = np.random.default_rng(0)
    p = (rng.standard_normal(net.count) * 0.05).astype(np.float32)
    net.set_params(p)
    x = rng.standard_normal((NET_IN, n, n)).astype(np.float32)
    dy = rng.standard_normal((NET_OUT, n, n)).astype(np.float32)
    net.forward(x)
    net.backward(dy)
    lib = net.lib
    import ctypes as C
    lib.casl_kernel_times(1, None, 0)
    for _ in range(reps):
        net.forward(x)
        net.backward(dy)
    buf = C.create_string_buffer(1 << 16)
    lib.casl_kernel_times(2, buf, len(buf))
    lib.casl_kernel_times(0, None, 0)
    net.close()
    peak, kind = peak_tflops()
    rows = []
    for line in buf.value.decode().splitlines():
        m = re.match(r"\s*(\S.*?)\s+(\d+)\s+([\d.]+)\s+ms\s+([\d.]+)\s+us\s*$", line)
        if not m:
            continue
        name, launches, total_ms, mean_us = m.group(1), int(m.group(2)), float(m.group(3)), float(m.group(4))
        k = _NAME.match(name)
        if not k:
            continue
        ci, co = int(k.group(2)), int(k.group(3))
        flops = 2.0 * n * n * 25 * ci * co  # per launch
        tf = flops / (mean_us * 1e-6) / 1e12
        rows.append(dict(kernel=name, launches=launches, mean_us=mean_us,
                         tflops=tf, frac=tf / peak))
    return dict(n=n, reps=reps, peak_tflops=peak, peak_source=kind, kernels=rows)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args()
    r = run(a.n, a.reps)
    print(f"closure network at {a.n}^2, {a.reps} forward + backward passes; peak "
          f"{r['peak_tflops']:.0f} TFLOP/s ({r['peak_source']})")
    for k in r["kernels"]:
        print(f"  {k['kernel']:28s} {k['launches']:5d} launches  {k['mean_us']:8.1f} us  "
              f"{k['tflops']:7.1f} TFLOP/s  {100 * k['frac']:5.1f} % of peak")
    print(json.dumps(r))


if __name__ == "__main__":
    main()
