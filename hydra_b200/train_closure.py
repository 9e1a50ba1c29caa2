"""Train the learned velocity closure on pairs the solver itself produces.

Each training pair is one state of a running simulation at the coarse grid n:
its inversion (contour PV, u, v on n^2; the plain bilinear node velocities)
against the fine-grid judge's node velocities (the same contours inverted on
(4n)^2 plus the coarse non-contour spectrum).  Every pair is used once, as it
is made, by the library's own tensor-core forward and backward kernels and an
Adam step (casl_closure_train).  States come from runs of the plain solver
(surgery every step, recontouring every 20 regularisations) started from
random-phase fields of seeds disjoint from the evaluation seeds; each run
gives its first 250 states (the node count about quadruples over them), after
which a new seed starts, so the pairs cover the early turbulent states that
the closure is evaluated on.

  python -m hydra_b200.train_closure --n 512 --pairs 20000 --out hydra_b200/closure_512.npz
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from .casl import CaslGPU, CaslNet
from .synthetic import random_pv

# the last layer's channels: the u and v correction at the points of the
# finer grid inside each coarse cell
HID = 16  # hidden channels (the library's HID)
NOUT = 8  # output channels (the library's NOUT, CASL_NET_OUT)
NIN = 12  # input channels (the library's NIN, CASL_NET_IN)
LAYERS = [(NIN, HID), (HID, HID), (HID, HID), (HID, NOUT)]


def init_params(seed: int) -> np.ndarray:
    """He-style weights (N(0, 2/fan_in) scaled by 1/2), zero biases, and a last
    layer 100x smaller so that training starts from an almost plain form."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (ci, co) in enumerate(LAYERS):
        w = rng.standard_normal(co * ci * 25) * 0.5 * np.sqrt(2.0 / (ci * 25))
        if l == len(LAYERS) - 1:
            w *= 0.01
        parts += [w, np.zeros(co)]
    return np.concatenate(parts).astype(np.float32)


def field_scales(g: CaslGPU) -> tuple[float, float]:
    """rms of the contour PV and of the speed of g's latest inversion."""
    g.inversion()
    u, v = g.field("uu"), g.field("vv")
    return float(np.sqrt(np.mean(g.con2grid() ** 2))), float(np.sqrt(np.mean(u * u + v * v)))


def save(path, params, qscale, uscale, meta):
    np.savez(path, params=params, qscale=np.float32(qscale), uscale=np.float32(uscale),
             **{k: np.asarray(v) for k, v in meta.items()})


def load(path):
    d = np.load(path)
    return d["params"], float(d["qscale"]), float(d["uscale"])


def train(n=512, pairs=20000, pairs_per_run=250, lr=1e-3, lr_end=1e-4, k0=12.0, levels=80,
          seed0=1000, fine=4, device=0, log_every=250, out=None, quiet=False):
    kw = dict(ncontq=levels, force_surgery=1, dtmax=0.05, npm=8_000_000, nm=500_000)
    g = CaslGPU(n, device=device, **kw)
    gf = CaslGPU(fine * n, device=device, ncontq=levels, npm=8_000_000, nm=500_000)
    net = CaslNet(n, device=device)
    g.initialise(random_pv(n, k0, seed0))
    qs, us = field_scales(g)
    net.set_params(init_params(seed0), qs, us)
    hist = []
    t0 = time.perf_counter()
    done, run = 0, 0
    while done < pairs:
        g.initialise(random_pv(n, k0, seed0 + run))
        if not quiet:
            print(f"run {run}: seed {seed0 + run}, {g.counts()[1]} nodes "
                  f"({time.perf_counter() - t0:.0f} s)", flush=True)
        for _ in range(min(pairs_per_run, pairs - done)):
            g.step(1)
            frac = done / max(pairs - 1, 1)
            rate = lr * (lr_end / lr) ** frac  # geometric decay
            hist.append(g.closure_train(net, gf, rate))
            done += 1
            if not quiet and done % log_every == 0:
                h = np.array(hist[-log_every:])
                print(f"pairs {done}: plain {h[:, 0].mean():.3e} net {h[:, 1].mean():.3e} "
                      f"loss {h[:, 2].mean():.3e}, nodes {g.counts()[1]} "
                      f"({time.perf_counter() - t0:.0f} s)", flush=True)
        run += 1
    secs = time.perf_counter() - t0
    params, qs, us = net.params()
    if out:
        save(out, params, qs, us, dict(n=n, pairs=pairs, fine=fine, k0=k0, levels=levels,
                                       seed0=seed0, runs=run, seconds=secs))
    net.close()
    g.close()
    gf.close()
    return params, qs, us, np.array(hist), secs


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--pairs-per-run", type=int, default=250)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-end", type=float, default=1e-4, help="final rate of the geometric decay")
    ap.add_argument("--k0", type=float, default=12.0)
    ap.add_argument("--levels", type=int, default=80)
    ap.add_argument("--seed0", type=int, default=1000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    _, _, _, hist, secs = train(a.n, a.pairs, a.pairs_per_run, a.lr, lr_end=a.lr_end, k0=a.k0,
                                levels=a.levels, seed0=a.seed0, out=a.out)
    print(f"trained on {len(hist)} pairs in {secs:.1f} s")


if __name__ == "__main__":
    main()
