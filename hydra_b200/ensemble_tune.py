"""Autotuner of the batched ensemble's batch size: how many members one
handle (casl_ensemble_*) steps together.

Every stage of a step is one launch across the handle's members, so larger
batches fill the GPU better; but a batch holds its members' fields, nodes
and scratch at once, and recontouring walks its members one at a time
through a view sized for the largest, so past some size a batch stops
paying.  Where that point lies depends on the member size, the node counts
and the GPU, so it is measured: each candidate batch size steps its share of
the members (every member, in consecutive batches) for a few steps after a
warm-up, timed with CUDA events on the library's stream, and the size with
the most node-steps per second is chosen.

    python -m hydra_b200.ensemble_tune --n 256 --members 256
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from .casl import CaslEnsemble
from .synthetic import ensemble_member_params, random_pv


def _capacity(fields, levels, batch):
    """Node and contour capacity for a batch: 80M / 4M per 256 members of
    256^2 (the bench's sizes), scaled by the batch and the grid."""
    n = fields[0].shape[0]
    scale = max(batch / 256.0, 1.0 / 16.0) * (n / 256.0) ** 2
    return int(80_000_000 * scale), int(4_000_000 * scale)


def time_batch(fields, levels, batch, steps=3, warmup=2, device=0, dtmax=0.05, timer=None):
    """Node-steps/s of stepping all members in consecutive batches of
    `batch`: each batch handle is initialised, warmed up and timed for
    `steps` steps; the times and node-steps add up over the batches.
    `timer(handle, steps) -> (ms, node_steps)` times one handle (default:
    CUDA events on the handle's stream)."""
    if timer is None:
        timer = _event_timer(device)
    n = fields[0].shape[0]
    npm, nm = _capacity(fields, levels, batch)
    ms_total, ns_total = 0.0, 0.0
    for b0 in range(0, len(fields), batch):
        fs, ls = fields[b0:b0 + batch], levels[b0:b0 + batch]
        e = CaslEnsemble(n, len(fs), dtmax=dtmax, nregmax=20, npm=npm, nm=nm, device=device)
        try:
            e.initialise_members(fs, ls)
            e.step(warmup)
            ms, ns = timer(e, steps)
        finally:
            e.close()
        ms_total += ms
        ns_total += ns
    return ns_total / (ms_total * 1e-3)


def tune_batch(fields, levels, candidates=(32, 64, 128, 256), steps=3, warmup=2, device=0,
               dtmax=0.05, timer=None):
    """Times every candidate batch size (those not above the member count)
    and returns ({batch: node-steps/s}, the fastest batch)."""
    rates = {}
    for b in candidates:
        if b > len(fields):
            continue
        rates[b] = time_batch(fields, levels, b, steps, warmup, device, dtmax, timer)
    if not rates:
        raise ValueError("no candidate batch size fits the member count")
    best = max(rates, key=rates.get)
    return rates, best


def _event_timer(device):
    import torch

    def timer(g, k):
        st = torch.cuda.ExternalStream(g.stream_ptr(), device=device)
        torch.cuda.synchronize()
        ns0 = g.scalar("node_steps")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        g.step(k)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), g.scalar("node_steps") - ns0

    return timer


def members(n, count):
    """The ensemble workload's members: seeds 0.., k0 ~ U[4, 12], 20-60 levels."""
    params = [ensemble_member_params(m) for m in range(count)]
    return [random_pv(n, k0, m) for m, (k0, _) in enumerate(params)], [lv for _, lv in params]


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--steps", type=int, default=3)
    a = ap.parse_args()
    fields, levels = members(a.n, a.members)
    rates, best = tune_batch(fields, levels, steps=a.steps)
    print(json.dumps({"n": a.n, "members": a.members,
                      "node_steps_per_s": {str(k): v for k, v in rates.items()}, "chosen": best}))


if __name__ == "__main__":
    main()
