#!/usr/bin/env python
"""Benchmark of the contour-advection time step (Hydra ca/plane/qg/caps) on B200.

Metric: node-steps/s -- the sum over steps of the contour nodes advanced,
divided by the device time of those steps.  A step is one pass of the
reference's advect loop body (evolution.f90:55-79): a regularisation (surgery
+ renode every step; prepare + recontour + init every 20th) followed by one
RK4 advance (4 inversions, 37 real 2-D FFTs, 4 con2grid, 4 velint).

Workload (the plain-CASL-at-scale configuration): doubly periodic
[-pi, pi)^2, 1024^2 inversion grid, random-phase PV with amplitude
k^3 exp(-(k/16)^2) normalised to rms 4 pi, 80 contour levels (about two
million FP64 nodes), surgery every step, recontouring every 20
regularisations, the reference's adaptive dt (dtmax 0.05).  Seeded synthetic
input; working set well above the 126 MB L2 (no flush needed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 (torchrun), every rank advances an independent ensemble member
(seed + rank): replicas, weak scaling, no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-steps/s on 1 B200, chosen vs plain form at <=1e-3 rel node-velocity err"
UNIT = "node-steps/s"


def workload_args(a):
    return dict(n=a.n, k0=a.k0, levels=a.levels, dtmax=a.dtmax)


def config_dict(a, nodes, mean_dt=None):
    return {
        "workload": f"plain CASL 2D Euler, {a.n}^2 grid, k0={a.k0:g}, {a.levels} levels, "
                    "surgery every step, recontour every 20 regularisations, adaptive dt",
        "n": a.n, "levels": a.levels, "k0": a.k0, "seed": a.seed, "dtmax": a.dtmax,
        "nodes_mean": nodes, "precision": "FP64 nodes and FP64 inversion",
        "l2": "working set > 126 MB L2 (fields + 4x fine grid + nodes); no flush",
        "parallelism": "replicas" if a.gpus > 1 else "single",
        "mean_dt": mean_dt, "host_nproc": os.cpu_count(),
    }


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock, its maximum, power and the active clock-event reasons of
    this process's GPU, read through NVML every 2 ms by a thread that stamps
    each sample with its own wall-clock time (a piped nvidia-smi delivers
    its lines in buffered bursts, whose arrival times say nothing about when
    they were taken).  Only reads; no setting of the GPU is touched."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, device):
        self.device = device
        self.samples = []  # (time, sm MHz, max sm MHz, power W, reason mask)
        self.window = None
        self.nvml = None
        self.stop_flag = threading.Event()

    def _handle(self, nv):
        try:
            import torch
            p = torch.cuda.get_device_properties(self.device)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nvml = nv
            self.h = self._handle(nv)
            self.max_sm = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        except Exception as e:
            self.nvml = None
            self.why = f"nvml unavailable: {type(e).__name__}"

    def _run(self):
        nv = self.nvml
        while not self.stop_flag.is_set():
            try:
                t = time.time()
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((t, sm, self.max_sm, pw, rs))
            except Exception:
                pass
            time.sleep(0.002)

    def mark(self, t0, t1):
        """The timed region in wall-clock seconds; only samples taken inside
        it are kept (the sampler runs from before the warm-up so that its
        start-up does not fall into the region)."""
        self.window = (t0, t1)

    def stop(self):
        if not self.nvml:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [getattr(self, "why", "nvml unavailable")]}
        self.stop_flag.set()
        self.thread.join(timeout=5)
        nv = self.nvml
        xs = self.samples
        if self.window:
            xs = [x for x in xs if self.window[0] <= x[0] <= self.window[1]]
        reasons = set()
        for x in xs:
            for nm, attr in self.REASONS:
                if x[4] & getattr(nv, attr, 0):
                    reasons.add(nm)
        try:
            nv.nvmlShutdown()
        except Exception:
            pass
        return {"sm_mhz": float(np.median([x[1] for x in xs])) if xs else None,
                "sm_max_mhz": float(self.max_sm),
                "power_w": float(np.median([x[3] for x in xs])) if xs else None,
                "reasons": sorted(reasons), "samples": len(xs)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes per launch of the transform pass at 1024^2, read off one ncu
# capture of the bench workload (dram__bytes_read.sum + dram__bytes_write.sum
# averaged over its k_rfft_r launches; profiles/rfft_pass_1024.md gives the
# command).  A stated constant, not a measurement of this run.
FFT_TRAFFIC_PER_LAUNCH_1024 = 30.7e6


# ---------------------------------------------------------------------------
# CPU legs (the oracle; test infrastructure, never the measured product)
# ---------------------------------------------------------------------------
def cpu_oracle_steps(state, a, budget_s, max_steps):
    """Time oracle steps on the given state (contours + fields); 1 core."""
    from oracle.oracle import Oracle
    c = state["contours"]
    o = Oracle(a.n, ncontq=a.levels, force_surgery=1, dtmax=a.dtmax,
               npm=max(4 * c["nptq"], 1 << 20), nm=max(4 * c["nq"], 1 << 16))
    o.set_contours(c)
    for f in ("qs", "qd", "qr"):
        o.set_field(f, state[f])
    o.set_scalar("t", state["t"])
    o.set_scalar("twist", 0.0)
    o.set_scalar("ireg", 0)
    node_steps, steps = 0, 0
    t0 = time.perf_counter()
    while steps < max_steps:
        node_steps += o.counts()[1]
        o.step()
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    return node_steps / dt, steps, dt


def run_reference(a):
    """--impl reference: the reference's CPU path (the oracle port; the Fortran
    reference cannot be compiled on these machines), serial as the reference
    is, on the same workload, with the same warm-up and timed steps as the
    GPU arm (a recontouring falls inside the timed steps on both arms)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle.oracle import Oracle
    from hydra_b200.synthetic import random_pv
    q0 = random_pv(a.n, a.k0, a.seed)
    o = Oracle(a.n, ncontq=a.levels, force_surgery=1, dtmax=a.dtmax,
               npm=16_000_000, nm=1_000_000)
    t_init = time.perf_counter()
    o.initialise(q0)
    t_init = time.perf_counter() - t_init
    for _ in range(a.warmup):
        o.step()
    node_steps, steps = 0, 0
    t_sim0 = o.scalar("t")
    t0 = time.perf_counter()
    while steps < a.steps:
        node_steps += o.counts()[1]
        o.step()
        steps += 1
    dt = time.perf_counter() - t0
    v = node_steps / dt
    nodes = node_steps / max(steps, 1)
    mean_dt = (o.scalar("t") - t_sim0) / max(steps, 1)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
        "steps": steps, "warmup": a.warmup, "ms_per_step": 1000.0 * dt / max(steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_dict(a, nodes, mean_dt),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": f"{steps} steps of the workload after {a.warmup} warm-up "
                                   f"steps (initialise {t_init:.0f} s untimed); the reference "
                                   "path is serial Fortran, restated in C (no Fortran compiler "
                                   "here)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# learned-closure leg (the "chosen" form of the metric)
# ---------------------------------------------------------------------------
CLOSURE_WEIGHTS = os.path.join(ROOT, "hydra_b200", "closure_512.npz")


def run_closure_leg(a, torch, device, steps=40, warmup=5, check_every=40, budget=1e-2):
    """The learned-closure configuration (512^2 grid, k0 = 12, 80 levels, the
    trained weights shipped with the library) against the plain form, every
    node-velocity error measured against the 2048^2 FP64 judge on states of
    an evaluation seed disjoint from the training seeds.  Throughput of the
    closure form includes its periodic fine-grid check (every check_every
    steps, inside the timed steps); the closure stays attached while its
    judged error is at most the budget and no larger than the plain form's,
    and a fallback is reported.  Plain forms at 512^2 and 1024^2 give the
    error-versus-cost curve the closure is placed on; their states are the
    same seed's field at that resolution.  Time to solution (simulated time
    per second) is reported beside node-steps/s because the node count grows
    with the grid."""
    from hydra_b200 import train_closure as tc
    from hydra_b200.casl import CaslGPU, CaslNet
    from hydra_b200.synthetic import random_pv
    if not os.path.exists(CLOSURE_WEIGHTS):
        return {"unavailable": "no trained weights (hydra_b200/closure_512.npz)"}
    d = np.load(CLOSURE_WEIGHTS)
    params, qs, us = tc.load(CLOSURE_WEIGHTS)
    n, k0, levels, seed = 512, 12.0, 80, 0
    kw = dict(ncontq=levels, force_surgery=1, dtmax=0.05, npm=8_000_000, nm=500_000, device=device)
    gf = CaslGPU(2048, ncontq=levels, npm=16_000_000, nm=1_000_000, device=device)
    out = {"config": f"learned closure: {n}^2 grid, k0={k0:g}, {levels} levels, seed {seed} "
                     "(training seeds from 1000), judge 2048^2 FP64",
           "training": {"pairs": int(d["pairs"]), "seconds": float(d["seconds"]),
                        "pairs_per_s": float(d["pairs"]) / float(d["seconds"])}}

    def timed(g, k):
        st = torch.cuda.ExternalStream(g.stream_ptr(), device=device)
        torch.cuda.synchronize()
        ns0, t0 = g.scalar("node_steps"), g.scalar("t")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        g.step(k)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        return {"ms_per_step": ms / k, "node_steps_per_s": (g.scalar("node_steps") - ns0) / (ms * 1e-3),
                "sim_time_per_s": (g.scalar("t") - t0) / (ms * 1e-3)}

    def errors(g, net=None, samples=4, gap=10):
        ep, en = [], []
        for _ in range(samples):
            g.step(gap)
            if net is not None:
                e = g.closure_evaluate(net, gf)
                ep.append(e[0]); en.append(e[1])
            else:
                uJ, vJ, uP, vP = g.judge(gf)
                ep.append(float(np.sqrt(((uP - uJ) ** 2 + (vP - vJ) ** 2).sum() / (uJ ** 2 + vJ ** 2).sum())))
        return float(np.mean(ep)), (float(np.mean(en)) if en else None)

    # closure and plain forms at 512^2, each on its own handle from the same
    # state (same seed, warm-up and error samples, all under the plain form),
    # timed over the same number of steps
    def form_512(closure):
        g = CaslGPU(n, **kw)
        g.initialise(random_pv(n, k0, seed))
        g.step(warmup)
        net = None
        if closure:
            net = CaslNet(n, device=device)
            net.set_params(params, qs, us)
        ep, en = errors(g, net)
        if closure:
            g.closure_attach(net, judge=gf, check_every=check_every, budget=budget)
        t = timed(g, steps)
        if closure:
            st = g.closure_status()
            g.closure_attach(None)
            t.update(err=en, active=st["active"], checks=st["checks"], fallbacks=st["fallbacks"])
            net.close()
        else:
            t.update(err=ep)
        g.close()
        return t

    out["closure_512"] = form_512(True)
    out["plain_512"] = form_512(False)
    # plain form at 1024^2 (judge twice as fine)
    g = CaslGPU(1024, ncontq=levels, force_surgery=1, dtmax=0.05, npm=16_000_000, nm=1_000_000,
                device=device)
    g.initialise(random_pv(1024, k0, seed))
    g.step(warmup)
    e1024, _ = errors(g)
    out["plain_1024"] = dict(timed(g, steps), err=e1024)
    g.close()
    gf.close()
    # the plain resolution with the closure's error, on the log-log line through
    # the two plain points, and the time to solution there
    c, p5, p10 = out["closure_512"], out["plain_512"], out["plain_1024"]
    if c["err"] and p5["err"] > p10["err"] > 0:
        order = np.log(p5["err"] / p10["err"]) / np.log(2.0)
        n_eq = 512.0 * (p5["err"] / c["err"]) ** (1.0 / order)
        cost_order = np.log(p5["sim_time_per_s"] / p10["sim_time_per_s"]) / np.log(2.0)
        sim_eq = p5["sim_time_per_s"] * (n_eq / 512.0) ** (-cost_order)
        out["equal_error"] = {"plain_grid_with_closure_error": n_eq, "error_order": order,
                              "speedup_time_to_solution": c["sim_time_per_s"] / sim_eq,
                              "note": "plain grid extrapolated on the log-log line through the "
                                      "512^2 and 1024^2 plain points"}
    return out


# ---------------------------------------------------------------------------
# batched-ensemble leg (the batched half of the "chosen" form)
# ---------------------------------------------------------------------------
def run_ensemble_leg(a, torch, device, members=256, n=256, steps=20, warmup=3, singles=8,
                     candidates=(32, 64, 128, 256)):
    """The batched ensemble configuration: `members` members of n^2 (seeds
    0.., k0 uniform in [4, 12], 20-60 levels, as ensemble_member_params
    draws them), surgery every step, recontouring every 20 regularisations.
    The members per handle are chosen by the autotuner
    (hydra_b200.ensemble_tune: every candidate batch steps all members, in
    consecutive batches, for 3 steps after 2); the chosen batch is then timed
    over `steps` steps after `warmup`.  Beside it the same members advanced
    one handle at a time (the plain form), on the first `singles` members.
    Both timed with CUDA events on the library's stream."""
    from hydra_b200.casl import CaslEnsemble, CaslGPU
    from hydra_b200 import ensemble_tune as et
    fields, levels = et.members(n, members)

    def timed(g, k):
        st = torch.cuda.ExternalStream(g.stream_ptr(), device=device)
        torch.cuda.synchronize()
        ns0 = g.scalar("node_steps")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        g.step(k)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), g.scalar("node_steps") - ns0

    rates, batch = et.tune_batch(fields, levels, candidates=candidates, steps=3, warmup=2,
                                 device=device, dtmax=a.dtmax, timer=timed)
    npm, nm = et._capacity(fields, levels, batch)
    ms, ns, sizes, t_init = 0.0, 0.0, [], 0.0
    for b0 in range(0, members, batch):
        e = CaslEnsemble(n, min(batch, members - b0), dtmax=a.dtmax, nregmax=20, npm=npm, nm=nm,
                         device=device)
        t0 = time.perf_counter()
        e.initialise_members(fields[b0:b0 + batch], levels[b0:b0 + batch])
        t_init += time.perf_counter() - t0
        e.step(warmup)
        x, y = timed(e, steps)
        ms += x
        ns += y
        sizes += [e.member_counts(m)[1] for m in range(e.members)]
        e.close()
    sms, sns = 0.0, 0.0
    for m in range(singles):
        g = CaslGPU(n, ncontq=levels[m], force_surgery=1, dtmax=a.dtmax, nregmax=20,
                    npm=4_000_000, nm=250_000, device=device)
        g.initialise(fields[m])
        g.step(warmup)
        x, y = timed(g, steps)
        sms += x
        sns += y
        g.close()
    return {"config": f"batched ensemble: {members} members of {n}^2, k0 ~ U[4,12], levels ~ "
                      f"U[20,60], seeds 0..{members - 1}, surgery every step, recontour every 20 "
                      f"regularisations; {steps} steps after {warmup} (one recontouring inside)",
            "autotune": {"members_per_handle": batch,
                         "node_steps_per_s": {str(k): v for k, v in rates.items()}},
            "node_steps_per_s": ns / (ms * 1e-3), "ms_per_step": ms / steps,
            "nodes_min": int(min(sizes)), "nodes_max": int(max(sizes)),
            "nodes_total": int(sum(sizes)), "initialise_s": t_init,
            "one_at_a_time": {"members_timed": singles, "node_steps_per_s": sns / (sms * 1e-3),
                              "ms_per_member_step": sms / (singles * steps)},
            "speedup_vs_one_at_a_time": (ns / ms) / (sns / sms) if sms > 0 else None}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def reduce_over_ranks(vals, world, device):
    """[ms, node_steps, e2e_ms, e2e_node_steps] of this rank -> the job's
    (max ms, summed node-steps, max e2e ms, summed e2e node-steps): the time
    of the slowest replica, the work of all of them.  The all-reduces run on
    the process group's backend (NCCL between GPUs)."""
    import torch
    import torch.distributed as dist
    if world <= 1:
        return vals[0], vals[1], vals[2], vals[3]
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = t.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx[0].item(), sm[1].item(), mx[2].item(), sm[3].item()


def run_gpu(a):
    import torch
    import torch.distributed as dist

    from hydra_b200.casl import CaslGPU, load_library
    from hydra_b200.synthetic import random_pv

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    load_library()

    q0 = random_pv(a.n, a.k0, a.seed + rank)
    g = CaslGPU(a.n, ncontq=a.levels, force_surgery=1, dtmax=a.dtmax,
                npm=16_000_000, nm=1_000_000, device=local)
    g.initialise(q0)
    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(a.warmup):
        g.step(1)
    stream = torch.cuda.ExternalStream(g.stream_ptr(), device=local)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- resident-data timed region ------------------------------------------------
    barrier()
    wall0 = time.time()
    ns0 = g.scalar("node_steps")
    tsim0 = g.scalar("t")
    l0 = g.launch_count()
    g.profile(1)  # the transform passes
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(a.steps):
        g.step(1)
    ev1.record(stream)
    barrier()
    clocks.mark(wall0, time.time())
    ms = ev0.elapsed_time(ev1)
    launches = g.launch_count() - l0
    fft_ms, fft_n, fft_bytes = g.profile_read()
    g.profile(0)
    node_steps = g.scalar("node_steps") - ns0
    mean_dt = (g.scalar("t") - tsim0) / a.steps
    clk = clocks.stop()

    # ---- end to end through the C-ABI with host buffers -----------------------------
    e2e = run_e2e(g, a, stream, torch)

    # CPU baseline on this host (rank 0, N = 1 only): the oracle on the same state
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        state = {"contours": g.contours(), "qs": g.field("qs"), "qd": g.field("qd"),
                 "qr": g.field("qr"), "t": g.scalar("t")}
        v, steps, dt = cpu_oracle_steps(state, a, a.cpu_seconds, 8)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{steps} oracle steps ({dt:.1f} s) from the GPU run's state after "
                         "its timed steps (surgery + advance; no recontouring in the sample)"}

    closure = None
    if rank == 0 and world == 1 and not a.no_closure:
        closure = run_closure_leg(a, torch, local)
    ensemble = None
    if rank == 0 and world == 1 and not a.no_ensemble:
        ensemble = run_ensemble_leg(a, torch, local)

    # ---- reduce over ranks ---------------------------------------------------------------
    ms_max, ns_sum, e2e_ms, e2e_ns = reduce_over_ranks(
        [ms, node_steps, e2e["ms"], e2e["node_steps"]], world, f"cuda:{local}")
    if rank == 0:
        peak, peak_kind = measured_peak()
        ach = fft_bytes / (fft_ms * 1e-3) / 1e9 if fft_ms > 0 else 0.0
        traffic = FFT_TRAFFIC_PER_LAUNCH_1024 if a.n == 1024 else None
        line = {
            "metric": METRIC,
            "value": ns_sum / (ms_max * 1e-3),
            "unit": UNIT,
            "n_gpus": world,
            "steps": a.steps,
            "warmup": a.warmup,
            "ms_per_step": ms_max / a.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": config_dict(a, node_steps / a.steps, mean_dt),
            "e2e": {"value": e2e_ns / (e2e_ms * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                    "steps": e2e["steps"]},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak if peak else None, "traffic": traffic,
                         "traffic_source": "constant: ncu DRAM bytes per k_rfft_r launch at "
                                           "1024^2 (profiles/rfft_pass_1024.md)",
                         "bytes_rule": "16 B per FP64 element per 2-D transform (one read, "
                                       "one write); a pass counts half",
                         "kernel": "k_rfft (batched real-FFT pass, all variants)",
                         "launches": fft_n, "kernel_ms_per_step": fft_ms / a.steps,
                         "peak_source": f"{peak_kind} hbm_gbs"},
            "cpu_baseline": cpu,
            "closure": closure,
            "ensemble": ensemble,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_e2e(g, a, stream, torch):
    """node-steps/s through the public C-ABI with the state in pinned host
    memory: every step uploads contours + spectral fields, steps, downloads."""
    import ctypes as C
    lib = g.lib
    n = a.n
    cap_n, cap_c = 16_000_000, 1_000_000

    def pinned(shape, dtype):
        t = torch.empty(shape, dtype=dtype, pin_memory=True)
        return t.numpy()

    xq = pinned(cap_n, torch.float64); yq = pinned(cap_n, torch.float64)
    nextq = pinned(cap_n, torch.int32)
    indq = pinned(cap_c, torch.int32); npq = pinned(cap_c, torch.int32)
    i1q = pinned(cap_c, torch.int32); i2q = pinned(cap_c, torch.int32)
    qs = pinned((n, n), torch.float64); qd = pinned((n, n), torch.float64)
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    D = lambda x: x.ctypes.data_as(dp)
    I = lambda x: x.ctypes.data_as(ip)

    def download():
        nq, npt, qj = g.counts()
        g._check(lib.casl_get_contours(g.h, D(xq), D(yq), I(nextq), I(indq), I(npq), I(i1q), I(i2q)),
                 "casl_get_contours")
        g._check(lib.casl_get_field(g.h, 0, D(qs)), "casl_get_field")
        g._check(lib.casl_get_field(g.h, 1, D(qd)), "casl_get_field")
        return nq, npt, qj

    nq, npt, qj = download()
    steps = max(1, a.steps)   # same steps as the timed region (recontourings included)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ns0 = g.scalar("node_steps")
    h2d = d2h = 0
    ev0.record(stream)
    for _ in range(steps):
        g._check(lib.casl_set_contours(g.h, nq, npt, qj, D(xq), D(yq), I(nextq), I(indq), I(npq),
                                       I(i1q), I(i2q)), "casl_set_contours")
        g._check(lib.casl_set_field(g.h, 0, D(qs)), "casl_set_field")
        g._check(lib.casl_set_field(g.h, 1, D(qd)), "casl_set_field")
        h2d += npt * 20 + nq * 16 + 2 * n * n * 8
        g.step(1)
        nq, npt, qj = download()
        d2h += npt * 20 + nq * 16 + 2 * n * n * 8
    ev1.record(stream)
    torch.cuda.synchronize()
    return {"ms": ev0.elapsed_time(ev1), "node_steps": g.scalar("node_steps") - ns0,
            "h2d": h2d // steps, "d2h": d2h // steps, "steps": steps}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["hydra", "reference"], default="hydra")
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--k0", type=float, default=16.0)
    ap.add_argument("--levels", type=int, default=80)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--dtmax", type=float, default=0.05)
    ap.add_argument("--cpu-seconds", type=float, default=20.0,
                    help="time budget of the cpu_baseline leg of the GPU arm")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-closure", action="store_true", help="skip the learned-closure leg")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble leg")
    a = ap.parse_args()
    if a.warmup < 3 and a.impl == "hydra":
        print("bench: at least 3 warm-up steps are required", file=sys.stderr)
        return 2
    if a.impl == "reference":
        return run_reference(a)
    return run_gpu(a)


if __name__ == "__main__":
    sys.exit(main())
