"""The FP32-inversion mode against the FP64 path, per field.

CASL_PREC_FP32_INVERSION stores the intermediate and the outputs of every
stage's inverse transform pair (the velocities and the x/y derivatives of qd
and qs) in FP32; the state stays FP64.  One RK4 step from the same state in
both modes, then 20 driver steps, with the error of each field reported and
held to a budget: stored-FP32 rounding is 2^-24 relative, the transform adds
two such roundings and the node update integrates the velocity over dt.
"""
import numpy as np
import pytest

from hydra_b200.synthetic import random_pv

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_fp32_inversion_errors_per_field(oracle_mod, gpu_lib, capsys):
    from hydra_b200.casl import CaslGPU
    n = 256
    o = oracle_mod.Oracle(n, ncontq=40, force_surgery=1, dtmax=0.05)
    o.initialise(random_pv(n, 8.0, 6))
    o.step()
    kw = dict(ncontq=40, force_surgery=1, dtmax=0.05)
    g64, g32 = CaslGPU(n, **kw), CaslGPU(n, **kw)
    for g in (g64, g32):
        g.set_contours(o.contours())
        for f in ("qs", "qd", "qr"):
            g.set_field(f, o.field(f))
        g.set_scalar("t", o.scalar("t"))
    g32.set_precision(1)
    g64.advance()
    g32.advance()
    err = {}
    for f in ("uu", "vv"):  # the last stage's velocity field
        err[f] = rel(g32.field(f), g64.field(f))
    for f in ("qs", "qd", "pp"):
        err[f] = rel(g32.field(f), g64.field(f))
    c64, c32 = g64.contours(), g32.contours()
    err["nodes"] = float(max(np.abs(c32["xq"] - c64["xq"]).max(), np.abs(c32["yq"] - c64["yq"]).max()))
    u64, v64 = g64.velint(g64.field("uu"), g64.field("vv"))
    u32, v32 = g32.velint(g32.field("uu"), g32.field("vv"))
    err["node_velocity"] = max(rel(u32, u64), rel(v32, v64))
    err["dt"] = abs(g32.scalar("dt") - g64.scalar("dt")) / g64.scalar("dt")
    # 20 driver steps (surgery, a recontouring) from there
    g64.step(20)
    g32.step(20)
    d64, d32 = g64.diagnostics(), g32.diagnostics()
    for k in ("ekin", "enstrophy", "circulation"):
        err["20 steps " + k] = abs(d32[k] - d64[k]) / abs(d64[k])
    with capsys.disabled():
        print("\nFP32 inversion vs FP64 (relative; nodes absolute):")
        for k, v in err.items():
            print(f"  {k:28s} {v:.2e}")
    for f in ("uu", "vv", "node_velocity"):
        assert err[f] <= 2e-6, (f, err[f])
    for f in ("qs", "qd"):
        assert err[f] <= 2e-6, (f, err[f])
    assert err["nodes"] <= 1e-7
    assert err["dt"] <= 1e-6
    for k in ("ekin", "enstrophy"):
        assert err["20 steps " + k] <= 1e-4, k
    # the contour circulation moves in steps when a surgery decision flips
    # (a filament kept by one run and dropped by the other)
    assert err["20 steps circulation"] <= 1e-2
    g64.close(); g32.close(); o.close()
