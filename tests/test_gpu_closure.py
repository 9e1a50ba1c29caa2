"""The closure network's tensor-core kernels against its CPU restatement
(oracle/closure_oracle.py), through the C ABI.

The GPU accumulates in FP32 on the tensor cores and rounds to BF16 where the
restatement does; the sums run in another order, so a stored BF16 value can
differ by one unit in the last place (2^-8 relative) where the FP32 value sits
at a rounding boundary.  Bars: the output within 1e-2 of its largest
magnitude (mean error below 1e-3 of it); every parameter gradient within 2e-2
of the largest gradient of its tensor.
"""
import numpy as np
import pytest

from oracle import closure_oracle as co

pytestmark = pytest.mark.gpu


def inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((co.NIN, n, n)).astype(np.float32)
    # smooth structure too, as the solver's fields have
    yy, xx = np.meshgrid(np.arange(n), np.arange(n))
    x[0] += np.sin(2 * np.pi * 3 * xx / n) * np.cos(2 * np.pi * 2 * yy / n)
    return x


@pytest.mark.parametrize("n", [128, 256])
def test_forward_matches_oracle(gpu_lib, n):
    from hydra_b200.casl import CaslNet
    p = co.init_params(3)
    p[co.param_count() - co.NOUT:] = np.linspace(-0.3, 0.3, co.NOUT)  # output bias
    x = inputs(n, n)
    net = CaslNet(n)
    net.set_params(p)
    y = net.forward(x)
    ref, _ = co.forward(p, x)
    scale = np.abs(ref).max()
    assert scale > 0.1
    err = np.abs(y - ref)
    assert err.max() <= 1e-2 * scale, (err.max(), scale)
    assert err.mean() <= 1e-3 * scale, (err.mean(), scale)
    net.close()


def test_backward_matches_oracle(gpu_lib):
    from hydra_b200.casl import CaslNet
    n = 128
    p = co.init_params(4)
    x = inputs(n, 5)
    dy = np.random.default_rng(6).standard_normal((co.NOUT, n, n)).astype(np.float32)
    net = CaslNet(n)
    net.set_params(p)
    net.forward(x)
    g = net.backward(dy)
    _, cache = co.forward(p, x)
    ref = co.backward(p, cache, dy)
    o = 0
    for l, (ci, cout) in enumerate(co.LAYERS):
        for size, what in ((cout * ci * 25, "W"), (cout, "b")):
            a, b = g[o:o + size], ref[o:o + size]
            scale = np.abs(b).max()
            assert np.abs(a - b).max() <= 2e-2 * scale, (l, what, np.abs(a - b).max(), scale)
            o += size
    net.close()


def test_adam_step(gpu_lib):
    """One Adam step from zero moments moves every parameter by lr * sign(g)
    (to within eps), as the update rule gives for the first step."""
    from hydra_b200.casl import CaslNet
    n = 128
    p = co.init_params(7)
    net = CaslNet(n)
    net.set_params(p)
    net.forward(inputs(n, 8))
    g = net.backward(np.random.default_rng(9).standard_normal((co.NOUT, n, n)).astype(np.float32))
    net.adam(1e-3)
    p1, _, _ = net.params()
    moved = p1 - p
    big = np.abs(g) > 1e-3 * np.abs(g).max()
    assert np.allclose(moved[big], -1e-3 * np.sign(g[big]), rtol=1e-3, atol=1e-7)
    net.close()


# ---------------------------------------------------------------------------
# the closure inside the solver
# ---------------------------------------------------------------------------
from hydra_b200.synthetic import ptospc_np, random_pv  # noqa: E402


def _state(oracle_mod, n, k0, levels, seed, steps):
    o = oracle_mod.Oracle(n, ncontq=levels, force_surgery=1, dtmax=0.05)
    o.initialise(random_pv(n, k0, seed))
    for _ in range(steps):
        o.step()
    return o


def _load(o, g):
    g.set_contours(o.contours())
    for f in ("qs", "qd", "qr"):
        g.set_field(f, o.field(f))
    for s in ("t", "twist"):
        g.set_scalar(s, o.scalar(s))


def test_judge_matches_oracle(oracle_mod, gpu_lib):
    """The fine-grid judge (4x) against the oracle's con2grid + main_invert at
    the fine resolution plus the padded non-contour spectrum, and velint on the
    fine grid; the plain node velocities against the oracle's velint."""
    from hydra_b200.casl import CaslGPU
    n, nf = 64, 256
    o = _state(oracle_mod, n, 6.0, 20, 2, 3)
    g = CaslGPU(n, ncontq=20, force_surgery=1, dtmax=0.05)
    gf = CaslGPU(nf, ncontq=20, npm=4_000_000)
    _load(o, g)
    uJ, vJ, uP, vP = g.judge(gf)
    o.inversion()
    qq, qc = o.field("qq"), o.field("qc")
    of = oracle_mod.Oracle(nf, ncontq=20, npm=4_000_000)
    of.set_contours(o.contours())
    qqf = ptospc_np(of.con2grid()) + co.pad_spectrum(qq - qc, nf)
    uf, vf, _ = of.main_invert(qqf)
    uJo, vJo = of.velint(uf, vf)
    uPo, vPo = o.velint(o.field("uu"), o.field("vv"))
    s = np.abs(uJo).max()
    assert np.abs(uJ - uJo).max() <= 1e-10 * s and np.abs(vJ - vJo).max() <= 1e-10 * s
    assert np.abs(uP - uPo).max() <= 1e-12 * s and np.abs(vP - vPo).max() <= 1e-12 * s
    # the judge differs from the plain form by the resolution error only
    rel = np.sqrt(((uP - uJ) ** 2 + (vP - vJ) ** 2).sum() / (uJ ** 2 + vJ ** 2).sum())
    assert 1e-6 < rel < 0.2, rel
    g.close(); gf.close(); of.close(); o.close()


def _pair(oracle_mod, n, seed, steps=2, levels=30, k0=8.0):
    from hydra_b200.casl import CaslGPU
    o = _state(oracle_mod, n, k0, levels, seed, steps)
    kw = dict(ncontq=levels, force_surgery=1, dtmax=0.05)
    a, b = CaslGPU(n, **kw), CaslGPU(n, **kw)
    _load(o, a)
    _load(o, b)
    o.close()
    return a, b


def test_features_are_the_inversion_fields(oracle_mod, gpu_lib):
    from hydra_b200.casl import CaslGPU, CaslNet
    n = 128
    g, _ = _pair(oracle_mod, n, 1)
    net = CaslNet(n)
    net.set_params(np.zeros(co.param_count(), np.float32), qscale=5.0, uscale=2.0)
    x = g.closure_features(net)
    qc, lv = g.con2grid(levels=True)
    ref = np.stack([qc / 5.0, g.field("uu") / 2.0, g.field("vv") / 2.0])
    assert np.abs(x[:3] - co.bf16(ref)).max() <= 1e-2 * np.abs(ref).max()
    # the sub-cell channels: fine levels against the coarse cell's 7 x 7
    # weighted sum C of the same levels (con2grid's coarsening, weights
    # [1,2,3,4,3,2,1]^2 centred on fine point 4cx, 4cy)
    qj = g.contours()["qjump"]
    nf = lv.shape[0]
    w7 = np.array([1, 2, 3, 4, 3, 2, 1], np.int64)
    cx = np.arange(n)
    C = np.zeros((n, n), np.int64)
    for a in range(7):
        for b in range(7):
            C += w7[a] * w7[b] * lv[np.ix_((4 * cx - 3 + a) % nf, (4 * cx - 3 + b) % nf)]
    sub = co.subcell_features(lv, C, qj, 1.0 / 5.0)
    assert np.abs(sub).max() > 0.0
    assert np.abs(x[3:12] - co.bf16(sub)).max() <= 1e-2 * np.abs(sub).max()
    net.close(); g.close(); _.close()


def test_node_correction_is_the_fine_grid_interpolation(oracle_mod, gpu_lib):
    """The correction added to each node's velocity is us times the bilinear
    interpolation, on the finer grid, of the network's output channels (restated in numpy by oracle/closure_oracle.node_correction)."""
    from hydra_b200.casl import CaslNet
    n = 128
    g, _ = _pair(oracle_mod, n, 2)
    p = co.init_params(7)
    p[-co.NOUT:] = np.linspace(-0.2, 0.2, co.NOUT)
    net = CaslNet(n)
    net.set_params(p, qscale=5.0, uscale=2.0)
    g.inversion()
    du, dv = g.closure_correction(net)
    y = net.forward(g.closure_features(net))
    c = g.contours()
    ru, rv = co.node_correction(y, c["xq"], c["yq"], 2.0, n)
    scale = max(np.abs(ru).max(), np.abs(rv).max())
    assert scale > 1e-3
    assert np.abs(du - ru).max() <= 1e-9 * scale
    assert np.abs(dv - rv).max() <= 1e-9 * scale
    net.close(); g.close(); _.close()


def test_zero_network_leaves_the_step_unchanged(oracle_mod, gpu_lib):
    """A network whose output is zero corrects nothing: the step is bit-for-bit
    the plain one."""
    from hydra_b200.casl import CaslNet
    n = 128
    a, b = _pair(oracle_mod, n, 3)
    net = CaslNet(n)
    net.set_params(np.zeros(co.param_count(), np.float32), 4.0, 2.0)
    b.closure_attach(net)
    a.advance()
    b.advance()
    ca, cb = a.contours(), b.contours()
    assert np.array_equal(ca["xq"], cb["xq"]) and np.array_equal(ca["yq"], cb["yq"])
    net.close(); a.close(); b.close()


def test_constant_correction_shifts_the_nodes(oracle_mod, gpu_lib):
    """Output bias b0 on the u channels, b1 on the v channels, zero
    weights: the correction is us*(b0, b1) everywhere on the fine grid, so
    every node moves with velint's velocity plus us*(b0, b1) at every stage.  With qjump = 0 and qs = qd = 0 the flow
    itself is zero, so the plain step leaves the nodes in place and one RK4
    step of the corrected one moves every node by exactly dt*us*b."""
    from hydra_b200.casl import CaslNet
    n = 128
    a, b = _pair(oracle_mod, n, 4)
    for g in (a, b):
        c = g.contours()
        c["qjump"] = 0.0
        g.set_contours(c)
        for f in ("qs", "qd"):
            g.set_field(f, np.zeros((n, n)))
    p = np.zeros(co.param_count(), np.float32)
    p[-co.NOUT:] = [0.5] * (co.NOUT // 2) + [-0.25] * (co.NOUT // 2)
    net = CaslNet(n)
    net.set_params(p, 4.0, 2.0)
    b.closure_attach(net)
    a.advance()
    b.advance()
    dt = a.scalar("dt")
    assert dt == b.scalar("dt")
    ca, cb = a.contours(), b.contours()
    L = 2 * np.pi
    dx = (cb["xq"] - ca["xq"] + np.pi) % L - np.pi
    dy = (cb["yq"] - ca["yq"] + np.pi) % L - np.pi
    assert dt > 0.0
    # every stage's wrap multiplies by oms = 1 - 1e-11 (evolution.f90:219)
    assert np.abs(dx - dt * 2.0 * 0.5).max() <= 1e-9
    assert np.abs(dy - dt * 2.0 * (-0.25)).max() <= 1e-9
    net.close(); a.close(); b.close()


def test_fallback_fires_and_recovers(oracle_mod, gpu_lib):
    """A network whose correction is far outside the budget is switched off
    by the periodic fine-grid check; the step then runs plain velint (bit-for-
    bit the plain step); a harmless network passes the check."""
    from hydra_b200.casl import CaslGPU, CaslNet
    n = 128
    a, b = _pair(oracle_mod, n, 5)
    gf = CaslGPU(4 * n, ncontq=30, npm=8_000_000)
    p = np.zeros(co.param_count(), np.float32)
    p[-2:] = [3.0, 3.0]
    net = CaslNet(n)
    net.set_params(p, 4.0, 2.0)
    b.closure_attach(net, judge=gf, check_every=2, budget=0.5)
    assert b.closure_status()["active"] == 1
    a.step(1)
    b.step(1)  # the check runs before this step's advance
    st = b.closure_status()
    assert st["checks"] == 1 and st["fallbacks"] == 1 and st["active"] == 0
    assert st["err_net"] > st["err_plain"]
    ca, cb = a.contours(), b.contours()
    assert np.array_equal(ca["xq"], cb["xq"])  # the fallback step is the plain step
    net.set_params(np.zeros(co.param_count(), np.float32), 4.0, 2.0)
    ep, en = b.closure_check()
    assert en == pytest.approx(ep, rel=1e-12) and b.closure_status()["active"] == 1
    net.close(); a.close(); b.close(); gf.close()


def test_training_reduces_node_velocity_error(oracle_mod, gpu_lib, capsys):
    """Trained on pairs the solver makes (128^2 states against the 512^2
    judge, seeds 1-3), the closure lowers the node-velocity error of a state
    from an unseen seed (seed 11) below the plain bilinear form's."""
    from hydra_b200.casl import CaslGPU, CaslNet
    n, levels = 128, 30
    kw = dict(ncontq=levels, force_surgery=1, dtmax=0.05)
    g = CaslGPU(n, **kw)
    gf = CaslGPU(4 * n, ncontq=levels, npm=8_000_000)
    net = CaslNet(n)
    g.initialise(random_pv(n, 8.0, 1))
    g.inversion()
    us = float(np.sqrt((g.field("uu") ** 2 + g.field("vv") ** 2).mean()))
    qs = float(np.sqrt((g.con2grid() ** 2).mean()))
    p = co.init_params(0, gain=0.5)
    p[co.param_count() - 2 - 32 * 32 * 25:co.param_count() - 2] *= 0.01  # small initial output
    net.set_params(p, qs, us)
    hist = []
    for seed in (1, 2, 3):
        g.initialise(random_pv(n, 8.0, seed))
        for it in range(100):
            if it % 4 == 0:
                g.step(1)
            hist.append(g.closure_train(net, gf, 1e-3))
    g.initialise(random_pv(n, 8.0, 11))
    g.step(3)
    ep, en, _ = g.closure_evaluate(net, gf)
    with capsys.disabled():
        print(f"\nclosure 128^2 vs 512^2 judge: first samples plain {hist[0][0]:.3e} net "
              f"{hist[0][1]:.3e}; last {hist[-1][0]:.3e} / {hist[-1][1]:.3e}; held-out seed 11: "
              f"plain {ep:.3e}, net {en:.3e} (gain {ep / en:.2f}x)")
    assert en < ep
    net.close(); g.close(); gf.close()


def test_closure_in_the_fp32_inversion_mode(oracle_mod, gpu_lib):
    """With FP32 storage of the inverse transforms the closure reads the FP32
    fields: one RK4 step moves the nodes by the same correction as in the
    FP64 mode.  The network's inputs are BF16, and a field value near a BF16
    rounding boundary rounds to neighbouring BF16 values (2^-8 apart,
    relative) in the two modes, so the bar is statistical: the median node
    within 1e-3 of the largest correction, every node within 5e-2."""
    from hydra_b200.casl import CaslNet
    n = 128
    p = co.init_params(11)
    p[-co.NOUT:] = np.linspace(-0.2, 0.2, co.NOUT)
    net = CaslNet(n)
    net.set_params(p, qscale=5.0, uscale=2.0)
    moves = []
    for prec in (0, 1):
        a, b = _pair(oracle_mod, n, 5)
        for g in (a, b):
            g.set_precision(prec)
        b.closure_attach(net)
        a.advance()
        b.advance()
        ca, cb = a.contours(), b.contours()
        assert ca["nptq"] == cb["nptq"]
        L = 2 * np.pi
        moves.append(np.stack([(cb["xq"] - ca["xq"] + np.pi) % L - np.pi,
                               (cb["yq"] - ca["yq"] + np.pi) % L - np.pi]))
        a.close(); b.close()
    d64, d32 = moves
    scale = np.abs(d64).max()
    assert scale > 0.0
    err = np.abs(d32 - d64)
    assert np.median(err) <= 1e-3 * scale
    assert err.max() <= 5e-2 * scale
    net.close()
