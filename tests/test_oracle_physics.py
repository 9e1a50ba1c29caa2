"""Self-checks of the oracle against analytic answers and internal identities.

The reference ships no tests or golden data, so these pin the oracle's
restatement of contours.f90 / evolution.f90 / congen.f90 instead.
"""
import numpy as np
import pytest

from hydra_b200.synthetic import random_pv


def circle_contour(n_nodes, r, x0=0.1, y0=-0.2, phase=0.0):
    th = (np.arange(n_nodes) + phase) * 2 * np.pi / n_nodes
    return x0 + r * np.cos(th), y0 + r * np.sin(th)


def single_contour(xq, yq, qjump, level=1):
    npt = len(xq)
    nxt = np.arange(2, npt + 2, dtype=np.int32)
    nxt[-1] = 1
    return dict(xq=xq, yq=yq, nextq=nxt, indq=np.array([level], np.int32),
                npq=np.array([npt], np.int32), i1q=np.array([1], np.int32),
                i2q=np.array([npt], np.int32), qjump=qjump)


def test_con2grid_circle_area(oracle_mod):
    """A counter-clockwise circle of radius r carries PV qjump inside, so the
    mean-removed grid field integrates to zero and its jump is qjump."""
    n = 64
    o = oracle_mod.Oracle(n, ncontq=10)
    x, y = circle_contour(400, 1.0)
    o.set_contours(single_contour(x, y, 1.0))
    qc, lv = o.con2grid(levels=True)
    assert abs(qc.sum()) < 1e-9
    # fine-grid levels: 0/1 indicator of the disc (up to an additive constant)
    lv = lv - lv.min()
    assert set(np.unique(lv)) <= {0, 1}
    area = lv.sum() * (2 * np.pi / (4 * n)) ** 2
    assert abs(area - np.pi) < 0.02
    # grid field range ~ qjump
    assert 0.9 < qc.max() - qc.min() < 1.01


def test_con2grid_levels_match_float_path(oracle_mod):
    """The fine-grid field the reference accumulates in floating point equals
    qjump times the integer level index the oracle counts alongside it."""
    n = 64
    o = oracle_mod.Oracle(n, ncontq=20)
    o.initialise(random_pv(n, 6.0, 7))
    qc, lv = o.con2grid(levels=True)
    qj = o.counts()[2]
    # coarsen the integer levels with the composed 7x7 stencil and compare
    nf = 4 * n
    w = np.array([1, 2, 3, 4, 3, 2, 1], float)
    L = lv.astype(float)            # [ix, iy] fine
    C = np.zeros((n, n))
    for a in range(7):
        for b in range(7):
            fx = (4 * np.arange(1, n + 1) - 6 + b - 1) % nf
            fy = (4 * np.arange(1, n + 1) - 6 + a - 1) % nf
            C += w[a] * w[b] * L[np.ix_(fx, fy)]
    q_exact = qj * (C - C.mean()) / 256.0
    assert np.abs(q_exact - qc).max() < 1e-11 * max(1.0, np.abs(qc).max())


def test_velint_bilinear_exact_for_linear_field(oracle_mod):
    n = 32
    o = oracle_mod.Oracle(n, ncontq=10)
    x, y = circle_contour(50, 0.7)
    o.set_contours(single_contour(x, y, 1.0))
    h = 2 * np.pi / n
    xg = -np.pi + h * np.arange(n)
    uu = np.repeat((0.3 * xg)[:, None], n, axis=1) + 0.0   # [ix, iy] = 0.3 x
    vv = np.repeat((0.2 * xg)[None, :], n, axis=0)          # 0.2 y
    uq, vq = o.velint(uu, vv)
    np.testing.assert_allclose(uq, 0.3 * x, atol=1e-12)
    np.testing.assert_allclose(vq, 0.2 * y, atol=1e-12)


def test_rankine_patch_velocity(oracle_mod):
    """Circular patch of PV q0, radius R (small vs the period): azimuthal
    velocity q0 r / 2 inside, q0 R^2 / (2 r) outside."""
    n, R, q0 = 128, 0.5, 1.0
    o = oracle_mod.Oracle(n, ncontq=10)
    x, y = circle_contour(800, R, 0.0, 0.0)
    o.set_contours(single_contour(x, y, q0))
    qc = o.con2grid()
    uu, vv, _ = o.main_invert(o.ptospc(qc))
    h = 2 * np.pi / n
    g = -np.pi + h * np.arange(n)
    X, Y = np.meshgrid(g, g, indexing="ij")
    r = np.hypot(X, Y)
    vt = (-uu * Y + vv * X) / np.maximum(r, 1e-9)
    inside = (r > 0.1) & (r < 0.35)
    outside = (r > 0.75) & (r < 1.0)
    np.testing.assert_allclose(vt[inside], q0 * r[inside] / 2, atol=0.03)
    # periodic images and the zero-mean PV reduce the far field slightly
    np.testing.assert_allclose(vt[outside], q0 * R**2 / (2 * r[outside]), atol=0.03)


def test_renode_circle(oracle_mod):
    """renode keeps a circle a circle, with node spacing set by curvature."""
    o = oracle_mod.Oracle(64, ncontq=10)
    x, y = circle_contour(300, 1.0)
    xr, yr = o.renode(x, y)
    assert 20 < len(xr) < 300
    r = np.hypot(xr - 0.1, yr + 0.2)
    assert np.abs(r - 1.0).max() < 1e-3
    # too-small contours are dropped
    x, y = circle_contour(6, 1e-4)
    xr, yr = o.renode(x, y)
    assert len(xr) == 0


def test_surgery_reconnects_close_contours(oracle_mod):
    """Two same-level circles closer than dm reconnect into one contour."""
    n = 64
    o = oracle_mod.Oracle(n, ncontq=10)
    glx = 2 * np.pi / n
    dm = 0.2**2 * 6.25 * glx / 4
    gap = 0.3 * dm
    # centre the gap inside a search box (boxes of width 2 pi / 24 start at -pi)
    xc = 0.13
    x1, y1 = circle_contour(200, 0.5, xc - 0.5 - gap / 2, 0.0)
    x2, y2 = circle_contour(200, 0.5, xc + 0.5 + gap / 2, 0.0, phase=0.5)
    xs = np.concatenate([x1, x2]); ys = np.concatenate([y1, y2])
    nxt = np.concatenate([np.arange(2, 201), [1], np.arange(202, 401), [201]]).astype(np.int32)
    c = dict(xq=xs, yq=ys, nextq=nxt, indq=np.array([1, 1], np.int32), npq=np.array([200, 200], np.int32),
             i1q=np.array([1, 201], np.int32), i2q=np.array([200, 400], np.int32), qjump=1.0)
    o.set_contours(c)
    o.surgery()
    nq, npt, _ = o.counts()
    assert nq == 1 and npt > 50
    # different levels never reconnect
    c["indq"] = np.array([1, 2], np.int32)
    o.set_contours(c)
    o.surgery()
    assert o.counts()[0] == 2


def test_initialise_and_steps_conserve_energy(oracle_mod):
    n = 64
    o = oracle_mod.Oracle(n, ncontq=20, force_surgery=1, dtmax=0.05)
    o.initialise(random_pv(n, 6.0, 0))
    nq, npt, qj = o.counts()
    assert nq > 50 and npt > 2000
    o.step()
    e0 = o.diagnostics()["ekin"]
    for _ in range(3):
        o.step()
    e1 = o.diagnostics()["ekin"]
    assert abs(e1 - e0) < 1e-3 * e0   # hyperdiffusion + surgery at 64^2
    assert o.scalar("dt") > 0


def test_recontour_every_nregmax(oracle_mod):
    """With forced surgery, the 20th regularisation recontours (ireg wraps)."""
    n = 32
    o = oracle_mod.Oracle(n, ncontq=10, force_surgery=1, nregmax=3, dtmax=0.05)
    o.initialise(random_pv(n, 4.0, 1))
    iregs = []
    for _ in range(5):
        o.step()
        iregs.append(int(o.scalar("ireg")))
    assert iregs == [1, 2, 1, 2, 1]
