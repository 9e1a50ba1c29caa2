"""GPU surgery and renode against the oracle, through the C-ABI.

Bar: after one surgery/renode pass the node count, the contour count, every
contour's length, start, end and level must be identical; node positions
agree within 1e-12 relative (the density sums are added in a different order).
"""
import numpy as np
import pytest

from hydra_b200.synthetic import random_pv

pytestmark = pytest.mark.gpu

REL = 1e-12


def circle(n_nodes, r, x0, y0, phase=0.0, wobble=0.0, k=3):
    th = (np.arange(n_nodes) + phase) * 2 * np.pi / n_nodes
    rr = r * (1 + wobble * np.cos(k * th))
    return x0 + rr * np.cos(th), y0 + rr * np.sin(th)


@pytest.fixture(scope="module")
def gpu64(gpu_lib):
    from hydra_b200.casl import CaslGPU
    g = CaslGPU(64, ncontq=20, dtmax=0.05)
    yield g
    g.close()


@pytest.mark.parametrize("case", ["circle", "wobbly", "corners", "tiny", "duplicates"])
def test_renode_single(oracle_mod, gpu64, case):
    o = oracle_mod.Oracle(64, ncontq=20)
    if case == "duplicates":
        # surgery joins nodes by moving one onto the other: zero-length
        # segments, whose density is zero, between every pair here; each
        # must receive no node however the density sums round
        x, y = circle(700, 0.9, 0.2, -0.1, wobble=0.25, k=7)
        x, y = np.repeat(x, 2), np.repeat(y, 2)
    elif case == "circle":
        x, y = circle(300, 1.0, 0.1, -0.2)
    elif case == "wobbly":
        x, y = circle(500, 0.8, -0.3, 0.4, wobble=0.3, k=5)
    elif case == "corners":
        # a square: every vertex is a corner
        s = np.linspace(0, 1, 40, endpoint=False)
        x = np.concatenate([s, np.ones(40), 1 - s, np.zeros(40)]) * 0.9 - 0.2
        y = np.concatenate([np.zeros(40), s, np.ones(40), 1 - s]) * 0.9 - 0.3
    else:
        x, y = circle(6, 1e-4, 0.0, 0.0)
    xo, yo = o.renode(x, y)
    xg, yg = gpu64.renode(x, y)
    assert len(xg) == len(xo)
    assert np.all(np.isfinite(xg)) and np.all(np.isfinite(yg))
    if len(xo):
        assert np.abs(xg - xo).max() <= REL * np.pi
        assert np.abs(yg - yo).max() <= REL * np.pi


def compare_contours(co, cg):
    assert cg["nq"] == co["nq"] and cg["nptq"] == co["nptq"]
    for k in ("npq", "i1q", "i2q", "indq", "nextq"):
        assert np.array_equal(cg[k], co[k]), k
    assert np.abs(cg["xq"] - co["xq"]).max() <= REL * np.pi
    assert np.abs(cg["yq"] - co["yq"]).max() <= REL * np.pi


def test_surgery_two_circles(oracle_mod, gpu64):
    glx = 2 * np.pi / 64
    dm = 0.2**2 * 6.25 * glx / 4
    gap = 0.3 * dm
    xc = 0.13
    x1, y1 = circle(200, 0.5, xc - 0.5 - gap / 2, 0.0)
    x2, y2 = circle(200, 0.5, xc + 0.5 + gap / 2, 0.0, phase=0.5)
    c = dict(xq=np.concatenate([x1, x2]), yq=np.concatenate([y1, y2]),
             nextq=np.concatenate([np.arange(2, 201), [1], np.arange(202, 401), [201]]).astype(np.int32),
             indq=np.array([1, 1], np.int32), npq=np.array([200, 200], np.int32),
             i1q=np.array([1, 201], np.int32), i2q=np.array([200, 400], np.int32), qjump=1.0)
    o = oracle_mod.Oracle(64, ncontq=20)
    o.set_contours(c)
    gpu64.set_contours(c)
    o.surgery()
    gpu64.surgery()
    co, cg = o.contours(), gpu64.contours()
    assert co["nq"] == 1
    compare_contours(co, cg)


@pytest.mark.parametrize("seed,steps", [(0, 0), (1, 3), (2, 6)])
def test_surgery_matches_oracle(oracle_mod, gpu64, seed, steps):
    n = 64
    o = oracle_mod.Oracle(n, ncontq=20, force_surgery=1, dtmax=0.05)
    o.initialise(random_pv(n, 6.0, seed))
    for _ in range(steps):
        o.step()
    c0 = o.contours()
    gpu64.set_contours(c0)
    o.surgery()
    gpu64.surgery()
    compare_contours(o.contours(), gpu64.contours())


def test_surgery_matches_oracle_large(oracle_mod, gpu_lib):
    """~120k nodes at 256^2: the binning, rebuild and renode scans run their
    multi-tile paths (more than 16 tiles of 4096)."""
    from hydra_b200.casl import CaslGPU
    n = 256
    o = oracle_mod.Oracle(n, ncontq=40, force_surgery=1, dtmax=0.05)
    o.initialise(random_pv(n, 8.0, 4))
    o.step()
    c0 = o.contours()
    assert c0["nptq"] > 16 * 4096
    g = CaslGPU(n, ncontq=40, force_surgery=1, dtmax=0.05)
    g.set_contours(c0)
    o.surgery()
    g.surgery()
    compare_contours(o.contours(), g.contours())
    g.close()
