"""The oracle's restatement of econgen.f90 (beta != 0 recontouring) on the
CPU: the contoured PV of a beta-plane state reproduces its anomaly to within
the contour interval, every node lies in the basic box, and a beta*Ly that
is not a whole number of contour intervals is refused (code 3), where the
reference stops (econgen.f90:52-60)."""
import numpy as np
import pytest

from hydra_b200.synthetic import random_pv

BETA, KD = 10.0, 2.5


def full_pv(n, k0, seed):
    y = -np.pi + 2 * np.pi * np.arange(n) / n
    return random_pv(n, k0, seed) + BETA * y[None, :]


def test_beta_contours_reproduce_the_anomaly(oracle_mod):
    n = 32
    q = random_pv(n, 4.0, 3)
    o = oracle_mod.Oracle(n, ncontq=20, beta=BETA, kd=KD)
    o.initialise(full_pv(n, 4.0, 3))
    c = o.contours()
    assert c["nq"] > 0 and c["qjump"] == pytest.approx(BETA * 2 * np.pi / 20)
    assert c["yq"].min() >= -np.pi and c["yq"].max() < np.pi
    assert c["xq"].min() >= -np.pi and c["xq"].max() < np.pi
    # the gridded contour PV (the anomaly, beta*y removed) against the input
    err = np.sqrt(np.mean((o.con2grid() - q) ** 2))
    assert err < c["qjump"]


def test_beta_steps_through_recontour(oracle_mod):
    n = 32
    o = oracle_mod.Oracle(n, ncontq=20, beta=BETA, kd=KD, force_surgery=1, dtmax=0.05)
    o.initialise(full_pv(n, 4.0, 3))
    for _ in range(22):
        o.step()
    c = o.contours()
    assert c["nq"] > 0
    assert c["yq"].min() >= -np.pi and c["yq"].max() < np.pi


def test_beta_ratio_refused(oracle_mod):
    n = 32
    o = oracle_mod.Oracle(n, ncontq=10, beta=BETA, kd=KD)
    o.initialise(full_pv(n, 4.0, 0))
    c = o.contours()
    c["qjump"] = c["qjump"] * 1.1
    o.set_contours(c)
    with pytest.raises(RuntimeError, match=r"\(3\)"):
        o.recontour(np.zeros((n, n)))
