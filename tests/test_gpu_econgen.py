"""Recontouring on a beta-plane (econgen.f90, the reference's ecaps build)
through the C-ABI, against the oracle's restatement of econgen.f90.

PV q = anomaly + beta*y is not periodic in y: the ultra-fine field is
extended over the rows its levels need, contours are traced on the extended
grid and one periodic image of each is kept.  Bars as for beta = 0: contour
and node counts and every contour's length, start, end, level and links
identical; nodes within 1e-10 of the domain after initialise (1e-8 with a
residual, whose ultra-fine sums run in another order than the reference's).
Cases use beta = 10 and kd = 2.5 (ncontq levels across beta*Ly).
"""
import numpy as np
import pytest

from hydra_b200.synthetic import random_pv

pytestmark = pytest.mark.gpu

BETA, KD = 10.0, 2.5


def same_topology(co, cg):
    assert cg["nq"] == co["nq"], (cg["nq"], co["nq"])
    assert cg["nptq"] == co["nptq"], (cg["nptq"], co["nptq"])
    for k in ("npq", "i1q", "i2q", "indq", "nextq"):
        assert np.array_equal(cg[k], co[k]), k


def close_nodes(co, cg, tol):
    assert np.abs(cg["xq"] - co["xq"]).max() <= tol * np.pi
    assert np.abs(cg["yq"] - co["yq"]).max() <= tol * np.pi


def full_pv(n, k0, seed, beta=BETA):
    """Anomaly of the usual construction plus beta*y ([ix][iy] layout)."""
    y = -np.pi + 2 * np.pi * np.arange(n) / n
    return random_pv(n, k0, seed) + beta * y[None, :]


@pytest.mark.parametrize("n,k0,levels,seed", [(32, 4.0, 10, 0), (64, 6.0, 20, 1), (128, 8.0, 30, 2)])
def test_beta_initialise(oracle_mod, gpu_lib, n, k0, levels, seed):
    from hydra_b200.casl import CaslGPU
    q = full_pv(n, k0, seed)
    o = oracle_mod.Oracle(n, ncontq=levels, beta=BETA, kd=KD, dtmax=0.05)
    o.initialise(q)
    g = CaslGPU(n, ncontq=levels, beta=BETA, kd=KD, dtmax=0.05)
    g.initialise(q)
    co, cg = o.contours(), g.contours()
    assert co["qjump"] == cg["qjump"]
    assert co["nq"] > 0
    same_topology(co, cg)
    close_nodes(co, cg, 1e-10)
    # every node folded into the basic box
    assert cg["yq"].min() >= -np.pi and cg["yq"].max() < np.pi
    for f in ("qs", "qd", "qc"):
        a, b = o.field(f), g.field(f)
        assert np.abs(a - b).max() <= 1e-10 * np.abs(a).max(), f
    g.close()


def test_beta_recontour_with_residual(oracle_mod, gpu_lib):
    from hydra_b200.casl import CaslGPU
    n = 64
    o = oracle_mod.Oracle(n, ncontq=20, beta=BETA, kd=KD, force_surgery=1, dtmax=0.05)
    o.initialise(full_pv(n, 6.0, 4))
    for _ in range(3):
        o.step()
    g = CaslGPU(n, ncontq=20, beta=BETA, kd=KD, dtmax=0.05)
    g.set_contours(o.contours())
    rng = np.random.default_rng(0)
    resid = 0.05 * o.counts()[2] * rng.standard_normal((n, n))
    o.recontour(resid)
    g.recontour(resid)
    co, cg = o.contours(), g.contours()
    same_topology(co, cg)
    close_nodes(co, cg, 1e-8)
    g.close()


def test_beta_driver_steps_through_recontour(oracle_mod, gpu_lib):
    """25 forced-surgery steps on the beta-plane: a recontour at step 20."""
    from hydra_b200.casl import CaslGPU
    n = 64
    q = full_pv(n, 6.0, 5)
    kw = dict(ncontq=20, beta=BETA, kd=KD, force_surgery=1, dtmax=0.05, nregmax=20)
    o = oracle_mod.Oracle(n, **kw)
    g = CaslGPU(n, **kw)
    o.initialise(q)
    g.initialise(q)
    for step in range(25):
        o.step()
        g.step(1)
        no, ng = o.counts(), g.counts()
        assert no[0] == ng[0] and no[1] == ng[1], (step, no, ng)
    co, cg = o.contours(), g.contours()
    same_topology(co, cg)
    close_nodes(co, cg, 1e-8)
    g.close()


def test_beta_ratio_must_be_integer(oracle_mod, gpu_lib):
    """beta*Ly/qjump not an integer: the reference stops (econgen.f90:52-60);
    here CASL_EINVAL, and the oracle's code 3."""
    from hydra_b200.casl import CaslError, CaslGPU
    n = 32
    o = oracle_mod.Oracle(n, ncontq=10, beta=BETA, kd=KD, dtmax=0.05)
    o.initialise(full_pv(n, 4.0, 0))
    c = o.contours()
    c["qjump"] = c["qjump"] * 1.1
    g = CaslGPU(n, ncontq=10, beta=BETA, kd=KD, dtmax=0.05)
    g.set_contours(c)
    with pytest.raises(CaslError) as ei:
        g.recontour(np.zeros((n, n)))
    assert ei.value.code == 1  # CASL_EINVAL
    g.close()
