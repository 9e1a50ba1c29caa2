"""The non-zero physics branches against the oracle, through the C ABI.

With kd > 0 the inversion is a Helmholtz problem (green = -1/(k^2 + kd^2),
spectral.f90:136-147); beta > 0 subtracts beta*y in con2grid
(contours.f90:279-286) and adds -beta*v to the source of qs
(evolution.f90:452-460); rekman and rtherm add Ekman friction and thermal
damping to the source of qd (evolution.f90:466-477).  The contour state is a
beta = 0 initialisation handed to both sides, so each case checks the
arithmetic of one branch on identical inputs.
"""
import numpy as np
import pytest

from hydra_b200.synthetic import random_pv

pytestmark = pytest.mark.gpu

REL = 1e-12

CASES = {
    "helmholtz": dict(kd=2.5),
    "beta": dict(beta=10.0),
    "ekman": dict(rekman=0.1),
    "qg_all": dict(kd=2.5, beta=10.0, rekman=0.1, rtherm=0.05),
}


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def base(oracle_mod):
    n = 64
    o = oracle_mod.Oracle(n, ncontq=20, dtmax=0.05)
    o.initialise(random_pv(n, 6.0, 5))
    st = dict(c=o.contours(), qs=o.field("qs"), qd=o.field("qd"), qr=o.field("qr"),
              t=o.scalar("t"))
    o.close()
    return n, st


def pair_for(oracle_mod, n, st, kw):
    from hydra_b200.casl import CaslGPU
    o = oracle_mod.Oracle(n, ncontq=20, dtmax=0.05, **kw)
    g = CaslGPU(n, ncontq=20, dtmax=0.05, **kw)
    for x in (o, g):
        x.set_contours(st["c"])
        for f in ("qs", "qd", "qr"):
            x.set_field(f, st[f])
        x.set_scalar("t", st["t"])
        x.set_scalar("twist", 0.0)
    return o, g


@pytest.mark.parametrize("case", list(CASES))
def test_main_invert_and_con2grid(oracle_mod, gpu_lib, base, case):
    n, st = base
    o, g = pair_for(oracle_mod, n, st, CASES[case])
    qq = st["qs"]
    uo, vo, po = o.main_invert(qq)
    ug, vg, pg = g.main_invert(qq)
    assert rel_err(ug, uo) < REL and rel_err(vg, vo) < REL
    assert rel_err(pg, po) < REL
    qc_o, lv_o = o.con2grid(levels=True)
    qc_g, lv_g = g.con2grid(levels=True)
    assert np.array_equal(lv_g, lv_o)
    assert rel_err(qc_g, qc_o) < REL
    assert rel_err(g.con2grid(), qc_o) < REL  # packed path
    g.close()
    o.close()


@pytest.mark.parametrize("case", list(CASES))
def test_advance_one_step(oracle_mod, gpu_lib, base, case):
    n, st = base
    o, g = pair_for(oracle_mod, n, st, CASES[case])
    o.advance()
    g.advance()
    co, cg = o.contours(), g.contours()
    assert rel_err(cg["xq"], co["xq"]) < REL
    assert rel_err(cg["yq"], co["yq"]) < REL
    assert abs(g.scalar("dt") - o.scalar("dt")) <= 1e-14 * o.scalar("dt")
    for f in ("qs", "qd"):
        assert rel_err(g.field(f), o.field(f)) < 1e-11, f
    for f in ("uu", "vv"):
        assert rel_err(g.field(f), o.field(f)) < REL, f
    dg, do = g.diagnostics(), o.diagnostics()
    for k in ("ekin", "epot", "enstrophy"):
        assert abs(dg[k] - do[k]) <= 1e-10 * max(abs(do[k]), 1e-300), k
    g.close()
    o.close()
