"""Forcing of qd (row f3) against the oracle, through the C ABI: pvforce's
point vortices and dipoles (evolution.f90:330-428) and the narrow-band
spectral forcing (spectral.f90:160-285), from the same random numbers.
Vortices sharing a grid point are summed in another order on the GPU, so qd
agrees to rounding (1e-12 of its largest value)."""
import numpy as np
import pytest

from hydra_b200.synthetic import random_pv

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def state(oracle_mod):
    n = 64
    o = oracle_mod.Oracle(n, ncontq=20, dtmax=0.05)
    o.initialise(random_pv(n, 6.0, 8))
    st = dict(c=o.contours(), qs=o.field("qs"), qd=o.field("qd"))
    o.close()
    return n, st


def pair(oracle_mod, n, st):
    from hydra_b200.casl import CaslGPU
    o = oracle_mod.Oracle(n, ncontq=20)
    g = CaslGPU(n, ncontq=20)
    for x in (o, g):
        x.set_contours(st["c"])
        x.set_field("qs", st["qs"])
        x.set_field("qd", st["qd"])
    return o, g


@pytest.mark.parametrize("ivor", [1, 2])
def test_pvforce_matches_oracle(oracle_mod, gpu_lib, state, ivor):
    n, st = state
    o, g = pair(oracle_mod, n, st)
    rng = np.random.default_rng(ivor)
    m = 2 if ivor == 1 else 3
    rnd = rng.random((37, m))
    rnd[3, -2:] = [0.0, 0.999999]  # grid corner and the periodic wrap
    o.pvforce(ivor, 12.5, rnd)
    g.pvforce(ivor, 12.5, rnd)
    qd_o, qd_g = o.field("qd"), g.field("qd")
    assert rel(qd_g, qd_o) <= 1e-12
    assert rel(qd_o, st["qd"]) > 1e-6  # the forcing changed qd
    g.close(); o.close()


def test_nb_forcing_matches_oracle(oracle_mod, gpu_lib, state):
    n, st = state
    o, g = pair(oracle_mod, n, st)
    k_o = o.nb_forcing_init(8.0, 1.5, 0.25)
    k_g = g.nb_forcing_init(8.0, 1.5, 0.25)
    assert k_o == k_g > 0
    rng = np.random.default_rng(3)
    for _ in range(2):
        rnd = 2.0 * rng.random(k_g) - 1.0
        o.nb_forcing(0.01, rnd)
        g.nb_forcing(0.01, rnd)
    assert rel(g.field("qd"), o.field("qd")) <= 1e-13
    g.close(); o.close()


def test_nb_forcing_band_checks(gpu_lib):
    from hydra_b200.casl import CaslError, CaslGPU
    g = CaslGPU(64, ncontq=20)
    for kfmid, fwid in ((2.0, 2.5), (30.0, 3.0)):  # reaches k = 0 / the Nyquist wavenumber
        with pytest.raises(CaslError) as e:
            g.nb_forcing_init(kfmid, fwid, 1.0)
        assert e.value.code == 1
    g.close()
