"""The oracle's 1-D spectrum (spec1d, spectral.f90:370-424) and its tables
(init_spectral, spectral.f90:109-134), pinned to closed forms: a single
Fourier mode puts all of its weight in the one shell nint(|k|/delk), the
shell sums add up to the weighted sum of squares of the Hermitian array,
and the tables follow from counting modes per shell."""
import numpy as np
import pytest


def _single_mode(n, kx, ky):
    x = -np.pi + 2 * np.pi * np.arange(n) / n
    X, Y = np.meshgrid(x, x, indexing="ij")  # (ix, iy)
    return np.cos(kx * X) * np.cos(ky * Y)


@pytest.mark.parametrize("kx,ky", [(3, 0), (0, 5), (3, 5), (7, 2)])
def test_single_mode_lands_in_one_shell(oracle_mod, kx, ky):
    n = 32
    o = oracle_mod.Oracle(n)
    ss = o.ptospc(_single_mode(n, kx, ky))
    spec, after = o.spec1d(ss, 0)
    assert np.array_equal(after, ss)  # iopt = 0 leaves the field alone
    shell = int(np.floor(np.hypot(kx, ky) / np.sqrt(2.0) + 0.5))
    nz = np.flatnonzero(np.abs(spec) > 1e-12 * np.abs(spec).max())
    assert list(nz) == [shell]


def test_shell_sums_are_weighted_sum_of_squares(oracle_mod):
    n = 64
    o = oracle_mod.Oracle(n)
    rng = np.random.default_rng(3)
    ss = o.ptospc(rng.standard_normal((n, n)))
    spec, _ = o.spec1d(ss, 0)
    w = np.ones((n, n))
    w[0, :] = 0.5
    w[:, 0] = 0.5
    w[0, 0] = 0.25
    assert spec[n // 2 + 1:].max() == 0.0
    assert abs(spec.sum() - (w * ss ** 2).sum()) <= 1e-12 * spec.sum()


def test_iopt1_multiplies_by_filtered_ksq(oracle_mod):
    n = 32
    o = oracle_mod.Oracle(n)
    rng = np.random.default_rng(4)
    ss = rng.standard_normal((n, n))
    spec1, after = o.spec1d(ss, 1)
    rksq = o.table("rksq")
    assert np.array_equal(after, ss * rksq)
    spec0, _ = o.spec1d(after, 0)
    assert np.array_equal(spec0, spec1)


@pytest.mark.parametrize("n", [32, 64, 128])
def test_tables_closed_form(oracle_mod, n):
    o = oracle_mod.Oracle(n)
    t = o.spec_tables()
    assert t["kmax"] == n // 2
    assert t["kmaxred"] == int(np.floor(n / 2 / np.sqrt(2.0) + 0.5))
    k1 = np.fft.fftfreq(n, 1.0 / n)
    K = np.floor(np.hypot(k1[:, None], k1[None, :]) / np.sqrt(2.0) + 0.5).astype(int)
    cnt = np.bincount(K.ravel(), minlength=n + 1)
    k = np.arange(1, t["kmax"] + 1)
    np.testing.assert_allclose(t["spmf"][k], 4 * np.pi / n ** 2 * k / cnt[k], rtol=1e-14)
    np.testing.assert_allclose(t["alk"][k], np.log10(np.sqrt(2.0) * k), rtol=1e-14)
