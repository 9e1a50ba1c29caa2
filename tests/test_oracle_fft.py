"""The oracle's FFT restates stafft's Hermitian layout and normalisation.

Known answers below are read off the reference's radix routines for the
lengths that reduce to one butterfly (lib/stafft/stafft.f90: forrdx4 k=0
branch lines 910-918, forrdx2 lines 1094-1097), times the 1/sqrt(n)
normalisation of forfft (stafft.f90:275).
"""
import numpy as np
import pytest

from hydra_b200.synthetic import herm_forward, herm_reverse, ptospc_np, spctop_np


def test_length4_known_answer(oracle_mod):
    # forrdx4, lv = 1: b0 = a0+a1+a2+a3, b1 = a0-a2, b2 = a0-a1+a2-a3, b3 = a3-a1
    a = np.array([[1.0], [2.0], [4.0], [8.0]])
    out = oracle_mod.forfft(a).ravel() * np.sqrt(4.0)
    np.testing.assert_allclose(out, [15.0, -3.0, -5.0, 6.0], rtol=0, atol=1e-14)


def test_layout_matches_numpy_formula(oracle_mod):
    rng = np.random.default_rng(1)
    for n in (8, 16, 64, 256):
        x = rng.standard_normal((n, 5))
        np.testing.assert_allclose(oracle_mod.forfft(x), herm_forward(x, 0), atol=1e-13)


def test_round_trip(oracle_mod):
    rng = np.random.default_rng(2)
    for n in (8, 32, 128, 1024):
        x = rng.standard_normal((n, 3))
        np.testing.assert_allclose(oracle_mod.revfft(oracle_mod.forfft(x)), x, atol=1e-12)
        np.testing.assert_allclose(herm_reverse(herm_forward(x, 0), 0), x, atol=1e-12)


def test_single_modes(oracle_mod):
    # cos(2 pi m j/n) -> X[m] = sqrt(n)/2 ; sin(2 pi m j/n) -> X[n-m] = -sqrt(n)/2
    n, m = 32, 5
    j = np.arange(n)
    c = oracle_mod.forfft(np.cos(2 * np.pi * m * j / n)[:, None]).ravel()
    s = oracle_mod.forfft(np.sin(2 * np.pi * m * j / n)[:, None]).ravel()
    assert abs(c[m] - np.sqrt(n) / 2) < 1e-13
    assert abs(s[n - m] + np.sqrt(n) / 2) < 1e-13
    c[m] = 0.0
    s[n - m] = 0.0
    assert np.abs(c).max() < 1e-13 and np.abs(s).max() < 1e-13


def test_2d_transforms(oracle_mod):
    o = oracle_mod.Oracle(32, ncontq=10)
    rng = np.random.default_rng(3)
    q = rng.standard_normal((32, 32))
    s = o.ptospc(q)
    np.testing.assert_allclose(s, ptospc_np(q), atol=1e-12)
    np.testing.assert_allclose(o.spctop(s), q, atol=1e-12)
    np.testing.assert_allclose(spctop_np(s), q, atol=1e-12)
