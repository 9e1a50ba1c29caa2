"""Seeded synthetic initial PV fields for the contour-advection workloads.

The field follows the structure of the reference's random-phase initial
condition (ca/plane/qg/init/ranpv.f90:38-117): a radial amplitude spectrum,
independent phases per (kx, ky) quadrant filled with the same cos/sin pattern
in the "Hermitian" spectral layout, a spectral-to-physical transform, then a
renormalisation.  The workloads fix the amplitude to k^3 exp(-(k/k0)^2) and
normalise the rms of q to 4 pi (ranpv normalises max|q| instead), with phases
drawn from numpy's PCG64 seeded generator in place of the GNU ``rand()``
stream, so that every run on every machine reads identical bytes.

Array convention (shared by the whole package): a physical field q(ny,nx) of
the Fortran code is a C-contiguous numpy array of shape (nx, ny) indexed
[ix-1, iy-1]; a spectral field s(nx,ny) is a (ny, nx) array indexed
[ky-1, kx-1].
"""
from __future__ import annotations

import numpy as np

__all__ = ["herm_forward", "herm_reverse", "ptospc_np", "spctop_np", "random_pv",
           "ensemble_member_params"]


def herm_forward(x: np.ndarray, axis: int) -> np.ndarray:
    """Real transform along ``axis`` in the stafft Hermitian layout
    (lib/stafft/stafft.f90:55-58,187-287): out[k] = Re F(k)/sqrt(n) for
    k <= n/2, out[n-k] = Im F(k)/sqrt(n) for 0 < k < n/2,
    F(k) = sum_j x_j exp(-2 pi i j k / n)."""
    x = np.moveaxis(np.asarray(x, np.float64), axis, 0)
    n = x.shape[0]
    F = np.fft.rfft(x, axis=0) / np.sqrt(n)
    out = np.empty_like(x)
    h = n // 2
    out[: h + 1] = F.real
    out[n - np.arange(1, h)] = F.imag[1:h]
    return np.moveaxis(out, 0, axis)


def herm_reverse(s: np.ndarray, axis: int) -> np.ndarray:
    """Exact inverse of :func:`herm_forward` (stafft.f90:290-406)."""
    s = np.moveaxis(np.asarray(s, np.float64), axis, 0)
    n = s.shape[0]
    h = n // 2
    F = np.zeros((h + 1,) + s.shape[1:], np.complex128)
    F.real = s[: h + 1]
    F.imag[1:h] = s[n - np.arange(1, h)]
    x = np.fft.irfft(F * np.sqrt(n), n=n, axis=0)
    return np.moveaxis(x, 0, axis)


def ptospc_np(q: np.ndarray) -> np.ndarray:
    """Physical (nx, ny) C array -> spectral (ny, nx) C array
    (lib/stafft/sta2dfft.f90:103-132)."""
    a = herm_forward(q, axis=0)        # along ix
    return herm_forward(a.T, axis=0)   # transpose, along iy


def spctop_np(s: np.ndarray) -> np.ndarray:
    """Spectral (ny, nx) C array -> physical (nx, ny) C array
    (lib/stafft/sta2dfft.f90:136-165)."""
    a = herm_reverse(s, axis=0)        # along ky
    return herm_reverse(a.T, axis=0)   # transpose, along kx


def random_pv(n: int, k0: float, seed: int, rms: float = 4.0 * np.pi,
              power: float = 3.0) -> np.ndarray:
    """Random-phase PV field on an n x n grid of [-pi, pi)^2.

    Amplitude |q_k| = k^power exp(-(k/k0)^2); phases filled in the
    quadrant pattern of ranpv.f90:51-111.  Returns the physical field as an
    (nx, ny) float64 array normalised to the given rms, with zero mean.
    """
    if n < 8 or n & (n - 1):
        raise ValueError("n must be a power of two >= 8")
    rng = np.random.Generator(np.random.PCG64(seed))
    nw = n // 2
    k = np.arange(nw + 1, dtype=np.float64)          # integer wavenumbers (L = 2 pi)
    K = np.sqrt(k[None, :] ** 2 + k[:, None] ** 2)   # [ky, kx]
    amp = K ** power * np.exp(-(K / k0) ** 2)
    s = np.zeros((n, n))                             # spectral, [ky-1, kx-1]
    two_pi = 2 * np.pi
    m = np.arange(2, nw + 1)                         # 2..nw
    mc = n + 2 - m                                   # conjugate (sine) index
    # interior quadrants (ranpv.f90:51-67); draws in (ky outer, kx inner, x then y) order
    r = rng.random((nw - 1, nw - 1, 2))
    phix = two_pi * r[..., 0] - np.pi
    phiy = two_pi * r[..., 1] - np.pi
    cx, sx, cy, sy = np.cos(phix), np.sin(phix), np.cos(phiy), np.sin(phiy)
    a = amp[1:nw, 1:nw]
    KY, KX = np.meshgrid(m, m, indexing="ij")
    KYC, KXC = np.meshgrid(mc, mc, indexing="ij")
    s[KY - 1, KX - 1] = a * cx * cy
    s[KY - 1, KXC - 1] = a * sx * cy
    s[KYC - 1, KX - 1] = a * cx * sy
    s[KYC - 1, KXC - 1] = a * sx * sy
    # ky = 1 row, kx = 1 column, Nyquist row and column (ranpv.f90:69-111)
    ph = two_pi * rng.random(nw - 1) - np.pi
    s[0, m - 1] = amp[0, 1:nw] * np.cos(ph); s[0, mc - 1] = amp[0, 1:nw] * np.sin(ph)
    ph = two_pi * rng.random(nw - 1) - np.pi
    s[m - 1, 0] = amp[1:nw, 0] * np.cos(ph); s[mc - 1, 0] = amp[1:nw, 0] * np.sin(ph)
    ph = two_pi * rng.random(nw - 1) - np.pi
    s[nw, m - 1] = amp[nw, 1:nw] * np.cos(ph); s[nw, mc - 1] = amp[nw, 1:nw] * np.sin(ph)
    ph = two_pi * rng.random(nw - 1) - np.pi
    s[m - 1, nw] = amp[1:nw, nw] * np.cos(ph); s[mc - 1, nw] = amp[1:nw, nw] * np.sin(ph)
    s[0, 0] = 0.0
    s[nw, nw] = 0.0
    q = spctop_np(s)
    q -= q.mean()
    q *= rms / np.sqrt(np.mean(q * q))
    return np.ascontiguousarray(q)


def ensemble_member_params(seed: int):
    """Per-member (k0, ncontq) of the batched ensemble workload: k0 uniform in
    [4, 12] and the level count uniform in [20, 60], drawn from the seed."""
    rng = np.random.Generator(np.random.PCG64(10_000 + seed))
    return float(rng.uniform(4.0, 12.0)), int(rng.integers(20, 61))
