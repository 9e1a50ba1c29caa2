"""CPU restatement of the learned velocity closure's network (numpy).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA network in
``hydra_b200/csrc/closure.cu``; nothing in the product imports it.  The
closure has no counterpart in the reference (Hydra corrects nothing: velint,
contours.f90:136-169, interpolates the coarse inversion bilinearly), so this
file restates the network the library defines, not a reference algorithm:

* four periodic 5x5 convolutions (cross-correlation: out[y, x] reads
  in[y + ky - 2, x + kx - 2], indices modulo n), NIN -> HID -> HID -> HID ->
  NOUT channels, GELU (0.5 x (1 + erf(x / sqrt 2))) after the first three;
* the output is the velocity correction on a grid SUB times as fine as n:
  channel comp*SUB^2 + a*SUB + b is component comp (u, v) at the fine point
  (SUB ix + a, SUB iy + b), interpolated bilinearly to the nodes on that grid
  (``node_correction``);
* parameters in the order W1[co][ci][ky][kx], b1, ..., W4, b4 (FP32);
* BF16 rounding (round to nearest even) wherever the GPU stores BF16: the
  input, the weights, every pre-activation and activation, the output
  gradient and every pre-activation gradient; sums in float64 here, FP32 on
  the tensor cores, so the two agree to accumulation order and occasional
  one-ulp BF16 flips.

Arrays are channel-major [C][n][n] with rows = ix and columns = iy, the
physical field order of the solver.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

HID = 16  # hidden channels
SUB = 2  # the output grid is SUB times as fine as the input
NOUT = 2 * SUB * SUB  # output channels
NIN = 12  # input channels: coarse PV, u, v, nine sub-cell level deviations
LAYERS = [(NIN, HID), (HID, HID), (HID, HID), (HID, NOUT)]


def param_count() -> int:
    return sum(co * ci * 25 + co for ci, co in LAYERS)


def split_params(p):
    """Flat parameters -> [(W[co][ci][5][5], b[co]), ...]."""
    out, o = [], 0
    for ci, co in LAYERS:
        w = np.asarray(p[o:o + co * ci * 25], np.float64).reshape(co, ci, 5, 5)
        o += co * ci * 25
        b = np.asarray(p[o:o + co], np.float64)
        o += co
        out.append((w, b))
    return out


def init_params(seed: int, gain: float = 1.0) -> np.ndarray:
    """He-style initial weights N(0, gain^2 * 2 / fan_in), zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co in LAYERS:
        parts.append(rng.standard_normal(co * ci * 25) * gain * np.sqrt(2.0 / (ci * 25)))
        parts.append(np.zeros(co))
    return np.concatenate(parts).astype(np.float32)


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def gelu(x):
    x = np.asarray(x, np.float64)
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_d(x):
    x = np.asarray(x, np.float64)
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def taps(x):
    """[C][n][n] -> [25][C][n][n], tap ky*5+kx holding x[c][y+ky-2][x+kx-2]."""
    return np.stack([np.roll(x, (-(ky - 2), -(kx - 2)), axis=(1, 2))
                     for ky in range(5) for kx in range(5)])


def conv(x, w, b):
    co, ci = w.shape[:2]
    return np.einsum("oit,tihw->ohw", w.reshape(co, ci, 25), taps(x), optimize=True) + b[:, None, None]


def conv_t(dz, w):
    """Gradient of conv's input: dx[ci][y][x] = sum W[co][ci][ky][kx] dz[co][y-ky+2][x-kx+2]."""
    co, ci = w.shape[:2]
    sh = np.stack([np.roll(dz, (ky - 2, kx - 2), axis=(1, 2)) for ky in range(5) for kx in range(5)])
    return np.einsum("oit,tohw->ihw", w.reshape(co, ci, 25), sh, optimize=True)


def conv_w(x, dz):
    """Gradient of conv's weights: dW[co][ci][tap] = sum dz[co] * taps(x)[tap][ci]."""
    return np.einsum("ohw,tihw->oit", dz, taps(x), optimize=True)


def forward(params, x, rounding=True):
    """Returns (y, cache).  x: [3][n][n]."""
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    L = split_params(params)
    a = r(x).astype(np.float64)
    cache = {"x0": a, "z": [], "a": []}
    for l in range(3):
        w, b = L[l]
        z = conv(a, r(w).astype(np.float64), b)
        zr = r(z).astype(np.float64)
        a = r(gelu(z)).astype(np.float64)
        cache["z"].append(zr)
        cache["a"].append(a)
    w, b = L[3]
    y = conv(a, r(w).astype(np.float64), b)
    return y, cache


def backward(params, cache, dy, rounding=True):
    """Flat gradient of sum(dy * y) with respect to the parameters."""
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    L = split_params(params)
    grads = [None] * 4
    dz = r(dy).astype(np.float64)
    ins = [cache["x0"]] + cache["a"]
    for l in range(3, -1, -1):
        w, _ = L[l]
        co, ci = w.shape[:2]
        dw = conv_w(ins[l], dz).reshape(co, ci, 5, 5)
        db = dz.sum(axis=(1, 2))
        grads[l] = (dw, db)
        if l == 0:
            break
        da = conv_t(dz, r(w).astype(np.float64))
        dz = r(da * gelu_d(cache["z"][l - 1])).astype(np.float64)
    return np.concatenate([np.concatenate([g[0].ravel(), g[1]]) for g in grads])


def pad_spectrum(s, nf):
    """Spectrum s (ny, nx) of an n x n grid in stafft's layout carried to an
    nf x nf grid: each wavenumber keeps its coefficient times sqrt(nf/n) per
    axis (sqrt(nf/n)/2 for the cosine at the coarse Nyquist wavenumber, a
    regular mode of the fine grid); wavenumbers the coarse grid lacks are 0.
    The judge's transfer of the non-contour PV, restated for the tests."""
    n = s.shape[0]
    out = np.zeros((nf, nf))
    r = np.sqrt(nf / n)

    def axis_map(m):
        idx, fac = [], []
        for i in range(m):
            sine = i > m // 2
            k = m - i if sine else i
            if k > n // 2 or (sine and k == n // 2):
                idx.append(-1); fac.append(0.0)
            else:
                idx.append(n - k if sine else k)
                fac.append(0.5 * r if k == n // 2 else r)
        return np.array(idx), np.array(fac)

    ix, fx = axis_map(nf)
    ok = ix >= 0
    sub = s[np.ix_(ix[ok], ix[ok])] * np.outer(fx[ok], fx[ok])
    out[np.ix_(np.nonzero(ok)[0], np.nonzero(ok)[0])] = sub
    return out


def node_correction(y, xq, yq, us, n, ell=2 * np.pi):
    """us times the bilinear interpolation of the output y ([NOUT][n][n]) on
    the SUB*n grid at the nodes (xq, yq) of the domain [-ell/2, ell/2)^2: fine
    point (I, J) is sub-cell (I % SUB, J % SUB) of coarse cell (I // SUB,
    J // SUB)."""
    m = SUB * n
    h = ell / m
    fx = (np.asarray(xq) + ell / 2) / h
    fy = (np.asarray(yq) + ell / 2) / h
    i0 = np.floor(fx).astype(np.int64)
    j0 = np.floor(fy).astype(np.int64)
    px, py = fx - i0, fy - j0
    i0 %= m
    j0 %= m
    i1, j1 = (i0 + 1) % m, (j0 + 1) % m
    y = np.asarray(y, np.float64)

    def at(comp, I, J):
        return y[comp * SUB * SUB + (I % SUB) * SUB + (J % SUB), I // SUB, J // SUB]

    out = []
    for comp in range(2):
        v = ((1 - px) * (1 - py) * at(comp, i0, j0) + px * (1 - py) * at(comp, i1, j0)
             + (1 - px) * py * at(comp, i0, j1) + px * py * at(comp, i1, j1))
        out.append(us * v)
    return out[0], out[1]


def subcell_features(levels, C, qjump, iq):
    """The network's sub-cell input channels 3..11 from the fine (4n) contour
    levels ([4n][4n], rows = fine x) and the coarse con2grid sums C ([n][n]):
    qjump (L(4cx + 2a - 2, 4cy + 2b - 2) - C/256) * iq, channel 3a + b."""
    nf = levels.shape[0]
    n = nf // 4
    cx = np.arange(n)[:, None]
    cy = np.arange(n)[None, :]
    out = []
    for a in range(3):
        for b in range(3):
            L = levels[(4 * cx + 2 * a - 2) % nf, (4 * cy + 2 * b - 2) % nf].astype(np.float64)
            out.append(qjump * (L - C.astype(np.float64) / 256.0) * iq)
    return np.stack(out)
