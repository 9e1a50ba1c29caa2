"""The closure network's CPU restatement against finite differences of
itself (float64, no BF16 rounding): its transposed and weight-gradient
convolutions are the exact derivatives of its forward pass."""
import numpy as np

from oracle import closure_oracle as co


def test_oracle_gradient_matches_finite_differences():
    n = 12
    rng = np.random.default_rng(0)
    p = co.init_params(1).astype(np.float64)
    p += 0.05 * rng.standard_normal(p.size)  # non-zero biases too
    x = rng.standard_normal((co.NIN, n, n))
    dy = rng.standard_normal((co.NOUT, n, n))
    y, cache = co.forward(p, x, rounding=False)
    g = co.backward(p, cache, dy, rounding=False)
    assert g.shape == (co.param_count(),)
    idx = rng.choice(p.size, 40, replace=False)
    L = lambda q: float((co.forward(q, x, rounding=False)[0] * dy).sum())
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (L(p + e) - L(p - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 1e-30], np.float32)
    r = co.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0          # tie to even (down)
    assert r[2] == 1.0 + 2 ** -6                  # tie to even (up)
    assert r[3] == 1.0                            # below half
    assert r[4] == -2.5
    assert abs(r[5] - 1e-30) <= 1e-32


def test_pad_spectrum_carries_a_band_limited_field():
    """A field of wavenumbers up to the coarse Nyquist one, sampled on 16^2
    and on 64^2: the padded coarse spectrum is the fine spectrum."""
    from hydra_b200.synthetic import ptospc_np
    rng = np.random.default_rng(2)
    n, nf = 16, 64

    def field(m):
        x = -np.pi + 2 * np.pi * np.arange(m) / m
        X, Y = np.meshgrid(x, x, indexing="ij")  # [ix, iy]
        f = np.zeros((m, m))
        for kx in range(0, n // 2 + 1):
            for ky in range(0, n // 2 + 1):
                a, b, c, d = rng.standard_normal(4) if m == n else coef[(kx, ky)]
                coef.setdefault((kx, ky), (a, b, c, d))
                cx = [np.cos(kx * X)] + ([np.sin(kx * X)] if 0 < kx < n // 2 else [])
                cy = [np.cos(ky * Y)] + ([np.sin(ky * Y)] if 0 < ky < n // 2 else [])
                w = [a, b, c, d]
                t = 0
                for u in cx:
                    for v in cy:
                        f += w[t] * u * v
                        t += 1
        return f

    coef = {}
    fc = field(n)
    ff = field(nf)
    sc, sf = ptospc_np(fc), ptospc_np(ff)
    assert np.abs(co.pad_spectrum(sc, nf) - sf).max() <= 1e-12 * np.abs(sf).max()
