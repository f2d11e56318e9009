"""Seeded initial conditions with the shapes of the benchmark configurations.

All arrays have shape (nk, nj, ni) (i fastest); x = (i+1/2)/ni pairs with i,
y with j, z with k.  The reference benchmarks on its analytic solution
(exactQ); the synthetic fields below are the stand-ins that the configuration
list names (no dataset is involved).
"""
import numpy as np


def centres(n):
    return (np.arange(n) + 0.5) / n


def gaussian_noise(ni, nj=None, nk=None, seed=0, sigma=0.1, amp=1e-3):
    """Gaussian bump (sigma, centred at 0.5^3, non-periodic distance) plus U(-amp, amp) noise."""
    nj = nj or ni
    nk = nk or ni
    z, y, x = np.meshgrid(centres(nk), centres(nj), centres(ni), indexing="ij")
    r2 = (x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2
    q = np.exp(-r2 / (2 * sigma ** 2))
    rng = np.random.default_rng(seed)
    return q + rng.uniform(-amp, amp, size=(nk, nj, ni))


def fourier_modes(ni, nj=None, nk=None, seed=1, modes=8):
    """Sum of `modes` sines, wavenumbers in {1..4}^3, N(0,1) amplitudes, U[0,2pi) phases."""
    nj = nj or ni
    nk = nk or ni
    rng = np.random.default_rng(seed)
    kv = rng.integers(1, 5, size=(modes, 3))
    a = rng.standard_normal(modes)
    phi = rng.uniform(0.0, 2 * np.pi, size=modes)
    z, y, x = np.meshgrid(centres(nk), centres(nj), centres(ni), indexing="ij")
    q = np.zeros((nk, nj, ni))
    for m in range(modes):
        q += a[m] * np.sin(2 * np.pi * (kv[m, 0] * x + kv[m, 1] * y + kv[m, 2] * z) + phi[m])
    return q


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
