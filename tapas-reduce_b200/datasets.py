"""Seeded synthetic body sets for the N-body evaluation path.

The reference's example driver generates its own bodies
(``sample/exafmm-dev-13274dd4ac68/include/dataset.h:86-310``: "cube" on
[-pi,pi]^3, "sphere", "plummer", charges ``drand48()-0.5``).  The workloads
measured here are the ones stated for this project instead; all draw from a
counter-based SplitMix64 stream so that any (seed, stream, index) triple is
reproducible on any machine and in any order:

* ``uniform_cube``   - positions uniform in [-1,1]^3, charges U[0,1] scaled to sum 1.
* ``plummer``        - Plummer sphere, scale radius a (default 1): r = a / sqrt(U^(-2/3) - 1),
                       redrawn while r >= rmax (default 100), isotropic direction;
                       equal charges 1/N.  (No 3*pi/16 virial rescaling, unlike
                       the reference's dataset.h:209.)
* ``sphere_surface`` - uniform on the unit sphere surface (normalised Gaussian
                       triples), charges U[-1,1] minus their mean.
* ``two_gaussians``  - two isotropic Gaussian clusters, sigma 0.1, centres
                       (+-0.5, 0, 0), charges 1/N.

All arrays are float64, returned as (x, y, z, q).
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_SEEDMUL = np.uint64(0xD1B54A32D192ED03)
_STREAMMUL = np.uint64(0x8CB92BA72F3D8DD7)


def splitmix64(seed: int, stream: int, index: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser applied to a counter: one uint64 per index."""
    with np.errstate(over="ignore"):
        z = (np.uint64(seed & 0xFFFFFFFFFFFFFFFF) * _SEEDMUL
             + np.uint64(stream & 0xFFFFFFFFFFFFFFFF) * _STREAMMUL
             + (index.astype(np.uint64) + np.uint64(1)) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, stream: int, n: int, offset: int = 0) -> np.ndarray:
    """Open-interval uniforms in (0, 1): ((z >> 11) + 0.5) * 2^-53."""
    idx = np.arange(offset, offset + n, dtype=np.uint64)
    z = splitmix64(seed, stream, idx)
    return ((z >> np.uint64(11)).astype(np.float64) + 0.5) * (2.0 ** -53)


def uniform_cube(n: int, seed: int = 1):
    x = 2.0 * uniform01(seed, 1, n) - 1.0
    y = 2.0 * uniform01(seed, 2, n) - 1.0
    z = 2.0 * uniform01(seed, 3, n) - 1.0
    q = uniform01(seed, 4, n)
    q = q / q.sum()
    return x, y, z, q


def _isotropic(seed: int, n: int, s_cos: int, s_phi: int):
    ct = 2.0 * uniform01(seed, s_cos, n) - 1.0
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    ph = 2.0 * np.pi * uniform01(seed, s_phi, n)
    return st * np.cos(ph), st * np.sin(ph), ct


def plummer(n: int, seed: int = 2, a: float = 1.0, rmax: float = 100.0):
    r = np.empty(n)
    todo = np.arange(n)
    attempt = 0
    while todo.size:
        u = uniform01(seed, 1000 + attempt, n)[todo]
        rr = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        ok = rr < rmax
        r[todo[ok]] = rr[ok]
        todo = todo[~ok]
        attempt += 1
    ux, uy, uz = _isotropic(seed, n, 11, 12)
    q = np.full(n, 1.0 / n)
    return r * ux, r * uy, r * uz, q


def _gauss(seed: int, n: int, s1: int, s2: int):
    u1 = uniform01(seed, s1, n)
    u2 = uniform01(seed, s2, n)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def sphere_surface(n: int, seed: int = 5):
    gx = _gauss(seed, n, 21, 22)
    gy = _gauss(seed, n, 23, 24)
    gz = _gauss(seed, n, 25, 26)
    nr = np.sqrt(gx * gx + gy * gy + gz * gz)
    q = 2.0 * uniform01(seed, 27, n) - 1.0
    q = q - q.mean()
    return gx / nr, gy / nr, gz / nr, q


def two_gaussians(n: int, seed: int = 4, sigma: float = 0.1, sep: float = 1.0):
    side = np.where(uniform01(seed, 31, n) < 0.5, -0.5 * sep, 0.5 * sep)
    x = side + sigma * _gauss(seed, n, 32, 33)
    y = sigma * _gauss(seed, n, 34, 35)
    z = sigma * _gauss(seed, n, 36, 37)
    q = np.full(n, 1.0 / n)
    return x, y, z, q


DISTRIBUTIONS = {
    "uniform_cube": uniform_cube,
    "plummer": plummer,
    "sphere_surface": sphere_surface,
    "two_gaussians": two_gaussians,
}


def make(dist: str, n: int, seed: int | None = None):
    f = DISTRIBUTIONS[dist]
    return f(n) if seed is None else f(n, seed=seed)


def sample_targets(n: int, k: int, seed: int = 99) -> np.ndarray:
    """k distinct target indices drawn uniformly from range(n), sorted."""
    k = min(k, n)
    z = splitmix64(seed, 77, np.arange(n, dtype=np.uint64))
    return np.sort(np.argsort(z, kind="stable")[:k]).astype(np.int64)
