"""Seeded synthetic bound-constrained problems (inputs for tests, smoke and bench).

The problem family: on an s x s grid (k = j*s + i, i fast, h = 1/(s+1), zero Dirichlet
neighbours)

    f(x) = sum_k 0.5*kappa_k*((x_{i+1,j}-x_k)^2 + (x_{i,j+1}-x_k)^2)
         + h^2 * sum_k [w_k*softplus(x_k - t_k) - b_k*x_k + 0.05*cos(3*x_k)]

with kappa ~ U[0.5, 2], w ~ U[0, 1], t ~ N(0, 1), b ~ N(0, 4) (variance 4, sigma 2), bounds
l = -1, u = 1, and nbd drawn per variable: 2 with probability 0.8, 1 with 0.1, 0 with 0.1.
The reference library ships no such objective (its example is MINPACK-2 dsscfg); this
generator is glue for its parity and benchmark runs.

Every field is a pure function of (seed, field id, k) built only from integer arithmetic
and correctly rounded IEEE operations (+, -, *, /, sqrt, frexp/ldexp): normals come from
the Marsaglia polar method with a series logarithm, so the same seed gives bit-identical
inputs on any IEEE-754 machine, here and on the GPU host.
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
FIELD_KAPPA, FIELD_W, FIELD_T, FIELD_B, FIELD_NBD = 1, 2, 3, 4, 5


def _mix64(z: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser on a uint64 array (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _stream_base(seed: int, field: int) -> np.uint64:
    with np.errstate(over="ignore"):
        key = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) ^ (
            np.uint64(field) * np.uint64(0xD1B54A32D192ED03))
    return _mix64(np.array([key], dtype=np.uint64))[0]


def _uniform(base: np.uint64, k: np.ndarray, draw: int) -> np.ndarray:
    """U[0,1) doubles: top 53 bits of mix64(base + 64*k + draw)."""
    with np.errstate(over="ignore"):
        z = _mix64(base + (k.astype(np.uint64) << np.uint64(6)) + np.uint64(draw))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _log_exact_ops(x: np.ndarray) -> np.ndarray:
    """ln(x) for x > 0 from frexp and the atanh series, exact IEEE operations only."""
    m, e = np.frexp(x)  # x = m * 2**e, m in [0.5, 1)
    adj = m < 0.7071067811865476
    m = np.where(adj, m * 2.0, m)
    e = np.where(adj, e - 1, e).astype(np.float64)
    z = (m - 1.0) / (m + 1.0)  # |z| <= 0.1716
    z2 = z * z
    acc = np.zeros_like(z)
    for odd in range(27, 1, -2):  # Horner in z^2 for sum z^(2j+1)/(2j+1)
        acc = acc * z2 + (1.0 / odd)
    acc = acc * z2 + 1.0
    return e * 0.6931471805599453 + 2.0 * z * acc


def _normal(base: np.uint64, k: np.ndarray) -> np.ndarray:
    """N(0,1) by the Marsaglia polar method, up to 32 attempts per element."""
    out = np.zeros(k.shape, dtype=np.float64)
    pending = np.ones(k.shape, dtype=bool)
    for attempt in range(32):
        idx = np.nonzero(pending)[0]
        if idx.size == 0:
            break
        kk = k[idx]
        u = 2.0 * _uniform(base, kk, 2 * attempt) - 1.0
        v = 2.0 * _uniform(base, kk, 2 * attempt + 1) - 1.0
        s = u * u + v * v
        ok = (s > 0.0) & (s < 1.0)
        sel = idx[ok]
        so = s[ok]
        out[sel] = u[ok] * np.sqrt(-2.0 * _log_exact_ops(so) / so)
        pending[sel] = False
    return out


def synth_problem(s: int, seed: int = 0, nbd_mix: bool = True):
    """Fields and bounds of one instance on an s x s grid.

    Returns a dict of float64 arrays kappa, w, t, b, l, u (length s*s), int32 nbd, and
    the grid side s.  With nbd_mix=False every variable is boxed (nbd = 2)."""
    n = s * s
    k = np.arange(n, dtype=np.uint64)
    kappa = 0.5 + 1.5 * _uniform(_stream_base(seed, FIELD_KAPPA), k, 0)
    w = _uniform(_stream_base(seed, FIELD_W), k, 0)
    t = _normal(_stream_base(seed, FIELD_T), k)
    b = 2.0 * _normal(_stream_base(seed, FIELD_B), k)
    if nbd_mix:
        r = _uniform(_stream_base(seed, FIELD_NBD), k, 0)
        nbd = np.where(r < 0.8, 2, np.where(r < 0.9, 1, 0)).astype(np.int32)
    else:
        nbd = np.full(n, 2, dtype=np.int32)
    l = np.full(n, -1.0)
    u = np.full(n, 1.0)
    return {"s": s, "kappa": kappa, "w": w, "t": t, "b": b, "l": l, "u": u, "nbd": nbd}


def grid_side_log_uniform(seed: int, count: int, lo: int, hi: int) -> np.ndarray:
    """Grid sides drawn log-uniform on [lo, hi] (rounded), one per instance."""
    r = _uniform(_stream_base(seed, 99), np.arange(count, dtype=np.uint64), 0)
    ln_lo = float(_log_exact_ops(np.array([float(lo)]))[0])
    ln_hi = float(_log_exact_ops(np.array([float(hi)]))[0])
    return np.rint(np.exp(ln_lo + r * (ln_hi - ln_lo))).astype(np.int64)
