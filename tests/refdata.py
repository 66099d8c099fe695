"""Inputs the reference's own tests use, regenerated bit for bit.

rustymath's tests draw matrices with `random::<T>(m, n, seed)` (tests/linalg.rs:331-334):
successive SplitMix64 outputs from index `seed` (tests/support/mod.rs:5-25), each read as
rand's standard f64 (the top 53 bits times 2^-53), mapped to 2x-1."""
import numpy as np

_M = (1 << 64) - 1


def splitmix(i):
    z = ((i + 1) * 0x9E3779B97F4A7C15) & _M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M
    return z ^ (z >> 31)


def ref_random(m, n, seed):
    """The reference tests' `random::<f64>(m, n, seed)` as an m x n row-major array."""
    out = np.empty(m * n)
    for i in range(m * n):
        out[i] = 2.0 * ((splitmix(seed + i) >> 11) * 2.0 ** -53) - 1.0
    return out.reshape(m, n)


def norm(x):
    """tests/linalg.rs `norm`: the Frobenius norm."""
    return float(np.sqrt(np.sum(np.asarray(x, dtype=np.float64) ** 2)))


def distance(x, y, scale):
    return norm(np.asarray(x) - np.asarray(y)) / scale


def lower_of(factors):
    """Lu::lower for column-major factors (row j holds column j)."""
    n = factors.shape[0]
    t = factors.T
    return np.tril(t, -1) + np.eye(n)


def upper_of(factors):
    return np.triu(factors.T)
