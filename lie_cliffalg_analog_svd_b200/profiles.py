"""Synthetic matrix generators.

``generate`` restates ``profiles::generate`` (src/lib.rs:230-319) and the named
test matrices of ``src/lie_svd_benchmarks.rs:106-300``.  The reference draws
from ``rand`` 0.8.7 ``StdRng`` (ChaCha12) + ``rand_distr`` 0.4.3; those streams
are not reproduced here.  Inputs come from numpy's PCG64 with a fixed seed and
the same distribution and construction (Gaussian entries; Haar orthogonal
factors by modified Gram-Schmidt of a Gaussian matrix, src/lib.rs:321-340;
``compose_from_svd`` src/lib.rs:342-345).  The same buffers are fed to the
oracle and to the CUDA library.

The ``*_workload`` functions build the benchmark inputs: uneven batches of
``Q1 diag(s) Q2^T``, large polar inputs, Phase-JADE families and the adjoint
batch.
"""
from __future__ import annotations

import numpy as np

PROFILES = ("uniform_random", "degenerate_spectrum", "extreme_ill_conditioned",
            "jordan_defective", "sparse_structured", "nearly_diagonal")


def random_orthogonal(n: int, rng: np.random.Generator) -> np.ndarray:
    """Haar-distributed orthogonal matrix: QR of a Gaussian with the sign fix
    (equal in distribution to MGS of a Gaussian, src/lib.rs:321-340)."""
    g = rng.standard_normal((n, n))
    q, r = np.linalg.qr(g)
    d = np.sign(np.diag(r))
    d[d == 0] = 1.0
    return q * d


def random_orthogonal_batch(b: int, n: int, rng: np.random.Generator) -> np.ndarray:
    g = rng.standard_normal((b, n, n))
    q, r = np.linalg.qr(g)
    d = np.sign(np.diagonal(r, axis1=1, axis2=2))
    d[d == 0] = 1.0
    return q * d[:, None, :]


def compose_from_svd(u, sigma, v):
    return (u * np.asarray(sigma)[None, :]) @ v.T


def generate(n: int, profile: str, seed: int):
    """Returns ``(a, sigma_ref or None)``; see src/lib.rs:230-319."""
    rng = np.random.default_rng(seed)
    if profile == "uniform_random":
        return rng.standard_normal((n, n)), None
    if profile == "degenerate_spectrum":
        u = random_orthogonal(n, rng)
        v = random_orthogonal(n, rng)
        s = np.array([100.0 if i < n // 8 else 50.0 if i < n // 4 else 1.0 if i < n // 2
                      else 1e-12 for i in range(n)])
        return compose_from_svd(u, s, v), s
    if profile == "extreme_ill_conditioned":
        u = random_orthogonal(n, rng)
        v = random_orthogonal(n, rng)
        denom = max(n - 1, 1)
        s = np.array([10.0 ** (-18.0 * i / denom) for i in range(n)])
        return compose_from_svd(u, s, v), s
    if profile == "jordan_defective":
        a = np.zeros((n, n))
        for i in range(n):
            a[i, i] = 1.0 - 0.5 * (i / max(n, 1))
            if i + 1 < n:
                a[i, i + 1] = 20.0
            if i + 2 < n and i % 4 == 0:
                a[i, i + 2] = -3.0
        return a, None
    if profile == "sparse_structured":
        a = np.zeros((n, n))
        for i in range(n):
            a[i, i] = 4.0 + (i % 7) * 0.25
            if i + 1 < n:
                a[i, i + 1] = -1.0
                a[i + 1, i] = 0.75
            if i + 8 < n:
                a[i, i + 8] = 0.15
                a[i + 8, i] = -0.10
        return a, None
    if profile == "nearly_diagonal":
        s = np.array([1.0 + (n - i) / n for i in range(n)])
        i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        a = 1e-6 * np.sin((i * 131 + j * 17).astype(np.float64))
        np.fill_diagonal(a, s)
        return a, s
    raise ValueError(f"unknown profile {profile!r}")


# Named matrices, src/lie_svd_benchmarks.rs:106-300.
def kahan_matrix(n: int, theta: float) -> np.ndarray:
    c, s = np.cos(theta), np.sin(theta)
    k = np.zeros((n, n))
    sp = 1.0
    for i in range(n):
        k[i, i] = sp
        k[i, i + 1:] = -c * sp
        sp *= s
    return k


def hilbert_matrix(n: int) -> np.ndarray:
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    return 1.0 / (i + j + 1)


def pei_matrix(n: int, alpha: float) -> np.ndarray:
    return np.ones((n, n)) + alpha * np.eye(n)


def pei_matrix_singular_values(n: int, alpha: float) -> np.ndarray:
    s = np.full(n, alpha)
    if n:
        s[-1] = alpha + n
    return s


def frank_matrix(n: int) -> np.ndarray:
    a = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            if j >= i:
                a[i, j] = n - j
            elif j + 1 == i:
                a[i, j] = n - i
    return a


def forsythe_matrix(n: int, lam: float, alpha: float) -> np.ndarray:
    a = lam * np.eye(n) + np.eye(n, k=1)
    if n > 0:
        a[n - 1, 0] = alpha if n > 1 else lam
    return a


def parter_matrix(n: int) -> np.ndarray:
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    return 1.0 / (i - j + 0.5)


def cauchy_matrix(n: int) -> np.ndarray:
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    return 1.0 / (i + j + 2.0)


def vandermonde_matrix(n: int) -> np.ndarray:
    x = np.arange(1, n + 1, dtype=np.float64)
    return x[:, None] ** np.arange(n)[None, :]


# ------------------------------------------------------------- workloads ----

def uneven_batch_workload(count: int, seed: int, n_lo: int = 2, n_hi: int = 64,
                          k_max: float = 12.0, degenerate_frac: float = 0.05):
    """Batched uneven SVD inputs: square f64 matrices with n ~ U{n_lo..n_hi},
    ``A = Q1 diag(s) Q2^T`` with Haar Q1, Q2 and ``s_i = 10^(-k i/(n-1))``,
    ``k ~ U[0, k_max]``; ``degenerate_frac`` of the matrices get one cluster
    of 2-4 repeated singular values.  Returns ``(ns int32[count],
    packed row-major A, packed sigma_ref)``."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_lo, n_hi + 1, size=count).astype(np.int32)
    ks = rng.uniform(0.0, k_max, size=count)
    degen = rng.uniform(size=count) < degenerate_frac
    a_off = np.zeros(count + 1, dtype=np.int64)
    a_off[1:] = np.cumsum(ns.astype(np.int64) ** 2)
    s_off = np.zeros(count + 1, dtype=np.int64)
    s_off[1:] = np.cumsum(ns)
    a = np.empty(int(a_off[-1]))
    sig = np.empty(int(s_off[-1]))
    for n in np.unique(ns):
        idx = np.nonzero(ns == n)[0]
        b = idx.size
        i = np.arange(n)
        s = 10.0 ** (-ks[idx, None] * i[None, :] / max(n - 1, 1))
        for t, mi in enumerate(idx):
            if degen[mi] and n >= 2:
                csize = int(rng.integers(2, min(4, n) + 1))
                start = int(rng.integers(0, n - csize + 1))
                s[t, start:start + csize] = s[t, start]
        s = -np.sort(-s, axis=1)
        q1 = random_orthogonal_batch(b, int(n), rng)
        q2 = random_orthogonal_batch(b, int(n), rng)
        mats = (q1 * s[:, None, :]) @ np.swapaxes(q2, 1, 2)
        for t, mi in enumerate(idx):
            a[a_off[mi]:a_off[mi + 1]] = mats[t].ravel()
            sig[s_off[mi]:s_off[mi + 1]] = s[t]
    return ns, a, sig


def conditioned_factors(m: int, n: int, kappa: float, seed: int):
    """``(Q1, s, Q2)``: Q1 m x k and Q2 n x k with orthonormal columns
    (k = min(m, n)), s geometric from 1 down to 1/kappa."""
    rng = np.random.default_rng(seed)
    k = min(m, n)
    s = kappa ** (-np.arange(k) / max(k - 1, 1))
    q1 = np.linalg.qr(rng.standard_normal((m, k)))[0]
    q2 = random_orthogonal(n, rng)[:, :k]
    return q1, s, q2


def conditioned_matrix(m: int, n: int, kappa: float, seed: int):
    """``Q1 diag(s) Q2^T`` with a geometric spectrum from 1 down to 1/kappa."""
    q1, s, q2 = conditioned_factors(m, n, kappa, seed)
    return (q1 * s[None, :]) @ q2.T, s


def jade_family_workload(families: int, K: int, n: int, eps: float, seed: int):
    """Phase-JADE families: ``A_k = Q diag(d_k) Q^T + eps E_k`` with Q Haar,
    d_k ~ N(0,1), E_k = (G+G^T)/2.  Returns (families, K, n, n) f64."""
    rng = np.random.default_rng(seed)
    out = np.empty((families, K, n, n))
    for f in range(families):
        q = random_orthogonal(n, rng)
        d = rng.standard_normal((K, n))
        fam = (q[None] * d[:, None, :]) @ q.T[None]
        if eps:
            g = rng.standard_normal((K, n, n))
            fam = fam + eps * 0.5 * (g + np.swapaxes(g, 1, 2))
        out[f] = fam
    return out


def adjoint_workload(count: int, m: int, n: int, seed: int, gap: float = 1e-3,
                     small_gap: float = 1e-6, small_gap_frac: float = 0.1):
    """Tall matrices with singular values uniform in [0.1, 10] and a minimum
    gap; ``small_gap_frac`` of them get one pair at ``small_gap``."""
    rng = np.random.default_rng(seed)
    a = np.empty((count, m, n))
    sig = np.empty((count, n))
    for t in range(count):
        while True:
            s = np.sort(rng.uniform(0.1, 10.0, size=n))[::-1]
            if np.min(-np.diff(s)) >= gap:
                break
        if rng.uniform() < small_gap_frac:
            j = int(rng.integers(0, n - 1))
            s[j + 1] = s[j] - small_gap
            s = np.sort(s)[::-1]
        q1 = np.linalg.qr(rng.standard_normal((m, n)))[0]
        q2 = random_orthogonal(n, rng)
        a[t] = (q1 * s[None, :]) @ q2.T
        sig[t] = s
    return a, sig


def bss_workload(channels: int, samples: int, seed: int, noise: float = 0.05):
    """Phase-BSS input: one sinusoid per source at 0.03 .. 0.43 cycles per
    sample (distinct lagged autocorrelations), plus Gaussian noise, mixed by
    I + 0.1 G.  Returns (sources, mixing, observations = mixing @ sources)."""
    rng = np.random.default_rng(seed)
    t = np.arange(samples, dtype=np.float64)
    src = np.empty((channels, samples))
    for k in range(channels):
        src[k] = np.sin(2 * np.pi * (0.03 + 0.4 * k / channels) * t + k) * (1 + 0.1 * k)
    src += noise * rng.standard_normal(src.shape)
    mix = np.eye(channels) + 0.1 * rng.standard_normal((channels, channels))
    return src, mix, mix @ src
