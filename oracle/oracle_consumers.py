"""Oracle restatement of the consumers of the exact solvers: Phase-BSS
(src/lie_svd_bss.rs) and the canonical-order wrappers of the phase normalizer
(src/phase_normalizer.rs:103-340).

TEST INFRASTRUCTURE ONLY, like the rest of ``oracle/``: the checker for
``lie_cliffalg_analog_svd_b200.consumers``.  Every step follows the reference
in its own order: the solves are the oracle's ``LieSvdSmall`` /
``LieSvdJoint`` (C++ restatements), the products the oracle's ``dot``
(ndarray's sequential product order), the lagged covariances the C++ loop
``oracle_lagged_covariance`` (the reference's t, i, j order), the other
per-entry loops numpy statements with the same operation order per entry."""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

import oracle as O


# ------------------------------------------------------------------ Phase-BSS
@dataclass
class PhaseBssParams:
    """``PhaseBssParams`` (src/lie_svd_bss.rs:12-33)."""
    lags: list = field(default_factory=lambda: [1, 2, 3, 5])
    eps: float = 1e-10
    joint: O.JointDiagonalizationParams = None

    @staticmethod
    def for_channels(channels: int) -> "PhaseBssParams":
        return PhaseBssParams([1, 2, 3, 5], 1e-10, O.JointDiagonalizationParams.for_n(channels))


@dataclass
class PhaseBssTrace:
    channels: int
    samples: int
    covariance_floor: float
    joint_initial_offdiag: float
    joint_final_offdiag: float
    joint_rotations: int
    mean_channel_coherence: float


@dataclass
class PhaseBssResult:
    unmixing: np.ndarray
    separated: np.ndarray
    channel_coherence: np.ndarray
    trace: PhaseBssTrace


def center_channels(x):
    """src/lie_svd_bss.rs:161-170: per-channel mean (sequential sum / T)."""
    x = np.asarray(x, dtype=np.float64)
    out = x.copy()
    for i in range(out.shape[0]):
        mean = np.cumsum(out[i])[-1] / out.shape[1]
        out[i] -= mean
    return out


def lagged_covariances(x, lags):
    """src/lie_svd_bss.rs:172-195: per lag, C += x[:, t+lag] x[:, t]^T / (T - lag)
    term by term (each product divided, then added), symmetrised -- the C++
    oracle's loop in the reference's order; lags 0 and >= T are skipped, and
    with none left the plain covariance x x^T / T stands in."""
    ch, t_len = x.shape
    out = []
    for lag in lags:
        if lag == 0 or lag >= t_len:
            continue
        out.append(O.lagged_covariance(x, lag))
    if not out:
        out.append(O.dot(x, x.T.copy()) / t_len)
    return out


def channel_phase_coherence(ch):
    """src/lie_svd_bss.rs:103-127."""
    ch = np.asarray(ch, dtype=np.float64)
    n, s = ch.shape
    out = np.zeros(n)
    if s <= 1:
        return out
    for i in range(n):
        x = ch[i]
        y = np.roll(x, -1)
        norm = np.cumsum(x * x)[-1]
        delay = np.cumsum(x * y)[-1]
        grad = np.cumsum((y - x) * (y - x))[-1]
        lock = abs(delay) / max(norm, 1e-300)
        smooth = 1.0 / (1.0 + np.sqrt(grad / max(norm, 1e-300)))
        out[i] = min(max(0.5 * lock + 0.5 * smooth, 0.0), 1.0)
    return out


def absolute_correlation_matrix(a, b):
    """src/lie_svd_bss.rs:197-214."""
    n = min(a.shape[0], b.shape[0])
    s = min(a.shape[1], b.shape[1])
    c = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            x, y = a[i, :s], b[j, :s]
            d = np.cumsum(x * y)[-1]
            na = np.cumsum(x * x)[-1]
            nb = np.cumsum(y * y)[-1]
            c[i, j] = abs(d) / max(np.sqrt(na) * np.sqrt(nb), 1e-300)
    return c


def estimate_sir_db(reference, separated) -> float:
    """src/lie_svd_bss.rs:129-159: greedy matching of |correlation|, signal =
    matched squares, interference = the other rows' squares in each matched column."""
    n = min(reference.shape[0], separated.shape[0])
    if n == 0:
        return 0.0
    corr = absolute_correlation_matrix(reference, separated)
    used_r, used_s = [False] * n, [False] * n
    sig = inter = 0.0
    for _ in range(n):
        best = (0, 0, -1.0)
        for i in range(n):
            if used_r[i]:
                continue
            for j in range(n):
                if not used_s[j] and corr[i, j] > best[2]:
                    best = (i, j, corr[i, j])
        used_r[best[0]] = used_s[best[1]] = True
        sig += best[2] * best[2]
        for i in range(n):
            if i != best[0]:
                inter += corr[i, best[1]] * corr[i, best[1]]
    return 10.0 * np.log10(sig / max(inter, 1e-12))


def bss_separate(observations, params: PhaseBssParams | None = None) -> PhaseBssResult:
    """``LieSvdBss::separate`` (src/lie_svd_bss.rs:57-100)."""
    x = np.asarray(observations, dtype=np.float64)
    ch, s = x.shape
    assert ch > 0 and s > 1, "PhaseBSS: empty observations"
    params = params or PhaseBssParams.for_channels(ch)
    xc = center_channels(x)
    cov = O.dot(xc, xc.T.copy()) / s
    u, sigma, _ = O.LieSvdSmall.solve(cov)
    floor = params.eps * max(max(float(sigma.max()), 0.0), 1.0)
    inv = 1.0 / np.sqrt(np.maximum(sigma, floor))
    w = inv[:, None] * u.T
    wh = O.dot(w, xc)
    lagged = lagged_covariances(wh, params.lags)
    basis, _, tr = O.LieSvdJoint.diagonalize_symmetric_with_params(lagged, params.joint)
    sep = O.dot(basis.T.copy(), wh)
    unmix = O.dot(basis.T.copy(), w)
    coh = channel_phase_coherence(sep)
    return PhaseBssResult(unmix, sep, coh, PhaseBssTrace(ch, s, floor, tr.initial_offdiag, tr.final_offdiag,
                                                         tr.rotations, float(coh.sum() / max(len(coh), 1))))


# ---------------------------------------------------------- phase normalizer
def row_wedge_capacity_from_gram(g):
    """src/phase_normalizer.rs:113-126: Omega_i = sum over j != i of
    sqrt(max(G_ii G_jj - G_ij^2, 0)), in j order."""
    n = g.shape[0]
    om = np.zeros(n)
    for i in range(n):
        for j in range(n):
            if i != j:
                om[i] += np.sqrt(max(g[i, i] * g[j, j] - g[i, j] * g[i, j], 0.0))
    return om


def row_leverage_scores(a):
    """src/phase_normalizer.rs:131-137: squared row norms of U from solve_rectangular."""
    u, _, _ = O.LieSvdSmall.solve_rectangular(a)
    return np.array([np.cumsum(u[i] * u[i])[-1] for i in range(u.shape[0])])


def canonical_row_scores(a):
    """src/phase_normalizer.rs:139-145: S_i = G_ii (1 + Omega_i) h_i, G = a a^T."""
    a = np.asarray(a, dtype=np.float64)
    g = O.dot(a, a.T.copy())
    om = row_wedge_capacity_from_gram(g)
    h = row_leverage_scores(a)
    return np.array([g[i, i] * (1.0 + om[i]) * h[i] for i in range(a.shape[0])])


def canonical_column_scores(a):
    return canonical_row_scores(np.asarray(a, dtype=np.float64).T.copy())


def order_from_scores(scores):
    """src/phase_normalizer.rs:182-200: descending, ties by original index."""
    n = len(scores)
    return sorted(range(n), key=lambda i: (-scores[i], i))


def canonical_family_order(matrices):
    """src/phase_normalizer.rs:253-279: one order from the summed row scores."""
    total = np.zeros(np.asarray(matrices[0]).shape[0])
    for m in matrices:
        total = total + canonical_row_scores(m)
    return order_from_scores(total), total


def solve_canonicalized(a):
    """src/phase_normalizer.rs:295-309: (U, sigma, Vt, row_order, col_order)."""
    a = np.asarray(a, dtype=np.float64)
    ro = order_from_scores(canonical_row_scores(a))
    co = order_from_scores(canonical_column_scores(a))
    u, s, vt = O.LieSvdSmall.solve_rectangular(a[np.ix_(ro, co)])
    inv_r, inv_c = np.argsort(ro), np.argsort(co)
    return u[inv_r], s, vt[:, inv_c], ro, co


def diagonalize_symmetric_canonicalized(matrices):
    """src/phase_normalizer.rs:326-340: (basis, diagonals, trace, order)."""
    order, _ = canonical_family_order(matrices)
    canon = [np.asarray(m, dtype=np.float64)[np.ix_(order, order)] for m in matrices]
    v, d, tr = O.LieSvdJoint.diagonalize_symmetric(canon)
    return v[np.argsort(order)], d, tr, order
