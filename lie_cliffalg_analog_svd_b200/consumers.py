"""Consumers of the exact solvers, on the GPU: Phase-BSS (``LieSvdBss``,
src/lie_svd_bss.rs) and the phase normalizer's canonical-order wrappers
(src/phase_normalizer.rs:103-340).

Device work: every product -- channel means, covariance, whitening, lagged
covariances, separation, unmixing, the coherence sums, row Gram matrices --
runs on the library's FP64 product kernel (``lsvd_gemm_f64``, which splits
a long inner dimension across the SMs), and every solve on ``LieSvdSmall``
(covariance SVD), ``LieSvdSmall.solve_rectangular`` (leverage scores, the
canonical solve) or Phase-JADE.  Host work is channels x channels glue: the
whitening matrix from the covariance's SVD, symmetrising the lagged
covariances, the wedge capacities of a Gram matrix, the permutation
bookkeeping.  The reference's evaluation helpers (``channel_phase_coherence``,
``estimate_sir_db``) are also provided for host arrays."""
from __future__ import annotations

import os
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .api import (Context, JointDiagonalizationParams, JointDiagonalizationTrace, LieSvdJoint, LieSvdSmall,
                  default_context, gemm_f64)


def _even(rows: int, cols: int, device):
    """A zeroed rows x cols float64 device view whose row stride is even
    (the product kernel's leading-dimension rule), starting 16-byte aligned."""
    import torch
    buf = torch.zeros((max(rows, 1), cols + (cols & 1)), dtype=torch.float64, device=device)
    return buf[:rows, :cols]


def _to_dev(a: np.ndarray, device):
    import torch
    t = _even(a.shape[0], a.shape[1], device)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)))
    return t


def _host(t) -> np.ndarray:
    return np.ascontiguousarray(t.cpu().numpy())


_tls = threading.local()


def _staging(elems: int):
    """This thread's grow-only page-locked float64 staging buffer (torch CPU
    tensor) of at least ``elems`` elements: large copies go host array ->
    staging -> device (and back) at DMA speed instead of through pageable memory."""
    import torch
    buf = getattr(_tls, "staging", None)
    if buf is None or buf.numel() < elems:
        buf = _tls.staging = None
        buf = _tls.staging = torch.empty(max(elems, 1), dtype=torch.float64, pin_memory=True)
    return buf


_STAGE_CHUNKS = 8
_copy_pool = None
_copy_pool_lock = threading.Lock()


def _copier():
    """Process-wide thread pool for the host side of the staged copies
    (numpy's copy releases the GIL, so the chunks copy in parallel)."""
    global _copy_pool
    with _copy_pool_lock:
        if _copy_pool is None:
            from concurrent.futures import ThreadPoolExecutor
            _copy_pool = ThreadPoolExecutor(max_workers=max(1, min(_STAGE_CHUNKS, os.cpu_count() or 1)))
        return _copy_pool


def _row_chunks(rows: int):
    step = max(1, -(-rows // _STAGE_CHUNKS))
    return [(r, min(rows, r + step)) for r in range(0, rows, step)]


def _to_dev_staged(a: np.ndarray, device):
    """``_to_dev`` of a large host array through the staging buffer, in row
    chunks copied into it by a thread pool; each chunk's DMA is issued as soon
    as its host copy is done, beside the copies still running."""
    import torch
    rows, cols = a.shape
    try:
        st = _staging(a.size)[:a.size].view(rows, cols)
    except RuntimeError:  # page-locked memory exhausted: copy straight from the pageable array
        return _to_dev(a, device)
    sn = st.numpy()
    t = _even(rows, cols, device)
    chunks = _row_chunks(rows)
    jobs = [_copier().submit(np.copyto, sn[r0:r1], a[r0:r1]) for r0, r1 in chunks]
    for (r0, r1), job in zip(chunks, jobs):
        job.result()
        t[r0:r1].copy_(st[r0:r1], non_blocking=True)
    torch.cuda.current_stream(device).synchronize()
    return t


def _host_staged(t) -> np.ndarray:
    """``_host`` of a large device view through the staging buffer, in row
    chunks: every chunk's DMA is enqueued at once, and each is copied out by
    the thread pool as soon as its event has completed."""
    import torch
    rows, cols = t.shape
    try:
        st = _staging(rows * cols)[:rows * cols].view(rows, cols)
    except RuntimeError:  # page-locked memory exhausted: copy straight into pageable memory
        return _host(t)
    sn = st.numpy()
    out = np.empty((rows, cols))
    stream = torch.cuda.current_stream(t.device)
    done = []
    for r0, r1 in _row_chunks(rows):
        st[r0:r1].copy_(t[r0:r1], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(stream)
        done.append((r0, r1, ev))
    jobs = []
    for r0, r1, ev in done:
        ev.synchronize()
        jobs.append(_copier().submit(np.copyto, out[r0:r1], sn[r0:r1]))
    for job in jobs:
        job.result()
    return out


def _device(ctx: Context):
    import torch
    return torch.device("cuda", ctx.device)


# ------------------------------------------------------------------ Phase-BSS
@dataclass
class PhaseBssParams:
    """``PhaseBssParams`` (src/lie_svd_bss.rs:12-33)."""
    lags: list = field(default_factory=lambda: [1, 2, 3, 5])
    eps: float = 1e-10
    joint: JointDiagonalizationParams = field(default_factory=lambda: JointDiagonalizationParams.for_n(4))

    @staticmethod
    def for_channels(channels: int) -> "PhaseBssParams":
        return PhaseBssParams([1, 2, 3, 5], 1e-10, JointDiagonalizationParams.for_n(channels))


@dataclass
class PhaseBssTrace:
    """``PhaseBssTrace`` (src/lie_svd_bss.rs:35-44)."""
    channels: int
    samples: int
    covariance_floor: float
    joint_initial_offdiag: float
    joint_final_offdiag: float
    joint_rotations: int
    mean_channel_coherence: float


@dataclass
class PhaseBssResult:
    """``PhaseBssResult`` (src/lie_svd_bss.rs:46-52)."""
    unmixing: np.ndarray
    separated: np.ndarray
    channel_coherence: np.ndarray
    trace: PhaseBssTrace


def channel_phase_coherence(channels) -> np.ndarray:
    """src/lie_svd_bss.rs:103-127: per channel, half the lag-1 circular
    autocorrelation magnitude plus half 1 / (1 + relative gradient norm)."""
    x = np.asarray(channels, dtype=np.float64)
    if x.shape[1] <= 1:
        return np.zeros(x.shape[0])
    y = np.roll(x, -1, axis=1)
    norm = np.maximum(np.sum(x * x, axis=1), 1e-300)
    lock = np.abs(np.sum(x * y, axis=1)) / norm
    smooth = 1.0 / (1.0 + np.sqrt(np.sum((y - x) ** 2, axis=1) / norm))
    return np.clip(0.5 * lock + 0.5 * smooth, 0.0, 1.0)


def _coherence_on_device(S, ctx: Context) -> np.ndarray:
    """``channel_phase_coherence`` of the device rows ``S`` (channels x T,
    T >= 2) from two products on the device: sum x_t^2 = diag(S S^T) and the
    circular lag-1 sum x_t x_(t+1 mod T) = diag(S_(+1) S^T) plus the wrap-around
    term; the gradient norm is 2 (sum x^2 - sum x x_(+1)) since the circular
    shift keeps sum y^2 = sum x^2."""
    ch, s = S.shape
    g0 = _host(gemm_f64(S, S, trans_b=True, c=_even(ch, ch, S.device), ctx=ctx))
    ahead = _even(ch, s - 1, S.device)
    ahead.copy_(S[:, 1:])
    g1 = _host(gemm_f64(ahead, S[:, :s - 1], trans_b=True, c=_even(ch, ch, S.device), ctx=ctx))
    ends = _host(S[:, [0, s - 1]])
    norm = np.diag(g0).copy()
    delay = np.diag(g1) + ends[:, 0] * ends[:, 1]
    n = np.maximum(norm, 1e-300)
    grad = np.maximum(2.0 * (norm - delay), 0.0)
    return np.clip(0.5 * np.abs(delay) / n + 0.5 / (1.0 + np.sqrt(grad / n)), 0.0, 1.0)


def estimate_sir_db(reference, separated) -> float:
    """src/lie_svd_bss.rs:129-159: greedy matching on the absolute
    correlation matrix; signal-to-interference ratio in dB."""
    a, b = np.asarray(reference, dtype=np.float64), np.asarray(separated, dtype=np.float64)
    n, s = min(a.shape[0], b.shape[0]), min(a.shape[1], b.shape[1])
    if n == 0:
        return 0.0
    a, b = a[:n, :s], b[:n, :s]
    corr = np.abs(a @ b.T) / np.maximum(np.outer(np.linalg.norm(a, axis=1), np.linalg.norm(b, axis=1)), 1e-300)
    used_r, used_s = np.zeros(n, bool), np.zeros(n, bool)
    sig = inter = 0.0
    for _ in range(n):
        masked = np.where(used_r[:, None] | used_s[None, :], -1.0, corr)
        i, j = np.unravel_index(int(np.argmax(masked)), masked.shape)  # first maximum in (i, j) order
        used_r[i] = used_s[j] = True
        sig += corr[i, j] ** 2
        inter += float(np.sum(np.delete(corr[:, j], i) ** 2))
    return float(10.0 * np.log10(sig / max(inter, 1e-12)))


class LieSvdBss:
    """``LieSvdBss`` (src/lie_svd_bss.rs:54-101)."""

    @staticmethod
    def separate(observations, params: PhaseBssParams | None = None, ctx: Context | None = None) -> PhaseBssResult:
        """Separates ``channels x samples`` observations: centre, whiten by
        the covariance's SVD, jointly diagonalise the lagged covariances of
        the whitened channels (Phase-JADE), rotate."""
        ctx = ctx or default_context()
        x = np.asarray(observations, dtype=np.float64)
        if x.ndim != 2 or x.shape[0] == 0 or x.shape[1] <= 1:
            raise L.LsvdError(L.BAD_SHAPE, "PhaseBSS: empty observations")
        ch, s = x.shape
        params = params or PhaseBssParams.for_channels(ch)
        dev = _device(ctx)
        X = _to_dev_staged(x, dev)
        # channel means (X 1 / T, as X E^T with E = [1^T; 0^T]: a narrow output over
        # the long sample axis) and X <- X - mean 1^T (E again, the inner
        # dimension padded to 2), both on the product kernel
        ones = _even(2, s, dev)
        ones[0, :] = 1.0
        mean = gemm_f64(X, ones, trans_b=True, alpha=1.0 / s, c=_even(ch, 2, dev), ctx=ctx)
        gemm_f64(mean, ones, alpha=-1.0, beta=1.0, c=X, ctx=ctx)
        cov = _host(gemm_f64(X, X, trans_b=True, alpha=1.0 / s, c=_even(ch, ch, dev), ctx=ctx))
        u, sigma, _ = LieSvdSmall.solve(cov, ctx=ctx)
        floor = params.eps * max(float(np.max(sigma)), 0.0, 1.0)
        w = (1.0 / np.sqrt(np.maximum(sigma, floor)))[:, None] * u.T
        W = _to_dev(w, dev)
        Wh = gemm_f64(W, X, c=_even(ch, s, dev), ctx=ctx)
        lagged = []
        for lag in params.lags:
            if lag == 0 or lag >= s:
                continue
            m = s - lag
            ahead = _even(ch, m, dev)
            ahead.copy_(Wh[:, lag:])  # a lag-offset view would start off the 16-byte boundary
            c = _host(gemm_f64(ahead, Wh[:, :m], trans_b=True, alpha=1.0 / m, c=_even(ch, ch, dev), ctx=ctx))
            lagged.append(0.5 * (c + c.T))
        if not lagged:
            lagged.append(_host(gemm_f64(Wh, Wh, trans_b=True, alpha=1.0 / s, c=_even(ch, ch, dev), ctx=ctx)))
        basis, _, tr = LieSvdJoint.diagonalize_symmetric_with_params(lagged, params.joint, ctx=ctx)
        V = _to_dev(basis, dev)
        Sep = gemm_f64(V, Wh, trans_a=True, c=_even(ch, s, dev), ctx=ctx)
        unmix = _host(gemm_f64(V, W, trans_a=True, c=_even(ch, ch, dev), ctx=ctx))
        coh = _coherence_on_device(Sep, ctx)
        sep = _host_staged(Sep)
        return PhaseBssResult(unmix, sep, coh,
                              PhaseBssTrace(ch, s, floor, tr.initial_offdiag, tr.final_offdiag, tr.rotations,
                                            float(coh.sum() / max(len(coh), 1))))


# ---------------------------------------------------------- phase normalizer
def _wedge_capacity(g: np.ndarray) -> np.ndarray:
    """src/phase_normalizer.rs:113-126: Omega_i = sum over j != i of
    sqrt(max(G_ii G_jj - G_ij^2, 0)) (the parallelogram areas of row i with
    every other row, from the Gram matrix alone)."""
    d = np.diag(g)
    area = np.sqrt(np.maximum(np.outer(d, d) - g * g, 0.0))
    np.fill_diagonal(area, 0.0)
    return area.sum(axis=1)


def row_wedge_capacity(a, ctx: Context | None = None) -> np.ndarray:
    """``row_wedge_capacity`` (src/phase_normalizer.rs:108-111)."""
    ctx = ctx or default_context()
    a = np.asarray(a, dtype=np.float64)
    A = _to_dev(a, _device(ctx))
    return _wedge_capacity(_host(gemm_f64(A, A, trans_b=True, c=_even(a.shape[0], a.shape[0], A.device), ctx=ctx)))


def row_leverage_scores(a, ctx: Context | None = None) -> np.ndarray:
    """``row_leverage_scores`` (src/phase_normalizer.rs:131-137): squared row
    norms of U from ``solve_rectangular``."""
    u, _, _ = LieSvdSmall.solve_rectangular(a, ctx=ctx)
    return np.sum(u * u, axis=1)


def canonical_row_scores(a, ctx: Context | None = None) -> np.ndarray:
    """``canonical_row_scores`` (src/phase_normalizer.rs:139-145):
    S_i = G_ii (1 + Omega_i) h_i with G = a a^T; invariant under a rotation of
    the columns, equivariant under a permutation of the rows."""
    ctx = ctx or default_context()
    a = np.asarray(a, dtype=np.float64)
    if a.ndim != 2 or a.size == 0:
        raise L.LsvdError(L.BAD_SHAPE, "canonical_row_scores: empty input")
    A = _to_dev(a, _device(ctx))
    g = _host(gemm_f64(A, A, trans_b=True, c=_even(a.shape[0], a.shape[0], A.device), ctx=ctx))
    return np.diag(g) * (1.0 + _wedge_capacity(g)) * row_leverage_scores(a, ctx=ctx)


def canonical_column_scores(a, ctx: Context | None = None) -> np.ndarray:
    """``canonical_column_scores`` (src/phase_normalizer.rs:147-150)."""
    return canonical_row_scores(np.asarray(a, dtype=np.float64).T, ctx=ctx)


class CanonicalOrder:
    """``CanonicalOrder`` (src/phase_normalizer.rs:156-238):
    ``order[new_position] = original_index``, ``inverse`` its inverse."""

    def __init__(self, order, scores=None):
        self.order = np.asarray(order, dtype=np.int64)
        self.inverse = np.empty_like(self.order)
        self.inverse[self.order] = np.arange(len(self.order))
        self.scores = np.zeros(0) if scores is None else np.asarray(scores, dtype=np.float64)

    @staticmethod
    def from_order(order) -> "CanonicalOrder":
        return CanonicalOrder(order)

    @staticmethod
    def from_scores(scores) -> "CanonicalOrder":
        """Descending scores, ties broken by the original index (a stable sort
        of the negated scores; NaN scores compare equal, as in the reference)."""
        s = np.asarray(scores, dtype=np.float64)
        key = np.where(np.isnan(s), 0.0, -s)
        return CanonicalOrder(np.argsort(key, kind="stable"), s)

    def permute_rows(self, a):
        return np.asarray(a)[self.order]

    def permute_cols(self, a):
        return np.asarray(a)[:, self.order]

    def restore_rows(self, p):
        return np.asarray(p)[self.inverse]

    def restore_cols(self, p):
        return np.asarray(p)[:, self.inverse]

    def permute_symmetric(self, a):
        return np.asarray(a)[np.ix_(self.order, self.order)]

    def restore_symmetric(self, p):
        return np.asarray(p)[np.ix_(self.inverse, self.inverse)]


def canonical_row_order(a, ctx: Context | None = None) -> CanonicalOrder:
    return CanonicalOrder.from_scores(canonical_row_scores(a, ctx=ctx))


def canonical_column_order(a, ctx: Context | None = None) -> CanonicalOrder:
    return CanonicalOrder.from_scores(canonical_column_scores(a, ctx=ctx))


def canonical_family_order(matrices, ctx: Context | None = None) -> CanonicalOrder:
    """``canonical_family_order`` (src/phase_normalizer.rs:253-279): one
    order for the whole family from the sum of the members' row scores."""
    if len(matrices) == 0:
        raise L.LsvdError(L.BAD_SHAPE, "canonical_family_order: empty family")
    n = np.asarray(matrices[0]).shape[0]
    total = np.zeros(n)
    for m in matrices:
        m = np.asarray(m)
        if m.shape != (n, n):
            raise L.LsvdError(L.BAD_SHAPE, "canonical_family_order: members must be square on the same axes")
        total = total + canonical_row_scores(m, ctx=ctx)
    return CanonicalOrder.from_scores(total)


@dataclass
class CanonicalSvdResult:
    """``CanonicalSvdResult`` (src/phase_normalizer.rs:286-293)."""
    u: np.ndarray
    sigma: np.ndarray
    vt: np.ndarray
    row_order: CanonicalOrder
    col_order: CanonicalOrder


def solve_canonicalized(a, ctx: Context | None = None) -> CanonicalSvdResult:
    """``solve_canonicalized`` (src/phase_normalizer.rs:295-309): permute rows
    and columns into canonical order, ``solve_rectangular``, restore U's rows
    and Vt's columns."""
    a = np.asarray(a, dtype=np.float64)
    ro, co = canonical_row_order(a, ctx=ctx), canonical_column_order(a, ctx=ctx)
    u, s, vt = LieSvdSmall.solve_rectangular(np.ascontiguousarray(co.permute_cols(ro.permute_rows(a))), ctx=ctx)
    return CanonicalSvdResult(ro.restore_rows(u), s, co.restore_cols(vt), ro, co)


@dataclass
class CanonicalJadeResult:
    """``CanonicalJadeResult`` (src/phase_normalizer.rs:318-324)."""
    basis: np.ndarray
    diagonals: list
    trace: JointDiagonalizationTrace
    order: CanonicalOrder


def diagonalize_symmetric_canonicalized(matrices, ctx: Context | None = None) -> CanonicalJadeResult:
    """``diagonalize_symmetric_canonicalized`` (src/phase_normalizer.rs:326-340):
    one shared order for the family, Phase-JADE on the permuted members, the
    basis rows restored to the caller's axis order."""
    order = canonical_family_order(matrices, ctx=ctx)
    canon = [np.ascontiguousarray(order.permute_symmetric(np.asarray(m, dtype=np.float64))) for m in matrices]
    v, d, tr = LieSvdJoint.diagonalize_symmetric(canon, ctx=ctx)
    return CanonicalJadeResult(order.restore_rows(v), d, tr, order)
