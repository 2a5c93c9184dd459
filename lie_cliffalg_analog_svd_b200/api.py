"""Python host mirror of the reference's API for the hot path, over the C ABI.

Names, argument meaning and error behaviour follow the Rust crate
``lie_cliffalg_analog_svd`` v0.44.0:

* ``LieSvdSmall.solve(a) -> (U, sigma, Vt)``      src/lie_svd_small.rs:296
* ``LieSvdSmall.solve_rectangular(a)``            src/lie_svd_small.rs:340
* ``LieSvdMicro.solve(a)``                        src/lie_svd_micro.rs:21
* ``LieSvd.solve(a)`` -- the exact tiers of the dispatcher: Micro for n <= 4
  (src/lie_svd_adaptive.rs:105-106), Small otherwise
* ``metrics.compute(a, u, sigma, vt, sigma_ref)``  src/lib.rs:149
* ``svd_batched(ns, a)`` -- the batched entry (no reference counterpart)

Where the reference panics (``assert!``) these raise ``LsvdError`` with status
``BAD_SHAPE``.  Every call runs on the GPU through ``liblsvd_b200.so``.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass

import numpy as np

from . import _lib as L


def _check(lib, ctx_ptr, status: int, what: str):
    if status in (L.OK,):
        return
    msg = lib.lsvd_status_string(status).decode()
    detail = lib.lsvd_context_last_error(ctx_ptr).decode() if ctx_ptr else ""
    raise L.LsvdError(status, f"{what}: {msg} {detail}".strip())


class Context:
    """One ``lsvd_context`` (device, CUDA stream, workspaces, plan cache)."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        st = self.lib.lsvd_context_create(device, C.byref(h))
        if st != L.OK:
            raise L.LsvdError(st, f"lsvd_context_create: {self.lib.lsvd_status_string(st).decode()}")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            self.lib.lsvd_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int):
        _check(self.lib, self.handle, self.lib.lsvd_context_set_stream(self.handle, C.c_void_p(stream_handle)),
               "set_stream")

    @property
    def stream(self) -> int:
        return self.lib.lsvd_context_get_stream(self.handle) or 0

    def synchronize(self):
        _check(self.lib, self.handle, self.lib.lsvd_synchronize(self.handle), "synchronize")

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.lsvd_context_kernel_launches(self.handle))


_tls = threading.local()


def default_context(device: int = 0) -> Context:
    """Per-thread default context (a context is not thread-safe)."""
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    if device not in ctxs:
        ctxs[device] = Context(device)
    return ctxs[device]


PRECISIONS = {"fp64": L.PREC_FP64, "tf32": L.PREC_MIXED_TF32, "bf16": L.PREC_MIXED_BF16}


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _diag_dict(d: L.Diag) -> dict:
    return {k: getattr(d, k) for k, _ in L.Diag._fields_}


@dataclass
class SmallResult:
    u: np.ndarray
    sigma: np.ndarray
    vt: np.ndarray
    diag: dict
    rotors: np.ndarray | None
    perm: np.ndarray


class LieSvdSmall:
    """``LieSvdSmall`` (src/lie_svd_small.rs:291-361) on the GPU."""

    @staticmethod
    def solve(a, ctx: Context | None = None):
        """Full SVD ``(U, sigma, Vt)`` of a square matrix (n <= 64 on the
        shared-memory kernels, larger n on the blocked large solve).  Like the
        reference's ``solve`` it computes no diagnostics (``solve_full`` does)."""
        r = LieSvdSmall.solve_full(a, ctx=ctx, want_diag=False)
        return r.u, r.sigma, r.vt

    @staticmethod
    def solve_full(a, ctx: Context | None = None, want_diag: bool = True,
                   rotor_cap: int = 0) -> SmallResult:
        """``solve`` plus diagnostics, the sort permutation and (if
        ``rotor_cap`` > 0) the accepted rotor stream of the eigensolve."""
        ctx = ctx or default_context()
        a = _f64(a)
        if a.ndim != 2 or a.shape[0] != a.shape[1]:
            raise L.LsvdError(L.BAD_SHAPE, "LieSvdSmall::solve: matrix must be square N×N")
        n = a.shape[0]
        u = np.empty((n, n)); s = np.empty(n); vt = np.empty((n, n))
        d = L.Diag()
        small = n <= 64  # the rotor stream and permutation exist on the shared-memory route
        if rotor_cap and not small:
            raise L.LsvdError(L.UNSUPPORTED, "LieSvdSmall::solve: rotor stream needs n <= 64")
        perm = np.empty(n, dtype=np.int32) if small else None
        rot = np.empty(max(rotor_cap, 1), dtype=L.ROTOR_DTYPE) if rotor_cap else None
        cnt = C.c_int64(0)
        st = ctx.lib.lsvd_small_solve_f64(
            ctx.handle, n, _ptr(a), n, _ptr(u), n, _ptr(s), _ptr(vt), n, C.byref(d),
            _ptr(rot) if rot is not None else None, rotor_cap, C.byref(cnt) if small else None,
            _ptr(perm) if small else None, L.WANT_DIAG if want_diag else 0)
        if st not in (L.OK, L.NOT_CONVERGED, L.NONFINITE_INPUT, L.ROTOR_OVERFLOW):
            _check(ctx.lib, ctx.handle, st, "LieSvdSmall::solve")
        dd = _diag_dict(d)
        dd["status"] = st
        dd["rotor_count"] = cnt.value
        return SmallResult(u, s, vt, dd, rot[:min(cnt.value, rotor_cap)] if rot is not None else None,
                           perm)

    @staticmethod
    def solve_rectangular(a, ctx: Context | None = None):
        """Thin SVD of an m×d matrix: U m×k, sigma k, Vt k×d (k = min(m, d))."""
        ctx = ctx or default_context()
        a = _f64(a)
        if a.ndim != 2 or a.shape[0] == 0 or a.shape[1] == 0:
            raise L.LsvdError(L.BAD_SHAPE, "LieSvdSmall::solve_rectangular: empty input")
        m, d = a.shape
        k = min(m, d)
        u = np.empty((m, k)); s = np.empty(k); vt = np.empty((k, d))
        st = ctx.lib.lsvd_small_solve_rectangular_f64(ctx.handle, m, d, _ptr(a), d, _ptr(u), k,
                                                      _ptr(s), _ptr(vt), d, None, 0)
        if st not in (L.OK, L.NOT_CONVERGED):
            _check(ctx.lib, ctx.handle, st, "LieSvdSmall::solve_rectangular")
        return u, s, vt


@dataclass
class LargeResult:
    u: object
    s: object
    vt: object
    info: L.LargeInfo
    diag: dict
    status: int


def svd_large(a, precision: str = "fp64", want_diag: bool = True, ctx: Context | None = None) -> LargeResult:
    """SVD of one large dense matrix (``lsvd_svd_large_f64``): ``a`` m×n (a
    numpy array, or a float64 CUDA torch tensor for the device-pointer path);
    returns the thin U (m×k), S (k), Vt (k×n) with the run's diagnostics."""
    ctx = ctx or default_context()
    if _is_torch(a):
        import torch
        assert a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()
        m, n = a.shape
        k = min(m, n)
        u = torch.empty((m, k), dtype=torch.float64, device=a.device)
        s = torch.empty(k, dtype=torch.float64, device=a.device)
        vt = torch.empty((k, n), dtype=torch.float64, device=a.device)
        pa, pu, ps, pv = (C.c_void_p(t.data_ptr()) for t in (a, u, s, vt))
        flags = L.DEVICE_POINTERS
    else:
        a = _f64(a)
        m, n = a.shape
        k = min(m, n)
        u = np.empty((m, k)); s = np.empty(k); vt = np.empty((k, n))
        pa, pu, ps, pv = _ptr(a), _ptr(u), _ptr(s), _ptr(vt)
        flags = 0
    info = L.LargeInfo()
    st = ctx.lib.lsvd_svd_large_f64(ctx.handle, m, n, pa, n, pu, k, ps, pv, n, PRECISIONS[precision],
                                    C.byref(info), flags | (L.WANT_DIAG if want_diag else 0))
    if st not in (L.OK, L.NOT_CONVERGED):
        _check(ctx.lib, ctx.handle, st, "svd_large")
    diag = {"rel_recon": info.rel_recon, "orth_u": info.orth_u, "orth_v": info.orth_v}
    return LargeResult(u, s, vt, info, diag, st)


class LieSvdMicro:
    """``LieSvdMicro`` (src/lie_svd_micro.rs:17-53) on the GPU."""

    @staticmethod
    def solve(a, ctx: Context | None = None, diag: bool = False):
        ctx = ctx or default_context()
        a = _f64(a)
        n = a.shape[0]
        if a.ndim != 2 or a.shape[1] != n:
            raise L.LsvdError(L.BAD_SHAPE, "LieSvdMicro: matrix must be square")
        if n > 4:
            raise L.LsvdError(L.BAD_SHAPE, "LieSvdMicro only supports N <= 4")
        u = np.empty((n, n)); s = np.empty(n); vt = np.empty((n, n))
        d = L.Diag()
        if n:
            st = ctx.lib.lsvd_micro_solve_f64(ctx.handle, n, _ptr(a), n, _ptr(u), n, _ptr(s),
                                              _ptr(vt), n, C.byref(d), L.WANT_DIAG)
            if st not in (L.OK, L.NONFINITE_INPUT):
                _check(ctx.lib, ctx.handle, st, "LieSvdMicro::solve")
        return (u, s, vt, _diag_dict(d)) if diag else (u, s, vt)


class LieSvd:
    """``LieSvd::solve`` (src/lie_svd.rs:49), which forwards to
    ``LieSvdAdaptive::solve``: the tiers that runs here -- Micro for
    n <= MICRO_MAX_N = 4, Small otherwise -- without computing the triage
    (``LieSvdAdaptive.solve_with_trace`` reports the route the reference's
    triage would pick, including its PhaseFlow/CoreFlow research routes)."""

    MICRO_MAX_N = 4

    @staticmethod
    def solve(a, ctx: Context | None = None):
        a = _f64(a)
        if a.shape[0] <= LieSvd.MICRO_MAX_N:
            return LieSvdMicro.solve(a, ctx=ctx)
        return LieSvdSmall.solve(a, ctx=ctx)


class solvers:  # noqa: N801 -- mirrors the Rust module name
    """``solvers::run_small`` / ``run_auto`` (src/lib.rs:56-60, :117-121):
    the SVD and its wall time in seconds (the reference returns a Duration)."""

    @staticmethod
    def run_small(a, ctx: Context | None = None):
        import time
        t0 = time.perf_counter()
        u, s, vt = LieSvdSmall.solve(a, ctx=ctx)
        return u, s, vt, time.perf_counter() - t0

    @staticmethod
    def run_auto(a, ctx: Context | None = None):
        import time
        t0 = time.perf_counter()
        u, s, vt = LieSvd.solve(a, ctx=ctx)
        return u, s, vt, time.perf_counter() - t0


ADAPTIVE_ROUTES = ("Micro", "Small", "PhaseFlow", "CoreFlowTopo", "Hybrid")
PASSPORT_ROUTES = ("RealSmall", "RealPhaseFlowPolished")


def triage_batched(mats, ctx: Context | None = None) -> np.ndarray:
    """Routing statistics of every matrix (``lsvd_triage_batched_f64``): a
    structured array with the AdaptiveTriage, PhaseSignature and passport
    fields, ``adaptive_route`` and ``passport_route`` per matrix."""
    ctx = ctx or default_context()
    mats = [_f64(m) for m in mats]
    rows = np.array([m.shape[0] for m in mats], dtype=np.int32)
    cols = np.array([m.shape[1] for m in mats], dtype=np.int32)
    flat = np.concatenate([m.ravel() for m in mats]) if mats else np.zeros(0)
    out = np.empty(len(mats), dtype=L.TRIAGE_DTYPE)
    if len(mats):
        st = ctx.lib.lsvd_triage_batched_f64(ctx.handle, len(mats), _ptr(rows), _ptr(cols), _ptr(flat),
                                             _ptr(out), 0)
        _check(ctx.lib, ctx.handle, st, "triage_batched")
    return out


def _triage_dict(rec) -> dict:
    d = {f: float(rec[f]) for f in L.TRIAGE_FIELDS}
    r = int(rec["adaptive_route"])
    d["route"] = ADAPTIVE_ROUTES[r] if r >= 0 else None
    d["passport_route"] = PASSPORT_ROUTES[int(rec["passport_route"])]
    return d


class LieSvdAdaptive:
    """``LieSvdAdaptive``'s triage (src/lie_svd_adaptive.rs:84-274) on the GPU.
    The routes themselves beyond the exact tiers (PhaseFlow, CoreFlowTopo,
    Hybrid) are research solvers this library does not provide: ``solve``
    runs the exact tier (Micro for n <= 4, Small otherwise) and reports the
    route the reference would have taken."""

    @staticmethod
    def analyze_matrix(a, ctx: Context | None = None) -> dict:
        a = _f64(a)
        if a.ndim != 2 or a.shape[0] != a.shape[1]:
            raise L.LsvdError(L.BAD_SHAPE, "adaptive SVD expects square matrices")
        return _triage_dict(triage_batched([a], ctx=ctx)[0])

    @staticmethod
    def choose_route(a, ctx: Context | None = None) -> str:
        return LieSvdAdaptive.analyze_matrix(a, ctx=ctx)["route"]

    @staticmethod
    def solve(a, ctx: Context | None = None):
        """``LieSvdAdaptive::solve`` (src/lie_svd_adaptive.rs:83-85)."""
        return LieSvdAdaptive.solve_with_trace(a, ctx=ctx)[0]

    @staticmethod
    def solve_with_trace(a, params=None, ctx: Context | None = None):
        """``LieSvdAdaptive::solve_with_trace`` (src/lie_svd_adaptive.rs:87-100)
        with the default ``LieSvdAdaptiveParams``: the triage picks the route
        as the reference does; Micro and Small run as there, and the research
        routes (PhaseFlow, CoreFlowTopo, Hybrid) run the exact Small tier
        instead.  Returns ``((U, sigma, Vt), trace)``, trace = {"route": the
        reference's route, "route_taken": the tier that ran, "triage": the
        analyze_matrix statistics}."""
        if params is not None:
            raise L.LsvdError(L.UNSUPPORTED, "LieSvdAdaptive: only the default parameters are mirrored")
        tri = LieSvdAdaptive.analyze_matrix(a, ctx=ctx)
        route = tri["route"]
        if route == "Micro":
            res, taken = LieSvdMicro.solve(a, ctx=ctx), "Micro"
        else:
            res, taken = LieSvdSmall.solve(a, ctx=ctx), "Small"
        return res, {"route": route, "route_taken": taken, "triage": tri}


@dataclass
class PhaseEngineReport:
    passport: dict
    route: str
    time_s: float
    rel_recon: float | None
    orth_u: float | None
    orth_v: float | None
    phase_stress: tuple | None
    schedule_events: int


class PhaseEngine:
    """``PhaseEngine``'s real-matrix facade (src/lie_svd_engine.rs:75-136,
    :246-275) over the GPU kernels."""

    @staticmethod
    def passport_real(a, ctx: Context | None = None) -> dict:
        a = _f64(a)
        d = _triage_dict(triage_batched([a], ctx=ctx)[0])
        d.update({"rows": a.shape[0], "cols": a.shape[1], "family": 1, "tensor_modes": None,
                  "route_hint": d.pop("passport_route")})
        return d

    @staticmethod
    def solve_real(a, ctx: Context | None = None):
        """``PhaseEngine::solve_real``: the passport on the GPU, then the SVD.
        The ``RealPhaseFlowPolished`` route is a research solver this library
        does not provide; inputs the passport sends there are solved by the
        exact route (LieSvdSmall::solve on the GPU) and the report says so
        (``route`` "RealSmall", ``passport['route_hint']`` unchanged)."""
        import time
        a = _f64(a)
        passport = PhaseEngine.passport_real(a, ctx=ctx)
        t0 = time.perf_counter()
        if a.shape[0] == a.shape[1]:
            u, s, vt = LieSvdSmall.solve(a, ctx=ctx)
        else:
            u, s, vt = LieSvdSmall.solve_rectangular(a, ctx=ctx)
        el = time.perf_counter() - t0
        m = metrics.compute(a, u, s, vt, ctx=ctx)
        return (u, s, vt), PhaseEngineReport(passport, "RealSmall", el, m.rel_recon, m.orth_u, m.orth_v, None, 0)

    @staticmethod
    def diagonalize_family(mats, ctx: Context | None = None):
        """``PhaseEngine::diagonalize_family``: Phase-JADE of the family on the
        GPU with the passport of its first matrix."""
        import time
        if not len(mats):
            raise L.LsvdError(L.BAD_SHAPE, "PhaseEngine: empty matrix family")
        t0 = time.perf_counter()
        v, diags, trace = LieSvdJoint.diagonalize_symmetric_with_params(
            mats, JointDiagonalizationParams.for_n(np.asarray(mats[0]).shape[0]), ctx=ctx)
        el = time.perf_counter() - t0
        passport = PhaseEngine.passport_real(mats[0], ctx=ctx)
        passport["family"] = len(mats)
        passport["route_hint"] = "JointPhaseJade"
        rep = PhaseEngineReport(passport, "JointPhaseJade", el, None, None,
                                float(np.linalg.norm(v.T @ v - np.eye(v.shape[1]))),
                                (trace.initial_offdiag, trace.final_offdiag), int(trace.rotations))
        return v, diags, trace, rep


@dataclass
class SvdMetrics:
    rel_recon: float
    orth_u: float
    orth_v: float
    sigma_max_rel: float | None
    sigma_tail_rel: float | None


class metrics:  # noqa: N801 -- mirrors the Rust module name
    """``metrics::compute`` (src/lib.rs:149-194) on the GPU."""

    @staticmethod
    def compute(a, u, sigma, vt, sigma_ref=None, ctx: Context | None = None) -> SvdMetrics:
        ctx = ctx or default_context()
        a, u, sigma, vt = _f64(a), _f64(u), _f64(sigma), _f64(vt)
        m, d = a.shape
        k = sigma.shape[0]
        ref = _f64(sigma_ref) if sigma_ref is not None else None
        out = np.empty(5)
        st = ctx.lib.lsvd_metrics_f64(ctx.handle, m, d, k, _ptr(a), _ptr(u), _ptr(sigma), _ptr(vt),
                                      _ptr(ref) if ref is not None else None, _ptr(out), 0)
        _check(ctx.lib, ctx.handle, st, "metrics::compute")
        return SvdMetrics(out[0], out[1], out[2], None if ref is None else out[3],
                          None if ref is None else out[4])




def packed_offsets(ns) -> tuple[np.ndarray, np.ndarray]:
    ns = np.asarray(ns, dtype=np.int64)
    ao = np.zeros(ns.size + 1, dtype=np.int64)
    ao[1:] = np.cumsum(ns * ns)
    so = np.zeros(ns.size + 1, dtype=np.int64)
    so[1:] = np.cumsum(ns)
    return ao, so


def svd_batched(ns, a, precision: str = "fp64", want_diag: bool = False,
                ctx: Context | None = None, out=None, device_async: bool = False):
    """Batched uneven SVD.  ``ns``: int sizes (1..64); ``a``: the matrices
    back to back, row-major (numpy array on the host, or a CUDA torch tensor
    for the device-pointer path).  Returns ``(U, S, Vt, diags, status)`` in the
    same packed layout (torch tensors when ``a`` is a torch tensor)."""
    ctx = ctx or default_context()
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    count = ns.size
    ao, so = packed_offsets(ns)
    prec = PRECISIONS[precision]
    flags = L.WANT_DIAG if want_diag else 0
    is_torch = _is_torch(a)
    if is_torch:
        import torch
        assert a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()
        if out is None:
            u = torch.empty(int(ao[-1]), dtype=torch.float64, device=a.device)
            s = torch.empty(int(so[-1]), dtype=torch.float64, device=a.device)
            vt = torch.empty(int(ao[-1]), dtype=torch.float64, device=a.device)
            dg = torch.empty(count * C.sizeof(L.Diag) if want_diag else 8, dtype=torch.uint8, device=a.device)
        else:
            u, s, vt, dg = out
        flags |= L.DEVICE_POINTERS | (L.ASYNC if device_async else 0)
        st = ctx.lib.lsvd_svd_batched_f64(ctx.handle, count, _ptr(ns), C.c_void_p(a.data_ptr()),
                                          C.c_void_p(u.data_ptr()), C.c_void_p(s.data_ptr()),
                                          C.c_void_p(vt.data_ptr()),
                                          C.c_void_p(dg.data_ptr()) if want_diag else None, prec,
                                          flags)
        if st not in (L.OK, L.NOT_CONVERGED, L.NONFINITE_INPUT):
            _check(ctx.lib, ctx.handle, st, "svd_batched")
        return u, s, vt, (dg if want_diag else None), st
    a = _f64(a)
    assert a.size == ao[-1], "packed A has the wrong length for ns"
    if out is None:
        u = np.empty(int(ao[-1])); s = np.empty(int(so[-1])); vt = np.empty(int(ao[-1]))
        dg = np.empty(count, dtype=L.DIAG_DTYPE) if want_diag else None
    else:
        u, s, vt, dg = out
    st = ctx.lib.lsvd_svd_batched_f64(ctx.handle, count, _ptr(ns), _ptr(a), _ptr(u), _ptr(s),
                                      _ptr(vt), _ptr(dg) if dg is not None else None, prec, flags)
    if st not in (L.OK, L.NOT_CONVERGED, L.NONFINITE_INPUT):
        _check(ctx.lib, ctx.handle, st, "svd_batched")
    return u, s, vt, dg, st


def autotune(per_class: int = 2000, cache_path: str | None = None, ctx: Context | None = None) -> str:
    """Times the batched FP64 kernel's team shapes per size class and writes
    the fastest to the shape cache (``lsvd_autotune_f64``); returns the
    per-class report."""
    ctx = ctx or default_context()
    buf = C.create_string_buffer(4096)
    st = ctx.lib.lsvd_autotune_f64(ctx.handle, per_class, cache_path.encode() if cache_path else None,
                                   C.cast(buf, C.c_void_p), len(buf))
    _check(ctx.lib, ctx.handle, st, "autotune")
    return buf.value.decode()


def class_shapes(precision: str = "fp64", ctx: Context | None = None) -> np.ndarray:
    """The (warps, tile, lanes per pair, matrices per team) of each of the 8
    size classes the batched planner uses now."""
    ctx = ctx or default_context()
    out = np.zeros(32, dtype=np.int32)
    _check(ctx.lib, ctx.handle, ctx.lib.lsvd_class_shapes(ctx.handle, PRECISIONS[precision], _ptr(out)),
           "class_shapes")
    return out.reshape(8, 4)


def unpack(ns, packed, square: bool = True):
    """Splits a packed buffer into per-matrix arrays."""
    ns = np.asarray(ns, dtype=np.int64)
    ao, so = packed_offsets(ns)
    off = ao if square else so
    out = []
    for t, n in enumerate(ns):
        blk = packed[off[t]:off[t + 1]]
        out.append(blk.reshape(n, n) if square else blk)
    return out


TARGETS = {"mzi_mesh": 0, "fpga_rotor_mesh": 1}


def _json_call(fn, *args) -> str:
    n = C.c_int64(0)
    st = fn(*args, None, 0, C.byref(n))
    if st not in (L.OK,):
        raise L.LsvdError(st, "schedule sizing failed")
    buf = C.create_string_buffer(n.value + 1)
    st = fn(*args, buf, n.value + 1, C.byref(n))
    if st != L.OK:
        raise L.LsvdError(st, "schedule serialisation failed")
    return buf.value.decode()


class HardwareSchedule:
    """``HardwareSchedule`` (src/lie_svd_compiler.rs:43-266) as produced by the
    library's host-side compiler; ``to_json_string`` is the library's JSON."""

    @staticmethod
    def from_orthogonal_matrix_json(v, target: str = "mzi_mesh") -> str:
        v = _f64(v)
        d = v.shape[0]
        if v.ndim != 2 or v.shape[1] != d:
            raise L.LsvdError(L.BAD_SHAPE, "HardwareSchedule::from_orthogonal_matrix: matrix must be square")
        lib = L.load()
        return _json_call(lib.lsvd_schedule_from_orthogonal, d, _ptr(v), TARGETS[target])

    @staticmethod
    def from_rotor_stream_json(rotors, channels: int, target: str = "mzi_mesh") -> str:
        r = np.ascontiguousarray(rotors, dtype=L.ROTOR_DTYPE)
        lib = L.load()
        return _json_call(lib.lsvd_schedule_from_rotors, _ptr(r) if r.size else None, r.size,
                          channels, TARGETS[target])

    @staticmethod
    def _mzi_events(events):
        """MziPhase events (src/lie_svd_phaseflow.rs:202-209) as a structured
        array: either already of MZI_PHASE_DTYPE, or (pass, i, j, theta_l,
        theta_r, kind) tuples with kind a PhaseRotorKind name or index."""
        if isinstance(events, np.ndarray) and events.dtype == np.dtype(L.MZI_PHASE_DTYPE):
            return np.ascontiguousarray(events)
        ev = np.zeros(len(events), dtype=L.MZI_PHASE_DTYPE)
        for k, (ps, i, j, tl, tr, kind) in enumerate(events):
            kind = L.PHASE_ROTOR_KINDS.index(kind) if isinstance(kind, str) else int(kind)
            ev[k] = (ps, i, j, tl, tr, kind, 0)
        return ev

    @staticmethod
    def from_real_phaseflow_json(events, channels: int, target: str = "mzi_mesh") -> str:
        """``HardwareSchedule::from_real_phaseflow(..).to_json_string()``
        (src/lie_svd_compiler.rs:59-88, :213-265)."""
        ev = HardwareSchedule._mzi_events(events)
        return _json_call(L.load().lsvd_schedule_from_real_phaseflow, _ptr(ev) if ev.size else None, ev.size,
                          channels, TARGETS[target])

    @staticmethod
    def _frame_call(fn, *args, tail=()) -> bytes:
        n = C.c_int64(0)
        st = fn(*args, None, 0, C.byref(n), *tail)
        if st != L.OK:
            raise L.LsvdError(st, "schedule frame sizing failed")
        buf = np.empty(n.value, dtype=np.uint8)
        st = fn(*args, _ptr(buf), n.value, C.byref(n), *tail)
        if st != L.OK:
            raise L.LsvdError(st, "schedule frame encoding failed")
        return buf.tobytes()

    @staticmethod
    def from_real_phaseflow_binary(events, channels: int, target: str = "mzi_mesh") -> bytes:
        """Binary phase-schedule frame of ``from_real_phaseflow``'s schedule."""
        ev = HardwareSchedule._mzi_events(events)
        return HardwareSchedule._frame_call(L.load().lsvd_schedule_binary_from_real_phaseflow,
                                            _ptr(ev) if ev.size else None, ev.size, channels, TARGETS[target])

    @staticmethod
    def from_rotor_stream_binary(rotors, channels: int, target: str = "mzi_mesh", ctx=None):
        """Binary phase-schedule frame of a rotor stream.  A CUDA tensor of
        16-byte rotors (any dtype viewing the lsvd_rotor records, e.g. the
        stream buffer of ``svd_batched_stream``) is encoded on the device and
        returned as a CUDA uint8 tensor; a numpy stream on the host, as bytes."""
        lib = L.load()
        if _is_torch(rotors) and rotors.is_cuda:
            import torch
            rb = rotors.contiguous().view(torch.uint8)
            if rb.numel() % 16:
                raise L.LsvdError(L.BAD_ARGUMENT, "rotor stream is not a whole number of 16-byte records")
            count = rb.numel() // 16
            ctx = ctx or default_context(rotors.device.index or 0)
            torch.cuda.current_stream(rotors.device).synchronize()
            n = C.c_int64(0)
            st = lib.lsvd_schedule_binary_from_rotors(ctx.handle, C.c_void_p(rb.data_ptr()), count, channels,
                                                      TARGETS[target], None, 0, C.byref(n), L.DEVICE_POINTERS)
            if st != L.OK:
                raise L.LsvdError(st, "schedule frame sizing failed")
            out = torch.empty(n.value, dtype=torch.uint8, device=rotors.device)
            st = lib.lsvd_schedule_binary_from_rotors(ctx.handle, C.c_void_p(rb.data_ptr()), count, channels,
                                                      TARGETS[target], C.c_void_p(out.data_ptr()), n.value,
                                                      C.byref(n), L.DEVICE_POINTERS)
            _check(lib, ctx.handle, st, "lsvd_schedule_binary_from_rotors")
            return out
        r = np.ascontiguousarray(rotors, dtype=L.ROTOR_DTYPE)
        return HardwareSchedule._frame_call(lib.lsvd_schedule_binary_from_rotors, None, _ptr(r) if r.size else None,
                                            r.size, channels, TARGETS[target], tail=(0,))

    @staticmethod
    def binary_to_json(frame) -> str:
        """phase-schedule-v1 JSON text of a binary frame (bytes, numpy or a
        CUDA uint8 tensor, copied to the host first)."""
        if _is_torch(frame):
            frame = frame.cpu().numpy()
        buf = np.frombuffer(bytes(frame), dtype=np.uint8) if not isinstance(frame, np.ndarray) else frame
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        return _json_call(L.load().lsvd_schedule_binary_to_json, _ptr(buf), buf.size)


@dataclass
class JointDiagonalizationParams:
    """``JointDiagonalizationParams`` (src/lie_svd_joint.rs:18-41)."""
    max_sweeps: int
    tol: float = 1e-12
    min_pair_scale: float = 1e-14
    line_search_steps: int = 6

    @staticmethod
    def for_n(n: int) -> "JointDiagonalizationParams":
        return JointDiagonalizationParams(max_sweeps=12 + max(n, 1))


@dataclass
class JointDiagonalizationTrace:
    initial_offdiag: float
    final_offdiag: float
    sweeps: int
    rotations: int
    rejected_rotations: int


class LieSvdJoint:
    """``LieSvdJoint`` (src/lie_svd_joint.rs:61-261) on the GPU: the symmetric
    Phase-JADE route and the two-sided joint SVD, each also batched over
    independent families."""

    @staticmethod
    def joint_svd(matrices, ctx: Context | None = None):
        """``joint_svd`` (src/lie_svd_joint.rs:163): (U, per-matrix |diagonals|,
        Vt, trace) with ``JointDiagonalizationParams::for_n(min(rows, cols))``."""
        return _joint_svd(matrices, None, ctx)

    @staticmethod
    def joint_svd_with_params(matrices, params: "JointDiagonalizationParams",
                              ctx: Context | None = None):
        """``joint_svd_with_params`` (src/lie_svd_joint.rs:170-261)."""
        return _joint_svd(matrices, params, ctx)

    @staticmethod
    def joint_svd_families(m, params: "JointDiagonalizationParams | None" = None,
                           ctx: Context | None = None):
        """``m``: (families, K, rows, cols).  Returns U (families, rows, rows),
        |diagonals| (families, K, min(rows, cols)), Vt (families, cols, cols) and
        one trace per family."""
        return _joint_svd_families(m, params, ctx)

    @staticmethod
    def diagonalize_symmetric(matrices, ctx: Context | None = None):
        n = np.asarray(matrices[0]).shape[0] if len(matrices) else 0
        return LieSvdJoint.diagonalize_symmetric_with_params(
            matrices, JointDiagonalizationParams.for_n(n), ctx=ctx)

    @staticmethod
    def diagonalize_symmetric_with_params(matrices, params: JointDiagonalizationParams,
                                          ctx: Context | None = None):
        if len(matrices) == 0:
            raise L.LsvdError(L.BAD_SHAPE, "LieSvdJoint: empty matrix set")
        m = _f64(np.stack([np.asarray(x, dtype=np.float64) for x in matrices]))
        if m.ndim != 3 or m.shape[1] != m.shape[2]:
            raise L.LsvdError(L.BAD_SHAPE, "LieSvdJoint: matrices must be square")
        v, d, tr = LieSvdJoint.diagonalize_families(m[None], params, ctx=ctx)
        return v[0], [d[0, k].copy() for k in range(m.shape[0])], tr[0]

    @staticmethod
    def diagonalize_families(m, params: JointDiagonalizationParams | None = None,
                             ctx: Context | None = None):
        """``m``: (families, K, n, n).  Returns V (families, n, n), diagonals
        (families, K, n) and one trace per family."""
        ctx = ctx or default_context()
        m = _f64(m)
        F, K, n, n2 = m.shape
        if n != n2:
            raise L.LsvdError(L.BAD_SHAPE, "LieSvdJoint: matrices must be square")
        v = np.empty((F, n, n)); d = np.empty((F, K, n))
        tr = (L.JointTrace * F)()
        p = None
        if params is not None:
            p = L.JointParams(params.max_sweeps, params.tol, params.min_pair_scale,
                              params.line_search_steps)
        st = ctx.lib.lsvd_jade_sym_f64(ctx.handle, F, K, n, _ptr(m), C.byref(p) if p else None,
                                       _ptr(v), _ptr(d), tr, 0)
        _check(ctx.lib, ctx.handle, st, "LieSvdJoint::diagonalize_symmetric")
        traces = [JointDiagonalizationTrace(t.initial_offdiag, t.final_offdiag, t.sweeps,
                                            t.rotations, t.rejected_rotations) for t in tr]
        return v, d, traces


def _joint_svd_families(m, params, ctx):
    ctx = ctx or default_context()
    m = _f64(m)
    F, K, r, c = m.shape
    kk = min(r, c)
    u = np.empty((F, r, r)); s = np.empty((F, K, kk)); vt = np.empty((F, c, c))
    tr = (L.JointTrace * F)()
    p = None
    if params is not None:
        p = L.JointParams(params.max_sweeps, params.tol, params.min_pair_scale, params.line_search_steps)
    st = ctx.lib.lsvd_joint_svd_f64(ctx.handle, F, K, r, c, _ptr(m), C.byref(p) if p else None,
                                    _ptr(u), _ptr(s), _ptr(vt), tr, 0)
    _check(ctx.lib, ctx.handle, st, "LieSvdJoint::joint_svd")
    traces = [JointDiagonalizationTrace(t.initial_offdiag, t.final_offdiag, t.sweeps, t.rotations,
                                        t.rejected_rotations) for t in tr]
    return u, s, vt, traces


def _joint_svd(matrices, params=None, ctx=None):
    mats = [_f64(x) for x in matrices]
    if not mats:
        raise L.LsvdError(L.BAD_SHAPE, "LieSvdJoint::joint_svd: empty matrix set")
    m = np.stack(mats)[None]
    u, s, vt, traces = _joint_svd_families(m, params, ctx)
    return u[0], [s[0, k].copy() for k in range(s.shape[1])], vt[0], traces[0]


class PolarResult:
    """Polar factor with the iteration's diagnostics."""

    def __init__(self, q, info: L.PolarInfo, status: int):
        self.q = q
        self.iters_lowp = int(info.iters_lowp)
        self.iters_fp64 = int(info.iters_fp64)
        self.orth = float(info.orth)
        self.flops_lowp = float(info.flops_lowp)
        self.flops_fp64 = float(info.flops_fp64)
        self.gemm_ms_lowp = float(info.gemm_ms_lowp)
        self.gemm_ms_fp64 = float(info.gemm_ms_fp64)
        self.converged = bool(info.converged)
        self.status = status


def polar(a, precision: str = "fp64", ctx: Context | None = None) -> PolarResult:
    """Polar factor Q of a large m x n matrix (m >= n) by Newton-Schulz
    (``newton_schulz_polar``, src/lie_svd_small.rs:158-183): FP64 throughout,
    or TF32/BF16 tensor-core iterations followed by FP64 refinement.  ``a``:
    numpy array (host path) or a contiguous float64 CUDA torch tensor (device
    path, Q returned as a torch tensor)."""
    ctx = ctx or default_context()
    prec = PRECISIONS[precision]
    info = L.PolarInfo()
    is_torch = _is_torch(a)
    if is_torch:
        import torch
        assert a.is_cuda and a.dtype == torch.float64 and a.is_contiguous() and a.dim() == 2
        m, n = a.shape
        q = torch.empty_like(a)
        st = ctx.lib.lsvd_polar_f64(ctx.handle, m, n, C.c_void_p(a.data_ptr()), n,
                                    C.c_void_p(q.data_ptr()), n, prec, C.byref(info),
                                    L.DEVICE_POINTERS)
    else:
        a = _f64(a)
        m, n = a.shape
        q = np.empty_like(a)
        st = ctx.lib.lsvd_polar_f64(ctx.handle, m, n, _ptr(a), n, _ptr(q), n, prec,
                                    C.byref(info), 0)
    if st not in (L.OK, L.NOT_CONVERGED):
        _check(ctx.lib, ctx.handle, st, "polar")
    return PolarResult(q, info, st)


def gemm_nt_lowp(a, b, precision: str = "tf32", ctx: Context | None = None):
    """C = A B^T on the tcgen05 tensor cores with TF32 or BF16 operands and
    FP32 accumulation (the product kernel of the mixed polar iteration).
    ``a`` (M x K), ``b`` (N x K): contiguous float32 CUDA torch tensors."""
    import torch
    ctx = ctx or default_context()
    assert a.is_cuda and b.is_cuda and a.dtype == torch.float32 and b.dtype == torch.float32
    a = a.contiguous(); b = b.contiguous()
    M, K = a.shape
    N, K2 = b.shape
    assert K == K2
    c = torch.empty((M, N), dtype=torch.float32, device=a.device)
    st = ctx.lib.lsvd_gemm_nt_lowp(ctx.handle, M, N, K, C.c_void_p(a.data_ptr()),
                                   C.c_void_p(b.data_ptr()), C.c_void_p(c.data_ptr()),
                                   PRECISIONS[precision])
    _check(ctx.lib, ctx.handle, st, "gemm_nt_lowp")
    return c


def gemm_f64(a, b, trans_a: bool = False, trans_b: bool = False, alpha: float = 1.0, beta: float = 0.0,
             c=None, ctx: Context | None = None):
    """C = alpha op(A) op(B) + beta C in FP64 on the FP64 tensor path (the
    product kernel of the FP64 polar iteration and the large SVD).  ``a``,
    ``b`` (and ``c``): float64 CUDA torch tensors, row-major, contiguous rows
    with an even row stride."""
    import torch
    ctx = ctx or default_context()
    assert a.is_cuda and b.is_cuda and a.dtype == torch.float64 and b.dtype == torch.float64
    M, K = (a.shape[1], a.shape[0]) if trans_a else a.shape
    K2, N = (b.shape[1], b.shape[0]) if trans_b else b.shape
    assert K == K2
    if c is None:
        c = torch.zeros((M, N), dtype=torch.float64, device=a.device)
    assert a.stride(1) == 1 and b.stride(1) == 1 and c.stride(1) == 1
    # the inputs come from torch's current stream, the product runs on the context's stream
    torch.cuda.current_stream(a.device).synchronize()
    st = ctx.lib.lsvd_gemm_f64(ctx.handle, int(trans_a), int(trans_b), M, N, K, alpha,
                               C.c_void_p(a.data_ptr()), a.stride(0), C.c_void_p(b.data_ptr()), b.stride(0),
                               beta, C.c_void_p(c.data_ptr()), c.stride(0))
    _check(ctx.lib, ctx.handle, st, "gemm_f64")
    ctx.synchronize()
    return c


class SvdStream:
    """Forward of the stream-keeping batched SVD: sigma, sort permutation and
    accepted rotor stream per matrix (U, Vt when requested)."""

    def __init__(self, m, n, a, s, perm, rotors, counts, u, vt, diags, status, cap):
        self.m, self.n = m, n
        self.a = a
        self.s = s
        self.perm = perm
        self.rotors = rotors
        self.counts = counts
        self.u = u
        self.vt = vt
        self.diags = diags
        self.status = status
        self.rotor_cap = cap

    def stream_bytes(self) -> int:
        """Bytes the adjoint needs beyond A: sigma, perm and the streams."""
        nel = lambda x: int(x.numel()) if hasattr(x, "numel") else int(x.size)  # noqa: E731
        return int(self.counts.sum()) * 16 + nel(self.s) * 8 + nel(self.perm) * 4

    def uv_bytes(self) -> int:
        """Bytes of the U and V intermediates this replaces."""
        cnt = self.s.shape[0]
        return cnt * (self.m * self.n + self.n * self.n) * 8


def svd_batched_stream(a, rotor_cap: int | None = None, want_uv: bool = False,
                       want_diag: bool = False, ctx: Context | None = None) -> SvdStream:
    """Thin SVD of ``a`` (count, m, n), m >= n, n <= 64, keeping each matrix's
    rotor stream (numpy host arrays, or a contiguous float64 CUDA torch tensor
    for the device path, whose outputs are then torch tensors)."""
    ctx = ctx or default_context()
    cnt, m, n = a.shape
    # default: room for 20 full sweeps of n (n - 1) / 2 rotations
    cap = rotor_cap if rotor_cap is not None else 20 * (n * (n - 1) // 2) + 1
    flags = L.WANT_DIAG if want_diag else 0
    if _is_torch(a):
        import torch
        assert a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()
        dv = a.device
        s = torch.empty((cnt, n), dtype=torch.float64, device=dv)
        perm = torch.empty((cnt, n), dtype=torch.int32, device=dv)
        rot = torch.empty((cnt, max(cap, 1), 16), dtype=torch.uint8, device=dv)
        counts = torch.empty(cnt, dtype=torch.int64, device=dv)
        u = torch.empty((cnt, m, n), dtype=torch.float64, device=dv) if want_uv else None
        vt = torch.empty((cnt, n, n), dtype=torch.float64, device=dv) if want_uv else None
        dg = torch.empty((cnt, C.sizeof(L.Diag)), dtype=torch.uint8, device=dv) if want_diag else None
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
        st = ctx.lib.lsvd_svd_batched_stream_f64(ctx.handle, cnt, m, n, ptr(a), ptr(u), ptr(s), ptr(vt),
                                                 ptr(rot), cap, ptr(counts), ptr(perm), ptr(dg),
                                                 flags | L.DEVICE_POINTERS)
    else:
        a = _f64(a)
        s = np.empty((cnt, n)); perm = np.empty((cnt, n), dtype=np.int32)
        rot = np.empty((cnt, max(cap, 1)), dtype=L.ROTOR_DTYPE)
        counts = np.empty(cnt, dtype=np.int64)
        u = np.empty((cnt, m, n)) if want_uv else None
        vt = np.empty((cnt, n, n)) if want_uv else None
        dg = np.empty(cnt, dtype=L.DIAG_DTYPE) if want_diag else None
        p = lambda x: _ptr(x) if x is not None else None  # noqa: E731
        st = ctx.lib.lsvd_svd_batched_stream_f64(ctx.handle, cnt, m, n, _ptr(a), p(u), _ptr(s), p(vt),
                                                 _ptr(rot), cap, _ptr(counts), _ptr(perm), p(dg), flags)
    if st not in (L.OK, L.NOT_CONVERGED, L.NONFINITE_INPUT):
        _check(ctx.lib, ctx.handle, st, "svd_batched_stream")
    return SvdStream(m, n, a, s, perm, rot, counts, u, vt, dg, st, cap)


def svd_vjp(fwd: SvdStream, ubar=None, sbar=None, vbar=None, qbar=None, gap_tol: float = 0.0,
            ctx: Context | None = None, stored_vt=None):
    """Abar for cotangents on U (count, m, n), sigma (count, n), V (count, n, n)
    and the polar factor U V^T (count, m, n), from the forward's rotor stream
    (host numpy or device torch, matching the forward).  ``stored_vt``: read V
    from it instead of replaying the stream (the comparison path)."""
    ctx = ctx or default_context()
    cnt, m, n = fwd.a.shape
    if _is_torch(fwd.a):
        import torch
        ab = torch.empty_like(fwd.a)
        ptr = lambda t: C.c_void_p(t.contiguous().data_ptr()) if t is not None else None  # noqa: E731
        st = ctx.lib.lsvd_svd_vjp_f64(ctx.handle, cnt, m, n, ptr(fwd.a), ptr(fwd.s), ptr(fwd.perm),
                                      ptr(fwd.rotors), fwd.rotor_cap, ptr(fwd.counts), ptr(ubar),
                                      ptr(sbar), ptr(vbar), ptr(qbar), ptr(stored_vt), float(gap_tol),
                                      ptr(ab), L.DEVICE_POINTERS)
    else:
        ab = np.empty((cnt, m, n))
        p = lambda x: _ptr(_f64(x)) if x is not None else None  # noqa: E731
        keep = [None if x is None else _f64(x) for x in (ubar, sbar, vbar, qbar, stored_vt)]
        st = ctx.lib.lsvd_svd_vjp_f64(ctx.handle, cnt, m, n, _ptr(fwd.a), _ptr(fwd.s), _ptr(fwd.perm),
                                      _ptr(fwd.rotors), fwd.rotor_cap, _ptr(fwd.counts),
                                      *[_ptr(x) if x is not None else None for x in keep],
                                      float(gap_tol), _ptr(ab), 0)
        del p
    _check(ctx.lib, ctx.handle, st, "svd_vjp")
    return ab
