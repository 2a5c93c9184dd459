"""ctypes binding for the CPU oracle (``oracle/_build/liblsvd_oracle.so``).

TEST INFRASTRUCTURE ONLY.  The oracle is a C++ f64 restatement of the Rust
crate ``lie_cliffalg_analog_svd`` v0.44.0 hot path (see ``lsvd_oracle.cpp``
for the file:line each routine follows).  Only ``tests/``, the smoke
entry point and ``bench.py``'s CPU-baseline legs import this module, always as the checker or the timed CPU baseline -- never as the
product path.

The names mirror the reference API: ``LieSvdSmall.solve``,
``LieSvdSmall.solve_rectangular``, ``LieSvdMicro.solve``,
``LieSvdJoint.diagonalize_symmetric(_with_params)``, ``LieSvdJoint.joint_svd``,
``HardwareSchedule.from_orthogonal_matrix``, ``metrics.compute``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liblsvd_oracle.so")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -O3)."""
    src = os.path.join(_HERE, "lsvd_oracle.cpp")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


class SmallInfo(C.Structure):
    _fields_ = [("ns_iters", C.c_int32), ("polar_ok", C.c_int32), ("jacobi_sweeps", C.c_int32),
                ("jacobi_rotations", C.c_int64), ("repaired", C.c_int32),
                ("micro_fallback", C.c_int32)]


class JointParams(C.Structure):
    _fields_ = [("max_sweeps", C.c_int32), ("tol", C.c_double), ("min_pair_scale", C.c_double),
                ("line_search_steps", C.c_int32)]


class JointTrace(C.Structure):
    _fields_ = [("initial_offdiag", C.c_double), ("final_offdiag", C.c_double),
                ("sweeps", C.c_int64), ("rotations", C.c_int64),
                ("rejected_rotations", C.c_int64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        P = C.POINTER(C.c_double)
        _lib.oracle_joint_params_for_n.restype = JointParams
        _lib.oracle_schedule_from_orthogonal.restype = C.c_int64
        _lib.oracle_jade_sym.argtypes = [C.c_int64, C.c_int64, P, JointParams, P, P,
                                         C.POINTER(JointTrace)]
        _lib.oracle_joint_svd.argtypes = [C.c_int64, C.c_int64, C.c_int64, P, JointParams, P, P,
                                          P, C.POINTER(JointTrace)]
        V = C.c_void_p
        _lib.oracle_triage.argtypes = [C.c_int64, C.c_int64, V, V, V]
        _lib.oracle_svd_batch.restype = C.c_int64
        _lib.oracle_svd_batch.argtypes = [C.c_int64, V, V, V, V, V, V, V, V, C.c_int32]
        _lib.oracle_dot.argtypes = [C.c_int64, C.c_int64, C.c_int64, P, P, P]
        _lib.oracle_lagged_covariance.argtypes = [C.c_int64, C.c_int64, P, C.c_int64, P]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


TRIAGE_FIELDS = ("offdiag_ratio", "diagonal_dominance", "row_cv", "col_cv", "row_col_mismatch",
                 "symmetry_ratio", "transpose_torsion_ratio", "diagonal_entropy", "row_mass_entropy",
                 "col_mass_entropy", "suspicious_score", "mean_stress", "max_twist", "causal_disbalance",
                 "entropy_gap", "global_phase", "torsion_energy", "chirality_balance", "phase_entropy",
                 "chirality", "golden_resonance")
ADAPTIVE_ROUTES = ("Micro", "Small", "PhaseFlow", "CoreFlowTopo", "Hybrid")
PASSPORT_ROUTES = ("RealSmall", "RealPhaseFlowPolished")


def triage(a) -> dict:
    """Oracle restatement of analyze_matrix / choose_route
    (src/lie_svd_adaptive.rs:84-274), phase_signature
    (src/lie_svd_phasehealth.rs:100-343) and the PhaseEngine passport
    extras (src/lie_svd_engine.rs:75-103): field name -> value, plus
    "route" (AdaptiveRoute name, None when not square) and "passport_route"."""
    a = _c(a)
    rows, cols = a.shape
    out = np.empty(21)
    routes = np.zeros(2, dtype=np.int32)
    v = lambda x: C.c_void_p(x.ctypes.data)  # noqa: E731
    assert lib().oracle_triage(rows, cols, v(a), v(out), v(routes)) == 0
    d = dict(zip(TRIAGE_FIELDS, out.tolist()))
    d["route"] = ADAPTIVE_ROUTES[routes[0]] if routes[0] >= 0 else None
    d["passport_route"] = PASSPORT_ROUTES[routes[1]]
    return d


def svd_batch(ns, a, idx, threads: int, out=None):
    """Solves matrices ``idx`` of the packed uneven batch ``(ns, a)`` on
    ``threads`` host threads in one call (micro route for n <= 4, small
    otherwise).  Returns ``(solved, U, S, Vt)`` in the packed layout."""
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    a = _c(a)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    aoff = np.zeros(ns.size + 1, dtype=np.int64)
    aoff[1:] = np.cumsum(ns.astype(np.int64) ** 2)
    soff = np.zeros(ns.size + 1, dtype=np.int64)
    soff[1:] = np.cumsum(ns.astype(np.int64))
    if out is None:
        out = (np.empty_like(a), np.empty(int(soff[-1])), np.empty_like(a))
    u, s, vt = out
    v = lambda x: C.c_void_p(x.ctypes.data)  # noqa: E731
    got = lib().oracle_svd_batch(idx.size, v(idx), v(ns), v(aoff), v(soff), v(a), v(u), v(s), v(vt),
                                 int(threads))
    return int(got), u, s, vt


class LieSvdSmall:
    """Oracle restatement of ``LieSvdSmall`` (src/lie_svd_small.rs:291-361)."""

    @staticmethod
    def solve(a, info: bool = False):
        a = _c(a)
        n = a.shape[0]
        assert a.ndim == 2 and a.shape[1] == n, "LieSvdSmall::solve: matrix must be square N×N"
        u = np.empty((n, n)); s = np.empty(n); vt = np.empty((n, n)); inf = SmallInfo()
        rc = lib().oracle_small_solve(C.c_int64(n), _p(a), _p(u), _p(s), _p(vt), C.byref(inf))
        assert rc == 0
        return (u, s, vt, inf) if info else (u, s, vt)

    @staticmethod
    def solve_rectangular(a):
        a = _c(a)
        m, d = a.shape
        assert m > 0 and d > 0, "LieSvdSmall::solve_rectangular: empty input"
        k = min(m, d)
        u = np.empty((m, k)); s = np.empty(k); vt = np.empty((k, d))
        assert lib().oracle_small_solve_rectangular(C.c_int64(m), C.c_int64(d), _p(a), _p(u),
                                                    _p(s), _p(vt)) == 0
        return u, s, vt


def ns_polar(a):
    """``newton_schulz_polar`` (src/lie_svd_small.rs:158-183) -> (Q, ok, iters)."""
    a = _c(a)
    n = a.shape[0]
    q = np.empty((n, n)); ok = C.c_int32(); it = C.c_int32()
    assert lib().oracle_ns_polar(C.c_int64(n), _p(a), _p(q), C.byref(ok), C.byref(it)) == 0
    return q, bool(ok.value), it.value


def eigh_jacobi_full(p):
    """``eigh_jacobi_full`` (src/lie_svd_small.rs:212-285) -> (V, eig, sweeps, rotations)."""
    p = _c(p)
    n = p.shape[0]
    v = np.empty((n, n)); e = np.empty(n); sw = C.c_int32(); rot = C.c_int64()
    assert lib().oracle_eigh_jacobi(C.c_int64(n), _p(p), _p(v), _p(e), C.byref(sw),
                                    C.byref(rot)) == 0
    return v, e, sw.value, rot.value


def qr_reduce(a):
    """``qr_reduce`` (src/lie_svd_small.rs:373-418) -> (Q m×d, R d×d)."""
    a = _c(a)
    m, d = a.shape
    q = np.empty((m, d)); r = np.empty((d, d))
    assert lib().oracle_qr_reduce(C.c_int64(m), C.c_int64(d), _p(a), _p(q), _p(r)) == 0
    return q, r


class LieSvdMicro:
    """Oracle restatement of ``LieSvdMicro`` (src/lie_svd_micro.rs:17-53)."""

    @staticmethod
    def solve(a, info: bool = False):
        a = _c(a)
        n = a.shape[0]
        assert a.shape[1] == n, "LieSvdMicro: matrix must be square"
        assert n <= 4, "LieSvdMicro only supports N <= 4"
        u = np.empty((n, n)); s = np.empty(n); vt = np.empty((n, n)); inf = SmallInfo()
        assert lib().oracle_micro_solve(C.c_int64(n), _p(a) if n else None, _p(u), _p(s),
                                        _p(vt), C.byref(inf)) == 0
        return (u, s, vt, inf) if info else (u, s, vt)


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

    def _c(self):
        return JointParams(self.max_sweeps, self.tol, self.min_pair_scale, self.line_search_steps)


@dataclass
class JointDiagonalizationTrace:
    initial_offdiag: float
    final_offdiag: float
    sweeps: int
    rotations: int
    rejected_rotations: int


def _trace(t: JointTrace) -> JointDiagonalizationTrace:
    return JointDiagonalizationTrace(t.initial_offdiag, t.final_offdiag, t.sweeps, t.rotations,
                                     t.rejected_rotations)


class LieSvdJoint:
    """Oracle restatement of ``LieSvdJoint`` (src/lie_svd_joint.rs:61-262)."""

    @staticmethod
    def diagonalize_symmetric(matrices):
        n = np.asarray(matrices[0]).shape[0] if len(matrices) else 0
        return LieSvdJoint.diagonalize_symmetric_with_params(
            matrices, JointDiagonalizationParams.for_n(n))

    @staticmethod
    def diagonalize_symmetric_with_params(matrices, params: JointDiagonalizationParams):
        m = _c(np.stack([np.asarray(x, dtype=np.float64) for x in matrices]))
        k, n, n2 = m.shape
        assert n == n2, "LieSvdJoint: matrices must be square"
        v = np.empty((n, n)); d = np.empty((k, n)); tr = JointTrace()
        assert lib().oracle_jade_sym(k, n, _p(m), params._c(), _p(v), _p(d), C.byref(tr)) == 0
        return v, [d[i].copy() for i in range(k)], _trace(tr)

    @staticmethod
    def joint_svd(matrices):
        r, c = np.asarray(matrices[0]).shape
        return LieSvdJoint.joint_svd_with_params(matrices,
                                                 JointDiagonalizationParams.for_n(min(r, c)))

    @staticmethod
    def joint_svd_with_params(matrices, params: JointDiagonalizationParams):
        m = _c(np.stack([np.asarray(x, dtype=np.float64) for x in matrices]))
        k, r, c = m.shape
        kk = min(r, c)
        u = np.empty((r, r)); s = np.empty((k, kk)); vt = np.empty((c, c)); tr = JointTrace()
        assert lib().oracle_joint_svd(k, r, c, _p(m), params._c(), _p(u), _p(s), _p(vt),
                                      C.byref(tr)) == 0
        return u, [s[i].copy() for i in range(k)], vt, _trace(tr)


@dataclass
class SvdMetrics:
    rel_recon: float
    orth_u: float
    orth_v: float
    sigma_max_rel: float | None
    sigma_tail_rel: float | None


class metrics:  # noqa: N801 -- mirrors the Rust module name
    """``metrics::compute`` (src/lib.rs:149-194)."""

    @staticmethod
    def compute(a, u, sigma, vt, sigma_ref=None) -> SvdMetrics:
        a, u, vt = _c(a), _c(u), _c(vt)
        sigma = _c(sigma)
        m, d = a.shape
        k = sigma.shape[0]
        out = np.empty(5)
        ref = _c(sigma_ref) if sigma_ref is not None else None
        assert lib().oracle_metrics(C.c_int64(m), C.c_int64(d), C.c_int64(k), _p(a), _p(u),
                                    _p(sigma), _p(vt), _p(ref) if ref is not None else None,
                                    _p(out)) == 0
        return SvdMetrics(out[0], out[1], out[2],
                          None if sigma_ref is None else out[3],
                          None if sigma_ref is None else out[4])


def set_dot_fma(on: bool) -> None:
    """Product rounding of the oracle's ndarray ``dot`` restatements: fused
    multiply-add per k (matrixmultiply's FMA kernel, the default) or multiply
    then add (its generic kernel on hosts without FMA).  Process-wide."""
    lib().oracle_set_dot_fma(C.c_int32(1 if on else 0))


def dot(a, b) -> np.ndarray:
    """ndarray ``a.dot(&b)`` in the reference's product order (sequential
    fused multiply-adds over k, matrixmultiply 0.3.11's f64 kernel)."""
    a, b = _c(a), _c(b)
    m, k = a.shape
    k2, n = b.shape
    assert k == k2
    c = np.empty((m, n))
    assert lib().oracle_dot(C.c_int64(m), C.c_int64(k), C.c_int64(n), _p(a), _p(b), _p(c)) == 0
    return c


def lagged_covariance(x, lag: int) -> np.ndarray:
    """One symmetrised lagged covariance of Phase-BSS (src/lie_svd_bss.rs:172-190)
    in the reference's loop order (t, i, j; each product divided, then added)."""
    x = _c(x)
    ch, s = x.shape
    out = np.empty((ch, ch))
    assert lib().oracle_lagged_covariance(C.c_int64(ch), C.c_int64(s), _p(x), C.c_int64(lag), _p(out)) == 0
    return out


def _next_centered(state: list) -> float:
    """``next_centered`` of the reference's stress binary
    (src/bin/stress_cpu.rs:829-833): a 64-bit LCG, top 53 bits, minus 1/2."""
    state[0] = (state[0] * 6364136223846793005 + 1) & 0xFFFFFFFFFFFFFFFF
    return (state[0] >> 11) / float(1 << 53) - 0.5


def deterministic_orthogonal(n: int, state: list) -> np.ndarray:
    """``deterministic_orthogonal`` (src/bin/stress_cpu.rs:805-827): LCG
    entries in row-major order, then Gram-Schmidt over the columns with the
    reference's sequential sums (each product rounded, summed left to right)."""
    q = np.array([_next_centered(state) for _ in range(n * n)]).reshape(n, n)
    for j in range(n):
        for k in range(j):
            d = np.cumsum(q[:, j] * q[:, k])[-1]
            q[:, j] -= d * q[:, k]
        nrm = max(float(np.sqrt(np.cumsum(q[:, j] * q[:, j])[-1])), 1e-300)
        q[:, j] /= nrm
    return q


def fmt_e17(x: float) -> str:
    """Rust ``format!("{:.17e}", x)`` (src/lie_svd_compiler.rs:227)."""
    buf = C.create_string_buffer(64)
    lib().oracle_fmt_e17(C.c_double(x), buf, C.c_int64(64))
    return buf.value.decode()


def fmt_display(x: float) -> str:
    """Rust ``format!("{}", x)`` for the values a sign vector holds (+-1, NaN)."""
    if x != x:
        return "NaN"
    if float(x).is_integer():
        return str(int(x)) if x != 0 or np.copysign(1.0, x) > 0 else "-0"
    return repr(float(x))


@dataclass
class HardwarePhaseEvent:
    layer: int
    i: int
    j: int
    phi_l: float
    phi_r: float
    theta: float
    theta_l: float
    theta_r: float
    source: str
    kind: str
    energy_before: float | None = None
    energy_after: float | None = None


class HardwareSchedule:
    """Oracle restatement of ``HardwareSchedule`` (src/lie_svd_compiler.rs:43-266)."""

    def __init__(self, target: str, channels: int, events, diagonal_signs):
        self.format_version = "phase-schedule-v1"
        self.target = target
        self.channels = channels
        self.events = list(events)
        self.diagonal_signs = list(diagonal_signs)

    @staticmethod
    def from_orthogonal_matrix(v, target: str = "mzi_mesh") -> "HardwareSchedule":
        v = _c(v)
        d = v.shape[0]
        assert v.shape[1] == d, (
            f"HardwareSchedule::from_orthogonal_matrix: matrix must be square, got {d}x{v.shape[1]}")
        cap = d * (d - 1) // 2
        ei = np.empty(max(cap, 1), dtype=np.int64); ej = np.empty_like(ei)
        th = np.empty(max(cap, 1)); sg = np.empty(max(d, 1))
        cnt = lib().oracle_schedule_from_orthogonal(
            C.c_int64(d), _p(v), C.c_int64(cap), ei.ctypes.data_as(C.POINTER(C.c_int64)),
            ej.ctypes.data_as(C.POINTER(C.c_int64)), _p(th), _p(sg))
        assert cnt >= 0
        evs = [HardwarePhaseEvent(layer=k, i=int(ei[k]), j=int(ej[k]), phi_l=0.0, phi_r=0.0,
                                  theta=float(th[k]), theta_l=float(th[k]), theta_r=0.0,
                                  source="orthogonal_givens", kind="givens_elimination")
               for k in range(cnt)]
        return HardwareSchedule(target, d, evs, [float(x) for x in sg[:d]])

    @staticmethod
    def from_real_phaseflow(events, channels: int, target: str = "mzi_mesh") -> "HardwareSchedule":
        """``from_real_phaseflow`` (src/lie_svd_compiler.rs:59-88): events are
        MziPhase tuples (pass, i, j, theta_l, theta_r, kind name)."""
        evs = [HardwarePhaseEvent(layer=int(ps), i=int(i), j=int(j), phi_l=0.0, phi_r=0.0,
                                  theta=0.5 * (float(tl) + float(tr)), theta_l=float(tl), theta_r=float(tr),
                                  source="real_phaseflow", kind=str(kind))
               for ps, i, j, tl, tr, kind in events]
        return HardwareSchedule(target, channels, evs, [])

    def total_events(self) -> int:
        return len(self.events)

    def conflict_free_layer_count(self) -> int:
        return max((e.layer for e in self.events), default=-1) + 1

    def to_json_string(self) -> str:
        """``to_json_string`` (src/lie_svd_compiler.rs:213-265)."""
        out = ["{\n", f'  "format_version": "{self.format_version}",\n',
               f'  "target": "{self.target}",\n', f'  "channels": {self.channels},\n',
               f'  "total_events": {len(self.events)},\n', '  "events": [\n']
        for idx, e in enumerate(self.events):
            s = ('    {' f'"layer": {e.layer}, "i": {e.i}, "j": {e.j}, '
                 f'"phi_l": {fmt_e17(e.phi_l)}, "phi_r": {fmt_e17(e.phi_r)}, '
                 f'"theta": {fmt_e17(e.theta)}, "theta_l": {fmt_e17(e.theta_l)}, '
                 f'"theta_r": {fmt_e17(e.theta_r)}, "source": "{e.source}", "kind": "{e.kind}"')
            if e.energy_before is not None:
                s += f', "energy_before": {fmt_e17(e.energy_before)}'
            if e.energy_after is not None:
                s += f', "energy_after": {fmt_e17(e.energy_after)}'
            s += "}"
            if idx + 1 != len(self.events):
                s += ","
            out.append(s + "\n")
        out.append("  ]")
        if self.diagonal_signs:
            out.append(',\n  "diagonal_signs": [' +
                       ", ".join(fmt_display(x) for x in self.diagonal_signs) + "]")
        out.append("\n}\n")
        return "".join(out)
