"""ctypes binding of ``liblsvd_b200.so`` (the C ABI declared in
``include/lsvd.h``).  Loading fails loudly when the library is missing: there
is no CPU fallback anywhere in this package."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "liblsvd_b200.so")

# status codes (lsvd_status)
OK, NOT_CONVERGED, NONFINITE_INPUT, BAD_SHAPE, BAD_ARGUMENT, CUDA_ERROR, OUT_OF_MEMORY, \
    ROTOR_OVERFLOW, NO_DEVICE, UNSUPPORTED = range(10)
# flags
DEVICE_POINTERS, WANT_DIAG, ASYNC = 0x1, 0x2, 0x4
# per-matrix outcome bits
MAT_POLAR_UNTRUSTED, MAT_REPAIRED, MAT_NS_CAP, MAT_JACOBI_CAP, MAT_MICRO_FALLBACK, \
    MAT_NONFINITE, MAT_ROTOR_OVERFLOW, MAT_NS_DIVERGED = (1 << i for i in range(8))
ROUTE_MICRO, ROUTE_SMALL = 0, 1
PREC_FP64, PREC_MIXED_TF32, PREC_MIXED_BF16 = 0, 1, 2


class Diag(C.Structure):
    _fields_ = [("rel_recon", C.c_double), ("orth_u", C.c_double), ("orth_v", C.c_double),
                ("ns_iters", C.c_int32), ("jacobi_sweeps", C.c_int32), ("rotations", C.c_int64),
                ("flags", C.c_int32), ("route", C.c_int32)]


class Rotor(C.Structure):
    _fields_ = [("i", C.c_uint16), ("j", C.c_uint16), ("round", C.c_uint32),
                ("theta", C.c_double)]


DIAG_DTYPE = [("rel_recon", "<f8"), ("orth_u", "<f8"), ("orth_v", "<f8"), ("ns_iters", "<i4"),
              ("jacobi_sweeps", "<i4"), ("rotations", "<i8"), ("flags", "<i4"), ("route", "<i4")]
ROTOR_DTYPE = [("i", "<u2"), ("j", "<u2"), ("round", "<u4"), ("theta", "<f8")]
# lsvd_mzi_phase (MziPhase of the real PhaseFlow route) and the binary
# phase-schedule frame's header and record
MZI_PHASE_DTYPE = [("pass", "<i8"), ("i", "<i8"), ("j", "<i8"), ("theta_l", "<f8"), ("theta_r", "<f8"),
                   ("kind", "<i4"), ("pad_", "<i4")]
SCHED_HEADER_DTYPE = [("magic", "S8"), ("header_bytes", "<u4"), ("record_bytes", "<u4"), ("target", "<u4"),
                      ("flags", "<u4"), ("channels", "<i8"), ("total_events", "<i8"), ("n_signs", "<i8"),
                      ("reserved", "<i8", (2,))]
SCHED_RECORD_DTYPE = [("layer", "<u4"), ("i", "<u2"), ("j", "<u2"), ("phi_l", "<f8"), ("phi_r", "<f8"),
                      ("theta", "<f8"), ("theta_l", "<f8"), ("theta_r", "<f8"), ("source", "u1"), ("kind", "u1"),
                      ("reserved0", "<u2"), ("reserved1", "<u4")]
PHASE_ROTOR_KINDS = ("golden_prespin", "causal_antispin", "cross_phase_yinyang", "phase_conjugate",
                     "bottleneck", "phase_jump", "unwrap", "directional", "surgery")
SCHED_CANONICAL = 0x1
SCHED_ENERGY = 0x2


class JointParams(C.Structure):
    _fields_ = [("max_sweeps", C.c_int32), ("tol", C.c_double), ("min_pair_scale", C.c_double),
                ("line_search_steps", C.c_int32)]


class JointTrace(C.Structure):
    _fields_ = [("initial_offdiag", C.c_double), ("final_offdiag", C.c_double),
                ("sweeps", C.c_int64), ("rotations", C.c_int64), ("rejected_rotations", C.c_int64)]


class PolarInfo(C.Structure):
    _fields_ = [("iters_lowp", C.c_int32), ("iters_fp64", C.c_int32), ("orth", C.c_double),
                ("flops_lowp", C.c_double), ("flops_fp64", C.c_double),
                ("gemm_ms_lowp", C.c_double), ("gemm_ms_fp64", C.c_double), ("converged", C.c_int32),
                ("pad_", C.c_int32)]


class LargeInfo(C.Structure):
    _fields_ = [("ns_iters_lowp", C.c_int32), ("ns_iters_fp64", C.c_int32), ("sweeps_lowp", C.c_int32),
                ("sweeps_fp64", C.c_int32), ("rotations", C.c_int64), ("flags", C.c_int32),
                ("inner_cap_pairs", C.c_int32), ("last_offdiag", C.c_double), ("flops_fp64", C.c_double),
                ("flops_lowp", C.c_double), ("ms_polar", C.c_double), ("ms_eig_lowp", C.c_double),
                ("ms_eig_fp64", C.c_double), ("ms_total", C.c_double), ("rel_recon", C.c_double),
                ("orth_u", C.c_double), ("orth_v", C.c_double)]


TRIAGE_FIELDS = ("offdiag_ratio", "diagonal_dominance", "row_cv", "col_cv", "row_col_mismatch",
                 "symmetry_ratio", "transpose_torsion_ratio", "diagonal_entropy", "row_mass_entropy",
                 "col_mass_entropy", "suspicious_score", "mean_stress", "max_twist", "causal_disbalance",
                 "entropy_gap", "global_phase", "torsion_energy", "chirality_balance", "phase_entropy",
                 "chirality", "golden_resonance")


class Triage(C.Structure):
    _fields_ = [(f, C.c_double) for f in TRIAGE_FIELDS] + [("adaptive_route", C.c_int32),
                                                             ("passport_route", C.c_int32)]


TRIAGE_DTYPE = [(f, "<f8") for f in TRIAGE_FIELDS] + [("adaptive_route", "<i4"), ("passport_route", "<i4")]


class LsvdError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"lsvd status {status}: {msg}")
        self.status = status


_lib = None

P = C.c_void_p
I64 = C.c_int64
U32 = C.c_uint32

SIGNATURES = {
    "lsvd_version": (C.c_char_p, []),
    "lsvd_status_string": (C.c_char_p, [C.c_int]),
    "lsvd_context_create": (C.c_int, [C.c_int, C.POINTER(P)]),
    "lsvd_context_destroy": (C.c_int, [P]),
    "lsvd_context_set_stream": (C.c_int, [P, P]),
    "lsvd_context_get_stream": (P, [P]),
    "lsvd_synchronize": (C.c_int, [P]),
    "lsvd_context_last_error": (C.c_char_p, [P]),
    "lsvd_context_kernel_launches": (I64, [P]),
    "lsvd_small_solve_f64": (C.c_int, [P, I64, P, I64, P, I64, P, P, I64, P, P, I64, P, P, U32]),
    "lsvd_micro_solve_f64": (C.c_int, [P, I64, P, I64, P, I64, P, P, I64, P, U32]),
    "lsvd_small_solve_rectangular_f64": (C.c_int, [P, I64, I64, P, I64, P, I64, P, P, I64, P,
                                                   U32]),
    "lsvd_svd_batched_f64": (C.c_int, [P, I64, P, P, P, P, P, P, C.c_int, U32]),
    "lsvd_svd_large_f64": (C.c_int, [P, I64, I64, P, I64, P, I64, P, P, I64, C.c_int, P, U32]),
    "lsvd_autotune_f64": (C.c_int, [P, I64, C.c_char_p, P, I64]),
    "lsvd_triage_batched_f64": (C.c_int, [P, I64, P, P, P, P, U32]),
    "lsvd_class_shapes": (C.c_int, [P, C.c_int, P]),
    "lsvd_metrics_f64": (C.c_int, [P, I64, I64, I64, P, P, P, P, P, P, U32]),
    "lsvd_svd_batched_noalloc_f64": (C.c_int, [P, I64, P, P, P, P, P, P, U32]),
    "lsvd_joint_params_for_n": (JointParams, [I64]),
    "lsvd_jade_sym_f64": (C.c_int, [P, I64, I64, I64, P, P, P, P, P, U32]),
    "lsvd_joint_svd_f64": (C.c_int, [P, I64, I64, I64, I64, P, P, P, P, P, P, U32]),
    "lsvd_polar_f64": (C.c_int, [P, I64, I64, P, I64, P, I64, C.c_int, P, U32]),
    "lsvd_gemm_nt_lowp": (C.c_int, [P, I64, I64, I64, P, P, P, C.c_int]),
    "lsvd_gemm_f64": (C.c_int, [P, C.c_int32, C.c_int32, I64, I64, I64, C.c_double, P, I64, P, I64,
                                C.c_double, P, I64]),
    "lsvd_svd_batched_stream_f64": (C.c_int, [P, I64, I64, I64, P, P, P, P, P, I64, P, P, P, U32]),
    "lsvd_svd_vjp_f64": (C.c_int, [P, I64, I64, I64, P, P, P, P, I64, P, P, P, P, P, P,
                                   C.c_double, P, U32]),
    "lsvd_schedule_from_orthogonal": (C.c_int, [I64, P, C.c_int32, P, I64, C.POINTER(I64)]),
    "lsvd_schedule_from_rotors": (C.c_int, [P, I64, I64, C.c_int32, P, I64, C.POINTER(I64)]),
    "lsvd_schedule_from_real_phaseflow": (C.c_int, [P, I64, I64, C.c_int32, P, I64, C.POINTER(I64)]),
    "lsvd_schedule_binary_from_rotors": (C.c_int, [P, P, I64, I64, C.c_int32, P, I64, C.POINTER(I64),
                                                   C.c_uint32]),
    "lsvd_schedule_binary_from_real_phaseflow": (C.c_int, [P, I64, I64, C.c_int32, P, I64, C.POINTER(I64)]),
    "lsvd_schedule_binary_to_json": (C.c_int, [P, I64, P, I64, C.POINTER(I64)]),
}

OPTIONAL_SIGNATURES: dict = {}


def load() -> C.CDLL:
    """Loads the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA extension with "
            "`python -m lie_cliffalg_analog_svd_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in {**SIGNATURES, **OPTIONAL_SIGNATURES}.items():
        if not hasattr(lib, name):
            if name in OPTIONAL_SIGNATURES:
                continue
            raise ImportError(f"{LIB_PATH} does not export {name}")
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return sorted(SIGNATURES)
