"""B200-native (sm_100a) implementation of the dense rotor-schedule hot path of
the Rust crate ``lie_cliffalg_analog_svd`` v0.44.0.

The compute lives in ``_lib/liblsvd_b200.so`` (CUDA, C ABI in
``include/lsvd.h``); this package is the Python host mirror of the reference
API over that ABI.  Importing the package does not load the library;
the first call does, and fails loudly if it was not built.
"""
from .api import (Context, LieSvd, LieSvdMicro, LieSvdSmall, SmallResult, SvdMetrics,  # noqa: F401
                  HardwareSchedule, JointDiagonalizationParams, LieSvdJoint, default_context,
                  PolarResult, SvdStream, metrics, packed_offsets, polar, svd_batched,
                  svd_batched_stream, svd_vjp, unpack, svd_large, LargeResult,
                  LieSvdAdaptive, PhaseEngine, triage_batched, solvers)
from ._lib import LsvdError  # noqa: F401
from .dist import svd_batched_sharded  # noqa: F401
from .consumers import (CanonicalOrder, LieSvdBss, PhaseBssParams,  # noqa: F401
                        diagonalize_symmetric_canonicalized, solve_canonicalized)

__all__ = ["Context", "HardwareSchedule", "JointDiagonalizationParams", "LieSvdJoint", "LieSvd", "LieSvdMicro", "LieSvdSmall", "SmallResult", "SvdMetrics",
           "PolarResult", "SvdStream", "svd_batched_stream", "svd_vjp", "default_context", "metrics", "packed_offsets", "polar", "svd_batched", "unpack", "LsvdError", "svd_large", "LargeResult",
           "LieSvdAdaptive", "PhaseEngine", "triage_batched", "svd_batched_sharded", "solvers",
           "LieSvdBss", "PhaseBssParams", "CanonicalOrder", "solve_canonicalized",
           "diagonalize_symmetric_canonicalized"]
