/*
 * lsvd.h -- C ABI of liblsvd_b200.so, the B200 (sm_100a) implementation of the
 * dense rotor-schedule hot path of the Rust crate `lie_cliffalg_analog_svd`
 * v0.44.0: polar/Jacobi SVD, the n<=4 micro kernels, Newton-Schulz polar,
 * Phase-JADE joint diagonalisation, the rotor stream that the
 * phase-schedule-v1 compiler consumes, and the SVD diagnostics.
 *
 * Conventions (all entry points):
 *   - matrices are dense row-major f64 (`ndarray::Array2<f64>` standard
 *     layout), with an explicit leading dimension where one is taken;
 *   - pointers are HOST pointers unless `LSVD_DEVICE_POINTERS` is set in
 *     `flags`, in which case every array argument (except the per-matrix
 *     size array `n` of batched calls, which is always host memory) is
 *     device memory on the context's device;
 *   - every entry point returns an `lsvd_status`; nothing traps, throws
 *     across the ABI or exits; the reference's `assert!` panics on bad
 *     shapes become `LSVD_BAD_SHAPE`;
 *   - a context owns one CUDA stream and its workspaces and is not
 *     thread-safe: use one context per host thread;
 *   - host-pointer calls are synchronous; device-pointer calls with
 *     `LSVD_ASYNC` return after enqueueing on the context's stream.
 */
#ifndef LSVD_H
#define LSVD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LSVD_API __attribute__((visibility("default")))

typedef enum lsvd_status {
    LSVD_OK = 0,
    LSVD_NOT_CONVERGED = 1,   /* an iteration cap was hit; results are returned */
    LSVD_NONFINITE_INPUT = 2, /* NaN/Inf in the input; outputs are NaN */
    LSVD_BAD_SHAPE = 3,       /* the reference would panic (assert!) */
    LSVD_BAD_ARGUMENT = 4,    /* NULL pointer, bad leading dimension, bad flag */
    LSVD_CUDA_ERROR = 5,      /* see lsvd_context_last_error */
    LSVD_OUT_OF_MEMORY = 6,
    LSVD_ROTOR_OVERFLOW = 7,  /* rotor buffer too small; count holds the need */
    LSVD_NO_DEVICE = 8,
    LSVD_UNSUPPORTED = 9      /* size or option outside what the library supports */
} lsvd_status;

/* flags */
#define LSVD_DEVICE_POINTERS 0x1u /* array arguments are device pointers */
#define LSVD_WANT_DIAG 0x2u       /* fill rel_recon / orth_u / orth_v in lsvd_diag */
#define LSVD_ASYNC 0x4u           /* with device pointers: do not synchronise */

/* per-matrix outcome bits (lsvd_diag.flags) */
#define LSVD_MAT_POLAR_UNTRUSTED 0x01 /* newton_schulz_polar returned ok=false */
#define LSVD_MAT_REPAIRED 0x02        /* U rebuilt by repair_left_basis_from_right */
#define LSVD_MAT_NS_CAP 0x04          /* 120 Newton-Schulz iterations without convergence */
#define LSVD_MAT_JACOBI_CAP 0x08      /* Jacobi sweep cap hit */
#define LSVD_MAT_MICRO_FALLBACK 0x10  /* LieSvdMicro escalated to LieSvdSmall */
#define LSVD_MAT_NONFINITE 0x20       /* non-finite input */
#define LSVD_MAT_ROTOR_OVERFLOW 0x40  /* rotor stream truncated */
#define LSVD_MAT_NS_DIVERGED 0x80     /* polar iteration diverged -> MGS(A) */

/* route (lsvd_diag.route) */
#define LSVD_ROUTE_MICRO 0
#define LSVD_ROUTE_SMALL 1

typedef struct lsvd_diag {
    double rel_recon; /* ||U S Vt - A||_F / ||A||_F      (src/lib.rs:158-159) */
    double orth_u;    /* ||U^T U - I||_F                  (src/lib.rs:161)     */
    double orth_v;    /* ||Vt Vt^T - I||_F                (src/lib.rs:162)     */
    int32_t ns_iters;      /* Newton-Schulz iterations executed */
    int32_t jacobi_sweeps; /* Jacobi sweeps started */
    int64_t rotations;     /* accepted plane rotations */
    int32_t flags;         /* LSVD_MAT_* bits */
    int32_t route;         /* LSVD_ROUTE_* */
} lsvd_diag;

/* One accepted plane rotation of the right basis: V <- V G, where G acts on
 * columns (i, j), i < j, as  v_i' = cos(theta) v_i - sin(theta) v_j,
 * v_j' = sin(theta) v_i + cos(theta) v_j  (the apply_basis_rotor convention,
 * src/lie_svd_joint.rs:428-437).  `round` numbers conflict-free layers:
 * round = sweep * layers_per_sweep + layer. */
typedef struct lsvd_rotor {
    uint16_t i;
    uint16_t j;
    uint32_t round;
    double theta;
} lsvd_rotor;

typedef enum lsvd_precision {
    LSVD_PREC_FP64 = 0,       /* the reference algorithm in FP64 throughout */
    LSVD_PREC_MIXED_TF32 = 1, /* TF32 tensor-core bulk + FP64 refinement/cleanup */
    LSVD_PREC_MIXED_BF16 = 2  /* BF16 tensor-core bulk + FP64 refinement/cleanup */
} lsvd_precision;

typedef struct lsvd_context lsvd_context;

LSVD_API const char* lsvd_version(void);
LSVD_API const char* lsvd_status_string(lsvd_status s);

LSVD_API lsvd_status lsvd_context_create(int device, lsvd_context** out);
LSVD_API lsvd_status lsvd_context_destroy(lsvd_context* ctx);
/* Use `stream` (a cudaStream_t) instead of the context's own stream. */
LSVD_API lsvd_status lsvd_context_set_stream(lsvd_context* ctx, void* stream);
LSVD_API void* lsvd_context_get_stream(lsvd_context* ctx);
LSVD_API lsvd_status lsvd_synchronize(lsvd_context* ctx);
LSVD_API const char* lsvd_context_last_error(const lsvd_context* ctx);
/* Number of kernels this context has launched since creation. */
LSVD_API int64_t lsvd_context_kernel_launches(const lsvd_context* ctx);

/* ---------------------------------------------------------------- SVD ---- */

/* Replaces LieSvdSmall::solve (src/lie_svd_small.rs:296-323): Newton-Schulz
 * polar A = QP, P = sym(Q^T A), Jacobi eigensolve of P, U = QV, left-basis
 * repair.  A n*n (lda), U n*n (ldu), S n (descending), Vt n*n (ldvt).
 * n in 1..64 runs on one CTA with everything in shared memory; `rotors` (may
 * be NULL) receives the accepted rotation stream of the eigensolve, up to
 * rotor_cap entries; *rotor_count gets the number produced.  `perm` (may be
 * NULL, n int32) receives the sort permutation: column k of the returned V is
 * column perm[k] of the rotor-stream product.  n in 65..16384 runs the
 * blocked solve of lsvd_svd_large_f64 (rotors, rotor_count and perm must then
 * be NULL: its block rotations are not a plane-rotation stream). */
LSVD_API lsvd_status lsvd_small_solve_f64(lsvd_context* ctx, int64_t n, const double* A,
                                          int64_t lda, double* U, int64_t ldu, double* S,
                                          double* Vt, int64_t ldvt, lsvd_diag* diag,
                                          lsvd_rotor* rotors, int64_t rotor_cap,
                                          int64_t* rotor_count, int32_t* perm, uint32_t flags);

/* Replaces LieSvdMicro::solve (src/lie_svd_micro.rs:21-52), n in 0..4. */
LSVD_API lsvd_status lsvd_micro_solve_f64(lsvd_context* ctx, int64_t n, const double* A,
                                          int64_t lda, double* U, int64_t ldu, double* S,
                                          double* Vt, int64_t ldvt, lsvd_diag* diag,
                                          uint32_t flags);

/* Replaces LieSvdSmall::solve_rectangular (src/lie_svd_small.rs:340-360):
 * thin SVD of an m*d matrix via QR reduction; k = min(m, d);
 * U m*k, S k, Vt k*d.  min(m, d) in 1..64 on the shared-memory kernels;
 * larger min(m, d) (up to 16384, max(m, d) up to 65536) through
 * lsvd_svd_large_f64's thin route. */
LSVD_API lsvd_status lsvd_small_solve_rectangular_f64(lsvd_context* ctx, int64_t m, int64_t d,
                                                      const double* A, int64_t lda, double* U,
                                                      int64_t ldu, double* S, double* Vt,
                                                      int64_t ldvt, lsvd_diag* diag,
                                                      uint32_t flags);

/* Diagnostics of lsvd_svd_large_f64 (phase times are CUDA-event times on
 * the context's stream). */
typedef struct lsvd_large_info {
    int32_t ns_iters_lowp;   /* TF32/BF16 Newton-Schulz iterations */
    int32_t ns_iters_fp64;   /* FP64 Newton-Schulz iterations */
    int32_t sweeps_lowp;     /* low-precision Jacobi sweeps (mixed routes) */
    int32_t sweeps_fp64;     /* FP64 Jacobi sweeps */
    int64_t rotations;       /* plane rotations inside the block solves */
    int32_t flags;           /* LSVD_MAT_* bits */
    int32_t inner_cap_pairs; /* block pairs whose inner sweeps hit their cap */
    double last_offdiag;     /* largest |g_i.g_j|/(|g_i||g_j|) seen in the last sweep */
    double flops_fp64;       /* executed FP64 flops (GEMMs, Gram and apply products) */
    double flops_lowp;       /* executed TF32/BF16 flops */
    double ms_polar;         /* Newton-Schulz phase */
    double ms_eig_lowp;      /* low-precision eigensolve */
    double ms_eig_fp64;      /* FP64 Jacobi sweeps */
    double ms_total;         /* device time from the polar phase to U */
    double rel_recon;        /* with LSVD_WANT_DIAG: ||U S Vt - A||_F / ||A||_F (src/lib.rs:158-159) */
    double orth_u;           /* ||U^T U - I||_F */
    double orth_v;           /* ||Vt Vt^T - I||_F */
} lsvd_large_info;

/* SVD of one large dense matrix (no size class of its own in the reference:
 * LieSvdSmall::solve, src/lie_svd_small.rs:296-323, and solve_rectangular,
 * :340-360, run at any size; the reference routes up to n = 512 there,
 * src/lie_svd_adaptive.rs:71).  A m x n (lda); k = min(m, n); U m x k (ldu),
 * S k (descending), Vt k x n (ldvt).
 *   LSVD_PREC_FP64: Newton-Schulz polar factor Q of A (or of A^T when n > m)
 *     on the FP64 tensor path, P = sym(Q^T A), V by blocked two-sided Jacobi
 *     on P (blocks of 32 indices, 64 x 64 block-pair rotations applied as
 *     FP64 tensor products, the reference's stop test off(P) < 1e-13 ||P||_F
 *     evaluated on the device), sigma = max(lambda, 0) from the Rayleigh
 *     quotients, U = Q V.
 *   LSVD_PREC_MIXED_TF32/BF16 (m, n multiples of 128): the Newton-Schulz
 *     bulk on the tcgen05 tensor cores gives Q0; the eigensolve of
 *     P0 = sym(Q0^T A) stops at the low-precision level (4 u ||P0||_F) and
 *     gives V0; FP64 blocked one-sided Jacobi on W = A V0 then orthogonalises
 *     the columns (accuracy comes from this FP64 stage on A itself):
 *     sigma_j = ||w_j||, U = W diag(sigma)^-1, V = V0 R.  A zero singular
 *     value leaves its U column zero (LSVD_MAT_REPAIRED set in info.flags).
 * Host or device pointers (LSVD_DEVICE_POINTERS); synchronous.  `info` may
 * be NULL. */
LSVD_API lsvd_status lsvd_svd_large_f64(lsvd_context* ctx, int64_t m, int64_t n, const double* A, int64_t lda,
                                        double* U, int64_t ldu, double* S, double* Vt, int64_t ldvt,
                                        lsvd_precision precision, lsvd_large_info* info, uint32_t flags);

/* Batched uneven SVD (no reference counterpart; each matrix takes the route
 * LieSvd::solve's exact tiers take: LieSvdMicro for n<=4
 * (src/lie_svd_adaptive.rs:105-106), LieSvdSmall otherwise).
 * Matrix t is n[t]*n[t] (n[t] in 1..64); A, U and Vt hold the matrices back
 * to back (row-major, no padding), S the singular values back to back.
 * `n` is host memory.  `diags` (may be NULL) gets one lsvd_diag per matrix.
 * The per-size schedule (sort, work items, tile shapes) is planned once per
 * distinct `n` array and cached in the context together with a captured CUDA
 * graph. */
LSVD_API lsvd_status lsvd_svd_batched_f64(lsvd_context* ctx, int64_t count, const int32_t* n,
                                          const double* A, double* U, double* S, double* Vt,
                                          lsvd_diag* diags, lsvd_precision precision,
                                          uint32_t flags);

/* Autotuner of the batched FP64 kernel (no counterpart in the reference):
 * for every size class (n = 5..8, 9..16, 17..24, 25..32, 33..48, 49..64)
 * times each feasible team shape (warps per team, GEMM register tile, lanes
 * per Jacobi pair, matrices per team) on a seeded batch of `per_class`
 * matrices (16..100000) with CUDA events on the context's stream, and writes
 * the fastest to the shape cache (`cache_path`, or NULL for
 * LSVD_AUTOTUNE_CACHE / $HOME/.cache/lsvd_b200/shapes.json) that the batched
 * planner reads; the context's cached plans are dropped.  `report` (may be
 * NULL) receives one line per class with the chosen and the default shape
 * and their times.  Synchronous. */
LSVD_API lsvd_status lsvd_autotune_f64(lsvd_context* ctx, int64_t per_class, const char* cache_path,
                                       char* report, int64_t report_cap);
/* The team shapes the batched planner uses now for `precision`
 * (LSVD_SHAPES, then the autotune cache, then the built-in defaults):
 * out[4c .. 4c+3] = warps per team, register tile, lanes per Jacobi pair,
 * matrices per team for size class c = 0..7 (out holds 32 int32). */
LSVD_API lsvd_status lsvd_class_shapes(lsvd_context* ctx, lsvd_precision precision, int32_t* out);

/* No counterpart in the reference.  The batched FP64 SVD of
 * lsvd_svd_batched_f64 for callers that cannot allocate device memory:
 * latency-critical loops that cannot absorb the device-wide synchronisation
 * of cudaMalloc/cudaFree, and hosts whose device memory belongs to their own
 * allocator or pool.  It allocates nothing: A, U, S, Vt (and diags, may be
 * NULL) are DEVICE buffers of the caller in the packed layout of
 * lsvd_svd_batched_f64, `n` is host memory, `stream` a cudaStream_t of the
 * current device (NULL = legacy default stream), and all working memory is a
 * static device array of LSVD_NOALLOC_SCRATCH_BYTES that every GPU loading
 * the library holds until exit.  At most LSVD_NOALLOC_MAX_COUNT matrices per
 * call (more returns LSVD_UNSUPPORTED).  The first successful call on a
 * device sets that device up (the array's device address, kernel
 * attributes); a failed set-up is retried by the next call.  Calls share the
 * static array, so calls that overlap on a GPU race; serialise them.
 * Without LSVD_ASYNC the call synchronises `stream` and reports the outcome
 * like lsvd_svd_batched_f64.  With LSVD_ASYNC it only enqueues work: `n` is
 * then copied to the device when the stream reaches the copy, so a pinned
 * (page-locked) `n` must stay alive and unchanged until the stream has run
 * past the call (a pageable `n` is read before the call returns); sizes that
 * left 1..64 in between are caught on the device and nothing is solved. */
#define LSVD_NOALLOC_MAX_COUNT 65536
#define LSVD_NOALLOC_SCRATCH_BYTES (4096 + 44 * LSVD_NOALLOC_MAX_COUNT)
LSVD_API lsvd_status lsvd_svd_batched_noalloc_f64(void* stream, int64_t count, const int32_t* n,
                                                  const double* A, double* U, double* S,
                                                  double* Vt, lsvd_diag* diags, uint32_t flags);

/* Replaces metrics::compute (src/lib.rs:149-194) for one matrix (general
 * thin shape: A m*d, U m*k, S k, Vt k*d).  out[0..4] = rel_recon, orth_u,
 * orth_v, sigma_max_rel, sigma_tail_rel (NaN when sigma_ref is NULL). */
LSVD_API lsvd_status lsvd_metrics_f64(lsvd_context* ctx, int64_t m, int64_t d, int64_t k,
                                      const double* A, const double* U, const double* S,
                                      const double* Vt, const double* sigma_ref, double* out,
                                      uint32_t flags);

/* --------------------------------------------------------- Phase-JADE ---- */

/* JointDiagonalizationParams (src/lie_svd_joint.rs:18-35). */
typedef struct lsvd_joint_params {
    int32_t max_sweeps;
    double tol;
    double min_pair_scale;
    int32_t line_search_steps;
} lsvd_joint_params;

/* JointDiagonalizationTrace (src/lie_svd_joint.rs:43-50). */
typedef struct lsvd_joint_trace {
    double initial_offdiag;
    double final_offdiag;
    int64_t sweeps;
    int64_t rotations;
    int64_t rejected_rotations;
} lsvd_joint_trace;

/* JointDiagonalizationParams::for_n (src/lie_svd_joint.rs:27-34). */
LSVD_API lsvd_joint_params lsvd_joint_params_for_n(int64_t n);

/* Replaces LieSvdJoint::diagonalize_symmetric_with_params
 * (src/lie_svd_joint.rs:71-158) for `families` independent families at once.
 * M: families x K matrices of n x n, back to back (row-major); V: families x
 * n x n (the shared basis, columns = joint eigenvectors); diag: families x K
 * x n (the diagonals of V^T M_k V); traces: `families` entries, HOST memory
 * always.  params NULL = lsvd_joint_params_for_n(n).  K in 1..93. */
LSVD_API lsvd_status lsvd_jade_sym_f64(lsvd_context* ctx, int64_t families, int64_t K, int64_t n,
                                       const double* M, const lsvd_joint_params* params,
                                       double* V, double* diag, lsvd_joint_trace* traces,
                                       uint32_t flags);

/* Replaces LieSvdJoint::joint_svd_with_params (src/lie_svd_joint.rs:170-261)
 * for `families` independent families at once.  M: families x K matrices of
 * rows x cols, back to back (row-major); U: families x rows x rows (left
 * basis); sig: families x K x min(rows, cols) (|diag| of U^T M_k V, the
 * reference's diagonal_corridor); Vt: families x cols x cols; traces: HOST
 * memory always.  params NULL = lsvd_joint_params_for_n(min(rows, cols)).
 * K <= 90 and max(rows, cols) up to ~500 (shared memory). */
LSVD_API lsvd_status lsvd_joint_svd_f64(lsvd_context* ctx, int64_t families, int64_t K, int64_t rows,
                                        int64_t cols, const double* M, const lsvd_joint_params* params,
                                        double* U, double* sig, double* Vt, lsvd_joint_trace* traces,
                                        uint32_t flags);

/* ----------------------------------------------------------- triage ---- */

/* Routing statistics of one matrix: AdaptiveTriage (src/lie_svd_adaptive.rs:
 * 14-34; NaN unless square), PhaseSignature with its GlobalPhaseInvariants
 * (src/lie_svd_phasehealth.rs:42-98) and the PhasePassport extras
 * (src/lie_svd_engine.rs:34-61). */
typedef struct lsvd_triage {
    double offdiag_ratio, diagonal_dominance, row_cv, col_cv, row_col_mismatch;
    double symmetry_ratio, transpose_torsion_ratio, diagonal_entropy, row_mass_entropy, col_mass_entropy;
    double suspicious_score;
    double mean_stress, max_twist, causal_disbalance, entropy_gap;
    double global_phase, torsion_energy, chirality_balance, phase_entropy;
    double chirality, golden_resonance;
    /* choose_route with LieSvdAdaptiveParams::default() (:84-119): 0 Micro,
     * 1 Small, 2 PhaseFlow, 3 CoreFlowTopo, 4 Hybrid; -1 for non-square */
    int32_t adaptive_route;
    /* PhaseEngine::passport_real's route_hint (src/lie_svd_engine.rs:75-82):
     * 0 RealSmall, 1 RealPhaseFlowPolished */
    int32_t passport_route;
} lsvd_triage;

/* Replaces analyze_matrix + choose_route (src/lie_svd_adaptive.rs:84-274),
 * phase_signature (src/lie_svd_phasehealth.rs:129-140) and the statistics
 * of PhaseEngine::passport_real (src/lie_svd_engine.rs:75-103) for a batch:
 * matrix t is rows[t] x cols[t] (each <= 4096), row-major, back to back in
 * A; out gets one lsvd_triage per matrix.  rows/cols are host memory; A and
 * out host or device (LSVD_DEVICE_POINTERS); with LSVD_ASYNC and device
 * pointers the call only enqueues.  One CTA per matrix. */
LSVD_API lsvd_status lsvd_triage_batched_f64(lsvd_context* ctx, int64_t count, const int32_t* rows,
                                             const int32_t* cols, const double* A, lsvd_triage* out,
                                             uint32_t flags);

/* ------------------------------------------------ large polar factor ---- */
/* Polar factor Q (m x n, Q^T Q = I) of a large dense A (m >= n) by the
 * Newton-Schulz iteration X <- X (3I - X^T X)/2 from X0 = A/||A||_F.
 * Replaces newton_schulz_polar (src/lie_svd_small.rs:158-183) -- the
 * reference applies it to square n <= 64 matrices inside LieSvdSmall::solve;
 * this entry runs the same iteration and stopping rule on large m x n inputs:
 *   LSVD_PREC_FP64       : FP64 GEMMs throughout, delta < 1e-13 sqrt(n) (cap 120);
 *   LSVD_PREC_MIXED_TF32 : tcgen05 TF32 products (FP32 accumulation) until the
 *   LSVD_PREC_MIXED_BF16   update reaches the low-precision floor, then FP64
 *                          refinement iterations to delta < 1e-13 sqrt(n).
 * The mixed precisions need m and n to be multiples of 128.  Singular values
 * of A below ~u sigma_1 (u = 2^-11 TF32, 2^-8 BF16) are not resolved by the
 * low-precision phase: the result is then orthogonal to working precision but
 * differs from A's polar factor in that subspace.  Returns LSVD_NOT_CONVERGED
 * (with Q written) when the cap is reached or the iteration diverged. */
typedef struct lsvd_polar_info {
    int32_t iters_lowp; /* TF32/BF16 iterations */
    int32_t iters_fp64; /* FP64 iterations (refinement, or all for FP64) */
    double orth;        /* ||Q^T Q - I||_F of the returned factor */
    double flops_lowp;  /* 4 m n^2 per low-precision iteration */
    double flops_fp64;  /* 4 m n^2 per FP64 iteration */
    double gemm_ms_lowp; /* summed CUDA-event durations of the TF32/BF16 GEMM launches */
    double gemm_ms_fp64; /* ... and of the FP64 iteration GEMM launches */
    int32_t converged;
    int32_t pad_;
} lsvd_polar_info;

LSVD_API lsvd_status lsvd_polar_f64(lsvd_context* ctx, int64_t m, int64_t n, const double* A,
                                    int64_t lda, double* Q, int64_t ldq, lsvd_precision precision,
                                    lsvd_polar_info* info, uint32_t flags);

/* C = A B^T (FP32, row-major M x N) with A (M x K), B (N x K) rounded to TF32
 * or BF16 and multiplied on the tcgen05 tensor cores with FP32 accumulation:
 * the product kernel of the mixed polar iteration, exposed for testing.
 * Device pointers; M, N multiples of 128, K of 32 (TF32) or 64 (BF16).
 * No counterpart in the reference. */
LSVD_API lsvd_status lsvd_gemm_nt_lowp(lsvd_context* ctx, int64_t M, int64_t N, int64_t K,
                                       const float* A, const float* B, float* C,
                                       lsvd_precision precision);

/* C = alpha op(A) op(B) + beta C in FP64 (row-major; op(X) = X^T when
 * trans_x != 0) on the FP64 tensor path (mma.sync m8n8k4): the product
 * kernel of the FP64 polar iteration and of the large SVD (the reference's
 * ndarray .dot, src/lie_svd_small.rs:172-173, :305, :313), also the
 * products of the Phase-BSS and canonical-order consumers
 * (src/lie_svd_bss.rs:64, :74, :81-82, :179-186; src/phase_normalizer.rs:109, :140).
 * Few output tiles over K >= 4096 split K across the SMs into partials in the
 * context's workspace, reduced in a second launch (A B^T with M, N <= 64 on
 * CUDA-core slices, larger outputs as batched tensor-core slices).  Device
 * pointers; lda, ldb even and A, B 16-byte aligned; enqueued on the
 * context's stream without synchronising. */
LSVD_API lsvd_status lsvd_gemm_f64(lsvd_context* ctx, int32_t trans_a, int32_t trans_b, int64_t M,
                                   int64_t N, int64_t K, double alpha, const double* A, int64_t lda,
                                   const double* B, int64_t ldb, double beta, double* C, int64_t ldc);

/* ------------------------------------------- rotor stream and adjoint ---- */
/* Batched thin SVD of `count` matrices of one shape m x n (m >= n, n <= 64,
 * m <= 4096; packed row-major), keeping each matrix's accepted rotor stream
 * and sort permutation so that U and V need not be stored.  Tall inputs go
 * through qr_reduce (src/lie_svd_small.rs:373-418) and the square solve of R,
 * square ones through the solve directly -- LieSvdSmall::solve
 * (src/lie_svd_small.rs:296-336) for every n (no LieSvdMicro route here).
 * Matrix t's stream is rotors[t*rotor_cap ..][0 .. rotor_count[t]); with
 * perm[t*n ..] it gives V = G_1 G_2 ... G_k P (G_r rotates columns i, j by
 * theta: v_i <- c v_i - s v_j, v_j <- s v_i + c v_j; P[:, j] = e_perm[j]).
 * U (m x n) and Vt (n x n) may be NULL.  A stream longer than rotor_cap
 * returns LSVD_ROTOR_OVERFLOW.  Host or device pointers (LSVD_DEVICE_POINTERS);
 * synchronous.  No counterpart in the reference. */
LSVD_API lsvd_status lsvd_svd_batched_stream_f64(lsvd_context* ctx, int64_t count, int64_t m, int64_t n,
                                                 const double* A, double* U, double* S, double* Vt,
                                                 lsvd_rotor* rotors, int64_t rotor_cap,
                                                 int64_t* rotor_count, int32_t* perm, lsvd_diag* diags,
                                                 uint32_t flags);

/* Vector-Jacobian product of the thin SVD A = U diag(S) V^T and of its polar
 * factor Q = U V^T: given the forward's A, S, perm and rotor stream (as
 * written by lsvd_svd_batched_stream_f64) and cotangents Ubar (m x n), Sbar
 * (n), Vbar (n x n, of V -- not of Vt) and Qbar (m x n), each may be NULL,
 * writes Abar (m x n) for every matrix.  V is rebuilt by replaying the stream
 * in reverse and U = A V S^-1 is recomputed; nothing of U or V is stored.
 * The analytic thin-SVD adjoint with F_ij = 1/(s_j^2 - s_i^2) is used; F_ij
 * is taken as 0 where |s_i - s_j| <= gap_tol * max(S) (gap_tol = 0: exact
 * formula).  Needs S > 0 (else LSVD_BAD_ARGUMENT and that Abar zeroed).
 * Vt (n x n per matrix) may be NULL; when given, V is read from it instead of
 * replayed (the path that keeps V, for comparison; perm/rotors then unused).
 * Host or device pointers; synchronous.  No counterpart in the reference. */
LSVD_API lsvd_status lsvd_svd_vjp_f64(lsvd_context* ctx, int64_t count, int64_t m, int64_t n,
                                      const double* A, const double* S, const int32_t* perm,
                                      const lsvd_rotor* rotors, int64_t rotor_cap,
                                      const int64_t* rotor_count, const double* Ubar,
                                      const double* Sbar, const double* Vbar, const double* Qbar,
                                      const double* Vt, double gap_tol, double* Abar, uint32_t flags);

/* ----------------------------------------------------- rotor schedule ---- */
/* target: 0 = "mzi_mesh", 1 = "fpga_rotor_mesh" (HardwareTarget,
 * src/lie_svd_compiler.rs:12-25).  The JSON text (NUL-terminated) is written
 * to json[0..cap); *len receives its length without the NUL.  A too-small
 * buffer returns LSVD_ROTOR_OVERFLOW with *len set (pass json=NULL to size).
 * Host-side serialisation; no GPU is needed. */

/* Replaces HardwareSchedule::from_orthogonal_matrix + to_json_string
 * (src/lie_svd_compiler.rs:144-198, :213-265).  V d*d row-major. */
LSVD_API lsvd_status lsvd_schedule_from_orthogonal(int64_t d, const double* V, int32_t target,
                                                   char* json, int64_t cap, int64_t* len);

/* phase-schedule-v1 schedule of a rotor stream (lsvd_small_solve_f64's
 * `rotors`): one event per accepted rotation, layer = round, in the
 * compiler's reconstruction convention (src/lie_svd_compiler.rs:396-411),
 * source "gpu_jacobi", kind "jacobi_rotation".  It reconstructs the
 * eigenbasis before the descending sort; the solver's `perm` orders it. */
LSVD_API lsvd_status lsvd_schedule_from_rotors(const lsvd_rotor* rotors, int64_t count,
                                               int64_t channels, int32_t target, char* json,
                                               int64_t cap, int64_t* len);

/* One event of the real PhaseFlow route: MziPhase (src/lie_svd_phaseflow.rs:
 * 202-209); kind = the PhaseRotorKind variant's position (:189-199),
 * LSVD_ROTOR_KIND_*. */
typedef struct lsvd_mzi_phase {
    int64_t pass;
    int64_t i;
    int64_t j;
    double theta_l;
    double theta_r;
    int32_t kind;
    int32_t pad_;
} lsvd_mzi_phase;

#define LSVD_ROTOR_KIND_GOLDEN_PRESPIN 0
#define LSVD_ROTOR_KIND_CAUSAL_ANTISPIN 1
#define LSVD_ROTOR_KIND_CROSS_PHASE_YINYANG 2
#define LSVD_ROTOR_KIND_PHASE_CONJUGATE 3
#define LSVD_ROTOR_KIND_BOTTLENECK 4
#define LSVD_ROTOR_KIND_PHASE_JUMP 5
#define LSVD_ROTOR_KIND_UNWRAP 6
#define LSVD_ROTOR_KIND_DIRECTIONAL 7
#define LSVD_ROTOR_KIND_SURGERY 8

/* Replaces HardwareSchedule::from_real_phaseflow + to_json_string
 * (src/lie_svd_compiler.rs:59-88, :213-265): layer = pass, theta =
 * (theta_l + theta_r) / 2, phi_l = phi_r = 0, source "real_phaseflow", kind
 * by name (:268-280), no diagonal_signs.  JSON out as lsvd_schedule_from_*. */
LSVD_API lsvd_status lsvd_schedule_from_real_phaseflow(const lsvd_mzi_phase* events, int64_t count,
                                                       int64_t channels, int32_t target, char* json,
                                                       int64_t cap, int64_t* len);

/* ---------------------------------------- binary phase-schedule frame ---- */
/* The phase-schedule-v1 data model (src/lie_svd_compiler.rs:27-57) as one
 * little-endian frame, for targets that take fixed records (the reference's
 * intended CBOR / FPGA-table / MZI-frame mappings, no counterpart of its
 * own): header, total_events records, n_signs doubles (diagonal_signs),
 * then, with LSVD_SCHED_ENERGY, two doubles per event (energy_before,
 * energy_after; NaN = absent).  Source and kind are codes into the fixed
 * name tables LSVD_SCHED_SOURCE_* / LSVD_SCHED_KIND_* (kinds 0..8 are the
 * LSVD_ROTOR_KIND_* names, 9 complex_golden_prespin, 10
 * complex_diagonal_phase, 11 givens_elimination, 12 jacobi_rotation).
 * With LSVD_SCHED_CANONICAL the JSON order is the records stably sorted by
 * (layer, j, i) -- the (round, i, j) order of the rotors they come from, whose
 * pair the record stores as (i, j) = (rotor j, rotor i); a device-written
 * stream carries its events in the order the sweeps produced them. */
#define LSVD_SCHED_MAGIC "PSCHEDv1"
#define LSVD_SCHED_CANONICAL 0x1u
#define LSVD_SCHED_ENERGY 0x2u
#define LSVD_SCHED_SOURCE_REAL_PHASEFLOW 0
#define LSVD_SCHED_SOURCE_COMPLEX_PHASEFLOW 1
#define LSVD_SCHED_SOURCE_ORTHOGONAL_GIVENS 2
#define LSVD_SCHED_SOURCE_GPU_JACOBI 3
#define LSVD_SCHED_KIND_GIVENS_ELIMINATION 11
#define LSVD_SCHED_KIND_JACOBI_ROTATION 12

typedef struct lsvd_schedule_header {
    char magic[8];         /* LSVD_SCHED_MAGIC, no NUL */
    uint32_t header_bytes; /* sizeof(lsvd_schedule_header) = 64 */
    uint32_t record_bytes; /* sizeof(lsvd_schedule_record) = 56 */
    uint32_t target;       /* 0 mzi_mesh, 1 fpga_rotor_mesh */
    uint32_t flags;        /* LSVD_SCHED_* */
    int64_t channels;
    int64_t total_events;
    int64_t n_signs;
    int64_t reserved[2];
} lsvd_schedule_header;

typedef struct lsvd_schedule_record {
    uint32_t layer;
    uint16_t i;
    uint16_t j;
    double phi_l;
    double phi_r;
    double theta;
    double theta_l;
    double theta_r;
    uint8_t source;
    uint8_t kind;
    uint16_t reserved0;
    uint32_t reserved1;
} lsvd_schedule_record;

/* Binary frame of a rotor stream: the events of lsvd_schedule_from_rotors
 * (same convention, diagonal_signs all +1) in stream order, with
 * LSVD_SCHED_CANONICAL.  With LSVD_DEVICE_POINTERS `rotors` and `out` are
 * device memory and one kernel writes the whole frame on the context's
 * stream (synchronous unless LSVD_ASYNC; a bad rotor -- i >= j or
 * j >= channels -- is then reported by LSVD_BAD_ARGUMENT only when not
 * asynchronous); otherwise both are host memory and ctx may be NULL.
 * *len (host) receives the frame's size in bytes; cap below it returns
 * LSVD_ROTOR_OVERFLOW with nothing written (out = NULL to size). */
LSVD_API lsvd_status lsvd_schedule_binary_from_rotors(lsvd_context* ctx, const lsvd_rotor* rotors,
                                                      int64_t count, int64_t channels, int32_t target,
                                                      void* out, int64_t cap, int64_t* len,
                                                      uint32_t flags);

/* Binary frame of lsvd_schedule_from_real_phaseflow's schedule (host). */
LSVD_API lsvd_status lsvd_schedule_binary_from_real_phaseflow(const lsvd_mzi_phase* events,
                                                              int64_t count, int64_t channels,
                                                              int32_t target, void* out, int64_t cap,
                                                              int64_t* len);

/* The phase-schedule-v1 JSON text of a binary frame (host), byte-identical
 * to the JSON entry that describes the same schedule.  A malformed frame
 * (magic, sizes, codes, length) returns LSVD_BAD_ARGUMENT. */
LSVD_API lsvd_status lsvd_schedule_binary_to_json(const void* frame, int64_t bytes, char* json,
                                                  int64_t cap, int64_t* len);

#ifdef __cplusplus
}
#endif

#endif /* LSVD_H */
