/*
 * lsvd_oracle.h -- CPU f64 restatement of the hot path of the Rust crate
 * `lie_cliffalg_analog_svd` v0.44.0 (polar/Jacobi SVD, n<=4 micro kernels,
 * Phase-JADE, rotor schedule compiler, diagnostics).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against, and the timed CPU baseline.  Nothing in the product
 * (the `lie_cliffalg_analog_svd_b200` package, `include/lsvd.h`) links,
 * loads or calls it.
 *
 * All matrices are dense row-major f64 with leading dimension = #columns.
 * Every entry point returns 0 on success and a negative value on a shape
 * error (the Rust code panics via `assert!` in those cases).
 */
#ifndef LSVD_ORACLE_H
#define LSVD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t ns_iters;        /* Newton-Schulz iterations executed */
    int32_t polar_ok;        /* 1 if the polar factor was trusted */
    int32_t jacobi_sweeps;   /* Jacobi sweeps started (incl. the converged test sweep) */
    int64_t jacobi_rotations;/* rotations applied */
    int32_t repaired;        /* 1 if U was rebuilt by repair_left_basis_from_right */
    int32_t micro_fallback;  /* 1 if LieSvdMicro escalated to LieSvdSmall */
} oracle_small_info;

/* LieSvdSmall::solve (src/lie_svd_small.rs:296-323). A n*n; U n*n, S n, Vt n*n. */
int oracle_small_solve(int64_t n, const double* A, double* U, double* S, double* Vt,
                       oracle_small_info* info);

/* newton_schulz_polar (src/lie_svd_small.rs:158-183). Q n*n. */
int oracle_ns_polar(int64_t n, const double* A, double* Q, int32_t* ok, int32_t* iters);

/* eigh_jacobi_full (src/lie_svd_small.rs:212-285). P n*n symmetric; V n*n, eig n. */
int oracle_eigh_jacobi(int64_t n, const double* P, double* V, double* eig, int32_t* sweeps,
                       int64_t* rotations);

/* LieSvdSmall::solve_rectangular (src/lie_svd_small.rs:340-360).
 * A m*d; k=min(m,d); U m*k, S k, Vt k*d. */
int oracle_small_solve_rectangular(int64_t m, int64_t d, const double* A, double* U, double* S,
                                   double* Vt);

/* qr_reduce (src/lie_svd_small.rs:373-418). A m*d (m>=d); Q m*d, R d*d. */
int oracle_qr_reduce(int64_t m, int64_t d, const double* A, double* Q, double* R);

/* Timed-baseline batch driver: matrices idx[0..count) of a packed uneven
 * batch (matrix t: n[t] x n[t] at element offset aoff[t], singular values at
 * soff[t]) on `threads` host threads, LieSvdMicro for n <= 4 and LieSvdSmall
 * otherwise.  Returns the number solved. */
int64_t oracle_svd_batch(int64_t count, const int32_t* idx, const int32_t* n, const int64_t* aoff,
                         const int64_t* soff, const double* A, double* U, double* S, double* Vt,
                         int32_t threads);

/* Triage of one rows x cols matrix: LieSvdAdaptive's analyze_matrix and
 * choose_route (src/lie_svd_adaptive.rs:84-274, default params), the
 * PhaseSignature of lie_svd_phasehealth::phase_signature (src/
 * lie_svd_phasehealth.rs:100-343) with its global invariants and the 4x4
 * block dual balance (src/lie_svd_block4.rs:210-266), and PhaseEngine's
 * passport extras (src/lie_svd_engine.rs:75-103, :277-326).  out[0..20]:
 * offdiag_ratio, diagonal_dominance, row_cv, col_cv, row_col_mismatch,
 * symmetry_ratio, transpose_torsion_ratio, diagonal_entropy,
 * row_mass_entropy, col_mass_entropy, suspicious_score (NaN unless square),
 * mean_stress, max_twist, causal_disbalance, entropy_gap, global_phase,
 * torsion_energy, chirality_balance, phase_entropy, chirality,
 * golden_resonance; routes[0] = AdaptiveRoute (0 Micro, 1 Small,
 * 2 PhaseFlow, 3 CoreFlowTopo, 4 Hybrid; -1 not square), routes[1] =
 * passport PhaseRoute (0 RealSmall, 1 RealPhaseFlowPolished). */
int oracle_triage(int64_t rows, int64_t cols, const double* A, double* out, int32_t* routes);

/* LieSvdMicro::solve (src/lie_svd_micro.rs:21-52), n in 0..4. */
int oracle_micro_solve(int64_t n, const double* A, double* U, double* S, double* Vt,
                       oracle_small_info* info);

typedef struct {
    int32_t max_sweeps;
    double tol;
    double min_pair_scale;
    int32_t line_search_steps;
} oracle_joint_params;

typedef struct {
    double initial_offdiag;
    double final_offdiag;
    int64_t sweeps;
    int64_t rotations;
    int64_t rejected_rotations;
} oracle_joint_trace;

/* JointDiagonalizationParams::for_n (src/lie_svd_joint.rs:27-34). */
oracle_joint_params oracle_joint_params_for_n(int64_t n);

/* LieSvdJoint::diagonalize_symmetric_with_params (src/lie_svd_joint.rs:71-158).
 * M: K matrices n*n back to back; V n*n; diag K*n. */
int oracle_jade_sym(int64_t K, int64_t n, const double* M, oracle_joint_params params,
                    double* V, double* diag, oracle_joint_trace* trace);

/* LieSvdJoint::joint_svd_with_params (src/lie_svd_joint.rs:170-261).
 * M: K matrices rows*cols; U rows*rows; sig K*min(rows,cols); Vt cols*cols. */
int oracle_joint_svd(int64_t K, int64_t rows, int64_t cols, const double* M,
                     oracle_joint_params params, double* U, double* sig, double* Vt,
                     oracle_joint_trace* trace);

/* metrics::compute (src/lib.rs:149-194).  sigma_ref may be NULL (then the two
 * sigma outputs are set to NaN).  out[0..5] = rel_recon, orth_u, orth_v,
 * sigma_max_rel, sigma_tail_rel.  U m*k, S k, Vt k*d, A m*d. */
int oracle_metrics(int64_t m, int64_t d, int64_t k, const double* A, const double* U,
                   const double* S, const double* Vt, const double* sigma_ref, double* out);

/* HardwareSchedule::from_orthogonal_matrix (src/lie_svd_compiler.rs:144-198).
 * V d*d.  Writes at most cap events: ev_i, ev_j (int64), ev_theta; signs d.
 * Returns the number of events (>= 0) or < 0 on error. */
int64_t oracle_schedule_from_orthogonal(int64_t d, const double* V, int64_t cap, int64_t* ev_i,
                                        int64_t* ev_j, double* ev_theta, double* signs);

/* Formats a Rust `{:.17e}` float (src/lie_svd_compiler.rs:227) into buf.
 * Returns the string length. */
/* Product rounding of every ndarray `dot` the oracle restates: 1 (default) =
 * fused multiply-add per k (matrixmultiply's FMA kernel), 0 = multiply then
 * add (its generic kernel, hosts without FMA).  Process-wide. */
void oracle_set_dot_fma(int32_t on);

/* ndarray `a.dot(&b)` (row-major m x k times k x n) in the reference's product
 * order: sequential fused multiply-adds over k. */
int oracle_dot(int64_t m, int64_t k, int64_t n, const double* A, const double* B, double* C);

/* One symmetrised lagged covariance of Phase-BSS (src/lie_svd_bss.rs:172-190)
 * of the ch x samples row-major signal x, in the reference's loop order. */
int oracle_lagged_covariance(int64_t ch, int64_t samples, const double* x, int64_t lag, double* out);

int oracle_fmt_e17(double x, char* buf, int64_t cap);

#ifdef __cplusplus
}
#endif

#endif
