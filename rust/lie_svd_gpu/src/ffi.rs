//! Raw declarations of liblsvd_b200's C ABI, one for every export of
//! `include/lsvd.h`, with the structs laid out as the header lays them out.
use std::os::raw::{c_char, c_int, c_void};

pub type Status = c_int;
pub type Ctx = *mut c_void;

pub const LSVD_OK: Status = 0;
pub const LSVD_NOT_CONVERGED: Status = 1;

pub const PREC_FP64: c_int = 0;
pub const PREC_TF32: c_int = 1;
pub const PREC_BF16: c_int = 2;

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdDiag {
    pub rel_recon: f64,
    pub orth_u: f64,
    pub orth_v: f64,
    pub ns_iters: i32,
    pub jacobi_sweeps: i32,
    pub rotations: i64,
    pub flags: i32,
    pub route: i32,
}

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdRotor {
    pub i: u16,
    pub j: u16,
    pub round: u32,
    pub theta: f64,
}

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdLargeInfo {
    pub ns_iters_lowp: i32,
    pub ns_iters_fp64: i32,
    pub sweeps_lowp: i32,
    pub sweeps_fp64: i32,
    pub rotations: i64,
    pub flags: i32,
    pub inner_cap_pairs: i32,
    pub last_offdiag: f64,
    pub flops_fp64: f64,
    pub flops_lowp: f64,
    pub ms_polar: f64,
    pub ms_eig_lowp: f64,
    pub ms_eig_fp64: f64,
    pub ms_total: f64,
    pub rel_recon: f64,
    pub orth_u: f64,
    pub orth_v: f64,
}

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdJointParams {
    pub max_sweeps: i32,
    pub tol: f64,
    pub min_pair_scale: f64,
    pub line_search_steps: i32,
}

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdJointTrace {
    pub initial_offdiag: f64,
    pub final_offdiag: f64,
    pub sweeps: i64,
    pub rotations: i64,
    pub rejected_rotations: i64,
}

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdTriage {
    pub offdiag_ratio: f64,
    pub diagonal_dominance: f64,
    pub row_cv: f64,
    pub col_cv: f64,
    pub row_col_mismatch: f64,
    pub symmetry_ratio: f64,
    pub transpose_torsion_ratio: f64,
    pub diagonal_entropy: f64,
    pub row_mass_entropy: f64,
    pub col_mass_entropy: f64,
    pub suspicious_score: f64,
    pub mean_stress: f64,
    pub max_twist: f64,
    pub causal_disbalance: f64,
    pub entropy_gap: f64,
    pub global_phase: f64,
    pub torsion_energy: f64,
    pub chirality_balance: f64,
    pub phase_entropy: f64,
    pub chirality: f64,
    pub golden_resonance: f64,
    pub adaptive_route: i32,
    pub passport_route: i32,
}

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdPolarInfo {
    pub iters_lowp: i32,
    pub iters_fp64: i32,
    pub orth: f64,
    pub flops_lowp: f64,
    pub flops_fp64: f64,
    pub gemm_ms_lowp: f64,
    pub gemm_ms_fp64: f64,
    pub converged: i32,
    pub pad_: i32,
}

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdMziPhase {
    pub pass: i64,
    pub i: i64,
    pub j: i64,
    pub theta_l: f64,
    pub theta_r: f64,
    pub kind: i32,
    pub pad_: i32,
}

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdScheduleHeader {
    pub magic: [u8; 8],
    pub header_bytes: u32,
    pub record_bytes: u32,
    pub target: u32,
    pub flags: u32,
    pub channels: i64,
    pub total_events: i64,
    pub n_signs: i64,
    pub reserved: [i64; 2],
}

#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct LsvdScheduleRecord {
    pub layer: u32,
    pub i: u16,
    pub j: u16,
    pub phi_l: f64,
    pub phi_r: f64,
    pub theta: f64,
    pub theta_l: f64,
    pub theta_r: f64,
    pub source: u8,
    pub kind: u8,
    pub reserved0: u16,
    pub reserved1: u32,
}

#[link(name = "lsvd_b200")]
extern "C" {
    pub fn lsvd_version() -> *const c_char;
    pub fn lsvd_status_string(s: Status) -> *const c_char;
    pub fn lsvd_context_create(device: c_int, out: *mut Ctx) -> Status;
    pub fn lsvd_context_destroy(ctx: Ctx) -> Status;
    pub fn lsvd_context_set_stream(ctx: Ctx, stream: *mut c_void) -> Status;
    pub fn lsvd_context_get_stream(ctx: Ctx) -> *mut c_void;
    pub fn lsvd_synchronize(ctx: Ctx) -> Status;
    pub fn lsvd_context_last_error(ctx: Ctx) -> *const c_char;
    pub fn lsvd_context_kernel_launches(ctx: Ctx) -> i64;
    pub fn lsvd_small_solve_f64(ctx: Ctx, n: i64, a: *const f64, lda: i64, u: *mut f64, ldu: i64,
        s: *mut f64, vt: *mut f64, ldvt: i64, diag: *mut LsvdDiag, rotors: *mut LsvdRotor,
        rotor_cap: i64, rotor_count: *mut i64, perm: *mut i32, flags: u32) -> Status;
    pub fn lsvd_micro_solve_f64(ctx: Ctx, n: i64, a: *const f64, lda: i64, u: *mut f64, ldu: i64,
        s: *mut f64, vt: *mut f64, ldvt: i64, diag: *mut LsvdDiag, flags: u32) -> Status;
    pub fn lsvd_small_solve_rectangular_f64(ctx: Ctx, m: i64, d: i64, a: *const f64, lda: i64,
        u: *mut f64, ldu: i64, s: *mut f64, vt: *mut f64, ldvt: i64, diag: *mut LsvdDiag,
        flags: u32) -> Status;
    pub fn lsvd_svd_large_f64(ctx: Ctx, m: i64, n: i64, a: *const f64, lda: i64, u: *mut f64,
        ldu: i64, s: *mut f64, vt: *mut f64, ldvt: i64, precision: c_int,
        info: *mut LsvdLargeInfo, flags: u32) -> Status;
    pub fn lsvd_svd_batched_f64(ctx: Ctx, count: i64, n: *const i32, a: *const f64, u: *mut f64,
        s: *mut f64, vt: *mut f64, diags: *mut LsvdDiag, precision: c_int, flags: u32) -> Status;
    pub fn lsvd_autotune_f64(ctx: Ctx, per_class: i64, cache_path: *const c_char,
        report: *mut c_char, report_cap: i64) -> Status;
    pub fn lsvd_class_shapes(ctx: Ctx, precision: c_int, out: *mut i32) -> Status;
    pub fn lsvd_svd_batched_noalloc_f64(stream: *mut c_void, count: i64, n: *const i32,
        a: *const f64, u: *mut f64, s: *mut f64, vt: *mut f64, diags: *mut LsvdDiag,
        flags: u32) -> Status;
    pub fn lsvd_metrics_f64(ctx: Ctx, m: i64, d: i64, k: i64, a: *const f64, u: *const f64,
        s: *const f64, vt: *const f64, sigma_ref: *const f64, out: *mut f64, flags: u32) -> Status;
    pub fn lsvd_joint_params_for_n(n: i64) -> LsvdJointParams;
    pub fn lsvd_jade_sym_f64(ctx: Ctx, families: i64, k: i64, n: i64, m: *const f64,
        params: *const LsvdJointParams, v: *mut f64, diag: *mut f64,
        traces: *mut LsvdJointTrace, flags: u32) -> Status;
    pub fn lsvd_joint_svd_f64(ctx: Ctx, families: i64, k: i64, rows: i64, cols: i64,
        m: *const f64, params: *const LsvdJointParams, u: *mut f64, sig: *mut f64, vt: *mut f64,
        traces: *mut LsvdJointTrace, flags: u32) -> Status;
    pub fn lsvd_triage_batched_f64(ctx: Ctx, count: i64, rows: *const i32, cols: *const i32,
        a: *const f64, out: *mut LsvdTriage, flags: u32) -> Status;
    pub fn lsvd_polar_f64(ctx: Ctx, m: i64, n: i64, a: *const f64, lda: i64, q: *mut f64,
        ldq: i64, precision: c_int, info: *mut LsvdPolarInfo, flags: u32) -> Status;
    pub fn lsvd_gemm_nt_lowp(ctx: Ctx, m: i64, n: i64, k: i64, a: *const f32, b: *const f32,
        c: *mut f32, precision: c_int) -> Status;
    pub fn lsvd_gemm_f64(ctx: Ctx, trans_a: i32, trans_b: i32, m: i64, n: i64, k: i64,
        alpha: f64, a: *const f64, lda: i64, b: *const f64, ldb: i64, beta: f64, c: *mut f64,
        ldc: i64) -> Status;
    pub fn lsvd_svd_batched_stream_f64(ctx: Ctx, count: i64, m: i64, n: i64, a: *const f64,
        u: *mut f64, s: *mut f64, vt: *mut f64, rotors: *mut LsvdRotor, rotor_cap: i64,
        rotor_count: *mut i64, perm: *mut i32, diags: *mut LsvdDiag, flags: u32) -> Status;
    pub fn lsvd_svd_vjp_f64(ctx: Ctx, count: i64, m: i64, n: i64, a: *const f64, s: *const f64,
        perm: *const i32, rotors: *const LsvdRotor, rotor_cap: i64, rotor_count: *const i64,
        ubar: *const f64, sbar: *const f64, vbar: *const f64, qbar: *const f64, vt: *const f64,
        gap_tol: f64, abar: *mut f64, flags: u32) -> Status;
    pub fn lsvd_schedule_from_orthogonal(d: i64, v: *const f64, target: i32, json: *mut c_char,
        cap: i64, len: *mut i64) -> Status;
    pub fn lsvd_schedule_from_rotors(rotors: *const LsvdRotor, count: i64, channels: i64,
        target: i32, json: *mut c_char, cap: i64, len: *mut i64) -> Status;
    pub fn lsvd_schedule_from_real_phaseflow(events: *const LsvdMziPhase, count: i64, channels: i64,
        target: i32, json: *mut c_char, cap: i64, len: *mut i64) -> Status;
    pub fn lsvd_schedule_binary_from_rotors(ctx: Ctx, rotors: *const LsvdRotor, count: i64, channels: i64,
        target: i32, out: *mut c_void, cap: i64, len: *mut i64, flags: u32) -> Status;
    pub fn lsvd_schedule_binary_from_real_phaseflow(events: *const LsvdMziPhase, count: i64, channels: i64,
        target: i32, out: *mut c_void, cap: i64, len: *mut i64) -> Status;
    pub fn lsvd_schedule_binary_to_json(frame: *const c_void, bytes: i64, json: *mut c_char, cap: i64,
        len: *mut i64) -> Status;
}
