//! GPU back end for the hot path of `lie_cliffalg_analog_svd`.
//!
//! Each function here has the signature of the reference function it
//! replaces, so the reference forwards to it with a one-line body:
//!
//! | reference (file:line)                                        | here                        |
//! |--------------------------------------------------------------|-----------------------------|
//! | `LieSvdSmall::solve` (src/lie_svd_small.rs:296)              | [`small_solve`]             |
//! | `LieSvdSmall::solve_rectangular` (src/lie_svd_small.rs:340)  | [`solve_rectangular`]       |
//! | `LieSvdMicro::solve` (src/lie_svd_micro.rs:21)               | [`micro_solve`]             |
//! | `LieSvdJoint::diagonalize_symmetric_with_params` (src/lie_svd_joint.rs:71) | [`diagonalize_symmetric_with_params`] |
//! | `LieSvdJoint::joint_svd_with_params` (src/lie_svd_joint.rs:170) | [`joint_svd_with_params`] |
//! | `HardwareSchedule::from_real_phaseflow` + `to_json_string` (src/lie_svd_compiler.rs:59, :213) | [`schedule_from_real_phaseflow_json`] |
//! | `HardwareSchedule::from_orthogonal_matrix` + `to_json_string` (src/lie_svd_compiler.rs:144, :213) | [`schedule_from_orthogonal_json`] |
//!
//! plus the batched and large entries that have no reference counterpart
//! ([`svd_batched`], [`svd_large`]).  Errors panic with the library's
//! message, as the reference's `assert!`s do for bad shapes.
use ndarray::{Array1, Array2, ArrayView2};
use std::ffi::CStr;
use std::os::raw::c_int;

pub mod ffi;
use ffi::*;

/// Arithmetic of the Newton-Schulz bulk (the Jacobi stages stay FP64).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum Precision {
    Fp64,
    Tf32,
    Bf16,
}

impl Precision {
    fn code(self) -> c_int {
        match self {
            Precision::Fp64 => PREC_FP64,
            Precision::Tf32 => PREC_TF32,
            Precision::Bf16 => PREC_BF16,
        }
    }
}

/// One library context per host thread, created on first use on device 0.
struct Context(Ctx);

impl Drop for Context {
    fn drop(&mut self) {
        unsafe {
            lsvd_context_destroy(self.0);
        }
    }
}

thread_local! {
    static CTX: Context = {
        let mut c: Ctx = std::ptr::null_mut();
        let st = unsafe { lsvd_context_create(0, &mut c) };
        assert_eq!(st, LSVD_OK, "lsvd_context_create failed: {}", status_text(st));
        Context(c)
    };
}

fn with_ctx<R>(f: impl FnOnce(Ctx) -> R) -> R {
    CTX.with(|c| f(c.0))
}

fn status_text(st: Status) -> String {
    unsafe { CStr::from_ptr(lsvd_status_string(st)).to_string_lossy().into_owned() }
}

fn check(ctx: Ctx, what: &str, st: Status, tolerate_not_converged: bool) {
    if st == LSVD_OK || (tolerate_not_converged && st == LSVD_NOT_CONVERGED) {
        return;
    }
    let detail = unsafe { CStr::from_ptr(lsvd_context_last_error(ctx)).to_string_lossy().into_owned() };
    panic!("{what} failed: {} ({detail})", status_text(st));
}

fn row_major(m: &Array2<f64>) -> ArrayView2<'_, f64> {
    m.view()
}

fn contiguous(m: &Array2<f64>) -> Vec<f64> {
    row_major(m).as_standard_layout().iter().copied().collect()
}

type Svd = (Array2<f64>, Array1<f64>, Array2<f64>);

/// `LieSvdSmall::solve` (src/lie_svd_small.rs:296): square `n x n`, every
/// n (n <= 64 on one CTA per matrix, larger n through the blocked solve).
/// An iteration cap returns the results, as the reference does.
pub fn small_solve(mat: &Array2<f64>) -> Svd {
    let n = mat.nrows();
    assert_eq!(n, mat.ncols(), "LieSvdSmall::solve: matrix must be square N×N");
    let a = contiguous(mat);
    let (mut u, mut s, mut vt) = (Array2::zeros((n, n)), Array1::zeros(n), Array2::zeros((n, n)));
    let ni = n as i64;
    with_ctx(|c| {
        let st = unsafe {
            lsvd_small_solve_f64(c, ni, a.as_ptr(), ni, u.as_mut_ptr(), ni, s.as_mut_ptr(), vt.as_mut_ptr(), ni,
                std::ptr::null_mut(), std::ptr::null_mut(), 0, std::ptr::null_mut(), std::ptr::null_mut(), 0)
        };
        check(c, "lsvd_small_solve_f64", st, true);
    });
    (u, s, vt)
}

/// `LieSvdSmall::solve_rectangular` (src/lie_svd_small.rs:340): `m x d`,
/// U is `m x k`, S has k = min(m, d) entries, Vt is `k x d`.
pub fn solve_rectangular(mat: &Array2<f64>) -> Svd {
    let (m, d) = mat.dim();
    let k = m.min(d);
    let a = contiguous(mat);
    let (mut u, mut s, mut vt) = (Array2::zeros((m, k)), Array1::zeros(k), Array2::zeros((k, d)));
    with_ctx(|c| {
        let st = unsafe {
            lsvd_small_solve_rectangular_f64(c, m as i64, d as i64, a.as_ptr(), d as i64, u.as_mut_ptr(), k as i64,
                s.as_mut_ptr(), vt.as_mut_ptr(), d as i64, std::ptr::null_mut(), 0)
        };
        check(c, "lsvd_small_solve_rectangular_f64", st, true);
    });
    (u, s, vt)
}

/// `LieSvdMicro::solve` (src/lie_svd_micro.rs:21): n <= 4 on registers,
/// larger n escalates to the small route exactly as the reference does.
pub fn micro_solve(mat: &Array2<f64>) -> Svd {
    let n = mat.nrows();
    assert_eq!(n, mat.ncols(), "LieSvdMicro::solve: matrix must be square");
    let a = contiguous(mat);
    let (mut u, mut s, mut vt) = (Array2::zeros((n, n)), Array1::zeros(n), Array2::zeros((n, n)));
    let ni = n as i64;
    with_ctx(|c| {
        let st = unsafe {
            lsvd_micro_solve_f64(c, ni, a.as_ptr(), ni, u.as_mut_ptr(), ni, s.as_mut_ptr(), vt.as_mut_ptr(), ni,
                std::ptr::null_mut(), 0)
        };
        check(c, "lsvd_micro_solve_f64", st, true);
    });
    (u, s, vt)
}

/// The reference's `JointDiagonalizationParams` fields.
#[derive(Clone, Copy, Debug)]
pub struct JointParams {
    pub max_sweeps: usize,
    pub tol: f64,
    pub min_pair_scale: f64,
    pub line_search_steps: usize,
}

impl JointParams {
    /// `JointDiagonalizationParams::for_n` (src/lie_svd_joint.rs:27).
    pub fn for_n(n: usize) -> Self {
        let p = unsafe { lsvd_joint_params_for_n(n as i64) };
        JointParams {
            max_sweeps: p.max_sweeps as usize,
            tol: p.tol,
            min_pair_scale: p.min_pair_scale,
            line_search_steps: p.line_search_steps as usize,
        }
    }

    fn raw(&self) -> LsvdJointParams {
        LsvdJointParams {
            max_sweeps: self.max_sweeps as i32,
            tol: self.tol,
            min_pair_scale: self.min_pair_scale,
            line_search_steps: self.line_search_steps as i32,
        }
    }
}

/// The reference's `JointDiagonalizationTrace` / `JointSvdTrace` fields.
#[derive(Clone, Copy, Debug, Default)]
pub struct JointTrace {
    pub initial_offdiag: f64,
    pub final_offdiag: f64,
    pub sweeps: usize,
    pub rotations: usize,
    pub rejected_rotations: usize,
}

impl From<LsvdJointTrace> for JointTrace {
    fn from(t: LsvdJointTrace) -> Self {
        JointTrace {
            initial_offdiag: t.initial_offdiag,
            final_offdiag: t.final_offdiag,
            sweeps: t.sweeps as usize,
            rotations: t.rotations as usize,
            rejected_rotations: t.rejected_rotations as usize,
        }
    }
}

fn flatten(mats: &[Array2<f64>]) -> Vec<f64> {
    mats.iter().flat_map(|m| contiguous(m)).collect()
}

/// `LieSvdJoint::diagonalize_symmetric_with_params` (src/lie_svd_joint.rs:71):
/// one shared basis V for K symmetric n x n matrices, the diagonals of
/// V^T M_k V, and the sweep trace.
pub fn diagonalize_symmetric_with_params(
    matrices: &[Array2<f64>],
    params: JointParams,
) -> (Array2<f64>, Vec<Array1<f64>>, JointTrace) {
    assert!(!matrices.is_empty(), "LieSvdJoint: empty matrix set");
    let n = matrices[0].nrows();
    for m in matrices {
        assert_eq!(m.dim(), (n, n), "LieSvdJoint: matrices must be square and of one size");
    }
    let k = matrices.len();
    let flat = flatten(matrices);
    let p = params.raw();
    let (mut v, mut d, mut t) = (Array2::zeros((n, n)), vec![0.0; k * n], LsvdJointTrace::default());
    with_ctx(|c| {
        let st = unsafe {
            lsvd_jade_sym_f64(c, 1, k as i64, n as i64, flat.as_ptr(), &p, v.as_mut_ptr(), d.as_mut_ptr(), &mut t, 0)
        };
        check(c, "lsvd_jade_sym_f64", st, true);
    });
    (v, d.chunks(n.max(1)).map(|c| Array1::from(c.to_vec())).collect(), t.into())
}

/// `LieSvdJoint::diagonalize_symmetric` (src/lie_svd_joint.rs:64).
pub fn diagonalize_symmetric(matrices: &[Array2<f64>]) -> (Array2<f64>, Vec<Array1<f64>>, JointTrace) {
    let n = matrices.first().map(|m| m.nrows()).unwrap_or(0);
    diagonalize_symmetric_with_params(matrices, JointParams::for_n(n))
}

/// `LieSvdJoint::joint_svd_with_params` (src/lie_svd_joint.rs:170): shared
/// bases U (rows x rows) and Vt (cols x cols), per-matrix |diag(U^T M_k V)|.
pub fn joint_svd_with_params(
    matrices: &[Array2<f64>],
    params: JointParams,
) -> (Array2<f64>, Vec<Array1<f64>>, Array2<f64>, JointTrace) {
    assert!(!matrices.is_empty(), "LieSvdJoint: empty matrix set");
    let (rows, cols) = matrices[0].dim();
    assert!(rows > 0 && cols > 0, "LieSvdJoint: empty matrix");
    for m in matrices {
        assert_eq!(m.nrows(), rows, "LieSvdJoint: row-size mismatch");
        assert_eq!(m.ncols(), cols, "LieSvdJoint: col-size mismatch");
    }
    let (k, r) = (matrices.len(), rows.min(cols));
    let flat = flatten(matrices);
    let p = params.raw();
    let (mut u, mut vt) = (Array2::zeros((rows, rows)), Array2::zeros((cols, cols)));
    let (mut sig, mut t) = (vec![0.0; k * r], LsvdJointTrace::default());
    with_ctx(|c| {
        let st = unsafe {
            lsvd_joint_svd_f64(c, 1, k as i64, rows as i64, cols as i64, flat.as_ptr(), &p, u.as_mut_ptr(),
                sig.as_mut_ptr(), vt.as_mut_ptr(), &mut t, 0)
        };
        check(c, "lsvd_joint_svd_f64", st, true);
    });
    (u, sig.chunks(r).map(|c| Array1::from(c.to_vec())).collect(), vt, t.into())
}

/// `LieSvdJoint::joint_svd` (src/lie_svd_joint.rs:160).
pub fn joint_svd(matrices: &[Array2<f64>]) -> (Array2<f64>, Vec<Array1<f64>>, Array2<f64>, JointTrace) {
    let n = matrices.first().map(|m| m.nrows().min(m.ncols())).unwrap_or(0);
    joint_svd_with_params(matrices, JointParams::for_n(n))
}

/// Many square matrices of sizes 1..=64 in one call (the exact tiers of
/// `LieSvd::solve` per matrix); returns one SVD per input, in order.
pub fn svd_batched(matrices: &[Array2<f64>], precision: Precision) -> Vec<Svd> {
    let ns: Vec<i32> = matrices
        .iter()
        .map(|m| {
            assert_eq!(m.nrows(), m.ncols(), "svd_batched: matrices must be square");
            m.nrows() as i32
        })
        .collect();
    let total: usize = ns.iter().map(|&n| (n as usize) * (n as usize)).sum();
    let sum_n: usize = ns.iter().map(|&n| n as usize).sum();
    let a = flatten(matrices);
    let (mut u, mut s, mut vt) = (vec![0.0; total], vec![0.0; sum_n], vec![0.0; total]);
    with_ctx(|c| {
        let st = unsafe {
            lsvd_svd_batched_f64(c, ns.len() as i64, ns.as_ptr(), a.as_ptr(), u.as_mut_ptr(), s.as_mut_ptr(),
                vt.as_mut_ptr(), std::ptr::null_mut(), precision.code(), 0)
        };
        check(c, "lsvd_svd_batched_f64", st, true);
    });
    let (mut off, mut soff, mut out) = (0usize, 0usize, Vec::with_capacity(ns.len()));
    for &n in &ns {
        let n = n as usize;
        let take = |v: &[f64]| Array2::from_shape_vec((n, n), v[off..off + n * n].to_vec()).unwrap();
        out.push((take(&u), Array1::from(s[soff..soff + n].to_vec()), take(&vt)));
        off += n * n;
        soff += n;
    }
    out
}

/// One large m x n matrix: FP64 polar + blocked two-sided Jacobi, or a
/// TF32/BF16 Newton-Schulz bulk followed by FP64 one-sided Jacobi on A V0.
/// Returns the thin SVD (k = min(m, n)) and the run's statistics.
pub fn svd_large(mat: &Array2<f64>, precision: Precision) -> (Svd, LsvdLargeInfo) {
    let (m, n) = mat.dim();
    let k = m.min(n);
    let a = contiguous(mat);
    let (mut u, mut s, mut vt) = (Array2::zeros((m, k)), Array1::zeros(k), Array2::zeros((k, n)));
    let mut info = LsvdLargeInfo::default();
    with_ctx(|c| {
        let st = unsafe {
            lsvd_svd_large_f64(c, m as i64, n as i64, a.as_ptr(), n as i64, u.as_mut_ptr(), k as i64, s.as_mut_ptr(),
                vt.as_mut_ptr(), n as i64, precision.code(), &mut info, 0)
        };
        check(c, "lsvd_svd_large_f64", st, true);
    });
    ((u, s, vt), info)
}

/// The reference's `HardwareTarget` (src/lie_svd_compiler.rs:12-25).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum HardwareTarget {
    MziMesh,
    FpgaRotorMesh,
}

impl HardwareTarget {
    fn code(self) -> i32 {
        match self {
            HardwareTarget::MziMesh => 0,
            HardwareTarget::FpgaRotorMesh => 1,
        }
    }
}

fn text_call(what: &str, f: impl Fn(*mut std::os::raw::c_char, i64, *mut i64) -> Status) -> String {
    let mut len = 0i64;
    let st = f(std::ptr::null_mut(), 0, &mut len);
    assert_eq!(st, LSVD_OK, "{what} sizing failed: {}", status_text(st));
    let mut buf = vec![0u8; len as usize + 1];
    let st = f(buf.as_mut_ptr() as *mut std::os::raw::c_char, len + 1, &mut len);
    assert_eq!(st, LSVD_OK, "{what} failed: {}", status_text(st));
    buf.truncate(len as usize);
    String::from_utf8(buf).expect("phase-schedule-v1 text is ASCII")
}

/// `HardwareSchedule::from_real_phaseflow(..).to_json_string()`
/// (src/lie_svd_compiler.rs:59-88, :213-265); `events` as `MziPhase`
/// (kind = the `PhaseRotorKind` variant's position).
pub fn schedule_from_real_phaseflow_json(events: &[LsvdMziPhase], channels: usize, target: HardwareTarget) -> String {
    text_call("lsvd_schedule_from_real_phaseflow", |buf, cap, len| unsafe {
        lsvd_schedule_from_real_phaseflow(events.as_ptr(), events.len() as i64, channels as i64, target.code(), buf,
            cap, len)
    })
}

/// `HardwareSchedule::from_orthogonal_matrix(..).to_json_string()`
/// (src/lie_svd_compiler.rs:144-198, :213-265).
pub fn schedule_from_orthogonal_json(v: &Array2<f64>, target: HardwareTarget) -> String {
    let d = v.nrows();
    assert_eq!(d, v.ncols(), "HardwareSchedule::from_orthogonal_matrix: matrix must be square");
    let a = contiguous(v);
    text_call("lsvd_schedule_from_orthogonal", |buf, cap, len| unsafe {
        lsvd_schedule_from_orthogonal(d as i64, a.as_ptr(), target.code(), buf, cap, len)
    })
}

/// The binary phase-schedule frame of a rotor stream held on the host.
pub fn schedule_binary_from_rotors(rotors: &[LsvdRotor], channels: usize, target: HardwareTarget) -> Vec<u8> {
    let mut len = 0i64;
    let st = unsafe {
        lsvd_schedule_binary_from_rotors(std::ptr::null_mut(), rotors.as_ptr(), rotors.len() as i64, channels as i64,
            target.code(), std::ptr::null_mut(), 0, &mut len, 0)
    };
    assert_eq!(st, LSVD_OK, "lsvd_schedule_binary_from_rotors sizing failed: {}", status_text(st));
    let mut out = vec![0u8; len as usize];
    let st = unsafe {
        lsvd_schedule_binary_from_rotors(std::ptr::null_mut(), rotors.as_ptr(), rotors.len() as i64, channels as i64,
            target.code(), out.as_mut_ptr() as *mut std::os::raw::c_void, len, &mut len, 0)
    };
    assert_eq!(st, LSVD_OK, "lsvd_schedule_binary_from_rotors failed: {}", status_text(st));
    out
}

/// The phase-schedule-v1 JSON text of a binary frame.
pub fn schedule_binary_to_json(frame: &[u8]) -> String {
    text_call("lsvd_schedule_binary_to_json", |buf, cap, len| unsafe {
        lsvd_schedule_binary_to_json(frame.as_ptr() as *const std::os::raw::c_void, frame.len() as i64, buf, cap, len)
    })
}
