// lsvd_mixed.cuh -- mixed-precision SVD of one n <= 64 matrix per team:
// tensor-core TF32/BF16 bulk, FP64 refinement and FP64 Jacobi cleanup.
//
//   1. Newton-Schulz polar iteration X <- 0.5 X (3I - X^T X) on tensor cores
//      (mma.sync m16n8k8 TF32 or m16n8k16 BF16, FP32 accumulation) until the
//      update reaches the low-precision floor;
//   2. P_lo = sym(X^T A) and an FP32 round-robin one-sided Jacobi on P_lo give
//      an approximate right singular basis V0;
//   3. FP64 Newton-Schulz refinement makes V0 orthogonal to working precision;
//   4. W = A V0 in FP64, then FP64 one-sided Jacobi cleanup sweeps with the
//      same rotation rule and convergence test as the FP64 path;
//      sigma_j = ||w_j||, U = W diag(1/sigma) with the repair of
//      repair_left_basis_from_right (src/lie_svd_small.rs:185-208) for
//      vanishing sigma.
// The FP64 cleanup works on A itself, so the result is a backward-stable FP64
// SVD whatever the accuracy of V0; the low-precision phases only decide how
// many FP64 sweeps are needed.  (Preconditioned one-sided Jacobi with a
// low-precision eigenbasis: Higham, Tisseur, Webb & Zhou, "Computing accurate
// eigenvalues using a mixed-precision Jacobi algorithm", SIMAX 2021.)
//
// The in-team products are 64x64x64 at most, so they use the warp-level
// mma.sync path; the large polar kernels use tcgen05 (lsvd_polar.cu).
#pragma once

#include "lsvd_device.cuh"

namespace lsvd {

enum { kPrecTF32 = 1, kPrecBF16 = 2 };

__host__ __device__ constexpr int pad16(int n) { return (n + 15) & ~15; }
// FP32 buffers: leading dimension == 4 (mod 32) keeps the fragment loads of
// the Gram products conflict-free.
__host__ __device__ constexpr int ld32_of(int n) { return pad16(n) + 4; }
// One slot holds an FP64 buffer ((np+1) x np) or two FP32 buffers.
__host__ __device__ constexpr int mixed_slot_doubles(int n) {
    return (pad4(n) + 1) * pad4(n) > pad16(n) * ld32_of(n) ? (pad4(n) + 1) * pad4(n)
                                                            : pad16(n) * ld32_of(n);
}
__host__ __device__ constexpr int mixed_smem_doubles(int n) {
    return 3 * mixed_slot_doubles(n) + int(sizeof(TeamScratch) / sizeof(double));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// C (ntc x ntc) = A (ntc x ntc) * B (ntc x ntc) on tensor cores, one 16x8
// output tile per warp at a time.  la(row, k) = A(row, k), lb(k, col) = B(k, col)
// return FP32 values; epi(row, col, value) consumes the FP32 results.
template <int PREC, class LA, class LB, class Epi>
__device__ __forceinline__ void tc_gemm(const Team& t, int ntc, LA la, LB lb, Epi epi) {
    const int g = t.lane >> 2, q = t.lane & 3;
    const int tm = ntc / 16, tn = ntc / 8;
    for (int tile = t.warp; tile < tm * tn; tile += t.nwarps) {
        const int m0 = (tile % tm) * 16, n0 = (tile / tm) * 8;
        float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
        if (PREC == kPrecTF32) {
            for (int k0 = 0; k0 < ntc; k0 += 8) {
                const uint32_t a0 = to_tf32(la(m0 + g, k0 + q)), a1 = to_tf32(la(m0 + g + 8, k0 + q));
                const uint32_t a2 = to_tf32(la(m0 + g, k0 + q + 4)), a3 = to_tf32(la(m0 + g + 8, k0 + q + 4));
                const uint32_t b0 = to_tf32(lb(k0 + q, n0 + g)), b1 = to_tf32(lb(k0 + q + 4, n0 + g));
                asm volatile(
                    "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, "
                    "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                    : "+f"(c0), "+f"(c1), "+f"(c2), "+f"(c3)
                    : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
            }
        } else {
            for (int k0 = 0; k0 < ntc; k0 += 16) {
                const int kk = k0 + 2 * q;
                const uint32_t a0 = pack_bf16(la(m0 + g, kk), la(m0 + g, kk + 1));
                const uint32_t a1 = pack_bf16(la(m0 + g + 8, kk), la(m0 + g + 8, kk + 1));
                const uint32_t a2 = pack_bf16(la(m0 + g, kk + 8), la(m0 + g, kk + 9));
                const uint32_t a3 = pack_bf16(la(m0 + g + 8, kk + 8), la(m0 + g + 8, kk + 9));
                const uint32_t b0 = pack_bf16(lb(kk, n0 + g), lb(kk + 1, n0 + g));
                const uint32_t b1 = pack_bf16(lb(kk + 8, n0 + g), lb(kk + 9, n0 + g));
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, "
                    "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                    : "+f"(c0), "+f"(c1), "+f"(c2), "+f"(c3)
                    : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
            }
        }
        epi(m0 + g, n0 + 2 * q, c0);
        epi(m0 + g, n0 + 2 * q + 1, c1);
        epi(m0 + g + 8, n0 + 2 * q, c2);
        epi(m0 + g + 8, n0 + 2 * q + 1, c3);
    }
}

__device__ __forceinline__ void write_nonfinite(const Team& t, const SmallJob& job, int flags) {
    const int n = job.n;
    const double qnan = __longlong_as_double(0x7ff8000000000000ULL);
    for (int idx = t.tid; idx < n * n; idx += t.nthreads) {
        const int i = idx / n, j = idx % n;
        job.U[i * job.ldu + j] = qnan;
        job.Vt[i * job.ldvt + j] = qnan;
    }
    for (int i = t.tid; i < n; i += t.nthreads) job.S[i] = qnan;
    if (t.tid == 0) {
        if (job.diag) {
            lsvd_diag d;
            d.rel_recon = d.orth_u = d.orth_v = qnan;
            d.ns_iters = 0;
            d.jacobi_sweeps = 0;
            d.rotations = 0;
            d.flags = flags | LSVD_MAT_NONFINITE;
            d.route = LSVD_ROUTE_SMALL;
            *job.diag = d;
        }
        if (job.agg) atomicOr(job.agg, flags | LSVD_MAT_NONFINITE);
    }
    t.sync();
}

template <int TS, int G, int PREC>
__device__ void mixed_solve_team(const Team& t, const SmallJob& job, double* sm) {
    const int n = job.n;
    const int np = pad4(n), ld = np + 1;
    const int ntc = pad16(n), l32 = ld32_of(n);
    const int slot = mixed_slot_doubles(n);
    double* S0 = sm;
    double* S1 = sm + slot;
    double* S2 = sm + 2 * slot;
    TeamScratch* sc = reinterpret_cast<TeamScratch*>(sm + 3 * slot);
    const double refn = sqrt(double(n));
    int flags = job.extra_flags;

    // ---- load A (FP64, column-major) into S2: norm, max entry, finiteness
    double fro2 = 0.0, amax = 0.0;
    int bad = 0;
    for (int idx = t.tid; idx < np * np; idx += t.nthreads) {
        const int i = idx / np, j = idx - (idx / np) * np;
        double v = 0.0;
        if (i < n && j < n) {
            v = job.A[i * job.lda + j];
            fro2 += v * v;
            amax = fmax(amax, fabs(v));
            if (!isfinite(v)) bad++;
        }
        S2[j * ld + i] = v;
    }
    fro2 = team_sum(t, fro2, sc->red);
    amax = team_max(t, amax, sc->red);
    if (team_sum(t, double(bad), sc->red) > 0.0) {
        write_nonfinite(t, job, flags);
        return;
    }
    const double afro = sqrt(fro2);
    // power-of-two scale of A for the FP64 phase (exact, undone on sigma)
    const double ascale = amax > 0.0 ? ldexp(1.0, max(-1000, min(1000, -ilogb(amax)))) : 1.0;
    const double inv_fro = 1.0 / fmax(afro, 1e-300);

    // ---- 1. low-precision Newton-Schulz: X32 (S0 lo), T32 (S0 hi), Y32 (S1 lo)
    float* X32 = reinterpret_cast<float*>(S0);
    float* T32 = X32 + ntc * l32;
    float* Y32 = reinterpret_cast<float*>(S1);
    float* A32 = Y32 + ntc * l32;  // S1 hi
    for (int idx = t.tid; idx < ntc * ntc; idx += t.nthreads) {
        const int i = idx % ntc, j = idx / ntc;
        const float v = (i < n && j < n) ? float(S2[j * ld + i] * inv_fro) : 0.0f;
        X32[j * l32 + i] = v;
        A32[j * l32 + i] = v;
    }
    t.sync();
    const float lo_floor = PREC == kPrecTF32 ? 4e-3f : 3e-2f;  // ~8 u_lo sqrt(n)/sqrt(n)
    int iters_lo = 0;
    for (int it = 0; it < 120; ++it) {
        tc_gemm<PREC>(
            t, ntc, [&](int i, int k) { return X32[i * l32 + k]; },
            [&](int k, int j) { return X32[j * l32 + k]; },
            [&](int i, int j, float v) { T32[j * l32 + i] = v; });
        t.sync();
        float d2 = 0.f;
        tc_gemm<PREC>(
            t, ntc, [&](int i, int k) { return X32[k * l32 + i]; },
            [&](int k, int j) { return T32[j * l32 + k]; },
            [&](int i, int j, float v) {
                const float x = X32[j * l32 + i];
                const float xn = 1.5f * x - 0.5f * v;
                Y32[j * l32 + i] = xn;
                d2 += (xn - x) * (xn - x);
            });
        const double dd = team_sum(t, double(d2), sc->red);
        iters_lo = it + 1;
        float* tmp = X32;
        X32 = Y32;
        Y32 = tmp;
        if (!(dd < 1e6 * n)) break;  // non-finite guard; FP64 phases still run on A
        if (sqrt(dd) < double(lo_floor) * refn) break;
    }
    // ---- 2. P_lo = sym(X^T A) (into T32), then FP32 Jacobi -> V0 (in Y32)
    tc_gemm<PREC>(
        t, ntc, [&](int i, int k) { return X32[i * l32 + k]; },
        [&](int k, int j) { return A32[j * l32 + k]; },
        [&](int i, int j, float v) { T32[j * l32 + i] = v; });
    t.sync();
    for (int idx = t.tid; idx < ntc * ntc; idx += t.nthreads) {
        const int i = idx % ntc, j = idx / ntc;
        if (i < j) {
            const float s = (i < n && j < n) ? 0.5f * (T32[j * l32 + i] + T32[i * l32 + j]) : 0.f;
            T32[j * l32 + i] = s;
            T32[i * l32 + j] = s;
        } else if (i == j && i >= n) {
            T32[j * l32 + i] = 0.f;
        }
        Y32[j * l32 + i] = (i == j && i < n) ? 1.f : 0.f;
    }
    t.sync();
    long long rot_lo = 0;
    bool cap_lo = false;
    SmallJob nojob = job;
    nojob.rotors = nullptr;
    const int sweeps_lo = jacobi_sweeps<float, G>(t, n, T32, Y32, l32, 2e-5f,
                                                  PREC == kPrecTF32 ? 3e-3f : 1e-2f, 12, sc, nojob,
                                                  &rot_lo, &cap_lo);
    // V0 -> FP64 (S2: A is reloaded from global when needed)
    double* Xb = S2;
    double* Tb = S0;
    double* Yb = S1;
    for (int idx = t.tid; idx < np * np; idx += t.nthreads) {
        const int i = idx % np, j = idx / np;
        Xb[j * ld + i] = (i < n && j < n) ? double(Y32[j * l32 + i]) : 0.0;
    }
    t.sync();
    // ---- 3. FP64 Newton-Schulz refinement of V0 (quadratic: stop once the
    // update is below 1e-8, the next one would be at rounding level)
    int iters_hi = 0;
    for (int it = 0; it < 8; ++it) {
        team_gemm<TS>(
            t, np, n, [&](int k, int i) { return Xb[i * ld + k]; },
            [&](int k, int j) { return Xb[j * ld + k]; },
            [&](int i, int j, double v) { Tb[j * ld + i] = v; });
        t.sync();
        double d2 = 0.0;
        team_gemm<TS>(
            t, np, n, [&](int k, int i) { return Xb[k * ld + i]; },
            [&](int k, int j) { return Tb[j * ld + k]; },
            [&](int i, int j, double v) {
                const double x = Xb[j * ld + i];
                const double xn = 0.5 * (3.0 * x - v);
                Yb[j * ld + i] = xn;
                d2 += (xn - x) * (xn - x);
            });
        d2 = team_sum(t, d2, sc->red);
        iters_hi = it + 1;
        double* tmp = Xb;
        Xb = Yb;
        Yb = tmp;
        if (sqrt(d2) < 1e-8) break;
    }
    double* Vb = Xb;
    double* Ab = Tb;
    double* Wb = Yb;
    // ---- 4. W = (ascale A) V0, FP64 Jacobi cleanup
    for (int idx = t.tid; idx < np * np; idx += t.nthreads) {
        const int i = idx / np, j = idx - (idx / np) * np;
        Ab[j * ld + i] = (i < n && j < n) ? job.A[i * job.lda + j] * ascale : 0.0;
    }
    t.sync();
    team_gemm<TS>(
        t, np, n, [&](int k, int i) { return Ab[k * ld + i]; },
        [&](int k, int j) { return Vb[j * ld + k]; },
        [&](int i, int j, double v) { Wb[j * ld + i] = v; });
    if (t.tid == 0) sc->rotor_idx = 0;
    t.sync();
    long long rotations = 0;
    bool jcap = false;
    const int sweeps = jacobi_sweeps<double, G>(t, n, Wb, Vb, ld, double(n) * 2.220446049250313e-16,
                                                1e-9f, 60 + 20 * n, sc, job, &rotations, &jcap);
    if (jcap) flags |= LSVD_MAT_JACOBI_CAP;

    // ---- sigma, sort, U = W / sigma (+ repair), outputs
    {
        const int gpw = 32 / G;
        for (int base = t.warp * gpw; base < n; base += t.nwarps * gpw) {
            const int j = base + t.lane / G;
            double s = 0.0;
            for (int row = t.lane % G; row < n; row += G) {
                const double w = j < n ? Wb[j * ld + row] : 0.0;
                s = fma(w, w, s);
            }
            s = group_sum<G>(s);
            if (j < n && t.lane % G == 0) sc->sig[j] = sqrt(s);
        }
    }
    t.sync();
    for (int j = t.tid; j < n; j += t.nthreads) {
        const double sj = sc->sig[j];
        int rank = 0;
        for (int k = 0; k < n; ++k) {
            const double sk = sc->sig[k];
            rank += (sk > sj) || (sk == sj && k < j);
        }
        sc->perm[rank] = j;
    }
    t.sync();
    const int* perm = sc->perm;
    double smax = 0.0;
    for (int k = 0; k < n; ++k) smax = fmax(smax, sc->sig[k]);
    const double stol = 1e-12 * fmax(smax, ascale);  // 1e-12 max(sigma_max, 1) in scaled units
    double* Ub = Ab;  // A is dead
    int zero_cols = 0;
    for (int idx = t.tid; idx < np * np; idx += t.nthreads) {
        const int i = idx % np, j = idx / np;
        double v = 0.0;
        if (i < n && j < n) {
            const double sj = sc->sig[perm[j]];
            v = sj > stol ? Wb[perm[j] * ld + i] / sj : 0.0;
            if (i == 0 && !(sj > stol)) zero_cols++;
        }
        Ub[j * ld + i] = v;
    }
    const double nzero = team_sum(t, double(zero_cols), sc->red);
    auto orth_of = [&](const double* B) -> double {
        double o2 = 0.0;
        team_gemm<TS>(
            t, np, n, [&](int k, int i) { return B[i * ld + k]; },
            [&](int k, int j) { return B[j * ld + k]; },
            [&](int i, int j, double v) {
                if (i < n && j < n) {
                    const double d = v - (i == j ? 1.0 : 0.0);
                    o2 += d * d;
                }
            });
        return sqrt(team_sum(t, o2, sc->red));
    };
    double orth_u = orth_of(Ub);
    if (nzero > 0.0 || orth_u > 1e-8 * refn) {
        flags |= LSVD_MAT_REPAIRED;
        warp_mgs(t, Ub, n, ld);
        t.sync();
        if (job.want_diag) orth_u = orth_of(Ub);
    }
    for (int idx = t.tid; idx < n * n; idx += t.nthreads) {
        const int i = idx / n, j = idx % n;
        job.U[i * job.ldu + j] = Ub[j * ld + i];
        job.Vt[i * job.ldvt + j] = Vb[perm[i] * ld + j];
    }
    for (int i = t.tid; i < n; i += t.nthreads) {
        job.S[i] = sc->sig[perm[i]] / ascale;
        if (job.perm_out) job.perm_out[i] = perm[i];
    }
    const double qnan = __longlong_as_double(0x7ff8000000000000ULL);
    double rel_recon = qnan, orth_v = qnan;
    if (job.want_diag) {
        orth_v = orth_of(Vb);
        // reload A (unscaled) into W's buffer: W is dead after sigma/U
        for (int idx = t.tid; idx < np * np; idx += t.nthreads) {
            const int i = idx / np, j = idx - (idx / np) * np;
            Wb[j * ld + i] = (i < n && j < n) ? job.A[i * job.lda + j] : 0.0;
        }
        t.sync();
        double r2 = 0.0;
        team_gemm<TS>(
            t, np, n, [&](int k, int i) { return Ub[k * ld + i]; },
            [&](int k, int j) {
                return j < n ? (sc->sig[perm[k]] / ascale) * Vb[perm[k] * ld + j] : 0.0;
            },
            [&](int i, int j, double v) {
                if (i < n && j < n) {
                    const double d = v - Wb[j * ld + i];
                    r2 += d * d;
                }
            });
        rel_recon = sqrt(team_sum(t, r2, sc->red)) / fmax(afro, 1e-300);
    }
    if (t.tid == 0) {
        if (job.rotor_count) *job.rotor_count = sc->rotor_idx;
        if (job.agg && flags) atomicOr(job.agg, flags);
        if (job.diag) {
            lsvd_diag d;
            d.rel_recon = rel_recon;
            d.orth_u = job.want_diag ? orth_u : qnan;
            d.orth_v = orth_v;
            // low-precision + FP64 Newton-Schulz iterations, low-precision + FP64 sweeps
            d.ns_iters = iters_lo * 1000 + iters_hi;
            d.jacobi_sweeps = sweeps_lo * 1000 + sweeps;
            d.rotations = rotations;
            d.flags = flags;
            d.route = LSVD_ROUTE_SMALL;
            *job.diag = d;
        }
    }
    t.sync();
}

}  // namespace lsvd
