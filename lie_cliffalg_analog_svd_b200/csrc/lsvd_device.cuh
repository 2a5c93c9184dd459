// lsvd_device.cuh -- device-side building blocks of the B200 SVD hot path.
//
// A "team" is 1, 2, 4 or 8 warps of a 256-thread CTA that solves one matrix
// with everything resident in shared memory (n <= 64: three n x n FP64
// buffers, column-major, leading dimension np+1 with np = n rounded up to 4,
// which makes column walks and the interleaved GEMM tiles bank-conflict free).
// Teams synchronise on their own named barrier (bar.sync id, 32*W), so up to
// eight matrices progress independently inside one CTA.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lsvd.h"

namespace lsvd {

constexpr int kMaxN = 64;
constexpr int kCtaThreads = 256;

struct Team {
    int tid;       // 0 .. nthreads-1
    int nthreads;  // 32 * nwarps
    int warp;      // warp index inside the team
    int lane;
    int nwarps;
    int bar;       // named barrier id (1..15)
    __device__ __forceinline__ void sync() const {
        if (nwarps == 1)
            __syncwarp();
        else
            asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nthreads) : "memory");
    }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over aligned groups of G lanes (all 32 lanes must call).
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Deterministic team-wide sum (same value on every thread).  red >= nwarps.
__device__ __forceinline__ double team_sum(const Team& t, double v, double* red) {
    v = warp_sum(v);
    if (t.nwarps == 1) return v;
    if (t.lane == 0) red[t.warp] = v;
    t.sync();
    double s = 0.0;
    for (int w = 0; w < t.nwarps; ++w) s += red[w];
    t.sync();
    return s;
}

__device__ __forceinline__ double team_max(const Team& t, double v, double* red) {
    v = warp_max(v);
    if (t.nwarps == 1) return v;
    if (t.lane == 0) red[t.warp] = v;
    t.sync();
    double s = 0.0;
    for (int w = 0; w < t.nwarps; ++w) s = fmax(s, red[w]);
    t.sync();
    return s;
}

// Register-tiled FP64 GEMM over a team: C(i, j) = sum_{k<kdim} a(k, i) b(k, j)
// for i, j < np.  Each thread owns TS x TS outputs at rows ti + r*nt and
// columns tj + c*nt (interleaved tiles, nt = np/TS): consecutive lanes touch
// consecutive rows, so column-major operands stream conflict-free.
// epi(i, j, value) consumes each output.
template <int TS, class LA, class LB, class Epi>
__device__ __forceinline__ void team_gemm(const Team& t, int np, int kdim, LA la, LB lb, Epi epi) {
    const int nt = np / TS;
    const int ntiles = nt * nt;
    for (int tile = t.tid; tile < ntiles; tile += t.nthreads) {
        const int ti = tile % nt, tj = tile / nt;
        double acc[TS][TS];
#pragma unroll
        for (int r = 0; r < TS; ++r)
#pragma unroll
            for (int c = 0; c < TS; ++c) acc[r][c] = 0.0;
#pragma unroll 4
        for (int k = 0; k < kdim; ++k) {
            double av[TS], bv[TS];
#pragma unroll
            for (int r = 0; r < TS; ++r) av[r] = la(k, ti + r * nt);
#pragma unroll
            for (int c = 0; c < TS; ++c) bv[c] = lb(k, tj + c * nt);
#pragma unroll
            for (int r = 0; r < TS; ++r)
#pragma unroll
                for (int c = 0; c < TS; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
        }
#pragma unroll
        for (int r = 0; r < TS; ++r)
#pragma unroll
            for (int c = 0; c < TS; ++c) epi(ti + r * nt, tj + c * nt, acc[r][c]);
    }
}

// D += A B on one 8 x 8 tile: FP64 mma.sync m8n8k4.  Fragments (lane =
// 4 g + q): a = A[g][q], b = B[q][g], d = D[g][2q], D[g][2q + 1].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// C[i][j] = sum_k A(k, i) B(k, j) for i, j < np (np a multiple of 8), the
// same contract as team_gemm, on the FP64 tensor path: each warp owns a block
// of 2 x wn 8 x 8 tiles (wn = ceil(np / 16) <= 4) and runs kdim rounded up to
// 4 in k-steps of 4 (A and B must read zeros for k in [kdim, that)).  Every
// lane calls epi for its two outputs of each tile it owns.
template <class LA, class LB, class Epi>
__device__ __forceinline__ void team_mma(const Team& t, int np, int kdim, LA la, LB lb, Epi epi) {
    const int nt8 = np >> 3;
    const int wn = (nt8 + 1) >> 1;
    const int nblk = ((nt8 + 1) >> 1) * 2;
    const int g = t.lane >> 2, q = t.lane & 3;
    const int kd = (kdim + 3) & ~3;
    for (int blk = t.warp; blk < nblk; blk += t.nwarps) {
        const int ti0 = (blk >> 1) * 2, tj0 = (blk & 1) * wn;
        bool vr[2], vc[4];
#pragma unroll
        for (int r = 0; r < 2; ++r) vr[r] = ti0 + r < nt8;
#pragma unroll
        for (int c = 0; c < 4; ++c) vc[c] = c < wn && tj0 + c < nt8;
        double acc[2][4][2];
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[r][c][0] = acc[r][c][1] = 0.0;
#pragma unroll 2
        for (int k0 = 0; k0 < kd; k0 += 4) {
            double a[2], b[4];
#pragma unroll
            for (int r = 0; r < 2; ++r) a[r] = vr[r] ? la(k0 + q, (ti0 + r) * 8 + g) : 0.0;
#pragma unroll
            for (int c = 0; c < 4; ++c) b[c] = vc[c] ? lb(k0 + q, (tj0 + c) * 8 + g) : 0.0;
#pragma unroll
            for (int r = 0; r < 2; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    if (vc[c]) dmma_8x8x4(acc[r][c][0], acc[r][c][1], a[r], b[c]);
        }
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (vr[r] && vc[c]) {
                    const int i = (ti0 + r) * 8 + g, j = (tj0 + c) * 8 + 2 * q;
                    epi(i, j, acc[r][c][0]);
                    epi(i, j + 1, acc[r][c][1]);
                }
    }
}

// Pair k of round-robin layer `layer` over m (= n rounded up to even)
// indices: the circle method of layer_pairs, src/lie_svd_joint.rs:524-539.
__device__ __forceinline__ void rr_pair(int m, int layer, int k, int& a, int& b) {
    const int ring = m - 1;
    if (k == 0) {
        a = m - 1;
        b = layer % ring;
    } else {
        a = (layer + k) % ring;
        b = (layer + ring - k) % ring;
    }
}

// ---------------------------------------------------------------- Micro ----
// LieSvdMicro::solve (src/lie_svd_micro.rs:21-214) for one matrix per thread,
// everything in registers.  Returns false when the reference would escalate
// to LieSvdSmall (off-diagonal > 1e-10 max(||A||_F, 1), :90-92).

__device__ __forceinline__ double wrap_half_pi(double a) {
    const double kPi = 3.141592653589793238462643383279502884;
    while (a > 0.5 * kPi) a -= kPi;
    while (a < -0.5 * kPi) a += kPi;
    return a;
}

template <int N>
__device__ __forceinline__ double micro_offdiag(const double (&w)[N][N]) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (i != j) s += w[i][j] * w[i][j];
    return sqrt(s);
}

template <int N>
__device__ __forceinline__ void micro_rot_rows(double (&w)[N][N], int i, int j, double s, double c) {
#pragma unroll
    for (int col = 0; col < N; ++col) {
        const double ai = w[i][col], aj = w[j][col];
        w[i][col] = c * ai - s * aj;
        w[j][col] = s * ai + c * aj;
    }
}
template <int N>
__device__ __forceinline__ void micro_rot_cols(double (&w)[N][N], int i, int j, double s, double c) {
#pragma unroll
    for (int r = 0; r < N; ++r) {
        const double ai = w[r][i], aj = w[r][j];
        w[r][i] = c * ai - s * aj;
        w[r][j] = s * ai + c * aj;
    }
}

struct MicroOut {
    int sweeps;
    int rotations;
    bool ok;
    bool nonfinite;
};

// Fixed pair schedules of src/lie_svd_micro.rs:41-48.
__device__ __forceinline__ void micro_pair(int n, int k, int& i, int& j) {
    if (n == 2) {
        i = 0; j = 1;
    } else if (n == 3) {
        const int pi[3] = {0, 0, 1}, pj[3] = {1, 2, 2};
        i = pi[k]; j = pj[k];
    } else {
        const int pi[6] = {0, 2, 0, 1, 0, 1}, pj[6] = {1, 3, 2, 3, 3, 2};
        i = pi[k]; j = pj[k];
    }
}

template <int N>
__device__ MicroOut micro_solve_regs(const double* __restrict__ A, int64_t lda, double* U,
                                     int64_t ldu, double* S, double* Vt, int64_t ldvt) {
    MicroOut out{0, 0, true, false};
    double w[N][N], ub[N][N], vb[N][N];
    double fro2 = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            w[i][j] = A[i * lda + j];
            fro2 += w[i][j] * w[i][j];
            ub[i][j] = vb[i][j] = (i == j) ? 1.0 : 0.0;
            if (!isfinite(w[i][j])) out.nonfinite = true;
        }
    const double ref = fmax(sqrt(fro2), 1e-300);
    const double tol = 1e-13 * fmax(ref, 1.0);  // MICRO_TOL, :15 and :65
    const int max_sweeps = (N == 2) ? 1 : 24;
    constexpr int NP = (N == 2) ? 1 : (N == 3 ? 3 : 6);
    for (int sw = 0; sw < max_sweeps; ++sw) {
        const double e = micro_offdiag<N>(w);
        if (e <= tol || !isfinite(e)) break;
        out.sweeps = sw + 1;
        bool changed = false;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            int i, j;
            micro_pair(N, k, i, j);
            if (fabs(w[i][j]) + fabs(w[j][i]) <= tol) continue;
            // local_pair_svd_angles, :128-139
            const double sum = atan2(-(w[i][j] + w[j][i]), w[i][i] - w[j][j]);
            const double diff = atan2(w[i][j] - w[j][i], w[i][i] + w[j][j]);
            const double tl = wrap_half_pi(0.5 * (sum + diff));
            const double tr = wrap_half_pi(0.5 * (sum - diff));
            if (fabs(tl) + fabs(tr) <= 1e-18) continue;
            double sl, cl, sr, cr;
            sincos(tl, &sl, &cl);
            sincos(tr, &sr, &cr);
            micro_rot_rows<N>(w, i, j, sl, cl);
            micro_rot_cols<N>(ub, i, j, sl, cl);
            micro_rot_cols<N>(w, i, j, sr, cr);
            micro_rot_cols<N>(vb, i, j, sr, cr);
            changed = true;
            out.rotations++;
        }
        if (!changed) break;
    }
    if (micro_offdiag<N>(w) > 1e-10 * fmax(ref, 1.0)) {
        out.ok = false;
        return out;
    }
    // extract_sorted_svd, :187-214: stable sort by |diag| descending.
    int order[N];
#pragma unroll
    for (int i = 0; i < N; ++i) order[i] = i;
#pragma unroll
    for (int i = 1; i < N; ++i) {
        // insertion sort (stable): move order[i] left past smaller |diag|
        for (int k = i; k > 0; --k) {
            const int a = order[k - 1], b = order[k];
            double da = 0, db = 0;
#pragma unroll
            for (int q = 0; q < N; ++q) {
                if (q == a) da = fabs(w[q][q]);
                if (q == b) db = fabs(w[q][q]);
            }
            if (da < db) {
                order[k - 1] = b;
                order[k] = a;
            }
        }
    }
#pragma unroll
    for (int dst = 0; dst < N; ++dst) {
        const int src = order[dst];
        double d = 0.0;
#pragma unroll
        for (int q = 0; q < N; ++q)
            if (q == src) d = w[q][q];
        S[dst] = fabs(d);
        const double sg = d < 0.0 ? -1.0 : 1.0;
#pragma unroll
        for (int r = 0; r < N; ++r) {
            double uv = 0.0, vv = 0.0;
#pragma unroll
            for (int q = 0; q < N; ++q)
                if (q == src) {
                    uv = ub[r][q];
                    vv = vb[r][q];
                }
            U[r * ldu + dst] = sg * uv;
            Vt[dst * ldvt + r] = vv;
        }
    }
    return out;
}

// ---------------------------------------------------------------- Small ----

struct alignas(16) TeamScratch {
    double red[8];
    double sig[kMaxN];
    // rotation of each pair of the current round-robin layer (two-sided sweep)
    double rc[kMaxN / 2], rs[kMaxN / 2], rt[kMaxN / 2];
    int rp[kMaxN / 2], rq[kMaxN / 2];
    int pidx[2][kMaxN];  // index held at each position (ping-pong by layer parity)
    int perm[kMaxN];
    int cnt[4];
    int rotor_idx;
    int pad_;
};

__host__ __device__ constexpr int pad4(int n) { return (n + 3) & ~3; }
__host__ __device__ constexpr int pad8(int n) { return (n + 7) & ~7; }
// Eight-warp teams with n > 32 run their products on the FP64 tensor path
// (mma.sync m8n8k4, team_mma): buffers padded to 8 with leading dimension
// np + 4 (= 4 mod 8, so that the 8 x 4 fragment loads of a half-warp hit 16
// distinct banks).  Other teams use the scalar register-tiled team_gemm with
// np = n rounded up to 4 and an odd leading dimension np + 1.
__host__ __device__ constexpr bool team_uses_mma(int n, int nwarps) { return nwarps == 8 && n > 32; }
__host__ __device__ constexpr int team_np(int n, bool mma) { return mma ? pad8(n) : pad4(n); }
__host__ __device__ constexpr int team_ld(int n, bool mma) { return mma ? pad8(n) + 4 : pad4(n) + 1; }
// Doubles of shared memory a team of `nwarps` warps needs for an n x n solve.
__host__ __device__ constexpr int team_smem_doubles(int n, int nwarps) {
    return 3 * team_ld(n, team_uses_mma(n, nwarps)) * team_np(n, team_uses_mma(n, nwarps)) +
           int(sizeof(TeamScratch) / sizeof(double));
}

struct SmallJob {
    int n;
    const double* A;
    int64_t lda;
    double* U;
    int64_t ldu;
    double* S;
    double* Vt;
    int64_t ldvt;
    lsvd_diag* diag;  // may be null
    lsvd_rotor* rotors;
    int64_t rotor_cap;
    int64_t* rotor_count;  // device, may be null
    int32_t* perm_out;     // may be null
    bool want_diag;
    int extra_flags;  // e.g. LSVD_MAT_MICRO_FALLBACK
    int* agg;         // OR of outcome flags over a batch (may be null)
};

// Loads row-major A (global) into column-major smem buffer B (np x np,
// zero-padded).  Returns sum of squares and counts non-finite entries.
__device__ __forceinline__ void load_colmajor(const Team& t, const SmallJob& job, int np, int ld,
                                              double* B, double& fro2, int& bad) {
    const int n = job.n;
    for (int idx = t.tid; idx < np * np; idx += t.nthreads) {
        const int i = idx / np, j = idx - (idx / np) * np;
        double v = 0.0;
        if (i < n && j < n) {
            v = job.A[i * job.lda + j];
            fro2 += v * v;
            if (!isfinite(v)) bad++;
        }
        B[j * ld + i] = v;
    }
}

// Modified Gram-Schmidt of the n columns of B (in place) with the
// rank-deficient fill of gram_schmidt_orthonormal, src/lie_svd_small.rs:82-144.
// Executed by warp 0 of the team (lanes hold rows lane and lane+32).
__device__ inline void warp_mgs(const Team& t, double* B, int n, int ld) {
    if (t.warp != 0) return;
    const int l0 = t.lane, l1 = t.lane + 32;
    auto col = [&](int j, int row) -> double { return row < n ? B[j * ld + row] : 0.0; };
    for (int j = 0; j < n; ++j) {
        double v0 = col(j, l0), v1 = col(j, l1);
        for (int k = 0; k < j; ++k) {
            const double q0 = col(k, l0), q1 = col(k, l1);
            const double d = warp_sum(q0 * v0 + q1 * v1);
            v0 -= d * q0;
            v1 -= d * q1;
        }
        const double nrm = sqrt(warp_sum(v0 * v0 + v1 * v1));
        if (nrm >= 1e-10) {
            v0 /= nrm;
            v1 /= nrm;
        } else {
            double best_norm = -1.0, b0 = 0.0, b1 = 0.0;
            for (int kk = 0; kk < n; ++kk) {
                double c0 = (l0 == kk) ? 1.0 : 0.0, c1 = (l1 == kk) ? 1.0 : 0.0;
                for (int cc = 0; cc < j; ++cc) {
                    const double q0 = col(cc, l0), q1 = col(cc, l1);
                    const double d = warp_sum(q0 * c0 + q1 * c1);
                    c0 -= d * q0;
                    c1 -= d * q1;
                }
                const double en = sqrt(warp_sum(c0 * c0 + c1 * c1));
                if (en > best_norm) {
                    best_norm = en;
                    b0 = c0;
                    b1 = c1;
                }
            }
            if (best_norm > 0.0 && isfinite(best_norm)) {
                v0 = b0 / best_norm;
                v1 = b1 / best_norm;
            } else {
                v0 = (l0 == j) ? 1.0 : 0.0;
                v1 = (l1 == j) ? 1.0 : 0.0;
            }
        }
        if (l0 < n) B[j * ld + l0] = v0;
        if (l1 < n) B[j * ld + l1] = v1;
        __syncwarp();
    }
}

template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }

struct LayerStats {
    int nrot;     // rotations recorded by this thread (group leaders only)
    float cmax2;  // largest squared cosine this thread saw before rotating
};

// One round-robin layer of one-sided (Hestenes) Jacobi on the columns of W,
// accumulating V, in precision Real (double, or float for the low-precision
// phase of the mixed path).  Each pair is handled by an aligned group of G
// lanes (rows gl + G*r); the three Gram entries are group-shuffle reductions.
template <class Real, int G>
__device__ __forceinline__ void jacobi_layer(const Team& t, int n, int m, int layer, Real* W,
                                             Real* V, int ld, Real tol2, TeamScratch* sc,
                                             const SmallJob& job, uint32_t round, LayerStats& st) {
    constexpr int R = kMaxN / G;
    constexpr int GPW = 32 / G;
    const int half = m >> 1;
    const int gl = t.lane % G;
    const int ngroups = t.nwarps * GPW;
    for (int base = t.warp * GPW; base < half; base += ngroups) {
        const int k = base + t.lane / G;
        int a = 0, b = 0;
        bool valid = k < half;
        if (valid) {
            rr_pair(m, layer, k, a, b);
            valid = a < n && b < n;
        }
        const int p = min(a, b), q = max(a, b);
        Real wp[R], wq[R], vp[R], vq[R];
        Real al = 0, be = 0, ga = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int row = gl + G * r;
            const bool in = valid && row < n;
            wp[r] = in ? W[p * ld + row] : Real(0);
            wq[r] = in ? W[q * ld + row] : Real(0);
            // V is prefetched so its latency overlaps the reductions
            vp[r] = in ? V[p * ld + row] : Real(0);
            vq[r] = in ? V[q * ld + row] : Real(0);
            al = fma(wp[r], wp[r], al);
            be = fma(wq[r], wq[r], be);
            ga = fma(wp[r], wq[r], ga);
        }
        al = group_sum<G>(al);
        be = group_sum<G>(be);
        ga = group_sum<G>(ga);
        // Columns are scaled so that al, be <= 4n: the squared test cannot
        // overflow, and it needs no square roots.
        const Real ab = al * be;
        const bool rot = valid && ga != Real(0) && al > Real(0) && be > Real(0) && ga * ga > tol2 * ab;
        if (rot) {
            st.cmax2 = fmaxf(st.cmax2, float((ga * ga) / ab));
            // Rutishauser's smaller-root tangent of eigh_jacobi_full
            // (src/lie_svd_small.rs:235-242) for the 2x2 Gram block
            // [[al, ga], [ga, be]]: with zeta = (be - al) / (2 ga),
            // t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2))
            //   = sign(be - al) * 2 ga / (|be - al| + hypot(be - al, 2 ga)).
            const Real dd = be - al, g2 = Real(2) * ga;
            const Real tt0 = g2 / (fabs(dd) + sqrt(fma(dd, dd, g2 * g2)));
            const Real tt = dd < Real(0) ? -tt0 : tt0;
            const Real c = rsqrt_t(fma(tt, tt, Real(1)));
            const Real s = tt * c;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int row = gl + G * r;
                if (row < n) {
                    W[p * ld + row] = c * wp[r] - s * wq[r];
                    W[q * ld + row] = s * wp[r] + c * wq[r];
                    V[p * ld + row] = c * vp[r] - s * vq[r];
                    V[q * ld + row] = s * vp[r] + c * vq[r];
                }
            }
            if (gl == 0) {
                st.nrot++;
                if (job.rotors) {
                    const int idx = atomicAdd(&sc->rotor_idx, 1);
                    if (idx < job.rotor_cap) {
                        lsvd_rotor rr;
                        rr.i = (uint16_t)p;
                        rr.j = (uint16_t)q;
                        rr.round = round;
                        rr.theta = atan(double(tt));
                        job.rotors[idx] = rr;
                    }
                }
            }
        }
    }
}

// Round-robin one-sided Jacobi sweeps on W (n columns) accumulating V until
// a sweep rotates nothing, or the largest cosine a sweep met is <= stop_cos
// (quadratic convergence: the next sweep would only see rounding noise), or
// max_sweeps.  Rotates pairs whose cosine exceeds tol.  Returns sweeps run;
// adds the rotation count to *rotations; sets *capped if max_sweeps was hit.
template <class Real, int G>
__device__ int jacobi_sweeps(const Team& t, int n, Real* W, Real* V, int ld, Real tol,
                             float stop_cos, int max_sweeps, TeamScratch* sc, const SmallJob& job,
                             long long* rotations, bool* capped) {
    const int m = (n % 2 == 0) ? n : n + 1;
    const int layers = (n % 2 == 0) ? (n > 0 ? n - 1 : 0) : n;  // round_robin_layer_count
    const Real tol2 = tol * tol;
    int sweeps = 0;
    *capped = false;
    for (int sw = 0; sw < max_sweeps; ++sw) {
        sweeps = sw + 1;
        LayerStats st{0, 0.0f};
        for (int layer = 0; layer < layers; ++layer) {
            jacobi_layer<Real, G>(t, n, m, layer, W, V, ld, tol2, sc, job,
                                  uint32_t(sw * layers + layer), st);
            t.sync();
        }
        const int rotated = int(team_sum(t, double(st.nrot), sc->red));
        const double cmax2 = team_max(t, double(st.cmax2), sc->red);
        *rotations += rotated;
        if (rotated == 0 || cmax2 <= double(stop_cos) * double(stop_cos)) break;
        if (sw + 1 == max_sweeps) *capped = true;
    }
    return sweeps;
}

// Position of index i in round-robin layer l over m indices (ring = m - 1):
// pair k occupies positions 2k (smaller index) and 2k + 1 (larger index).
__device__ __forceinline__ int rr_position(int m, int l, int i) {
    const int ring = m - 1, half = m >> 1;
    if (i == m - 1) return 1;  // always in pair 0 with l % ring, and the larger index
    int d = i - l;  // 0 <= i, l < ring
    if (d < 0) d += ring;
    int k, j;
    if (d == 0) {
        k = 0;
        j = m - 1;
    } else if (d <= half - 1) {
        k = d;
        j = l + ring - k;
        if (j >= ring) j -= ring;
    } else {
        k = ring - d;
        j = l + k;
        if (j >= ring) j -= ring;
    }
    return 2 * k + (i > j ? 1 : 0);
}

// Two-sided round-robin Jacobi of eigh_jacobi_full (src/lie_svd_small.rs:
// 212-285) with P kept in pair-position order: in layer l, positions 2k and
// 2k+1 hold the pair (p_k < q_k), so every 2x2 block R_a^T P[a,b] R_b is two
// contiguous double2 loads, and the transformed block is written straight to
// the next layer's positions in the other buffer (ping-pong B0/B1, leading
// dimension m).  V stays in natural order.  Every warp computes the angles of
// all pairs of the layer itself (lane k <-> pair k, m <= 64) and fetches them
// by shuffle, so a layer costs one barrier.  Rotation: the reference's
// smaller-root tangent (:235-242) written t = sign(d) 2 a_pq / (|d| +
// hypot(d, 2 a_pq)), d = a_qq - a_pp; skip if |a_pq| < 1e-300; exact diagonal
// update (:244-249).  Convergence test at sweep start: sqrt(sum_{p<q}
// P_pq^2) < 1e-13 ||P||_F (:220-228).  On return *Pout holds P in the
// positions of sc->pidx[*par]; returns the sweeps started.
__device__ inline int jacobi2pp_sweeps(const Team& t, int n, double* B0, double* B1, double* V,
                                       int ldv, double ref_norm, int max_sweeps, TeamScratch* sc,
                                       const SmallJob& job, long long* rotations, bool* capped,
                                       double** Pout, int* par) {
    const int m = (n % 2 == 0) ? n : n + 1;
    const int half = m >> 1;
    const int layers = (n % 2 == 0) ? (n > 0 ? n - 1 : 0) : n;
    int sweeps = 0;
    *capped = false;
    double* cur = B0;
    double* nxt = B1;
    int cp = 0;  // parity of sc->pidx describing cur
    const int lane = t.lane;
    // The per-item indices below advance by t.nthreads each pass; their
    // starts and steps are divided out once here, so the layer loops carry
    // no integer division (runtime divisors cost ~20 instructions each).
    const int p_a0 = (t.warp * 32 + lane) % half, p_b0 = (t.warp * 32 + lane) / half;
    const int p_da = t.nthreads % half, p_db = t.nthreads / half;
    const int v_i0 = n > 0 ? (t.warp * 32 + lane) % n : 0, v_b0 = n > 0 ? (t.warp * 32 + lane) / n : 0;
    const int v_di = n > 0 ? t.nthreads % n : 0, v_db = n > 0 ? t.nthreads / n : 0;
    for (int sw = 0; sw < max_sweeps; ++sw) {
        sweeps = sw + 1;
        double off = 0.0;
        for (int idx = t.tid; idx < m * m; idx += t.nthreads) {
            const int x = idx % m, y = idx / m;
            if (x != y) off = fma(cur[y * m + x], cur[y * m + x], off);
        }
        off = 0.5 * team_sum(t, off, sc->red);
        if (sqrt(off) < 1e-13 * ref_norm) break;  // JACOBI_TOL, :69
        if (sw + 1 == max_sweeps) *capped = true;
        int nrot = 0;
        for (int l = 0; l < layers; ++l) {
            const int lnext = (l + 1 == layers) ? 0 : l + 1;
            // every warp: lane k computes the rotation of pair k
            double c = 1.0, s = 0.0, tt = 0.0;
            int xk = 0, yk = 0;
            if (lane < half) {
                const int k = lane;
                const int p = sc->pidx[cp][2 * k], q = sc->pidx[cp][2 * k + 1];
                if (q < n) {
                    const double2 d0 = *reinterpret_cast<const double2*>(cur + (2 * k) * m + 2 * k);
                    const double2 d1 = *reinterpret_cast<const double2*>(cur + (2 * k + 1) * m + 2 * k);
                    const double apq = d1.x;
                    if (fabs(apq) >= 1e-300) {
                        const double dd = d1.y - d0.x, g2 = 2.0 * apq;
                        const double t0 = g2 / (fabs(dd) + sqrt(fma(dd, dd, g2 * g2)));
                        tt = dd < 0.0 ? -t0 : t0;
                        c = rsqrt(fma(tt, tt, 1.0));
                        s = tt * c;
                    }
                }
                xk = rr_position(m, lnext, p);
                yk = rr_position(m, lnext, q);
                if (t.warp == 0) {
                    sc->pidx[cp ^ 1][xk] = p;
                    sc->pidx[cp ^ 1][yk] = q;
                    if (s != 0.0) {
                        nrot++;
                        if (job.rotors) {
                            const int ri = atomicAdd(&sc->rotor_idx, 1);
                            if (ri < job.rotor_cap) {
                                lsvd_rotor rr;
                                rr.i = (uint16_t)p;
                                rr.j = (uint16_t)q;
                                rr.round = uint32_t(sw * layers + l);
                                rr.theta = atan(tt);
                                job.rotors[ri] = rr;
                            }
                        }
                    }
                }
            }
            // P <- J^T P J into the next layer's positions
            const int nb = half * half;
            int a = p_a0, b = p_b0;
            for (int base = t.warp * 32; base < nb; base += t.nthreads, a += p_da, b += p_db) {
                if (a >= half) {
                    a -= half;
                    b++;
                }
                const int bi = base + lane;
                const double ca = __shfl_sync(0xffffffffu, c, a), sa = __shfl_sync(0xffffffffu, s, a);
                const double cb = __shfl_sync(0xffffffffu, c, b & 31), sb = __shfl_sync(0xffffffffu, s, b & 31);
                const double ta = __shfl_sync(0xffffffffu, tt, a);
                const int xa = __shfl_sync(0xffffffffu, xk, a), ya = __shfl_sync(0xffffffffu, yk, a);
                const int xb = __shfl_sync(0xffffffffu, xk, b & 31), yb = __shfl_sync(0xffffffffu, yk, b & 31);
                if (bi >= nb) continue;
                const double2 c0 = *reinterpret_cast<const double2*>(cur + (2 * b) * m + 2 * a);
                const double2 c1 = *reinterpret_cast<const double2*>(cur + (2 * b + 1) * m + 2 * a);
                if (a == b) {
                    // c0 = (P_pp, P_qp), c1 = (P_pq, P_qq)
                    double d00 = c0.x, d11 = c1.y, d01 = c1.x, d10 = c0.y;
                    if (sa != 0.0) {
                        d00 = c0.x - ta * c1.x;
                        d11 = c1.y + ta * c1.x;
                        d01 = 0.0;
                        d10 = 0.0;
                    }
                    nxt[xa * m + xa] = d00;
                    nxt[ya * m + ya] = d11;
                    nxt[ya * m + xa] = d01;
                    nxt[xa * m + ya] = d10;
                    continue;
                }
                // block rows (p_a, q_a) x cols (p_b, q_b): b00 = c0.x, b10 = c0.y, b01 = c1.x, b11 = c1.y
                const double x00 = cb * c0.x - sb * c1.x, x01 = sb * c0.x + cb * c1.x;
                const double x10 = cb * c0.y - sb * c1.y, x11 = sb * c0.y + cb * c1.y;
                nxt[xb * m + xa] = ca * x00 - sa * x10;
                nxt[xb * m + ya] = sa * x00 + ca * x10;
                nxt[yb * m + xa] = ca * x01 - sa * x11;
                nxt[yb * m + ya] = sa * x01 + ca * x11;
            }
            // V <- V J (natural order); item = (pair b, row i)
            const int nv = half * n;
            int vb = v_b0, vi_ = v_i0;
            for (int base = t.warp * 32; base < nv; base += t.nthreads, vi_ += v_di, vb += v_db) {
                if (vi_ >= n) {
                    vi_ -= n;
                    vb++;
                }
                const int vi = base + lane;
                const int b = vb, i = vi_;
                const double cb = __shfl_sync(0xffffffffu, c, b & 31), sb = __shfl_sync(0xffffffffu, s, b & 31);
                if (vi >= nv) continue;
                const int ib = sc->pidx[cp][2 * b], jb = sc->pidx[cp][2 * b + 1];
                if (jb >= n || sb == 0.0) continue;
                const double vp = V[ib * ldv + i], vq = V[jb * ldv + i];
                V[ib * ldv + i] = cb * vp - sb * vq;
                V[jb * ldv + i] = sb * vp + cb * vq;
            }
            t.sync();
            double* tmp = cur;
            cur = nxt;
            nxt = tmp;
            cp ^= 1;
        }
        *rotations += (long long)team_sum(t, double(nrot), sc->red);
    }
    *Pout = cur;
    *par = cp;
    return sweeps;
}

// Blocked two-sided Jacobi for the same eigensolve (eigh_jacobi_full,
// src/lie_svd_small.rs:212-285), used when no rotor stream is requested.
// Indices are cut into blocks of B (8 for n >= 45, else 4) and the blocks
// are paired by the circle method; in block layer l every block pair k owns
// 2B indices.  One warp solves the 2B x 2B principal sub-block S_k of its
// block pair: B rounds of B disjoint rotations (cross pairs; at layer 0 also
// the B-1 rounds of pairs inside the blocks), each with the reference's
// tangent, skip rule and exact diagonal update, accumulated into R_k.  The
// team then applies all R_k at once, W = P R and V <- V R (rows of P and V,
// in place, one (row, block pair) segment per item), then P' = R^T W
// (columns, in place), writing the solved S_k on the diagonal tiles.  Every
// index pair is visited once per sweep, as in the reference; the pair order
// differs.  The P data in shared memory move once per block layer instead of
// once per rotation layer, and R is applied with 2B FMAs per load.
// P: natural order, column-major, leading dimension pld; scr: scratch of
// nbp * 2 * (2B)^2 doubles.  Returns the sweeps started.
// Smallest n for the blocked sweep (where it overtakes the layer-by-layer
// sweep on B200; a build may override it).
#ifndef LSVD_BLOCK_JACOBI_MIN_N
#define LSVD_BLOCK_JACOBI_MIN_N 33
#endif

// Whether the blocked sweep with block size B fits in scr_doubles of scratch:
// sub-blocks S, R per block pair, then the block-pair table (64 ints).
__device__ __forceinline__ bool block_jacobi_fits_b(int n, int B, int scr_doubles) {
    const int B2 = 2 * B;
    const int nbl = (n + B - 1) / B, nbe = nbl + (nbl & 1);
    return (nbe / 2) * 2 * B2 * (B2 + 2) + 32 <= scr_doubles && nbe >= 2 && (nbe / 2) * B <= 32;
}

// Block size of the blocked sweep: 8 from n = 41 where the scratch holds it
// (fewer layers; the team's tensor-path layout does for every n > 32), else
// 4; 0 when neither fits.
__device__ __forceinline__ int block_jacobi_b(int n, int scr_doubles) {
    if (n >= 41 && block_jacobi_fits_b(n, 8, scr_doubles)) return 8;
    return block_jacobi_fits_b(n, 4, scr_doubles) ? 4 : 0;
}

// M[:, pair k columns] <- M[:, pair k columns] R_k for every block pair k of
// the layer: one (row i, block pair k) segment per item, in place (the item
// owns those 2B entries of row i).
template <int B>
__device__ __forceinline__ void seg_right_multiply(const Team& t, int n, int nbp, double* M, int ldm,
                                                   const double* scr, const int* bp_lo, const int* bp_hi) {
    constexpr int B2 = 2 * B, SLD = B2 + 2, BB = B2 * SLD;  // sub-block stride B2 + 2: conflict-free columns
    const int nit = n * nbp;
    int k = 0, i = t.tid;
    while (i >= n) {
        i -= n;
        k++;
    }
    const int dk = t.nthreads / n, di = t.nthreads % n;
    for (int it = t.tid; it < nit; it += t.nthreads, i += di, k += dk) {
        if (i >= n) {
            i -= n;
            k++;
        }
        const int lo = bp_lo[k] * B, hi = bp_hi[k] * B - B;
        const double* R = scr + k * 2 * BB + BB;
        double x[B2];
#pragma unroll
        for (int cc = 0; cc < B2; ++cc) {
            const int g = (cc < B ? lo : hi) + cc;
            x[cc] = g < n ? M[g * ldm + i] : 0.0;
        }
#pragma unroll 1
        for (int cc = 0; cc < B2; cc += 2) {
            double y0 = 0.0, y1 = 0.0;
#pragma unroll
            for (int cp = 0; cp < B2; ++cp) {
                const double2 rr = *reinterpret_cast<const double2*>(R + cp * SLD + cc);
                y0 = fma(x[cp], rr.x, y0);
                y1 = fma(x[cp], rr.y, y1);
            }
            const int g0 = (cc < B ? lo : hi) + cc, g1 = g0 + 1;
            if (g0 < n) M[g0 * ldm + i] = y0;
            if (g1 < n) M[g1 * ldm + i] = y1;
        }
    }
}

// Pair j (0..B-1) of round rd of a block-pair solve over the 2B local indices:
// rounds rd < B pair lo-block index j with hi-block index B + (j + rd) mod B
// (every inter-block pair once); layer 0 adds B - 1 rounds that pair indices
// inside each block (round-robin over B, pairs j < B/2 in the lo block).
template <int B>
__device__ __forceinline__ void bp_pair(int rd, int j, int& p, int& q) {
    if (rd < B) {
        p = j;
        q = B + ((j + rd) & (B - 1));
    } else {
        int x, y;
        rr_pair(B, rd - B, j & (B / 2 - 1), x, y);
        const int o = j < B / 2 ? 0 : B;
        p = o + min(x, y);
        q = o + max(x, y);
    }
}

// Rotation of pair (p, q) by the reference's rule (src/lie_svd_small.rs:
// 235-249): tan(theta) = t with t the smaller root, the new diagonal
// app - t apq, aqq + t apq.  Written in half-angle form so that the chain has
// two reciprocal square roots and one reciprocal in place of a square root,
// a division and a reciprocal square root:
//   h = hypot(d, 2 apq), cos 2theta = |d| / h, sin 2theta = 2 apq / h,
//   w = 1 + cos 2theta, cos theta = sqrt(w / 2), sin theta = sin 2theta / sqrt(2 w),
//   |t| = sin 2theta / w.
// Branch-free; expects the block scaled so that |entries| <= 1 (then
// d^2 + 4 apq^2 cannot overflow; it is floored at the smallest normal).
__device__ __forceinline__ void jacobi_rotation(double app, double aqq, double apq, double& c, double& s,
                                                double& npp, double& nqq) {
    const double d = aqq - app, g = 2.0 * apq;
    // sign of t: that of theta = d / (2 apq), and + for theta = +-0 (the
    // reference's theta >= 0 branch)
    const double sg = d < 0.0 ? -1.0 : (d > 0.0 || g >= 0.0 ? 1.0 : -1.0);
    const double x = fmax(fma(d, d, g * g), 2.2250738585072014e-308);
    const double y = rsqrt(x);
    const double w = fma(fabs(d), y, 1.0);
    const double v = g * y;
    const double z = rsqrt(2.0 * w);
    const double rw = 1.0 / w;
    c = w * z;
    s = sg * (v * z);
    const double ta = sg * (v * rw) * apq;
    npp = app - ta;
    nqq = aqq + ta;
}

// Two-sided Jacobi on one 2B x 2B sub-block S (stride B2 + 2) by one warp,
// accumulating the rotations into R (R <- R J each round).  Lane j < B
// computes pair j's rotation and writes pair j's 2 x 2 diagonal block (exact
// new diagonal, zero off-diagonal); the rotations reach the other lanes by
// shuffles.  Each lane owns whole 2 x 2 off-diagonal pair-blocks (row pair r,
// column pair c) and applies both sides in registers:
// S[{p_r,q_r}][{p_c,q_c}] <- J_r^T X J_c.
// B = 8: pair-blocks (r, c0), (r, c0 + 4) and R rows {r, r + 8} x pairs {c0, c0 + 4};
// B = 4: pair-block (r, c0) on lanes < 16 and R row lane & 7 x pair lane >> 3.
// Returns the rotations this lane computed.
template <int B, class Pairs>
__device__ __forceinline__ int block_pair_round(int lane, int lo, int hi, int n, double thr, double* S, double* R,
                                                Pairs pairs) {
    constexpr int B2 = 2 * B, SLD = B2 + 2;
    constexpr int NSB = B == 8 ? 2 : 1;  // S pair-blocks per lane
    constexpr int NRI = B == 8 ? 4 : 1;  // R (row, pair) items per lane
    constexpr unsigned FULL = 0xffffffffu;
    const int r = lane & (B - 1);
    int sc[NSB], rx[NRI], rc[NRI];
    if constexpr (B == 8) {
        sc[0] = lane >> 3;
        sc[1] = (lane >> 3) + 4;
        rx[0] = r; rc[0] = 0;
        rx[1] = r; rc[1] = 1;
        rx[2] = r + 8; rc[2] = 0;
        rx[3] = r + 8; rc[3] = 1;
    } else {
        sc[0] = (lane >> 2) & 3;
        rx[0] = lane & 7;
        rc[0] = lane >> 3;
    }
    // ---- reads
    int p, q;
    pairs(r, p, q);  // lane j < B: its own pair j (r == lane there)
    const int pr = p, qr = q;
    double app = 0.0, aqq = 0.0, apq = 0.0;
    if (lane < B) {
        app = S[p * SLD + p];
        aqq = S[q * SLD + q];
        apq = S[p * SLD + q];
    }
    int pc[NSB], qc[NSB];
    double xs[NSB][4];
#pragma unroll
    for (int u = 0; u < NSB; ++u) {
        pairs(sc[u], pc[u], qc[u]);
        xs[u][0] = S[pr * SLD + pc[u]];
        xs[u][1] = S[pr * SLD + qc[u]];
        xs[u][2] = S[qr * SLD + pc[u]];
        xs[u][3] = S[qr * SLD + qc[u]];
    }
    int rpc[NRI], rqc[NRI];
    double xr[NRI][2];
#pragma unroll
    for (int v = 0; v < NRI; ++v) {
        if constexpr (B == 8) {
            rpc[v] = pc[rc[v]];
            rqc[v] = qc[rc[v]];
        } else {
            pairs(rc[v], rpc[v], rqc[v]);
        }
        xr[v][0] = R[rx[v] * SLD + rpc[v]];
        xr[v][1] = R[rx[v] * SLD + rqc[v]];
    }
    // ---- pair `lane`'s rotation
    double c = 1.0, s = 0.0, npp = app, nqq = aqq;
    int nrot = 0;
    bool rot = false;
    if (lane < B) {
        const int gp = (p < B ? lo : hi - B) + p, gq = (q < B ? lo : hi - B) + q;
        if (gp < n && gq < n && fabs(apq) >= thr && apq != 0.0) {  // :232
            jacobi_rotation(app, aqq, apq, c, s, npp, nqq);
            rot = true;
            nrot = 1;
        }
    }
    const double cr = __shfl_sync(FULL, c, r), sr = __shfl_sync(FULL, s, r);
    double cc[NSB], ss[NSB];
#pragma unroll
    for (int u = 0; u < NSB; ++u) {
        cc[u] = __shfl_sync(FULL, c, sc[u]);
        ss[u] = __shfl_sync(FULL, s, sc[u]);
    }
    double rcc[NRI], rss[NRI];
#pragma unroll
    for (int v = 0; v < NRI; ++v) {
        if constexpr (B == 8) {
            rcc[v] = cc[rc[v]];
            rss[v] = ss[rc[v]];
        } else {
            rcc[v] = __shfl_sync(FULL, c, rc[v]);
            rss[v] = __shfl_sync(FULL, s, rc[v]);
        }
    }
    __syncwarp();  // every lane has read this round's S and R
    // ---- writes
    if (B == 8 || lane < 16) {
#pragma unroll
        for (int u = 0; u < NSB; ++u) {
            if (sc[u] != r) {
                // rows (p_r, q_r), then columns (p_c, q_c)
                const double y00 = cr * xs[u][0] - sr * xs[u][2], y10 = sr * xs[u][0] + cr * xs[u][2];
                const double y01 = cr * xs[u][1] - sr * xs[u][3], y11 = sr * xs[u][1] + cr * xs[u][3];
                S[pr * SLD + pc[u]] = cc[u] * y00 - ss[u] * y01;
                S[pr * SLD + qc[u]] = ss[u] * y00 + cc[u] * y01;
                S[qr * SLD + pc[u]] = cc[u] * y10 - ss[u] * y11;
                S[qr * SLD + qc[u]] = ss[u] * y10 + cc[u] * y11;
            }
        }
    }
    if (rot) {
        S[p * SLD + p] = npp;
        S[p * SLD + q] = 0.0;
        S[q * SLD + p] = 0.0;
        S[q * SLD + q] = nqq;
    }
#pragma unroll
    for (int v = 0; v < NRI; ++v) {
        R[rx[v] * SLD + rpc[v]] = rcc[v] * xr[v][0] - rss[v] * xr[v][1];
        R[rx[v] * SLD + rqc[v]] = rss[v] * xr[v][0] + rcc[v] * xr[v][1];
    }
    __syncwarp();
    return nrot;
}

// The B inter-block rounds of a block-pair solve (pair j of round rd is
// (j, B + (j + rd) mod B)), software-pipelined across rounds.  Every lane
// computes the rotation of its row pair r = lane mod B itself (lanes with the
// same r agree bit for bit), so the rotation of round rd + 1 starts as soon as
// round rd's values are in registers: its a_pp is pair r's new diagonal, its
// a_qq pair r + 1's, and its a_pq the (p_r, q_{r+1}) entry of pair-block
// (r, r + 1) after round rd, taken from the lane that owns that block.  The
// shared-memory stores and loads of the pair-blocks overlap that chain (the
// rounds are unrolled and branch-free).  Lane roles as in block_pair_round.
// Returns the rotations of lanes < B.
template <int B>
__device__ __forceinline__ int inter_rounds(int lane, int lo, int hi, int n, double thr, double* S, double* R) {
    constexpr int B2 = 2 * B, SLD = B2 + 2;
    constexpr int NSB = B == 8 ? 2 : 1;
    constexpr int NRI = B == 8 ? 4 : 1;
    constexpr unsigned FULL = 0xffffffffu;
    const int r = lane & (B - 1), r1 = (r + 1) & (B - 1);
    int sc[NSB], rx[NRI], rc[NRI];
    int owner;  // lane owning pair-block (r, r + 1); it sits in slot r1 >> 2 there (B = 8)
    if constexpr (B == 8) {
        sc[0] = lane >> 3;
        sc[1] = (lane >> 3) + 4;
        rx[0] = r; rc[0] = 0;
        rx[1] = r; rc[1] = 1;
        rx[2] = r + 8; rc[2] = 0;
        rx[3] = r + 8; rc[3] = 1;
        owner = r + 8 * (r1 & 3);
    } else {
        sc[0] = (lane >> 2) & 3;
        rx[0] = lane & 7;
        rc[0] = lane >> 3;
        owner = r + 4 * r1;
    }
    const bool s_writer = B == 8 || lane < 16;
    bool own_diag = sc[0] == r;
    if constexpr (NSB == 2) own_diag = own_diag || sc[1] == r;
    const bool p_ok = lo + r < n;
    // round 0 from shared memory
    double app = S[r * SLD + r], aqq = S[(B + r) * SLD + B + r], apq = S[r * SLD + B + r];
    double c, s, npp, nqq;
    bool rot = p_ok && hi + r < n && fabs(apq) >= thr && apq != 0.0;  // :232
    jacobi_rotation(app, aqq, apq, c, s, npp, nqq);
    c = rot ? c : 1.0;
    s = rot ? s : 0.0;
    npp = rot ? npp : app;
    nqq = rot ? nqq : aqq;
    int nrot = 0;
#pragma unroll
    for (int rd = 0; rd < B; ++rd) {
        const int qr = B + ((r + rd) & (B - 1));
        int qc[NSB];
        double xs[NSB][4];
#pragma unroll
        for (int u = 0; u < NSB; ++u) {
            qc[u] = B + ((sc[u] + rd) & (B - 1));
            xs[u][0] = S[r * SLD + sc[u]];
            xs[u][1] = S[r * SLD + qc[u]];
            xs[u][2] = S[qr * SLD + sc[u]];
            xs[u][3] = S[qr * SLD + qc[u]];
        }
        int rpc[NRI], rqc[NRI];
        double xr[NRI][2];
#pragma unroll
        for (int v = 0; v < NRI; ++v) {
            if constexpr (B == 8) {
                rpc[v] = sc[rc[v]];
                rqc[v] = qc[rc[v]];
            } else {
                rpc[v] = rc[v];
                rqc[v] = B + ((rc[v] + rd) & (B - 1));
            }
            xr[v][0] = R[rx[v] * SLD + rpc[v]];
            xr[v][1] = R[rx[v] * SLD + rqc[v]];
        }
        nrot += (rot && lane < B) ? 1 : 0;
        double cc[NSB], ss[NSB];
#pragma unroll
        for (int u = 0; u < NSB; ++u) {
            cc[u] = __shfl_sync(FULL, c, sc[u]);
            ss[u] = __shfl_sync(FULL, s, sc[u]);
        }
        double z[NSB][4];
#pragma unroll
        for (int u = 0; u < NSB; ++u) {
            // rows (p_r, q_r), then columns (p_c, q_c); the diagonal pair-block
            // is overwritten below with the exact values
            const double y00 = c * xs[u][0] - s * xs[u][2], y10 = s * xs[u][0] + c * xs[u][2];
            const double y01 = c * xs[u][1] - s * xs[u][3], y11 = s * xs[u][1] + c * xs[u][3];
            z[u][0] = cc[u] * y00 - ss[u] * y01;
            z[u][1] = ss[u] * y00 + cc[u] * y01;
            z[u][2] = cc[u] * y10 - ss[u] * y11;
            z[u][3] = ss[u] * y10 + cc[u] * y11;
        }
        double zr[NRI][2];
#pragma unroll
        for (int v = 0; v < NRI; ++v) {
            double rcv, rsv;
            if constexpr (B == 8) {
                rcv = cc[rc[v]];
                rsv = ss[rc[v]];
            } else {
                rcv = __shfl_sync(FULL, c, rc[v]);
                rsv = __shfl_sync(FULL, s, rc[v]);
            }
            zr[v][0] = rcv * xr[v][0] - rsv * xr[v][1];
            zr[v][1] = rsv * xr[v][0] + rcv * xr[v][1];
        }
        // this round's exact diagonal (the next round's rotation replaces rot, npp, nqq)
        const bool rot_d = rot;
        const double npp_d = npp, nqq_d = nqq;
        if (rd + 1 < B) {
            // next round's rotation of pair r, from registers
            double pz = z[0][1];
            if constexpr (B == 8) pz = (r1 >> 2) ? z[1][1] : z[0][1];
            const double apq_n = __shfl_sync(FULL, pz, owner);
            const double aqq_n = __shfl_sync(FULL, nqq, r1);
            const double app_n = npp;
            rot = p_ok && hi + ((r + rd + 1) & (B - 1)) < n && fabs(apq_n) >= thr && apq_n != 0.0;
            jacobi_rotation(app_n, aqq_n, apq_n, c, s, npp, nqq);
            c = rot ? c : 1.0;
            s = rot ? s : 0.0;
            npp = rot ? npp : app_n;
            nqq = rot ? nqq : aqq_n;
        }
        __syncwarp();  // every lane has read this round's S and R
        if (s_writer) {
#pragma unroll
            for (int u = 0; u < NSB; ++u) {
                S[r * SLD + sc[u]] = z[u][0];
                S[r * SLD + qc[u]] = z[u][1];
                S[qr * SLD + sc[u]] = z[u][2];
                S[qr * SLD + qc[u]] = z[u][3];
            }
            // the owner of the diagonal pair-block (r, r) of a rotated pair stores the
            // exact new diagonal and a zero off-diagonal (:244-249) over its values
            // (without a rotation c = 1, s = 0 left the block unchanged)
            if (own_diag && rot_d) {
                S[r * SLD + r] = npp_d;
                S[r * SLD + qr] = 0.0;
                S[qr * SLD + r] = 0.0;
                S[qr * SLD + qr] = nqq_d;
            }
        }
#pragma unroll
        for (int v = 0; v < NRI; ++v) {
            R[rx[v] * SLD + rpc[v]] = zr[v][0];
            R[rx[v] * SLD + rqc[v]] = zr[v][1];
        }
        __syncwarp();
    }
    return nrot;
}

// One block-pair solve: B rounds over the inter-block pairs (j, B + (j + rd)
// mod B), then on layer 0 the B - 1 round-robin rounds inside each block.
template <int B>
__device__ __forceinline__ int solve_block_pair(int lane, int layer, int lo, int hi, int n, double thr, double* S,
                                                double* R) {
    int nrot = inter_rounds<B>(lane, lo, hi, n, thr, S, R);
    if (layer == 0) {
#pragma unroll 1
        for (int rd = B; rd < 2 * B - 1; ++rd)
            nrot += block_pair_round<B>(lane, lo, hi, n, thr, S, R,
                                        [rd](int j, int& p, int& q) { bp_pair<B>(rd, j, p, q); });
    }
    return nrot;
}

template <int B>
__device__ inline int jacobi_block_sweeps_t(const Team& t, int n, double* P, int pld, double* scr,
                                            double* V, int ldv, double ref_norm, double thr, int max_sweeps,
                                            TeamScratch* sc, long long* rotations, bool* capped) {
    constexpr int B2 = 2 * B, SLD = B2 + 2, BB = B2 * SLD;  // sub-block stride B2 + 2: conflict-free columns
    const int nbl = (n + B - 1) / B, nbe = nbl + (nbl & 1), nbp = nbe / 2, layers = nbe - 1;
    const int lane = t.lane;
    // block-pair table of the current layer: bp_lo[k], bp_hi[k] (block indices)
    int* bp_lo = reinterpret_cast<int*>(scr + nbp * 2 * BB);
    int* bp_hi = bp_lo + 32;
    int sweeps = 0;
    *capped = false;
    for (int sw = 0; sw < max_sweeps; ++sw) {
        sweeps = sw + 1;
        double off = 0.0;
        for (int y = t.warp; y < n; y += t.nwarps)
            for (int x = lane; x < n; x += 32)
                if (x != y) off = fma(P[y * pld + x], P[y * pld + x], off);
        off = 0.5 * team_sum(t, off, sc->red);
        if (sqrt(off) < 1e-13 * ref_norm) break;  // JACOBI_TOL, :69
        if (sw + 1 == max_sweeps) *capped = true;
        int nrot = 0;
        for (int l = 0; l < layers; ++l) {
            if (t.warp == 0 && lane < nbp) {
                int A, Bk;
                rr_pair(nbe, l, lane, A, Bk);
                bp_lo[lane] = min(A, Bk);
                bp_hi[lane] = max(A, Bk);
            }
            t.sync();
            // ---- solve: one warp per block pair, warp-synchronous
            for (int k = t.warp; k < nbp; k += t.nwarps) {
                const int lo = bp_lo[k] * B, hi = bp_hi[k] * B;  // first global index of each block
                double* S = scr + k * 2 * BB;
                double* R = S + BB;
#pragma unroll
                for (int u = 0; u < B2 * B2 / 32; ++u) {
                    const int e = lane + 32 * u;
                    const int r = e / B2, c = e % B2;
                    const int gr = (r < B ? lo : hi - B) + r, gc = (c < B ? lo : hi - B) + c;
                    S[r * SLD + c] = (gr < n && gc < n) ? P[gc * pld + gr] : 0.0;
                    R[r * SLD + c] = (r == c) ? 1.0 : 0.0;
                }
                __syncwarp();
                nrot += solve_block_pair<B>(lane, l, lo, hi, n, thr, S, R);
            }
            t.sync();
            // ---- apply, pass 1: W = P R and V <- V R, one (row, block pair) segment per item
            const int nit = n * nbp;
            seg_right_multiply<B>(t, n, nbp, P, pld, scr, bp_lo, bp_hi);
            seg_right_multiply<B>(t, n, nbp, V, ldv, scr, bp_lo, bp_hi);
            t.sync();
            // ---- apply, pass 2: P' = R^T W, one (column, block pair) segment per item
            {
                int k = 0, j = t.tid;
                while (j >= n) {
                    j -= n;
                    k++;
                }
                const int dk = t.nthreads / n, dj = t.nthreads % n;
                for (int it = t.tid; it < nit; it += t.nthreads, j += dj, k += dk) {
                    if (j >= n) {
                        j -= n;
                        k++;
                    }
                    const int blo = bp_lo[k], bhi = bp_hi[k];
                    const int lo = blo * B, hi = bhi * B - B;
                    const double* S = scr + k * 2 * BB;
                    const double* R = S + BB;
                    const int jb = j / B;
                    const int jloc = jb == blo ? j - lo : (jb == bhi ? j - hi : -1);
                    double x[B2];
#pragma unroll
                    for (int r = 0; r < B2; ++r) {
                        const int g = (r < B ? lo : hi) + r;
                        x[r] = g < n ? P[j * pld + g] : 0.0;
                    }
#pragma unroll 1
                    for (int r = 0; r < B2; r += 2) {
                        double y0 = 0.0, y1 = 0.0;
#pragma unroll
                        for (int rp = 0; rp < B2; ++rp) {
                            const double2 rr = *reinterpret_cast<const double2*>(R + rp * SLD + r);
                            y0 = fma(rr.x, x[rp], y0);
                            y1 = fma(rr.y, x[rp], y1);
                        }
                        if (jloc >= 0) {  // diagonal tile: the solved sub-block
                            y0 = S[r * SLD + jloc];
                            y1 = S[(r + 1) * SLD + jloc];
                        }
                        const int g0 = (r < B ? lo : hi) + r, g1 = g0 + 1;
                        if (g0 < n) P[j * pld + g0] = y0;
                        if (g1 < n) P[j * pld + g1] = y1;
                    }
                }
            }
            t.sync();
        }
        *rotations += (long long)team_sum(t, double(nrot), sc->red);
    }
    return sweeps;
}

__device__ inline int jacobi_block_sweeps(const Team& t, int n, int bsize, double* P, int pld, double* scr,
                                          double* V, int ldv, double ref_norm, double thr, int max_sweeps,
                                          TeamScratch* sc, long long* rotations, bool* capped) {
    if (bsize == 8)
        return jacobi_block_sweeps_t<8>(t, n, P, pld, scr, V, ldv, ref_norm, thr, max_sweeps, sc, rotations, capped);
    return jacobi_block_sweeps_t<4>(t, n, P, pld, scr, V, ldv, ref_norm, thr, max_sweeps, sc, rotations, capped);
}

// LieSvdSmall::solve (src/lie_svd_small.rs:296-323) by one team, n <= 64.
//   1. newton_schulz_polar (:158-183)  X <- 0.5 X (3I - X^T X), FP64 GEMMs in smem
//   2. P = sym(Q^T A)                  (:305-309)
//   3. eigensolve of P                 two-sided Jacobi (eigh_jacobi_full, :212-285) in a
//      parallel order: blocked for n > 32 without a rotor stream, else
//      layer by layer over round-robin pairs
//   4. U = Q V, orthogonality check, repair_left_basis_from_right (:185-208, :317-320)
template <int TS, int G>
__device__ void small_solve_team(const Team& t, const SmallJob& job, double* sm) {
    const int n = job.n;
    const bool mma = team_uses_mma(n, t.nwarps);
    const int np = team_np(n, mma);
    const int ld = team_ld(n, mma);
    // products on the FP64 tensor path or the scalar register tiles
    auto gemm = [&](auto la, auto lb, auto epi) {
        if (mma)
            team_mma(t, np, n, la, lb, epi);
        else
            team_gemm<TS>(t, np, n, la, lb, epi);
    };
    double* X = sm;
    double* T = X + ld * np;
    double* Xn = T + ld * np;
    TeamScratch* sc = reinterpret_cast<TeamScratch*>(Xn + ld * np);
    const double refn = sqrt(double(n));
    int flags = job.extra_flags;

    // ---- load A, Frobenius norm, finiteness
    double fro2 = 0.0;
    int bad = 0;
    load_colmajor(t, job, np, ld, X, fro2, bad);
    fro2 = team_sum(t, fro2, sc->red);
    const double nbad = team_sum(t, double(bad), sc->red);  // also syncs X
    const double afro = sqrt(fro2);
    if (nbad > 0.0) {
        const double qnan = __longlong_as_double(0x7ff8000000000000ULL);
        for (int idx = t.tid; idx < n * n; idx += t.nthreads) {
            const int i = idx / n, j = idx % n;
            job.U[i * job.ldu + j] = qnan;
            job.Vt[i * job.ldvt + j] = qnan;
        }
        for (int i = t.tid; i < n; i += t.nthreads) {
            job.S[i] = qnan;
            if (job.perm_out) job.perm_out[i] = i;
        }
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
            if (job.rotor_count) *job.rotor_count = 0;
        }
        t.sync();
        return;
    }

    // ---- 1. Newton-Schulz polar
    const double scale = fmax(afro, 1e-300);
    for (int idx = t.tid; idx < n * n; idx += t.nthreads) {
        const int i = idx % n, j = idx / n;
        X[j * ld + i] = X[j * ld + i] / scale;
    }
    t.sync();
    bool conv = false, diverged = false;
    int iters = 0;
    for (;;) {
        gemm(
            [&](int k, int i) { return X[i * ld + k]; },
            [&](int k, int j) { return X[j * ld + k]; },
            [&](int i, int j, double v) { T[j * ld + i] = v; });
        t.sync();
        if (conv || iters == 120) break;  // POLAR_MAX_ITERS, :67
        iters++;
        double d2 = 0.0;
        gemm(
            [&](int k, int i) { return X[k * ld + i]; },
            [&](int k, int j) { return T[j * ld + k]; },
            [&](int i, int j, double v) {
                const double x = X[j * ld + i];
                const double xn = 0.5 * (3.0 * x - v);
                Xn[j * ld + i] = xn;
                d2 += (xn - x) * (xn - x);
            });
        d2 = team_sum(t, d2, sc->red);
        const double delta = sqrt(d2);
        if (!isfinite(d2) || delta > 1e6 * refn) {
            diverged = true;
            break;
        }
        double* tmp = X;
        X = Xn;
        Xn = tmp;
        if (delta < 1e-13 * refn) conv = true;  // POLAR_TOL, :68
    }
    bool polar_ok;
    if (!diverged) {
        double o2 = 0.0;
        for (int idx = t.tid; idx < n * n; idx += t.nthreads) {
            const int i = idx % n, j = idx / n;
            const double d = T[j * ld + i] - (i == j ? 1.0 : 0.0);
            o2 += d * d;
        }
        o2 = team_sum(t, o2, sc->red);
        polar_ok = sqrt(o2) <= 1e-8 * refn;
        if (!conv) flags |= LSVD_MAT_NS_CAP;
    } else {
        // (gram_schmidt_orthonormal(a), false), :169-171
        polar_ok = false;
        flags |= LSVD_MAT_NS_DIVERGED;
        double f = 0.0;
        int b2 = 0;
        load_colmajor(t, job, np, ld, X, f, b2);
        t.sync();
        warp_mgs(t, X, n, ld);
        t.sync();
    }
    if (!polar_ok) flags |= LSVD_MAT_POLAR_UNTRUSTED;
    double* Q = X;
    double* Wb = T;
    double* Vb = Xn;

    // ---- 2. P = sym(Q^T A)
    {
        double f = 0.0;
        int b2 = 0;
        load_colmajor(t, job, np, ld, Vb, f, b2);
    }
    t.sync();
    gemm(
        [&](int k, int i) { return Q[i * ld + k]; },
        [&](int k, int j) { return Vb[j * ld + k]; },
        [&](int i, int j, double v) { Wb[j * ld + i] = v; });
    t.sync();
    // P = (P + P^T) / 2 (:309) written straight into layer-0 pair positions
    // of the ping-pong buffer Vb (leading dimension m); Q is parked in the U
    // output (global) so that Q's buffer can be the second ping-pong buffer.
    const int m = (n % 2 == 0) ? n : n + 1;
    // Without a rotor stream to record, n >= LSVD_BLOCK_JACOBI_MIN_N takes the
    // blocked sweep (P in natural order, odd leading dimension m + 1);
    // otherwise the layer-by-layer sweep with P in pair-position order
    // (leading dimension m).
    const int bsize = (job.rotors == nullptr && n >= LSVD_BLOCK_JACOBI_MIN_N) ? block_jacobi_b(n, ld * np) : 0;
    const bool blocked = bsize != 0;
    const int pstride = blocked ? m + 1 : m;
    for (int x = t.tid; x < m; x += t.nthreads) {
        // layer 0: pair k = (m-1, 0) for k = 0, else (k, m-1-k) in ring m-1
        const int k = x >> 1;
        int a = k == 0 ? m - 1 : k, bb = k == 0 ? 0 : (m - 1 - k) % (m - 1);
        const int lo = min(a, bb), hi = max(a, bb);
        sc->pidx[0][x] = blocked ? x : ((x & 1) ? hi : lo);
    }
    for (int idx = t.tid; idx < n * n; idx += t.nthreads) {
        const int i = idx / n, j = idx % n;
        job.U[i * job.ldu + j] = Q[j * ld + i];
    }
    t.sync();
    double pf2 = 0.0;
    for (int idx = t.tid; idx < m * m; idx += t.nthreads) {
        const int x = idx % m, y = idx / m;
        const int i = sc->pidx[0][x], j = sc->pidx[0][y];
        double v = 0.0;
        if (i < n && j < n) v = (Wb[j * ld + i] + Wb[i * ld + j]) * 0.5;
        Vb[y * pstride + x] = v;
        pf2 = fma(v, v, pf2);
    }
    const double pref = fmax(sqrt(team_sum(t, pf2, sc->red)), 1e-300);  // syncs Vb
    // The blocked sweep works on P scaled by a power of two to ||P||_F in
    // [0.5, 1) (exact; the eigenvalues are scaled back), which keeps its
    // rotation formula in range.
    int pe = 0;
    if (blocked) {
        frexp(pref, &pe);
        pe = max(min(pe, 1000), -1000);
        const double pscale = ldexp(1.0, -pe);
        for (int idx = t.tid; idx < m * m; idx += t.nthreads) {
            const int x = idx % m, y = idx / m;
            Vb[y * pstride + x] *= pscale;
        }
    }
    // V = I in the (now free) W buffer; P ping-pongs between Vb and Q's buffer
    double* Vn = Wb;
    for (int idx = t.tid; idx < np * np; idx += t.nthreads) {
        const int i = idx % np, j = idx / np;
        Vn[j * ld + i] = (i == j && i < n) ? 1.0 : 0.0;
    }
    if (t.tid == 0) sc->rotor_idx = 0;
    t.sync();

    // ---- 3. two-sided round-robin Jacobi eigensolve of P (eigh_jacobi_full)
    long long rotations = 0;
    bool jcap = false;
    double* Pfin = nullptr;
    int par = 0;
    int sweeps;
    if (blocked) {
        const double pscale = ldexp(1.0, -pe);
        sweeps = jacobi_block_sweeps(t, n, bsize, Vb, pstride, Q, Vn, ld, pref * pscale, 1e-300 * pscale,
                                     60 + 20 * n /* :216 */, sc, &rotations, &jcap);
        Pfin = Vb;
        par = 0;
    } else {
        sweeps = jacobi2pp_sweeps(t, n, Vb, Q, Vn, ld, pref, 60 + 20 * n /* :216 */, sc, job, &rotations,
                                  &jcap, &Pfin, &par);
    }
    if (jcap) flags |= LSVD_MAT_JACOBI_CAP;
    double* const Pother = (Pfin == Vb) ? Q : Vb;
    Vb = Vn;

    // ---- eigenvalues on the diagonal, stable descending sort, sigma = max(eig, 0)
    for (int x = t.tid; x < m; x += t.nthreads) {
        const int i = sc->pidx[par][x];
        if (i < n) sc->sig[i] = ldexp(Pfin[x * pstride + x], pe);
    }
    t.sync();
    for (int j = t.tid; j < n; j += t.nthreads) {
        const double sj = sc->sig[j];
        const double kj = isnan(sj) ? -INFINITY : sj;
        int rank = 0;
        for (int k = 0; k < n; ++k) {
            const double sk = sc->sig[k];
            const double kk = isnan(sk) ? -INFINITY : sk;
            rank += (kk > kj) || (kk == kj && k < j);
        }
        sc->perm[rank] = j;
    }
    t.sync();
    for (int j = t.tid; j < n; j += t.nthreads) sc->sig[j] = fmax(sc->sig[j], 0.0);
    // both ping-pong buffers are free again: Q comes back from the U output
    double* Ub = Pfin;
    Q = (Pfin == Q) ? Pother : Q;
    t.sync();
    for (int idx = t.tid; idx < np * np; idx += t.nthreads) {
        const int i = idx / np, j = idx - (idx / np) * np;
        Q[j * ld + i] = (i < n && j < n) ? job.U[i * job.ldu + j] : 0.0;
    }
    t.sync();
    const int* perm = sc->perm;
    // ---- 4. U = Q V (sorted); orthogonality check (:317-318)
    gemm(
        [&](int k, int i) { return Q[k * ld + i]; },
        [&](int k, int j) { return j < n ? Vb[perm[j] * ld + k] : 0.0; },
        [&](int i, int j, double v) { Ub[j * ld + i] = v; });
    t.sync();
    auto orth_of = [&](const double* B) -> double {
        double o2 = 0.0;
        gemm(
            [&](int k, int i) { return B[i * ld + k]; },
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
    bool a_in_x = false;
    if (!polar_ok || orth_u > 1e-8 * refn) {
        // repair_left_basis_from_right, :185-208 (Q is dead: reuse its buffer for A)
        flags |= LSVD_MAT_REPAIRED;
        double f = 0.0;
        int b2 = 0;
        load_colmajor(t, job, np, ld, Q, f, b2);
        a_in_x = true;
        double smax = 0.0;
        for (int k = 0; k < n; ++k) smax = fmax(smax, sc->sig[k]);
        const double stol = 1e-12 * fmax(smax, 1.0);
        t.sync();
        gemm(
            [&](int k, int i) { return Q[k * ld + i]; },
            [&](int k, int j) { return j < n ? Vb[perm[j] * ld + k] : 0.0; },
            [&](int i, int j, double v) {
                const double sj = j < n ? sc->sig[perm[j]] : 0.0;
                Ub[j * ld + i] = (j < n && sj > stol) ? v / sj : 0.0;
            });
        t.sync();
        warp_mgs(t, Ub, n, ld);
        t.sync();
        if (job.want_diag) orth_u = orth_of(Ub);
    }

    // ---- outputs (row-major)
    for (int idx = t.tid; idx < n * n; idx += t.nthreads) {
        const int i = idx / n, j = idx % n;
        job.U[i * job.ldu + j] = Ub[j * ld + i];
        job.Vt[i * job.ldvt + j] = Vb[perm[i] * ld + j];
    }
    for (int i = t.tid; i < n; i += t.nthreads) {
        job.S[i] = sc->sig[perm[i]];
        if (job.perm_out) job.perm_out[i] = perm[i];
    }

    double rel_recon = __longlong_as_double(0x7ff8000000000000ULL), orth_v = rel_recon;
    if (job.want_diag) {
        orth_v = orth_of(Vb);
        if (!a_in_x) {
            double f = 0.0;
            int b2 = 0;
            load_colmajor(t, job, np, ld, Q, f, b2);
            t.sync();
        }
        // metrics::compute rel_recon (src/lib.rs:157-159): ||U S V^T - A||_F / ||A||_F
        double r2 = 0.0;
        gemm(
            [&](int k, int i) { return Ub[k * ld + i]; },
            [&](int k, int j) { return (j < n && k < n) ? sc->sig[perm[k]] * Vb[perm[k] * ld + j] : 0.0; },
            [&](int i, int j, double v) {
                if (i < n && j < n) {
                    const double d = v - Q[j * ld + i];
                    r2 += d * d;
                }
            });
        rel_recon = sqrt(team_sum(t, r2, sc->red)) / fmax(afro, 1e-300);
    }
    if (t.tid == 0) {
        int nrot = sc->rotor_idx;
        if (job.rotors && nrot > job.rotor_cap) flags |= LSVD_MAT_ROTOR_OVERFLOW;
        if (job.rotor_count) *job.rotor_count = nrot;
        if (job.agg && flags) atomicOr(job.agg, flags);
        if (job.diag) {
            lsvd_diag d;
            d.rel_recon = rel_recon;
            d.orth_u = job.want_diag ? orth_u : __longlong_as_double(0x7ff8000000000000ULL);
            d.orth_v = orth_v;
            d.ns_iters = iters;
            d.jacobi_sweeps = sweeps;
            d.rotations = rotations;
            d.flags = flags;
            d.route = LSVD_ROUTE_SMALL;
            *job.diag = d;
        }
    }
    t.sync();
}

}  // namespace lsvd
