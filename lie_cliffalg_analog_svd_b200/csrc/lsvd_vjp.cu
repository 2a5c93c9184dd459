// lsvd_vjp.cu -- batched thin SVD that keeps the rotor stream instead of U/V,
// and the SVD / polar-factor adjoint computed from that stream.
//
// Forward (lsvd_svd_batched_stream_f64): count matrices of one shape m x n
// (m >= n, n <= 64).  Tall inputs are reduced by qr_reduce (modified
// Gram-Schmidt, src/lie_svd_small.rs:373-418); R (or A itself when square)
// goes through LieSvdSmall::solve (src/lie_svd_small.rs:296-336: Newton-Schulz
// polar, Jacobi eigensolve of P = sym(Q^T A), U = Q V) on one CTA per matrix,
// which records the accepted rotations (i, j, round, theta) of the eigensolve
// and the descending sort permutation: V = G_1 G_2 ... G_k P, where G_r
// rotates columns i, j by theta (v_i <- c v_i - s v_j, v_j <- s v_i + c v_j)
// and P[:, j] = e_perm[j].  U and Vt are optional outputs.
//
// Adjoint (lsvd_svd_vjp_f64): from A, sigma, perm and the stream alone, one
// CTA per matrix
//   * rebuilds V by replaying the stream in reverse, V = G_1 (G_2 (... (G_k P))),
//     one column per thread (rotations act on rows, so columns are independent);
//   * applies the analytic thin-SVD adjoint, with U = A V S^-1 recomputed
//     (not stored):
//       Abar = U [F o (G - G^T) S + diag(Sbar) + S F o (H - H^T)] V^T
//              + (I - U U^T) Ubar S^-1 V^T,
//     G = U^T Ubar, H = V^T Vbar, F_ij = 1/(s_j^2 - s_i^2) (i != j), plus the
//     polar-factor (Q = U V^T) adjoint
//       U [(M - M^T) / (s_i + s_j)] V^T + (I - U U^T) Qbar V S^-1 V^T,
//     M = U^T Qbar V.  Both together are Abar = A E + Ubar S^-1 V^T
//     + Qbar V S^-1 V^T with E = V S^-1 D V^T and
//     D = F o (G - G^T) S + S F o (H - H^T) + (M - M^T)/(s_i + s_j)
//         + diag(Sbar) - (G + M) S^-1.
//   F_ij is set to 0 where |s_i - s_j| <= gap_tol * s_max (a near-degenerate
//   pair, whose in-plane rotation the loss must not depend on).
// Given a stored V^T instead, the same kernel skips the replay: the
// comparison path that keeps the V intermediate.
// No counterpart in the reference (it has no derivatives).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "lsvd.h"
#include "lsvd_internal.h"
#define LSVD_KERNELS_DEVICE_ONLY
#include "lsvd_kernels.cuh"

namespace {

using lsvd::kCtaThreads;
using lsvd::kMaxN;
using lsvd::Team;

constexpr int kVjpThreads = 256;
constexpr int kReplayChunk = 512;  // rotations staged in shared memory per replay chunk
constexpr int kReplayThreads = 64;  // one column of V per thread (n <= 64)
constexpr int kMaxRows = 4096;

__device__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < int(blockDim.x) / 32; ++w) s += red[w];
    __syncthreads();
    return s;
}

// qr_reduce of matrix blockIdx.x (m x n, row-major, packed): Q (m x n) and
// R (n x n, upper triangular) row-major.  Column j is staged in shared
// memory; a column whose residual norm is below 1e-10 ||X||_F gets a zero Q
// column (src/lie_svd_small.rs:399-410).
__global__ void __launch_bounds__(kCtaThreads) qr_batched_kernel(int m, int n, const double* A,
                                                                 double* Qo, double* Ro) {
    extern __shared__ double v[];
    __shared__ double red[kCtaThreads / 32];
    const size_t mi = blockIdx.x;
    const double* X = A + mi * size_t(m) * n;
    double* Q = Qo + mi * size_t(m) * n;
    double* R = Ro + mi * size_t(n) * n;
    double f2 = 0.0;
    for (int idx = threadIdx.x; idx < m * n; idx += kCtaThreads) f2 += X[idx] * X[idx];
    const double floor_ = 1e-10 * fmax(sqrt(block_sum(f2, red)), 1e-300);
    for (int j = 0; j < n; ++j) {
        for (int i = threadIdx.x; i < m; i += kCtaThreads) v[i] = X[size_t(i) * n + j];
        for (int r = threadIdx.x; r < n; r += kCtaThreads)
            if (r > j) R[r * n + j] = 0.0;
        __syncthreads();
        for (int k = 0; k < j; ++k) {
            double p = 0.0;
            for (int i = threadIdx.x; i < m; i += kCtaThreads) p = fma(Q[size_t(i) * n + k], v[i], p);
            const double dot = block_sum(p, red);
            if (threadIdx.x == 0) R[k * n + j] = dot;
            for (int i = threadIdx.x; i < m; i += kCtaThreads) v[i] -= dot * Q[size_t(i) * n + k];
            __syncthreads();
        }
        double p = 0.0;
        for (int i = threadIdx.x; i < m; i += kCtaThreads) p = fma(v[i], v[i], p);
        const double nrm = sqrt(block_sum(p, red));
        if (threadIdx.x == 0) R[j * n + j] = nrm;
        for (int i = threadIdx.x; i < m; i += kCtaThreads)
            Q[size_t(i) * n + j] = nrm >= floor_ ? v[i] / nrm : 0.0;
        __syncthreads();
    }
}

struct StreamArgs {
    int n;
    const double* A;  // n x n per matrix (R or the square input)
    double* U;        // n x n per matrix
    double* S;
    double* Vt;       // n x n per matrix
    lsvd_diag* diag;  // may be null
    lsvd_rotor* rotors;
    int64_t cap;
    int64_t* counts;
    int32_t* perm;
    int want_diag;
    int* agg;
};

// LieSvdSmall::solve of matrix blockIdx.x on one CTA (one team of eight
// warps), recording its rotor stream and sort permutation.
template <int TS, int G>
__global__ void __launch_bounds__(kCtaThreads, 2) stream_solve_kernel(StreamArgs a) {
    extern __shared__ __align__(16) double smem[];
    const size_t mi = blockIdx.x;
    const size_t nn = size_t(a.n) * a.n;
    lsvd::SmallJob job;
    job.n = a.n;
    job.A = a.A + mi * nn;
    job.lda = a.n;
    job.U = a.U + mi * nn;
    job.ldu = a.n;
    job.S = a.S + mi * a.n;
    job.Vt = a.Vt + mi * nn;
    job.ldvt = a.n;
    job.diag = a.diag ? a.diag + mi : nullptr;
    job.rotors = a.rotors + mi * size_t(a.cap);
    job.rotor_cap = a.cap;
    job.rotor_count = a.counts + mi;
    job.perm_out = a.perm + mi * a.n;
    job.want_diag = a.want_diag != 0;
    job.extra_flags = 0;
    job.agg = a.agg;
    Team tm;
    tm.tid = threadIdx.x;
    tm.nthreads = kCtaThreads;
    tm.warp = threadIdx.x / 32;
    tm.lane = threadIdx.x % 32;
    tm.nwarps = kCtaThreads / 32;
    tm.bar = 1;
    lsvd::small_solve_team<TS, G>(tm, job, smem);
}

// U (m x n) = Q (m x n) U_r (n x n) for matrix blockIdx.x.
__global__ void qu_kernel(int m, int n, const double* Q, const double* Ur, double* U) {
    const size_t mi = blockIdx.x;
    const double* q = Q + mi * size_t(m) * n;
    const double* ur = Ur + mi * size_t(n) * n;
    double* u = U + mi * size_t(m) * n;
    for (int idx = threadIdx.x; idx < m * n; idx += blockDim.x) {
        const int i = idx / n, j = idx % n;
        double s = 0.0;
        for (int k = 0; k < n; ++k) s = fma(q[size_t(i) * n + k], ur[k * n + j], s);
        u[idx] = s;
    }
}

// ------------------------------------------------------------------ adjoint

// C(i, j) = sum_k la(k, i) lb(k, j), 0 <= i < M, 0 <= j < N, on the FP64
// tensor path (mma.sync m8n8k4, lsvd::dmma_8x8x4): the block's warps take
// blocks of 2 x 4 tiles of 8 x 8 in turn; i >= M, j >= N and k >= K read as
// zero (no accessor is called there) and only i < M, j < N reach epi.
template <class LA, class LB, class Epi>
__device__ __forceinline__ void cta_mma(int M, int N, int K, LA la, LB lb, Epi epi) {
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const int mt = (M + 7) >> 3, nt = (N + 7) >> 3;
    const int mb = (mt + 1) >> 1, nb = (nt + 3) >> 2;
    for (int blk = warp; blk < mb * nb; blk += nwarps) {
        const int ti0 = (blk % mb) * 2, tj0 = (blk / mb) * 4;
        double acc[2][4][2];
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[r][c][0] = acc[r][c][1] = 0.0;
#pragma unroll 2
        for (int k0 = 0; k0 < K; k0 += 4) {
            const int k = k0 + q;
            double av[2], bv[4];
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const int i = (ti0 + r) * 8 + g;
                av[r] = (k < K && i < M) ? la(k, i) : 0.0;
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int j = (tj0 + c) * 8 + g;
                bv[c] = (k < K && j < N) ? lb(k, j) : 0.0;
            }
#pragma unroll
            for (int r = 0; r < 2; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    if (ti0 + r < mt && tj0 + c < nt) lsvd::dmma_8x8x4(acc[r][c][0], acc[r][c][1], av[r], bv[c]);
        }
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int i = (ti0 + r) * 8 + g, j = (tj0 + c) * 8 + 2 * q + e;
                    if (i < M && j < N) epi(i, j, acc[r][c][e]);
                }
    }
}

// Leading dimension of the n x n shared buffers: n rounded up to 8, plus 4
// (= 4 mod 8: the 8 x 4 fragment loads of a half-warp hit 16 distinct banks).
__host__ __device__ constexpr int vjp_ld(int n) { return ((n + 7) & ~7) + 4; }

struct VjpArgs {
    int m, n;
    const double* A;
    const double* S;
    const int32_t* perm;
    const lsvd_rotor* rotors;
    int64_t cap;
    const int64_t* counts;
    const double* Ub;  // m x n, may be null
    const double* Sb;  // n, may be null
    const double* Vb;  // n x n (cotangent of V), may be null
    const double* Qb;  // m x n (cotangent of the polar factor U V^T), may be null
    const double* Vt;  // n x n V^T: stored by the forward, or rebuilt by vjp_replay_kernel
    const int* vstat;  // per matrix replay status (non-zero: stream overflow), may be null
    double gap_tol;
    double* Ab;        // m x n
    int* status;       // per matrix: 0 ok, 1 stream overflow, 2 sigma <= 0
};

// V = G_1 (G_2 (... (G_k P))) rebuilt from a matrix's rotor stream, replayed
// from its end, written as V^T (n x n row-major).  One CTA of kReplayThreads
// per matrix and a small shared footprint (V plus one chunk of the stream),
// so that several matrices replay per SM.  A rotation only mixes rows i and
// j of each column, so the thread that owns column `col` replays the whole
// stream on it with no barrier; the stream comes through shared memory in
// chunks with cos/sin computed once.  status: 1 when the count is outside
// [0, cap] (V^T is then zero).
__global__ void __launch_bounds__(kReplayThreads) vjp_replay_kernel(int n, const int32_t* perm,
                                                                   const lsvd_rotor* rotors, int64_t cap,
                                                                   const int64_t* counts, double* Vt,
                                                                   int* status) {
    extern __shared__ __align__(16) double shr[];
    const int ld = n + 1;  // odd: column walks are bank-conflict free
    double* V = shr;
    double2* g_cs = reinterpret_cast<double2*>(V + ((n * ld + 1) & ~1));
    int* g_ij = reinterpret_cast<int*>(g_cs + kReplayChunk);
    int* g_safe = g_ij + kReplayChunk;
    const size_t mi = blockIdx.x;
    const int tid = threadIdx.x;
    const int64_t cnt = counts[mi];
    double* vt = Vt + mi * size_t(n) * n;
    if (cnt < 0 || cnt > cap) {
        for (int idx = tid; idx < n * n; idx += blockDim.x) vt[idx] = 0.0;
        if (tid == 0) status[mi] = 1;
        return;
    }
    const int32_t* pm = perm + mi * n;
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int i = idx / n, j = idx % n;
        V[i * ld + j] = (pm[j] == i) ? 1.0 : 0.0;
    }
    __syncthreads();
    const lsvd_rotor* rot = rotors + mi * size_t(cap);
    for (int64_t hi = cnt; hi > 0;) {
        const int64_t lo = hi > kReplayChunk ? hi - kReplayChunk : 0;
        const int len = int(hi - lo);
        for (int e = tid; e < len; e += blockDim.x) {
            const lsvd_rotor r = rot[lo + e];
            double sn, cs;
            sincos(r.theta, &sn, &cs);
            g_cs[e] = make_double2(cs, sn);
            g_ij[e] = int(r.i) | (int(r.j) << 16);
        }
        // groups of four entries of one round are disjoint: replayed with all
        // loads first (the stream is in round order)
        for (int g = tid; g < len / 4; g += blockDim.x)
            g_safe[g] = rot[lo + 4 * g].round == rot[lo + 4 * g + 3].round;
        __syncthreads();
        for (int col = tid; col < n; col += blockDim.x) {
            auto one = [&](int e) {
                const double2 cs = g_cs[e];
                const int ij = g_ij[e];
                const int ri = ij & 0xffff, rj = ij >> 16;
                const double xi = V[ri * ld + col], xj = V[rj * ld + col];
                V[ri * ld + col] = cs.x * xi + cs.y * xj;
                V[rj * ld + col] = -cs.y * xi + cs.x * xj;
            };
            const int ng = len / 4;
            for (int e = len - 1; e >= 4 * ng; --e) one(e);
            for (int gi = ng - 1; gi >= 0; --gi) {
                const int e0 = 4 * gi;
                if (g_safe[gi]) {
                    int ri[4], rj[4];
                    double2 cs[4];
                    double xi[4], xj[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        cs[u] = g_cs[e0 + u];
                        const int ij = g_ij[e0 + u];
                        ri[u] = ij & 0xffff;
                        rj[u] = ij >> 16;
                        xi[u] = V[ri[u] * ld + col];
                        xj[u] = V[rj[u] * ld + col];
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        V[ri[u] * ld + col] = cs[u].x * xi[u] + cs[u].y * xj[u];
                        V[rj[u] * ld + col] = -cs[u].y * xi[u] + cs[u].x * xj[u];
                    }
                } else {
                    one(e0 + 3);
                    one(e0 + 2);
                    one(e0 + 1);
                    one(e0);
                }
            }
        }
        __syncthreads();
        hi = lo;
    }
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int j = idx / n, i = idx % n;
        vt[j * n + i] = V[i * ld + j];
    }
    if (tid == 0) status[mi] = 0;
}

size_t replay_smem_bytes(int n) {
    return size_t((n * (n + 1) + 1) & ~1) * sizeof(double) + kReplayChunk * (sizeof(double2) + sizeof(int)) +
           (kReplayChunk / 4) * sizeof(int);
}

__global__ void __launch_bounds__(kVjpThreads, 1) svd_vjp_kernel(VjpArgs a) {
    extern __shared__ __align__(16) double sh[];
    const int m = a.m, n = a.n, ld = vjp_ld(n);
    const size_t mi = blockIdx.x;
    double* V = sh;              // n x ld, row-major
    double* S1 = V + n * ld;
    double* S2 = S1 + n * ld;
    double* S3 = S2 + n * ld;
    double* S4 = S3 + n * ld;
    double* sg = S4 + n * ld;    // sigma
    double* si = sg + kMaxN;     // 1/sigma
    __shared__ int grp_bad;
    const int tid = threadIdx.x;
    const double* A = a.A + mi * size_t(m) * n;
    const double* Ub = a.Ub ? a.Ub + mi * size_t(m) * n : nullptr;
    const double* Qb = a.Qb ? a.Qb + mi * size_t(m) * n : nullptr;
    const double* Vb = a.Vb ? a.Vb + mi * size_t(n) * n : nullptr;
    const double* Sb = a.Sb ? a.Sb + mi * n : nullptr;
    double* Ab = a.Ab + mi * size_t(m) * n;
    if (tid == 0) grp_bad = 0;
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) {
        const double s = a.S[mi * n + i];
        sg[i] = s;
        si[i] = s > 0.0 ? 1.0 / s : 0.0;
        if (!(s > 0.0)) grp_bad = 2;
    }
    if (tid == 0 && a.vstat && a.vstat[mi]) grp_bad = a.vstat[mi];
    // V from V^T (stored by the forward, or rebuilt from the rotor stream)
    const double* Vst = a.Vt + mi * size_t(n) * n;
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int i = idx / n, j = idx % n;
        V[i * ld + j] = Vst[j * n + i];
    }
    __syncthreads();
    if (grp_bad) {
        for (int idx = tid; idx < m * n; idx += blockDim.x) Ab[idx] = 0.0;
        if (tid == 0) a.status[mi] = grp_bad;
        return;
    }
    // ---- G = U^T Ubar = S^-1 V^T A^T Ubar into S3
    for (int idx = tid; idx < n * ld; idx += blockDim.x) {
        S1[idx] = 0.0;
        S2[idx] = 0.0;
        S4[idx] = 0.0;
    }
    __syncthreads();
    if (Ub)
        cta_mma(n, n, m, [&](int k, int i) { return A[size_t(k) * n + i]; },
                    [&](int k, int j) { return Ub[size_t(k) * n + j]; },
                    [&](int i, int j, double v) { S1[i * ld + j] = v; });
    __syncthreads();
    cta_mma(n, n, n, [&](int k, int i) { return V[k * ld + i]; },
                [&](int k, int j) { return S1[k * ld + j]; },
                [&](int i, int j, double v) { S3[i * ld + j] = si[i] * v; });
    // ---- H = V^T Vbar into S4
    if (Vb)
        cta_mma(n, n, n, [&](int k, int i) { return V[k * ld + i]; },
                    [&](int k, int j) { return Vb[k * n + j]; },
                    [&](int i, int j, double v) { S4[i * ld + j] = v; });
    __syncthreads();
    // ---- M = U^T Qbar V = S^-1 V^T (A^T Qbar) V into S2 (polar cotangent)
    if (Qb) {
        cta_mma(n, n, m, [&](int k, int i) { return A[size_t(k) * n + i]; },
                    [&](int k, int j) { return Qb[size_t(k) * n + j]; },
                    [&](int i, int j, double v) { S2[i * ld + j] = v; });
        __syncthreads();
        cta_mma(n, n, n, [&](int k, int i) { return S2[i * ld + k]; },
                    [&](int k, int j) { return V[k * ld + j]; },
                    [&](int i, int j, double v) { S1[i * ld + j] = v; });
        __syncthreads();
        cta_mma(n, n, n, [&](int k, int i) { return V[k * ld + i]; },
                    [&](int k, int j) { return S1[k * ld + j]; },
                    [&](int i, int j, double v) { S2[i * ld + j] = si[i] * v; });
        __syncthreads();
    }
    // ---- D (into S1):
    //   F o (G - G^T) S + S F o (H - H^T) + (M - M^T) / (s_i + s_j) + diag(Sbar)
    //   - (G + M) S^-1
    // The polar part uses its exact 1/(s_i + s_j) form, which stays finite for
    // equal singular values.
    double smax = 0.0;
    for (int k = 0; k < n; ++k) smax = fmax(smax, sg[k]);
    const double gtol = a.gap_tol * smax;
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int i = idx / n, j = idx % n;
        const double g = S3[i * ld + j], mm = S2[i * ld + j];
        double d = -(g + mm) * si[j];
        if (i == j) {
            d += Sb ? Sb[i] : 0.0;
        } else {
            const double den = sg[j] * sg[j] - sg[i] * sg[i];
            const double f = (fabs(sg[j] - sg[i]) <= gtol || den == 0.0) ? 0.0 : 1.0 / den;
            d += f * ((g - S3[j * ld + i]) * sg[j] + sg[i] * (S4[i * ld + j] - S4[j * ld + i]));
            d += (mm - S2[j * ld + i]) / (sg[i] + sg[j]);
        }
        S1[i * ld + j] = d;
    }
    __syncthreads();
    // ---- E = V S^-1 D V^T: S4 = V (S^-1 D), S3 = S4 V^T
    cta_mma(n, n, n, [&](int k, int i) { return V[i * ld + k]; },
                [&](int k, int j) { return si[k] * S1[k * ld + j]; },
                [&](int i, int j, double v) { S4[i * ld + j] = v; });
    __syncthreads();
    cta_mma(n, n, n, [&](int k, int i) { return S4[i * ld + k]; },
                [&](int k, int j) { return V[j * ld + k]; },
                [&](int i, int j, double v) { S3[i * ld + j] = v; });
    // ---- Z = V S^-1 V^T into S2 (polar cotangent only)
    if (Qb)
        cta_mma(n, n, n, [&](int k, int i) { return V[i * ld + k] * si[k]; },
                    [&](int k, int j) { return V[j * ld + k]; },
                    [&](int i, int j, double v) { S2[i * ld + j] = v; });
    __syncthreads();
    // ---- Abar = A E + Ub S^-1 V^T + Qb Z   (K = n for each term)
    const int K3 = n * (1 + (Ub ? 1 : 0) + (Qb ? 1 : 0));
    cta_mma(
        m, n, K3,
        [&](int k, int i) {
            const int part = k / n, kk = k % n;
            const double* src = part == 0 ? A : (part == 1 && Ub) ? Ub : Qb;
            return src[size_t(i) * n + kk];
        },
        [&](int k, int j) {
            const int part = k / n, kk = k % n;
            if (part == 0) return S3[kk * ld + j];
            if (part == 1 && Ub) return si[kk] * V[j * ld + kk];
            return S2[kk * ld + j];
        },
        [&](int i, int j, double v) { Ab[size_t(i) * n + j] = v; });
    if (tid == 0) a.status[mi] = 0;
}

size_t vjp_smem_bytes(int n) { return size_t(5 * n * vjp_ld(n) + 2 * kMaxN) * sizeof(double); }

template <class T>
T* carve(char*& p, size_t count) {
    T* r = reinterpret_cast<T*>(p);
    p += (count * sizeof(T) + 255) & ~size_t(255);
    return r;
}

}  // namespace

extern "C" lsvd_status lsvd_svd_batched_stream_f64(lsvd_context* ctx, int64_t count, int64_t m, int64_t n,
                                                   const double* A, double* U, double* S, double* Vt,
                                                   lsvd_rotor* rotors, int64_t rotor_cap,
                                                   int64_t* rotor_count, int32_t* perm, lsvd_diag* diags,
                                                   uint32_t flags) {
    LSVD_TRACE("lsvd_svd_batched_stream_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (count < 0 || m < 1 || n < 1 || m < n)
        return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "svd_batched_stream: need m >= n >= 1");
    if (count == 0) return LSVD_OK;
    if (n > kMaxN || m > kMaxRows || count > (int64_t(1) << 31) - 1)
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "svd_batched_stream: n <= 64, m <= 4096");
    if (!A || !S || !rotors || !rotor_count || !perm || rotor_cap < 0)
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "svd_batched_stream: null pointer");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool dev = (flags & LSVD_DEVICE_POINTERS) != 0;
    const size_t cnt = size_t(count), mn = size_t(m) * n, nn = size_t(n) * n;
    cudaError_t e;
    // workspace: [A | S | rotors | counts | perm | diags (host path)] | Q | R | Ur | Vr | U | agg
    size_t bytes = 16 * 256 + (m > n ? (mn + nn) * 8 * cnt : 0) + 2 * nn * 8 * cnt;
    if (!dev)
        bytes += mn * 8 * cnt + n * 8 * cnt + size_t(rotor_cap) * 16 * cnt + 8 * cnt + 4 * n * cnt +
                 (diags ? sizeof(lsvd_diag) * cnt : 0) + (U ? mn * 8 * cnt : 0);
    char* ws = static_cast<char*>(ctx->ws_polar.get(bytes + 64 * 256, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "stream workspace");
    char* p = ws;
    const double* dA = A;
    double* dS = S;
    lsvd_rotor* dRot = rotors;
    int64_t* dCnt = rotor_count;
    int32_t* dPerm = perm;
    lsvd_diag* dDiag = diags;
    double* dU = U;
    if (!dev) {
        double* a = carve<double>(p, mn * cnt);
        if ((e = cudaMemcpyAsync(a, A, mn * cnt * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "copy A");
        dA = a;
        dS = carve<double>(p, size_t(n) * cnt);
        dRot = carve<lsvd_rotor>(p, size_t(rotor_cap) * cnt);
        dCnt = carve<int64_t>(p, cnt);
        dPerm = carve<int32_t>(p, size_t(n) * cnt);
        dDiag = diags ? carve<lsvd_diag>(p, cnt) : nullptr;
        dU = U ? carve<double>(p, mn * cnt) : nullptr;
    }
    const double* Rin = dA;
    double* dQ = nullptr;
    if (m > n) {
        dQ = carve<double>(p, mn * cnt);
        double* dR = carve<double>(p, nn * cnt);
        const size_t smem = size_t(m) * 8;
        if (smem > 48 * 1024 &&
            (e = cudaFuncSetAttribute(qr_batched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(smem))) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "qr smem");
        qr_batched_kernel<<<unsigned(cnt), kCtaThreads, smem, st>>>(int(m), int(n), dA, dQ, dR);
        ctx->launches++;
        Rin = dR;
    }
    // U_r: written straight to U when square; V_r to Vt when given
    double* dUr = (m == n && dU) ? dU : carve<double>(p, nn * cnt);
    double* dVt = (dev && Vt) ? Vt : carve<double>(p, nn * cnt);
    int* agg = carve<int>(p, 1);
    if ((e = cudaMemsetAsync(agg, 0, 4, st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "agg");
    StreamArgs sa;
    sa.n = int(n);
    sa.A = Rin;
    sa.U = dUr;
    sa.S = dS;
    sa.Vt = dVt;
    sa.diag = dDiag;
    sa.rotors = dRot;
    sa.cap = rotor_cap;
    sa.counts = dCnt;
    sa.perm = dPerm;
    sa.want_diag = (flags & LSVD_WANT_DIAG) && dDiag ? 1 : 0;
    sa.agg = agg;
    const int smem = lsvd::team_smem_doubles(int(n), lsvd::kCtaThreads / 32) * 8;
    if (n > 32) {
        if ((e = cudaFuncSetAttribute(stream_solve_kernel<4, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "stream smem");
        stream_solve_kernel<4, 8><<<unsigned(cnt), kCtaThreads, smem, st>>>(sa);
    } else {
        if ((e = cudaFuncSetAttribute(stream_solve_kernel<2, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "stream smem");
        stream_solve_kernel<2, 8><<<unsigned(cnt), kCtaThreads, smem, st>>>(sa);
    }
    ctx->launches++;
    if (m > n && dU) {
        qu_kernel<<<unsigned(cnt), 256, 0, st>>>(int(m), int(n), dQ, dUr, dU);
        ctx->launches++;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "stream kernels");
    int hagg = 0;
    if ((e = cudaMemcpyAsync(&hagg, agg, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "agg");
    if (!dev) {
        if ((e = cudaMemcpyAsync(S, dS, size_t(n) * cnt * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(rotors, dRot, size_t(rotor_cap) * cnt * 16, cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess ||
            (e = cudaMemcpyAsync(rotor_count, dCnt, cnt * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(perm, dPerm, size_t(n) * cnt * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "copy out");
        if (U && (e = cudaMemcpyAsync(U, dU, mn * cnt * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "copy U");
        if (Vt && (e = cudaMemcpyAsync(Vt, dVt, nn * cnt * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "copy Vt");
        if (diags &&
            (e = cudaMemcpyAsync(diags, dDiag, sizeof(lsvd_diag) * cnt, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "copy diags");
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "stream sync");
    if (hagg & LSVD_MAT_ROTOR_OVERFLOW)
        return lsvd_ctx_fail(ctx, LSVD_ROTOR_OVERFLOW, "svd_batched_stream: rotor_cap too small");
    if (hagg & LSVD_MAT_NONFINITE) return LSVD_NONFINITE_INPUT;
    if (hagg & (LSVD_MAT_NS_CAP | LSVD_MAT_JACOBI_CAP)) return LSVD_NOT_CONVERGED;
    return LSVD_OK;
}

extern "C" lsvd_status lsvd_svd_vjp_f64(lsvd_context* ctx, int64_t count, int64_t m, int64_t n,
                                        const double* A, const double* S, const int32_t* perm,
                                        const lsvd_rotor* rotors, int64_t rotor_cap,
                                        const int64_t* rotor_count, const double* Ubar,
                                        const double* Sbar, const double* Vbar, const double* Qbar,
                                        const double* Vt, double gap_tol, double* Abar, uint32_t flags) {
    LSVD_TRACE("lsvd_svd_vjp_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (count < 0 || m < 1 || n < 1 || m < n)
        return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "svd_vjp: need m >= n >= 1");
    if (count == 0) return LSVD_OK;
    if (n > kMaxN || m > kMaxRows || count > (int64_t(1) << 31) - 1)
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "svd_vjp: n <= 64, m <= 4096");
    if (!A || !S || !Abar || rotor_cap < 0 || !(gap_tol >= 0.0) || (!Vt && (!perm || !rotors || !rotor_count)))
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "svd_vjp: null pointer or bad gap_tol");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool dev = (flags & LSVD_DEVICE_POINTERS) != 0;
    const size_t cnt = size_t(count), mn = size_t(m) * n, nn = size_t(n) * n;
    cudaError_t e;
    size_t bytes = 8 * 256 + 4 * cnt + (Vt ? 0 : nn * 8 * cnt + 4 * cnt + 2 * 256);
    if (!dev)
        bytes += mn * 8 * cnt * (2 + (Ubar ? 1 : 0) + (Qbar ? 1 : 0)) + n * 8 * cnt * (Sbar ? 2 : 1) +
                 ((Vbar ? 1 : 0) + (Vt ? 1 : 0)) * nn * 8 * cnt + 4 * n * cnt + size_t(rotor_cap) * 16 * cnt +
                 8 * cnt;
    char* ws = static_cast<char*>(ctx->ws_polar.get(bytes + 16 * 256, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "vjp workspace");
    char* p = ws;
    VjpArgs va;
    va.m = int(m);
    va.n = int(n);
    va.cap = rotor_cap;
    va.gap_tol = gap_tol;
    auto up = [&](const void* src, size_t bytes_, const char* what, const void** dst) -> bool {
        if (!src) {
            *dst = nullptr;
            return true;
        }
        if (dev) {
            *dst = src;
            return true;
        }
        void* d = carve<char>(p, bytes_);
        if ((e = cudaMemcpyAsync(d, src, bytes_, cudaMemcpyHostToDevice, st)) != cudaSuccess) {
            lsvd_ctx_cuda(ctx, e, what);
            return false;
        }
        *dst = d;
        return true;
    };
    const void *pA, *pS, *pP, *pR, *pC, *pU, *pSb, *pV, *pQ, *pVt;
    if (!up(A, mn * 8 * cnt, "copy A", &pA) || !up(S, n * 8 * cnt, "copy S", &pS) ||
        !up(perm, 4 * n * cnt, "copy perm", &pP) || !up(rotors, size_t(rotor_cap) * 16 * cnt, "copy rotors", &pR) ||
        !up(rotor_count, 8 * cnt, "copy counts", &pC) || !up(Ubar, mn * 8 * cnt, "copy Ubar", &pU) ||
        !up(Sbar, n * 8 * cnt, "copy Sbar", &pSb) || !up(Vbar, nn * 8 * cnt, "copy Vbar", &pV) ||
        !up(Qbar, mn * 8 * cnt, "copy Qbar", &pQ) || !up(Vt, nn * 8 * cnt, "copy Vt", &pVt))
        return LSVD_CUDA_ERROR;
    va.A = static_cast<const double*>(pA);
    va.S = static_cast<const double*>(pS);
    va.perm = static_cast<const int32_t*>(pP);
    va.rotors = static_cast<const lsvd_rotor*>(pR);
    va.counts = static_cast<const int64_t*>(pC);
    va.Ub = static_cast<const double*>(pU);
    va.Sb = static_cast<const double*>(pSb);
    va.Vb = static_cast<const double*>(pV);
    va.Qb = static_cast<const double*>(pQ);
    va.Vt = static_cast<const double*>(pVt);
    va.Ab = dev ? Abar : carve<double>(p, mn * cnt);
    va.status = carve<int>(p, cnt);
    va.vstat = nullptr;
    if (!Vt) {
        // V rebuilt from the rotor streams first, several matrices per SM
        double* vrep = carve<double>(p, nn * cnt);
        int* rstat = carve<int>(p, cnt);
        const size_t rsmem = replay_smem_bytes(int(n));
        if ((e = cudaFuncSetAttribute(vjp_replay_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(rsmem))) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "replay smem");
        vjp_replay_kernel<<<unsigned(cnt), kReplayThreads, rsmem, st>>>(
            int(n), va.perm, va.rotors, rotor_cap, va.counts, vrep, rstat);
        ctx->launches++;
        if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "vjp_replay_kernel");
        va.Vt = vrep;
        va.vstat = rstat;
    }
    const size_t smem = vjp_smem_bytes(int(n));
    if ((e = cudaFuncSetAttribute(svd_vjp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))) !=
        cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "vjp smem");
    svd_vjp_kernel<<<unsigned(cnt), kVjpThreads, smem, st>>>(va);
    ctx->launches++;
    if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "svd_vjp_kernel");
    std::vector<int> hst(cnt);
    if ((e = cudaMemcpyAsync(hst.data(), va.status, 4 * cnt, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "vjp status");
    if (!dev && (e = cudaMemcpyAsync(Abar, va.Ab, mn * 8 * cnt, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "copy Abar");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "vjp sync");
    int worst = 0;
    for (int s : hst) worst = std::max(worst, s);
    if (worst == 1) return lsvd_ctx_fail(ctx, LSVD_ROTOR_OVERFLOW, "svd_vjp: a rotor count exceeds rotor_cap");
    if (worst == 2) return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "svd_vjp: a singular value is <= 0 (Abar zeroed)");
    return LSVD_OK;
}
