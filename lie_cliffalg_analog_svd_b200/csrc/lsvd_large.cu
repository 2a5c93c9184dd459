// lsvd_large.cu -- SVD of one large dense matrix (n > 64, or thin m x n with
// n > 64): LieSvdSmall::solve (src/lie_svd_small.rs:296-323) and
// LieSvdSmall::solve_rectangular (:340-360) beyond the shared-memory-resident
// batched kernels.
//
// FP64 route (the reference's): Newton-Schulz polar A = Q H on the FP64
// tensor path (lsvd_polar_run), P = sym(Q^T A) (:305-309), the eigenvectors V
// of P by Jacobi, sigma = max(lambda, 0) in descending order, U = Q V (:313).
// A tall m x n input runs the polar iteration on the m x n matrix itself
// (Q^T Q = I), which gives the same thin SVD as the reference's qr_reduce +
// solve(R) (:340-360); a wide one runs on A^T (:343-348).
//
// The eigensolve is eigh_jacobi_full (:212-285) blocked for the GPU: indices
// are grouped in blocks of 32, and round-robin layers (the circle method of
// layer_pairs, src/lie_svd_joint.rs:524-539) pair the blocks.  Per sweep the
// reference's start-of-sweep test off(P) < 1e-13 ||P||_F (offnorm_part_kernel, offnorm_final_kernel);
// per layer
//   solve2_kernel   diagonalises the 64 x 64 diagonal block of every block
//                   pair by cyclic Jacobi sweeps (the reference's tangent,
//                   parallel round-robin order) into one orthogonal R
//   twoside_kernel  P <- R^T P R, one CTA per 64 x 64 block of the
//                   block-pair triangle (R_a^T P_ab R_b)
//   apply_kernel    V <- V R on V's column-major store
// with every product on the FP64 tensor path (mma.sync m8n8k4).  The
// eigenvalues are the Rayleigh quotients v_j^T P v_j of the converged basis.
// Parity with the reference is numerical (a parallel order), not bitwise.
//
// The one-sided (Hestenes) form of the same blocking -- Gram of a block pair
// (gram_kernel), its diagonalisation (solve_kernel), and the column update of
// the panel store H = [G; V] (apply_kernel) -- orthogonalises the columns of
// an m x n matrix G; the mixed-precision route runs it on G = A V0.
// Each sweep is one captured CUDA graph; every kernel reads the device-side
// convergence flag and returns at once after it is set.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "lsvd.h"
#include "lsvd_dgemm.cuh"
#include "lsvd_internal.h"

namespace {

using lsvd::dg::cp_async16;
using lsvd::dg::cp_async_commit;
using lsvd::dg::cp_async_wait;
using lsvd::dg::dmma;

constexpr int BW = 32;   // columns per block
constexpr int PW = 64;   // columns per block pair
constexpr int GLD = 36;  // gram tile: [64 columns][32 rows + 4], = 4 mod 16
constexpr int XLD = 68;  // apply tile: [64 columns][64 rows + 4]
constexpr int MLD = 65;  // 64 x 64 Gram / rotation in the solve kernel

struct SweepState {
    double scale2;                 // sigma_1^2 estimate of this sweep (largest squared column norm seen)
    unsigned long long next_scale2;  // bits of the largest squared column norm seen this sweep
    unsigned long long max_off;  // bits of the largest scaled off-diagonal seen this sweep (>= 0)
    int rotated;                 // some pair rotated this sweep
    int converged;
    int sweeps;                  // completed sweeps
    int inner_cap;               // pairs whose inner sweeps hit the cap
    unsigned long long rotations;  // plane rotations applied inside the block solves
    double last_off;             // max_off of the last completed sweep
};

// Block pair k of round-robin layer `layer` over nb blocks (nb even).
__device__ __forceinline__ void block_pair(int nb, int layer, int k, int& a, int& b) {
    const int ring = nb - 1;
    if (k == 0) {
        a = nb - 1;
        b = layer % ring;
    } else {
        a = (layer + k) % ring;
        b = (layer + ring - k) % ring;
    }
}

__device__ __forceinline__ int hrow_of(int col, int P, int Q) {
    return col < BW ? P * BW + col : Q * BW + (col - BW);
}

// M partial of block pair blockIdx.x over rows [chunk*kchunk, +kchunk) of G.
__global__ void __launch_bounds__(256) gram_kernel(const double* __restrict__ H, int64_t ldh, int nb, int layer,
                                                   int kchunk, int gpad, double* __restrict__ Mpart,
                                                   const SweepState* __restrict__ stt) {
    if (stt->converged) return;
    extern __shared__ __align__(16) double gsmem[];
    double(*Xs)[PW * GLD] = reinterpret_cast<double(*)[PW * GLD]>(gsmem);  // three stages
    const int pair = blockIdx.x, chunk = blockIdx.y, nchunk = gridDim.y;
    int P, Q;
    block_pair(nb, layer, pair, P, Q);
    const int k_lo = chunk * kchunk;
    const int k_hi = min(gpad, k_lo + kchunk);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wi = warp >> 2, wj = warp & 3;
    const int g = lane >> 2, q = lane & 3;
    double acc[4][2][2];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int u = 0; u < 2; ++u) acc[t][u][0] = acc[t][u][1] = 0.0;
    const int KT = k_hi > k_lo ? (k_hi - k_lo) / 32 : 0;
    auto load = [&](int s, int kt) {
        const int k0 = k_lo + kt * 32;
#pragma unroll
        for (int it = 0; it < 4; ++it) {
            const int c = tid + it * 256;
            const int col = c >> 4, kc = (c & 15) * 2;
            cp_async16(&Xs[s][col * GLD + kc], H + int64_t(hrow_of(col, P, Q)) * ldh + k0 + kc, 16);
        }
    };
    if (KT > 0) load(0, 0);
    cp_async_commit();
    if (KT > 1) load(1, 1);
    cp_async_commit();
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<1>();
        __syncthreads();
        if (kt + 2 < KT) load((kt + 2) % 3, kt + 2);
        cp_async_commit();
        const double* X = Xs[kt % 3];
#pragma unroll
        for (int kk = 0; kk < 32; kk += 4) {
            double a[4], b[2];
#pragma unroll
            for (int t = 0; t < 4; ++t) a[t] = X[(wi * 32 + t * 8 + g) * GLD + kk + q];
#pragma unroll
            for (int u = 0; u < 2; ++u) b[u] = X[(wj * 16 + u * 8 + g) * GLD + kk + q];
#pragma unroll
            for (int t = 0; t < 4; ++t)
#pragma unroll
                for (int u = 0; u < 2; ++u) dmma(acc[t][u][0], acc[t][u][1], a[t], b[u]);
        }
    }
    cp_async_wait<0>();
    double* out = Mpart + (int64_t(pair) * nchunk + chunk) * (PW * PW);
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int i = wi * 32 + t * 8 + g, j = wj * 16 + u * 8 + 2 * q;
            out[i * PW + j] = acc[t][u][0];
            out[i * PW + j + 1] = acc[t][u][1];
        }
}

// Maximum over the CTA's NT threads (same value on every thread); red >= NT / 32.
template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) r = fmax(r, red[w]);
    __syncthreads();
    return r;
}

// The scale a Gram entry M_ij is measured against: the larger of
// sqrt(M_ii M_jj) (the cosine of the two columns) and sqrt(S max(M_ii, M_jj))
// (the normwise scale, S = sigma_1^2).  A pair is rotated when |M_ij| exceeds
// tol times this scale: columns far below sigma_1 are orthogonalised down to
// an absolute error tol sigma_1 |g|, the normwise accuracy of the reference's
// own stopping rule (off(P) < 1e-13 ||P||_F, src/lie_svd_small.rs:226),
// instead of to a relative cosine that rounding in the larger columns (about
// eps sigma_1) puts out of reach.
__device__ __forceinline__ double pair_scale(double mii, double mjj, double S) {
    return fmax(sqrt(mii * mjj), sqrt(S * fmax(mii, mjj)));
}

// Largest scaled off-diagonal |M_ij| / pair_scale over i < j of the 64 x 64
// Gram in shared memory.
template <int NT>
__device__ __forceinline__ void scaled_offdiag(const double* Ms, double S, double* red, double& all, double& cross) {
    double off = 0.0, offc = 0.0;
    for (int e = threadIdx.x; e < PW * PW; e += NT) {
        const int i = e >> 6, j = e & 63;
        if (i < j) {
            const double d = pair_scale(Ms[i * MLD + i], Ms[j * MLD + j], S);
            if (d > 0.0) {
                const double v = fabs(Ms[i * MLD + j]) / d;
                off = fmax(off, v);
                if (i < BW && j >= BW) offc = fmax(offc, v);
            }
        }
    }
    all = block_max<NT>(off, red);
    cross = block_max<NT>(offc, red);
}



// Index of column/row `c` (0..63) of block pair (P, Q) in the full matrix.
__device__ __forceinline__ int pair_index(int c, int P, int Q) { return hrow_of(c, P, Q); }

// Two-sided route, sweep start: off(P)^2 = sum_{p<q} P_pq^2 over the
// symmetric P (npad x npad, row-major); the solve stops before the sweep when
// sqrt(off) < tol_ref ||P0||_F -- the test eigh_jacobi_full makes at the start
// of every sweep (src/lie_svd_small.rs:220-228).  Partial sums per CTA, then
// one CTA adds them and sets the flag.
__global__ void __launch_bounds__(256) offnorm_part_kernel(const double* __restrict__ P, int64_t ldp, int n,
                                                           const SweepState* __restrict__ stt,
                                                           double* __restrict__ part) {
    if (stt->converged) return;
    __shared__ double red[8];
    double s = 0.0;
    // rows i = blockIdx.x + k gridDim.x, the upper triangle of each row
    for (int i = blockIdx.x; i < n; i += gridDim.x)
        for (int j = i + 1 + threadIdx.x; j < n; j += 256) {
            const double v = P[int64_t(i) * ldp + j];
            s += v * v;
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}

__global__ void offnorm_final_kernel(const double* __restrict__ part, int nparts, SweepState* __restrict__ stt,
                                     double limit) {
    if (stt->converged) return;
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += 256) s += part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double off = sqrt(red[0]);
        stt->last_off = off;
        if (off < limit) stt->converged = 1;
    }
}

// Slot k (0..31) of round `round` of a block-pair solve over the 64 local
// indices (block lo = 0..31, block hi = 32..63).  Cross rounds (round 0..31)
// pair lo index k with hi index 32 + (k + round) mod 32; the 31 inner rounds
// pair the indices inside each block by the circle method of
// src/lie_svd_joint.rs:524-539 over 32 (index 31 fixed; slots 0..15 in lo,
// 16..31 the same pairs in hi).
__device__ __forceinline__ void bp2_slot(bool inner, int round, int k, int& p, int& q) {
    if (!inner) {
        p = k;
        q = BW + ((k + round) & (BW - 1));
        return;
    }
    const int off = k < BW / 2 ? 0 : BW, kk = k & (BW / 2 - 1);
    if (kk == 0) {
        p = BW - 1;
        q = round;
    } else {
        p = round + kk;
        p -= p >= BW - 1 ? BW - 1 : 0;
        q = round - kk;
        q += q < 0 ? BW - 1 : 0;
    }
    p += off;
    q += off;
}

// The rounds of one block-pair solve by a 1024-thread CTA (see
// solve2_kernel): cross rounds on every layer, the inner rounds of both
// blocks first when with_inner; up to inner_max passes while some pair
// rotates.  rotate(app, aqq, apq) decides a pair.  On return this thread
// holds rows warp, warp + 32 of R's lo column `lane` (l0, l1) and hi column
// 32 + lane (h0, h1); *cnt (lane 0 of warp 0) counts the rotations.
// Returns the passes run (inner_max + 1 when the cap was hit).
template <class Rot>
__device__ int pair_rounds(double* Ms, bool with_inner, int inner_max, Rot rotate, double* cs, double* sn,
                           int* s_flag_p, int& cnt, double& l0, double& l1, double& h0, double& h1) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int& s_flag = *s_flag_p;
    int ka = 0, kb = 0;
    const bool upd = tid < 32 * 33 / 2;
    if (upd) {
        int rem = tid;
        while (rem >= 32 - ka) {
            rem -= 32 - ka;
            ++ka;
        }
        kb = ka + rem;
    }
    l0 = warp == lane ? 1.0 : 0.0, h0 = warp == lane + BW ? 1.0 : 0.0;
    l1 = warp + 32 == lane ? 1.0 : 0.0, h1 = warp + 32 == lane + BW ? 1.0 : 0.0;
    int sweep = 0;
    for (; sweep < inner_max; ++sweep) {
        if (tid == 0) s_flag = 0;
        __syncthreads();
        const int nround = with_inner ? (BW - 1) + BW : BW;
        for (int it = 0; it < nround; ++it) {
            const bool inner = with_inner && it < BW - 1;
            const int round = inner ? it : it - (with_inner ? BW - 1 : 0);
            if (warp == 0) {
                int p, qq;
                bp2_slot(inner, round, lane, p, qq);
                const double app = Ms[p * MLD + p], aqq = Ms[qq * MLD + qq], apq = Ms[p * MLD + qq];
                double c = 1.0, s = 0.0;
                const bool rot = apq != 0.0 && rotate(app, aqq, apq);
                if (rot) {
                    // the reference's smaller-root tangent (src/lie_svd_small.rs:235-242, its
                    // theta >= 0 branch for theta = -0 included); the cosine by one reciprocal
                    // square root: each column of V takes tens of thousands of rotations
                    // here, and 1 / sqrt(.) with its two roundings leaves c^2 + s^2 biased
                    // enough that the orthogonality drifts (10-20x larger at n = 2048)
                    const double theta = (aqq - app) / (2.0 * apq);
                    const double t = theta >= 0.0 ? 1.0 / (theta + sqrt(theta * theta + 1.0))
                                                  : -1.0 / (-theta + sqrt(theta * theta + 1.0));
                    c = rsqrt(t * t + 1.0);
                    s = t * c;
                }
                const unsigned msk = __ballot_sync(0xffffffffu, rot);
                if (lane == 0 && msk) {
                    cnt += __popc(msk);
                    s_flag = 1;
                }
                cs[lane] = c;
                sn[lane] = s;
            }
            __syncthreads();
            if (upd) {
                const double ca = cs[ka], sa = sn[ka], cb = cs[kb], sb = sn[kb];
                if (sa != 0.0 || sb != 0.0) {
                    int ra, rb, ca_, cb_;
                    bp2_slot(inner, round, ka, ra, rb);
                    bp2_slot(inner, round, kb, ca_, cb_);
                    const double x = Ms[ra * MLD + ca_], y = Ms[ra * MLD + cb_];
                    const double z = Ms[rb * MLD + ca_], w = Ms[rb * MLD + cb_];
                    const double x1 = cb * x - sb * y, y1 = sb * x + cb * y;
                    const double z1 = cb * z - sb * w, w1 = sb * z + cb * w;
                    const double x2 = ca * x1 - sa * z1, w2 = sa * y1 + ca * w1;
                    double y2 = ca * y1 - sa * w1, z2 = sa * x1 + ca * z1;
                    if (ka == kb) y2 = z2 = 0.0;  // the pair this rotation annihilates
                    Ms[ra * MLD + ca_] = x2;
                    Ms[ra * MLD + cb_] = y2;
                    Ms[rb * MLD + ca_] = z2;
                    Ms[rb * MLD + cb_] = w2;
                    if (ka != kb) {
                        Ms[ca_ * MLD + ra] = x2;
                        Ms[cb_ * MLD + ra] = y2;
                        Ms[ca_ * MLD + rb] = z2;
                        Ms[cb_ * MLD + rb] = w2;
                    }
                }
            }
            if (inner) {
                // lane's index x in its block: role and partner in the circle method
                int k, partner;
                bool role_p;
                if (lane == BW - 1) {
                    k = 0, role_p = true, partner = round;
                } else if (lane == round) {
                    k = 0, role_p = false, partner = BW - 1;
                } else {
                    int d = lane - round;
                    d += d < 0 ? BW - 1 : 0;
                    role_p = d <= BW / 2 - 1;
                    k = role_p ? d : BW - 1 - d;
                    partner = role_p ? round - k : round + k;
                    partner += partner < 0 ? BW - 1 : 0;
                    partner -= partner >= BW - 1 ? BW - 1 : 0;
                }
                const double cl = cs[k], sl = sn[k], ch = cs[BW / 2 + k], sh = sn[BW / 2 + k];
                const double pl0 = __shfl_sync(0xffffffffu, l0, partner), pl1 = __shfl_sync(0xffffffffu, l1, partner);
                const double ph0 = __shfl_sync(0xffffffffu, h0, partner), ph1 = __shfl_sync(0xffffffffu, h1, partner);
                if (role_p) {
                    l0 = cl * l0 - sl * pl0, l1 = cl * l1 - sl * pl1;
                    h0 = ch * h0 - sh * ph0, h1 = ch * h1 - sh * ph1;
                } else {
                    l0 = sl * pl0 + cl * l0, l1 = sl * pl1 + cl * l1;
                    h0 = sh * ph0 + ch * h0, h1 = sh * ph1 + ch * h1;
                }
            } else {
                const double c = cs[lane], s = sn[lane];
                const double u0 = c * l0 - s * h0, v0 = s * l0 + c * h0;
                const double u1 = c * l1 - s * h1, v1 = s * l1 + c * h1;
                l0 = u0, l1 = u1;
                h0 = __shfl_sync(0xffffffffu, v0, (lane + 1) & 31);
                h1 = __shfl_sync(0xffffffffu, v1, (lane + 1) & 31);
            }
            __syncthreads();
        }
        const int any = s_flag;
        __syncthreads();
        if (!any) break;
    }
    return sweep == inner_max ? inner_max + 1 : sweep + 1;
}

// Two-sided route (1024 threads: the rounds of a block-pair solve are the
// critical path of every layer): gathers the 64 x 64 diagonal block M of
// block pair blockIdx.x from P, rotates (|a_pq| > tau; the reference rotates
// every |a_pq| >= 1e-300, src/lie_svd_small.rs:233-235, with the smaller-root
// tangent of :235-242) and writes R / skip like solve_kernel.  Every index pair
// is visited once per sweep, as in the reference: its 32 cross rounds
// (lo x hi pairs) on every layer, the 31 inner rounds of both blocks on
// layer 0 only (every block is in a layer-0 pair).  Per round, warp 0
// computes the 32 rotations (lane k <-> slot k); threads t < 528 update one
// 2 x 2 block (slot a <= slot b) of the symmetric M as J_a^T M_ab J_b and
// store it and its transpose.  R stays in registers: thread (warp w, lane k)
// holds rows w and w + 32 of lo column k and of one hi column; a cross round
// rotates the pair in place and passes the hi column to lane k - 1, an inner
// round fetches the partner column of the same block from its lane.
__global__ void __launch_bounds__(1024) solve2_kernel(const double* __restrict__ P, int64_t ldp, int nb, int layer,
                                                     double* __restrict__ Rg, int* __restrict__ skip,
                                                     SweepState* __restrict__ stt, double tau, int inner_max) {
    if (stt->converged) return;
    extern __shared__ __align__(16) double ssmem[];
    double* Ms = ssmem;
    __shared__ double cs[32], sn[32];
    __shared__ double red[32];
    __shared__ int s_flag;
    const int pair = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool with_inner = layer == 0;
    int Pb, Qb;
    block_pair(nb, layer, pair, Pb, Qb);
    for (int e = tid; e < PW * PW; e += 1024) {
        const int i = e >> 6, j = e & 63;
        Ms[i * MLD + j] = P[int64_t(pair_index(i, Pb, Qb)) * ldp + pair_index(j, Pb, Qb)];
    }
    __syncthreads();
    // largest entry this solve may rotate: every off-diagonal on layer 0,
    // the cross block otherwise
    double off = 0.0;
    for (int e = tid; e < PW * PW; e += 1024) {
        const int i = e >> 6, j = e & 63;
        if (with_inner ? i < j : (i < BW && j >= BW)) off = fmax(off, fabs(Ms[i * MLD + j]));
    }
    off = block_max<1024>(off, red);
    if (!(off > tau)) {
        if (tid == 0) skip[pair] = 1;
        return;
    }
    double l0, l1, h0, h1;
    int cnt = 0;
    const int sw = pair_rounds(
        Ms, with_inner, inner_max, [&](double, double, double apq) { return fabs(apq) > tau; }, cs, sn, &s_flag,
        cnt, l0, l1, h0, h1);
    double* R = Rg + int64_t(pair) * (PW * PW);
    R[warp * PW + lane] = l0;
    R[warp * PW + BW + lane] = h0;
    R[(warp + 32) * PW + lane] = l1;
    R[(warp + 32) * PW + BW + lane] = h1;
    if (tid == 0) {
        skip[pair] = 0;
        stt->rotated = 1;
        atomicAdd(&stt->rotations, (unsigned long long)cnt);
        if (sw > inner_max) atomicAdd(&stt->inner_cap, 1);
    }
}

// One-sided route: sums the Gram partials of a block pair, tests it, and
// rotates its pairs as solve2_kernel does (pair_rounds; a pair rotates when
// |g_pq| > tol * pair_scale), writing R (64 x 64, row-major, Rg[pair]) and
// skip[pair] = 1 when no pair this solve visits needs a rotation.  The
// sweep's convergence measure is the largest scaled off-diagonal over every
// pair of every Gram the sweep forms.
__global__ void __launch_bounds__(1024) solve_kernel(const double* __restrict__ Mpart, int nchunk, int layer,
                                                     double* __restrict__ Rg, int* __restrict__ skip,
                                                     SweepState* __restrict__ stt, double tol, int inner_max) {
    if (stt->converged) return;
    extern __shared__ __align__(16) double ssmem[];
    double* Ms = ssmem;  // 64 x 64 Gram, leading dimension 65
    __shared__ double cs[32], sn[32];
    __shared__ double red[32];
    __shared__ int s_flag;
    const int pair = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool with_inner = layer == 0;
    const double* mp = Mpart + int64_t(pair) * nchunk * (PW * PW);
    for (int e = tid; e < PW * PW; e += 1024) {
        double v = 0.0;
        for (int c = 0; c < nchunk; ++c) v += mp[int64_t(c) * (PW * PW) + e];
        Ms[(e >> 6) * MLD + (e & 63)] = v;
    }
    __syncthreads();
    const double S = stt->scale2;
    {
        double dmax = 0.0;
        for (int i = tid; i < PW; i += 1024) dmax = fmax(dmax, Ms[i * MLD + i]);
        dmax = block_max<1024>(dmax, red);
        if (tid == 0)
            atomicMax(&stt->next_scale2, static_cast<unsigned long long>(__double_as_longlong(dmax)));
    }
    double off_all, off_cross;
    scaled_offdiag<1024>(Ms, S, red, off_all, off_cross);
    if (tid == 0) atomicMax(&stt->max_off, static_cast<unsigned long long>(__double_as_longlong(off_all)));
    if (!((with_inner ? off_all : off_cross) > tol)) {  // also catches NaN: nothing to rotate
        if (tid == 0) skip[pair] = 1;
        return;
    }
    double l0, l1, h0, h1;
    int cnt = 0;
    const int sw = pair_rounds(
        Ms, with_inner, inner_max,
        [&](double app, double aqq, double apq) { return fabs(apq) > tol * pair_scale(app, aqq, S); }, cs, sn,
        &s_flag, cnt, l0, l1, h0, h1);
    double* R = Rg + int64_t(pair) * (PW * PW);
    R[warp * PW + lane] = l0;
    R[warp * PW + BW + lane] = h0;
    R[(warp + 32) * PW + lane] = l1;
    R[(warp + 32) * PW + BW + lane] = h1;
    if (tid == 0) {
        skip[pair] = 0;
        stt->rotated = 1;
        atomicAdd(&stt->rotations, (unsigned long long)cnt);
        if (sw > inner_max) atomicAdd(&stt->inner_cap, 1);
    }
}

// Two-sided route: P <- R^T P R for the block-diagonal R of one layer.  CTA
// (a, b), a <= b, computes the 64 x 64 block C = R_a^T P_ab R_b of block
// pairs a and b (R = I for a skipped pair) and writes C to P_ab and C^T to
// P_ba; the blocks are disjoint, so every block of P is written once.
// Both products on the FP64 tensor path.
// tiles: NULL for every block pair (a, b) of the triangle (CTA i = the i-th
// in row order), else CTA i takes tile tiles[i] = a * 65536 + b.
__global__ void __launch_bounds__(256, 2) twoside_kernel(double* __restrict__ P, int64_t ldp, int nb, int layer,
                                                         const double* __restrict__ Rg,
                                                         const int* __restrict__ skip,
                                                         const SweepState* __restrict__ stt,
                                                         const int* __restrict__ tiles) {
    if (stt->converged) return;
    int a = 0, b = 0;
    if (tiles) {
        a = tiles[blockIdx.x] >> 16;
        b = tiles[blockIdx.x] & 0xffff;
    } else {
        // (a, b) from the linear CTA index over the upper triangle of npairs x npairs
        const int npairs = nb / 2;
        int rem = blockIdx.x;
        while (rem >= npairs - a) {
            rem -= npairs - a;
            ++a;
        }
        b = a + rem;
    }
    const bool ra = !skip[a], rb = !skip[b];
    if (!ra && !rb) return;
    extern __shared__ __align__(16) double tsm[];
    double* Ps = tsm;                // P_ab, then T = P_ab R_b   [64][68]
    double* Ra = tsm + PW * XLD;     // R_a                        [64][68]
    double* Rb = tsm + 2 * PW * XLD; // R_b                        [64][68]
    int Pa, Qa, Pb2, Qb2;
    block_pair(nb, layer, a, Pa, Qa);
    block_pair(nb, layer, b, Pb2, Qb2);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wi = warp >> 1, wj = warp & 1;  // 4 x 2 warps; warp tile 16 rows x 32 columns
    const int g = lane >> 2, q = lane & 3;
    for (int c = tid; c < PW * PW / 2; c += 256) {
        const int i = c >> 5, jc = (c & 31) * 2;
        cp_async16(&Ps[i * XLD + jc], P + int64_t(pair_index(i, Pa, Qa)) * ldp + pair_index(jc, Pb2, Qb2), 16);
        if (ra) cp_async16(&Ra[i * XLD + jc], Rg + int64_t(a) * (PW * PW) + i * PW + jc, 16);
        if (rb) cp_async16(&Rb[i * XLD + jc], Rg + int64_t(b) * (PW * PW) + i * PW + jc, 16);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    double acc[2][4][2];
    if (rb) {  // T = P_ab R_b
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[t][u][0] = acc[t][u][1] = 0.0;
#pragma unroll 4
        for (int k0 = 0; k0 < PW; k0 += 4) {
            double av[2], bv[4];
#pragma unroll
            for (int t = 0; t < 2; ++t) av[t] = Ps[(wi * 16 + t * 8 + g) * XLD + k0 + q];
#pragma unroll
            for (int u = 0; u < 4; ++u) bv[u] = Rb[(k0 + q) * XLD + wj * 32 + u * 8 + g];
#pragma unroll
            for (int t = 0; t < 2; ++t)
#pragma unroll
                for (int u = 0; u < 4; ++u) dmma(acc[t][u][0], acc[t][u][1], av[t], bv[u]);
        }
        __syncthreads();  // every warp has read P_ab
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = wi * 16 + t * 8 + g, j = wj * 32 + u * 8 + 2 * q;
                Ps[i * XLD + j] = acc[t][u][0];
                Ps[i * XLD + j + 1] = acc[t][u][1];
            }
        __syncthreads();
    }
    // C = R_a^T T (or C = T when a is skipped)
#pragma unroll
    for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[t][u][0] = acc[t][u][1] = 0.0;
    if (ra) {
#pragma unroll 4
        for (int k0 = 0; k0 < PW; k0 += 4) {
            double av[2], bv[4];
#pragma unroll
            for (int t = 0; t < 2; ++t) av[t] = Ra[(k0 + q) * XLD + wi * 16 + t * 8 + g];
#pragma unroll
            for (int u = 0; u < 4; ++u) bv[u] = Ps[(k0 + q) * XLD + wj * 32 + u * 8 + g];
#pragma unroll
            for (int t = 0; t < 2; ++t)
#pragma unroll
                for (int u = 0; u < 4; ++u) dmma(acc[t][u][0], acc[t][u][1], av[t], bv[u]);
        }
    } else {
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = wi * 16 + t * 8 + g, j = wj * 32 + u * 8 + 2 * q;
                acc[t][u][0] = Ps[i * XLD + j];
                acc[t][u][1] = Ps[i * XLD + j + 1];
            }
    }
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int i = wi * 16 + t * 8 + g;
        const int gi = pair_index(i, Pa, Qa);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int j = wj * 32 + u * 8 + 2 * q;
            const int gj = pair_index(j, Pb2, Qb2);  // j, j + 1 in the same 32-block
            *reinterpret_cast<double2*>(P + int64_t(gi) * ldp + gj) = make_double2(acc[t][u][0], acc[t][u][1]);
            if (a != b) {
                P[int64_t(gj) * ldp + gi] = acc[t][u][0];
                P[int64_t(gj + 1) * ldp + gi] = acc[t][u][1];
            }
        }
    }
}

// [G_p G_q; V_p V_q] <- [G_p G_q; V_p V_q] R over rows [chunk*rows, +rows) of H.
// Computed transposed, C'(j, row) = sum_i R(i, j) H(row, col_i), so that the
// result lands on H's column-major storage in 16-byte pairs.
__global__ void __launch_bounds__(256, 2) apply_kernel(double* __restrict__ H, int64_t ldh, int nb, int layer,
                                                       int rows, const double* __restrict__ Rg,
                                                       const int* __restrict__ skip,
                                                       const SweepState* __restrict__ stt) {
    if (stt->converged) return;
    const int pair = blockIdx.x;
    if (skip[pair]) return;
    extern __shared__ __align__(16) double asmem[];
    double* Rs = asmem;                 // [64][68]
    double* Xs0 = asmem + PW * XLD;     // two [64][68] stages
    int P, Q;
    block_pair(nb, layer, pair, P, Q);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wj = warp >> 1, wr = warp & 1;  // 4 (j) x 2 (rows); warp tile 16 j x 32 rows
    const int g = lane >> 2, q = lane & 3;
    const double* R = Rg + int64_t(pair) * (PW * PW);
    for (int c = tid; c < PW * PW / 2; c += 256) {
        const int i = c >> 5, jc = (c & 31) * 2;
        cp_async16(&Rs[i * XLD + jc], R + i * PW + jc, 16);
    }
    cp_async_commit();
    const int64_t r_lo = int64_t(blockIdx.y) * rows;
    const int64_t r_hi = min(int64_t(ldh), r_lo + rows);
    const int NT = r_hi > r_lo ? int((r_hi - r_lo) / 64) : 0;
    auto load = [&](int s, int t) {
        double* X = Xs0 + s * PW * XLD;
        const int64_t r0 = r_lo + int64_t(t) * 64;
#pragma unroll
        for (int it = 0; it < 8; ++it) {
            const int c = tid + it * 256;
            const int i = c >> 5, rc = (c & 31) * 2;
            cp_async16(&X[i * XLD + rc], H + int64_t(hrow_of(i, P, Q)) * ldh + r0 + rc, 16);
        }
    };
    if (NT > 0) load(0, 0);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    // A = R^T fragments for this warp's 16 columns j over all 64 i, kept in registers
    double ra[16][2];
#pragma unroll
    for (int kk = 0; kk < 16; ++kk)
#pragma unroll
        for (int t = 0; t < 2; ++t) ra[kk][t] = Rs[(kk * 4 + q) * XLD + wj * 16 + t * 8 + g];
    for (int t = 0; t < NT; ++t) {
        if (t + 1 < NT) load((t + 1) & 1, t + 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const double* X = Xs0 + (t & 1) * PW * XLD;
        double acc[2][4][2];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[a][u][0] = acc[a][u][1] = 0.0;
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            double b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) b[u] = X[(kk * 4 + q) * XLD + wr * 32 + u * 8 + g];
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int u = 0; u < 4; ++u) dmma(acc[a][u][0], acc[a][u][1], ra[kk][a], b[u]);
        }
        const int64_t r0 = r_lo + int64_t(t) * 64;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            const int j = wj * 16 + a * 8 + g;
            double* hcol = H + int64_t(hrow_of(j, P, Q)) * ldh + r0 + wr * 32 + 2 * q;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                *reinterpret_cast<double2*>(hcol + u * 8) = make_double2(acc[a][u][0], acc[a][u][1]);
        }
        __syncthreads();  // the stage just read is the next prefetch's target
    }
    cp_async_wait<0>();
}

// End of a sweep: converged when no pair rotated, or when every pair started
// the sweep within tol_conv -- the sweep's own rotations then leave every
// scaled off-diagonal at about tol_conv^2 (Jacobi's quadratic convergence),
// far below the rotation threshold.
__global__ void sweep_end_kernel(SweepState* stt, double tol_conv) {
    if (stt->converged) return;
    stt->sweeps += 1;
    const double off = __longlong_as_double(static_cast<long long>(stt->max_off));
    stt->last_off = off;
    if (!stt->rotated || off <= tol_conv) stt->converged = 1;
    stt->rotated = 0;
    stt->max_off = 0ull;
    stt->scale2 = fmax(stt->scale2, __longlong_as_double(static_cast<long long>(stt->next_scale2)));
    stt->next_scale2 = 0ull;
}

// P2 (npad x npad) = scale sym(P) with zero padding; Vc (npad x npad) = I.
__global__ void fill_p2v_kernel(const double* P, int64_t ld, int n, double scale, double* P2, double* Vc, int npad) {
    const int64_t tot = int64_t(npad) * npad;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < tot; e += int64_t(gridDim.x) * blockDim.x) {
        const int r = int(e / npad), j = int(e % npad);
        P2[e] = (r < n && j < n) ? 0.5 * scale * (P[int64_t(r) * ld + j] + P[int64_t(j) * ld + r]) : 0.0;
        Vc[e] = r == j ? 1.0 : 0.0;
    }
}

// sigma_j = ||g_j||, and the sign test of the plain route: lambda_j = v_j . g_j
// (G = P V, so g_j = lambda_j v_j at convergence).  One warp per column.
__global__ void colnorm_kernel(const double* H, int64_t ldh, int n, int gm, int gpad, int sign_test, double* sig) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double* col = H + int64_t(warp) * ldh;
    double s2 = 0.0, dot = 0.0;
    for (int r = lane; r < gm; r += 32) {
        const double gv = col[r];
        s2 += gv * gv;
        if (sign_test) dot += gv * col[gpad + r];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        dot += __shfl_xor_sync(0xffffffffu, dot, o);
    }
    if (lane == 0) sig[warp] = (sign_test && !(dot > 0.0)) ? 0.0 : sqrt(s2);
}

// lambda_j = v_j . (P0 v_j): the Rayleigh quotients of the original P0 for
// the converged basis (Vc row j = v_j, Gt row j = (P0 v_j)^T).  One warp per j.
__global__ void rayleigh_kernel(const double* Vc, int64_t ldv, const double* Gt, int64_t ldg, int n, double* lam) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += Vc[int64_t(warp) * ldv + i] * Gt[int64_t(warp) * ldg + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) lam[warp] = s;
}

// Vt (n x n, ldv): row k = v_{perm[k]} (H's V part).
__global__ void gather_vt_kernel(const double* H, int64_t ldh, int gpad, int n, const int* perm, double* Vt,
                                 int64_t ldv) {
    const int64_t tot = int64_t(n) * n;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < tot; e += int64_t(gridDim.x) * blockDim.x) {
        const int k = int(e / n), i = int(e % n);
        Vt[int64_t(k) * ldv + i] = H[int64_t(perm[k]) * ldh + gpad + i];
    }
}

// U (m x k, ldu) column k = g_{perm[k]} / sigma_k from the one-sided panel
// store (H row j = column j of G), transposed through 32 x 32 shared tiles.
__global__ void gather_u_kernel(const double* H, int64_t ldh, int m, int k, const int* perm, const double* inv,
                                double* U, int64_t ldu) {
    __shared__ double tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int k0 = blockIdx.y * 32; k0 < k; k0 += gridDim.y * 32)
        for (int i0 = blockIdx.x * 32; i0 < m; i0 += gridDim.x * 32) {
            for (int r = ty; r < 32; r += 8) {
                const int kk = k0 + r, i = i0 + tx;
                tile[r][tx] = (kk < k && i < m) ? H[int64_t(perm[kk]) * ldh + i] * inv[kk] : 0.0;
            }
            __syncthreads();
            for (int r = ty; r < 32; r += 8) {
                const int i = i0 + r, kk = k0 + tx;
                if (i < m && kk < k) U[int64_t(i) * ldu + kk] = tile[tx][r];
            }
            __syncthreads();
        }
}

// G (n x n, UᵀU) -> F = strictly upper part of G plus half of diag(G) - I/2,
// so that F + F^T = G - I.  U <- U (I - F) is then Gram-Schmidt to first
// order: column j only takes out columns i < j (larger singular values), and
// the departure G - I squares at every step.
__global__ void gs_factor_kernel(int n, double* G, int64_t ld) {
    const int64_t tot = int64_t(n) * n;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < tot; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = e / n, j = e % n;
        double& g = G[i * ld + j];
        g = i < j ? g : (i == j ? 0.5 * (g - 1.0) : 0.0);
    }
}

// X <- X - Y on the m x n part (leading dimension ld).
__global__ void sub_kernel(int m, int n, double* X, const double* Y, int64_t ld) {
    const int64_t tot = int64_t(m) * n;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < tot; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = e / n, j = e % n;
        X[i * ld + j] -= Y[i * ld + j];
    }
}

__global__ void frob2_part_kernel(int m, int n, const double* A, int64_t lda, double* part) {
    __shared__ double red[256];
    double s = 0.0;
    const int64_t tot = int64_t(m) * n;
    for (int64_t e = blockIdx.x * int64_t(256) + threadIdx.x; e < tot; e += int64_t(gridDim.x) * 256) {
        const double v = A[(e / n) * lda + e % n];
        s += v * v;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Sum of squares of (X - I) over an n x n matrix (ld), or of X - Y over m x n
// (Y != nullptr, ldy), per block.
__global__ void diff2_kernel(int m, int n, const double* X, int64_t ldx, const double* Y, int64_t ldy,
                             double* part) {
    __shared__ double red[256];
    double s = 0.0;
    const int64_t tot = int64_t(m) * n;
    for (int64_t e = blockIdx.x * int64_t(256) + threadIdx.x; e < tot; e += int64_t(gridDim.x) * 256) {
        const int64_t i = e / n, j = e % n;
        const double d = X[i * ldx + j] - (Y ? Y[i * ldy + j] : (i == j ? 1.0 : 0.0));
        s += d * d;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// X (m x n, ldx) columns scaled by s (U diag(S)).
__global__ void scale_cols_kernel(int m, int n, const double* X, int64_t ldx, const double* s, double* Y,
                                  int64_t ldy) {
    const int64_t tot = int64_t(m) * n;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < tot; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = e / n, j = e % n;
        Y[i * ldy + j] = X[i * ldx + j] * s[j];
    }
}

__global__ void sum_parts_kernel(int count, const double* part, double* out) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += 256) s += part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// out (cols x rows, ldo) = in (rows x cols, ldi)^T through 32 x 32 shared tiles.
__global__ void transpose_kernel(int rows, int cols, const double* in, int64_t ldi, double* out, int64_t ldo) {
    __shared__ double tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int r0 = blockIdx.y * 32; r0 < rows; r0 += gridDim.y * 32)
        for (int c0 = blockIdx.x * 32; c0 < cols; c0 += gridDim.x * 32) {
            for (int k = ty; k < 32; k += 8) {
                const int r = r0 + k, c = c0 + tx;
                tile[k][tx] = (r < rows && c < cols) ? in[int64_t(r) * ldi + c] : 0.0;
            }
            __syncthreads();
            for (int k = ty; k < 32; k += 8) {
                const int c = c0 + k, r = r0 + tx;
                if (c < cols && r < rows) out[int64_t(c) * ldo + r] = tile[tx][k];
            }
            __syncthreads();
        }
}

constexpr int kApplySmem = 3 * PW * XLD * 8;  // R + two stages: 104448 bytes
constexpr int kGramSmem = 3 * PW * GLD * 8;   // three stages: 55296 bytes
constexpr int kSolve2Smem = PW * MLD * 8;  // M: 33280 bytes (solve_kernel, solve2_kernel)
constexpr int kTwoSmem = 3 * PW * XLD * 8;    // P_ab / T, R_a, R_b: 104448 bytes

struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    EventTimer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~EventTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    void start(cudaStream_t s) { cudaEventRecord(a, s); }
    void stop(cudaStream_t s) { cudaEventRecord(b, s); }
    double ms() {
        float t = 0.f;
        return cudaEventElapsedTime(&t, a, b) == cudaSuccess ? double(t) : 0.0;
    }
};

}  // namespace

// Blocked one-sided Jacobi on H = [G; V] (see the file comment).  H: npad
// columns of ldh doubles (G rows [0, gm), zero rows up to gpad, V rows
// [gpad, gpad + npad)).  Returns the completed sweeps, rotations and the last
// sweep's largest relative off-diagonal through the out-parameters.
static lsvd_status run_sweeps(lsvd_context* ctx, double* H, int64_t ldh, int gm, int gpad, int npad, double tol,
                              double tol_conv, double scale2, int max_sweeps, int inner_max, char* ws,
                              int* sweeps_out, int64_t* rot_out, double* off_out, int* inner_cap_out,
                              double* ms_out) {
    LSVD_TRACE("large/jacobi_one_sided");
    cudaStream_t st = ctx->stream;
    const int nb = npad / BW;
    const int npairs = nb / 2;
    const int sms = ctx->num_sms;
    int nchunk = std::max(1, std::min(gpad / 64, (3 * sms + npairs - 1) / npairs));
    int kchunk = ((gpad / 64 + nchunk - 1) / nchunk) * 64;
    nchunk = (gpad + kchunk - 1) / kchunk;
    int napply = std::max(1, (4 * sms + npairs - 1) / npairs);
    int rows = int(((ldh / 64 + napply - 1) / napply) * 64);
    napply = int((ldh + rows - 1) / rows);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    char* p = ws;
    SweepState* stt = reinterpret_cast<SweepState*>(p); p += al(sizeof(SweepState));
    int* skip = reinterpret_cast<int*>(p); p += al(size_t(npairs) * 4);
    double* Rg = reinterpret_cast<double*>(p); p += al(size_t(npairs) * PW * PW * 8);
    double* Mpart = reinterpret_cast<double*>(p);
    SweepState init;
    std::memset(&init, 0, sizeof(init));
    init.scale2 = scale2;
    SweepState* hinit = static_cast<SweepState*>(lsvd_ctx_pinned(ctx, 2 * sizeof(SweepState)));
    if (!hinit) return lsvd_ctx_fail(ctx, LSVD_OUT_OF_MEMORY, "large: pinned state");
    *hinit = init;
    cudaError_t e = cudaMemcpyAsync(stt, hinit, sizeof(SweepState), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // hinit is reused for the sweep reads below
    if (e == cudaSuccess) e = cudaFuncSetAttribute(apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kApplySmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGramSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolve2Smem);
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "large: sweep setup");
    // one sweep = nb - 1 layers of (gram, solve, apply) + the sweep-end test, captured once
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "large: begin capture");
    for (int layer = 0; layer < nb - 1; ++layer) {
        gram_kernel<<<dim3(npairs, nchunk), 256, kGramSmem, st>>>(H, ldh, nb, layer, kchunk, gpad, Mpart, stt);
        solve_kernel<<<npairs, 1024, kSolve2Smem, st>>>(Mpart, nchunk, layer, Rg, skip, stt, tol, inner_max);
        apply_kernel<<<dim3(npairs, napply), 256, kApplySmem, st>>>(H, ldh, nb, layer, rows, Rg, skip, stt);
    }
    sweep_end_kernel<<<1, 1, 0, st>>>(stt, tol_conv);
    cudaError_t e2 = cudaGetLastError();
    e = cudaStreamEndCapture(st, &graph);
    if (e2 != cudaSuccess || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return lsvd_ctx_cuda(ctx, e2 != cudaSuccess ? e2 : e, "large: sweep capture");
    }
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "large: graph instantiate");
    const int launches_per_sweep = 3 * (nb - 1) + 1;
    // The host runs one sweep ahead of the flag it reads: sweep k+1 is queued
    // before sweep k's state (copied into pinned memory after sweep k) is
    // examined; once the flag is set, a queued sweep's kernels return at once.
    SweepState* hst = static_cast<SweepState*>(lsvd_ctx_pinned(ctx, 2 * sizeof(SweepState)));
    cudaEvent_t ev[2] = {nullptr, nullptr};
    lsvd_status out = LSVD_OK;
    if (!hst) out = lsvd_ctx_fail(ctx, LSVD_OUT_OF_MEMORY, "large: pinned state");
    for (int i = 0; i < 2 && out == LSVD_OK; ++i)
        if ((e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming)) != cudaSuccess)
            out = lsvd_ctx_cuda(ctx, e, "large: events");
    EventTimer tm;
    tm.start(st);
    int launched = 0;
    while (out == LSVD_OK && launched < max_sweeps) {
        const int k = launched;
        if ((e = cudaGraphLaunch(exec, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(&hst[k & 1], stt, sizeof(SweepState), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaEventRecord(ev[k & 1], st)) != cudaSuccess) {
            out = lsvd_ctx_cuda(ctx, e, "large: sweep launch");
            break;
        }
        ++launched;
        ctx->launches += launches_per_sweep;
        if (k >= 1) {
            if ((e = cudaEventSynchronize(ev[(k - 1) & 1])) != cudaSuccess) {
                out = lsvd_ctx_cuda(ctx, e, "large: sweep sync");
                break;
            }
            if (hst[(k - 1) & 1].converged) break;
        }
    }
    tm.stop(st);
    SweepState hs;
    std::memset(&hs, 0, sizeof(hs));
    if (out == LSVD_OK) {
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
            out = lsvd_ctx_cuda(ctx, e, "large: sweep state");
        else
            hs = hst[(launched - 1) & 1];
    }
    for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    cudaGraphExecDestroy(exec);
    if (out != LSVD_OK) return out;
    *sweeps_out = hs.sweeps;
    *rot_out = hs.rotations;
    *off_out = hs.last_off;
    *inner_cap_out = hs.inner_cap;
    *ms_out = tm.ms();
    return hs.converged ? LSVD_OK : LSVD_NOT_CONVERGED;
}

// Blocked two-sided Jacobi on the symmetric P (npad x npad, row-major, padding
// zero) accumulating V into Vc (row j = v_j; I on entry): per sweep the
// reference's start-of-sweep test off(P) < limit (offnorm_part_kernel, offnorm_final_kernel), then for
// every round-robin layer the block solves (solve2_kernel), P <- R^T P R
// (twoside_kernel) and V <- V R (apply_kernel on Vc).
// Host twin of block_pair.
static void block_pair_host(int nb, int layer, int k, int& a, int& b) {
    const int ring = nb - 1;
    if (k == 0) {
        a = nb - 1;
        b = layer % ring;
    } else {
        a = (layer + k) % ring;
        b = (layer + ring - k) % ring;
    }
}

// The twoside tiles (a <= b, a * 65536 + b) of every layer of a sweep, split
// for the next layer's solves: first the n1[L] tiles that hold the next
// layer's diagonal block-pair blocks -- tile (x, x) and (y, y) and the one
// between them, x, y the layer-L pairs of the next pair's two blocks -- then
// the rest, which can run beside the next layer's solves.  The last layer of
// a sweep has no next layer in the sweep: all its tiles come first.
static void twoside_tiles(int nb, std::vector<int>& tiles, std::vector<int>& n1) {
    const int npairs = nb / 2, ntri = npairs * (npairs + 1) / 2, layers = nb - 1;
    tiles.assign(size_t(layers) * ntri, 0);
    n1.assign(size_t(layers), ntri);
    std::vector<int> pof(size_t(nb), 0);
    std::vector<char> need(size_t(npairs) * npairs);
    for (int L = 0; L < layers; ++L) {
        for (int k = 0; k < npairs; ++k) {
            int a, b;
            block_pair_host(nb, L, k, a, b);
            pof[size_t(a)] = pof[size_t(b)] = k;
        }
        std::fill(need.begin(), need.end(), char(L + 1 == layers));
        if (L + 1 < layers)
            for (int k = 0; k < npairs; ++k) {
                int a, b;
                block_pair_host(nb, L + 1, k, a, b);
                const int x = pof[size_t(a)], y = pof[size_t(b)];
                need[size_t(x) * npairs + x] = need[size_t(y) * npairs + y] = 1;
                need[size_t(std::min(x, y)) * npairs + std::max(x, y)] = 1;
            }
        int* t = tiles.data() + size_t(L) * ntri;
        int c = 0;
        for (int pass = 0; pass < 2; ++pass)
            for (int a = 0; a < npairs; ++a)
                for (int b = a; b < npairs; ++b)
                    if ((need[size_t(a) * npairs + b] != 0) == (pass == 0)) t[c++] = a * 65536 + b;
        int first = 0;
        for (int a = 0; a < npairs; ++a)
            for (int b = a; b < npairs; ++b) first += need[size_t(a) * npairs + b] != 0;
        n1[size_t(L)] = first;
    }
}

static lsvd_status run_sweeps2(lsvd_context* ctx, double* P, double* Vc, int n, int npad, double limit, double tau,
                               int max_sweeps, int inner_max, char* ws, int* sweeps_out, int64_t* rot_out,
                               double* off_out, int* inner_cap_out, double* ms_out) {
    LSVD_TRACE("large/jacobi_two_sided");
    cudaStream_t st = ctx->stream;
    const int nb = npad / BW;
    const int npairs = nb / 2;
    const int ntri = npairs * (npairs + 1) / 2;
    const int sms = ctx->num_sms;
    int napply = std::max(1, (4 * sms + npairs - 1) / npairs);
    int rows = ((npad / 64 + napply - 1) / napply) * 64;
    napply = (npad + rows - 1) / rows;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    char* p = ws;
    SweepState* stt = reinterpret_cast<SweepState*>(p); p += al(sizeof(SweepState));
    // rotations and skip flags double-buffered by layer parity: V's update of
    // layer L runs on a side branch of the graph while the next layer solves
    int* skip2[2];
    double* Rg2[2];
    skip2[0] = reinterpret_cast<int*>(p); p += al(size_t(npairs) * 4);
    skip2[1] = reinterpret_cast<int*>(p); p += al(size_t(npairs) * 4);
    Rg2[0] = reinterpret_cast<double*>(p); p += al(size_t(npairs) * PW * PW * 8);
    Rg2[1] = reinterpret_cast<double*>(p); p += al(size_t(npairs) * PW * PW * 8);
    double* offpart = reinterpret_cast<double*>(p);  // 256 partial sums of the off-norm test
    p += al(256 * 8);
    // twoside's tile lists per layer
    int* tiles_d = reinterpret_cast<int*>(p);
    std::vector<int> tiles_h, n1;
    twoside_tiles(nb, tiles_h, n1);
    cudaError_t e = cudaMemcpy(tiles_d, tiles_h.data(), tiles_h.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemsetAsync(stt, 0, sizeof(SweepState), st);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kApplySmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(solve2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolve2Smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(twoside_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTwoSmem);
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "large: sweep setup");
    if (!ctx->side_stream && (e = cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "large: side stream");
    if (!ctx->side_stream2 && (e = cudaStreamCreateWithFlags(&ctx->side_stream2, cudaStreamNonBlocking)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "large: side stream");
    cudaStream_t sv = ctx->side_stream, s2 = ctx->side_stream2;
    cudaEvent_t evs[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // solved, join, applied[2], rest done
    for (auto& x : evs)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
    auto destroy_events = [&]() {
        for (auto& x : evs)
            if (x) cudaEventDestroy(x);
    };
    if (e != cudaSuccess) {
        destroy_events();
        return lsvd_ctx_cuda(ctx, e, "large: capture events");
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
        destroy_events();
        return lsvd_ctx_cuda(ctx, e, "large: begin capture");
    }
    offnorm_part_kernel<<<256, 256, 0, st>>>(P, npad, n, stt, offpart);
    offnorm_final_kernel<<<1, 256, 0, st>>>(offpart, 256, stt, limit);
    // Per layer L: solve2(L); V <- V R on sv; P <- R^T P R split in two: the tiles the
    // next layer's solves read, on st, and the rest on s2, beside solve2(L + 1).  The
    // rest of layer L - 1 finishes before any tile of layer L starts (a tile of L
    // reads blocks that tiles of L - 1 wrote); R / skip of parity b are rewritten by
    // solve2(L + 2) only after V's update of L (applied[b]) and the rest of L (which
    // precedes the first part of L + 1 on st).
    bool rest_pending = false;  // the previous layer left tiles on s2
    for (int layer = 0; layer < nb - 1; ++layer) {
        const int b = layer & 1;
        const int* tl = tiles_d + size_t(layer) * ntri;
        const int k1 = n1[size_t(layer)];
        if (layer >= 2) cudaStreamWaitEvent(st, evs[2 + b], 0);
        solve2_kernel<<<npairs, 1024, kSolve2Smem, st>>>(P, npad, nb, layer, Rg2[b], skip2[b], stt, tau, inner_max);
        cudaEventRecord(evs[0], st);
        cudaStreamWaitEvent(sv, evs[0], 0);
        apply_kernel<<<dim3(npairs, napply), 256, kApplySmem, sv>>>(Vc, npad, nb, layer, rows, Rg2[b], skip2[b], stt);
        cudaEventRecord(evs[2 + b], sv);
        if (rest_pending) cudaStreamWaitEvent(st, evs[4], 0);  // the rest of layer - 1
        twoside_kernel<<<k1, 256, kTwoSmem, st>>>(P, npad, nb, layer, Rg2[b], skip2[b], stt, tl);
        rest_pending = k1 < ntri;
        if (rest_pending) {
            cudaStreamWaitEvent(s2, evs[0], 0);
            twoside_kernel<<<ntri - k1, 256, kTwoSmem, s2>>>(P, npad, nb, layer, Rg2[b], skip2[b], stt, tl + k1);
            cudaEventRecord(evs[4], s2);
        }
    }
    if (rest_pending) cudaStreamWaitEvent(st, evs[4], 0);
    cudaEventRecord(evs[1], sv);
    cudaStreamWaitEvent(st, evs[1], 0);
    sweep_end_kernel<<<1, 1, 0, st>>>(stt, -1.0);
    cudaError_t e2 = cudaGetLastError();
    e = cudaStreamEndCapture(st, &graph);
    destroy_events();
    if (e2 != cudaSuccess || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return lsvd_ctx_cuda(ctx, e2 != cudaSuccess ? e2 : e, "large: sweep capture");
    }
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "large: graph instantiate");
    int launches_per_sweep = 3;  // off-norm test, its final step, sweep end
    for (int L = 0; L < nb - 1; ++L) launches_per_sweep += 3 + (n1[size_t(L)] < ntri ? 1 : 0);
    SweepState* hst = static_cast<SweepState*>(lsvd_ctx_pinned(ctx, 2 * sizeof(SweepState)));
    cudaEvent_t ev[2] = {nullptr, nullptr};
    lsvd_status out = LSVD_OK;
    if (!hst) out = lsvd_ctx_fail(ctx, LSVD_OUT_OF_MEMORY, "large: pinned state");
    for (int i = 0; i < 2 && out == LSVD_OK; ++i)
        if ((e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming)) != cudaSuccess)
            out = lsvd_ctx_cuda(ctx, e, "large: events");
    EventTimer tm;
    tm.start(st);
    int launched = 0;
    // one sweep ahead of the flag the host reads (see run_sweeps)
    while (out == LSVD_OK && launched < max_sweeps + 1) {
        const int k = launched;
        if ((e = cudaGraphLaunch(exec, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(&hst[k & 1], stt, sizeof(SweepState), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaEventRecord(ev[k & 1], st)) != cudaSuccess) {
            out = lsvd_ctx_cuda(ctx, e, "large: sweep launch");
            break;
        }
        ++launched;
        ctx->launches += launches_per_sweep;
        if (k >= 1) {
            if ((e = cudaEventSynchronize(ev[(k - 1) & 1])) != cudaSuccess) {
                out = lsvd_ctx_cuda(ctx, e, "large: sweep sync");
                break;
            }
            if (hst[(k - 1) & 1].converged) break;
        }
    }
    tm.stop(st);
    SweepState hs;
    std::memset(&hs, 0, sizeof(hs));
    if (out == LSVD_OK) {
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
            out = lsvd_ctx_cuda(ctx, e, "large: sweep state");
        else
            hs = hst[(launched - 1) & 1];
    }
    for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    cudaGraphExecDestroy(exec);
    if (out != LSVD_OK) return out;
    *sweeps_out = hs.sweeps;
    *rot_out = int64_t(hs.rotations);
    *off_out = hs.last_off;
    *inner_cap_out = hs.inner_cap;
    *ms_out = tm.ms();
    return hs.converged ? LSVD_OK : LSVD_NOT_CONVERGED;
}

static size_t sweep_ws_bytes(int gpad, int npad, int num_sms) {
    const int nb = npad / BW, npairs = nb / 2;
    const int nchunk = std::max(1, std::min(gpad / 64, (3 * num_sms + npairs - 1) / npairs));
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    // state | skip x 2 | rotations x 2 | Gram partials (the two-sided route uses the second
    // skip and rotation buffers, the one-sided route the partials)
    // | twoside's tile lists per layer (the two-sided route)
    const size_t ntri = size_t(npairs) * (npairs + 1) / 2;
    return al(sizeof(SweepState)) + 2 * al(size_t(npairs) * 4) + 2 * al(size_t(npairs) * PW * PW * 8) +
           al(256 * 8) + al(size_t(npairs) * (nchunk + 1) * PW * PW * 8) + al(size_t(nb - 1) * ntri * 4);
}

static lsvd_status large_impl(lsvd_context* ctx, int64_t m, int64_t n, const double* A, int64_t lda,
                              bool transpose_in, double* U, int64_t ldu, double* S, double* Vt, int64_t ldvt,
                              lsvd_precision precision, lsvd_large_info* info, lsvd_diag* diag, bool want_diag) {
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    const int64_t ld = (n + 7) & ~int64_t(7);
    const int gpad = int((n + 63) & ~int64_t(63));  // G = P is n x n on this route
    const int npad = gpad;
    const int64_t ldh = int64_t(gpad) + npad;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t b_a = al(size_t(m) * ld * 8), b_p = al(size_t(ld) * ld * 8), b_h = al(size_t(npad) * ldh * 8);
    const size_t b_u = al(size_t(m) * ld * 8), b_v = al(size_t(ld) * ld * 8);
    const size_t b_misc = al(4096 * 8 + 64) + al(size_t(n) * 8) * 2 + al(size_t(n) * 4);
    const bool lowp = precision == LSVD_PREC_MIXED_TF32 || precision == LSVD_PREC_MIXED_BF16;
    // mixed route: the one-sided panel store [W; V] with W = A V0 (m rows)
    const int gpadm = int((m + 63) & ~int64_t(63));
    const int64_t ldh1 = int64_t(gpadm) + npad;
    const size_t b_h1 = lowp ? al(size_t(npad) * ldh1 * 8) : 0;
    const size_t b_sw = sweep_ws_bytes(std::max(gpad, lowp ? gpadm : 0), npad, ctx->num_sms);
    char* ws = static_cast<char*>(ctx->ws_large.get(b_a + b_p + b_h + b_u + b_v + b_misc + b_h1 + b_sw, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "large: workspace");
    char* p = ws;
    double* A64 = reinterpret_cast<double*>(p); p += b_a;
    double* Pm = reinterpret_cast<double*>(p); p += b_p;
    double* H = reinterpret_cast<double*>(p); p += b_h;
    double* Ud = reinterpret_cast<double*>(p); p += b_u;
    double* Vd = reinterpret_cast<double*>(p); p += b_v;
    double* part = reinterpret_cast<double*>(p);
    double* dsum = part + 4096;
    p += al(4096 * 8 + 64);
    double* sig = reinterpret_cast<double*>(p); p += al(size_t(n) * 8);
    double* sig2 = reinterpret_cast<double*>(p); p += al(size_t(n) * 8);
    int* perm_d = reinterpret_cast<int*>(p); p += al(size_t(n) * 4);
    double* H1 = lowp ? reinterpret_cast<double*>(p) : nullptr;
    p += b_h1;
    char* sw = p;
    // A (m x n) into A64 with an even leading dimension (transposed input: A is n x m)
    if ((e = cudaMemsetAsync(A64, 0, size_t(m) * ld * 8, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "large: clear A");
    if (!transpose_in) {
        e = cudaMemcpy2DAsync(A64, size_t(ld) * 8, A, size_t(lda) * 8, size_t(n) * 8, size_t(m), cudaMemcpyDefault, st);
    } else {
        // A given as n x m (lda): stage it in Ud (n x ldm), then transpose on the device
        const int64_t ldm = (m + 7) & ~int64_t(7);
        e = cudaMemcpy2DAsync(Ud, size_t(ldm) * 8, A, size_t(lda) * 8, size_t(m) * 8, size_t(n), cudaMemcpyDefault, st);
        if (e == cudaSuccess) {
            transpose_kernel<<<dim3(32, 32), 256, 0, st>>>(int(n), int(m), Ud, ldm, A64, ld);
            e = cudaGetLastError();
            ctx->launches += 1;
        }
    }
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "large: copy A");
    frob2_part_kernel<<<1024, 256, 0, st>>>(int(m), int(n), A64, ld, part);
    sum_parts_kernel<<<1, 256, 0, st>>>(1024, part, dsum);
    double f2 = 0.0;
    if ((e = cudaMemcpyAsync(&f2, dsum, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "large: norm");
    if (!std::isfinite(f2)) return lsvd_ctx_fail(ctx, LSVD_NONFINITE_INPUT, "large: non-finite input");
    lsvd_large_info li;
    std::memset(&li, 0, sizeof(li));
    EventTimer total;
    total.start(st);
    int32_t mflags = 0;
    // 1. polar factor Q (m x n, ldq)
    lsvd_polar_info pinfo;
    std::memset(&pinfo, 0, sizeof(pinfo));
    double* X = nullptr;
    int64_t ldx = 0;
    EventTimer tpol;
    tpol.start(st);
    lsvd_status pst = LSVD_OK;
    if (f2 > 0.0) {
        // FP64: the reference's iteration to delta < 1e-13 sqrt(n).  Mixed: the
        // TF32/BF16 tensor-core bulk only (no FP64 iterations): its factor Q0
        // preconditions the eigensolve below and accuracy comes from the FP64
        // cleanup on A itself.
        LSVD_TRACE("large/polar");
        pst = lsvd_polar_run(ctx, m, n, A64, ld, lowp ? precision : LSVD_PREC_FP64, lowp ? 0 : 120, &X, &ldx,
                             &pinfo);
        if (pst != LSVD_OK && pst != LSVD_NOT_CONVERGED) return pst;
        if (lowp) pst = LSVD_OK;
    }
    tpol.stop(st);
    if (pst == LSVD_NOT_CONVERGED) mflags |= LSVD_MAT_NS_CAP;
    if (!lowp && f2 > 0.0 && pinfo.orth > 1e-8 * std::sqrt(double(n))) mflags |= LSVD_MAT_POLAR_UNTRUSTED;
    li.ns_iters_fp64 = pinfo.iters_fp64;
    li.ns_iters_lowp = pinfo.iters_lowp;
    li.flops_fp64 += pinfo.flops_fp64;
    li.flops_lowp += pinfo.flops_lowp;
    // scale G so that ||P||_F = ||A||_F is near 1 (a power of two: exact)
    const double scale = f2 > 0.0 ? std::ldexp(1.0, -std::ilogb(std::sqrt(f2))) : 1.0;
    int sweeps = 0, inner_cap = 0;
    int64_t rots = 0;
    double off = 0.0, ms_eig = 0.0;
    lsvd_status jst = LSVD_OK;
    double* P2 = H;                       // npad x npad, row-major (the H slot holds both)
    double* Vc = H + size_t(npad) * npad;  // npad x npad, row j = v_j
    if (f2 > 0.0) {
        // 2. P = Q^T A (n x n); P2 = scale sym(P), Vc = I
        if ((e = lsvd::dg::dgemm(st, true, false, int(n), int(n), int(m), 1.0, X, ldx, A64, ld, 0.0, Pm, ld)) !=
            cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "large: P = Q^T A");
        li.flops_fp64 += 2.0 * double(m) * double(n) * double(n);
        fill_p2v_kernel<<<2048, 256, 0, st>>>(Pm, ld, int(n), scale, P2, Vc, npad);
        frob2_part_kernel<<<1024, 256, 0, st>>>(int(n), int(n), P2, npad, part);
        sum_parts_kernel<<<1, 256, 0, st>>>(1024, part, dsum);
        ctx->launches += 4;
        double p2 = 0.0;
        if ((e = cudaMemcpyAsync(&p2, dsum, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "large: ||P||");
        // 3. eigenvectors of P by blocked two-sided Jacobi: the reference's
        //    stop test off(P) < 1e-13 ||P||_F at every sweep start
        //    (src/lie_svd_small.rs:216-228); rotations of |a_pq| above the
        //    rounding level eps ||P||_F / sqrt(n) of the entries
        const double refn = std::max(std::sqrt(p2), 1e-300);
        const double tau = 2.220446049250313e-16 * refn / std::sqrt(double(npad));
        // mixed: P0 = Q0^T A is accurate to ~u_lo ||A|| only, so its eigensolve
        // stops at off(P0) < 4 u_lo ||P0||_F (TF32 u = 2^-11, BF16 2^-8)
        const double stop = lowp ? 4.0 * (precision == LSVD_PREC_MIXED_BF16 ? 3.90625e-3 : 4.8828125e-4) : 1e-13;
        // one inner Jacobi sweep per block solve: a full diagonalisation of
        // every 64 x 64 block saves about one outer sweep but costs eight
        jst = run_sweeps2(ctx, P2, Vc, int(n), npad, stop * refn, tau, 40, 1, sw, &sweeps, &rots, &off,
                          &inner_cap, &ms_eig);
        if (jst != LSVD_OK && jst != LSVD_NOT_CONVERGED) return jst;
        if (jst == LSVD_NOT_CONVERGED) mflags |= LSVD_MAT_JACOBI_CAP;
        off /= scale;
        // per sweep and layer: R_a^T P_ab R_b over the block-pair triangle, and V R
        const double np2 = double(npad / PW);
        li.flops_fp64 += double(sweeps) * double(npad / BW - 1) *
                         (np2 * (np2 + 1) / 2 * 4.0 * PW * PW * PW + np2 * 2.0 * PW * PW * npad);
        if (!lowp) {
            // 4. eigenvalues: Rayleigh quotients of the original P for the converged basis
            if ((e = lsvd::dg::dgemm(st, false, true, int(n), int(n), int(n), 1.0, Vc, npad, Pm, ld, 0.0, Ud,
                                     ld)) != cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: P V");
            li.flops_fp64 += 2.0 * double(n) * double(n) * double(n);
            rayleigh_kernel<<<(int(n) * 32 + 255) / 256, 256, 0, st>>>(Vc, npad, Ud, ld, int(n), sig);
            ctx->launches += 2;
        } else {
            // 4'. FP64 cleanup on A itself: W = A V0, then blocked one-sided Jacobi on
            //     the panel store [W; V0] until the columns of W are orthogonal (the
            //     normwise-scaled test of solve_kernel); sigma_j = ||w_j||, U = W / sigma
            li.sweeps_lowp = sweeps;
            li.ms_eig_lowp = ms_eig;
            if ((e = lsvd::dg::dgemm(st, false, true, int(m), int(n), int(n), 1.0, A64, ld, Vc, npad, 0.0, Ud,
                                     ld)) != cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: W = A V0");
            li.flops_fp64 += 2.0 * double(m) * double(n) * double(n);
            if ((e = cudaMemsetAsync(H1, 0, size_t(npad) * ldh1 * 8, st)) != cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: clear H");
            transpose_kernel<<<dim3(64, 32), 256, 0, st>>>(int(m), int(n), Ud, ld, H1, ldh1);
            if ((e = cudaMemcpy2DAsync(H1 + gpadm, size_t(ldh1) * 8, Vc, size_t(npad) * 8, size_t(npad) * 8,
                                       size_t(npad), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: V0 into H");
            colnorm_kernel<<<(int(n) * 32 + 255) / 256, 256, 0, st>>>(H1, ldh1, int(n), int(m), gpadm, 0, sig);
            ctx->launches += 3;
            std::vector<double> c0(static_cast<size_t>(n));
            if ((e = cudaMemcpyAsync(c0.data(), sig, size_t(n) * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                (e = cudaStreamSynchronize(st)) != cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: column norms");
            double s2 = 0.0;
            for (double v : c0) s2 = std::max(s2, v * v);
            const double tol1 = std::max(1e-14, 8.0 * 2.220446049250313e-16 * std::sqrt(double(gpadm)));
            int sw1 = 0, cap1 = 0;
            int64_t rot1 = 0;
            double off1 = 0.0, ms1 = 0.0;
            jst = run_sweeps(ctx, H1, ldh1, int(m), gpadm, npad, tol1, 1e-10, s2, 40, 2, sw, &sw1, &rot1, &off1,
                             &cap1, &ms1);
            if (jst != LSVD_OK && jst != LSVD_NOT_CONVERGED) return jst;
            if (jst == LSVD_NOT_CONVERGED) mflags |= LSVD_MAT_JACOBI_CAP;
            sweeps = sw1;
            rots += rot1;
            off = off1;
            inner_cap += cap1;
            ms_eig = ms1;
            // per sweep and layer: Gram over gpadm rows and the apply over ldh1 rows, per block pair
            li.flops_fp64 += double(sw1) * double(npad / BW - 1) * double(npad / PW) * 2.0 * PW * PW *
                             double(gpadm + ldh1);
            colnorm_kernel<<<(int(n) * 32 + 255) / 256, 256, 0, st>>>(H1, ldh1, int(n), int(m), gpadm, 0, sig);
            ctx->launches += 1;
        }
    } else {
        // A = 0: sigma = 0, V = I, U = the first n columns of I (MGS fill of zero seeds)
        fill_p2v_kernel<<<2048, 256, 0, st>>>(Pm, ld, 0, 0.0, P2, Vc, npad);
        if ((e = cudaMemsetAsync(sig, 0, size_t(n) * 8, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "large: zero sigma");
        ctx->launches += 1;
    }
    // sigma = max(lambda, 0) in descending eigenvalue order (src/lie_svd_small.rs:270-284, :311)
    std::vector<double> hs(static_cast<size_t>(n));
    if ((e = cudaMemcpyAsync(hs.data(), sig, size_t(n) * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "large: sigma");
    std::vector<int> perm(static_cast<size_t>(n));
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return hs[a] > hs[b]; });
    std::vector<double> hsorted(static_cast<size_t>(n));
    for (int64_t k = 0; k < n; ++k) hsorted[size_t(k)] = std::max(hs[size_t(perm[size_t(k)])], 0.0);
    if ((e = cudaMemcpyAsync(perm_d, perm.data(), size_t(n) * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "large: perm");
    if (lowp && f2 > 0.0) {
        // U = W / sigma and Vt from the one-sided panel store
        std::vector<double> inv(static_cast<size_t>(n));
        for (int64_t k = 0; k < n; ++k) {
            inv[size_t(k)] = hsorted[size_t(k)] > 0.0 ? 1.0 / hsorted[size_t(k)] : 0.0;
            if (!(hsorted[size_t(k)] > 0.0)) mflags |= LSVD_MAT_REPAIRED;  // zero column left zero
        }
        if ((e = cudaMemcpyAsync(sig2, inv.data(), size_t(n) * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "large: 1/sigma");
        gather_vt_kernel<<<2048, 256, 0, st>>>(H1, ldh1, gpadm, int(n), perm_d, Vd, ld);
        gather_u_kernel<<<dim3(64, 32), 256, 0, st>>>(H1, ldh1, int(m), int(n), perm_d, sig2, Ud, ld);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess)  // `inv` is pageable host memory
            return lsvd_ctx_cuda(ctx, e, "large: gather");
        // W's columns are orthogonal to the normwise scale only: columns with
        // sigma_j << sigma_1 keep cosines up to ~tol sigma_1 / sigma_j.  Gram-
        // Schmidt in descending sigma order (the order of the reference's MGS
        // repair, src/lie_svd_small.rs:82-144) restores orthonormal columns and
        // moves column j by at most its cosines with larger columns, i.e. the
        // product U S V^T by ~tol sigma_1: U <- U (I - F), F the upper half of
        // U^T U - I, until ||U^T U - I|| reaches rounding.  X (Q0, no longer
        // needed) holds U F.
        for (int it = 0; it < 8; ++it) {
            if ((e = lsvd::dg::dgemm(st, true, false, int(n), int(n), int(m), 1.0, Ud, ld, Ud, ld, 0.0, Pm, ld)) !=
                cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: U^T U");
            diff2_kernel<<<1024, 256, 0, st>>>(int(n), int(n), Pm, ld, nullptr, 0, part);
            sum_parts_kernel<<<1, 256, 0, st>>>(1024, part, dsum);
            double o2 = 0.0;
            if ((e = cudaMemcpyAsync(&o2, dsum, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                (e = cudaStreamSynchronize(st)) != cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: U orthogonality");
            li.flops_fp64 += 2.0 * double(m) * double(n) * double(n);
            ctx->launches += 3;
            if (!(std::sqrt(o2) > 1e-14 * std::sqrt(double(n)))) break;
            gs_factor_kernel<<<2048, 256, 0, st>>>(int(n), Pm, ld);
            if ((e = lsvd::dg::dgemm(st, false, false, int(m), int(n), int(n), 1.0, Ud, ld, Pm, ld, 0.0, X, ld)) !=
                cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: U F");
            sub_kernel<<<2048, 256, 0, st>>>(int(m), int(n), Ud, X, ld);
            li.flops_fp64 += 2.0 * double(m) * double(n) * double(n);
            ctx->launches += 3;
        }
    } else {
        gather_vt_kernel<<<2048, 256, 0, st>>>(Vc, npad, 0, int(n), perm_d, Vd, ld);
    }
    if (f2 > 0.0 && !lowp) {
        if ((e = lsvd::dg::dgemm(st, false, true, int(m), int(n), int(n), 1.0, X, ldx, Vd, ld, 0.0, Ud, ld)) !=
            cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "large: U = Q V");
        li.flops_fp64 += 2.0 * double(m) * double(n) * double(n);
    } else if (f2 == 0.0) {
        std::vector<double> eye(size_t(m) * ld, 0.0);
        for (int64_t i = 0; i < n; ++i) eye[size_t(i) * ld + i] = 1.0;
        if ((e = cudaMemcpyAsync(Ud, eye.data(), eye.size() * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "large: U");
    }
    ctx->launches += 3;
    total.stop(st);
    // 5. outputs: the thin SVD of A, or of A^T for a transposed input (U and Vt swap roles)
    LSVD_TRACE("large/outputs");
    double* dS = sig;  // sorted sigma back to the device for the diagnostics
    if ((e = cudaMemcpyAsync(dS, hsorted.data(), size_t(n) * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "large: sorted sigma");
    if (want_diag || diag) {
        double o_u = 0.0, o_v = 0.0, rec = 0.0;
        auto norm2 = [&](double* out) -> cudaError_t {
            sum_parts_kernel<<<1, 256, 0, st>>>(1024, part, dsum);
            cudaError_t ee = cudaMemcpyAsync(out, dsum, 8, cudaMemcpyDeviceToHost, st);
            return ee == cudaSuccess ? cudaStreamSynchronize(st) : ee;
        };
        if (want_diag) {
            // ||U^T U - I||, ||Vt Vt^T - I||, ||U S Vt - A|| / ||A|| with the GEMMs of this file
            if ((e = lsvd::dg::dgemm(st, true, false, int(n), int(n), int(m), 1.0, Ud, ld, Ud, ld, 0.0, Pm, ld)) !=
                cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: diag");
            diff2_kernel<<<1024, 256, 0, st>>>(int(n), int(n), Pm, ld, nullptr, 0, part);
            if ((e = norm2(&o_u)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "large: diag");
            if ((e = lsvd::dg::dgemm(st, false, true, int(n), int(n), int(n), 1.0, Vd, ld, Vd, ld, 0.0, Pm, ld)) !=
                cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "large: diag");
            diff2_kernel<<<1024, 256, 0, st>>>(int(n), int(n), Pm, ld, nullptr, 0, part);
            if ((e = norm2(&o_v)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "large: diag");
            // U diag(S) in X's slot (Q is no longer needed once U = Q V is formed), then
            // A64 <- U S Vt - A64 and its sum of squares
            if (X) {
                scale_cols_kernel<<<2048, 256, 0, st>>>(int(m), int(n), Ud, ld, dS, X, ld);
                if ((e = lsvd::dg::dgemm(st, false, false, int(m), int(n), int(n), 1.0, X, ld, Vd, ld, -1.0, A64,
                                         ld)) != cudaSuccess)
                    return lsvd_ctx_cuda(ctx, e, "large: diag");
            }
            frob2_part_kernel<<<1024, 256, 0, st>>>(int(m), int(n), A64, ld, part);
            if ((e = norm2(&rec)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "large: diag");
            ctx->launches += 10;
            o_u = std::sqrt(o_u);
            o_v = std::sqrt(o_v);
            rec = f2 > 0.0 ? std::sqrt(rec / f2) : 0.0;
        }
        if (diag) {
            diag->rel_recon = rec;
            diag->orth_u = transpose_in ? o_v : o_u;
            diag->orth_v = transpose_in ? o_u : o_v;
            diag->ns_iters = pinfo.iters_fp64;
            diag->jacobi_sweeps = f2 > 0.0 ? sweeps + 1 : 0;  // + the sweep whose start test stopped the solve
            diag->rotations = rots;
            diag->flags = mflags;
            diag->route = LSVD_ROUTE_SMALL;
        }
    }
    if (!transpose_in) {
        if ((e = cudaMemcpy2DAsync(U, size_t(ldu) * 8, Ud, size_t(ld) * 8, size_t(n) * 8, size_t(m), cudaMemcpyDefault,
                                   st)) != cudaSuccess ||
            (e = cudaMemcpy2DAsync(Vt, size_t(ldvt) * 8, Vd, size_t(ld) * 8, size_t(n) * 8, size_t(n),
                                   cudaMemcpyDefault, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "large: copy out");
    } else {
        // A^T = U S Vt  =>  A = Vt^T S U^T: the caller's U (n x n) = Vd^T and Vt (n x m) = Ud^T,
        // transposed on the device into the free P and A64 slots
        const int64_t ldm = (m + 7) & ~int64_t(7);
        transpose_kernel<<<dim3(32, 32), 256, 0, st>>>(int(n), int(n), Vd, ld, Pm, ld);
        transpose_kernel<<<dim3(32, 32), 256, 0, st>>>(int(m), int(n), Ud, ld, A64, ldm);
        ctx->launches += 2;
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpy2DAsync(U, size_t(ldu) * 8, Pm, size_t(ld) * 8, size_t(n) * 8, size_t(n),
                                   cudaMemcpyDefault, st)) != cudaSuccess ||
            (e = cudaMemcpy2DAsync(Vt, size_t(ldvt) * 8, A64, size_t(ldm) * 8, size_t(m) * 8, size_t(n),
                                   cudaMemcpyDefault, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "large: copy out");
    }
    if ((e = cudaMemcpyAsync(S, hsorted.data(), size_t(n) * 8, cudaMemcpyDefault, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "large: copy S");
    li.sweeps_fp64 = sweeps;  // mixed: the FP64 cleanup sweeps
    li.rotations = rots;
    li.flags = mflags;
    li.last_offdiag = off;
    li.inner_cap_pairs = inner_cap;
    li.ms_polar = tpol.ms();
    li.ms_eig_fp64 = ms_eig;
    li.ms_total = total.ms();
    if (diag) {
        li.rel_recon = diag->rel_recon;
        li.orth_u = diag->orth_u;
        li.orth_v = diag->orth_v;
    }
    if (info) *info = li;
    if (jst == LSVD_NOT_CONVERGED || pst == LSVD_NOT_CONVERGED) return LSVD_NOT_CONVERGED;
    return LSVD_OK;
}

lsvd_status lsvd_large_solve(lsvd_context* ctx, int64_t rows, int64_t cols, const double* A, int64_t lda,
                             double* U, int64_t ldu, double* S, double* Vt, int64_t ldvt,
                             lsvd_precision precision, lsvd_large_info* info, lsvd_diag* diag, bool want_diag) {
    // wide inputs run on A^T (the reference transposes, src/lie_svd_small.rs:343-348)
    const bool tr = cols > rows;
    const int64_t m = tr ? cols : rows, n = tr ? rows : cols;
    return large_impl(ctx, m, n, A, lda, tr, U, ldu, S, Vt, ldvt, precision, info, diag, want_diag);
}

extern "C" lsvd_status lsvd_svd_large_f64(lsvd_context* ctx, int64_t m, int64_t n, const double* A, int64_t lda,
                                          double* U, int64_t ldu, double* S, double* Vt, int64_t ldvt,
                                          lsvd_precision precision, lsvd_large_info* info, uint32_t flags) {
    LSVD_TRACE("lsvd_svd_large_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (m < 1 || n < 1) return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "lsvd_svd_large_f64: empty matrix");
    const int64_t k = std::min(m, n);
    if (!A || !U || !S || !Vt || lda < n || ldu < k || ldvt < n)
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_svd_large_f64: bad pointer or leading dimension");
    if (std::max(m, n) > (int64_t(1) << 16) || k > 16384)
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "lsvd_svd_large_f64: larger than 65536 x 16384");
    if (precision != LSVD_PREC_FP64 && precision != LSVD_PREC_MIXED_TF32 && precision != LSVD_PREC_MIXED_BF16)
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_svd_large_f64: unknown precision");
    if (precision != LSVD_PREC_FP64 && (std::max(m, n) % 128 || std::min(m, n) % 128))
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "lsvd_svd_large_f64: TF32/BF16 need m, n multiples of 128");
    cudaSetDevice(ctx->device);
    lsvd_diag d;
    return lsvd_large_solve(ctx, m, n, A, lda, U, ldu, S, Vt, ldvt, precision, info, &d,
                            (flags & LSVD_WANT_DIAG) != 0);
}
