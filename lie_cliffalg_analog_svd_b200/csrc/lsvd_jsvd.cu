// lsvd_jsvd.cu -- two-sided joint SVD of families of rows x cols matrices,
// LieSvdJoint::joint_svd_with_params (src/lie_svd_joint.rs:170-261), batched
// over independent families and blocked like the Phase-JADE kernels.
//
// The reference sweeps the kk = min(rows, cols) leading indices in
// round-robin layers (layer_pairs, :524-539); for each pair (i, j) it
//   * skips it if sum_k |m_ij| + |m_ji| <= pair_tol                  (:195)
//   * takes left/right angles from the normalised 2 x 2 blocks
//     (joint_svd_pair_angles :264-277, pair_block_norm :279-282) and skips
//     |theta_l| + |theta_r| <= 1e-18                                  (:199)
//   * rotates rows i, j of every matrix by theta_l and columns by theta_r,
//     accepting if the local off-diagonal energy does not grow beyond
//     1e-14 max(before, 1), else halving both angles, line_search_steps
//     times (accept_joint_svd_rotor, :303-336); U takes the left rotation
//     on its columns, V the right one
// and stops when the joint off-diagonal norm is <= tol or stopped
// decreasing by 1e-10 (:226-229).
//
// Blocked on the GPU: blocks of 8 of the kk indices are paired by the circle
// method; for each block pair the K principal 16 x 16 sub-blocks are staged
// in shared memory (jsvd_solve_kernel), every index pair inside is treated by
// the rules above, and the accepted rotations compose into a left RL and a
// right RR (16 x 16 each).  jsvd_apply_kernel then streams every matrix in
// strips of 16 rows, M <- RL^T M RR (rows and columns past kk untouched by
// the respective side), and the bases U <- U RL, V <- V RR.  The rotations
// preserve the norms of rows i, j and columns i, j outside the 2 x 2 block,
// so the acceptance test uses the exact change of the block's off-diagonal
// energy; the slack uses the sub-block's local energy (decisions identical in
// exact arithmetic, up to that slack).  The pair order inside a sweep differs
// from the reference's, so parity is on the converged result.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "lsvd.h"
#include "lsvd_internal.h"
#include "lsvd_joint_common.cuh"

namespace {

using namespace lsvd::joint;

struct JsvdArgs {
    int F, K, rows, cols, kk, nbe;  // families, matrices, shape, min(rows, cols), blocks (even)
    int layer;
    int steps;                      // line_search_steps
    const double* pair_tol;         // per family
    double* W;                      // F*K*rows*cols
    double* U;                      // F*rows*rows
    double* V;                      // F*cols*cols
    double* RL;                     // F*(nbe/2)*B2*B2 (row-major)
    double* RR;
    long long* rot;                 // per family: accepted, rejected
    const int* active;
    double* part;                   // last layer: per matrix (offdiag^2, all^2), else null
};

// pair_svd_angles (the micro 2 x 2 SVD angles, src/lie_svd_micro.rs:128-139):
// theta_l, theta_r = (atan2(-(b + c), a - d) +- atan2(b - c, a + d)) / 2,
// each wrapped to (-pi/2, pi/2].
__device__ __forceinline__ void pair_svd_angles(double a, double b, double c, double d, double& tl,
                                                double& tr) {
    const double sum = atan2(-(b + c), a - d);
    const double diff = atan2(b - c, a + d);
    tl = wrap_half(0.5 * (sum + diff));
    tr = wrap_half(0.5 * (sum - diff));
}

// grid (nbe/2, F).  Shared: K padded 16 x 16 sub-blocks + RL, RR.
__global__ void __launch_bounds__(kThreads, 1) jsvd_solve_kernel(JsvdArgs a) {
    extern __shared__ __align__(16) double sh[];
    const int bp = blockIdx.x, f = blockIdx.y;
    const int nbp = a.nbe / 2;
    double* RLg = a.RL + (size_t(f) * nbp + bp) * B2 * B2;
    double* RRg = a.RR + (size_t(f) * nbp + bp) * B2 * B2;
    __shared__ int idx[B2];
    __shared__ int pl[B], pm[B];
    __shared__ double pcl[B], psl[B], pcr[B], psr[B];  // accepted rotation; s = 0 on both: none
    __shared__ long long nacc, nrej;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (!a.active[f]) {
        for (int e = tid; e < B2 * B2; e += kThreads) {
            const double v = (e / B2 == e % B2) ? 1.0 : 0.0;
            RLg[e] = v;
            RRg[e] = v;
        }
        return;
    }
    if (tid < B2) {
        int A, Bb;
        rr_pair(a.nbe, a.layer, bp, A, Bb);
        idx[tid] = block_pos(min(A, Bb), max(A, Bb), tid, a.kk);
    }
    if (tid == 0) {
        nacc = 0;
        nrej = 0;
    }
    __syncthreads();
    const int K = a.K, rows = a.rows, cols = a.cols;
    double* S = sh;                        // S[k] at k * MST, row stride SLD
    double* RLs = sh + size_t(K) * MST;    // B2 x SLD
    double* RRs = RLs + B2 * SLD;
    const double* Wf = a.W + size_t(f) * K * rows * cols;
    for (int e = tid; e < K * B2 * B2; e += kThreads) {
        const int k = e / (B2 * B2), r = (e / B2) % B2, c = e % B2;
        const int gi = idx[r], gj = idx[c];
        S[k * MST + r * SLD + c] = (gi >= 0 && gj >= 0) ? Wf[(size_t(k) * rows + gi) * cols + gj] : 0.0;
    }
    for (int e = tid; e < B2 * B2; e += kThreads) {
        const double v = (e / B2 == e % B2) ? 1.0 : 0.0;
        RLs[(e / B2) * SLD + e % B2] = v;
        RRs[(e / B2) * SLD + e % B2] = v;
    }
    __syncthreads();
    const double ptol = a.pair_tol[f];
    const int rounds = B + (a.layer == 0 ? B - 1 : 0);
    for (int round = 0; round < rounds; ++round) {
        if (tid < B) {
            int l, m;
            if (round < B) {  // cross pairs (t, B + (t + round) % B)
                l = tid;
                m = B + (tid + round) % B;
            } else {  // pairs inside each block
                const int rr = round - B, k = tid % (B / 2);
                int x, y;
                rr_pair(B, rr, k, x, y);
                const int off = tid < B / 2 ? 0 : B;
                l = off + min(x, y);
                m = off + max(x, y);
            }
            pl[tid] = l;
            pm[tid] = m;
            pcl[tid] = 1.0;
            psl[tid] = 0.0;
            pcr[tid] = 1.0;
            psr[tid] = 0.0;
        }
        __syncthreads();
        if (warp < B) {  // one warp per pair, lanes over the K matrices
            const int li = pl[warp], lj = pm[warp];
            const bool valid = idx[li] >= 0 && idx[lj] >= 0;
            double poff = 0.0, sa = 0.0, sb = 0.0, sc = 0.0, sd = 0.0;
            if (valid)
                for (int k = lane; k < K; k += 32) {
                    const double* Sk = S + size_t(k) * MST;
                    const double m00 = Sk[li * SLD + li], m01 = Sk[li * SLD + lj];
                    const double m10 = Sk[lj * SLD + li], m11 = Sk[lj * SLD + lj];
                    poff += fabs(m01) + fabs(m10);
                    // pair_block_norm (:279-282), floored at 1e-300
                    const double wt = fmax(sqrt(m00 * m00 + m01 * m01 + m10 * m10 + m11 * m11), 1e-300);
                    sa += m00 / wt;
                    sb += m01 / wt;
                    sc += m10 / wt;
                    sd += m11 / wt;
                }
            poff = warp_sum(poff);
            sa = warp_sum(sa);
            sb = warp_sum(sb);
            sc = warp_sum(sc);
            sd = warp_sum(sd);
            if (valid && poff > ptol) {
                double tl, tr;
                pair_svd_angles(sa, sb, sc, sd, tl, tr);
                if (fabs(tl) + fabs(tr) > 1e-18) {
                    // local off-diagonal energy restricted to the sub-block
                    double before = 0.0;
                    for (int k = lane; k < K; k += 32) {
                        const double* Sk = S + size_t(k) * MST;
                        for (int c = 0; c < B2; ++c) {
                            if (c != li) before += Sk[li * SLD + c] * Sk[li * SLD + c];
                            if (c != lj) before += Sk[lj * SLD + c] * Sk[lj * SLD + c];
                            if (c != li && c != lj)
                                before += Sk[c * SLD + li] * Sk[c * SLD + li] + Sk[c * SLD + lj] * Sk[c * SLD + lj];
                        }
                    }
                    before = warp_sum(before);
                    const double slack = 1e-14 * fmax(before, 1.0);
                    double scale = 1.0, cl = 1.0, sl = 0.0, cr = 1.0, sr = 0.0;
                    bool ok = false;
                    for (int stp = 0; stp < max(a.steps, 1); ++stp) {
                        double s1, c1, s2, c2;
                        sincos(tl * scale, &s1, &c1);
                        sincos(tr * scale, &s2, &c2);
                        double delta = 0.0;
                        for (int k = lane; k < K; k += 32) {
                            const double* Sk = S + size_t(k) * MST;
                            const double m00 = Sk[li * SLD + li], m01 = Sk[li * SLD + lj];
                            const double m10 = Sk[lj * SLD + li], m11 = Sk[lj * SLD + lj];
                            // rows by theta_l, then columns by theta_r
                            const double r00 = c1 * m00 - s1 * m10, r01 = c1 * m01 - s1 * m11;
                            const double r10 = s1 * m00 + c1 * m10, r11 = s1 * m01 + c1 * m11;
                            const double n01 = s2 * r00 + c2 * r01;
                            const double n10 = c2 * r10 - s2 * r11;
                            delta += n01 * n01 + n10 * n10 - m01 * m01 - m10 * m10;
                        }
                        delta = warp_sum(delta);
                        const double after = before + delta;
                        if (after <= before + slack && isfinite(after)) {
                            ok = true;
                            cl = c1;
                            sl = s1;
                            cr = c2;
                            sr = s2;
                            break;
                        }
                        scale *= 0.5;
                    }
                    if (lane == 0) {
                        if (ok) {
                            pcl[warp] = cl;
                            psl[warp] = sl;
                            pcr[warp] = cr;
                            psr[warp] = sr;
                            atomicAdd((unsigned long long*)&nacc, 1ull);
                        } else {
                            atomicAdd((unsigned long long*)&nrej, 1ull);
                        }
                    }
                }
            }
        }
        __syncthreads();
        // rows by theta_l (apply_left_rotor, :406-415)
        for (int e = tid; e < B * K * B2; e += kThreads) {
            const int p = e / (K * B2), k = (e / B2) % K, col = e % B2;
            const double s = psl[p], c = pcl[p];
            if (s == 0.0 && psr[p] == 0.0) continue;
            double* Sk = S + size_t(k) * MST;
            const int li = pl[p], lj = pm[p];
            const double x = Sk[li * SLD + col], y = Sk[lj * SLD + col];
            Sk[li * SLD + col] = c * x - s * y;
            Sk[lj * SLD + col] = s * x + c * y;
        }
        __syncthreads();
        // columns by theta_r (apply_right_rotor, :417-426) and the bases:
        // RR by theta_r, RL by theta_l (apply_basis_rotor, :428-437)
        for (int e = tid; e < B * (K + 2) * B2; e += kThreads) {
            const int p = e / ((K + 2) * B2), k = (e / B2) % (K + 2), row = e % B2;
            if (psl[p] == 0.0 && psr[p] == 0.0) continue;
            const bool left = k == K + 1;
            const double s = left ? psl[p] : psr[p], c = left ? pcl[p] : pcr[p];
            double* Mk = k < K ? S + size_t(k) * MST : (left ? RLs : RRs);
            const int li = pl[p], lj = pm[p];
            const double x = Mk[row * SLD + li], y = Mk[row * SLD + lj];
            Mk[row * SLD + li] = c * x - s * y;
            Mk[row * SLD + lj] = s * x + c * y;
        }
        __syncthreads();
    }
    for (int e = tid; e < B2 * B2; e += kThreads) {
        RLg[e] = RLs[(e / B2) * SLD + e % B2];
        RRg[e] = RRs[(e / B2) * SLD + e % B2];
    }
    if (tid == 0) {
        atomicAdd((unsigned long long*)&a.rot[2 * f], (unsigned long long)nacc);
        atomicAdd((unsigned long long*)&a.rot[2 * f + 1], (unsigned long long)nrej);
    }
}

// grid (K + 2, F), kThreads: matrix k of family f (k == K: U, left basis;
// k == K + 1: V, right basis).  W_k <- RL^T W_k RR; U <- U RL; V <- V RR.
// Streamed in strips of 16 rows: for W_k the layer's row block pairs (left
// product) and then the rows past kk in groups of 16; for U and V plain
// groups of 16 rows.  Each strip: coalesced load (left product in registers),
// shared strip (row stride ncols + 1), right product by one warp per column
// block pair in place (columns past kk unchanged), coalesced store.
__global__ void __launch_bounds__(kThreads, 2) jsvd_apply_kernel(JsvdArgs a) {
    const int k = blockIdx.x, f = blockIdx.y;
    if (!a.active[f]) return;
    extern __shared__ __align__(16) double ash[];
    const int kk = a.kk, nbp = a.nbe / 2;
    const bool isW = k < a.K, isU = k == a.K;
    const int nrows = isW ? a.rows : (isU ? a.rows : a.cols);
    const int ncols = isW ? a.cols : nrows;
    double* M = isW ? a.W + (size_t(f) * a.K + k) * a.rows * a.cols
                    : (isU ? a.U + size_t(f) * a.rows * a.rows : a.V + size_t(f) * a.cols * a.cols);
    const int ldt = ncols + 1;
    double* RLall = ash;                                // nbp * B2 * B2
    double* RRall = RLall + size_t(nbp) * B2 * B2;      // nbp * B2 * B2
    double* T = RRall + size_t(nbp) * B2 * B2;          // B2 x ldt
    int* blo = reinterpret_cast<int*>(T + size_t(B2) * ldt);
    int* bhi = blo + 32 * 4;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double sum_off = 0.0, sum_all = 0.0;
    const double* RLg = a.RL + size_t(f) * nbp * B2 * B2;
    const double* RRg = a.RR + size_t(f) * nbp * B2 * B2;
    for (int e = tid; e < nbp * B2 * B2; e += kThreads) {
        RLall[e] = RLg[e];
        RRall[e] = RRg[e];
    }
    for (int q = tid; q < nbp; q += kThreads) {
        int A, Bb;
        rr_pair(a.nbe, a.layer, q, A, Bb);
        blo[q] = min(A, Bb);
        bhi[q] = max(A, Bb);
    }
    __syncthreads();
    const double* RQall = (isW || !isU) ? RRall : RLall;  // right factor: W, V -> RR; U -> RL
    const int left_strips = isW ? nbp : 0;
    const int base = isW ? kk : 0;  // first row of the plain strips
    const int nstrips = left_strips + (nrows - base + B2 - 1) / B2;
    for (int st = 0; st < nstrips; ++st) {
        const bool lft = st < left_strips;
        const int plo = lft ? blo[st] : 0, phi = lft ? bhi[st] : 0;
        const int row0 = lft ? 0 : base + (st - left_strips) * B2;
        auto row_of = [&](int r) -> int {
            if (lft) return block_pos(plo, phi, r, kk);
            const int g = row0 + r;
            return g < nrows ? g : -1;
        };
        const double* RP = RLall + size_t(lft ? st : 0) * B2 * B2;
        // ---- load (+ left product for the W strips of block pairs)
        for (int col = tid; col < ncols; col += kThreads) {
            double x[B2];
#pragma unroll
            for (int r = 0; r < B2; ++r) {
                const int g = row_of(r);
                x[r] = g >= 0 ? M[size_t(g) * ncols + col] : 0.0;
            }
            if (!lft) {
#pragma unroll
                for (int r = 0; r < B2; ++r) T[r * ldt + col] = x[r];
            } else {
#pragma unroll 1
                for (int r = 0; r < B2; r += 2) {
                    double y0 = 0.0, y1 = 0.0;
#pragma unroll
                    for (int rp = 0; rp < B2; ++rp) {
                        const double2 rr = *reinterpret_cast<const double2*>(RP + rp * B2 + r);
                        y0 = fma(rr.x, x[rp], y0);
                        y1 = fma(rr.y, x[rp], y1);
                    }
                    T[r * ldt + col] = y0;
                    T[(r + 1) * ldt + col] = y1;
                }
            }
        }
        __syncthreads();
        // ---- right product on the column block pairs (columns < kk)
        {
            const int rr = lane % B, c0 = 4 * (lane / B);
            for (int Q = warp; Q < nbp; Q += kThreads / 32) {
                const int qlo = blo[Q], qhi = bhi[Q];
                const double* RQ = RQall + size_t(Q) * B2 * B2;
                double x0[B2], x1[B2];
#pragma unroll
                for (int c = 0; c < B2; ++c) {
                    const int g = block_pos(qlo, qhi, c, kk);
                    x0[c] = g >= 0 ? T[rr * ldt + g] : 0.0;
                    x1[c] = g >= 0 ? T[(rr + B) * ldt + g] : 0.0;
                }
                double y0[4] = {0.0, 0.0, 0.0, 0.0}, y1[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int cp = 0; cp < B2; ++cp) {
                    const double2 ra = *reinterpret_cast<const double2*>(RQ + cp * B2 + c0);
                    const double2 rb = *reinterpret_cast<const double2*>(RQ + cp * B2 + c0 + 2);
                    y0[0] = fma(x0[cp], ra.x, y0[0]);
                    y0[1] = fma(x0[cp], ra.y, y0[1]);
                    y0[2] = fma(x0[cp], rb.x, y0[2]);
                    y0[3] = fma(x0[cp], rb.y, y0[3]);
                    y1[0] = fma(x1[cp], ra.x, y1[0]);
                    y1[1] = fma(x1[cp], ra.y, y1[1]);
                    y1[2] = fma(x1[cp], rb.x, y1[2]);
                    y1[3] = fma(x1[cp], rb.y, y1[3]);
                }
                __syncwarp();  // every lane of the warp read its rows before any writes
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int g = block_pos(qlo, qhi, c0 + u, kk);
                    if (g >= 0) {
                        T[rr * ldt + g] = y0[u];
                        T[(rr + B) * ldt + g] = y1[u];
                    }
                }
            }
        }
        __syncthreads();
        // ---- store (last layer of a sweep: squared norms of W_k)
        for (int col = tid; col < ncols; col += kThreads) {
#pragma unroll
            for (int r = 0; r < B2; ++r) {
                const int g = row_of(r);
                if (g >= 0) {
                    const double v = T[r * ldt + col];
                    M[size_t(g) * ncols + col] = v;
                    sum_all = fma(v, v, sum_all);
                    if (g != col) sum_off = fma(v, v, sum_off);
                }
            }
        }
        __syncthreads();
    }
    if (a.part && isW) {
        __shared__ double red[2][kThreads / 32];
        for (int o = 16; o > 0; o >>= 1) {
            sum_off += __shfl_xor_sync(0xffffffffu, sum_off, o);
            sum_all += __shfl_xor_sync(0xffffffffu, sum_all, o);
        }
        if (lane == 0) {
            red[0][warp] = sum_off;
            red[1][warp] = sum_all;
        }
        __syncthreads();
        if (tid == 0) {
            double so = 0.0, sa = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) {
                so += red[0][w];
                sa += red[1][w];
            }
            a.part[2 * (size_t(f) * a.K + k)] = so;
            a.part[2 * (size_t(f) * a.K + k) + 1] = sa;
        }
    }
}

// Per family: sums over k and all entries with i != j of m_ij^2
// (joint_offdiag_norm^2, :439-441 on rectangular matrices) and of all m_ij^2.
__global__ void jsvd_norms_kernel(int F, int K, int rows, int cols, const double* W, double* off2,
                                  double* all2) {
    const int f = blockIdx.x;
    __shared__ double red[2][kThreads / 32];
    const double* Wf = W + size_t(f) * K * rows * cols;
    double so = 0.0, sa = 0.0;
    const size_t tot = size_t(K) * rows * cols, rc = size_t(rows) * cols;
    for (size_t e = threadIdx.x; e < tot; e += kThreads) {
        const double v = Wf[e];
        const size_t ij = e % rc;
        sa += v * v;
        if (ij / cols != ij % cols) so += v * v;
    }
    so = warp_sum(so);
    sa = warp_sum(sa);
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = so;
        red[1][threadIdx.x >> 5] = sa;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) {
            x += red[0][w];
            y += red[1][w];
        }
        off2[f] = x;
        all2[f] = y;
    }
}

__global__ void jsvd_part_sum_kernel(int F, int K, const double* part, const int* active, double* off2,
                                     double* all2) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F || !active[f]) return;
    double so = 0.0, sa = 0.0;
    for (int k = 0; k < K; ++k) {
        so += part[2 * (size_t(f) * K + k)];
        sa += part[2 * (size_t(f) * K + k) + 1];
    }
    off2[f] = so;
    all2[f] = sa;
}

__global__ void eye_kernel(size_t count, int n, double* M) {
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < count; e += size_t(gridDim.x) * blockDim.x) {
        const size_t ij = e % (size_t(n) * n);
        M[e] = (ij / n == ij % n) ? 1.0 : 0.0;
    }
}

// sig[f][k][i] = |W_k[i][i]| (diagonal_corridor, :501-504); Vt[f] = V[f]^T.
__global__ void jsvd_out_kernel(int F, int K, int rows, int cols, int kk, const double* W, double* sig,
                                const double* V, double* Vt) {
    const size_t ns = size_t(F) * K * kk, nv = size_t(F) * cols * cols;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < ns + nv; e += size_t(gridDim.x) * blockDim.x) {
        if (e < ns) {
            const size_t fk = e / kk, i = e % kk;
            sig[e] = fabs(W[fk * rows * cols + i * cols + i]);
        } else {
            const size_t x = e - ns, f = x / (size_t(cols) * cols), ij = x % (size_t(cols) * cols);
            const size_t i = ij / cols, j = ij % cols;
            Vt[f * cols * cols + i * cols + j] = V[f * cols * cols + j * cols + i];
        }
    }
}

}  // namespace

extern "C" lsvd_status lsvd_joint_svd_f64(lsvd_context* ctx, int64_t families, int64_t K, int64_t rows,
                                          int64_t cols, const double* M, const lsvd_joint_params* params,
                                          double* U, double* sig, double* Vt, lsvd_joint_trace* traces,
                                          uint32_t flags) {
    LSVD_TRACE("lsvd_joint_svd_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (families < 0 || K < 0 || rows < 0 || cols < 0)
        return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "LieSvdJoint::joint_svd: bad shape");
    if (families == 0) return LSVD_OK;
    if (K == 0 || rows == 0 || cols == 0)  // :174-181
        return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "LieSvdJoint::joint_svd: empty input");
    if (!M || !U || !sig || !Vt || !traces) return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "null pointer");
    const int64_t kk = std::min(rows, cols);
    const int nb = int((kk + B - 1) / B), nbe = nb % 2 == 0 ? std::max(nb, 2) : nb + 1;
    const int nbp = nbe / 2, layers = nbe - 1;
    const size_t smem = size_t(K) * MST * 8 + 2 * B2 * SLD * 8;
    const int64_t wide = std::max(rows, cols);
    const size_t asmem = 2 * size_t(nbp) * B2 * B2 * 8 + size_t(B2) * (wide + 1) * 8 + 2 * 32 * 4 * 4;
    if (smem > 200 * 1024 || asmem > 200 * 1024 || nbp > 128 || families > (1 << 30))
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "LieSvdJoint::joint_svd: K <= 90 and max(rows, cols) <= ~500");
    const lsvd_joint_params p = params ? *params : lsvd_joint_params_for_n(kk);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool dev = (flags & LSVD_DEVICE_POINTERS) != 0;
    const int F = int(families);
    const size_t wsz = size_t(F) * K * rows * cols, usz = size_t(F) * rows * rows, vsz = size_t(F) * cols * cols;
    const size_t ssz = size_t(F) * K * kk, rsz = size_t(F) * nbp * B2 * B2, psz = 2 * size_t(F) * K;
    auto al = [](size_t x) { return (x + 31) & ~size_t(31); };
    const size_t bytes = 8 * (al(wsz) + al(vsz) + 2 * al(rsz) + al(psz) + 4 * al(F) +
                              (dev ? 0 : al(usz) + al(ssz) + al(vsz))) +
                         16 * al(F) + 4 * al(F);
    cudaError_t e;
    char* ws = static_cast<char*>(ctx->ws_rot.get(bytes, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "joint_svd workspace");
    char* q = ws;
    auto take = [&](size_t doubles) {
        double* r = reinterpret_cast<double*>(q);
        q += 8 * al(doubles);
        return r;
    };
    double* dW = take(wsz);
    double* dV = take(vsz);
    double* dRL = take(rsz);
    double* dRR = take(rsz);
    double* dPart = take(psz);
    double* off2 = take(F);
    double* all2 = take(F);
    double* ptol = take(F);
    take(F);
    double* dU = dev ? U : take(usz);
    double* dS = dev ? sig : take(ssz);
    double* dVt = dev ? Vt : take(vsz);
    long long* rot = reinterpret_cast<long long*>(q);
    q += 16 * al(F);
    int* active = reinterpret_cast<int*>(q);
    if ((e = cudaMemcpyAsync(dW, M, wsz * 8, cudaMemcpyDefault, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(rot, 0, size_t(F) * 16, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "joint_svd setup");
    eye_kernel<<<std::min<size_t>((usz + 255) / 256, 4096), 256, 0, st>>>(usz, int(rows), dU);
    eye_kernel<<<std::min<size_t>((vsz + 255) / 256, 4096), 256, 0, st>>>(vsz, int(cols), dV);
    jsvd_norms_kernel<<<F, kThreads, 0, st>>>(F, int(K), int(rows), int(cols), dW, off2, all2);
    ctx->launches += 3;
    std::vector<double> h_off(F), h_all(F), h_tol(F), h_ptol(F), before(F), init(F);
    std::vector<int> h_act(F, kk > 1 ? 1 : 0);
    std::vector<long long> h_sweeps(F, 0);
    if ((e = cudaMemcpyAsync(h_off.data(), off2, 8 * F, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h_all.data(), all2, 8 * F, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "joint_svd norms");
    for (int f = 0; f < F; ++f) {
        const double ref = std::max(std::sqrt(h_all[f]), 1e-300);  // :185
        h_ptol[f] = p.min_pair_scale * std::max(ref, 1.0);        // :186
        h_tol[f] = p.tol * std::max(ref, 1.0);                    // :187
        init[f] = std::sqrt(h_off[f]);                            // :188
        before[f] = init[f];
    }
    if ((e = cudaMemcpyAsync(ptol, h_ptol.data(), 8 * F, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(active, h_act.data(), 4 * F, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "joint_svd upload");
    if ((e = cudaFuncSetAttribute(jsvd_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))) !=
            cudaSuccess ||
        (e = cudaFuncSetAttribute(jsvd_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(asmem))) !=
            cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "joint_svd smem");
    JsvdArgs a;
    a.F = F;
    a.K = int(K);
    a.rows = int(rows);
    a.cols = int(cols);
    a.kk = int(kk);
    a.nbe = nbe;
    a.steps = p.line_search_steps;
    a.pair_tol = ptol;
    a.W = dW;
    a.U = dU;
    a.V = dV;
    a.RL = dRL;
    a.RR = dRR;
    a.rot = rot;
    a.active = active;
    a.part = nullptr;
    int live = 0;
    for (int f = 0; f < F; ++f) live += h_act[f];
    for (int sw = 0; sw < p.max_sweeps && live > 0; ++sw) {
        for (int f = 0; f < F; ++f)
            if (h_act[f]) h_sweeps[f] = sw + 1;
        for (int l = 0; l < layers; ++l) {
            a.layer = l;
            a.part = (l + 1 == layers) ? dPart : nullptr;
            jsvd_solve_kernel<<<dim3(nbp, F), kThreads, smem, st>>>(a);
            jsvd_apply_kernel<<<dim3(unsigned(K + 2), F), kThreads, asmem, st>>>(a);
            ctx->launches += 2;
        }
        jsvd_part_sum_kernel<<<(F + 127) / 128, 128, 0, st>>>(F, int(K), dPart, active, off2, all2);
        ctx->launches++;
        if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "joint_svd sweep");
        if ((e = cudaMemcpyAsync(h_off.data(), off2, 8 * F, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "joint_svd sweep sync");
        live = 0;
        for (int f = 0; f < F; ++f) {
            if (!h_act[f]) continue;
            const double after = std::sqrt(h_off[f]);
            if (after <= h_tol[f] || after >= before[f] * (1.0 - 1e-10)) h_act[f] = 0;  // :226-229
            before[f] = after;
            live += h_act[f];
        }
        if ((e = cudaMemcpyAsync(active, h_act.data(), 4 * F, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "joint_svd active");
    }
    jsvd_norms_kernel<<<F, kThreads, 0, st>>>(F, int(K), int(rows), int(cols), dW, off2, all2);  // :232
    jsvd_out_kernel<<<std::min<size_t>((ssz + vsz + 255) / 256, 8192), 256, 0, st>>>(
        F, int(K), int(rows), int(cols), int(kk), dW, dS, dV, dVt);
    ctx->launches += 2;
    std::vector<long long> h_rot(2 * size_t(F));
    if ((e = cudaMemcpyAsync(h_off.data(), off2, 8 * F, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h_rot.data(), rot, 16 * size_t(F), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "joint_svd out");
    if (!dev) {
        if ((e = cudaMemcpyAsync(U, dU, usz * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(sig, dS, ssz * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(Vt, dVt, vsz * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "joint_svd copy out");
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "joint_svd sync");
    for (int f = 0; f < F; ++f) {
        lsvd_joint_trace t;
        t.initial_offdiag = kk > 1 ? init[f] : 0.0;
        t.final_offdiag = kk > 1 ? std::sqrt(h_off[f]) : 0.0;
        t.sweeps = h_sweeps[f];
        t.rotations = h_rot[2 * f];
        t.rejected_rotations = h_rot[2 * f + 1];
        traces[f] = t;
    }
    return LSVD_OK;
}
