// lsvd_jade.cu -- Phase-JADE joint diagonalisation of symmetric families,
// LieSvdJoint::diagonalize_symmetric_with_params (src/lie_svd_joint.rs:71-158),
// batched over independent families.
//
// One family is K matrices of n x n; the reference sweeps n-1 round-robin
// layers (layer_pairs, :524-539) of disjoint index pairs, and for each pair
//   * skips it if sum_k |m_ij| + |m_ji| <= pair_tol              (:118)
//   * takes the Cardoso angle 1/4 atan2(2 sxy, syy - sxx), or its pi/4
//     alternative if that leaves less 2x2 off-diagonal energy   (:338-357)
//   * skips |theta| <= 1e-18                                      (:122)
//   * applies the symmetric rotor to all K matrices and accepts it if the
//     local off-diagonal energy does not grow beyond 1e-14 max(before, 1),
//     else rolls back and halves theta, line_search_steps times (:359-386)
// and stops a sweep loop when the joint off-diagonal norm is <= tol or
// stopped decreasing by 1e-10 (:139-142).
//
// Blocked on the GPU: indices are cut into blocks of B = 8 and the blocks are
// paired by the same circle method; for each block pair the K principal
// 16 x 16 sub-blocks are staged in shared memory (jade_solve_kernel) and every
// index pair inside is treated by the rules above -- cross pairs in every
// block layer, pairs inside a block in block layer 0, so each index pair is
// visited once per sweep, as in the reference.  The accepted rotations of a
// block pair compose into one 16 x 16 orthogonal R, and a second pass
// (jade_apply_kernel) applies all of a layer's R to every 16 x 16 tile of
// every matrix, M[P,Q] <- R_P^T M[P,Q] R_Q, and to V: the family is streamed
// once per block layer instead of once per index layer.
//
// The acceptance test uses the exact change of the pair's 2 x 2 block energy
// (the energy of rows/columns i, j outside the block is invariant under the
// pair's rotation) and the sub-block's local energy for the slack, so it
// differs from the reference only in rounding (decisions are identical in
// exact arithmetic); the pair order inside a sweep differs, so parity is on
// the converged result (final off-diagonal, V orthogonality, diagonals).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "lsvd.h"
#include "lsvd_internal.h"
#include "lsvd_dgemm.cuh"
#include "lsvd_joint_common.cuh"

namespace {

using namespace lsvd::joint;
using lsvd::dg::cp_async16;
using lsvd::dg::cp_async_commit;
using lsvd::dg::cp_async_wait;

struct JadeArgs {
    int F, K, n, nbe;        // families, matrices per family, order, blocks (even)
    int layer;               // block layer
    int steps;               // line_search_steps
    const double* pair_tol;  // per family
    double* W;               // F*K*n*n, rotated in place
    double* V;               // F*n*n
    double* R;               // F*(nbe/2)*B2*B2
    long long* rot;          // per family: accepted, rejected
    const int* active;       // per family
    double* part;            // last layer of a sweep: per matrix (offdiag^2, all^2), else null
    int prefetch;            // apply: strips staged by cp.async one strip ahead (n even)
};

// Block pair (A, Bk) of `layer` -> the 16 global indices (B of block A, then
// B of block Bk); -1 marks padding past n.
__device__ __forceinline__ void block_indices(const JadeArgs& a, int bp, int* idx) {
    int A, Bb;
    rr_pair(a.nbe, a.layer, bp, A, Bb);
    const int lo = min(A, Bb), hi = max(A, Bb);
    for (int t = 0; t < B; ++t) {
        const int i0 = lo * B + t, i1 = hi * B + t;
        idx[t] = i0 < a.n ? i0 : -1;
        idx[B + t] = i1 < a.n ? i1 : -1;
    }
}

// grid (nbe/2, F).  Shared: K x 16 x 16 sub-blocks + R + pair tables.
__global__ void __launch_bounds__(kThreads, 1) jade_solve_kernel(JadeArgs a) {
    extern __shared__ __align__(16) double sh[];
    const int bp = blockIdx.x, f = blockIdx.y;
    const int nbp = a.nbe / 2;
    double* R = a.R + (size_t(f) * nbp + bp) * B2 * B2;
    __shared__ int idx[B2];
    __shared__ int pl[B], pm[B];          // pairs of the current round (local indices)
    __shared__ double pc[B], ps[B];       // accepted rotation (cos, sin), s = 0: none
    __shared__ long long nacc, nrej;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (!a.active[f]) {
        // keep R = I so the apply pass is a no-op for finished families
        for (int e = tid; e < B2 * B2; e += kThreads) R[e] = (e / B2 == e % B2) ? 1.0 : 0.0;
        return;
    }
    if (tid == 0) {
        block_indices(a, bp, idx);
        nacc = 0;
        nrej = 0;
    }
    __syncthreads();
    const int K = a.K, n = a.n;
    double* S = sh;                    // S[k][r][c]
    double* Rs = sh + size_t(K) * MST;
    const double* Wf = a.W + size_t(f) * K * n * n;
    for (int e = tid; e < K * B2 * B2; e += kThreads) {
        const int k = e / (B2 * B2), r = (e / B2) % B2, c = e % B2;
        const int se = k * MST + r * SLD + c;
        const int gi = idx[r], gj = idx[c];
        S[se] = (gi >= 0 && gj >= 0) ? Wf[(size_t(k) * n + gi) * n + gj] : 0.0;
    }
    for (int e = tid; e < B2 * B2; e += kThreads) Rs[(e / B2) * SLD + e % B2] = (e / B2 == e % B2) ? 1.0 : 0.0;
    __syncthreads();
    const double ptol = a.pair_tol[f];
    const int rounds_cross = B, rounds_intra = (a.layer == 0) ? B - 1 : 0;
    for (int round = 0; round < rounds_cross + rounds_intra; ++round) {
        if (tid < B) {
            int l, m;
            if (round < rounds_cross) {  // cross pairs (t, B + (t + round) % B)
                l = tid;
                m = B + (tid + round) % B;
            } else {  // pairs inside each block: round robin over B, I and J at once
                const int rr = round - rounds_cross, k = tid % (B / 2);
                int x, y;
                rr_pair(B, rr, k, x, y);
                const int off = tid < B / 2 ? 0 : B;
                l = off + min(x, y);
                m = off + max(x, y);
            }
            pl[tid] = l;
            pm[tid] = m;
            pc[tid] = 1.0;
            ps[tid] = 0.0;
        }
        __syncthreads();
        // one warp per pair: angle, line search over the K matrices
        if (warp < B) {
            const int li = pl[warp], lj = pm[warp];
            const bool valid = idx[li] >= 0 && idx[lj] >= 0;
            double poff = 0.0, sxx = 0.0, syy = 0.0, sxy = 0.0;
            if (valid)
                for (int k = lane; k < K; k += 32) {
                    const double* Sk = S + size_t(k) * MST;
                    const double mij = Sk[li * SLD + lj], mji = Sk[lj * SLD + li];
                    poff += fabs(mij) + fabs(mji);
                    const double x = 0.5 * (Sk[li * SLD + li] - Sk[lj * SLD + lj]);
                    const double y = 0.5 * (mij + mji);
                    sxx += x * x;
                    syy += y * y;
                    sxy += x * y;
                }
            poff = warp_sum(poff);
            sxx = warp_sum(sxx);
            syy = warp_sum(syy);
            sxy = warp_sum(sxy);
            if (valid && poff > ptol) {
                double th = 0.25 * atan2(2.0 * sxy, syy - sxx);
                const double alt = wrap_quarter(th + 0.25 * kPi);
                th = wrap_quarter(th);
                // joint_pair_energy_after (:388-399) for both candidates
                double st, ct, sa, ca;
                sincos(th, &st, &ct);
                sincos(alt, &sa, &ca);
                double et = 0.0, ea = 0.0, before = 0.0;
                for (int k = lane; k < K; k += 32) {
                    const double* Sk = S + size_t(k) * MST;
                    const double av = Sk[li * SLD + li], dv = Sk[lj * SLD + lj];
                    const double bv = 0.5 * (Sk[li * SLD + lj] + Sk[lj * SLD + li]);
                    const double ot = 0.5 * (av - dv) * (2.0 * st * ct) + bv * (ct * ct - st * st);
                    const double oa = 0.5 * (av - dv) * (2.0 * sa * ca) + bv * (ca * ca - sa * sa);
                    et += 2.0 * ot * ot;
                    ea += 2.0 * oa * oa;
                    // local_offdiag_sq_for_axes (:475-494) restricted to the sub-block
                    for (int c = 0; c < B2; ++c) {
                        if (c != li) before += Sk[li * SLD + c] * Sk[li * SLD + c];
                        if (c != lj) before += Sk[lj * SLD + c] * Sk[lj * SLD + c];
                        if (c != li && c != lj)
                            before += Sk[c * SLD + li] * Sk[c * SLD + li] + Sk[c * SLD + lj] * Sk[c * SLD + lj];
                    }
                }
                et = warp_sum(et);
                ea = warp_sum(ea);
                before = warp_sum(before);
                const double theta = ea < et ? alt : th;
                if (fabs(theta) > 1e-18) {
                    // accept_joint_rotor (:359-386): the rotor changes the local
                    // energy only through the pair's 2x2 block
                    const double slack = 1e-14 * fmax(before, 1.0);
                    double scale = 1.0, cacc = 1.0, sacc = 0.0;
                    bool ok = false;
                    for (int stp = 0; stp < max(a.steps, 1); ++stp) {
                        double s, c;
                        sincos(theta * scale, &s, &c);
                        double delta = 0.0;
                        for (int k = lane; k < K; k += 32) {
                            const double* Sk = S + size_t(k) * MST;
                            const double m00 = Sk[li * SLD + li], m01 = Sk[li * SLD + lj];
                            const double m10 = Sk[lj * SLD + li], m11 = Sk[lj * SLD + lj];
                            // rows then columns (apply_symmetric_rotor, :401-404)
                            const double r00 = c * m00 - s * m10, r01 = c * m01 - s * m11;
                            const double r10 = s * m00 + c * m10, r11 = s * m01 + c * m11;
                            const double n01 = s * r00 + c * r01;
                            const double n10 = c * r10 - s * r11;
                            delta += n01 * n01 + n10 * n10 - m01 * m01 - m10 * m10;
                        }
                        delta = warp_sum(delta);
                        const double after = before + delta;
                        if (after <= before + slack && isfinite(after)) {
                            ok = true;
                            cacc = c;
                            sacc = s;
                            break;
                        }
                        scale *= 0.5;
                    }
                    if (lane == 0) {
                        if (ok) {
                            pc[warp] = cacc;
                            ps[warp] = sacc;
                            atomicAdd((unsigned long long*)&nacc, 1ull);
                        } else {
                            atomicAdd((unsigned long long*)&nrej, 1ull);
                        }
                    }
                }
            }
        }
        __syncthreads();
        // rows (apply_left_rotor, :406-415) of every pair in the round
        for (int e = tid; e < B * K * B2; e += kThreads) {
            const int p = e / (K * B2), k = (e / B2) % K, col = e % B2;
            const double s = ps[p];
            if (s == 0.0) continue;
            const double c = pc[p];
            double* Sk = S + size_t(k) * MST;
            const int li = pl[p], lj = pm[p];
            const double x = Sk[li * SLD + col], y = Sk[lj * SLD + col];
            Sk[li * SLD + col] = c * x - s * y;
            Sk[lj * SLD + col] = s * x + c * y;
        }
        __syncthreads();
        // columns (apply_right_rotor, :417-426) and the basis (apply_basis_rotor, :428-437)
        for (int e = tid; e < B * (K + 1) * B2; e += kThreads) {
            const int p = e / ((K + 1) * B2), k = (e / B2) % (K + 1), row = e % B2;
            const double s = ps[p];
            if (s == 0.0) continue;
            const double c = pc[p];
            double* Sk = k < K ? S + size_t(k) * MST : Rs;
            const int li = pl[p], lj = pm[p];
            const double x = Sk[row * SLD + li], y = Sk[row * SLD + lj];
            Sk[row * SLD + li] = c * x - s * y;
            Sk[row * SLD + lj] = s * x + c * y;
        }
        __syncthreads();
    }
    for (int e = tid; e < B2 * B2; e += kThreads) R[e] = Rs[(e / B2) * SLD + e % B2];
    if (tid == 0) {
        atomicAdd((unsigned long long*)&a.rot[2 * f], (unsigned long long)nacc);
        atomicAdd((unsigned long long*)&a.rot[2 * f + 1], (unsigned long long)nrej);
    }
}

// grid (K + 1, F), kThreads: matrix k of family f (k == K: the basis V).
// M <- R^T M R with R = blockdiag over the layer's block pairs (for V:
// V <- V R), streamed one strip of 2B rows (a row block pair P) at a time:
//   load  : each thread takes columns, reads the strip's 2B rows from global
//           (coalesced) into registers and left-multiplies by R_P^T;
//   stage : the product goes to a shared strip (row stride n + 1);
//   right : one warp per column block pair Q; lane (rr, quarter) holds rows
//           rr and rr + B and 4 of the 2B columns, R_Q read as 16-byte
//           broadcasts; results in place (each lane owns its entries);
//   store : coalesced row stores back to global.
// All R of the family sit in shared memory for the whole matrix, so M's data
// cross HBM once per layer.  Positions past n are padding (R is the
// identity there and they are never loaded or stored).
__global__ void __launch_bounds__(kThreads, 2) jade_apply_kernel(JadeArgs a) {
    const int k = blockIdx.x, f = blockIdx.y;
    if (!a.active[f]) return;
    extern __shared__ __align__(16) double ash[];
    const int n = a.n, nbp = a.nbe / 2, ldt = n + 1;
    const bool isV = k == a.K;
    double* M = isV ? a.V + size_t(f) * n * n : a.W + (size_t(f) * a.K + k) * n * n;
    double* Rall = ash;                              // nbp * B2 * B2
    double* T = Rall + size_t(nbp) * B2 * B2;        // B2 x ldt
    // with prefetch: the next strip's rows, row stride n + 2 (16-byte rows for cp.async)
    const bool pre = a.prefetch != 0;
    const int ldi = n + 2;
    double* Tin = T + size_t(B2) * ldt;
    int* blo = reinterpret_cast<int*>(Tin + (pre ? size_t(B2) * ldi : 0));
    int* bhi = blo + 32 * 4;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double sum_off = 0.0, sum_all = 0.0;
    const double* Rg = a.R + size_t(f) * nbp * B2 * B2;
    for (int e = tid; e < nbp * B2 * B2; e += kThreads) Rall[e] = Rg[e];
    for (int q = tid; q < nbp; q += kThreads) {
        int A, Bb;
        rr_pair(a.nbe, a.layer, q, A, Bb);
        blo[q] = min(A, Bb);
        bhi[q] = max(A, Bb);
    }
    // strip P's 2B rows into Tin: 16-byte cp.async chunks (padding rows zeroed)
    auto stage = [&](int P) {
        const int pl = blo[P], ph = bhi[P], per_row = n / 2;
        for (int c = tid; c < B2 * per_row; c += kThreads) {
            const int r = c / per_row, ch = c - r * per_row;
            const int g = block_pos(pl, ph, r, n);
            double* dst = Tin + size_t(r) * ldi + 2 * ch;
            if (g >= 0) {
                cp_async16(dst, M + size_t(g) * n + 2 * ch, 16);
            } else {
                dst[0] = 0.0;
                dst[1] = 0.0;
            }
        }
        cp_async_commit();
    };
    __syncthreads();
    if (pre) stage(0);
    for (int P = 0; P < nbp; ++P) {
        const int plo = blo[P], phi = bhi[P];
        const double* RP = Rall + size_t(P) * B2 * B2;
        if (pre) {
            cp_async_wait<0>();
            __syncthreads();  // strip P is in Tin for every thread
        }
        // ---- load + left multiply (V: plain copy)
        for (int col = tid; col < n; col += kThreads) {
            double x[B2];
#pragma unroll
            for (int r = 0; r < B2; ++r) {
                if (pre) {
                    x[r] = Tin[r * ldi + col];
                } else {
                    const int g = block_pos(plo, phi, r, n);
                    x[r] = g >= 0 ? M[size_t(g) * n + col] : 0.0;
                }
            }
            if (isV) {
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
        // every thread is done with Tin: fetch the next strip behind the right multiply and store
        if (pre && P + 1 < nbp) stage(P + 1);
        // ---- right multiply by R_Q, in place in the strip
        {
            const int rr = lane % B, c0 = 4 * (lane / B);  // rows rr, rr + B; columns c0 .. c0 + 3
            for (int Q = warp; Q < nbp; Q += kThreads / 32) {
                const int qlo = blo[Q], qhi = bhi[Q];
                const double* RQ = Rall + size_t(Q) * B2 * B2;
                double x0[B2], x1[B2];
#pragma unroll
                for (int c = 0; c < B2; ++c) {
                    const int g = block_pos(qlo, qhi, c, n);
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
                    const int g = block_pos(qlo, qhi, c0 + u, n);
                    if (g >= 0) {
                        T[rr * ldt + g] = y0[u];
                        T[(rr + B) * ldt + g] = y1[u];
                    }
                }
            }
        }
        __syncthreads();
        // ---- store the strip (last layer of a sweep: also the squared norms
        // of the new matrix, joint_offdiag_norm / joint_frobenius_norm terms)
        for (int col = tid; col < n; col += kThreads) {
#pragma unroll
            for (int r = 0; r < B2; ++r) {
                const int g = block_pos(plo, phi, r, n);
                if (g >= 0) {
                    const double v = T[r * ldt + col];
                    M[size_t(g) * n + col] = v;
                    sum_all = fma(v, v, sum_all);
                    if (g != col) sum_off = fma(v, v, sum_off);
                }
            }
        }
        __syncthreads();
    }
    if (a.part && !isV) {
        // per-matrix partials in a fixed reduction order (deterministic)
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

// off2[f], all2[f] = sums of the K per-matrix partials, in order.
__global__ void jade_part_sum_kernel(int F, int K, const double* part, const int* active, double* off2,
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

// Per family: sum over k, i != j of m_ij^2 (joint_offdiag_norm^2, :439-441)
// and sum of all squares (joint_frobenius_norm^2, :443-449).
__global__ void jade_norms_kernel(int F, int K, int n, const double* W, const int* active,
                                  double* off2, double* all2) {
    const int f = blockIdx.x;
    if (active && !active[f]) return;
    __shared__ double red[2][kThreads / 32];
    const double* Wf = W + size_t(f) * K * n * n;
    double so = 0.0, sa = 0.0;
    const size_t tot = size_t(K) * n * n;
    for (size_t e = threadIdx.x; e < tot; e += kThreads) {
        const double v = Wf[e];
        const size_t ij = e % (size_t(n) * n);
        sa += v * v;
        if (ij / n != ij % n) so += v * v;
    }
    so = warp_sum(so);
    sa = warp_sum(sa);
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = so;
        red[1][threadIdx.x >> 5] = sa;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        off2[f] = a;
        all2[f] = b;
    }
}

__global__ void jade_init_kernel(int F, int n, double* V) {
    const size_t tot = size_t(F) * n * n;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < tot;
         e += size_t(gridDim.x) * blockDim.x) {
        const size_t ij = e % (size_t(n) * n);
        V[e] = (ij / n == ij % n) ? 1.0 : 0.0;
    }
}

__global__ void jade_diag_kernel(int F, int K, int n, const double* W, double* D) {
    const size_t tot = size_t(F) * K * n;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < tot;
         e += size_t(gridDim.x) * blockDim.x) {
        const size_t fk = e / n, i = e % n;
        D[e] = W[fk * n * n + i * n + i];
    }
}

}  // namespace

extern "C" lsvd_joint_params lsvd_joint_params_for_n(int64_t n) {
    lsvd_joint_params p;
    p.max_sweeps = int32_t(12 + std::max<int64_t>(n, 1));
    p.tol = 1e-12;
    p.min_pair_scale = 1e-14;
    p.line_search_steps = 6;
    return p;
}

extern "C" lsvd_status lsvd_jade_sym_f64(lsvd_context* ctx, int64_t families, int64_t K, int64_t n,
                                         const double* M, const lsvd_joint_params* params,
                                         double* V, double* diag, lsvd_joint_trace* traces,
                                         uint32_t flags) {
    LSVD_TRACE("lsvd_jade_sym_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (families < 0 || K < 0 || n < 0) return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "LieSvdJoint: bad shape");
    if (families == 0) return LSVD_OK;
    if (K == 0) return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "LieSvdJoint: empty matrix set");
    if (!M || !V || !diag || !traces) return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "null pointer");
    const size_t smem = size_t(K) * MST * 8 + B2 * SLD * 8;
    if (smem > 200 * 1024 || n > 32768)
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "LieSvdJoint: K must be <= 93 (shared memory)");
    const lsvd_joint_params p = params ? *params : lsvd_joint_params_for_n(n);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool dev = (flags & LSVD_DEVICE_POINTERS) != 0;
    const int F = int(families);
    const size_t wsz = size_t(F) * K * n * n, vsz = size_t(F) * n * n;
    const int nb = int((n + B - 1) / B), nbe = nb % 2 == 0 ? std::max(nb, 2) : nb + 1;
    const int nbp = nbe / 2, layers = nbe - 1;
    cudaError_t e;
    // workspace: W (work copy) | V | R | off2, all2, tol | rot | active
    const size_t rsz = size_t(F) * nbp * B2 * B2;
    auto al = [](size_t x) { return (x + 31) & ~size_t(31); };
    const size_t psz = 2 * size_t(F) * K;  // per-matrix norm partials of the last layer
    const size_t bytes = 8 * (al(wsz) + (dev ? 0 : al(vsz)) + al(rsz) + 4 * al(F) + al(psz)) + 16 * al(F) + 4 * al(F);
    char* ws = static_cast<char*>(ctx->ws_rot.get(bytes, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "jade workspace");
    char* q = ws;
    double* dW = reinterpret_cast<double*>(q); q += 8 * al(wsz);
    double* dV = dev ? V : reinterpret_cast<double*>(q);
    if (!dev) q += 8 * al(vsz);
    double* dR = reinterpret_cast<double*>(q); q += 8 * al(rsz);
    double* dPart = reinterpret_cast<double*>(q); q += 8 * al(psz);
    double* off2 = reinterpret_cast<double*>(q); q += 8 * al(F);
    double* all2 = reinterpret_cast<double*>(q); q += 8 * al(F);
    double* ptol = reinterpret_cast<double*>(q); q += 8 * al(F);
    q += 8 * al(F);
    long long* rot = reinterpret_cast<long long*>(q); q += 16 * al(F);
    int* active = reinterpret_cast<int*>(q);
    if ((e = cudaMemcpyAsync(dW, M, wsz * 8, cudaMemcpyDefault, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(rot, 0, size_t(F) * 16, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "jade setup");
    jade_init_kernel<<<std::min<size_t>((vsz + 255) / 256, 4096), 256, 0, st>>>(F, int(n), dV);
    jade_norms_kernel<<<F, kThreads, 0, st>>>(F, int(K), int(n), dW, nullptr, off2, all2);
    ctx->launches += 2;
    std::vector<double> h_off(F), h_all(F), h_tol(F), h_ptol(F), h_init(F), h_final(F);
    std::vector<int> h_act(F, 1);
    std::vector<long long> h_sweeps(F, 0);
    if ((e = cudaMemcpyAsync(h_off.data(), off2, 8 * F, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h_all.data(), all2, 8 * F, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "jade norms");
    for (int f = 0; f < F; ++f) {
        const double ref = std::max(std::sqrt(h_all[f]), 1e-300);  // :105
        h_ptol[f] = p.min_pair_scale * std::max(ref, 1.0);        // :106
        h_tol[f] = p.tol * std::max(ref, 1.0);                    // :107
        h_init[f] = std::sqrt(h_off[f]);                          // :108
        if (n <= 1) h_act[f] = 0;                                 // :87-101
    }
    if ((e = cudaMemcpyAsync(ptol, h_ptol.data(), 8 * F, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(active, h_act.data(), 4 * F, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "jade upload");
    if ((e = cudaFuncSetAttribute(jade_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem))) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "jade smem");
    // apply: all R of a family + one strip of 2B rows (row stride n + 1) + block tables
    size_t asmem = size_t(nbp) * B2 * B2 * 8 + size_t(B2) * (n + 1) * 8 + 2 * 32 * 4 * 4;
    if (asmem > 200 * 1024)
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "LieSvdJoint: n too large for the apply pass");
    // the prefetch buffer (next strip, row stride n + 2) where rows are 16-byte multiples and it fits
    const size_t pre_bytes = size_t(B2) * (n + 2) * 8;
    const bool prefetch = n % 2 == 0 && asmem + pre_bytes <= 100 * 1024;
    if (prefetch) asmem += pre_bytes;
    if ((e = cudaFuncSetAttribute(jade_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(asmem))) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "jade apply smem");
    JadeArgs a;
    a.F = F;
    a.K = int(K);
    a.n = int(n);
    a.nbe = nbe;
    a.steps = p.line_search_steps;
    a.prefetch = prefetch ? 1 : 0;
    a.pair_tol = ptol;
    a.W = dW;
    a.V = dV;
    a.R = dR;
    a.rot = rot;
    a.active = active;
    a.part = nullptr;
    std::vector<double> before(h_init);
    int live = 0;
    for (int f = 0; f < F; ++f) live += h_act[f];
    for (int sw = 0; sw < p.max_sweeps && live > 0; ++sw) {
        for (int f = 0; f < F; ++f)
            if (h_act[f]) h_sweeps[f] = sw + 1;
        for (int l = 0; l < layers; ++l) {
            a.layer = l;
            a.part = (l + 1 == layers) ? dPart : nullptr;
            jade_solve_kernel<<<dim3(nbp, F), kThreads, smem, st>>>(a);
            jade_apply_kernel<<<dim3(unsigned(K + 1), F), kThreads, asmem, st>>>(a);
            ctx->launches += 2;
        }
        // the sweep's norms came out of the last layer's apply pass
        jade_part_sum_kernel<<<(F + 127) / 128, 128, 0, st>>>(F, int(K), dPart, active, off2, all2);
        ctx->launches++;
        if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "jade sweep");
        if ((e = cudaMemcpyAsync(h_off.data(), off2, 8 * F, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "jade sweep sync");
        live = 0;
        for (int f = 0; f < F; ++f) {
            if (!h_act[f]) continue;
            const double after = std::sqrt(h_off[f]);
            if (after <= h_tol[f] || after >= before[f] * (1.0 - 1e-10)) h_act[f] = 0;  // :139-142
            before[f] = after;
            live += h_act[f];
        }
        if ((e = cudaMemcpyAsync(active, h_act.data(), 4 * F, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "jade active");
    }
    // final_offdiag (:145), diagonals (:146), outputs
    jade_norms_kernel<<<F, kThreads, 0, st>>>(F, int(K), int(n), dW, nullptr, off2, all2);
    double* dD = dev ? diag : dR;  // R is dead: reuse it for the diagonals on the host path
    if (!dev && rsz < size_t(F) * K * n) {
        dD = reinterpret_cast<double*>(static_cast<char*>(ctx->ws_u.get(size_t(F) * K * n * 8, &e)));
        if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "jade diag");
    }
    jade_diag_kernel<<<std::min<size_t>((size_t(F) * K * n + 255) / 256, 4096), 256, 0, st>>>(
        F, int(K), int(n), dW, dD);
    ctx->launches += 2;
    std::vector<long long> h_rot(2 * size_t(F));
    if ((e = cudaMemcpyAsync(h_off.data(), off2, 8 * F, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h_rot.data(), rot, 16 * size_t(F), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "jade out");
    if (!dev) {
        if ((e = cudaMemcpyAsync(V, dV, vsz * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(diag, dD, size_t(F) * K * n * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "jade copy out");
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "jade sync");
    for (int f = 0; f < F; ++f) {
        lsvd_joint_trace t;
        const bool trivial = n <= 1;
        t.initial_offdiag = trivial ? 0.0 : h_init[f];
        t.final_offdiag = trivial ? 0.0 : std::sqrt(h_off[f]);
        t.sweeps = trivial ? 0 : h_sweeps[f];
        t.rotations = h_rot[2 * size_t(f)];
        t.rejected_rotations = h_rot[2 * size_t(f) + 1];
        traces[f] = t;
    }
    return LSVD_OK;
}
