// lsvd_triage.cu -- batched triage of matrices on the GPU: the statistics
// LieSvdAdaptive::choose_route and PhaseEngine::passport_real compute before
// they route a matrix (src/lie_svd_adaptive.rs:84-274,
// src/lie_svd_phasehealth.rs:100-343, src/lie_svd_block4.rs:210-266,
// src/lie_svd_engine.rs:75-103, :277-326), so that a batch can be routed on
// the device.  One CTA per matrix: every row is a warp's vector (coalesced),
// every column a thread's (coalesced across the warp); each statistic is
// reduced in a fixed order, so results are deterministic.  O(rows x cols)
// reads per matrix: a bandwidth-bound kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "lsvd.h"
#include "lsvd_internal.h"

namespace {

constexpr int TT = 256;  // threads per CTA
constexpr int kMaxDim = 4096;

// Deterministic CTA sum (same value on every thread); red holds TT / 32.
__device__ __forceinline__ double csum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
#pragma unroll
    for (int w = 0; w < TT / 32; ++w) r += red[w];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double cmax(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
#pragma unroll
    for (int w = 0; w < TT / 32; ++w) r = fmax(r, red[w]);
    __syncthreads();
    return r;
}

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per-vector phase health (analyze_vector_phase_by, src/lie_svd_phasehealth.rs:
// 146-207) folded into the running summaries of summarize (:274-311) and the
// weighted phase sums of global_phase_invariants (:219-232).
struct Acc {
    double dbsq, gsq, max_twist, twist, ent, sin_w, cos_w, w;
    __device__ void zero() { dbsq = gsq = max_twist = twist = ent = sin_w = cos_w = w = 0.0; }
    __device__ void add(int64_t len, double sum, double norm_sq, double delay, double grad, double vector_sq,
                        double plogp) {
        if (len == 0) return;  // an empty vector adds zeros (analyze_vector_phase_by's n == 0 case)
        const double mean = sum / double(len);
        const double scalar_sq = double(len) * mean * mean;
        const double db = fmax(norm_sq * norm_sq - delay * delay, 0.0);
        const double ent_v = (len > 1 && norm_sq > 1e-300) ? -plogp / log(double(len)) : 0.0;
        const double tw = sqrt(db) / fmax(norm_sq, 1e-300);
        const double ph = (delay >= 0.0 ? 1.0 : -1.0) * atan2(sqrt(grad), fabs(mean) + sqrt(vector_sq) + 1e-300);
        dbsq += db;
        gsq += grad;
        max_twist = fmax(max_twist, tw);
        twist += tw;
        ent += ent_v;
        const double wt = sqrt(scalar_sq + vector_sq);
        double sn, cs;
        sincos(ph, &sn, &cs);
        sin_w += wt * sn;
        cos_w += wt * cs;
        w += wt;
    }
};

struct TriageArgs {
    int count;
    const int32_t* rows;
    const int32_t* cols;
    const int64_t* aoff;
    const double* A;
    lsvd_triage* out;
    int max_rows, max_cols;
};

}  // namespace

namespace {

// coeff_var (src/lie_svd_adaptive.rs:341-355) of v[0..len) in shared memory.
__device__ double coeff_var_dev(const double* v, int len, double* red) {
    double s = 0.0;
    for (int i = threadIdx.x; i < len; i += TT) s += v[i];
    const double l = double(max(len, 1));
    const double mean = csum(s, red) / l;
    if (fabs(mean) <= 1e-300) return 0.0;
    double q = 0.0;
    for (int i = threadIdx.x; i < len; i += TT) q += (v[i] - mean) * (v[i] - mean);
    return sqrt(csum(q, red) / l) / fabs(mean);
}

// entropy01 (:368-380) of v[0..len).
__device__ double entropy01_dev(const double* v, int len, double* red) {
    double s = 0.0;
    for (int i = threadIdx.x; i < len; i += TT) s += v[i];
    const double sum = csum(s, red);
    if (sum <= 1e-300 || len <= 1) return 1.0;
    double h = 0.0;
    for (int i = threadIdx.x; i < len; i += TT) {
        const double p = v[i] / sum;
        if (p > 0.0) h -= p * log(p);
    }
    return csum(h, red) / fmax(log(double(len)), 1e-300);
}

__global__ void __launch_bounds__(TT) triage_kernel(const TriageArgs args) {
    extern __shared__ __align__(16) double tsm[];
    __shared__ double red[TT / 32];
    __shared__ double wacc[TT / 32][12];
    const int t = blockIdx.x;
    const int n = args.rows[t], m = args.cols[t];
    const double* A = args.A + args.aoff[t];
    double* rl1 = tsm;
    double* rl2 = rl1 + args.max_rows;
    double* cl1 = rl2 + args.max_rows;
    double* cl2 = cl1 + args.max_cols;
    double* dabs = cl2 + args.max_cols;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int cor = min(n, m);
    // rows: one warp per row
    Acc ra;
    ra.zero();
    double all_sq = 0.0, diag_sq = 0.0, off_sq = 0.0, g_re = 0.0, g_im = 0.0, g_mass = 0.0;
    for (int i = warp; i < n; i += TT / 32) {
        const double* row = A + int64_t(i) * m;
        double s = 0.0, nq = 0.0, dl = 0.0, gr = 0.0, ab = 0.0, dq = 0.0;
        for (int j = lane; j < m; j += 32) {
            const double x = row[j], xn = row[j + 1 < m ? j + 1 : 0];
            s += x;
            nq += x * x;
            dl += x * xn;
            gr += (xn - x) * (xn - x);
            ab += fabs(x);
            if (j == i) dq = x * x;
        }
        s = wsum(s);
        nq = wsum(nq);
        dl = wsum(dl);
        gr = wsum(gr);
        ab = wsum(ab);
        dq = wsum(dq);
        const double mean = m ? s / double(m) : 0.0;
        double vq = 0.0, pl = 0.0;
        for (int j = lane; j < m; j += 32) {
            const double x = row[j];
            vq += (x - mean) * (x - mean);
            if (nq > 1e-300) {
                const double p = (x * x) / nq;
                if (p > 0.0) pl += p * log(p);
            }
        }
        vq = wsum(vq);
        pl = wsum(pl);
        if (lane == 0) {
            ra.add(m, s, nq, dl, gr, vq, pl);
            rl1[i] = ab;
            rl2[i] = sqrt(nq);
            if (i < cor) dabs[i] = sqrt(dq);
            all_sq += nq;
            diag_sq += dq;
            off_sq += nq - dq;
            double sn, cs;
            sincos(2.39996322972865332 * double(i), &sn, &cs);  // golden_resonance_real (src/lie_svd_engine.rs:310-326)
            g_re += ab * cs;
            g_im += ab * sn;
            g_mass += ab;
        }
    }
    if (lane == 0) {
        const double v[12] = {ra.dbsq, ra.gsq, ra.max_twist, ra.twist, ra.ent, ra.sin_w,
                              ra.cos_w, ra.w, all_sq, diag_sq, off_sq, 0.0};
        for (int k = 0; k < 12; ++k) wacc[warp][k] = v[k];
    }
    // columns: one thread per column
    Acc ca;
    ca.zero();
    for (int j = tid; j < m; j += TT) {
        double s = 0.0, nq = 0.0, dl = 0.0, gr = 0.0, ab = 0.0;
        for (int i = 0; i < n; ++i) {
            const double x = A[int64_t(i) * m + j], xn = A[int64_t(i + 1 < n ? i + 1 : 0) * m + j];
            s += x;
            nq += x * x;
            dl += x * xn;
            gr += (xn - x) * (xn - x);
            ab += fabs(x);
        }
        const double mean = n ? s / double(n) : 0.0;
        double vq = 0.0, pl = 0.0;
        for (int i = 0; i < n; ++i) {
            const double x = A[int64_t(i) * m + j];
            vq += (x - mean) * (x - mean);
            if (nq > 1e-300) {
                const double p = (x * x) / nq;
                if (p > 0.0) pl += p * log(p);
            }
        }
        ca.add(n, s, nq, dl, gr, vq, pl);
        cl1[j] = ab;
        cl2[j] = sqrt(nq);
    }
    __syncthreads();
    // row summaries in warp order
    double R[12] = {0};
    for (int w = 0; w < TT / 32; ++w)
        for (int k = 0; k < 12; ++k) R[k] = (k == 2) ? fmax(R[k], wacc[w][k]) : R[k] + wacc[w][k];
    const double c_dbsq = csum(ca.dbsq, red), c_gsq = csum(ca.gsq, red), c_max = cmax(ca.max_twist, red);
    const double c_ent = csum(ca.ent, red);
    const double c_sin = csum(ca.sin_w, red), c_cos = csum(ca.cos_w, red), c_w = csum(ca.w, red);
    const double gre = csum(lane == 0 ? g_re : 0.0, red), gim = csum(lane == 0 ? g_im : 0.0, red);
    const double gmass = csum(lane == 0 ? g_mass : 0.0, red);
    // corridor pairs: triangular disbalance, torsion, symmetry split, chirality
    double up = 0.0, lo = 0.0, skq = 0.0, syq = 0.0, chs = 0.0, cht = 0.0;
    for (int64_t e = tid; e < int64_t(cor) * cor; e += TT) {
        const int i = int(e / cor), j = int(e % cor);
        const double x = A[int64_t(i) * m + j];
        cht += x * x;
        if (i < j) {
            const double y = A[int64_t(j) * m + i];
            up += x * x;
            lo += y * y;
            const double sy = 0.5 * (x + y), sk = 0.5 * (x - y);
            syq += 2.0 * sy * sy;
            skq += 2.0 * sk * sk;
            chs += (x - y) * (x - y);
        }
    }
    up = csum(up, red);
    lo = csum(lo, red);
    skq = csum(skq, red);
    syq = csum(syq, red);
    chs = csum(chs, red);
    cht = csum(cht, red);
    // phase entropy of the whole operator (:253-266)
    const double tot = R[8];
    double pl = 0.0;
    if (tot > 1e-300)
        for (int64_t e = tid; e < int64_t(n) * m; e += TT) {
            const double p = (A[e] * A[e]) / tot;
            if (p > 0.0) pl += p * log(p);
        }
    pl = csum(pl, red);
    // 4x4 block self-dual / anti-self-dual balance (src/lie_svd_block4.rs:210-262)
    double sd2 = 0.0, asd2 = 0.0;
    for (int b = tid; b < cor / 4; b += TT) {
        const int st = 4 * b;
        auto wv = [&](int p, int q) { return 0.5 * (A[int64_t(st + q) * m + st + p] - A[int64_t(st + p) * m + st + q]); };
        const double w12 = wv(0, 1), w13 = wv(0, 2), w14 = wv(0, 3), w23 = wv(1, 2), w24 = wv(1, 3), w34 = wv(2, 3);
        const double r = 0.70710678118654752440;
        const double s0 = (w12 + w34) * r, s1 = (w13 - w24) * r, s2 = (w14 + w23) * r;
        const double a0 = (w12 - w34) * r, a1 = (w13 + w24) * r, a2 = (w14 - w23) * r;
        sd2 += s0 * s0 + s1 * s1 + s2 * s2;
        asd2 += a0 * a0 + a1 * a1 + a2 * a2;
    }
    sd2 = csum(sd2, red);
    asd2 = csum(asd2, red);
    // analyze_matrix's vector statistics (square inputs)
    const bool sq = n == m;
    double rcv = 0.0, ccv = 0.0, mism = 0.0, dent = 0.0, rent = 0.0, cent = 0.0;
    if (sq) {
        rcv = coeff_var_dev(rl2, n, red);
        ccv = coeff_var_dev(cl2, n, red);
        double num = 0.0, den = 0.0;
        for (int i = tid; i < n; i += TT) {
            const double d = rl1[i] - cl1[i];
            num += d * d;
            den += rl1[i] * rl1[i] + cl1[i] * cl1[i];
        }
        mism = sqrt(csum(num, red)) / fmax(sqrt(csum(den, red)), 1e-300);
        dent = entropy01_dev(dabs, n, red);
        rent = entropy01_dev(rl1, n, red);
        cent = entropy01_dev(cl1, n, red);
    }
    if (tid != 0) return;
    lsvd_triage o;
    const double nan = __longlong_as_double(0x7ff8000000000000ULL);
    const double cnt = double(max(n + m, 1));
    o.mean_stress = (sqrt(R[0] + c_dbsq) + sqrt(R[1] + c_gsq)) / cnt;
    o.max_twist = fmax(R[2], c_max);
    o.causal_disbalance = fabs(up - lo) / fmax(up + lo, 1e-300);
    o.entropy_gap = fabs((n ? R[4] / n : 0.0) - (m ? c_ent / m : 0.0));
    const double sw = R[5] + c_sin, cw = R[6] + c_cos, ww = R[7] + c_w;
    o.global_phase = ww > 1e-300 ? atan2(sw, cw) : 0.0;
    o.torsion_energy = sqrt(skq);
    const double sdn = sqrt(sd2), asdn = sqrt(asd2);
    o.chirality_balance = cor >= 4 ? fabs(sdn - asdn) / fmax(sdn + asdn, 1e-300) : 0.0;
    o.phase_entropy = (int64_t(n) * m > 1 && tot > 1e-300) ? -pl / log(double(int64_t(n) * m)) : 0.0;
    o.chirality = sqrt(chs) / fmax(sqrt(cht), 1e-300);
    o.golden_resonance = sqrt(gre * gre + gim * gim) / fmax(gmass, 1e-300);
    o.passport_route = (sq && (o.max_twist > 0.8 || o.causal_disbalance > 0.65 || o.entropy_gap > 0.2) && n <= 128) ? 1 : 0;
    if (!sq) {
        o.offdiag_ratio = o.diagonal_dominance = o.row_cv = o.col_cv = o.row_col_mismatch = nan;
        o.symmetry_ratio = o.transpose_torsion_ratio = o.diagonal_entropy = nan;
        o.row_mass_entropy = o.col_mass_entropy = o.suspicious_score = nan;
        o.adaptive_route = -1;
    } else {
        const double norm = fmax(sqrt(R[8]), 1e-300);
        const double off = sqrt(R[10]) / norm, dd = sqrt(R[9]) / norm;
        const double symr = sqrt(syq) / fmax(sqrt(syq + skq), 1e-300), torr = sqrt(skq) / fmax(sqrt(syq + skq), 1e-300);
        double score = 0.0;  // suspicious_score (src/lie_svd_adaptive.rs:325-339)
        score += fmax(off - 0.55, 0.0) * 0.9;
        score += fmax(0.35 - dd, 0.0) * 0.8;
        score += fmax(rcv, ccv) * 1.4;
        score += mism * 1.6;
        score += torr * 0.45;
        score += off * fmax(symr - 0.82, 0.0) * 1.8;
        score += fmax(0.78 - dent, 0.0) * 1.2;
        o.offdiag_ratio = off;
        o.diagonal_dominance = dd;
        o.row_cv = rcv;
        o.col_cv = ccv;
        o.row_col_mismatch = mism;
        o.symmetry_ratio = symr;
        o.transpose_torsion_ratio = torr;
        o.diagonal_entropy = dent;
        o.row_mass_entropy = rent;
        o.col_mass_entropy = cent;
        o.suspicious_score = score;
        // choose_route with the default LieSvdAdaptiveParams (:55-65, :103-184)
        const double thr = 1.15;
        const bool bal = score >= thr + 0.25 && off > 0.90 && dd < 0.25 && rcv >= 0.20 && ccv >= 0.20 && rcv < 0.45 &&
                         ccv < 0.45 && mism < 0.45;
        const bool pf = bal || (o.causal_disbalance > 0.88 && off > 0.20 && o.mean_stress > 1.0) ||
                        (o.mean_stress > 50.0 && o.max_twist > 0.92 && rcv < 0.42 && ccv < 0.42 && mism < 0.30 &&
                         off > 0.85 && dd < 0.35) ||
                        (o.chirality_balance > 0.30 && off > 0.20 && o.torsion_energy > 1.0 && dd < 0.5);
        const bool topo = (symr > 0.96 && off > 0.35 && dd < 0.95) || bal ||
                          (score >= thr && (rent < 0.92 || cent < 0.92) && mism < 0.22 && (torr < 0.62 || dent < 0.62) &&
                           rcv < 0.42 && ccv < 0.42);
        o.adaptive_route = n <= 4 ? 0 : off <= 1e-5 ? 1 : (n <= 64 && pf) ? 2 : (n <= 64 && topo) ? 3 : n <= 512 ? 1 : 4;
    }
    args.out[t] = o;
}

}  // namespace

extern "C" lsvd_status lsvd_triage_batched_f64(lsvd_context* ctx, int64_t count, const int32_t* rows,
                                               const int32_t* cols, const double* A, lsvd_triage* out,
                                               uint32_t flags) {
    LSVD_TRACE("lsvd_triage_batched_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (count < 0 || (count > 0 && (!rows || !cols || !A || !out)))
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_triage_batched_f64: bad pointer");
    if (count == 0) return LSVD_OK;
    if (count > (int64_t(1) << 30)) return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "triage: batch too large");
    std::vector<int64_t> aoff(static_cast<size_t>(count));
    int64_t tot = 0;
    int mr = 1, mc = 1;
    for (int64_t t = 0; t < count; ++t) {
        if (rows[t] < 0 || cols[t] < 0) return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "triage: negative size");
        if (rows[t] > kMaxDim || cols[t] > kMaxDim)
            return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "triage: rows and cols must be <= 4096");
        aoff[size_t(t)] = tot;
        tot += int64_t(rows[t]) * cols[t];
        mr = std::max(mr, int(rows[t]));
        mc = std::max(mc, int(cols[t]));
    }
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool dev = (flags & LSVD_DEVICE_POINTERS) != 0;
    cudaError_t e;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t b_meta = 2 * al(size_t(count) * 4) + al(size_t(count) * 8);
    const size_t b_out = al(size_t(count) * sizeof(lsvd_triage));
    char* meta = static_cast<char*>(ctx->ws_diag.get(b_meta + (dev ? 0 : b_out), &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "triage metadata");
    int32_t* d_rows = reinterpret_cast<int32_t*>(meta);
    int32_t* d_cols = reinterpret_cast<int32_t*>(meta + al(size_t(count) * 4));
    int64_t* d_aoff = reinterpret_cast<int64_t*>(meta + 2 * al(size_t(count) * 4));
    lsvd_triage* d_out = dev ? out : reinterpret_cast<lsvd_triage*>(meta + b_meta);
    const double* d_a = A;
    if (!dev) {
        double* stage = static_cast<double*>(ctx->ws_a.get(size_t(std::max<int64_t>(tot, 1)) * 8, &e));
        if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "triage staging");
        if (tot && (e = cudaMemcpyAsync(stage, A, size_t(tot) * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "triage copy A");
        d_a = stage;
    }
    if ((e = cudaMemcpyAsync(d_rows, rows, size_t(count) * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_cols, cols, size_t(count) * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_aoff, aoff.data(), size_t(count) * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "triage metadata upload");
    const int smem = (2 * mr + 2 * mc + std::min(mr, mc)) * 8;
    if ((e = cudaFuncSetAttribute(triage_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "triage smem attribute");
    TriageArgs args{int(count), d_rows, d_cols, d_aoff, d_a, d_out, mr, mc};
    triage_kernel<<<unsigned(count), TT, smem, st>>>(args);
    ctx->launches += 1;
    if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "triage launch");
    if (!dev && (e = cudaMemcpyAsync(out, d_out, size_t(count) * sizeof(lsvd_triage), cudaMemcpyDeviceToHost, st)) !=
                    cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "triage copy out");
    if (dev && (flags & LSVD_ASYNC)) return LSVD_OK;
    // the host arrays above (aoff) must outlive their copies
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "triage sync");
    return LSVD_OK;
}
