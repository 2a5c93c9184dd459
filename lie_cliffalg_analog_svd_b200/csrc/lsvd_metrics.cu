// lsvd_metrics.cu -- metrics::compute (src/lib.rs:149-194) on the device.
//
// rel_recon = ||U diag(S) Vt - A||_F / max(||A||_F, 1e-300)
// orth_u    = ||U^T U - I||_F ,  orth_v = ||Vt Vt^T - I||_F
// sigma_max_rel / sigma_tail_rel over both spectra sorted descending, the
// tail starting at index 3k/4.  Written for the general thin shape (A m*d,
// U m*k, Vt k*d); on square input this is the reference formula exactly.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "lsvd.h"
#include "lsvd_internal.h"

namespace {

constexpr int kThreads = 256;

__device__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kThreads / 32; ++i) s += red[i];
    __syncthreads();
    return s;
}

// part[blockIdx.x * 4 + {0,1,2,3}] = partial sums of recon^2, A^2, Gu^2, Gv^2.
__global__ void metrics_partial(int64_t m, int64_t d, int64_t k, const double* A, const double* U,
                                const double* S, const double* Vt, double* part) {
    __shared__ double red[kThreads / 32];
    double r2 = 0.0, a2 = 0.0, u2 = 0.0, v2 = 0.0;
    const int64_t stride = int64_t(gridDim.x) * kThreads;
    const int64_t t0 = int64_t(blockIdx.x) * kThreads + threadIdx.x;
    for (int64_t idx = t0; idx < m * d; idx += stride) {
        const int64_t i = idx / d, j = idx % d;
        double rec = 0.0;
        for (int64_t q = 0; q < k; ++q) rec = fma(U[i * k + q] * S[q], Vt[q * d + j], rec);
        const double a = A[i * d + j];
        r2 += (rec - a) * (rec - a);
        a2 += a * a;
    }
    for (int64_t idx = t0; idx < k * k; idx += stride) {
        const int64_t i = idx / k, j = idx % k;
        double gu = 0.0, gv = 0.0;
        for (int64_t q = 0; q < m; ++q) gu = fma(U[q * k + i], U[q * k + j], gu);
        for (int64_t q = 0; q < d; ++q) gv = fma(Vt[i * d + q], Vt[j * d + q], gv);
        const double e = (i == j) ? 1.0 : 0.0;
        u2 += (gu - e) * (gu - e);
        v2 += (gv - e) * (gv - e);
    }
    r2 = block_sum(r2, red);
    a2 = block_sum(a2, red);
    u2 = block_sum(u2, red);
    v2 = block_sum(v2, red);
    if (threadIdx.x == 0) {
        part[blockIdx.x * 4 + 0] = r2;
        part[blockIdx.x * 4 + 1] = a2;
        part[blockIdx.x * 4 + 2] = u2;
        part[blockIdx.x * 4 + 3] = v2;
    }
}

// Final reduction + sigma errors (rank sort, descending, stable) in one block.
__global__ void metrics_final(int nblocks, int64_t k, const double* part, const double* S,
                              const double* ref, double* out) {
    __shared__ double red[kThreads / 32];
    double acc[4] = {0, 0, 0, 0};
    for (int b = 0; b < nblocks; ++b)
        for (int q = 0; q < 4; ++q) acc[q] += part[b * 4 + q];
    double mx = 0.0, tail = 0.0;
    if (ref) {
        const int64_t tail_start = (k * 3) / 4;
        for (int64_t i = threadIdx.x; i < k; i += kThreads) {
            // i-th largest of each spectrum
            double gi = 0.0, wi = 0.0;
            for (int64_t c = 0; c < k; ++c) {
                int64_t rg = 0, rw = 0;
                for (int64_t q = 0; q < k; ++q) {
                    rg += (S[q] > S[c]) || (S[q] == S[c] && q < c);
                    rw += (ref[q] > ref[c]) || (ref[q] == ref[c] && q < c);
                }
                if (rg == i) gi = S[c];
                if (rw == i) wi = ref[c];
            }
            const double r = fabs(gi - wi) / fmax(fabs(wi), 1e-300);
            if (!isnan(r)) {
                mx = fmax(mx, r);
                if (i >= tail_start) tail = fmax(tail, r);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        tail = fmax(tail, __shfl_xor_sync(0xffffffffu, tail, o));
    }
    __shared__ double smx[kThreads / 32], stl[kThreads / 32];
    if (threadIdx.x % 32 == 0) {
        smx[threadIdx.x / 32] = mx;
        stl[threadIdx.x / 32] = tail;
    }
    __syncthreads();
    (void)red;
    if (threadIdx.x == 0) {
        for (int w = 0; w < kThreads / 32; ++w) {
            mx = fmax(mx, smx[w]);
            tail = fmax(tail, stl[w]);
        }
        out[0] = sqrt(acc[0]) / fmax(sqrt(acc[1]), 1e-300);
        out[1] = sqrt(acc[2]);
        out[2] = sqrt(acc[3]);
        const double qnan = __longlong_as_double(0x7ff8000000000000ULL);
        out[3] = ref ? mx : qnan;
        out[4] = ref ? tail : qnan;
    }
}

}  // namespace

extern "C" lsvd_status lsvd_metrics_f64(lsvd_context* ctx, int64_t m, int64_t d, int64_t k,
                                        const double* A, const double* U, const double* S,
                                        const double* Vt, const double* sigma_ref, double* out,
                                        uint32_t flags) {
    LSVD_TRACE("lsvd_metrics_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (m <= 0 || d <= 0 || k <= 0 || k > (m < d ? m : d))
        return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "lsvd_metrics_f64: bad shape");
    if (!A || !U || !S || !Vt || !out) return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "null pointer");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool dev = (flags & LSVD_DEVICE_POINTERS) != 0;
    cudaError_t e;
    const size_t ba = size_t(m * d) * 8, bu = size_t(m * k) * 8, bs = size_t(k) * 8,
                 bv = size_t(k * d) * 8;
    const int nblocks = int(std::min<int64_t>(2 * ctx->num_sms, (m * d + kThreads - 1) / kThreads + 1));
    char* ws = static_cast<char*>(ctx->ws_diag.get(ba + bu + 2 * bs + bv + size_t(nblocks) * 32 + 64 + 1024, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "metrics workspace");
    const double *dA = A, *dU = U, *dS = S, *dV = Vt, *dR = sigma_ref;
    char* p = ws;
    if (!dev) {
        double* hA = reinterpret_cast<double*>(p); p += ba;
        double* hU = reinterpret_cast<double*>(p); p += bu;
        double* hS = reinterpret_cast<double*>(p); p += bs;
        double* hV = reinterpret_cast<double*>(p); p += bv;
        double* hR = reinterpret_cast<double*>(p); p += bs;
        if ((e = cudaMemcpyAsync(hA, A, ba, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(hU, U, bu, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(hS, S, bs, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(hV, Vt, bv, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (sigma_ref && (e = cudaMemcpyAsync(hR, sigma_ref, bs, cudaMemcpyHostToDevice, st)) != cudaSuccess))
            return lsvd_ctx_cuda(ctx, e, "metrics copy");
        dA = hA; dU = hU; dS = hS; dV = hV; dR = sigma_ref ? hR : nullptr;
    } else {
        p += ba + bu + 2 * bs + bv;
    }
    p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 255) & ~uintptr_t(255));
    double* part = reinterpret_cast<double*>(p);
    double* dout = part + size_t(nblocks) * 4;
    metrics_partial<<<nblocks, kThreads, 0, st>>>(m, d, k, dA, dU, dS, dV, part);
    metrics_final<<<1, kThreads, 0, st>>>(nblocks, k, part, dS, dR, dout);
    ctx->launches += 2;
    if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "metrics launch");
    if ((e = cudaMemcpyAsync(out, dout, 5 * 8, cudaMemcpyDefault, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "metrics out");
    if (!(dev && (flags & LSVD_ASYNC)) && (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "metrics sync");
    return LSVD_OK;
}
