// lsvd_rect.cu -- LieSvdSmall::solve_rectangular (src/lie_svd_small.rs:340-360)
// for one m x d matrix with min(m, d) <= 64.
//
//   d == m : the square solve;
//   d >  m : SVD of A^T (read through strides, no copy), outputs swapped;
//   m >  d : qr_reduce (modified Gram-Schmidt, :373-418) -> square solve of
//            R (d x d) -> U = Q U_r.
#include <cuda_runtime.h>

#include "lsvd.h"
#include "lsvd_device.cuh"
#include "lsvd_internal.h"

namespace {

using lsvd::kCtaThreads;

__device__ double cta_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < kCtaThreads / 32; ++w) s += red[w];
    __syncthreads();
    return s;
}

// qr_reduce on X(i, j) = A[i*rs + j*cs], i < m, j < d (m >= d).  Q m x d and
// R d x d row-major.  Column j of X is staged in shared memory (m doubles).
__global__ void __launch_bounds__(kCtaThreads, 1)
    qr_reduce_kernel(int64_t m, int64_t d, const double* A, int64_t rs, int64_t cs, double* Q,
                     double* R) {
    extern __shared__ double v[];
    __shared__ double red[kCtaThreads / 32];
    double f2 = 0.0;
    for (int64_t idx = threadIdx.x; idx < m * d; idx += kCtaThreads) {
        const double x = A[(idx / d) * rs + (idx % d) * cs];
        f2 += x * x;
    }
    const double floor_ = 1e-10 * fmax(sqrt(cta_sum(f2, red)), 1e-300);
    for (int64_t j = 0; j < d; ++j) {
        for (int64_t i = threadIdx.x; i < m; i += kCtaThreads) v[i] = A[i * rs + j * cs];
        for (int64_t r = threadIdx.x; r < d; r += kCtaThreads)
            if (r > j) R[r * d + j] = 0.0;
        __syncthreads();
        for (int64_t k = 0; k < j; ++k) {
            double p = 0.0;
            for (int64_t i = threadIdx.x; i < m; i += kCtaThreads) p = fma(Q[i * d + k], v[i], p);
            const double dot = cta_sum(p, red);
            if (threadIdx.x == 0) R[k * d + j] = dot;
            for (int64_t i = threadIdx.x; i < m; i += kCtaThreads) v[i] -= dot * Q[i * d + k];
            __syncthreads();
        }
        double p = 0.0;
        for (int64_t i = threadIdx.x; i < m; i += kCtaThreads) p = fma(v[i], v[i], p);
        const double nrm = sqrt(cta_sum(p, red));
        if (threadIdx.x == 0) R[j * d + j] = nrm;
        for (int64_t i = threadIdx.x; i < m; i += kCtaThreads)
            Q[i * d + j] = nrm >= floor_ ? v[i] / nrm : 0.0;
        __syncthreads();
    }
}

// C (m x k, row-major, ldc) = Q (m x d) * B (d x k); C is written through
// strides (crs, ccs) so the transposed branch can store U^T / V directly.
__global__ void gemm_store_kernel(int64_t m, int64_t d, int64_t k, const double* Q,
                                  const double* B, double* C, int64_t crs, int64_t ccs) {
    const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= m * k) return;
    const int64_t i = idx / k, j = idx % k;
    double s = 0.0;
    for (int64_t q = 0; q < d; ++q) s = fma(Q[i * d + q], B[q * k + j], s);
    C[i * crs + j * ccs] = s;
}

__global__ void strided_copy_kernel(int64_t rows, int64_t cols, const double* src, int64_t srs,
                                    int64_t scs, double* dst, int64_t drs, int64_t dcs) {
    const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= rows * cols) return;
    const int64_t i = idx / cols, j = idx % cols;
    dst[i * drs + j * dcs] = src[i * srs + j * scs];
}

}  // namespace

extern "C" lsvd_status lsvd_small_solve_rectangular_f64(lsvd_context* ctx, int64_t m, int64_t d,
                                                        const double* A, int64_t lda, double* U,
                                                        int64_t ldu, double* S, double* Vt,
                                                        int64_t ldvt, lsvd_diag* diag,
                                                        uint32_t flags) {
    LSVD_TRACE("lsvd_small_solve_rectangular_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (m <= 0 || d <= 0)
        return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "LieSvdSmall::solve_rectangular: empty input");
    const int64_t k = m < d ? m : d;
    if (!A || !U || !S || !Vt || lda < d || ldu < k || ldvt < d)
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "solve_rectangular: bad pointer or leading dimension");
    if (k > lsvd::kMaxN) {
        // beyond the shared-memory kernels: the thin route of the large solve
        if (k > 16384 || (m > d ? m : d) > (int64_t(1) << 16))
            return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "solve_rectangular: larger than 65536 x 16384");
        cudaSetDevice(ctx->device);
        lsvd_diag hd;
        const lsvd_status st = lsvd_large_solve(ctx, m, d, A, lda, U, ldu, S, Vt, ldvt, LSVD_PREC_FP64, nullptr,
                                                &hd, (flags & LSVD_WANT_DIAG) != 0);
        if (diag && st != LSVD_CUDA_ERROR && st != LSVD_OUT_OF_MEMORY && st != LSVD_NONFINITE_INPUT) {
            if (flags & LSVD_DEVICE_POINTERS) {
                if (cudaMemcpy(diag, &hd, sizeof(hd), cudaMemcpyHostToDevice) != cudaSuccess)
                    return lsvd_ctx_fail(ctx, LSVD_CUDA_ERROR, "copy diag out");
            } else {
                *diag = hd;
            }
        }
        return st;
    }
    if ((m > d ? m : d) > (int64_t(1) << 24))
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "solve_rectangular: too many rows");
    if (m == d)
        return lsvd_single_small(ctx, m, A, lda, U, ldu, S, Vt, ldvt, diag, nullptr, 0, nullptr,
                                 nullptr, flags, 0, false);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool dev = (flags & LSVD_DEVICE_POINTERS) != 0;
    const bool wide = d > m;
    // tall view X (mm x dd) of the input: X = A, or X = A^T for the wide case
    const int64_t mm = wide ? d : m, dd = k;
    cudaError_t e;
    const size_t bx = size_t(m * d) * 8, bq = size_t(mm * dd) * 8, br = size_t(dd * dd) * 8;
    char* ws = static_cast<char*>(ctx->ws_rot.get(bx + bq + 3 * br + 4096, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "rect workspace");
    double* dA = reinterpret_cast<double*>(ws);
    double* dQ = reinterpret_cast<double*>(ws + bx);
    double* dR = reinterpret_cast<double*>(ws + bx + bq);
    double* dUr = dR + dd * dd;
    double* dVr = dUr + dd * dd;
    double* dS = dVr + dd * dd;
    // packed copy of A (m x d) regardless of pointer kind
    if ((e = cudaMemcpy2DAsync(dA, size_t(d) * 8, A, size_t(lda) * 8, size_t(d) * 8, size_t(m),
                               cudaMemcpyDefault, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "copy A");
    const int64_t rs = wide ? 1 : d, cs = wide ? d : 1;
    const size_t smem = size_t(mm) * 8;
    if (smem > 200 * 1024) return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "solve_rectangular: too many rows");
    if ((e = cudaFuncSetAttribute(qr_reduce_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem))) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "qr smem attribute");
    qr_reduce_kernel<<<1, kCtaThreads, smem, st>>>(mm, dd, dA, rs, cs, dQ, dR);
    ctx->launches++;
    if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "qr_reduce");
    // square solve of R (device pointers, synchronous)
    lsvd_diag local;
    lsvd_status s2 = lsvd_single_small(ctx, dd, dR, dd, dUr, dd, dS, dVr, dd, &local, nullptr, 0,
                                       nullptr, nullptr, LSVD_DEVICE_POINTERS | (flags & LSVD_WANT_DIAG), 0,
                                       true);
    if (s2 != LSVD_OK && s2 != LSVD_NOT_CONVERGED && s2 != LSVD_NONFINITE_INPUT) return s2;
    if (diag) {
        if (dev) {
            if ((e = cudaMemcpy(diag, &local, sizeof(local), cudaMemcpyHostToDevice)) != cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "copy diag out");
        } else {
            *diag = local;
        }
    }
    // outputs: tall: U = Q U_r (m x k), Vt = Vt_r (k x d)
    //          wide: SVD(A^T) = (Q U_r, s, Vt_r) -> U = Vt_r^T (m x m), Vt = (Q U_r)^T (k x d)
    double* outU = U;
    double* outV = Vt;
    double* tmp = nullptr;
    if (!dev) {
        tmp = static_cast<double*>(ctx->ws_u.get(size_t(m * k + k * d) * 8 + 64, &e));
        if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "rect out");
        outU = tmp;
        outV = tmp + m * k;
    }
    const int64_t lu = dev ? ldu : k, lv = dev ? ldvt : d;
    const int blk = 256;
    if (!wide) {
        gemm_store_kernel<<<unsigned((mm * dd + blk - 1) / blk), blk, 0, st>>>(mm, dd, dd, dQ, dUr, outU, lu, 1);
        strided_copy_kernel<<<unsigned((dd * dd + blk - 1) / blk), blk, 0, st>>>(dd, dd, dVr, dd, 1, outV, lv, 1);
    } else {
        gemm_store_kernel<<<unsigned((mm * dd + blk - 1) / blk), blk, 0, st>>>(mm, dd, dd, dQ, dUr, outV, 1, lv);
        strided_copy_kernel<<<unsigned((dd * dd + blk - 1) / blk), blk, 0, st>>>(dd, dd, dVr, dd, 1, outU, 1, lu);
    }
    ctx->launches += 2;
    if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "rect outputs");
    if ((e = cudaMemcpyAsync(S, dS, size_t(k) * 8, cudaMemcpyDefault, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "copy S");
    if (!dev) {
        if ((e = cudaMemcpy2DAsync(U, size_t(ldu) * 8, outU, size_t(k) * 8, size_t(k) * 8, size_t(m),
                                   cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpy2DAsync(Vt, size_t(ldvt) * 8, outV, size_t(d) * 8, size_t(d) * 8, size_t(k),
                                   cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "copy out");
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "sync");
    return s2;
}
