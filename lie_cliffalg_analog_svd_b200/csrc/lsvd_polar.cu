// lsvd_polar.cu -- Newton-Schulz polar factor of a large m x n matrix
// (newton_schulz_polar, src/lie_svd_small.rs:158-183, generalised to m >= n)
// in three precisions:
//   FP64       : X <- 0.5 X (3I - X^T X) from X0 = A/||A||_F with FP64 GEMMs
//                on the FP64 tensor path (lsvd_dgemm.cuh, mma.sync m8n8k4)
//                and the reference's stopping rule (delta < 1e-13 sqrt(n),
//                cap 120);
//   TF32, BF16 : the same iteration on tensor cores (lsvd_tcgemm.cuh,
//                tcgen05, FP32 accumulation) until the update reaches the
//                low-precision floor, then FP64 refinement iterations until
//                delta < 1e-13 sqrt(n).
// The refinement restores orthogonality to working precision, but it
// converges to the polar factor of the low-precision iterate: rounding in the
// TF32/BF16 products perturbs X at ~u_lo ||X|| in every direction, so the
// mixed result differs from A's polar factor by about u_lo sqrt(n) in
// Frobenius norm (u_lo = 2^-11 TF32, 2^-8 BF16), more where A's singular
// values fall below ~u_lo sigma_1.  The FP64 path has no such floor.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <vector>

#include "lsvd.h"
#include "lsvd_dgemm.cuh"
#include "lsvd_internal.h"
#include "lsvd_tcgemm.cuh"

namespace {

using namespace lsvd::tc;

__device__ __forceinline__ float round_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Low-precision operand store: BF16 (2 bytes) or TF32-rounded FP32 (4 bytes).
template <int PREC>
__device__ __forceinline__ void store_lo(void* base, size_t idx, float v) {
    if (PREC == kBF16)
        reinterpret_cast<__nv_bfloat16*>(base)[idx] = __float2bfloat16_rn(v);
    else
        reinterpret_cast<float*>(base)[idx] = round_tf32(v);
}

// X (m x n, FP32) = A / ||A||_F; Xlo = lo(X); Xt = lo(X)^T (n x m).
// Also: the NS update X <- 1.5 X - 0.5 Y when Y != nullptr, with the squared
// update norm accumulated per block into part[b] and the squared norm of the
// new X into part[nblocks + b].  32x32 tiles through shared memory make the
// transposed store coalesced.
template <int PREC>
__global__ void ns_update_kernel(int m, int n, float* X, const float* Y, const double* A, int lda,
                                 double inv_scale, void* Xlo, void* Xt, double* part) {
    __shared__ float tile[32][33];
    __shared__ double red[8], redx[8];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // bx: column, by: row
    const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 32 x 8 threads
    double d2 = 0.0, x2 = 0.0;
    for (int r = ty; r < 32; r += 8) {
        const int i = by + r, j = bx + tx;
        const size_t e = size_t(i) * n + j;
        float x;
        if (Y) {
            const float x0 = X[e];
            x = 1.5f * x0 - 0.5f * Y[e];
            d2 += double(x - x0) * double(x - x0);
        } else {
            x = float(A[size_t(i) * lda + j] * inv_scale);
        }
        X[e] = x;
        x2 += double(x) * double(x);
        store_lo<PREC>(Xlo, e, x);
        tile[r][tx] = x;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int j = bx + r, i = by + tx;  // transposed: row j of X^T, column i
        store_lo<PREC>(Xt, size_t(j) * m + i, tile[tx][r]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        d2 += __shfl_xor_sync(0xffffffffu, d2, o);
        x2 += __shfl_xor_sync(0xffffffffu, x2, o);
    }
    if (tx == 0) {
        red[ty] = d2;
        redx[ty] = x2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0, sx = 0.0;
        for (int w = 0; w < 8; ++w) {
            s += red[w];
            sx += redx[w];
        }
        const int b = blockIdx.y * gridDim.x + blockIdx.x;
        part[b] = s;
        part[gridDim.x * gridDim.y + b] = sx;
    }
}

template <int PREC>
__global__ void to_lo_kernel(size_t count, const float* src, void* dst) {
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < count;
         e += size_t(gridDim.x) * blockDim.x)
        store_lo<PREC>(dst, e, src[e]);
}

__global__ void sum_kernel(int count, const double* part, double* out) {
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

__global__ void frob2_kernel(int m, int n, const double* A, int64_t lda, double* part) {
    __shared__ double red[256];
    double s = 0.0;
    const size_t tot = size_t(m) * n;
    for (size_t e = blockIdx.x * size_t(256) + threadIdx.x; e < tot; e += size_t(gridDim.x) * 256) {
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

// FP64: X <- 1.5 X - 0.5 Y over the whole padded buffer (padding columns are
// zero in X and Y and stay zero), squared update norm per block.
__global__ void ns_update64_kernel(size_t count, double* X, const double* Y, double* part) {
    __shared__ double red[256];
    double s = 0.0;
    for (size_t e = blockIdx.x * size_t(256) + threadIdx.x; e < count; e += size_t(gridDim.x) * 256) {
        const double x0 = X[e];
        const double x = 0.5 * (3.0 * x0 - Y[e]);
        X[e] = x;
        s += (x - x0) * (x - x0);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// X (m x ld, padding columns zero) = A (m x n, lda) * inv.
__global__ void scale64_kernel(int m, int n, const double* A, int64_t lda, double inv, double* X, int64_t ld) {
    const size_t tot = size_t(m) * ld;
    for (size_t e = blockIdx.x * size_t(256) + threadIdx.x; e < tot; e += size_t(gridDim.x) * 256) {
        const size_t i = e / ld, j = e % ld;
        X[e] = j < size_t(n) ? A[i * lda + j] * inv : 0.0;
    }
}

__global__ void widen_kernel(int m, int n, const float* X32, double* X64, int64_t ld) {
    const size_t tot = size_t(m) * ld;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < tot;
         e += size_t(gridDim.x) * blockDim.x) {
        const size_t i = e / ld, j = e % ld;
        X64[e] = j < size_t(n) ? double(X32[i * n + j]) : 0.0;
    }
}

// ||T - I||_F^2 partials (T n x n with leading dimension ld).
__global__ void orth2_kernel(int n, const double* T, int64_t ld, double* part) {
    __shared__ double red[256];
    double s = 0.0;
    const size_t tot = size_t(n) * n;
    for (size_t e = blockIdx.x * size_t(256) + threadIdx.x; e < tot; e += size_t(gridDim.x) * 256) {
        const size_t i = e / n, j = e % n;
        const double d = T[i * ld + j] - (i == j ? 1.0 : 0.0);
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

// cuTensorMapEncodeTiled through the runtime's driver entry point, so the
// library does not link libcuda directly (it loads on hosts without a driver).
typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                             const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                             CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                             CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
    static EncodeFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeFn>(p);
    }();
    return fn;
}

// 2-D K-major map: rows x cols (cols = K contiguous), box box_rows x 128 bytes.
bool make_map(CUtensorMap* map, int prec, const void* ptr, int rows, int cols, int box_rows) {
    EncodeFn fn = encode_fn();
    if (!fn) return false;
    const int elem = prec == kBF16 ? 2 : 4;
    cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
    cuuint64_t strides[1] = {cuuint64_t(cols) * elem};
    cuuint32_t box[2] = {cuuint32_t(kSliceBytes / elem), cuuint32_t(box_rows)};
    cuuint32_t es[2] = {1, 1};
    return fn(map, prec == kBF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
              const_cast<void*>(ptr), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int PREC, int TN>
cudaError_t launch_gemm_t(cudaStream_t st, const void* A, const void* B, float* C, int M, int N, int K,
                          int* err) {
    CUtensorMap ma, mb;
    if (!make_map(&ma, PREC, A, M, K, kTile) || !make_map(&mb, PREC, B, N, K, TN))
        return cudaErrorInvalidValue;
    // the persistent kernel (one CTA per SM, two TMEM accumulators, epilogue beside the next
    // tile's main loop); LSVD_TC_GEMM_SIMPLE=1 selects the one-tile-per-CTA kernel
    static const bool simple = [] {
        const char* v = std::getenv("LSVD_TC_GEMM_SIMPLE");
        return v && v[0] == '1';
    }();
    cudaError_t e;
    if (simple) {
        e = cudaFuncSetAttribute(tc_gemm_kernel<PREC, TN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem_bytes(TN));
        if (e != cudaSuccess) return e;
        tc_gemm_kernel<PREC, TN><<<dim3(N / TN, M / kTile), 128, smem_bytes(TN), st>>>(ma, mb, C, N, K, err);
        return cudaGetLastError();
    }
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    e = cudaFuncSetAttribute(tc_gemm_persistent_kernel<PREC, TN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem_bytes(TN));
    if (e != cudaSuccess) return e;
    const int tiles = (M / kTile) * (N / TN);
    tc_gemm_persistent_kernel<PREC, TN><<<std::max(1, std::min(tiles, sms)), 192, smem_bytes(TN), st>>>(
        ma, mb, C, N, M, N, K, err);
    return cudaGetLastError();
}

// 128 x 256 tiles where N allows them (half the A traffic per flop), else 128 x 128.
template <int PREC>
cudaError_t launch_gemm(cudaStream_t st, const void* A, const void* B, float* C, int M, int N, int K,
                        int* err) {
    return N % 256 == 0 ? launch_gemm_t<PREC, 256>(st, A, B, C, M, N, K, err)
                        : launch_gemm_t<PREC, kTile>(st, A, B, C, M, N, K, err);
}

// Start/stop events around the GEMM launches of one iteration; the summed
// durations are read after the iteration's own synchronisation.
struct GemmTimer {
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    double ms = 0.0;
    bool ok = true;
    GemmTimer() {
        for (auto& e : ev)
            if (cudaEventCreate(&e) != cudaSuccess) ok = false;
    }
    ~GemmTimer() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
    void mark(int i, cudaStream_t st) {
        if (ok) cudaEventRecord(ev[i], st);
    }
    void accumulate() {  // after the stream synchronised
        float a = 0.f, b = 0.f;
        if (ok && cudaEventElapsedTime(&a, ev[0], ev[1]) == cudaSuccess &&
            cudaEventElapsedTime(&b, ev[2], ev[3]) == cudaSuccess)
            ms += double(a) + double(b);
    }
};

}  // namespace

extern "C" lsvd_status lsvd_gemm_nt_lowp(lsvd_context* ctx, int64_t M, int64_t N, int64_t K,
                                         const float* A, const float* B, float* C,
                                         lsvd_precision precision) {
    LSVD_TRACE("lsvd_gemm_nt_lowp");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (precision != LSVD_PREC_MIXED_TF32 && precision != LSVD_PREC_MIXED_BF16)
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_gemm_nt_lowp: precision must be TF32 or BF16");
    const int prec = precision == LSVD_PREC_MIXED_BF16 ? kBF16 : kTF32;
    const int kq = kSliceBytes / (prec == kBF16 ? 2 : 4);
    if (M <= 0 || N <= 0 || K <= 0 || M % kTile || N % kTile || K % kq || M > (1 << 20) ||
        N > (1 << 20) || K > (1 << 24))
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "lsvd_gemm_nt_lowp: M, N multiples of 128, K of the slice");
    if (!A || !B || !C) return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "null pointer");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    const size_t ea = size_t(M) * K, eb = size_t(N) * K;
    const size_t esz = prec == kBF16 ? 2 : 4;
    char* ws = static_cast<char*>(ctx->ws_a.get((ea + eb) * esz + 1024 + 16, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "gemm workspace");
    void* alo = ws;
    void* blo = ws + ((ea * esz + 255) & ~size_t(255));
    int* err = reinterpret_cast<int*>(static_cast<char*>(ws) + ctx->ws_a.bytes - 16);
    cudaMemsetAsync(err, 0, 4, st);
    if (prec == kBF16) {
        to_lo_kernel<kBF16><<<1024, 256, 0, st>>>(ea, A, alo);
        to_lo_kernel<kBF16><<<1024, 256, 0, st>>>(eb, B, blo);
        e = launch_gemm<kBF16>(st, alo, blo, C, int(M), int(N), int(K), err);
    } else {
        to_lo_kernel<kTF32><<<1024, 256, 0, st>>>(ea, A, alo);
        to_lo_kernel<kTF32><<<1024, 256, 0, st>>>(eb, B, blo);
        e = launch_gemm<kTF32>(st, alo, blo, C, int(M), int(N), int(K), err);
    }
    ctx->launches += 3;
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "tc gemm launch");
    int herr = 0;
    if ((e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "tc gemm sync");
    if (herr) return lsvd_ctx_fail(ctx, LSVD_CUDA_ERROR, "tc gemm: pipeline wait timed out");
    return LSVD_OK;
}

// C = alpha * (sum over z < parts of W[z], each M x N with row stride N) + beta C,
// one thread per element (consecutive threads on consecutive columns).
__global__ void splitk_reduce_kernel(const double* __restrict__ W, int parts, int64_t M, int64_t N, double alpha,
                                     double beta, double* __restrict__ C, int64_t ldc) {
    const int64_t mn = M * N;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < mn; i += int64_t(gridDim.x) * blockDim.x) {
        double s = 0.0;
        for (int z = 0; z < parts; ++z) s += W[z * mn + i];
        const int64_t r = i / N;
        double* c = C + r * ldc + (i - r * N);
        const double v = alpha * s;
        *c = beta == 0.0 ? v : v + beta * *c;
    }
}

// Partial products C_z = A_z B_z^T of a split inner dimension for small outputs
// (M, N <= 16 T; A row-major M x K, B row-major N x K): CTA z accumulates the K
// columns [z Kc, min(K, (z + 1) Kc)) with CUDA-core FMAs -- an M x N output on
// 128-wide tensor tiles would waste most of each tile -- and writes its M x N
// partial to W + z M N (row stride N).  256 threads as 16 x 16, each owning a
// T x T block of C.  Slabs of BK = 2048 / (16 T) columns are staged k-major in
// shared memory (a warp's reads of A broadcast, its reads of B are
// consecutive); each thread holds its 8 + 8 elements of the next slab in
// registers while the current slab is multiplied.
template <int T>
__global__ void __launch_bounds__(256) gram_slices_kernel(const double* __restrict__ A, int64_t lda,
                                                          const double* __restrict__ B, int64_t ldb, int M, int N,
                                                          int64_t K, int64_t Kc, double* __restrict__ W) {
    constexpr int R = 16 * T, BK = 2048 / R, PER = R * BK / 256;  // PER = 8
    static_assert(BK >= 32 && PER * 256 == R * BK, "slab shape");
    __shared__ double As[BK][R + 1];
    __shared__ double Bs[BK][R + 1];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int64_t k0 = int64_t(blockIdx.x) * Kc, k1 = k0 + Kc < K ? k0 + Kc : K;
    double acc[T][T];
#pragma unroll
    for (int i = 0; i < T; ++i)
#pragma unroll
        for (int j = 0; j < T; ++j) acc[i][j] = 0.0;
    double ra[PER], rb[PER];
    auto fetch = [&](int64_t kb) {
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int e = tid + 256 * q, r = e / BK, c = e - r * BK;  // a warp: 32 consecutive columns of a row
            const int64_t k = kb + c;
            ra[q] = (r < M && k < k1) ? A[r * lda + k] : 0.0;
            rb[q] = (r < N && k < k1) ? B[r * ldb + k] : 0.0;
        }
    };
    fetch(k0);
    for (int64_t kb = k0; kb < k1; kb += BK) {
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int e = tid + 256 * q, r = e / BK, c = e - r * BK;
            As[c][r] = ra[q];
            Bs[c][r] = rb[q];
        }
        __syncthreads();
        if (kb + BK < k1) fetch(kb + BK);
#pragma unroll 8
        for (int c = 0; c < BK; ++c) {
            double a[T], b[T];
#pragma unroll
            for (int i = 0; i < T; ++i) a[i] = As[c][ty * T + i];
#pragma unroll
            for (int j = 0; j < T; ++j) b[j] = Bs[c][tx * T + j];
#pragma unroll
            for (int i = 0; i < T; ++i)
#pragma unroll
                for (int j = 0; j < T; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
    double* Wz = W + int64_t(blockIdx.x) * M * N;
#pragma unroll
    for (int i = 0; i < T; ++i) {
        const int r = ty * T + i;
#pragma unroll
        for (int j = 0; j < T; ++j) {
            const int c = tx * T + j;
            if (r < M && c < N) Wz[int64_t(r) * N + c] = acc[i][j];
        }
    }
}

extern "C" lsvd_status lsvd_gemm_f64(lsvd_context* ctx, int32_t trans_a, int32_t trans_b, int64_t M,
                                     int64_t N, int64_t K, double alpha, const double* A, int64_t lda,
                                     const double* B, int64_t ldb, double beta, double* C, int64_t ldc) {
    LSVD_TRACE("lsvd_gemm_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (M < 0 || N < 0 || K < 0 || M > (1 << 24) || N > (1 << 24) || K > (1 << 24))
        return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "lsvd_gemm_f64: bad sizes");
    if (!A || !B || !C || ldc < N || lda < (trans_a ? M : K) || ldb < (trans_b ? K : N))
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_gemm_f64: bad pointer or leading dimension");
    if ((lda | ldb) & 1 || (reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "lsvd_gemm_f64: lda, ldb even and A, B 16-byte aligned");
    cudaSetDevice(ctx->device);
    // A B^T with both output dimensions <= 64 over a long inner dimension (a
    // covariance of a few channels over many samples): CUDA-core slices of at
    // least 1024 columns, up to four per SM, then the reduction below.
    if (!trans_a && trans_b && M > 0 && N > 0 && M <= 64 && N <= 64 && K >= 4096) {
        const int64_t S = std::min<int64_t>(4 * int64_t(ctx->num_sms), (K + 1023) / 1024);
        const int64_t Kc = (K + S - 1) / S, parts = (K + Kc - 1) / Kc, mn = M * N;
        cudaError_t e = cudaSuccess;
        double* W = static_cast<double*>(ctx->ws_splitk.get(size_t(parts) * size_t(mn) * 8, &e));
        if (!W) return lsvd_ctx_cuda(ctx, e, "lsvd_gemm_f64: split-K workspace");
        const int mx = int(std::max(M, N));
        const unsigned g = unsigned(parts);
        if (mx <= 16)
            gram_slices_kernel<1><<<g, 256, 0, ctx->stream>>>(A, lda, B, ldb, int(M), int(N), K, Kc, W);
        else if (mx <= 32)
            gram_slices_kernel<2><<<g, 256, 0, ctx->stream>>>(A, lda, B, ldb, int(M), int(N), K, Kc, W);
        else
            gram_slices_kernel<4><<<g, 256, 0, ctx->stream>>>(A, lda, B, ldb, int(M), int(N), K, Kc, W);
        const int blocks = int(std::min<int64_t>((mn + 255) / 256, 4 * int64_t(ctx->num_sms)));
        splitk_reduce_kernel<<<blocks, 256, 0, ctx->stream>>>(W, int(parts), M, N, alpha, beta, C, ldc);
        ctx->launches += 2;
        return lsvd_ctx_cuda(ctx, cudaGetLastError(), "lsvd_gemm_f64: small-output slices");
    }
    // Few output tiles over a long inner dimension (a Gram or covariance of a
    // few rows over many samples): one CTA per tile would walk all of K alone.
    // Split K into S even slices run as one batched launch into the context's
    // workspace (slice z reads A and B from column / row z * Kc on), the
    // remainder as one more product, then C = alpha * (sum of the partials) + beta C.
    const int64_t tiles = ((M + 127) / 128) * ((N + 63) / 64);
    const int64_t S = std::min<int64_t>(2 * ctx->num_sms / std::max<int64_t>(tiles, 1), K / 2048);
    if (S >= 2 && M > 0 && N > 0) {
        const int64_t Kc = (K / S) & ~int64_t(1), Kr = K - S * Kc, mn = M * N;
        const int parts = int(S + (Kr > 0 ? 1 : 0));
        cudaError_t e = cudaSuccess;
        double* W = static_cast<double*>(ctx->ws_splitk.get(size_t(parts) * size_t(mn) * 8, &e));
        if (!W) return lsvd_ctx_cuda(ctx, e, "lsvd_gemm_f64: split-K workspace");
        const int64_t sA = trans_a ? Kc * lda : Kc, sB = trans_b ? Kc : Kc * ldb;
        e = lsvd::dg::dgemm(ctx->stream, trans_a != 0, trans_b != 0, int(M), int(N), int(Kc), 1.0, A, lda, B, ldb,
                            0.0, W, N, int(S), sA, sB, mn);
        if (e == cudaSuccess && Kr > 0)
            e = lsvd::dg::dgemm(ctx->stream, trans_a != 0, trans_b != 0, int(M), int(N), int(Kr), 1.0,
                                A + S * sA, lda, B + S * sB, ldb, 0.0, W + S * mn, N);
        if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "lsvd_gemm_f64: split-K slices");
        const int blocks = int(std::min<int64_t>((mn + 255) / 256, 4 * int64_t(ctx->num_sms)));
        splitk_reduce_kernel<<<blocks, 256, 0, ctx->stream>>>(W, parts, M, N, alpha, beta, C, ldc);
        ctx->launches += 2 + (Kr > 0 ? 1 : 0);
        return lsvd_ctx_cuda(ctx, cudaGetLastError(), "lsvd_gemm_f64: split-K reduction");
    }
    cudaError_t e = lsvd::dg::dgemm(ctx->stream, trans_a != 0, trans_b != 0, int(M), int(N), int(K), alpha, A,
                                    lda, B, ldb, beta, C, ldc);
    ctx->launches += 1;
    return lsvd_ctx_cuda(ctx, e, "lsvd_gemm_f64");
}

lsvd_status lsvd_polar_run(lsvd_context* ctx, int64_t m, int64_t n, const double* A, int64_t lda,
                           lsvd_precision precision, int fp64_cap, double** Xout, int64_t* ldx_out,
                           lsvd_polar_info* info) {
    LSVD_TRACE("polar/newton_schulz");
    const bool lowp = precision == LSVD_PREC_MIXED_TF32 || precision == LSVD_PREC_MIXED_BF16;
    if (lowp && (m % kTile || n % kTile))
        return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "polar: TF32/BF16 need m, n multiples of 128");
    if (m * n > (int64_t(1) << 31)) return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "polar: too large");
    cudaStream_t st = ctx->stream;
    const int64_t ld = (n + 7) & ~int64_t(7);  // FP64 buffers: even leading dimension for the GEMMs
    const size_t mn = size_t(m) * ld, nn = size_t(ld) * ld;
    const size_t mn32 = size_t(m) * n, nn32 = size_t(n) * n;
    const int prec = precision == LSVD_PREC_MIXED_BF16 ? kBF16 : kTF32;
    const size_t lo = prec == kBF16 ? 2 : 4;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    // workspace: A64 | X64 | Y64 | T64 | part | (X32 | Y32 | T32 | Xlo | Xt | Tlo | err)
    const int nparts = 4096;
    size_t bytes = al(mn * 8) * 3 + al(nn * 8) + al(nparts * 8) + 64;
    if (lowp) bytes += al(mn32 * 4) * 2 + al(nn32 * 4) + al(mn32 * lo) * 2 + al(nn32 * lo) + 64;
    cudaError_t e;
    char* ws = static_cast<char*>(ctx->ws_polar.get(bytes, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "polar workspace");
    char* p = ws;
    double* A64 = reinterpret_cast<double*>(p); p += al(mn * 8);
    double* X64 = reinterpret_cast<double*>(p); p += al(mn * 8);
    double* Y64 = reinterpret_cast<double*>(p); p += al(mn * 8);
    double* T64 = reinterpret_cast<double*>(p); p += al(nn * 8);
    double* part = reinterpret_cast<double*>(p); p += al(nparts * 8);
    double* dsum = reinterpret_cast<double*>(p); p += 64;
    // padding columns of the FP64 buffers must read as zero: the GEMMs write
    // only the n valid columns, and the update and its norm run over the
    // whole padded buffer
    if ((e = cudaMemsetAsync(Y64, 0, mn * 8, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(T64, 0, nn * 8, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(A64, 0, mn * 8, st)) != cudaSuccess ||
        (e = cudaMemcpy2DAsync(A64, size_t(ld) * 8, A, size_t(lda) * 8, size_t(n) * 8, size_t(m),
                               cudaMemcpyDefault, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "polar copy A");
    const double refn = std::sqrt(double(n));
    auto read_sum = [&](int count, double* out) -> cudaError_t {
        sum_kernel<<<1, 256, 0, st>>>(count, part, dsum);
        cudaError_t ee = cudaMemcpyAsync(out, dsum, 8, cudaMemcpyDeviceToHost, st);
        if (ee == cudaSuccess) ee = cudaStreamSynchronize(st);
        return ee;
    };
    frob2_kernel<<<1024, 256, 0, st>>>(int(m), int(n), A64, ld, part);
    double f2 = 0.0;
    if ((e = read_sum(1024, &f2)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "polar norm");
    const double inv = 1.0 / std::max(std::sqrt(f2), 1e-300);
    int it_lo = 0, it_hi = 0;
    double flops_lo = 0.0, flops_hi = 0.0;
    GemmTimer tlo, thi;
    if (lowp) {
        float* X32 = reinterpret_cast<float*>(p); p += al(mn32 * 4);
        float* Y32 = reinterpret_cast<float*>(p); p += al(mn32 * 4);
        float* T32 = reinterpret_cast<float*>(p); p += al(nn32 * 4);
        void* Xlo = p; p += al(mn32 * lo);
        void* Xt = p; p += al(mn32 * lo);
        void* Tlo = p; p += al(nn32 * lo);
        int* err = reinterpret_cast<int*>(p);
        cudaMemsetAsync(err, 0, 4, st);
        const dim3 ug(unsigned(n / 32), unsigned(m / 32));
        const int nub = int(ug.x * ug.y);
        double* upart = Y64;  // Y64 is unused in the low-precision phase: 2 partials per block
        if (prec == kBF16)
            ns_update_kernel<kBF16><<<ug, 256, 0, st>>>(int(m), int(n), X32, nullptr, A64, int(ld), inv, Xlo, Xt, upart);
        else
            ns_update_kernel<kTF32><<<ug, 256, 0, st>>>(int(m), int(n), X32, nullptr, A64, int(ld), inv, Xlo, Xt, upart);
        // Stop the low-precision phase when the relative update
        // delta/||X||_F reaches a few units of the low precision: beyond it
        // the iterate only moves by rounding noise, and from there the FP64
        // iteration is in its quadratic regime (e <- 1.5 e^2).
        const double floor_rel = prec == kBF16 ? 8 * 3.90625e-3 : 8 * 4.8828125e-4;
        for (int it = 0; it < 100; ++it) {
            // T = X^T X = Xt Xt^T (n x n, K = m); Y = X T = Xlo T^T (m x n, K = n)
            if (prec == kBF16) {
                tlo.mark(0, st);
                e = launch_gemm<kBF16>(st, Xt, Xt, T32, int(n), int(n), int(m), err);
                tlo.mark(1, st);
                if (e == cudaSuccess) to_lo_kernel<kBF16><<<1024, 256, 0, st>>>(nn32, T32, Tlo);
                tlo.mark(2, st);
                if (e == cudaSuccess) e = launch_gemm<kBF16>(st, Xlo, Tlo, Y32, int(m), int(n), int(n), err);
                tlo.mark(3, st);
                if (e == cudaSuccess)
                    ns_update_kernel<kBF16><<<ug, 256, 0, st>>>(int(m), int(n), X32, Y32, nullptr, 0, 0.0, Xlo, Xt, upart);
            } else {
                tlo.mark(0, st);
                e = launch_gemm<kTF32>(st, Xt, Xt, T32, int(n), int(n), int(m), err);
                tlo.mark(1, st);
                if (e == cudaSuccess) to_lo_kernel<kTF32><<<1024, 256, 0, st>>>(nn32, T32, Tlo);
                tlo.mark(2, st);
                if (e == cudaSuccess) e = launch_gemm<kTF32>(st, Xlo, Tlo, Y32, int(m), int(n), int(n), err);
                tlo.mark(3, st);
                if (e == cudaSuccess)
                    ns_update_kernel<kTF32><<<ug, 256, 0, st>>>(int(m), int(n), X32, Y32, nullptr, 0, 0.0, Xlo, Xt, upart);
            }
            ctx->launches += 4;
            if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "polar tc iteration");
            sum_kernel<<<1, 256, 0, st>>>(nub, upart, dsum);
            sum_kernel<<<1, 256, 0, st>>>(nub, upart + nub, dsum + 1);
            double d2x2[2] = {0.0, 0.0};
            int herr = 0;
            if ((e = cudaMemcpyAsync(d2x2, dsum, 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                (e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                (e = cudaStreamSynchronize(st)) != cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "polar tc sync");
            if (herr) return lsvd_ctx_fail(ctx, LSVD_CUDA_ERROR, "tc gemm: pipeline wait timed out");
            tlo.accumulate();
            it_lo = it + 1;
            flops_lo += 4.0 * double(m) * double(n) * double(n);
            if (!std::isfinite(d2x2[0]) || !std::isfinite(d2x2[1])) break;
            if (std::sqrt(d2x2[0]) < floor_rel * std::sqrt(d2x2[1])) break;
        }
        widen_kernel<<<2048, 256, 0, st>>>(int(m), int(n), X32, X64, ld);
        if ((e = cudaMemsetAsync(Y64, 0, mn * 8, st)) != cudaSuccess)  // held the partials
            return lsvd_ctx_cuda(ctx, e, "polar clear Y");
    } else {
        scale64_kernel<<<2048, 256, 0, st>>>(int(m), int(n), A64, ld, inv, X64, ld);
    }
    // FP64 iterations (refinement, or the whole FP64 iteration) on the FP64
    // tensor path: T = X^T X (K = m), Y = X T (K = n), row-major throughout.
    bool conv = false;
    const int cap = std::min(fp64_cap, lowp ? 120 - it_lo : 120);
    for (int it = 0; it < cap; ++it) {
        thi.mark(0, st);
        e = lsvd::dg::dgemm(st, true, false, int(n), int(n), int(m), 1.0, X64, ld, X64, ld, 0.0, T64, ld);
        thi.mark(1, st);
        thi.mark(2, st);
        if (e == cudaSuccess)
            e = lsvd::dg::dgemm(st, false, false, int(m), int(n), int(n), 1.0, X64, ld, T64, ld, 0.0, Y64, ld);
        thi.mark(3, st);
        if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "polar fp64 gemm");
        ns_update64_kernel<<<nparts, 256, 0, st>>>(mn, X64, Y64, part);
        ctx->launches += 3;
        double d2 = 0.0;
        if ((e = read_sum(nparts, &d2)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "polar fp64 sync");
        thi.accumulate();
        it_hi = it + 1;
        flops_hi += 4.0 * double(m) * double(n) * double(n);
        const double delta = std::sqrt(d2);
        if (!std::isfinite(d2) || delta > 1e6 * refn) break;  // divergence (:169)
        if (delta < 1e-13 * refn) {                            // POLAR_TOL (:173)
            conv = true;
            break;
        }
    }
    // orthogonality of the returned factor: ||X^T X - I||_F
    if ((e = lsvd::dg::dgemm(st, true, false, int(n), int(n), int(m), 1.0, X64, ld, X64, ld, 0.0, T64, ld)) !=
        cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "polar orth gemm");
    orth2_kernel<<<nparts, 256, 0, st>>>(int(n), T64, ld, part);
    ctx->launches += 2;
    double o2 = 0.0;
    if ((e = read_sum(nparts, &o2)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "polar orth");
    if (info) {
        info->iters_lowp = it_lo;
        info->iters_fp64 = it_hi;
        info->orth = std::sqrt(o2);
        info->flops_lowp = flops_lo;
        info->flops_fp64 = flops_hi;
        info->gemm_ms_lowp = tlo.ms;
        info->gemm_ms_fp64 = thi.ms;
        info->converged = conv ? 1 : 0;
        info->pad_ = 0;
    }
    *Xout = X64;
    *ldx_out = ld;
    return conv ? LSVD_OK : LSVD_NOT_CONVERGED;
}

extern "C" lsvd_status lsvd_polar_f64(lsvd_context* ctx, int64_t m, int64_t n, const double* A,
                                      int64_t lda, double* Q, int64_t ldq, lsvd_precision precision,
                                      lsvd_polar_info* info, uint32_t flags) {
    LSVD_TRACE("lsvd_polar_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (m <= 0 || n <= 0 || m < n) return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "polar: need m >= n >= 1");
    if (!A || !Q || lda < n || ldq < n) return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "polar: bad pointer");
    if (precision != LSVD_PREC_FP64 && precision != LSVD_PREC_MIXED_TF32 && precision != LSVD_PREC_MIXED_BF16)
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "polar: unknown precision");
    (void)flags;  // host and device pointers are both handled by cudaMemcpy2DAsync's default kind
    cudaSetDevice(ctx->device);
    double* X = nullptr;
    int64_t ldx = 0;
    const lsvd_status st = lsvd_polar_run(ctx, m, n, A, lda, precision, 120, &X, &ldx, info);
    if (st != LSVD_OK && st != LSVD_NOT_CONVERGED) return st;
    cudaError_t e;
    if ((e = cudaMemcpy2DAsync(Q, size_t(ldq) * 8, X, size_t(ldx) * 8, size_t(n) * 8, size_t(m),
                               cudaMemcpyDefault, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "polar copy out");
    return st;
}
