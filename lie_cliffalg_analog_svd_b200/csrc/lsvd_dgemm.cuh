// lsvd_dgemm.cuh -- FP64 GEMM on the FP64 tensor path (mma.sync m8n8k4.f64)
// for the large-matrix products of the hot path: the Newton-Schulz products
// X^T X and X T (newton_schulz_polar, src/lie_svd_small.rs:172-173), P = Q^T A
// (:305), U = Q V (:313) and the preconditioning products of the large SVD.
//
//   C (M x N, row-major, ldc) = alpha op(A) op(B) + beta C
//   op(A) = A   (A row-major M x K, lda >= K)   or A^T (A row-major K x M)
//   op(B) = B   (B row-major K x N, ldb >= N)   or B^T (B row-major N x K)
//
// One CTA of 8 warps computes a 128 x 128 tile (or 128 x 64 when the product
// has too few 128 x 128 tiles to fill the GPU twice); warps are arranged 4 (M)
// x 2 (N) and own 32 x 64 (32 x 32) each (4 x 8 (4 x 4) tiles of 8 x 8).
// Operands stream through a 3-stage cp.async ring of BK = 32; each operand
// tile sits in shared memory either K-contiguous (leading dimension 36
// doubles) or M/N-contiguous (leading dimension 132 doubles), both = 4 mod 16,
// so the 8 x 4 fragment reads of a half-warp hit 16 distinct 8-byte bank
// pairs.  Edges are zero-filled by the cp.async source size; the caller keeps
// every leading dimension even and every base 16-byte aligned.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace lsvd {
namespace dg {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, THREADS = 256;
constexpr int LDK = BK + 4;   // K-contiguous tiles: [128][36]
constexpr int LDMN = BM + 4;  // M/N-contiguous tiles: [32][132]
constexpr int TILE_DOUBLES = (BM * LDK > BK * LDMN) ? BM * LDK : BK * LDMN;  // 4608
constexpr int SMEM_BYTES = STAGES * 2 * TILE_DOUBLES * 8;                       // 221184

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Loads the BK-slice starting at k0 of an R-wide operand tile (rows/cols
// [r0, r0 + R) of op(X), R = 128 or 64) into shared memory.  KCONT: the
// operand's K index is contiguous in global memory (A not transposed, or B
// transposed).
template <bool KCONT, int R = 128>
__device__ __forceinline__ void load_tile(double* sm, const double* X, int64_t ldx, int r0, int rdim,
                                          int k0, int kdim, int tid) {
    constexpr int KCH = BK / 2;  // two-double chunks per row of a slice
    if (KCONT) {
        // R rows x BK k = KCH R chunks of two doubles
#pragma unroll
        for (int it = 0; it < R * KCH / THREADS; ++it) {
            const int c = tid + it * THREADS;
            const int row = c / KCH, kc = (c % KCH) * 2;
            const int gr = r0 + row, gk = k0 + kc;
            int valid = kdim - gk;
            valid = valid > 2 ? 2 : (valid < 0 ? 0 : valid);
            if (gr >= rdim) valid = 0;
            const double* src = valid ? X + int64_t(gr) * ldx + gk : X;
            cp_async16(sm + row * LDK + kc, src, valid * 8);
        }
    } else {
        // BK k-rows x R = KCH R chunks
#pragma unroll
        for (int it = 0; it < R * KCH / THREADS; ++it) {
            const int c = tid + it * THREADS;
            const int kr = c / (R / 2), mc = (c % (R / 2)) * 2;
            const int gk = k0 + kr, gm = r0 + mc;
            int valid = rdim - gm;
            valid = valid > 2 ? 2 : (valid < 0 ? 0 : valid);
            if (gk >= kdim) valid = 0;
            const double* src = valid ? X + int64_t(gk) * ldx + gm : X;
            cp_async16(sm + kr * LDMN + mc, src, valid * 8);
        }
    }
}

// Fragment element (row r of the 128-wide tile, k index kk of the slice).
template <bool KCONT>
__device__ __forceinline__ double frag(const double* sm, int r, int kk) {
    return KCONT ? sm[r * LDK + kk] : sm[kk * LDMN + r];
}

struct GemmArgs {
    int M, N, K;
    const double* A;
    int64_t lda, strideA;
    const double* B;
    int64_t ldb, strideB;
    double* C;
    int64_t ldc, strideC;
    double alpha, beta;
};

template <bool TA, bool TB, int TBN = BN>
__global__ void __launch_bounds__(THREADS, 1) dgemm_kernel(const GemmArgs g) {
    constexpr int WJ = TBN / 16;  // 8 x 8 tiles per warp along N
    extern __shared__ __align__(16) double dsm[];
    // A's K is contiguous when A is not transposed; B's when B is transposed
    constexpr bool AK = !TA, BKC = TB;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const int gq = lane >> 2, q = lane & 3;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * TBN;
    const double* A = g.A + int64_t(blockIdx.z) * g.strideA;
    const double* B = g.B + int64_t(blockIdx.z) * g.strideB;
    double* Cz = g.C + int64_t(blockIdx.z) * g.strideC;
    const int KT = (g.K + BK - 1) / BK;

    double acc[4][WJ][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < WJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    auto sa = [&](int s) { return dsm + s * 2 * TILE_DOUBLES; };
    auto sb = [&](int s) { return dsm + s * 2 * TILE_DOUBLES + TILE_DOUBLES; };
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < KT) {
            load_tile<AK>(sa(s), A, g.lda, m0, g.M, s * BK, g.K, tid);
            load_tile<BKC, TBN>(sb(s), B, g.ldb, n0, g.N, s * BK, g.K, tid);
        }
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        {
            const int nk = kt + STAGES - 1;
            if (nk < KT) {
                const int s = nk % STAGES;
                load_tile<AK>(sa(s), A, g.lda, m0, g.M, nk * BK, g.K, tid);
                load_tile<BKC, TBN>(sb(s), B, g.ldb, n0, g.N, nk * BK, g.K, tid);
            }
            cp_async_commit();
        }
        const double* As = sa(kt % STAGES);
        const double* Bs = sb(kt % STAGES);
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double a[4], b[WJ];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = frag<AK>(As, wm * 32 + i * 8 + gq, kk + q);
#pragma unroll
            for (int j = 0; j < WJ; ++j) b[j] = frag<BKC>(Bs, wn * (TBN / 2) + j * 8 + gq, kk + q);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < WJ; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }
    cp_async_wait<0>();
    // epilogue: lane holds C[row gq][cols 2q, 2q + 1] of every 8 x 8 tile
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = m0 + wm * 32 + i * 8 + gq;
        if (r >= g.M) continue;
        double* crow = Cz + int64_t(r) * g.ldc;
#pragma unroll
        for (int j = 0; j < WJ; ++j) {
            const int c = n0 + wn * (TBN / 2) + j * 8 + 2 * q;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                if (c + e < g.N) {
                    const double v = g.alpha * acc[i][j][e];
                    crow[c + e] = g.beta == 0.0 ? v : v + g.beta * crow[c + e];
                }
            }
        }
    }
}

// Launches C = alpha op(A) op(B) + beta C on `st` (batch = gridDim.z).
// Leading dimensions must be even and the bases 16-byte aligned.
inline cudaError_t dgemm(cudaStream_t st, bool ta, bool tb, int M, int N, int K, double alpha,
                         const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
                         double* C, int64_t ldc, int batch = 1, int64_t sA = 0, int64_t sB = 0,
                         int64_t sC = 0) {
    if (M <= 0 || N <= 0) return cudaSuccess;
    if ((lda | ldb) & 1 || (reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15 ||
        (sA | sB) & 1)
        return cudaErrorInvalidValue;
    GemmArgs g{M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, alpha, beta};
    // 128 x 64 tiles when 128 x 128 tiles would not fill the GPU twice over
    static int sms = [] {
        int d = 0, v = 148;
        if (cudaGetDevice(&d) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d) != cudaSuccess)
            v = 148;
        return v;
    }();
    const int64_t tiles = int64_t((N + BN - 1) / BN) * ((M + BM - 1) / BM) * batch;
    const bool narrow = tiles < 2 * sms;
    const int bn = narrow ? 64 : BN;
    const dim3 grid(unsigned((N + bn - 1) / bn), unsigned((M + BM - 1) / BM), unsigned(batch));
    cudaError_t e;
#define LSVD_DGEMM_LAUNCH(TA_, TB_)                                                                          \
    if (narrow) {                                                                                             \
        e = cudaFuncSetAttribute(dgemm_kernel<TA_, TB_, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                 SMEM_BYTES);                                                                 \
        if (e == cudaSuccess) dgemm_kernel<TA_, TB_, 64><<<grid, THREADS, SMEM_BYTES, st>>>(g);              \
    } else {                                                                                                  \
        e = cudaFuncSetAttribute(dgemm_kernel<TA_, TB_, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                 SMEM_BYTES);                                                                 \
        if (e == cudaSuccess) dgemm_kernel<TA_, TB_, BN><<<grid, THREADS, SMEM_BYTES, st>>>(g);              \
    }
    if (!ta && !tb) {
        LSVD_DGEMM_LAUNCH(false, false)
    } else if (ta && !tb) {
        LSVD_DGEMM_LAUNCH(true, false)
    } else if (!ta && tb) {
        LSVD_DGEMM_LAUNCH(false, true)
    } else {
        LSVD_DGEMM_LAUNCH(true, true)
    }
#undef LSVD_DGEMM_LAUNCH
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace dg
}  // namespace lsvd
