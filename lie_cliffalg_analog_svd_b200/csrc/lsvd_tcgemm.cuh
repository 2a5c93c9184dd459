// lsvd_tcgemm.cuh -- tcgen05 GEMM for the large Newton-Schulz polar iteration.
//
//   C[M x N] (FP32, row-major) = A[M x K] * B[N x K]^T
//
// A and B are K-major (row-major, K contiguous), BF16 or FP32-stored TF32.
// One CTA computes a 128 x TN tile (TN = 256 where N allows it, else 128):
// TMA (cp.async.bulk.tensor.2d, 128-byte swizzle, no multicast) brings
// 128-byte K-slices of 128 rows of A and TN rows of B into a 4-stage
// shared-memory ring guarded by mbarriers; one elected thread issues
// tcgen05.mma (cta_group::1, M = 128, N = TN, FP32 accumulator in TN TMEM
// columns) and releases each stage with tcgen05.commit; after the last
// K-slice the four warps read their 32 TMEM lanes with tcgen05.ld and store
// FP32 rows.  Every mbarrier wait is bounded: on timeout the kernel records
// an error code, drains the copies it issued (bounded), frees its TMEM and
// returns.  M, N must be multiples of 128 and K a multiple of the K-slice
// (64 BF16 or 32 TF32 elements).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace lsvd {
namespace tc {

constexpr int kTile = 128;                             // M of a tile (and the smallest N)
constexpr int kStages = 4;
constexpr int kSliceBytes = 128;                       // K bytes per stage row
// Stage: an A slice of 128 rows and a B slice of TN rows (TN = 128 or 256).
__host__ __device__ constexpr int stage_bytes(int tn) { return (kTile + tn) * kSliceBytes; }
__host__ __device__ constexpr int smem_bytes(int tn) { return kStages * stage_bytes(tn) + 1024 + 256; }
constexpr unsigned kSpinLimit = 1u << 26;              // bounded mbarrier waits: polls
constexpr uint64_t kWaitNs = 2000000000ull;           // ... and wall time (2 s)

enum Prec { kBF16 = 1, kTF32 = 2 };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the phase with the given parity; false once kWaitNs of
// wall time (or kSpinLimit polls) passed without the phase completing.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    for (unsigned it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255u) == 255u && global_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1)
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (LBO unused for swizzled K-major, = 1), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= uint64_t((addr & 0x3FFFF) >> 4);   // start address, bits [0,14)
    d |= uint64_t(1) << 16;                  // leading byte offset (unused), bits [16,30)
    d |= uint64_t(1024 >> 4) << 32;          // stride byte offset, bits [32,46)
    d |= uint64_t(1) << 46;                  // descriptor version
    d |= uint64_t(2) << 61;                  // SWIZZLE_128B
    return d;
}

// Instruction descriptor: FP32 accumulator, A/B format (1 = BF16 under
// kind::f16, 2 = TF32 under kind::tf32), K-major A and B, N = TN, M = 128.
template <int PREC, int TN>
__host__ __device__ constexpr uint32_t instr_desc() {
    return (1u << 4) | ((PREC == kBF16 ? 1u : 2u) << 7) | ((PREC == kBF16 ? 1u : 2u) << 10) |
           (uint32_t(TN >> 3) << 17) | (uint32_t(kTile >> 4) << 24);
}

template <int PREC, int TN>
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc) {
    constexpr uint32_t idesc = instr_desc<PREC, TN>();
    if (PREC == kBF16) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
    }
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// grid (N/TN, M/128), 128 threads.  err: set to a nonzero code on timeout.
// mapB's box is TN rows high.
template <int PREC, int TN>
__global__ void __launch_bounds__(128, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                   float* __restrict__ C, int ldc, int K, int* err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte alignment of the swizzled stages
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* bufs = smem_raw + (base - raw);
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
    __shared__ uint32_t tmem_base;
    __shared__ int s_err;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    constexpr int kStageBytes = stage_bytes(TN);
    const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * TN;
    constexpr int elem = (PREC == kBF16) ? 2 : 4;
    constexpr int kslice = kSliceBytes / elem;       // K elements per stage
    constexpr int kmma = (PREC == kBF16) ? 16 : 8;   // K per tcgen05.mma
    const int nk = K / kslice;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(&done), 1);
        s_err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(TN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    if (warp == 0 && lane == 0) {
        // producer: K-slices of A (rows m0..) and B (rows n0..)
        int issued = 0;
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kStages;
            if (kb >= kStages && !mbar_wait(smem_u32(&empty[s]), ((kb / kStages) - 1) & 1)) {
                s_err = 1;
                break;
            }
            const uint32_t a_dst = base + s * kStageBytes;
            const uint32_t b_dst = a_dst + kTile * kSliceBytes;
            mbar_expect_tx(smem_u32(&full[s]), kStageBytes);
            tma_load_2d(a_dst, &mapA, smem_u32(&full[s]), kb * kslice, m0);
            tma_load_2d(b_dst, &mapB, smem_u32(&full[s]), kb * kslice, n0);
            issued = kb + 1;
        }
        // drain: wait (bounded) until every issued copy has landed before leaving
        if (s_err)
            for (int kb = (issued > kStages ? issued - kStages : 0); kb < issued; ++kb)
                mbar_wait(smem_u32(&full[kb % kStages]), (kb / kStages) & 1);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kStages;
            if (!mbar_wait(smem_u32(&full[s]), (kb / kStages) & 1)) {
                s_err = 2;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a_src = base + s * kStageBytes;
            const uint32_t b_src = a_src + kTile * kSliceBytes;
            const uint64_t da = smem_desc(a_src), db = smem_desc(b_src);
#pragma unroll
            for (int k = 0; k < kslice / kmma; ++k) {
                // advance 32 bytes along K inside the swizzle atom (16-byte units)
                const uint64_t off = uint64_t((k * kmma * elem) >> 4);
                mma<PREC, TN>(tmem, da + off, db + off, (kb > 0 || k > 0) ? 1u : 0u);
            }
            mma_commit(smem_u32(&empty[s]));
        }
        mma_commit(smem_u32(&done));
    }
    __syncwarp();
    // epilogue: warp w owns TMEM lanes (rows) 32w .. 32w+31; the warp-wide
    // vote keeps the .sync.aligned TMEM loads converged and uniform
    const bool ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(&done), 0));
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (__all_sync(0xffffffffu, ok && *reinterpret_cast<volatile int*>(&s_err) == 0)) {
        const int row = m0 + warp * 32 + lane;
        float* crow = C + size_t(row) * ldc + n0;
#pragma unroll 1
        for (int c0 = 0; c0 < TN; c0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                  "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                  "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                  "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                  "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                  "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 32; j += 4) {
                float4 f;
                f.x = __uint_as_float(v[j]);
                f.y = __uint_as_float(v[j + 1]);
                f.z = __uint_as_float(v[j + 2]);
                f.w = __uint_as_float(v[j + 3]);
                *reinterpret_cast<float4*>(crow + c0 + j) = f;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (threadIdx.x == 0 && (s_err || !ok)) atomicExch(err, s_err ? s_err : 3);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
}


__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Persistent variant, grid = min(tiles, SMs), 192 threads (6 warps), one CTA
// per SM, tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... (row of tiles
// major: consecutive CTAs share the A row panel in L2):
//   warp 0 (one lane)  TMA producer over every (tile, K-slice) of the CTA;
//   warp 1 (one lane)  MMA issuer; the accumulator of the CTA's i-th tile lives
//                      in TMEM columns (i & 1) * TN .. + TN (2 TN allocated);
//   warps 2..5         epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its
//                      lane quadrant), stores FP32 rows, releases the accumulator.
// So tile i's epilogue overlaps tile i + 1's main loop.  Barriers: full/empty
// per stage, tfull[2] (MMA -> epilogue, tcgen05.commit), tempty[2] (epilogue ->
// MMA, one arrival per epilogue warp).  Every wait is bounded; a timeout sets
// an error code, the roles stop issuing, the producer drains its copies, the
// MMA issuer waits (bounded) for its MMAs, and the CTA frees its TMEM.
template <int PREC, int TN>
__global__ void __launch_bounds__(192, 1)
    tc_gemm_persistent_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                              float* __restrict__ C, int ldc, int M, int N, int K, int* err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], tfull[2], tempty[2], mdone;
    __shared__ uint32_t tmem_base;
    __shared__ int s_err;
    volatile int* verr = &s_err;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    constexpr int kStageBytes = stage_bytes(TN);
    constexpr int elem = (PREC == kBF16) ? 2 : 4;
    constexpr int kslice = kSliceBytes / elem;
    constexpr int kmma = (PREC == kBF16) ? 16 : 8;
    const int nk = K / kslice;
    const int ntn = N / TN, tiles = (M / kTile) * ntn;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(smem_u32(&tfull[a]), 1);
            mbar_init(smem_u32(&tempty[a]), 4);
        }
        mbar_init(smem_u32(&mdone), 1);
        s_err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(2 * TN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    if (warp == 0 && lane == 0) {
        int it = 0;  // K-slices issued (ring position)
        bool stop = false;
        for (int t = blockIdx.x; t < tiles && !stop; t += gridDim.x) {
            const int m0 = (t / ntn) * kTile, n0 = (t % ntn) * TN;
            for (int kb = 0; kb < nk; ++kb) {
                const int s = it % kStages;
                if (*verr || (it >= kStages && !mbar_wait(smem_u32(&empty[s]), ((it / kStages) - 1) & 1))) {
                    if (!*verr) *verr = 1;
                    stop = true;
                    break;
                }
                const uint32_t a_dst = base + s * kStageBytes;
                const uint32_t b_dst = a_dst + kTile * kSliceBytes;
                mbar_expect_tx(smem_u32(&full[s]), kStageBytes);
                tma_load_2d(a_dst, &mapA, smem_u32(&full[s]), kb * kslice, m0);
                tma_load_2d(b_dst, &mapB, smem_u32(&full[s]), kb * kslice, n0);
                ++it;
            }
        }
        // drain: every copy issued lands before the CTA leaves
        if (stop)
            for (int j = (it > kStages ? it - kStages : 0); j < it; ++j)
                mbar_wait(smem_u32(&full[j % kStages]), (j / kStages) & 1);
    } else if (warp == 1 && lane == 0) {
        int it = 0, lt = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++lt) {
            const int acc = lt & 1;
            if (*verr || (lt >= 2 && !mbar_wait(smem_u32(&tempty[acc]), ((lt >> 1) - 1) & 1))) {
                if (!*verr) *verr = 2;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t d = tmem + uint32_t(acc * TN);
            bool stop = false;
            for (int kb = 0; kb < nk; ++kb, ++it) {
                const int s = it % kStages;
                if (!mbar_wait(smem_u32(&full[s]), (it / kStages) & 1)) {
                    *verr = 3;
                    stop = true;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t a_src = base + s * kStageBytes;
                const uint32_t b_src = a_src + kTile * kSliceBytes;
                const uint64_t da = smem_desc(a_src), db = smem_desc(b_src);
#pragma unroll
                for (int k = 0; k < kslice / kmma; ++k) {
                    const uint64_t off = uint64_t((k * kmma * elem) >> 4);
                    mma<PREC, TN>(d, da + off, db + off, (kb > 0 || k > 0) ? 1u : 0u);
                }
                mma_commit(smem_u32(&empty[s]));
            }
            if (stop) break;
            mma_commit(smem_u32(&tfull[acc]));
        }
        // every MMA this thread issued is complete before TMEM can be freed
        mma_commit(smem_u32(&mdone));
        if (!mbar_wait(smem_u32(&mdone), 0) && !*verr) *verr = 5;
    } else if (warp >= 2) {
        const int q = warp & 3;  // the TMEM lane quadrant this warp may read
        int lt = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++lt) {
            const int acc = lt & 1;
            const bool ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(&tfull[acc]), (lt >> 1) & 1));
            if (!ok || *verr) {
                if (!ok && lane == 0) *verr = 4;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int m0 = (t / ntn) * kTile, n0 = (t % ntn) * TN;
            float* crow = C + size_t(m0 + q * 32 + lane) * ldc + n0;
#pragma unroll 1
            for (int c0 = 0; c0 < TN; c0 += 32) {
                uint32_t v[32];
                const uint32_t taddr = tmem + (uint32_t(q * 32) << 16) + uint32_t(acc * TN + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                    "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                      "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                      "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                      "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                      "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                      "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 32; j += 4) {
                    float4 f;
                    f.x = __uint_as_float(v[j]);
                    f.y = __uint_as_float(v[j + 1]);
                    f.z = __uint_as_float(v[j + 2]);
                    f.w = __uint_as_float(v[j + 3]);
                    *reinterpret_cast<float4*>(crow + c0 + j) = f;
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&tempty[acc]));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (threadIdx.x == 0 && *verr) atomicExch(err, *verr);
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TN));
}

}  // namespace tc
}  // namespace lsvd
