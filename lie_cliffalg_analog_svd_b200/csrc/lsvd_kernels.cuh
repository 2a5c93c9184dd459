// lsvd_kernels.cuh -- kernel entry points of the small/micro/batched SVD path.
#pragma once

#include "lsvd_device.cuh"
#include "lsvd_internal.h"
#include "lsvd_mixed.cuh"

namespace lsvd {


struct BatchArgs {
    const int32_t* n;
    const int64_t* aoff;  // element offset of matrix t in A/U/Vt
    const int64_t* soff;  // element offset of matrix t in S
    const int32_t* perm;  // matrices sorted by n descending
    const double* A;
    double* U;
    double* S;
    double* Vt;
    lsvd_diag* diag;  // may be null
    const Item* items;
    int n_items;
    int want_diag;
    int* head;      // work-queue head (zeroed before launch)
    int* fb_count;  // micro -> small escalations (zeroed before launch)
    int32_t* fb_list;
    int* agg_flags;  // OR of all per-matrix flags (zeroed before launch)
    ClassCfg cls[kMaxClasses];
};

template <int TS, int G>
__device__ __forceinline__ void run_variant(const Team& t, const SmallJob& job, double* sm) {
    small_solve_team<TS, G>(t, job, sm);
}

__device__ __forceinline__ void dispatch_small(int variant, const Team& t, const SmallJob& job,
                                               double* sm) {
    switch (variant) {
        case 0: run_variant<2, 8>(t, job, sm); break;
        case 1: run_variant<2, 16>(t, job, sm); break;
        case 2: run_variant<2, 32>(t, job, sm); break;
        case 3: run_variant<4, 8>(t, job, sm); break;
        case 4: run_variant<4, 16>(t, job, sm); break;
        default: run_variant<4, 32>(t, job, sm); break;
    }
}

__device__ __forceinline__ SmallJob make_job(const BatchArgs& a, int mi) {
    SmallJob j;
    j.n = a.n[mi];
    const int64_t ao = a.aoff[mi], so = a.soff[mi];
    j.A = a.A + ao;
    j.lda = j.n;
    j.U = a.U + ao;
    j.ldu = j.n;
    j.S = a.S + so;
    j.Vt = a.Vt + ao;
    j.ldvt = j.n;
    j.diag = a.diag ? a.diag + mi : nullptr;
    j.rotors = nullptr;
    j.rotor_cap = 0;
    j.rotor_count = nullptr;
    j.perm_out = nullptr;
    j.want_diag = a.want_diag != 0;
    j.extra_flags = 0;
    j.agg = a.agg_flags;
    return j;
}

// metrics::compute (src/lib.rs:149-194) for an n <= 4 result, one thread.
__device__ __forceinline__ void micro_metrics(int n, const double* A, const double* U,
                                              const double* S, const double* Vt, double& rel,
                                              double& ou, double& ov) {
    double r2 = 0.0, a2 = 0.0, u2 = 0.0, v2 = 0.0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double rec = 0.0, gu = 0.0, gv = 0.0;
            for (int k = 0; k < n; ++k) {
                rec += U[i * n + k] * S[k] * Vt[k * n + j];
                gu += U[k * n + i] * U[k * n + j];
                gv += Vt[i * n + k] * Vt[j * n + k];
            }
            const double d = rec - A[i * n + j];
            r2 += d * d;
            a2 += A[i * n + j] * A[i * n + j];
            const double e = (i == j) ? 1.0 : 0.0;
            u2 += (gu - e) * (gu - e);
            v2 += (gv - e) * (gv - e);
        }
    rel = sqrt(r2) / fmax(sqrt(a2), 1e-300);
    ou = sqrt(u2);
    ov = sqrt(v2);
}

// One matrix with n <= 4 on the calling thread.  Returns false if it must be
// escalated to LieSvdSmall (src/lie_svd_micro.rs:90-92).
__device__ __forceinline__ bool micro_one(int n, const double* A, double* U, double* S, double* Vt,
                                          lsvd_diag* diag, bool want_diag, int* agg) {
    MicroOut mo{0, 0, true, false};
    if (n == 1) {  // src/lie_svd_micro.rs:32-40
        const double d = A[0];
        U[0] = d < 0.0 ? -1.0 : 1.0;
        S[0] = fabs(d);
        Vt[0] = 1.0;
        mo.nonfinite = !isfinite(d);
    } else if (n == 2) {
        mo = micro_solve_regs<2>(A, 2, U, 2, S, Vt, 2);
    } else if (n == 3) {
        mo = micro_solve_regs<3>(A, 3, U, 3, S, Vt, 3);
    } else {
        mo = micro_solve_regs<4>(A, 4, U, 4, S, Vt, 4);
    }
    if (!mo.ok) return false;
    const int fl = mo.nonfinite ? LSVD_MAT_NONFINITE : 0;
    if (fl) atomicOr(agg, fl);
    if (diag) {
        lsvd_diag d;
        const double qnan = __longlong_as_double(0x7ff8000000000000ULL);
        d.rel_recon = d.orth_u = d.orth_v = qnan;
        if (want_diag) micro_metrics(n, A, U, S, Vt, d.rel_recon, d.orth_u, d.orth_v);
        d.ns_iters = 0;
        d.jacobi_sweeps = mo.sweeps;
        d.rotations = mo.rotations;
        d.flags = fl;
        d.route = LSVD_ROUTE_MICRO;
        *diag = d;
    }
    return true;
}

#ifndef LSVD_KERNELS_DEVICE_ONLY
// Persistent batched kernel: CTAs pull work items (largest n first) from an
// atomic queue until it drains.  Micro items: one matrix per thread.  Small
// items: teams of W warps, one matrix per team at a time.
__global__ void __launch_bounds__(kCtaThreads, 2) batched_kernel(const BatchArgs args) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(args.head, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= args.n_items) break;
        const Item item = args.items[it];
        const ClassCfg cfg = args.cls[item.cls];
        if (cfg.nwarps == 0) {
            const int t = threadIdx.x;
            if (t < item.count) {
                const int mi = args.perm[item.first + t];
                const int n = args.n[mi];
                const int64_t ao = args.aoff[mi], so = args.soff[mi];
                const bool ok = micro_one(n, args.A + ao, args.U + ao, args.S + so, args.Vt + ao,
                                          args.diag ? args.diag + mi : nullptr,
                                          args.want_diag != 0, args.agg_flags);
                if (!ok) {
                    const int slot = atomicAdd(args.fb_count, 1);
                    args.fb_list[slot] = mi;
                }
            }
        } else {
            const int tsize = 32 * cfg.nwarps;
            const int teams = kCtaThreads / tsize;
            const int team = threadIdx.x / tsize;
            Team tm;
            tm.tid = threadIdx.x % tsize;
            tm.nthreads = tsize;
            tm.warp = tm.tid / 32;
            tm.lane = threadIdx.x % 32;
            tm.nwarps = cfg.nwarps;
            tm.bar = 1 + team;
            double* sm = smem + size_t(team) * cfg.slice;
            for (int k = team; k < item.count; k += teams) {
                const int mi = args.perm[item.first + k];
                SmallJob job = make_job(args, mi);
                dispatch_small(cfg.variant, tm, job, sm);
            }
        }
        __syncthreads();
    }
}

template <int PREC>
__device__ __forceinline__ void dispatch_mixed(int variant, const Team& t, const SmallJob& job,
                                               double* sm) {
    switch (variant) {
        case 1: mixed_solve_team<2, 16, PREC>(t, job, sm); break;
        case 3: case 4: case 5: mixed_solve_team<4, 8, PREC>(t, job, sm); break;
        default: mixed_solve_team<2, 8, PREC>(t, job, sm); break;
    }
}

// Persistent batched kernel of the mixed-precision path (same work queue and
// size classes as batched_kernel; n <= 4 keeps the FP64 micro kernel).
template <int PREC>
__global__ void __launch_bounds__(kCtaThreads, 2) batched_mixed_kernel(const BatchArgs args) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(args.head, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= args.n_items) break;
        const Item item = args.items[it];
        const ClassCfg cfg = args.cls[item.cls];
        if (cfg.nwarps == 0) {
            const int t = threadIdx.x;
            if (t < item.count) {
                const int mi = args.perm[item.first + t];
                const int n = args.n[mi];
                const int64_t ao = args.aoff[mi], so = args.soff[mi];
                const bool ok = micro_one(n, args.A + ao, args.U + ao, args.S + so, args.Vt + ao,
                                          args.diag ? args.diag + mi : nullptr,
                                          args.want_diag != 0, args.agg_flags);
                if (!ok) {
                    const int slot = atomicAdd(args.fb_count, 1);
                    args.fb_list[slot] = mi;
                }
            }
        } else {
            const int tsize = 32 * cfg.nwarps;
            const int teams = kCtaThreads / tsize;
            const int team = threadIdx.x / tsize;
            Team tm;
            tm.tid = threadIdx.x % tsize;
            tm.nthreads = tsize;
            tm.warp = tm.tid / 32;
            tm.lane = threadIdx.x % 32;
            tm.nwarps = cfg.nwarps;
            tm.bar = 1 + team;
            double* sm = smem + size_t(team) * cfg.slice;
            for (int k = team; k < item.count; k += teams) {
                const int mi = args.perm[item.first + k];
                SmallJob job = make_job(args, mi);
                dispatch_mixed<PREC>(cfg.variant, tm, job, sm);
            }
        }
        __syncthreads();
    }
}

// Escalations from the micro kernel (rare): LieSvdSmall on a whole CTA.
__global__ void __launch_bounds__(kCtaThreads, 1) fallback_kernel(const BatchArgs args) {
    extern __shared__ __align__(16) double smem[];
    const int cnt = *args.fb_count;
    Team tm;
    tm.tid = threadIdx.x;
    tm.nthreads = kCtaThreads;
    tm.warp = threadIdx.x / 32;
    tm.lane = threadIdx.x % 32;
    tm.nwarps = kCtaThreads / 32;
    tm.bar = 1;
    for (int idx = blockIdx.x; idx < cnt; idx += gridDim.x) {
        const int mi = args.fb_list[idx];
        SmallJob job = make_job(args, mi);
        job.extra_flags = LSVD_MAT_MICRO_FALLBACK;
        small_solve_team<2, 8>(tm, job, smem);
        __syncthreads();
    }
}

// Single-matrix LieSvdSmall::solve on one CTA (all eight warps, one team),
// with the rotor stream and sort permutation outputs.
template <int TS, int G>
__global__ void __launch_bounds__(kCtaThreads, 1) single_kernel(SmallJob job) {
    extern __shared__ __align__(16) double smem[];
    Team tm;
    tm.tid = threadIdx.x;
    tm.nthreads = kCtaThreads;
    tm.warp = threadIdx.x / 32;
    tm.lane = threadIdx.x % 32;
    tm.nwarps = kCtaThreads / 32;
    tm.bar = 1;
    small_solve_team<TS, G>(tm, job, smem);
}

// LieSvdMicro::solve for one matrix (thread 0), with escalation flag.
__global__ void micro_single_kernel(int n, const double* A, double* U, double* S, double* Vt,
                                    lsvd_diag* diag, int want_diag, int* need_fallback,
                                    int* agg) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    *need_fallback = micro_one(n, A, U, S, Vt, diag, want_diag != 0, agg) ? 0 : 1;
}

#endif  // LSVD_KERNELS_DEVICE_ONLY

}  // namespace lsvd
