// lsvd_api.cu -- host side of liblsvd_b200.so: contexts, workspaces, the
// batched planner (size classes, LPT work items, CUDA-graph capture) and the
// C ABI declared in include/lsvd.h.
#include <cuda_runtime.h>

#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <unordered_map>
#include <vector>

#include "lsvd.h"
#include "lsvd_internal.h"
#include "lsvd_kernels.cuh"

using namespace lsvd;

// ------------------------------------------------------------ context ----

lsvd_status lsvd_ctx_fail(lsvd_context* ctx, lsvd_status st, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return st;
}

void* lsvd_ctx_pinned(lsvd_context* ctx, size_t bytes) {
    if (ctx->pinned && ctx->pinned_bytes >= bytes) return ctx->pinned;
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    const size_t sz = std::max(bytes, size_t(4096));
    if (cudaHostAlloc(&ctx->pinned, sz, cudaHostAllocDefault) != cudaSuccess) {
        ctx->pinned = nullptr;
        return nullptr;
    }
    ctx->pinned_bytes = sz;
    return ctx->pinned;
}

lsvd_status lsvd_ctx_cuda(lsvd_context* ctx, cudaError_t e, const char* where) {
    if (e == cudaSuccess) return LSVD_OK;
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return lsvd_ctx_fail(ctx, LSVD_OUT_OF_MEMORY, m);
    return lsvd_ctx_fail(ctx, LSVD_CUDA_ERROR, m);
}

void* DeviceBuffer::get(size_t want, cudaError_t* err) {
    *err = cudaSuccess;
    if (want <= bytes) return ptr;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t sz = std::max(want, size_t(256));
    *err = cudaMalloc(&ptr, sz);
    if (*err != cudaSuccess) {
        ptr = nullptr;
        return nullptr;
    }
    bytes = sz;
    return ptr;
}
void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

extern "C" const char* lsvd_version(void) { return "lsvd_b200 0.1.0 (sm_100a)"; }

extern "C" const char* lsvd_status_string(lsvd_status s) {
    switch (s) {
        case LSVD_OK: return "ok";
        case LSVD_NOT_CONVERGED: return "iteration cap reached";
        case LSVD_NONFINITE_INPUT: return "non-finite input";
        case LSVD_BAD_SHAPE: return "bad shape";
        case LSVD_BAD_ARGUMENT: return "bad argument";
        case LSVD_CUDA_ERROR: return "CUDA error";
        case LSVD_OUT_OF_MEMORY: return "out of device memory";
        case LSVD_ROTOR_OVERFLOW: return "rotor buffer too small";
        case LSVD_NO_DEVICE: return "no CUDA device";
        case LSVD_UNSUPPORTED: return "unsupported size or option";
    }
    return "unknown status";
}

extern "C" lsvd_status lsvd_context_create(int device, lsvd_context** out) {
    if (!out) return LSVD_BAD_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return LSVD_NO_DEVICE;
    }
    if (device < 0 || device >= count) return LSVD_BAD_ARGUMENT;
    auto* ctx = new lsvd_context();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        delete ctx;
        return LSVD_CUDA_ERROR;
    }
    ctx->own_stream = true;
    *out = ctx;
    return LSVD_OK;
}

lsvd_context::~lsvd_context() {
    cudaSetDevice(device);
    for (auto& kv : plans) kv.second.reset();
    for (auto& pp : pipe_plans) pp.reset();
    for (auto* b : {&ws_a, &ws_u, &ws_s, &ws_vt, &ws_diag, &ws_misc, &ws_rot, &ws_polar, &ws_large, &ws_splitk})
        b->release();
    if (pinned) cudaFreeHost(pinned);
    if (h2d_stream) cudaStreamDestroy(h2d_stream);
    if (side_stream) cudaStreamDestroy(side_stream);
    if (side_stream2) cudaStreamDestroy(side_stream2);
    if (d2h_stream) cudaStreamDestroy(d2h_stream);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

extern "C" lsvd_status lsvd_context_destroy(lsvd_context* ctx) {
    if (!ctx) return LSVD_BAD_ARGUMENT;
    delete ctx;
    return LSVD_OK;
}

extern "C" lsvd_status lsvd_context_set_stream(lsvd_context* ctx, void* stream) {
    if (!ctx) return LSVD_BAD_ARGUMENT;
    cudaSetDevice(ctx->device);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = static_cast<cudaStream_t>(stream);
    ctx->own_stream = false;
    for (auto& kv : ctx->plans) kv.second->invalidate_graph();
    for (auto& pp : ctx->pipe_plans)
        if (pp) pp->invalidate_graph();
    return LSVD_OK;
}

extern "C" void* lsvd_context_get_stream(lsvd_context* ctx) { return ctx ? ctx->stream : nullptr; }

extern "C" lsvd_status lsvd_synchronize(lsvd_context* ctx) {
    if (!ctx) return LSVD_BAD_ARGUMENT;
    cudaSetDevice(ctx->device);
    return lsvd_ctx_cuda(ctx, cudaStreamSynchronize(ctx->stream), "lsvd_synchronize");
}

extern "C" const char* lsvd_context_last_error(const lsvd_context* ctx) {
    return ctx ? ctx->last_error.c_str() : "null context";
}

extern "C" int64_t lsvd_context_kernel_launches(const lsvd_context* ctx) {
    return ctx ? ctx->launches : -1;
}

// ---------------------------------------------------------- helpers ----

static bool is_dev(uint32_t flags) { return (flags & LSVD_DEVICE_POINTERS) != 0; }

// 2-D copy of a rows x cols f64 block between (possibly) strided buffers.
static cudaError_t copy2d(double* dst, int64_t ldd, const double* src, int64_t lds, int64_t rows,
                          int64_t cols, cudaStream_t s) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    return cudaMemcpy2DAsync(dst, size_t(ldd) * 8, src, size_t(lds) * 8, size_t(cols) * 8,
                             size_t(rows), cudaMemcpyDefault, s);
}

static int variant_of(int ts, int g) { return (ts == 4 ? 3 : 0) + (g == 16 ? 1 : g == 32 ? 2 : 0); }

// ------------------------------------------------------- single SVD ----

static cudaError_t launch_single(lsvd_context* ctx, const SmallJob& job) {
    const int n = job.n;
    const size_t smem = size_t(team_smem_doubles(n, kCtaThreads / 32)) * sizeof(double);
    const bool big = n > 32;
    cudaError_t e;
    if (big) {
        e = cudaFuncSetAttribute(single_kernel<4, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
        single_kernel<4, 8><<<1, kCtaThreads, smem, ctx->stream>>>(job);
    } else {
        e = cudaFuncSetAttribute(single_kernel<2, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
        single_kernel<2, 8><<<1, kCtaThreads, smem, ctx->stream>>>(job);
    }
    ctx->launches++;
    return cudaGetLastError();
}

lsvd_status lsvd_single_small(lsvd_context* ctx, int64_t n, const double* A, int64_t lda,
                              double* U, int64_t ldu, double* S, double* Vt, int64_t ldvt,
                              lsvd_diag* diag, lsvd_rotor* rotors, int64_t rotor_cap,
                              int64_t* rotor_count, int32_t* perm, uint32_t flags,
                              int extra_flags, bool host_meta) {
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (n < 1 || n > kMaxN)
        return lsvd_ctx_fail(ctx, n < 1 ? LSVD_BAD_SHAPE : LSVD_UNSUPPORTED,
                             "LieSvdSmall::solve (shared-memory kernel): n must be in 1..64");
    if (!A || !U || !S || !Vt || lda < n || ldu < n || ldvt < n || rotor_cap < 0 ||
        (rotors && rotor_cap > 0 && !rotor_count))
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_small_solve_f64: bad pointer or leading dimension");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool dev = is_dev(flags);
    cudaError_t e;
    const size_t nn = size_t(n) * size_t(n);
    double* dA = static_cast<double*>(ctx->ws_a.get(nn * 8, &e));
    double* dU = e == cudaSuccess ? static_cast<double*>(ctx->ws_u.get(nn * 8, &e)) : nullptr;
    double* dS = e == cudaSuccess ? static_cast<double*>(ctx->ws_s.get(size_t(n) * 8, &e)) : nullptr;
    double* dV = e == cudaSuccess ? static_cast<double*>(ctx->ws_vt.get(nn * 8, &e)) : nullptr;
    char* misc = e == cudaSuccess ? static_cast<char*>(ctx->ws_misc.get(4096, &e)) : nullptr;
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "workspace");
    lsvd_diag* dDiag = reinterpret_cast<lsvd_diag*>(misc);
    int64_t* dRotCount = reinterpret_cast<int64_t*>(misc + 256);
    int32_t* dPerm = reinterpret_cast<int32_t*>(misc + 512);
    lsvd_rotor* dRot = nullptr;
    if (rotors && rotor_cap > 0) {
        if (dev)
            dRot = rotors;
        else {
            dRot = static_cast<lsvd_rotor*>(ctx->ws_rot.get(size_t(rotor_cap) * sizeof(lsvd_rotor), &e));
            if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "rotor workspace");
        }
    }
    if ((e = copy2d(dA, n, A, lda, n, n, st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "copy A");
    SmallJob job;
    job.n = int(n);
    job.A = dA;
    job.lda = n;
    job.U = dU;
    job.ldu = n;
    job.S = dS;
    job.Vt = dV;
    job.ldvt = n;
    job.diag = dDiag;
    job.rotors = dRot;
    job.rotor_cap = dRot ? rotor_cap : 0;
    job.rotor_count = dRotCount;
    job.perm_out = dPerm;
    job.want_diag = (flags & LSVD_WANT_DIAG) != 0;
    job.extra_flags = extra_flags;
    job.agg = nullptr;
    if ((e = launch_single(ctx, job)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "single_kernel");
    if ((e = copy2d(U, ldu, dU, n, n, n, st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "copy U");
    if ((e = copy2d(Vt, ldvt, dV, n, n, n, st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "copy Vt");
    if ((e = cudaMemcpyAsync(S, dS, size_t(n) * 8, cudaMemcpyDefault, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "copy S");
    if (perm && (e = cudaMemcpyAsync(perm, dPerm, size_t(n) * 4, cudaMemcpyDefault, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "copy perm");
    lsvd_diag hdiag;
    int64_t hcount = 0;
    if ((e = cudaMemcpyAsync(&hdiag, dDiag, sizeof(hdiag), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&hcount, dRotCount, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "copy diag");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "sync");
    if (rotors && rotor_cap > 0 && !dev) {
        const int64_t got = std::min(hcount, rotor_cap);
        if (got > 0 &&
            (e = cudaMemcpy(rotors, dRot, size_t(got) * sizeof(lsvd_rotor), cudaMemcpyDeviceToHost)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "copy rotors");
    }
    if (rotor_count) {
        if (dev && !host_meta)
            e = cudaMemcpy(rotor_count, &hcount, 8, cudaMemcpyHostToDevice);
        else
            *rotor_count = hcount;
    }
    if (diag) {
        if (dev && !host_meta)
            e = cudaMemcpy(diag, &hdiag, sizeof(hdiag), cudaMemcpyHostToDevice);
        else
            *diag = hdiag;
    }
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "copy diag out");
    if (hdiag.flags & LSVD_MAT_NONFINITE) return LSVD_NONFINITE_INPUT;
    if (hdiag.flags & LSVD_MAT_JACOBI_CAP) return LSVD_NOT_CONVERGED;
    if (rotors && hcount > rotor_cap) return LSVD_ROTOR_OVERFLOW;
    return LSVD_OK;
}

extern "C" lsvd_status lsvd_small_solve_f64(lsvd_context* ctx, int64_t n, const double* A,
                                            int64_t lda, double* U, int64_t ldu, double* S,
                                            double* Vt, int64_t ldvt, lsvd_diag* diag,
                                            lsvd_rotor* rotors, int64_t rotor_cap,
                                            int64_t* rotor_count, int32_t* perm, uint32_t flags) {
    LSVD_TRACE("lsvd_small_solve_f64");
    if (ctx && n > kMaxN) {
        // beyond the shared-memory kernels: the blocked large solve (no plane-rotation stream)
        if (rotors || rotor_count || perm)
            return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "LieSvdSmall::solve: rotor stream and perm need n <= 64");
        if (!A || !U || !S || !Vt || lda < n || ldu < n || ldvt < n)
            return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_small_solve_f64: bad pointer or leading dimension");
        if (n > 16384) return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "LieSvdSmall::solve: n above 16384");
        cudaSetDevice(ctx->device);
        lsvd_diag hd;
        const lsvd_status st = lsvd_large_solve(ctx, n, n, A, lda, U, ldu, S, Vt, ldvt, LSVD_PREC_FP64, nullptr,
                                                &hd, (flags & LSVD_WANT_DIAG) != 0);
        if (diag && st != LSVD_CUDA_ERROR && st != LSVD_OUT_OF_MEMORY && st != LSVD_NONFINITE_INPUT) {
            if (is_dev(flags)) {
                if (cudaMemcpy(diag, &hd, sizeof(hd), cudaMemcpyHostToDevice) != cudaSuccess)
                    return lsvd_ctx_fail(ctx, LSVD_CUDA_ERROR, "copy diag out");
            } else {
                *diag = hd;
            }
        }
        return st;
    }
    return lsvd_single_small(ctx, n, A, lda, U, ldu, S, Vt, ldvt, diag, rotors, rotor_cap,
                             rotor_count, perm, flags, 0, false);
}

extern "C" lsvd_status lsvd_micro_solve_f64(lsvd_context* ctx, int64_t n, const double* A,
                                            int64_t lda, double* U, int64_t ldu, double* S,
                                            double* Vt, int64_t ldvt, lsvd_diag* diag,
                                            uint32_t flags) {
    LSVD_TRACE("lsvd_micro_solve_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (n < 0 || n > 4) return lsvd_ctx_fail(ctx, LSVD_BAD_SHAPE, "LieSvdMicro only supports N <= 4");
    if (n == 0) return LSVD_OK;  // empty result, src/lie_svd_micro.rs:27-31
    if (!A || !U || !S || !Vt || lda < n || ldu < n || ldvt < n)
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_micro_solve_f64: bad pointer or leading dimension");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    double* dA = static_cast<double*>(ctx->ws_a.get(16 * 8, &e));
    double* dU = e == cudaSuccess ? static_cast<double*>(ctx->ws_u.get(16 * 8, &e)) : nullptr;
    double* dS = e == cudaSuccess ? static_cast<double*>(ctx->ws_s.get(4 * 8, &e)) : nullptr;
    double* dV = e == cudaSuccess ? static_cast<double*>(ctx->ws_vt.get(16 * 8, &e)) : nullptr;
    char* misc = e == cudaSuccess ? static_cast<char*>(ctx->ws_misc.get(4096, &e)) : nullptr;
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "workspace");
    lsvd_diag* dDiag = reinterpret_cast<lsvd_diag*>(misc);
    int* dFlag = reinterpret_cast<int*>(misc + 1024);
    int* dAgg = dFlag + 1;
    if ((e = copy2d(dA, n, A, lda, n, n, st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "copy A");
    if ((e = cudaMemsetAsync(dFlag, 0, 8, st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "memset");
    micro_single_kernel<<<1, 32, 0, st>>>(int(n), dA, dU, dS, dV, dDiag,
                                          (flags & LSVD_WANT_DIAG) ? 1 : 0, dFlag, dAgg);
    ctx->launches++;
    if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "micro kernel");
    int hflag = 0;
    if ((e = cudaMemcpyAsync(&hflag, dFlag, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "sync");
    if (hflag) {  // LieSvdMicro -> LieSvdSmall escalation, src/lie_svd_micro.rs:90-92
        return lsvd_single_small(ctx, n, A, lda, U, ldu, S, Vt, ldvt, diag, nullptr, 0, nullptr,
                                 nullptr, flags, LSVD_MAT_MICRO_FALLBACK, false);
    }
    if ((e = copy2d(U, ldu, dU, n, n, n, st)) != cudaSuccess ||
        (e = copy2d(Vt, ldvt, dV, n, n, n, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(S, dS, size_t(n) * 8, cudaMemcpyDefault, st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "copy out");
    lsvd_diag hdiag;
    if ((e = cudaMemcpyAsync(&hdiag, dDiag, sizeof(hdiag), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "sync");
    if (diag) {
        if (is_dev(flags)) {
            if ((e = cudaMemcpy(diag, &hdiag, sizeof(hdiag), cudaMemcpyHostToDevice)) != cudaSuccess)
                return lsvd_ctx_cuda(ctx, e, "copy diag out");
        } else {
            *diag = hdiag;
        }
    }
    return (hdiag.flags & LSVD_MAT_NONFINITE) ? LSVD_NONFINITE_INPUT : LSVD_OK;
}

// ------------------------------------------------------------ batched ----

// Default size classes (n ranges, team shape, tile variant).  The autotuner
// (lsvd_autotune.cu) may override the shape per class.
static const int kClassHi[kMaxClasses] = {4, 8, 16, 24, 32, 48, 64, 64};

int lsvd_class_of(int n) {
    for (int c = 0; c < kMaxClasses; ++c)
        if (n <= kClassHi[c]) return c;
    return kMaxClasses - 1;
}

static const ClassShape kDefaultShapes[kMaxClasses] = {
    {0, 2, 8, 64},  // micro: thread per matrix, up to 256 per item
    {1, 2, 8, 2},   // 5..8
    {1, 2, 16, 1},  // 9..16
    {2, 2, 8, 1},   // 17..24
    {2, 4, 8, 1},   // 25..32
    {8, 4, 8, 1},   // 33..48
    {8, 4, 8, 1},   // 49..64
    {8, 4, 8, 1},
};

ClassShape lsvd_default_shape(int cls) { return kDefaultShapes[cls]; }

BatchPlan::~BatchPlan() {
    invalidate_graph();
    for (auto* b : {&d_meta, &d_scratch, &d_a, &d_u, &d_s, &d_vt, &d_diag}) b->release();
}

void BatchPlan::invalidate_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    bound_key.clear();
}

static uint64_t hash_ns(int64_t count, const int32_t* n) {
    uint64_t h = 1469598103934665603ull ^ uint64_t(count);
    for (int64_t i = 0; i < count; ++i) {
        h ^= uint64_t(uint32_t(n[i]));
        h *= 1099511628211ull;
    }
    return h;
}

// Builds the LPT schedule: matrices sorted by n descending, grouped into work
// items of one size class each.
static lsvd_status build_plan(lsvd_context* ctx, int64_t count, const int32_t* n,
                              const ClassShape* shapes, lsvd_precision prec, BatchPlan& P) {
    P.count = count;
    P.precision = prec;
    P.ns.assign(n, n + count);
    std::vector<int32_t> perm(static_cast<size_t>(count));
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) { return n[a] > n[b]; });
    std::vector<int64_t> aoff(static_cast<size_t>(count)), soff(static_cast<size_t>(count));
    int64_t ao = 0, so = 0;
    for (int64_t t = 0; t < count; ++t) {
        aoff[size_t(t)] = ao;
        soff[size_t(t)] = so;
        ao += int64_t(n[t]) * n[t];
        so += n[t];
    }
    P.a_elems = ao;
    P.s_elems = so;
    std::vector<Item> items;
    int max_smem = 0;
    for (int c = 0; c < kMaxClasses; ++c) {
        const ClassShape& s = shapes[c];
        ClassCfg& cfg = P.cls[c];
        cfg.nwarps = s.nwarps;
        cfg.variant = variant_of(s.ts, s.g);
        const int lo = c == 0 ? 1 : kClassHi[c - 1] + 1;
        const int hi = kClassHi[c];
        cfg.slice = !s.nwarps ? 0 : (prec == LSVD_PREC_FP64 ? team_smem_doubles(hi, s.nwarps)
                                                             : mixed_smem_doubles(hi));
        if (lo > hi) continue;
    }
    size_t i = 0;
    while (i < perm.size()) {
        const int c = lsvd_class_of(n[perm[i]]);
        size_t j = i;
        while (j < perm.size() && lsvd_class_of(n[perm[j]]) == c) ++j;
        const ClassShape& s = shapes[c];
        int per_item;
        if (s.nwarps == 0) {
            per_item = kCtaThreads;
        } else {
            const int teams = kCtaThreads / (32 * s.nwarps);
            per_item = teams * std::max(1, s.per_team);
            max_smem = std::max(max_smem, teams * P.cls[c].slice * 8);
        }
        for (size_t k = i; k < j; k += size_t(per_item)) {
            Item it;
            it.cls = c;
            it.first = int(k);
            it.count = int(std::min(j - k, size_t(per_item)));
            it.pad_ = 0;
            items.push_back(it);
        }
        i = j;
    }
    P.n_items = int(items.size());
    P.smem_bytes = max_smem;
    // metadata in one device allocation: n | aoff | soff | perm | items
    const size_t b_n = size_t(count) * 4, b_off = size_t(count) * 8;
    const size_t b_items = items.size() * sizeof(Item);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t total = al(b_n) + 2 * al(b_off) + al(b_n) + al(b_items);
    cudaError_t e;
    char* base = static_cast<char*>(P.d_meta.get(total, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "plan metadata");
    size_t off = 0;
    P.m_n = reinterpret_cast<int32_t*>(base + off); off += al(b_n);
    P.m_aoff = reinterpret_cast<int64_t*>(base + off); off += al(b_off);
    P.m_soff = reinterpret_cast<int64_t*>(base + off); off += al(b_off);
    P.m_perm = reinterpret_cast<int32_t*>(base + off); off += al(b_n);
    P.m_items = reinterpret_cast<Item*>(base + off);
    cudaStream_t st = ctx->stream;
    if ((e = cudaMemcpyAsync(P.m_n, n, b_n, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(P.m_aoff, aoff.data(), b_off, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(P.m_soff, soff.data(), b_off, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(P.m_perm, perm.data(), b_n, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (b_items && (e = cudaMemcpyAsync(P.m_items, items.data(), b_items, cudaMemcpyHostToDevice, st)) != cudaSuccess))
        return lsvd_ctx_cuda(ctx, e, "plan upload");
    // scratch: head | fb_count | agg_flags | pad | fb_list[count]
    char* sc = static_cast<char*>(P.d_scratch.get(256 + size_t(count) * 4, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "plan scratch");
    P.s_head = reinterpret_cast<int*>(sc);
    P.s_fb_count = P.s_head + 1;
    P.s_agg = P.s_head + 2;
    P.s_fb_list = reinterpret_cast<int32_t*>(sc + 256);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "plan sync");
    return LSVD_OK;
}

static cudaError_t enqueue_plan(lsvd_context* ctx, BatchPlan& P, const double* A, double* U,
                                double* S, double* Vt, lsvd_diag* diag, bool want_diag) {
    cudaStream_t st = ctx->stream;
    BatchArgs a;
    a.n = P.m_n;
    a.aoff = P.m_aoff;
    a.soff = P.m_soff;
    a.perm = P.m_perm;
    a.A = A;
    a.U = U;
    a.S = S;
    a.Vt = Vt;
    a.diag = diag;
    a.items = P.m_items;
    a.n_items = P.n_items;
    a.want_diag = want_diag ? 1 : 0;
    a.head = P.s_head;
    a.fb_count = P.s_fb_count;
    a.fb_list = P.s_fb_list;
    a.agg_flags = P.s_agg;
    for (int c = 0; c < kMaxClasses; ++c) a.cls[c] = P.cls[c];
    cudaError_t e = cudaMemsetAsync(P.s_head, 0, 16, st);
    if (e != cudaSuccess) return e;
    const int smem = std::max(P.smem_bytes, 16);
    const int grid = std::max(1, std::min(P.n_items, 2 * ctx->num_sms));
    if (P.precision == LSVD_PREC_MIXED_TF32)
        batched_mixed_kernel<kPrecTF32><<<grid, kCtaThreads, smem, st>>>(a);
    else if (P.precision == LSVD_PREC_MIXED_BF16)
        batched_mixed_kernel<kPrecBF16><<<grid, kCtaThreads, smem, st>>>(a);
    else
        batched_kernel<<<grid, kCtaThreads, smem, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int fsmem = team_smem_doubles(4, kCtaThreads / 32) * 8;
    fallback_kernel<<<std::max(1, std::min(ctx->num_sms, int(P.count))), kCtaThreads, fsmem, st>>>(a);
    return cudaGetLastError();
}

lsvd_status lsvd_run_plan(lsvd_context* ctx, BatchPlan& P, const double* A, double* U, double* S,
                          double* Vt, lsvd_diag* diag, bool want_diag, bool use_graph) {
    LSVD_TRACE("batched/run_plan");
    const int sm_bytes = std::max(P.smem_bytes, 16);
    cudaError_t e = P.precision == LSVD_PREC_MIXED_TF32
                        ? cudaFuncSetAttribute(batched_mixed_kernel<kPrecTF32>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, sm_bytes)
                    : P.precision == LSVD_PREC_MIXED_BF16
                        ? cudaFuncSetAttribute(batched_mixed_kernel<kPrecBF16>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, sm_bytes)
                        : cudaFuncSetAttribute(batched_kernel,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, sm_bytes);
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "smem attribute");
    if (!use_graph) {
        if ((e = enqueue_plan(ctx, P, A, U, S, Vt, diag, want_diag)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "batched launch");
        ctx->launches += 2;
        return LSVD_OK;
    }
    char key[160];
    std::snprintf(key, sizeof(key), "%p|%p|%p|%p|%p|%d|%p", (const void*)A, (void*)U, (void*)S,
                  (void*)Vt, (void*)diag, int(want_diag), (void*)ctx->stream);
    if (!P.graph_exec || P.bound_key != key) {
        P.invalidate_graph();
        cudaGraph_t g;
        if ((e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "begin capture");
        cudaError_t e2 = enqueue_plan(ctx, P, A, U, S, Vt, diag, want_diag);
        e = cudaStreamEndCapture(ctx->stream, &g);
        if (e2 != cudaSuccess) return lsvd_ctx_cuda(ctx, e2, "capture batched");
        if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "end capture");
        e = cudaGraphInstantiate(&P.graph_exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            P.graph_exec = nullptr;
            return lsvd_ctx_cuda(ctx, e, "graph instantiate");
        }
        P.bound_key = key;
    }
    if ((e = cudaGraphLaunch(P.graph_exec, ctx->stream)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "graph launch");
    ctx->launches += 2;
    return LSVD_OK;
}

static bool plan_matches(const BatchPlan& P, int64_t count, const int32_t* n, lsvd_precision prec) {
    return P.count == count && P.precision == prec && std::equal(P.ns.begin(), P.ns.end(), n);
}

BatchPlan* lsvd_get_plan(lsvd_context* ctx, int64_t count, const int32_t* n, lsvd_precision prec,
                         lsvd_status* st) {
    LSVD_TRACE("batched/plan");
    const uint64_t key = hash_ns(count, n) ^ (uint64_t(prec) << 61);
    auto it = ctx->plans.find(key);
    if (it != ctx->plans.end() && plan_matches(*it->second, count, n, prec)) {
        *st = LSVD_OK;
        return it->second.get();
    }
    auto P = std::make_unique<BatchPlan>();
    ClassShape shapes[kMaxClasses];
    lsvd_autotune_shapes(ctx, prec, shapes);
    *st = build_plan(ctx, count, n, shapes, prec, *P);
    if (*st != LSVD_OK) return nullptr;
    if (ctx->plans.size() > 16) ctx->plans.clear();
    BatchPlan* raw = P.get();
    ctx->plans[key] = std::move(P);
    return raw;
}

// The plan of chunk `slot` of the pipelined path: kept in its own slot (not
// in the shared cache), so two chunks never share staging buffers or a graph.
static BatchPlan* pipe_plan(lsvd_context* ctx, int slot, int64_t count, const int32_t* n,
                            lsvd_precision prec, lsvd_status* st) {
    std::unique_ptr<BatchPlan>& P = ctx->pipe_plans[slot];
    if (P && plan_matches(*P, count, n, prec)) {
        *st = LSVD_OK;
        return P.get();
    }
    P = std::make_unique<BatchPlan>();
    ClassShape shapes[kMaxClasses];
    lsvd_autotune_shapes(ctx, prec, shapes);
    *st = build_plan(ctx, count, n, shapes, prec, *P);
    if (*st != LSVD_OK) {
        P.reset();
        return nullptr;
    }
    return P.get();
}

// ----------------------------------------------------------- autotuner ----
//
// For every size class of the FP64 batched kernel (n = 5..64), times each
// feasible team shape -- warps per team {1, 2, 4, 8}, GEMM register tile
// {2, 4}, lanes per Jacobi pair {8, 16, 32}, matrices per team {1, 2}, with
// the CTA's teams fitting in 227 KB of shared memory -- on a seeded batch of
// `per_class` matrices spread over the class's sizes (CUDA events on the
// context's stream, best of three after one untimed run), keeps the fastest,
// and writes the choice to the cache that lsvd_autotune_shapes reads.
static void lcg_gauss(uint64_t& st, double* out, size_t count) {
    for (size_t i = 0; i < count; i += 2) {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        const double u1 = double((st >> 11) + 1) * (1.0 / 9007199254740993.0);
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        const double u2 = double(st >> 11) * (1.0 / 9007199254740992.0);
        const double r = std::sqrt(-2.0 * std::log(u1)), t = 6.283185307179586 * u2;
        out[i] = r * std::cos(t);
        if (i + 1 < count) out[i + 1] = r * std::sin(t);
    }
}

extern "C" lsvd_status lsvd_autotune_f64(lsvd_context* ctx, int64_t per_class, const char* cache_path,
                                         char* report, int64_t report_cap) {
    LSVD_TRACE("lsvd_autotune_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (per_class < 16 || per_class > 100000)
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_autotune_f64: per_class in 16..100000");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    ClassShape best[kMaxClasses];
    for (int c = 0; c < kMaxClasses; ++c) best[c] = lsvd_default_shape(c);
    std::string rep;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "autotune events");
    lsvd_status out = LSVD_OK;
    uint64_t seed = 0x5eed1234abcdull;
    for (int c = 1; c < kMaxClasses && out == LSVD_OK; ++c) {
        const int lo = kClassHi[c - 1] + 1, hi = kClassHi[c];
        if (lo > hi) continue;
        std::vector<int32_t> ns(static_cast<size_t>(per_class));
        int64_t elems = 0, selems = 0;
        for (int64_t t = 0; t < per_class; ++t) {
            ns[size_t(t)] = lo + int(t % (hi - lo + 1));
            elems += int64_t(ns[size_t(t)]) * ns[size_t(t)];
            selems += ns[size_t(t)];
        }
        std::vector<double> ha(static_cast<size_t>(elems));
        lcg_gauss(seed, ha.data(), ha.size());
        double* dA = static_cast<double*>(ctx->ws_a.get(size_t(elems) * 8, &e));
        double* dU = e == cudaSuccess ? static_cast<double*>(ctx->ws_u.get(size_t(elems) * 8, &e)) : nullptr;
        double* dS = e == cudaSuccess ? static_cast<double*>(ctx->ws_s.get(size_t(selems) * 8, &e)) : nullptr;
        double* dV = e == cudaSuccess ? static_cast<double*>(ctx->ws_vt.get(size_t(elems) * 8, &e)) : nullptr;
        if (e != cudaSuccess ||
            (e = cudaMemcpyAsync(dA, ha.data(), ha.size() * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess) {
            out = lsvd_ctx_cuda(ctx, e, "autotune batch");
            break;
        }
        double t_best = 1e30, t_def = -1.0;
        const ClassShape def = lsvd_default_shape(c);
        std::vector<ClassShape> cands;
        for (int w : {1, 2, 4, 8})
            for (int ts : {2, 4})
                for (int g : {8, 16, 32})
                    for (int pt : {1, 2})
                        if (size_t(kCtaThreads / (32 * w)) * team_smem_doubles(hi, w) * 8 <= 227 * 1024)
                            cands.push_back(ClassShape{w, ts, g, pt});
        for (const ClassShape& cand : cands) {
            ClassShape shapes[kMaxClasses];
            for (int k = 0; k < kMaxClasses; ++k) shapes[k] = lsvd_default_shape(k);
            shapes[c] = cand;
            BatchPlan P;
            if ((out = build_plan(ctx, per_class, ns.data(), shapes, LSVD_PREC_FP64, P)) != LSVD_OK) break;
            double t = 1e30;
            for (int rep_i = 0; rep_i < 4; ++rep_i) {
                float ms = 0.f;
                if ((e = cudaEventRecord(e0, st)) != cudaSuccess) break;
                if ((out = lsvd_run_plan(ctx, P, dA, dU, dS, dV, nullptr, false, false)) != LSVD_OK) break;
                if ((e = cudaEventRecord(e1, st)) != cudaSuccess || (e = cudaEventSynchronize(e1)) != cudaSuccess ||
                    (e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess)
                    break;
                if (rep_i > 0) t = std::min(t, double(ms));
            }
            if (out == LSVD_OK && e != cudaSuccess) out = lsvd_ctx_cuda(ctx, e, "autotune timing");
            if (out != LSVD_OK) break;
            if (cand.nwarps == def.nwarps && cand.ts == def.ts && cand.g == def.g && cand.per_team == def.per_team)
                t_def = t;
            if (t < t_best) {
                t_best = t;
                best[c] = cand;
            }
        }
        if (out != LSVD_OK) break;
        char line[200];
        std::snprintf(line, sizeof(line), "class %d (n %d..%d): %d,%d,%d,%d %.3f ms (default %d,%d,%d,%d %.3f ms)\n",
                      c, lo, hi, best[c].nwarps, best[c].ts, best[c].g, best[c].per_team, t_best, def.nwarps, def.ts,
                      def.g, def.per_team, t_def);
        rep += line;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (out != LSVD_OK) return out;
    // write the cache: keep a "shapes" entry for every precision, replace "shapes_fp64"
    std::string path = cache_path ? std::string(cache_path) : lsvd_autotune_cache_path();
    std::string tuned;
    for (int c = 1; c < kMaxClasses; ++c) {
        char b[48];
        std::snprintf(b, sizeof(b), "%s%d:%d,%d,%d,%d", tuned.empty() ? "" : ";", c, best[c].nwarps, best[c].ts,
                      best[c].g, best[c].per_team);
        tuned += b;
    }
    std::string shared;
    if (FILE* f = std::fopen(path.c_str(), "r")) {
        char buf[4096] = {0};
        const size_t got = std::fread(buf, 1, sizeof(buf) - 1, f);
        std::fclose(f);
        buf[got] = 0;
        if (const char* q = std::strstr(buf, "\"shapes\": \"")) {
            const char* end = std::strchr(q + 11, '"');
            if (end) shared.assign(q + 11, end);
        }
    }
    const size_t slash = path.find_last_of('/');
    if (slash != std::string::npos && slash > 0) {  // create the parent directories
        const std::string dir = path.substr(0, slash);
        for (size_t i = 1; i <= dir.size(); ++i)
            if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
    }
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_autotune_f64: cannot write " + path);
    std::fprintf(f, "{\"shapes_fp64\": \"%s\"%s%s%s, \"per_class\": %lld, \"sms\": %d}\n", tuned.c_str(),
                 shared.empty() ? "" : ", \"shapes\": \"", shared.c_str(), shared.empty() ? "" : "\"",
                 static_cast<long long>(per_class), ctx->num_sms);
    std::fclose(f);
    // plans built under the old shapes are stale now
    ctx->plans.clear();
    for (auto& pp : ctx->pipe_plans) pp.reset();
    if (report && report_cap > 0) std::snprintf(report, size_t(report_cap), "%s", rep.c_str());
    return LSVD_OK;
}

// The team shapes the planner would use now for `precision` (LSVD_SHAPES, the
// autotune cache, the defaults): out[4 c + {0..3}] = warps, tile, lanes per
// pair, matrices per team of class c (8 classes).
extern "C" lsvd_status lsvd_class_shapes(lsvd_context* ctx, lsvd_precision precision, int32_t* out) {
    if (!ctx || !out) return LSVD_BAD_ARGUMENT;
    ClassShape shapes[kMaxClasses];
    lsvd_autotune_shapes(ctx, precision, shapes);
    for (int c = 0; c < kMaxClasses; ++c) {
        out[4 * c] = shapes[c].nwarps;
        out[4 * c + 1] = shapes[c].ts;
        out[4 * c + 2] = shapes[c].g;
        out[4 * c + 3] = shapes[c].per_team;
    }
    return LSVD_OK;
}

// Host-pointer batches of at least kPipeMin matrices are cut into kPipeChunks
// contiguous chunks, each with its own plan and staging buffers (its own slot,
// even when two chunks have equal size lists), so that the copies overlap the
// solves: H2D of every chunk on one copy stream, the solves in order on the
// context stream, D2H of chunk c on a second copy stream as soon as its solve
// is done.  Only the first chunk's H2D and the last chunk's D2H stay exposed,
// so the chunk costs (sum of n^3) ramp up and down, kPipeWeight / 20 of the
// total each.  The results are those of the unchunked call (every matrix is
// solved independently).
constexpr int64_t kPipeMin = 16384;
constexpr int kPipeChunks = 8;
constexpr int kPipeWeight[kPipeChunks] = {1, 2, 3, 4, 4, 3, 2, 1};

static lsvd_status batched_pipelined(lsvd_context* ctx, int64_t count, const int32_t* n, const double* A,
                                     double* U, double* S, double* Vt, lsvd_diag* diags,
                                     lsvd_precision precision, bool want_diag) {
    LSVD_TRACE("batched/host_pipeline");
    constexpr int C = kPipeChunks;
    cudaError_t e = cudaSuccess;
    if (!ctx->h2d_stream && (e = cudaStreamCreateWithFlags(&ctx->h2d_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "copy stream");
    if (!ctx->d2h_stream && (e = cudaStreamCreateWithFlags(&ctx->d2h_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "copy stream");
    // cost-balanced cuts (every chunk non-empty) and the element offsets of every chunk
    std::vector<double> pre(size_t(count) + 1, 0.0);
    for (int64_t t = 0; t < count; ++t) pre[t + 1] = pre[t] + double(n[t]) * n[t] * n[t];
    int64_t cut[C + 1];
    cut[0] = 0;
    int wsum = 0, wtot = 0;
    for (int c = 0; c < C; ++c) wtot += kPipeWeight[c];
    for (int c = 1; c < C; ++c) {
        wsum += kPipeWeight[c - 1];
        const int64_t x = std::lower_bound(pre.begin(), pre.end(), pre[count] * wsum / wtot) - pre.begin();
        cut[c] = std::min(std::max(x, cut[c - 1] + 1), count - (C - c));
    }
    cut[C] = count;
    int64_t aoff[C + 1], soff[C + 1];
    {
        int64_t a = 0, s = 0, t = 0;
        for (int c = 0; c <= C; ++c) {
            for (; t < cut[c]; ++t) {
                a += int64_t(n[t]) * n[t];
                s += n[t];
            }
            aoff[c] = a;
            soff[c] = s;
        }
    }
    static_assert(C <= int(sizeof(ctx->pipe_plans) / sizeof(ctx->pipe_plans[0])), "one slot per chunk");
    BatchPlan* plans[C];
    for (int c = 0; c < C; ++c) {
        lsvd_status st;
        plans[c] = pipe_plan(ctx, c, cut[c + 1] - cut[c], n + cut[c], precision, &st);
        if (!plans[c]) return st;
    }
    cudaEvent_t ev[2 * C + 1];
    int created = 0;
    for (; created < 2 * C + 1; ++created)
        if ((e = cudaEventCreateWithFlags(&ev[created], cudaEventDisableTiming)) != cudaSuccess) break;
    auto destroy = [&]() {
        for (int i = 0; i < created; ++i) cudaEventDestroy(ev[i]);
    };
    if (e != cudaSuccess) {
        destroy();
        return lsvd_ctx_cuda(ctx, e, "events");
    }
    cudaEvent_t ev_start = ev[2 * C];
    lsvd_status out = LSVD_OK;
    double *dA[C], *dU[C], *dS[C], *dV[C];
    lsvd_diag* dD[C];
    // the copy streams start after everything already queued on the context stream
    if ((e = cudaEventRecord(ev_start, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(ctx->h2d_stream, ev_start, 0)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(ctx->d2h_stream, ev_start, 0)) != cudaSuccess)
        out = lsvd_ctx_cuda(ctx, e, "pipeline start");
    for (int c = 0; c < C && out == LSVD_OK; ++c) {
        BatchPlan& P = *plans[c];
        const int64_t cnt = cut[c + 1] - cut[c];
        dA[c] = static_cast<double*>(P.d_a.get(size_t(P.a_elems) * 8, &e));
        if (e == cudaSuccess) dU[c] = static_cast<double*>(P.d_u.get(size_t(P.a_elems) * 8, &e));
        if (e == cudaSuccess) dS[c] = static_cast<double*>(P.d_s.get(size_t(P.s_elems) * 8, &e));
        if (e == cudaSuccess) dV[c] = static_cast<double*>(P.d_vt.get(size_t(P.a_elems) * 8, &e));
        dD[c] = nullptr;
        if (e == cudaSuccess && diags)
            dD[c] = static_cast<lsvd_diag*>(P.d_diag.get(size_t(cnt) * sizeof(lsvd_diag), &e));
        if (e != cudaSuccess) {
            out = lsvd_ctx_cuda(ctx, e, "batch buffers");
            break;
        }
        if ((e = cudaMemcpyAsync(dA[c], A + aoff[c], size_t(P.a_elems) * 8, cudaMemcpyHostToDevice,
                                 ctx->h2d_stream)) != cudaSuccess ||
            (e = cudaEventRecord(ev[c], ctx->h2d_stream)) != cudaSuccess)
            out = lsvd_ctx_cuda(ctx, e, "copy A");
    }
    for (int c = 0; c < C && out == LSVD_OK; ++c) {
        BatchPlan& P = *plans[c];
        const int64_t cnt = cut[c + 1] - cut[c];
        if ((e = cudaStreamWaitEvent(ctx->stream, ev[c], 0)) != cudaSuccess) {
            out = lsvd_ctx_cuda(ctx, e, "pipeline wait");
            break;
        }
        if ((out = lsvd_run_plan(ctx, P, dA[c], dU[c], dS[c], dV[c], dD[c], want_diag, true)) != LSVD_OK) break;
        cudaStream_t s = ctx->d2h_stream;
        if ((e = cudaEventRecord(ev[C + c], ctx->stream)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(s, ev[C + c], 0)) != cudaSuccess ||
            (e = cudaMemcpyAsync(U + aoff[c], dU[c], size_t(P.a_elems) * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(S + soff[c], dS[c], size_t(P.s_elems) * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(Vt + aoff[c], dV[c], size_t(P.a_elems) * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (diags && (e = cudaMemcpyAsync(diags + cut[c], dD[c], size_t(cnt) * sizeof(lsvd_diag),
                                           cudaMemcpyDeviceToHost, s)) != cudaSuccess))
            out = lsvd_ctx_cuda(ctx, e, "copy out");
    }
    // wait for all three streams, then the per-chunk outcome flags
    if ((e = cudaStreamSynchronize(ctx->h2d_stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->d2h_stream)) != cudaSuccess) {
        if (out == LSVD_OK) out = lsvd_ctx_cuda(ctx, e, "pipeline sync");
    }
    int agg = 0;
    for (int c = 0; c < C && out == LSVD_OK; ++c) {
        int a = 0;
        if ((e = cudaMemcpy(&a, plans[c]->s_agg, 4, cudaMemcpyDeviceToHost)) != cudaSuccess) {
            out = lsvd_ctx_cuda(ctx, e, "flags");
            break;
        }
        agg |= a;
    }
    destroy();
    if (out != LSVD_OK) return out;
    if (agg & LSVD_MAT_NONFINITE) return LSVD_NONFINITE_INPUT;
    if (agg & LSVD_MAT_JACOBI_CAP) return LSVD_NOT_CONVERGED;
    return LSVD_OK;
}

extern "C" lsvd_status lsvd_svd_batched_f64(lsvd_context* ctx, int64_t count, const int32_t* n,
                                            const double* A, double* U, double* S, double* Vt,
                                            lsvd_diag* diags, lsvd_precision precision,
                                            uint32_t flags) {
    LSVD_TRACE("lsvd_svd_batched_f64");
    if (!ctx) return LSVD_BAD_ARGUMENT;
    if (count < 0 || (count > 0 && (!n || !A || !U || !S || !Vt)))
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "lsvd_svd_batched_f64: bad pointer");
    if (count == 0) return LSVD_OK;
    if (count > (int64_t(1) << 30)) return lsvd_ctx_fail(ctx, LSVD_UNSUPPORTED, "batch too large");
    for (int64_t t = 0; t < count; ++t)
        if (n[t] < 1 || n[t] > kMaxN)
            return lsvd_ctx_fail(ctx, n[t] < 1 ? LSVD_BAD_SHAPE : LSVD_UNSUPPORTED,
                                 "lsvd_svd_batched_f64: every n must be in 1..64");
    if (precision != LSVD_PREC_FP64 && precision != LSVD_PREC_MIXED_TF32 &&
        precision != LSVD_PREC_MIXED_BF16)
        return lsvd_ctx_fail(ctx, LSVD_BAD_ARGUMENT, "unknown precision");
    cudaSetDevice(ctx->device);
    if (!is_dev(flags) && count >= kPipeMin)
        return batched_pipelined(ctx, count, n, A, U, S, Vt, diags, precision, (flags & LSVD_WANT_DIAG) != 0);
    lsvd_status st;
    BatchPlan* P = lsvd_get_plan(ctx, count, n, precision, &st);
    if (!P) return st;
    const bool dev = is_dev(flags);
    const bool want_diag = (flags & LSVD_WANT_DIAG) != 0;
    cudaError_t e;
    const double* dA = A;
    double *dU = U, *dS = S, *dV = Vt;
    lsvd_diag* dD = diags;
    if (!dev) {
        dA = static_cast<double*>(P->d_a.get(size_t(P->a_elems) * 8, &e));
        if (e == cudaSuccess) dU = static_cast<double*>(P->d_u.get(size_t(P->a_elems) * 8, &e));
        if (e == cudaSuccess) dS = static_cast<double*>(P->d_s.get(size_t(P->s_elems) * 8, &e));
        if (e == cudaSuccess) dV = static_cast<double*>(P->d_vt.get(size_t(P->a_elems) * 8, &e));
        if (e == cudaSuccess && diags)
            dD = static_cast<lsvd_diag*>(P->d_diag.get(size_t(count) * sizeof(lsvd_diag), &e));
        if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "batch buffers");
        if ((e = cudaMemcpyAsync(const_cast<double*>(dA), A, size_t(P->a_elems) * 8,
                                 cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
            return lsvd_ctx_cuda(ctx, e, "copy A");
    }
    if ((st = lsvd_run_plan(ctx, *P, dA, dU, dS, dV, dD, want_diag, true)) != LSVD_OK) return st;
    if (!dev) {
        cudaStream_t s = ctx->stream;
        if ((e = cudaMemcpyAsync(U, dU, size_t(P->a_elems) * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(S, dS, size_t(P->s_elems) * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(Vt, dV, size_t(P->a_elems) * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (diags && (e = cudaMemcpyAsync(diags, dD, size_t(count) * sizeof(lsvd_diag),
                                           cudaMemcpyDeviceToHost, s)) != cudaSuccess))
            return lsvd_ctx_cuda(ctx, e, "copy out");
    }
    if (dev && (flags & LSVD_ASYNC)) return LSVD_OK;
    int agg = 0;
    if ((e = cudaMemcpyAsync(&agg, P->s_agg, 4, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "sync");
    if (agg & LSVD_MAT_NONFINITE) return LSVD_NONFINITE_INPUT;
    if (agg & LSVD_MAT_JACOBI_CAP) return LSVD_NOT_CONVERGED;
    return LSVD_OK;
}
