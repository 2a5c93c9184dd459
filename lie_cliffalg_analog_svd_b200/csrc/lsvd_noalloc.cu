// lsvd_noalloc.cu -- the batched FP64 SVD for callers that cannot allocate.
//
// Some callers may not allocate device memory at the point where they need
// an SVD: real-time loops where the implicit device synchronisation of
// cudaMalloc/cudaFree would stall other streams, and hosts whose device
// memory is owned by their own pool or allocator (a framework arena, a Rust
// or JVM runtime handing out preallocated buffers) and must not see a second
// allocator.  lsvd_svd_batched_noalloc_f64 serves them: the caller passes
// device buffers for the inputs and outputs, and every piece of working
// memory the solve needs (the work queue head, outcome flags, the per-size
// schedule and the micro->small escalation list) lives in one file-scope
// device array, g_noalloc_scratch, of LSVD_NOALLOC_SCRATCH_BYTES.  That array
// is part of the library image: every GPU that loads the library holds it
// until the process exits.  The schedule is built on the device by a setup
// kernel, so no host or device memory is allocated on any call.
//
// All calls share the one array.  Calls whose work overlaps on a GPU (two
// streams, or two host threads, at the same time on the same device) race on
// it and corrupt each other's schedules; serialise them.  The array keeps the
// last call's contents; each call rebuilds everything it reads and clears the
// counters that must start at zero.
#include <cuda_runtime.h>

#include <mutex>

#include "lsvd.h"
#include "lsvd_internal.h"
// device functions only: the kernels of lsvd_kernels.cuh live in lsvd_api.cu
#define LSVD_KERNELS_DEVICE_ONLY
#include "lsvd_kernels.cuh"

// The scratch of every no-allocation call (see the file comment).
static __device__ __align__(256) unsigned char g_noalloc_scratch[LSVD_NOALLOC_SCRATCH_BYTES];

namespace {

using namespace lsvd;

constexpr int64_t kMaxCount = LSVD_NOALLOC_MAX_COUNT;
constexpr size_t kHeader = 4096;
// per matrix: n (4) + aoff (8) + soff (8) + perm (4) + escalation slot (4) + item (16)
constexpr size_t kPerMatrix = 4 + 8 + 8 + 4 + 4 + sizeof(Item);
static_assert(kHeader + kPerMatrix * size_t(kMaxCount) <= LSVD_NOALLOC_SCRATCH_BYTES,
              "scratch too small for the stated maximum count");

struct ClassCfgArray {
    int per_item[kMaxClasses];
};

// header layout (ints): head, fb_count, agg, n_items, bad_n, hist[65], start[65]
struct Header {
    int head, fb_count, agg, n_items;
    int bad_n;  // sizes outside 1..64 seen on the device (the call then solves nothing)
    int hist[65];
    int start[65];
};

struct Layout {
    Header* hdr;
    int32_t* n;
    int64_t* aoff;
    int64_t* soff;
    int32_t* perm;
    int32_t* fb_list;
    Item* items;
};

__host__ __device__ inline Layout layout_of(unsigned char* base) {
    Layout L;
    L.hdr = reinterpret_cast<Header*>(base);
    unsigned char* p = base + kHeader;
    L.aoff = reinterpret_cast<int64_t*>(p);
    p += 8 * size_t(kMaxCount);
    L.soff = reinterpret_cast<int64_t*>(p);
    p += 8 * size_t(kMaxCount);
    L.items = reinterpret_cast<Item*>(p);
    p += sizeof(Item) * size_t(kMaxCount);
    L.n = reinterpret_cast<int32_t*>(p);
    p += 4 * size_t(kMaxCount);
    L.perm = reinterpret_cast<int32_t*>(p);
    p += 4 * size_t(kMaxCount);
    L.fb_list = reinterpret_cast<int32_t*>(p);
    return L;
}

// Size classes and work-item sizes of the batched planner (lsvd_api.cu):
// upper n of each class and matrices per item.
__constant__ int c_class_hi[kMaxClasses] = {4, 8, 16, 24, 32, 48, 64, 64};

// One CTA: offsets (prefix sums in input order), counting sort by n
// descending, and work items (one size class each, largest n first).
__global__ void __launch_bounds__(256, 1)
    noalloc_setup_kernel(int count, unsigned char* base, ClassCfgArray cfg) {
    Layout L = layout_of(base);
    Header* h = L.hdr;
    __shared__ int64_t carry_a, carry_s;
    const int tid = threadIdx.x;
    __shared__ int s_bad;
    if (tid == 0) {
        h->head = 0;
        h->fb_count = 0;
        h->agg = 0;
        h->n_items = 0;
        h->bad_n = 0;
        carry_a = 0;
        carry_s = 0;
        s_bad = 0;
    }
    for (int i = tid; i < 65; i += 256) h->hist[i] = 0;
    __syncthreads();
    // The host checked the sizes when the call was made; with LSVD_ASYNC the
    // caller's array is only read when the copy runs, so check again here and
    // solve nothing (n_items = 0) if a size left 1..64 in between.
    for (int t = tid; t < count; t += 256) {
        const int v = L.n[t];
        if (v < 1 || v > kMaxN) atomicOr(&s_bad, 1);
    }
    __syncthreads();
    if (s_bad) {
        if (tid == 0) h->bad_n = 1;
        return;
    }
    for (int t = tid; t < count; t += 256) atomicAdd(&h->hist[L.n[t]], 1);
    // exclusive prefix sums of n^2 and n, chunks of 256
    __shared__ int64_t sa[256], ss[256];
    for (int base0 = 0; base0 < count; base0 += 256) {
        const int t = base0 + tid;
        const int64_t nn = t < count ? int64_t(L.n[t]) : 0;
        sa[tid] = nn * nn;
        ss[tid] = nn;
        __syncthreads();
        for (int o = 1; o < 256; o <<= 1) {
            const int64_t va = tid >= o ? sa[tid - o] : 0, vs = tid >= o ? ss[tid - o] : 0;
            __syncthreads();
            sa[tid] += va;
            ss[tid] += vs;
            __syncthreads();
        }
        if (t < count) {
            L.aoff[t] = carry_a + sa[tid] - nn * nn;
            L.soff[t] = carry_s + ss[tid] - nn;
        }
        __syncthreads();
        if (tid == 255) {
            carry_a += sa[255];
            carry_s += ss[255];
        }
        __syncthreads();
    }
    if (tid == 0) {
        int acc = 0;
        for (int v = 64; v >= 1; --v) {  // descending n
            h->start[v] = acc;
            acc += h->hist[v];
        }
    }
    __syncthreads();
    for (int t = tid; t < count; t += 256) {
        const int pos = atomicAdd(&h->start[L.n[t]], 1);
        L.perm[pos] = t;
    }
    __syncthreads();
    // items: classes in descending n, each cut into chunks of per_item
    // matrices; class ranges follow from the histogram
    __shared__ int cstart[kMaxClasses], citems[kMaxClasses + 1];
    if (tid == 0) {
        int pos = 0, items = 0;
        for (int c = kMaxClasses - 1; c >= 0; --c) {
            const int lo = c == 0 ? 1 : c_class_hi[c - 1] + 1, hi = c_class_hi[c];
            int cnt = 0;
            for (int v = lo; v <= hi; ++v) cnt += h->hist[v];
            cstart[c] = pos;
            citems[c] = items;
            pos += cnt;
            items += (cnt + cfg.per_item[c] - 1) / cfg.per_item[c];
        }
        citems[kMaxClasses] = items;
        h->n_items = items;
    }
    __syncthreads();
    for (int c = 0; c < kMaxClasses; ++c) {
        const int lo = c == 0 ? 1 : c_class_hi[c - 1] + 1, hi = c_class_hi[c];
        int cnt = 0;
        for (int v = lo; v <= hi; ++v) cnt += h->hist[v];
        const int ni = (cnt + cfg.per_item[c] - 1) / cfg.per_item[c];
        for (int k = tid; k < ni; k += 256) {
            Item it;
            it.cls = c;
            it.first = cstart[c] + k * cfg.per_item[c];
            it.count = min(cnt - k * cfg.per_item[c], cfg.per_item[c]);
            it.pad_ = 0;
            L.items[citems[c] + k] = it;
        }
    }
}

struct NoallocArgs {
    unsigned char* base;
    const double* A;
    double* U;
    double* S;
    double* Vt;
    lsvd_diag* diag;
    int want_diag;
    ClassCfg cls[kMaxClasses];
};

__device__ __forceinline__ BatchArgs args_of(const NoallocArgs& na, const Layout& L) {
    BatchArgs a;
    a.n = L.n;
    a.aoff = L.aoff;
    a.soff = L.soff;
    a.perm = L.perm;
    a.A = na.A;
    a.U = na.U;
    a.S = na.S;
    a.Vt = na.Vt;
    a.diag = na.diag;
    a.items = L.items;
    a.n_items = L.hdr->n_items;
    a.want_diag = na.want_diag;
    a.head = &L.hdr->head;
    a.fb_count = &L.hdr->fb_count;
    a.fb_list = L.fb_list;
    a.agg_flags = &L.hdr->agg;
    for (int c = 0; c < kMaxClasses; ++c) a.cls[c] = na.cls[c];
    return a;
}

// The persistent loop of batched_kernel, reading its schedule from the
// static scratch.
__global__ void __launch_bounds__(kCtaThreads, 2) noalloc_batched_kernel(const NoallocArgs na) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_item;
    const Layout L = layout_of(na.base);
    const BatchArgs args = args_of(na, L);
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

__global__ void __launch_bounds__(kCtaThreads, 1) noalloc_fallback_kernel(const NoallocArgs na) {
    extern __shared__ __align__(16) double smem[];
    const Layout L = layout_of(na.base);
    const BatchArgs args = args_of(na, L);
    const int cnt = L.hdr->fb_count;
    Team tm;
    tm.tid = threadIdx.x;
    tm.nthreads = kCtaThreads;
    tm.warp = threadIdx.x / 32;
    tm.lane = threadIdx.x % 32;
    tm.nwarps = kCtaThreads / 32;
    tm.bar = 1;
    for (int idx = blockIdx.x; idx < cnt; idx += gridDim.x) {
        SmallJob job = make_job(args, L.fb_list[idx]);
        job.extra_flags = LSVD_MAT_MICRO_FALLBACK;
        small_solve_team<2, 8>(tm, job, smem);
        __syncthreads();
    }
}

// Per-device set-up: the device address of g_noalloc_scratch (the host-side
// symbol is only a stand-in and must never be passed to a kernel), the
// dynamic shared-memory limit of the persistent kernel and the SM count.
struct DeviceSetup {
    std::mutex mu;
    bool done = false;  // set only by a set-up that succeeded; a failed one is retried
    unsigned char* scratch = nullptr;
    int num_sms = 0;
};
DeviceSetup g_setup[64];

// Runs the per-device set-up once it succeeds; returns its error otherwise.
cudaError_t device_setup(DeviceSetup& ds, int dev, int smem) {
    std::lock_guard<std::mutex> lock(ds.mu);
    if (ds.done) return cudaSuccess;
    void* p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(noalloc_batched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int sms = 0;
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (err != cudaSuccess) {
        cudaGetLastError();  // leave no pending error behind; the next call retries
        return err;
    }
    ds.scratch = static_cast<unsigned char*>(p);
    ds.num_sms = sms;
    ds.done = true;
    return cudaSuccess;
}

int noalloc_smem_bytes(const ClassCfg* cls) {
    int mx = 0;
    for (int c = 0; c < kMaxClasses; ++c)
        if (cls[c].nwarps) {
            const int teams = kCtaThreads / (32 * cls[c].nwarps);
            mx = mx > teams * cls[c].slice * 8 ? mx : teams * cls[c].slice * 8;
        }
    return mx;
}

}  // namespace

extern "C" lsvd_status lsvd_svd_batched_noalloc_f64(void* stream, int64_t count, const int32_t* n,
                                                    const double* A, double* U, double* S,
                                                    double* Vt, lsvd_diag* diags, uint32_t flags) {
    LSVD_TRACE("lsvd_svd_batched_noalloc_f64");
    if (count < 0 || (count > 0 && (!n || !A || !U || !S || !Vt))) return LSVD_BAD_ARGUMENT;
    if (count > kMaxCount) return LSVD_UNSUPPORTED;  // more matrices than the scratch holds
    if (count == 0) return LSVD_OK;
    for (int64_t t = 0; t < count; ++t)
        if (n[t] < 1 || n[t] > kMaxN) return n[t] < 1 ? LSVD_BAD_SHAPE : LSVD_UNSUPPORTED;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return LSVD_NO_DEVICE;
    // classes: the batched planner's default team shapes
    NoallocArgs na;
    ClassCfgArray cfga;
    for (int c = 0; c < kMaxClasses; ++c) {
        const ClassShape s = lsvd_default_shape(c);
        const int hi = c == 0 ? 4 : (c == 1 ? 8 : c == 2 ? 16 : c == 3 ? 24 : c == 4 ? 32 : c == 5 ? 48 : 64);
        na.cls[c].nwarps = s.nwarps;
        na.cls[c].variant = (s.ts == 4 ? 3 : 0) + (s.g == 16 ? 1 : s.g == 32 ? 2 : 0);
        na.cls[c].slice = s.nwarps ? team_smem_doubles(hi, s.nwarps) : 0;
        na.cls[c].pad_ = 0;
        cfga.per_item[c] = s.nwarps == 0 ? kCtaThreads
                                         : (kCtaThreads / (32 * s.nwarps)) * (s.per_team > 0 ? s.per_team : 1);
    }
    const int smem = noalloc_smem_bytes(na.cls);
    DeviceSetup& ds = g_setup[dev];
    // The first successful call on a device does the set-up (the device
    // address of the static array, kernel attributes); a set-up that failed
    // is tried again on the next call.
    if (device_setup(ds, dev, smem) != cudaSuccess) return LSVD_CUDA_ERROR;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Layout L = layout_of(ds.scratch);
    na.base = ds.scratch;
    na.A = A;
    na.U = U;
    na.S = S;
    na.Vt = Vt;
    na.diag = diags;
    na.want_diag = (flags & LSVD_WANT_DIAG) ? 1 : 0;
    cudaError_t e = cudaMemcpyAsync(L.n, n, size_t(count) * 4, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return LSVD_CUDA_ERROR;
    noalloc_setup_kernel<<<1, 256, 0, st>>>(int(count), ds.scratch, cfga);
    const int grid = ds.num_sms * 2 < count ? ds.num_sms * 2 : int(count);
    noalloc_batched_kernel<<<grid > 0 ? grid : 1, kCtaThreads, smem, st>>>(na);
    const int fgrid = ds.num_sms < count ? ds.num_sms : int(count);
    noalloc_fallback_kernel<<<fgrid > 0 ? fgrid : 1, kCtaThreads, team_smem_doubles(4, kCtaThreads / 32) * 8, st>>>(na);
    if ((e = cudaGetLastError()) != cudaSuccess) return LSVD_CUDA_ERROR;
    if (flags & LSVD_ASYNC) return LSVD_OK;
    int agg_bad[5] = {0, 0, 0, 0, 0};  // head, fb_count, agg, n_items, bad_n
    if (cudaMemcpyAsync(agg_bad, L.hdr, sizeof(agg_bad), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return LSVD_CUDA_ERROR;
    const int agg = agg_bad[2];
    if (agg_bad[4]) return LSVD_BAD_ARGUMENT;
    if (agg & LSVD_MAT_NONFINITE) return LSVD_NONFINITE_INPUT;
    if (agg & LSVD_MAT_JACOBI_CAP) return LSVD_NOT_CONVERGED;
    return LSVD_OK;
}
