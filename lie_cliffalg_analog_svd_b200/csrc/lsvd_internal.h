// lsvd_internal.h -- host-side internals shared by the .cu files of
// liblsvd_b200.so (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "lsvd.h"
#include "lsvd_trace.h"

namespace lsvd {
constexpr int kMaxClasses = 8;

// Work-item size class: team shape and tile variant for a range of n.
struct ClassCfg {
    int nwarps;   // warps per team (1, 2, 4, 8); 0 = micro (thread per matrix)
    int variant;  // 0..5 = (TS, G) in {2,4} x {8,16,32}
    int slice;    // shared-memory doubles per team
    int pad_;
};

struct Item {
    int cls;
    int first;  // index into the sorted permutation
    int count;
    int pad_;
};
}  // namespace lsvd

// Grow-only device allocation owned by a context or plan.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    void* get(size_t want, cudaError_t* err);
    void release();
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

// Team shape for one size class of the batched kernel.
struct ClassShape {
    int nwarps;    // warps per team (0 = micro, thread per matrix)
    int ts;        // GEMM register tile (2 or 4)
    int g;         // lanes per Jacobi pair (8, 16 or 32)
    int per_team;  // matrices per team per work item
};

struct BatchPlan {
    int64_t count = 0;
    std::vector<int32_t> ns;
    int64_t a_elems = 0, s_elems = 0;
    int n_items = 0;
    int smem_bytes = 0;
    lsvd_precision precision = LSVD_PREC_FP64;
    // device metadata
    DeviceBuffer d_meta, d_scratch;
    int32_t* m_n = nullptr;
    int64_t* m_aoff = nullptr;
    int64_t* m_soff = nullptr;
    int32_t* m_perm = nullptr;
    lsvd::Item* m_items = nullptr;
    int* s_head = nullptr;
    int* s_fb_count = nullptr;
    int* s_agg = nullptr;
    int32_t* s_fb_list = nullptr;
    // staging buffers for host-pointer calls
    DeviceBuffer d_a, d_u, d_s, d_vt, d_diag;
    // captured graph, bound to one set of device pointers
    cudaGraphExec_t graph_exec = nullptr;
    std::string bound_key;
    lsvd::ClassCfg cls[lsvd::kMaxClasses];
    void invalidate_graph();
    ~BatchPlan();
};

struct lsvd_context {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;
    int64_t launches = 0;
    DeviceBuffer ws_a, ws_u, ws_s, ws_vt, ws_diag, ws_misc, ws_rot, ws_polar;
    DeviceBuffer ws_large;  // large SVD: A, the [G; V] panel store, Gram partials, rotations
    DeviceBuffer ws_splitk;  // lsvd_gemm_f64: per-slice partial products of a split inner dimension
    // copy streams of the pipelined host-pointer batched path, created on first use
    cudaStream_t h2d_stream = nullptr, d2h_stream = nullptr;
    // side branch of the large solve's sweep graph (V's update), created on first use
    cudaStream_t side_stream = nullptr;
    cudaStream_t side_stream2 = nullptr;  // large solve: the P update tiles the next layer does not read
    std::unordered_map<uint64_t, std::unique_ptr<BatchPlan>> plans;
    // one plan per chunk of the pipelined host-pointer path: every chunk owns
    // its staging buffers, even when two chunks have the same size list
    std::unique_ptr<BatchPlan> pipe_plans[8];
    void* pinned = nullptr;  // small page-locked host buffer (device-to-host status reads)
    size_t pinned_bytes = 0;
    ~lsvd_context();
};

lsvd_status lsvd_ctx_fail(lsvd_context* ctx, lsvd_status st, const std::string& msg);
lsvd_status lsvd_ctx_cuda(lsvd_context* ctx, cudaError_t e, const char* where);
// The context's page-locked host buffer of at least `bytes` (grow-only); NULL on failure.
void* lsvd_ctx_pinned(lsvd_context* ctx, size_t bytes);

// lsvd_api.cu
int lsvd_class_of(int n);
ClassShape lsvd_default_shape(int cls);
BatchPlan* lsvd_get_plan(lsvd_context* ctx, int64_t count, const int32_t* n, lsvd_precision prec,
                         lsvd_status* st);
lsvd_status lsvd_run_plan(lsvd_context* ctx, BatchPlan& P, const double* A, double* U, double* S,
                          double* Vt, lsvd_diag* diag, bool want_diag, bool use_graph);
lsvd_status lsvd_single_small(lsvd_context* ctx, int64_t n, const double* A, int64_t lda,
                              double* U, int64_t ldu, double* S, double* Vt, int64_t ldvt,
                              lsvd_diag* diag, lsvd_rotor* rotors, int64_t rotor_cap,
                              int64_t* rotor_count, int32_t* perm, uint32_t flags,
                              int extra_flags, bool host_meta);

// lsvd_polar.cu
// Newton-Schulz polar iteration on the device matrix A (m x n, leading
// dimension lda) in `precision`, with at most fp64_cap FP64 iterations after
// the low-precision phase (all iterations for FP64).  The factor is left in
// the context's polar workspace: *X (m x n, leading dimension *ldx, even).
lsvd_status lsvd_polar_run(lsvd_context* ctx, int64_t m, int64_t n, const double* A, int64_t lda,
                           lsvd_precision precision, int fp64_cap, double** X, int64_t* ldx,
                           lsvd_polar_info* info);

// lsvd_large.cu: SVD of one matrix beyond the shared-memory kernels (rows x
// cols, either orientation; wide inputs run on the transpose).  U rows x k,
// S k, Vt k x cols with k = min(rows, cols); pointers host or device.
lsvd_status lsvd_large_solve(lsvd_context* ctx, int64_t rows, int64_t cols, const double* A, int64_t lda,
                             double* U, int64_t ldu, double* S, double* Vt, int64_t ldvt,
                             lsvd_precision precision, lsvd_large_info* info, lsvd_diag* diag, bool want_diag);

// lsvd_autotune.cu
void lsvd_autotune_shapes(lsvd_context* ctx, lsvd_precision prec, ClassShape* shapes);
std::string lsvd_autotune_cache_path();
