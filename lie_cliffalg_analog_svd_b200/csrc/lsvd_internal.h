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
    void* cublas = nullptr;  // cublasHandle_t of the large-polar FP64 GEMMs, created on first use
    // copy streams of the pipelined host-pointer batched path, created on first use
    cudaStream_t h2d_stream = nullptr, d2h_stream = nullptr;
    std::unordered_map<uint64_t, std::unique_ptr<BatchPlan>> plans;
    ~lsvd_context();
};

lsvd_status lsvd_ctx_fail(lsvd_context* ctx, lsvd_status st, const std::string& msg);
lsvd_status lsvd_ctx_cuda(lsvd_context* ctx, cudaError_t e, const char* where);

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
void lsvd_destroy_blas(void* handle);

// lsvd_autotune.cu
void lsvd_autotune_shapes(lsvd_context* ctx, lsvd_precision prec, ClassShape* shapes);
