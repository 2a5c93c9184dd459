// lsvd_trace.h -- NVTX ranges around the library's C-ABI entries and the
// phases of its multi-kernel solves, all in the NVTX domain "lsvd".
//
// NVTX3 is header-only.  With no tool attached (no NVTX_INJECTION64_PATH, no
// profiler) the first range resolves every NVTX call to a no-op and each later
// range costs one indirect call.  Under Nsight Systems, or any NVTX injection
// library, the ranges nest as: entry ("lsvd_svd_large_f64") > phase
// ("large/polar", "large/jacobi", ...).  Ranges mark host time: the kernels a
// range enqueues run later on their stream unless the entry synchronises.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace lsvd {

inline nvtxDomainHandle_t trace_domain() {
    static const nvtxDomainHandle_t d = nvtxDomainCreateA("lsvd");
    return d;
}

// Pushes a range named `name` (a string literal: NVTX keeps the pointer only for
// the call) on construction and pops it on destruction, so every return path of
// the enclosing scope closes it.
class TraceRange {
  public:
    explicit TraceRange(const char* name) {
        nvtxEventAttributes_t a = {};
        a.version = NVTX_VERSION;
        a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
        a.messageType = NVTX_MESSAGE_TYPE_ASCII;
        a.message.ascii = name;
        nvtxDomainRangePushEx(trace_domain(), &a);
    }
    ~TraceRange() { nvtxDomainRangePop(trace_domain()); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace lsvd

#define LSVD_TRACE_CAT2(a, b) a##b
#define LSVD_TRACE_CAT(a, b) LSVD_TRACE_CAT2(a, b)
// One range for the rest of the enclosing scope.
#define LSVD_TRACE(name) ::lsvd::TraceRange LSVD_TRACE_CAT(lsvd_trace_range_, __LINE__)(name)
