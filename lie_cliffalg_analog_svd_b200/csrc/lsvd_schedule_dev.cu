// lsvd_schedule_dev.cu -- the binary phase-schedule frame of a rotor stream
// written on the device: the stream the Jacobi sweeps left in HBM becomes
// the frame in HBM without a trip through the host (the JSON text of the same
// schedule is the host compiler's, lsvd_schedule.cpp).
//
// One thread per event: a 256-event block stages its records (7 words each)
// in shared memory and stores the block's contiguous 14 KB span with
// coalesced 8-byte stores; the same threads write the +1 diagonal signs and
// block 0 the header.  HBM-bound: 16 bytes read and 56 written per event.
#include <cuda_runtime.h>

#include "lsvd.h"
#include "lsvd_internal.h"
#include "lsvd_schedule_frame.h"

lsvd_status lsvd_schedule_binary_rotors_host(const lsvd_rotor* rotors, int64_t count, int64_t channels,
                                             int32_t target, void* out, int64_t cap, int64_t* len);

namespace {

constexpr int kThreads = 256;
constexpr int kWords = int(sizeof(lsvd_schedule_record) / 8);  // 7

__global__ void __launch_bounds__(kThreads) frame_kernel(const lsvd_rotor* __restrict__ rotors, int64_t count,
                                                         int64_t channels, int32_t target,
                                                         unsigned long long* __restrict__ frame,
                                                         int* __restrict__ bad) {
    __shared__ unsigned long long st[kThreads * kWords];
    const int64_t base = int64_t(blockIdx.x) * kThreads;
    const int64_t t = base + threadIdx.x;
    if (t == 0) {
        const lsvd_schedule_header h =
            lsvd::sched::make_header(target, LSVD_SCHED_CANONICAL, channels, count, channels);
        const unsigned long long* hw = reinterpret_cast<const unsigned long long*>(&h);
#pragma unroll
        for (int w = 0; w < 8; ++w) frame[w] = hw[w];
    }
    unsigned long long* rec_out = frame + 8;  // 64-byte header
    if (t < count) {
        const lsvd_rotor r = rotors[t];
        if (!lsvd::sched::rotor_ok(r, channels)) atomicAdd(bad, 1);
        const lsvd_schedule_record e = lsvd::sched::rotor_record(r);
        const unsigned long long* ew = reinterpret_cast<const unsigned long long*>(&e);
#pragma unroll
        for (int w = 0; w < kWords; ++w) st[threadIdx.x * kWords + w] = ew[w];
    }
    __syncthreads();
    const int64_t here = count - base < kThreads ? count - base : kThreads;
    for (int64_t w = threadIdx.x; w < here * kWords; w += kThreads) rec_out[base * kWords + w] = st[w];
    // diagonal signs after the records: all +1 (the stream's rotations are
    // the whole orthogonal factor)
    if (t < channels) {
        double* signs = reinterpret_cast<double*>(rec_out + count * kWords);
        signs[t] = 1.0;
    }
}

}  // namespace

extern "C" LSVD_API lsvd_status lsvd_schedule_binary_from_rotors(lsvd_context* ctx, const lsvd_rotor* rotors,
                                                                 int64_t count, int64_t channels, int32_t target,
                                                                 void* out, int64_t cap, int64_t* len,
                                                                 uint32_t flags) {
    LSVD_TRACE("lsvd_schedule_binary_from_rotors");
    if (count < 0 || channels < 0 || (count > 0 && !rotors) || (target != 0 && target != 1) ||
        (flags & ~(LSVD_DEVICE_POINTERS | LSVD_ASYNC)) != 0)
        return LSVD_BAD_ARGUMENT;
    if (channels > lsvd::sched::kMaxChannels || count > 0xffffffffLL) return LSVD_UNSUPPORTED;
    if (!(flags & LSVD_DEVICE_POINTERS))
        return lsvd_schedule_binary_rotors_host(rotors, count, channels, target, out, cap, len);
    if (!ctx) return LSVD_BAD_ARGUMENT;
    const int64_t bytes = lsvd::sched::frame_bytes(count, channels, false);
    if (len) *len = bytes;
    if (!out) return LSVD_OK;
    if (cap < bytes) return LSVD_ROTOR_OVERFLOW;
    if ((reinterpret_cast<uintptr_t>(out) & 7) || (reinterpret_cast<uintptr_t>(rotors) & 7))
        return LSVD_BAD_ARGUMENT;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "set device");
    cudaStream_t st = ctx->stream;
    int* bad = static_cast<int*>(ctx->ws_misc.get(256, &e));
    if (e != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "frame flag");
    if ((e = cudaMemsetAsync(bad, 0, sizeof(int), st)) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "frame flag");
    const int64_t work = count > channels ? count : channels;
    const int64_t blocks = work > 0 ? (work + kThreads - 1) / kThreads : 1;
    frame_kernel<<<unsigned(blocks), kThreads, 0, st>>>(rotors, count, channels, target,
                                                        static_cast<unsigned long long*>(out), bad);
    if ((e = cudaGetLastError()) != cudaSuccess) return lsvd_ctx_cuda(ctx, e, "frame kernel");
    ctx->launches += 1;
    if (flags & LSVD_ASYNC) return LSVD_OK;
    int* hb = static_cast<int*>(lsvd_ctx_pinned(ctx, sizeof(int)));
    if (!hb) return lsvd_ctx_cuda(ctx, cudaErrorMemoryAllocation, "pinned flag");
    if ((e = cudaMemcpyAsync(hb, bad, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return lsvd_ctx_cuda(ctx, e, "frame sync");
    return *hb ? LSVD_BAD_ARGUMENT : LSVD_OK;
}
