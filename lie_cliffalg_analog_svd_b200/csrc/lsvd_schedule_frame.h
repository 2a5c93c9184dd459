// lsvd_schedule_frame.h -- the binary phase-schedule frame's layout helpers,
// shared by the host encoder/decoder (lsvd_schedule.cpp) and the device
// encoder of rotor streams (lsvd_schedule_dev.cu).
#pragma once
#include <cstdint>
#include <cstring>

#include "lsvd.h"

#ifdef __CUDACC__
#define LSVD_HD __host__ __device__ __forceinline__
#else
#define LSVD_HD inline
#endif

namespace lsvd {
namespace sched {

static_assert(sizeof(lsvd_schedule_header) == 64, "frame header is 64 bytes");
static_assert(sizeof(lsvd_schedule_record) == 56, "frame record is 56 bytes");
static_assert(sizeof(lsvd_mzi_phase) == 48, "lsvd_mzi_phase layout");

constexpr int64_t kMaxChannels = 65535;  // record indices are 16-bit

LSVD_HD int64_t frame_bytes(int64_t events, int64_t signs, bool energy) {
    return int64_t(sizeof(lsvd_schedule_header)) + events * int64_t(sizeof(lsvd_schedule_record)) + signs * 8 +
           (energy ? events * 16 : 0);
}

LSVD_HD lsvd_schedule_header make_header(int32_t target, uint32_t flags, int64_t channels, int64_t events,
                                         int64_t signs) {
    lsvd_schedule_header h;
    const char m[8] = {'P', 'S', 'C', 'H', 'E', 'D', 'v', '1'};
    for (int k = 0; k < 8; ++k) h.magic[k] = m[k];
    h.header_bytes = uint32_t(sizeof(lsvd_schedule_header));
    h.record_bytes = uint32_t(sizeof(lsvd_schedule_record));
    h.target = uint32_t(target);
    h.flags = flags;
    h.channels = channels;
    h.total_events = events;
    h.n_signs = signs;
    h.reserved[0] = h.reserved[1] = 0;
    return h;
}

// Event of one accepted rotation V <- V G(i, j, t) in the compiler's
// reconstruction convention (src/lie_svd_compiler.rs:396-411): rows (j, i),
// angle -t on both sides, source gpu_jacobi, kind jacobi_rotation.
LSVD_HD lsvd_schedule_record rotor_record(const lsvd_rotor& r) {
    lsvd_schedule_record e;
    e.layer = r.round;
    e.i = r.j;
    e.j = r.i;
    e.phi_l = 0.0;
    e.phi_r = 0.0;
    e.theta = -r.theta;
    e.theta_l = -r.theta;
    e.theta_r = -r.theta;
    e.source = uint8_t(LSVD_SCHED_SOURCE_GPU_JACOBI);
    e.kind = uint8_t(LSVD_SCHED_KIND_JACOBI_ROTATION);
    e.reserved0 = 0;
    e.reserved1 = 0;
    return e;
}

LSVD_HD bool rotor_ok(const lsvd_rotor& r, int64_t channels) { return r.i < r.j && int64_t(r.j) < channels; }

}  // namespace sched
}  // namespace lsvd
