// lsvd_schedule.cpp -- the phase-schedule-v1 compiler on the host:
// HardwareSchedule (src/lie_svd_compiler.rs:27-266) fed by the GPU rotor
// stream or by a finished orthogonal matrix.  Serialisation only; the rotor
// stream itself is produced on the device by the Jacobi sweeps.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lsvd.h"
#include "lsvd_schedule_frame.h"

namespace {

struct Event {
    int64_t layer, i, j;
    double phi_l, phi_r, theta, theta_l, theta_r;
    const char* source;
    const char* kind;
    bool has_before = false, has_after = false;  // Option<f64> energy_before / energy_after
    double energy_before = 0.0, energy_after = 0.0;
};

// Rust `{:.17e}`: 17 fractional digits, exponent without '+' or zero padding.
std::string fmt_e17(double x) {
    if (std::isnan(x)) return "NaN";
    if (std::isinf(x)) return x < 0 ? "-inf" : "inf";
    char tmp[64];
    std::snprintf(tmp, sizeof(tmp), "%.17e", x);
    std::string t(tmp);
    const size_t e = t.find('e');
    return t.substr(0, e) + "e" + std::to_string(std::atoi(t.c_str() + e + 1));
}

// Rust `{}` for the +-1 / NaN entries of diagonal_signs.
std::string fmt_display(double x) {
    if (std::isnan(x)) return "NaN";
    if (x == std::floor(x) && std::fabs(x) < 1e15) {
        char tmp[32];
        std::snprintf(tmp, sizeof(tmp), "%s%lld", std::signbit(x) ? "-" : "",
                      (long long)std::fabs(x));
        return tmp;
    }
    char tmp[64];
    std::snprintf(tmp, sizeof(tmp), "%.17g", x);
    return tmp;
}

const char* target_name(int target) { return target == 1 ? "fpga_rotor_mesh" : "mzi_mesh"; }

// Name tables of the binary frame's codes: sources as HardwareSchedule's
// constructors write them, kinds as real_kind / complex_kind
// (src/lie_svd_compiler.rs:268-287) and the two solver-side kinds.
constexpr const char* kSources[] = {"real_phaseflow", "complex_phaseflow", "orthogonal_givens", "gpu_jacobi"};
constexpr const char* kKinds[] = {"golden_prespin", "causal_antispin", "cross_phase_yinyang",
                                  "phase_conjugate", "bottleneck", "phase_jump",
                                  "unwrap", "directional", "surgery",
                                  "complex_golden_prespin", "complex_diagonal_phase", "givens_elimination",
                                  "jacobi_rotation"};
constexpr int kNumSources = int(sizeof(kSources) / sizeof(kSources[0]));
constexpr int kNumKinds = int(sizeof(kKinds) / sizeof(kKinds[0]));
constexpr int kNumRealKinds = 9;

// to_json_string, src/lie_svd_compiler.rs:213-265.
std::string to_json(int target, int64_t channels, const std::vector<Event>& ev,
                    const std::vector<double>& signs) {
    std::string out = "{\n";
    out += "  \"format_version\": \"phase-schedule-v1\",\n";
    out += std::string("  \"target\": \"") + target_name(target) + "\",\n";
    out += "  \"channels\": " + std::to_string(channels) + ",\n";
    out += "  \"total_events\": " + std::to_string(ev.size()) + ",\n";
    out += "  \"events\": [\n";
    for (size_t k = 0; k < ev.size(); ++k) {
        const Event& e = ev[k];
        out += "    {\"layer\": " + std::to_string(e.layer) + ", \"i\": " + std::to_string(e.i) +
               ", \"j\": " + std::to_string(e.j) + ", \"phi_l\": " + fmt_e17(e.phi_l) +
               ", \"phi_r\": " + fmt_e17(e.phi_r) + ", \"theta\": " + fmt_e17(e.theta) +
               ", \"theta_l\": " + fmt_e17(e.theta_l) + ", \"theta_r\": " + fmt_e17(e.theta_r) +
               ", \"source\": \"" + e.source + "\", \"kind\": \"" + e.kind + "\"";
        if (e.has_before) out += ", \"energy_before\": " + fmt_e17(e.energy_before);
        if (e.has_after) out += ", \"energy_after\": " + fmt_e17(e.energy_after);
        out += "}";
        if (k + 1 != ev.size()) out += ",";
        out += "\n";
    }
    out += "  ]";
    if (!signs.empty()) {
        out += ",\n  \"diagonal_signs\": [";
        for (size_t k = 0; k < signs.size(); ++k) {
            if (k) out += ", ";
            out += fmt_display(signs[k]);
        }
        out += "]";
    }
    out += "\n}\n";
    return out;
}

lsvd_status emit(const std::string& s, char* json, int64_t cap, int64_t* len) {
    if (len) *len = int64_t(s.size());
    if (!json || cap <= 0) return json ? LSVD_ROTOR_OVERFLOW : LSVD_OK;
    if (int64_t(s.size()) + 1 > cap) {
        std::memcpy(json, s.data(), size_t(cap - 1));
        json[cap - 1] = 0;
        return LSVD_ROTOR_OVERFLOW;
    }
    std::memcpy(json, s.data(), s.size() + 1);
    return LSVD_OK;
}

}  // namespace

// HardwareSchedule::from_orthogonal_matrix + to_json_string
// (src/lie_svd_compiler.rs:144-198, :213-265): Givens elimination of the
// strict lower triangle, one layer per event, +-1 diagonal signs.
extern "C" LSVD_API lsvd_status lsvd_schedule_from_orthogonal(int64_t d, const double* V,
                                                              int32_t target, char* json,
                                                              int64_t cap, int64_t* len) {
    if (d < 0 || (d > 0 && !V) || (target != 0 && target != 1)) return LSVD_BAD_ARGUMENT;
    std::vector<double> r(V, V + d * d);
    std::vector<Event> ev;
    int64_t layer = 0;
    for (int64_t j = 0; j < d; ++j) {
        for (int64_t i = j + 1; i < d; ++i) {
            const double a = r[size_t(j * d + j)], b = r[size_t(i * d + j)];
            if (std::fabs(b) <= 1e-300) continue;
            const double nrm = std::sqrt(a * a + b * b);
            const double c = a / nrm, s = b / nrm;
            for (int64_t k = 0; k < d; ++k) {
                const double rj = r[size_t(j * d + k)], ri = r[size_t(i * d + k)];
                r[size_t(j * d + k)] = c * rj + s * ri;
                r[size_t(i * d + k)] = -s * rj + c * ri;
            }
            const double th = std::atan2(s, c);
            ev.push_back(Event{layer, i, j, 0.0, 0.0, th, th, 0.0, "orthogonal_givens",
                               "givens_elimination"});
            ++layer;
        }
    }
    std::vector<double> signs(static_cast<size_t>(d));
    for (int64_t k = 0; k < d; ++k) {
        const double x = r[size_t(k * d + k)];
        signs[size_t(k)] = std::isnan(x) ? x : (std::signbit(x) ? -1.0 : 1.0);
    }
    return emit(to_json(target, d, ev, signs), json, cap, len);
}

// Schedule of a GPU rotor stream.  Each accepted rotation V <- V G(i, j, t)
// (columns i < j) becomes one event in layer `round` (rounds are
// conflict-free round-robin layers).  In the compiler's reconstruction
// convention (src/lie_svd_compiler.rs:396-411: V = G_1^T ... G_m^T D with
// row rotations on (j_ev, i_ev)) the event is (i_ev, j_ev) = (j, i) and
// theta_l = -t; theta_r = theta_l marks the symmetric (two-sided) rotor of
// the eigensolve; diagonal_signs are all +1.  The stream reconstructs the
// unsorted eigenbasis; `perm` (optional) is returned unchanged by the solver
// and orders its columns.  Events are emitted in (round, i, j) order.
extern "C" LSVD_API lsvd_status lsvd_schedule_from_rotors(const lsvd_rotor* rotors, int64_t count,
                                                          int64_t channels, int32_t target,
                                                          char* json, int64_t cap, int64_t* len) {
    if (count < 0 || channels < 0 || (count > 0 && !rotors) || (target != 0 && target != 1))
        return LSVD_BAD_ARGUMENT;
    std::vector<lsvd_rotor> rs(rotors, rotors + count);
    for (const auto& r : rs)
        if (r.i >= r.j || int64_t(r.j) >= channels) return LSVD_BAD_ARGUMENT;
    std::stable_sort(rs.begin(), rs.end(), [](const lsvd_rotor& a, const lsvd_rotor& b) {
        if (a.round != b.round) return a.round < b.round;
        if (a.i != b.i) return a.i < b.i;
        return a.j < b.j;
    });
    std::vector<Event> ev;
    ev.reserve(rs.size());
    for (const auto& r : rs)
        ev.push_back(Event{int64_t(r.round), int64_t(r.j), int64_t(r.i), 0.0, 0.0, -r.theta,
                           -r.theta, -r.theta, "gpu_jacobi", "jacobi_rotation"});
    std::vector<double> signs(static_cast<size_t>(channels), 1.0);
    return emit(to_json(target, channels, ev, signs), json, cap, len);
}

namespace {

bool phaseflow_ok(const lsvd_mzi_phase* events, int64_t count, int64_t channels, int32_t target) {
    if (count < 0 || channels < 0 || (count > 0 && !events) || (target != 0 && target != 1)) return false;
    for (int64_t k = 0; k < count; ++k)
        if (events[k].kind < 0 || events[k].kind >= kNumRealKinds || events[k].pass < 0 || events[k].i < 0 ||
            events[k].j < 0)
            return false;
    return true;
}

// Copies a finished frame (or reports its size): *len = bytes; cap too small
// writes nothing.
lsvd_status emit_frame(const std::vector<unsigned char>& f, void* out, int64_t cap, int64_t* len) {
    if (len) *len = int64_t(f.size());
    if (!out) return LSVD_OK;
    if (cap < int64_t(f.size())) return LSVD_ROTOR_OVERFLOW;
    std::memcpy(out, f.data(), f.size());
    return LSVD_OK;
}

std::vector<unsigned char> build_frame(int32_t target, uint32_t flags, int64_t channels,
                                       const std::vector<lsvd_schedule_record>& rec,
                                       const std::vector<double>& signs) {
    std::vector<unsigned char> f(size_t(lsvd::sched::frame_bytes(int64_t(rec.size()), int64_t(signs.size()), false)));
    const lsvd_schedule_header h =
        lsvd::sched::make_header(target, flags, channels, int64_t(rec.size()), int64_t(signs.size()));
    std::memcpy(f.data(), &h, sizeof(h));
    if (!rec.empty()) std::memcpy(f.data() + sizeof(h), rec.data(), rec.size() * sizeof(lsvd_schedule_record));
    if (!signs.empty())
        std::memcpy(f.data() + sizeof(h) + rec.size() * sizeof(lsvd_schedule_record), signs.data(),
                    signs.size() * 8);
    return f;
}

}  // namespace

// HardwareSchedule::from_real_phaseflow + to_json_string
// (src/lie_svd_compiler.rs:59-88, :213-265).
extern "C" LSVD_API lsvd_status lsvd_schedule_from_real_phaseflow(const lsvd_mzi_phase* events, int64_t count,
                                                                  int64_t channels, int32_t target, char* json,
                                                                  int64_t cap, int64_t* len) {
    if (!phaseflow_ok(events, count, channels, target)) return LSVD_BAD_ARGUMENT;
    std::vector<Event> ev;
    ev.reserve(size_t(count));
    for (int64_t k = 0; k < count; ++k) {
        const lsvd_mzi_phase& e = events[k];
        ev.push_back(Event{e.pass, e.i, e.j, 0.0, 0.0, 0.5 * (e.theta_l + e.theta_r), e.theta_l, e.theta_r,
                           kSources[LSVD_SCHED_SOURCE_REAL_PHASEFLOW], kKinds[e.kind]});
    }
    return emit(to_json(target, channels, ev, {}), json, cap, len);
}

extern "C" LSVD_API lsvd_status lsvd_schedule_binary_from_real_phaseflow(const lsvd_mzi_phase* events,
                                                                         int64_t count, int64_t channels,
                                                                         int32_t target, void* out, int64_t cap,
                                                                         int64_t* len) {
    if (!phaseflow_ok(events, count, channels, target)) return LSVD_BAD_ARGUMENT;
    std::vector<lsvd_schedule_record> rec(static_cast<size_t>(count));
    for (int64_t k = 0; k < count; ++k) {
        const lsvd_mzi_phase& e = events[k];
        if (e.pass > 0xffffffffLL || e.i > lsvd::sched::kMaxChannels || e.j > lsvd::sched::kMaxChannels)
            return LSVD_UNSUPPORTED;
        lsvd_schedule_record& r = rec[size_t(k)];
        std::memset(&r, 0, sizeof(r));
        r.layer = uint32_t(e.pass);
        r.i = uint16_t(e.i);
        r.j = uint16_t(e.j);
        r.theta = 0.5 * (e.theta_l + e.theta_r);
        r.theta_l = e.theta_l;
        r.theta_r = e.theta_r;
        r.source = uint8_t(LSVD_SCHED_SOURCE_REAL_PHASEFLOW);
        r.kind = uint8_t(e.kind);
    }
    return emit_frame(build_frame(target, 0u, channels, rec, {}), out, cap, len);
}

// Host half of lsvd_schedule_binary_from_rotors (the device half is in
// lsvd_schedule_dev.cu).
lsvd_status lsvd_schedule_binary_rotors_host(const lsvd_rotor* rotors, int64_t count, int64_t channels,
                                             int32_t target, void* out, int64_t cap, int64_t* len) {
    std::vector<lsvd_schedule_record> rec(static_cast<size_t>(count));
    for (int64_t k = 0; k < count; ++k) {
        if (!lsvd::sched::rotor_ok(rotors[k], channels)) return LSVD_BAD_ARGUMENT;
        rec[size_t(k)] = lsvd::sched::rotor_record(rotors[k]);
    }
    const std::vector<double> signs(size_t(channels), 1.0);
    return emit_frame(build_frame(target, LSVD_SCHED_CANONICAL, channels, rec, signs), out, cap, len);
}

extern "C" LSVD_API lsvd_status lsvd_schedule_binary_to_json(const void* frame, int64_t bytes, char* json,
                                                             int64_t cap, int64_t* len) {
    const int64_t hb = int64_t(sizeof(lsvd_schedule_header));
    if (!frame || bytes < hb) return LSVD_BAD_ARGUMENT;
    lsvd_schedule_header h;
    std::memcpy(&h, frame, sizeof(h));
    if (std::memcmp(h.magic, LSVD_SCHED_MAGIC, 8) != 0 || h.header_bytes != sizeof(lsvd_schedule_header) ||
        h.record_bytes != sizeof(lsvd_schedule_record) || h.target > 1 ||
        (h.flags & ~(LSVD_SCHED_CANONICAL | LSVD_SCHED_ENERGY)) != 0 || h.channels < 0 || h.total_events < 0 ||
        h.n_signs < 0 || h.total_events > bytes || h.n_signs > bytes)
        return LSVD_BAD_ARGUMENT;
    const bool energy = (h.flags & LSVD_SCHED_ENERGY) != 0;
    if (lsvd::sched::frame_bytes(h.total_events, h.n_signs, energy) != bytes) return LSVD_BAD_ARGUMENT;
    const unsigned char* base = static_cast<const unsigned char*>(frame);
    const unsigned char* rp = base + hb;
    const unsigned char* sp = rp + h.total_events * int64_t(sizeof(lsvd_schedule_record));
    const unsigned char* ep = sp + h.n_signs * 8;
    std::vector<Event> ev;
    ev.reserve(size_t(h.total_events));
    for (int64_t k = 0; k < h.total_events; ++k) {
        lsvd_schedule_record r;
        std::memcpy(&r, rp + k * int64_t(sizeof(r)), sizeof(r));
        if (r.source >= kNumSources || r.kind >= kNumKinds) return LSVD_BAD_ARGUMENT;
        Event e{int64_t(r.layer), int64_t(r.i), int64_t(r.j), r.phi_l, r.phi_r, r.theta, r.theta_l, r.theta_r,
                kSources[r.source], kKinds[r.kind]};
        if (energy) {
            double eb[2];
            std::memcpy(eb, ep + k * 16, 16);
            e.has_before = !std::isnan(eb[0]);
            e.has_after = !std::isnan(eb[1]);
            e.energy_before = eb[0];
            e.energy_after = eb[1];
        }
        ev.push_back(e);
    }
    if (h.flags & LSVD_SCHED_CANONICAL)
        std::stable_sort(ev.begin(), ev.end(), [](const Event& a, const Event& b) {
            if (a.layer != b.layer) return a.layer < b.layer;
            if (a.j != b.j) return a.j < b.j;
            return a.i < b.i;
        });
    std::vector<double> signs(size_t(h.n_signs));
    if (h.n_signs) std::memcpy(signs.data(), sp, size_t(h.n_signs) * 8);
    return emit(to_json(int(h.target), h.channels, ev, signs), json, cap, len);
}
