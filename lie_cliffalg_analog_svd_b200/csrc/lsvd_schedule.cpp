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

namespace {

struct Event {
    int64_t layer, i, j;
    double phi_l, phi_r, theta, theta_l, theta_r;
    const char* source;
    const char* kind;
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
               ", \"source\": \"" + e.source + "\", \"kind\": \"" + e.kind + "\"}";
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
