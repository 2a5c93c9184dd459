// lsvd_oracle.cpp -- CPU f64 restatement of the hot path of the Rust crate
// `lie_cliffalg_analog_svd` v0.44.0.
//
// TEST INFRASTRUCTURE ONLY: this is the oracle the CUDA library is checked
// against and the timed CPU baseline; the product never links or calls it.
//
// Each function names the Rust lines it follows.  The arithmetic is the
// reference's: same iteration formulas, thresholds, loop orders and caps, and
// the reference's `.dot` (ndarray 0.15.6 -> matrixmultiply 0.3.11) restated
// in its per-element order, sequential fused multiply-adds over k.  Pinned:
// the reference's printed rounding statistics and rotation counts for its
// RNG-free inputs are reproduced to every printed digit
// (tests/test_oracle_pinned.py).
#include "lsvd_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <atomic>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Mat {
    int64_t r = 0, c = 0;
    std::vector<double> a;
    Mat() = default;
    Mat(int64_t rr, int64_t cc) : r(rr), c(cc), a(size_t(rr * cc), 0.0) {}
    double& operator()(int64_t i, int64_t j) { return a[size_t(i * c + j)]; }
    double operator()(int64_t i, int64_t j) const { return a[size_t(i * c + j)]; }
    static Mat eye(int64_t n) {
        Mat m(n, n);
        for (int64_t i = 0; i < n; ++i) m(i, i) = 1.0;
        return m;
    }
    static Mat from(int64_t rr, int64_t cc, const double* p) {
        Mat m(rr, cc);
        std::memcpy(m.a.data(), p, sizeof(double) * size_t(rr * cc));
        return m;
    }
    Mat t() const {
        Mat m(c, r);
        for (int64_t i = 0; i < r; ++i)
            for (int64_t j = 0; j < c; ++j) m(j, i) = (*this)(i, j);
        return m;
    }
    void store(double* p) const { std::memcpy(p, a.data(), sizeof(double) * a.size()); }
};

// ndarray's `dot` (ndarray 0.15.6 over matrixmultiply 0.3.11, the versions
// of the reference's Cargo.lock): the dgemm micro-kernel accumulates every
// C(i, j) over k = 0, 1, ... in order from zero, then scales by alpha = 1
// (exact) -- with a fused multiply-add per k on hosts with FMA (the default
// here), with a multiply then an add on hosts without (oracle_set_dot_fma(0)).
// The products below keep that order and rounding, so rounding-level outputs
// (orthogonality, reconstruction residuals) reproduce the reference's printed
// ones on either kind of host.
bool g_dot_fma = true;

template <bool FMA>
void mm_rows(const Mat& A, const Mat& B, Mat& C, bool trans_a) {
    const int64_t kk = trans_a ? A.r : A.c, mi = trans_a ? A.c : A.r;
    for (int64_t i = 0; i < mi; ++i)
        for (int64_t k = 0; k < kk; ++k) {
            const double a = trans_a ? A(k, i) : A(i, k);
            const double* brow = &B.a[size_t(k * B.c)];
            double* crow = &C.a[size_t(i * C.c)];
            for (int64_t j = 0; j < B.c; ++j) {
                if (FMA)
                    crow[j] = std::fma(a, brow[j], crow[j]);
                else
                    crow[j] += a * brow[j];
            }
        }
}

// C = A * B
Mat matmul(const Mat& A, const Mat& B) {
    Mat C(A.r, B.c);
    if (g_dot_fma)
        mm_rows<true>(A, B, C, false);
    else
        mm_rows<false>(A, B, C, false);
    return C;
}
// C = A^T * B
Mat matmul_tn(const Mat& A, const Mat& B) {
    Mat C(A.c, B.c);
    if (g_dot_fma)
        mm_rows<true>(A, B, C, true);
    else
        mm_rows<false>(A, B, C, true);
    return C;
}

double frob(const Mat& m) {
    double s = 0.0;
    for (double x : m.a) s += x * x;
    return std::sqrt(s);
}

// ---------------------------------------------------------------- Small ----

// gram_schmidt_orthonormal, src/lie_svd_small.rs:82-144.  MGS on the columns;
// a column whose residual norm is < 1e-10 is replaced by the standard basis
// vector with the largest residual after projection (never a zero column).
Mat mgs_orthonormal(const Mat& a) {
    const int64_t n = a.r;
    Mat out(n, n);
    std::vector<double> v(static_cast<size_t>(n)), cand(static_cast<size_t>(n)), best(static_cast<size_t>(n));
    for (int64_t j = 0; j < n; ++j) {
        for (int64_t i = 0; i < n; ++i) v[size_t(i)] = a(i, j);
        for (int64_t k = 0; k < j; ++k) {
            double d = 0.0;
            for (int64_t i = 0; i < n; ++i) d += out(i, k) * v[size_t(i)];
            for (int64_t i = 0; i < n; ++i) v[size_t(i)] -= d * out(i, k);
        }
        double nrm = 0.0;
        for (double x : v) nrm += x * x;
        nrm = std::sqrt(nrm);
        if (nrm >= 1e-10) {
            for (double& x : v) x /= nrm;
        } else {
            double best_norm = -1.0;
            for (int64_t k = 0; k < n; ++k) {
                std::fill(cand.begin(), cand.end(), 0.0);
                cand[size_t(k)] = 1.0;
                for (int64_t col = 0; col < j; ++col) {
                    double d = 0.0;
                    for (int64_t i = 0; i < n; ++i) d += out(i, col) * cand[size_t(i)];
                    for (int64_t i = 0; i < n; ++i) cand[size_t(i)] -= d * out(i, col);
                }
                double en = 0.0;
                for (double x : cand) en += x * x;
                en = std::sqrt(en);
                if (en > best_norm) {
                    best_norm = en;
                    best = cand;
                }
            }
            if (best_norm > 0.0 && std::isfinite(best_norm)) {
                for (int64_t i = 0; i < n; ++i) v[size_t(i)] = best[size_t(i)] / best_norm;
            } else {
                std::fill(v.begin(), v.end(), 0.0);
                v[size_t(j)] = 1.0;
            }
        }
        for (int64_t i = 0; i < n; ++i) out(i, j) = v[size_t(i)];
    }
    return out;
}

// orthogonality_err, src/lie_svd_small.rs:146-150: ||Q^T Q - I||_F.
double orth_err(const Mat& q) {
    Mat g = matmul_tn(q, q);
    double s = 0.0;
    for (int64_t i = 0; i < g.r; ++i)
        for (int64_t j = 0; j < g.c; ++j) {
            const double d = g(i, j) - (i == j ? 1.0 : 0.0);
            s += d * d;
        }
    return std::sqrt(s);
}

// Constants of src/lie_svd_small.rs:67-69.
constexpr int kPolarMaxIters = 120;
constexpr double kPolarTol = 1e-13;
constexpr double kJacobiTol = 1e-13;

// newton_schulz_polar, src/lie_svd_small.rs:158-183.
//   X0 = A / max(||A||_F, 1e-300);  X+ = 0.5 X (3I - X^T X);  delta = ||X+ - X||_F
//   non-finite or delta > 1e6 sqrt(n) -> (MGS(A), false)
//   delta < 1e-13 sqrt(n)             -> (X, ||X^T X - I|| <= 1e-8 sqrt(n))
//   cap 120 iterations                -> (X, same orthogonality test)
Mat ns_polar(const Mat& a, bool* ok, int* iters) {
    const int64_t n = a.r;
    const double scale = std::max(frob(a), 1e-300);
    Mat x(n, n);
    for (size_t i = 0; i < x.a.size(); ++i) x.a[i] = a.a[i] / scale;
    const double ref = std::sqrt(double(n));
    *iters = 0;
    for (int it = 0; it < kPolarMaxIters; ++it) {
        *iters = it + 1;
        Mat xtx = matmul_tn(x, x);
        Mat m(n, n);  // 3I - X^T X
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < n; ++j) m(i, j) = (i == j ? 3.0 : 0.0) - xtx(i, j);
        Mat xn = matmul(x, m);
        bool finite = true;
        double dsq = 0.0;
        for (size_t i = 0; i < xn.a.size(); ++i) {
            xn.a[i] *= 0.5;
            if (!std::isfinite(xn.a[i])) finite = false;
            const double d = xn.a[i] - x.a[i];
            dsq += d * d;
        }
        const double delta = std::sqrt(dsq);
        if (!finite || delta > 1e6 * ref) {
            *ok = false;
            return mgs_orthonormal(a);
        }
        x = std::move(xn);
        if (delta < kPolarTol * ref) {
            *ok = orth_err(x) <= 1e-8 * ref;
            return x;
        }
    }
    *ok = orth_err(x) <= 1e-8 * ref;
    return x;
}

// repair_left_basis_from_right, src/lie_svd_small.rs:185-208.
Mat repair_left(const Mat& mat, const Mat& v, const std::vector<double>& sigma) {
    const int64_t n = mat.r;
    double smax = 0.0;
    for (double s : sigma) smax = std::max(smax, s);
    const double stol = 1e-12 * std::max(smax, 1.0);
    Mat seed(n, n);
    for (int64_t j = 0; j < n; ++j) {
        if (sigma[size_t(j)] > stol) {
            for (int64_t row = 0; row < n; ++row) {
                double s = 0.0;
                for (int64_t k = 0; k < n; ++k) s += mat(row, k) * v(k, j);
                seed(row, j) = s / sigma[size_t(j)];
            }
        }
    }
    return mgs_orthonormal(seed);
}

// eigh_jacobi_full, src/lie_svd_small.rs:212-285: classical cyclic (row order
// p<q) two-sided Jacobi with the Rutishauser tangent, off-norm test at sweep
// start, cap 60+20n sweeps, skip |a_pq| < 1e-300, stable descending sort.
void eigh_jacobi(const Mat& p, Mat& vs, std::vector<double>& eig, int* sweeps_out,
                 int64_t* rot_out) {
    const int64_t n = p.r;
    Mat a = p;
    Mat v = Mat::eye(n);
    const int64_t max_sweeps = 60 + 20 * n;
    const double ref = std::max(frob(p), 1e-300);
    int sweeps = 0;
    int64_t rots = 0;
    for (int64_t sw = 0; sw < max_sweeps; ++sw) {
        sweeps = int(sw + 1);
        double off = 0.0;
        for (int64_t pp = 0; pp < n; ++pp)
            for (int64_t qq = pp + 1; qq < n; ++qq) off += a(pp, qq) * a(pp, qq);
        if (std::sqrt(off) < kJacobiTol * ref) break;
        for (int64_t pp = 0; pp < n; ++pp) {
            for (int64_t qq = pp + 1; qq < n; ++qq) {
                const double apq = a(pp, qq);
                if (std::fabs(apq) < 1e-300) continue;
                const double theta = (a(qq, qq) - a(pp, pp)) / (2.0 * apq);
                const double t = theta >= 0.0 ? 1.0 / (theta + std::sqrt(theta * theta + 1.0))
                                               : -1.0 / (-theta + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0);
                const double s = t * c;
                const double app = a(pp, pp), aqq = a(qq, qq);
                a(pp, pp) = app - t * apq;
                a(qq, qq) = aqq + t * apq;
                a(pp, qq) = 0.0;
                a(qq, pp) = 0.0;
                for (int64_t i = 0; i < n; ++i) {
                    if (i != pp && i != qq) {
                        const double aip = a(i, pp), aiq = a(i, qq);
                        a(i, pp) = c * aip - s * aiq;
                        a(pp, i) = a(i, pp);
                        a(i, qq) = s * aip + c * aiq;
                        a(qq, i) = a(i, qq);
                    }
                }
                for (int64_t i = 0; i < n; ++i) {
                    const double vip = v(i, pp), viq = v(i, qq);
                    v(i, pp) = c * vip - s * viq;
                    v(i, qq) = s * vip + c * viq;
                }
                ++rots;
            }
        }
    }
    std::vector<int64_t> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), 0);
    // Rust's sort_by is stable; NaN compares as Equal (partial_cmp -> None).
    std::stable_sort(order.begin(), order.end(), [&](int64_t i, int64_t j) {
        return a(j, j) < a(i, i);
    });
    vs = Mat(n, n);
    eig.assign(size_t(n), 0.0);
    for (int64_t nj = 0; nj < n; ++nj) {
        const int64_t oj = order[size_t(nj)];
        eig[size_t(nj)] = a(oj, oj);
        for (int64_t i = 0; i < n; ++i) vs(i, nj) = v(i, oj);
    }
    if (sweeps_out) *sweeps_out = sweeps;
    if (rot_out) *rot_out = rots;
}

// LieSvdSmall::solve, src/lie_svd_small.rs:296-323.
void small_solve(const Mat& mat, Mat& u, std::vector<double>& sigma, Mat& vt,
                 oracle_small_info* info) {
    const int64_t n = mat.r;
    bool ok = false;
    int iters = 0;
    Mat q = ns_polar(mat, &ok, &iters);
    Mat p = matmul_tn(q, mat);
    Mat ps(n, n);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = 0; j < n; ++j) ps(i, j) = (p(i, j) + p(j, i)) * 0.5;
    Mat v;
    std::vector<double> eig;
    int sweeps = 0;
    int64_t rots = 0;
    eigh_jacobi(ps, v, eig, &sweeps, &rots);
    sigma.assign(size_t(n), 0.0);
    for (int64_t j = 0; j < n; ++j) sigma[size_t(j)] = std::max(eig[size_t(j)], 0.0);
    u = matmul(q, v);
    bool repaired = false;
    if (!ok || orth_err(u) > 1e-8 * std::sqrt(double(n))) {
        u = repair_left(mat, v, sigma);
        repaired = true;
    }
    vt = v.t();
    if (info) {
        info->ns_iters = iters;
        info->polar_ok = ok ? 1 : 0;
        info->jacobi_sweeps = sweeps;
        info->jacobi_rotations = rots;
        info->repaired = repaired ? 1 : 0;
        info->micro_fallback = 0;
    }
}

// qr_reduce, src/lie_svd_small.rs:373-418: MGS QR; a column whose residual is
// below 1e-10 ||X||_F keeps a zero Q column and R[j,j] = residual norm.
void qr_reduce(const Mat& mat, Mat& q, Mat& r) {
    const int64_t n = mat.r, d = mat.c;
    q = Mat(n, d);
    r = Mat(d, d);
    Mat v(n, d);
    const double scale = std::max(frob(mat), 1e-300);
    const double floor_ = 1e-10 * scale;
    for (int64_t j = 0; j < d; ++j) {
        for (int64_t i = 0; i < n; ++i) v(i, j) = mat(i, j);
        for (int64_t k = 0; k < j; ++k) {
            double dot = 0.0;
            for (int64_t i = 0; i < n; ++i) dot += q(i, k) * v(i, j);
            r(k, j) = dot;
            for (int64_t i = 0; i < n; ++i) v(i, j) -= dot * q(i, k);
        }
        double nrm = 0.0;
        for (int64_t i = 0; i < n; ++i) nrm += v(i, j) * v(i, j);
        nrm = std::sqrt(nrm);
        r(j, j) = nrm;
        if (nrm >= floor_)
            for (int64_t i = 0; i < n; ++i) q(i, j) = v(i, j) / nrm;
    }
}

// LieSvdSmall::solve_rectangular, src/lie_svd_small.rs:340-360.
void small_solve_rect(const Mat& mat, Mat& u, std::vector<double>& s, Mat& vt) {
    const int64_t n = mat.r, d = mat.c;
    if (n == d) {
        small_solve(mat, u, s, vt, nullptr);
        return;
    }
    if (d > n) {
        Mat ut, vtt;
        small_solve_rect(mat.t(), ut, s, vtt);
        u = vtt.t();
        vt = ut.t();
        return;
    }
    Mat q, r;
    qr_reduce(mat, q, r);
    Mat ur;
    small_solve(r, ur, s, vt, nullptr);
    u = matmul(q, ur);
}

// ---------------------------------------------------------------- Micro ----
// src/lie_svd_micro.rs

constexpr double kMicroTol = 1e-13;  // :15

double offdiag_norm(const Mat& a) {  // :101-112
    double s = 0.0;
    for (int64_t i = 0; i < a.r; ++i)
        for (int64_t j = 0; j < a.c; ++j)
            if (i != j) s += a(i, j) * a(i, j);
    return std::sqrt(s);
}

double wrap_half_pi(double ang) {  // :118-126 and src/lie_svd_joint.rs:293-301
    while (ang > M_PI_2) ang -= M_PI;
    while (ang < -M_PI_2) ang += M_PI;
    return ang;
}

// local_pair_svd_angles, :128-139 (and local_pair_svd_angles_from_values,
// src/lie_svd_joint.rs:284-291).
void pair_svd_angles(double a, double b, double c, double d, double* tl, double* tr) {
    const double sum = std::atan2(-(b + c), a - d);
    const double diff = std::atan2(b - c, a + d);
    *tl = wrap_half_pi(0.5 * (sum + diff));
    *tr = wrap_half_pi(0.5 * (sum - diff));
}

// apply_left_rotor (rows i,j), src/lie_svd_micro.rs:141-162 / joint.rs:406-415.
void rot_rows(Mat& w, int64_t i, int64_t j, double th) {
    const double s = std::sin(th), c = std::cos(th);
    for (int64_t col = 0; col < w.c; ++col) {
        const double ai = w(i, col), aj = w(j, col);
        w(i, col) = c * ai - s * aj;
        w(j, col) = s * ai + c * aj;
    }
}
// apply_right_rotor / apply_basis_rotor (columns i,j), micro.rs:164-185,
// joint.rs:417-437.
void rot_cols(Mat& w, int64_t i, int64_t j, double th) {
    const double s = std::sin(th), c = std::cos(th);
    for (int64_t row = 0; row < w.r; ++row) {
        const double ai = w(row, i), aj = w(row, j);
        w(row, i) = c * ai - s * aj;
        w(row, j) = s * ai + c * aj;
    }
}

// solve_fixed_schedule + extract_sorted_svd, src/lie_svd_micro.rs:55-95,187-214.
void micro_fixed(const Mat& mat, const int (*pairs)[2], int npairs, int max_sweeps, Mat& u,
                 std::vector<double>& sigma, Mat& vt, oracle_small_info* info) {
    const int64_t n = mat.r;
    Mat work = mat;
    Mat ub = Mat::eye(n), vb = Mat::eye(n);
    const double ref = std::max(frob(mat), 1e-300);
    const double tol = kMicroTol * std::max(ref, 1.0);
    int sweeps = 0;
    int64_t rots = 0;
    for (int sw = 0; sw < std::max(max_sweeps, 1); ++sw) {
        const double e = offdiag_norm(work);
        if (e <= tol || !std::isfinite(e)) break;
        sweeps = sw + 1;
        bool changed = false;
        for (int k = 0; k < npairs; ++k) {
            const int i = pairs[k][0], j = pairs[k][1];
            if (std::fabs(work(i, j)) + std::fabs(work(j, i)) <= tol) continue;
            double tl, tr;
            pair_svd_angles(work(i, i), work(i, j), work(j, i), work(j, j), &tl, &tr);
            if (std::fabs(tl) + std::fabs(tr) <= 1e-18) continue;
            rot_rows(work, i, j, tl);
            rot_cols(ub, i, j, tl);
            rot_cols(work, i, j, tr);
            rot_cols(vb, i, j, tr);
            changed = true;
            ++rots;
        }
        if (!changed) break;
    }
    if (offdiag_norm(work) > 1e-10 * std::max(ref, 1.0)) {
        small_solve(mat, u, sigma, vt, info);
        if (info) info->micro_fallback = 1;
        return;
    }
    std::vector<int64_t> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
        return std::fabs(work(b, b)) < std::fabs(work(a, a));
    });
    u = Mat(n, n);
    Mat vs(n, n);
    sigma.assign(size_t(n), 0.0);
    for (int64_t dst = 0; dst < n; ++dst) {
        const int64_t src = order[size_t(dst)];
        const double d = work(src, src);
        sigma[size_t(dst)] = std::fabs(d);
        const double sg = d < 0.0 ? -1.0 : 1.0;
        for (int64_t r = 0; r < n; ++r) {
            u(r, dst) = sg * ub(r, src);
            vs(r, dst) = vb(r, src);
        }
    }
    vt = vs.t();
    if (info) {
        info->ns_iters = 0;
        info->polar_ok = 1;
        info->jacobi_sweeps = sweeps;
        info->jacobi_rotations = rots;
        info->repaired = 0;
        info->micro_fallback = 0;
    }
}

// LieSvdMicro::solve, src/lie_svd_micro.rs:21-52.
void micro_solve(const Mat& mat, Mat& u, std::vector<double>& s, Mat& vt,
                 oracle_small_info* info) {
    const int64_t n = mat.r;
    if (info) std::memset(info, 0, sizeof(*info));
    if (n == 0) {
        u = Mat(0, 0);
        vt = Mat(0, 0);
        s.clear();
        return;
    }
    if (n == 1) {
        const double d = mat(0, 0);
        u = Mat(1, 1);
        u(0, 0) = d < 0.0 ? -1.0 : 1.0;
        s.assign(1, std::fabs(d));
        vt = Mat::eye(1);
        if (info) info->polar_ok = 1;
        return;
    }
    static const int p2[][2] = {{0, 1}};
    static const int p3[][2] = {{0, 1}, {0, 2}, {1, 2}};
    static const int p4[][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {0, 3}, {1, 2}};
    if (n == 2) micro_fixed(mat, p2, 1, 1, u, s, vt, info);
    if (n == 3) micro_fixed(mat, p3, 3, 24, u, s, vt, info);
    if (n == 4) micro_fixed(mat, p4, 6, 24, u, s, vt, info);
}

// ---------------------------------------------------------------- Joint ----
// src/lie_svd_joint.rs

double joint_offdiag_norm(const std::vector<Mat>& w) {  // :439-441, offdiag_sq :461-473
    double s = 0.0;
    for (const Mat& m : w)
        for (int64_t i = 0; i < m.r; ++i)
            for (int64_t j = 0; j < m.c; ++j)
                if (i != j) s += m(i, j) * m(i, j);
    return std::sqrt(s);
}
double joint_frob(const std::vector<Mat>& w) {  // :443-449
    double s = 0.0;
    for (const Mat& m : w)
        for (double x : m.a) s += x * x;
    return std::sqrt(s);
}
double joint_pair_offdiag(const std::vector<Mat>& w, int64_t i, int64_t j) {  // :451-453
    double s = 0.0;
    for (const Mat& m : w) s += std::fabs(m(i, j)) + std::fabs(m(j, i));
    return s;
}
double local_offdiag_sq(const Mat& m, int64_t i, int64_t j) {  // :475-494
    double s = 0.0;
    for (int64_t col = 0; col < m.c; ++col) {
        if (col != i) s += m(i, col) * m(i, col);
        if (col != j) s += m(j, col) * m(j, col);
    }
    for (int64_t row = 0; row < m.r; ++row) {
        if (row != i && row != j) {
            s += m(row, i) * m(row, i);
            s += m(row, j) * m(row, j);
        }
    }
    return s;
}
double joint_local(const std::vector<Mat>& w, int64_t i, int64_t j) {  // :455-459
    double s = 0.0;
    for (const Mat& m : w) s += local_offdiag_sq(m, i, j);
    return s;
}
double wrap_quarter_pi(double ang) {  // wrap_jacobi_angle :506-514
    while (ang > M_PI_4) ang -= M_PI_2;
    while (ang < -M_PI_4) ang += M_PI_2;
    return ang;
}
int64_t rr_layer_count(int64_t n) { return n % 2 == 0 ? std::max<int64_t>(n - 1, 0) : n; }  // :516-522
// layer_pairs :524-539 -- circle-method round robin with a dummy for odd n.
std::vector<std::pair<int64_t, int64_t>> layer_pairs(int64_t n, int64_t layer) {
    const int64_t m = n % 2 == 0 ? n : n + 1;
    const int64_t ring = m - 1;
    std::vector<std::pair<int64_t, int64_t>> out;
    for (int64_t k = 0; k < m / 2; ++k) {
        int64_t a, b;
        if (k == 0) {
            a = m - 1;
            b = layer % ring;
        } else {
            a = (layer + k) % ring;
            b = (layer + ring - k) % ring;
        }
        if (a < n && b < n) out.push_back(a < b ? std::make_pair(a, b) : std::make_pair(b, a));
    }
    return out;
}
double pair_energy_after(const std::vector<Mat>& w, int64_t i, int64_t j, double th) {  // :388-399
    const double s = std::sin(th), c = std::cos(th);
    double out = 0.0;
    for (const Mat& m : w) {
        const double a = m(i, i), b = 0.5 * (m(i, j) + m(j, i)), d = m(j, j);
        const double off = 0.5 * (a - d) * (2.0 * s * c) + b * (c * c - s * s);
        out += 2.0 * off * off;
    }
    return out;
}
double sym_pair_angle(const std::vector<Mat>& w, int64_t i, int64_t j) {  // :338-357
    double sxx = 0.0, syy = 0.0, sxy = 0.0;
    for (const Mat& m : w) {
        const double x = 0.5 * (m(i, i) - m(j, j));
        const double y = 0.5 * (m(i, j) + m(j, i));
        sxx += x * x;
        syy += y * y;
        sxy += x * y;
    }
    double th = 0.25 * std::atan2(2.0 * sxy, syy - sxx);
    const double alt = wrap_quarter_pi(th + M_PI_4);
    th = wrap_quarter_pi(th);
    return pair_energy_after(w, i, j, alt) < pair_energy_after(w, i, j, th) ? alt : th;
}
void sym_rotor(Mat& m, int64_t i, int64_t j, double th) {  // apply_symmetric_rotor :401-404
    rot_rows(m, i, j, th);
    rot_cols(m, i, j, th);
}
bool accept_sym(std::vector<Mat>& w, Mat& basis, int64_t i, int64_t j, double theta,
                int steps) {  // accept_joint_rotor :359-386
    const double before = joint_local(w, i, j);
    const double slack = 1e-14 * std::max(before, 1.0);
    double scale = 1.0;
    for (int it = 0; it < std::max(steps, 1); ++it) {
        const double ang = theta * scale;
        for (Mat& m : w) sym_rotor(m, i, j, ang);
        const double after = joint_local(w, i, j);
        if (after <= before + slack && std::isfinite(after)) {
            rot_cols(basis, i, j, ang);
            return true;
        }
        for (Mat& m : w) sym_rotor(m, i, j, -ang);
        scale *= 0.5;
    }
    return false;
}

// diagonalize_symmetric_with_params, :71-158.
void jade_sym(std::vector<Mat>& work, const oracle_joint_params& p, Mat& basis,
              oracle_joint_trace* tr) {
    const int64_t n = work[0].r;
    basis = Mat::eye(n);
    std::memset(tr, 0, sizeof(*tr));
    if (n <= 1) return;
    const double ref = std::max(joint_frob(work), 1e-300);
    const double pair_tol = p.min_pair_scale * std::max(ref, 1.0);
    const double tol = p.tol * std::max(ref, 1.0);
    tr->initial_offdiag = joint_offdiag_norm(work);
    for (int64_t sw = 0; sw < p.max_sweeps; ++sw) {
        tr->sweeps = sw + 1;
        const double before = joint_offdiag_norm(work);
        for (int64_t layer = 0; layer < rr_layer_count(n); ++layer) {
            for (auto [i, j] : layer_pairs(n, layer)) {
                if (joint_pair_offdiag(work, i, j) <= pair_tol) continue;
                const double th = sym_pair_angle(work, i, j);
                if (std::fabs(th) <= 1e-18) continue;
                if (accept_sym(work, basis, i, j, th, p.line_search_steps))
                    tr->rotations++;
                else
                    tr->rejected_rotations++;
            }
        }
        const double after = joint_offdiag_norm(work);
        if (after <= tol || after >= before * (1.0 - 1e-10)) break;
    }
    tr->final_offdiag = joint_offdiag_norm(work);
}

// joint_svd_pair_angles :264-277 with pair_block_norm :279-282.
void joint_svd_angles(const std::vector<Mat>& w, int64_t i, int64_t j, double* tl, double* trr) {
    double a = 0, b = 0, c = 0, d = 0;
    for (const Mat& m : w) {
        const double wt = std::max(std::sqrt(m(i, i) * m(i, i) + m(i, j) * m(i, j) +
                                             m(j, i) * m(j, i) + m(j, j) * m(j, j)),
                                   1e-300);
        a += m(i, i) / wt;
        b += m(i, j) / wt;
        c += m(j, i) / wt;
        d += m(j, j) / wt;
    }
    pair_svd_angles(a, b, c, d, tl, trr);
}
bool accept_svd(std::vector<Mat>& w, Mat& ub, Mat& vb, int64_t i, int64_t j, double tl,
                double trr, int steps) {  // accept_joint_svd_rotor :303-336
    const double before = joint_local(w, i, j);
    const double slack = 1e-14 * std::max(before, 1.0);
    double scale = 1.0;
    for (int it = 0; it < std::max(steps, 1); ++it) {
        const double a = tl * scale, b = trr * scale;
        for (Mat& m : w) {
            rot_rows(m, i, j, a);
            rot_cols(m, i, j, b);
        }
        const double after = joint_local(w, i, j);
        if (after <= before + slack && std::isfinite(after)) {
            rot_cols(ub, i, j, a);
            rot_cols(vb, i, j, b);
            return true;
        }
        for (Mat& m : w) {
            rot_cols(m, i, j, -b);
            rot_rows(m, i, j, -a);
        }
        scale *= 0.5;
    }
    return false;
}

}  // namespace

// ================================================================ C ABI ====

extern "C" {

int oracle_small_solve(int64_t n, const double* A, double* U, double* S, double* Vt,
                       oracle_small_info* info) {
    if (n <= 0 || !A || !U || !S || !Vt) return -1;
    Mat a = Mat::from(n, n, A), u, vt;
    std::vector<double> s;
    small_solve(a, u, s, vt, info);
    u.store(U);
    vt.store(Vt);
    std::memcpy(S, s.data(), sizeof(double) * size_t(n));
    return 0;
}

int oracle_ns_polar(int64_t n, const double* A, double* Q, int32_t* ok, int32_t* iters) {
    if (n <= 0 || !A || !Q) return -1;
    bool o = false;
    int it = 0;
    Mat q = ns_polar(Mat::from(n, n, A), &o, &it);
    q.store(Q);
    if (ok) *ok = o ? 1 : 0;
    if (iters) *iters = it;
    return 0;
}

int oracle_eigh_jacobi(int64_t n, const double* P, double* V, double* eig, int32_t* sweeps,
                       int64_t* rotations) {
    if (n <= 0 || !P || !V || !eig) return -1;
    Mat v;
    std::vector<double> e;
    int sw = 0;
    eigh_jacobi(Mat::from(n, n, P), v, e, &sw, rotations);
    v.store(V);
    std::memcpy(eig, e.data(), sizeof(double) * size_t(n));
    if (sweeps) *sweeps = sw;
    return 0;
}

int oracle_small_solve_rectangular(int64_t m, int64_t d, const double* A, double* U, double* S,
                                   double* Vt) {
    if (m <= 0 || d <= 0 || !A) return -1;  // src/lie_svd_small.rs:343-346
    Mat u, vt;
    std::vector<double> s;
    small_solve_rect(Mat::from(m, d, A), u, s, vt);
    u.store(U);
    vt.store(Vt);
    std::memcpy(S, s.data(), sizeof(double) * s.size());
    return 0;
}

int oracle_qr_reduce(int64_t m, int64_t d, const double* A, double* Q, double* R) {
    if (m <= 0 || d <= 0 || m < d) return -1;
    Mat q, r;
    qr_reduce(Mat::from(m, d, A), q, r);
    q.store(Q);
    r.store(R);
    return 0;
}

int oracle_micro_solve(int64_t n, const double* A, double* U, double* S, double* Vt,
                       oracle_small_info* info) {
    if (n < 0 || n > 4) return -1;  // src/lie_svd_micro.rs:23-24
    Mat u, vt;
    std::vector<double> s;
    micro_solve(n == 0 ? Mat(0, 0) : Mat::from(n, n, A), u, s, vt, info);
    if (n > 0) {
        u.store(U);
        vt.store(Vt);
        std::memcpy(S, s.data(), sizeof(double) * size_t(n));
    }
    return 0;
}

oracle_joint_params oracle_joint_params_for_n(int64_t n) {
    oracle_joint_params p;
    p.max_sweeps = int32_t(12 + std::max<int64_t>(n, 1));
    p.tol = 1e-12;
    p.min_pair_scale = 1e-14;
    p.line_search_steps = 6;
    return p;
}

int oracle_jade_sym(int64_t K, int64_t n, const double* M, oracle_joint_params params, double* V,
                    double* diag, oracle_joint_trace* trace) {
    if (K <= 0 || n < 0 || !M) return -1;  // :75-85
    std::vector<Mat> work;
    for (int64_t k = 0; k < K; ++k) work.push_back(Mat::from(n, n, M + size_t(k * n * n)));
    Mat basis;
    oracle_joint_trace tr;
    jade_sym(work, params, basis, &tr);
    if (V) basis.store(V);
    if (diag)
        for (int64_t k = 0; k < K; ++k)
            for (int64_t i = 0; i < n; ++i) diag[size_t(k * n + i)] = work[size_t(k)](i, i);
    if (trace) *trace = tr;
    return 0;
}

int oracle_joint_svd(int64_t K, int64_t rows, int64_t cols, const double* M,
                     oracle_joint_params params, double* U, double* sig, double* Vt,
                     oracle_joint_trace* trace) {
    if (K <= 0 || rows <= 0 || cols <= 0 || !M) return -1;  // :174-181
    std::vector<Mat> work;
    for (int64_t k = 0; k < K; ++k)
        work.push_back(Mat::from(rows, cols, M + size_t(k * rows * cols)));
    const int64_t kk = std::min(rows, cols);
    Mat ub = Mat::eye(rows), vb = Mat::eye(cols);
    oracle_joint_trace tr;
    std::memset(&tr, 0, sizeof(tr));
    if (kk > 1) {
        const double ref = std::max(joint_frob(work), 1e-300);
        const double pair_tol = params.min_pair_scale * std::max(ref, 1.0);
        const double tol = params.tol * std::max(ref, 1.0);
        tr.initial_offdiag = joint_offdiag_norm(work);
        for (int64_t sw = 0; sw < params.max_sweeps; ++sw) {
            tr.sweeps = sw + 1;
            const double before = joint_offdiag_norm(work);
            for (int64_t layer = 0; layer < rr_layer_count(kk); ++layer) {
                for (auto [i, j] : layer_pairs(kk, layer)) {
                    if (joint_pair_offdiag(work, i, j) <= pair_tol) continue;
                    double tl, trr;
                    joint_svd_angles(work, i, j, &tl, &trr);
                    if (std::fabs(tl) + std::fabs(trr) <= 1e-18) continue;
                    if (accept_svd(work, ub, vb, i, j, tl, trr, params.line_search_steps))
                        tr.rotations++;
                    else
                        tr.rejected_rotations++;
                }
            }
            const double after = joint_offdiag_norm(work);
            if (after <= tol || after >= before * (1.0 - 1e-10)) break;
        }
        tr.final_offdiag = joint_offdiag_norm(work);
    }
    if (U) ub.store(U);
    if (Vt) vb.t().store(Vt);
    if (sig)  // diagonal_corridor :501-504
        for (int64_t k = 0; k < K; ++k)
            for (int64_t i = 0; i < kk; ++i)
                sig[size_t(k * kk + i)] = std::fabs(work[size_t(k)](i, i));
    if (trace) *trace = tr;
    return 0;
}

// metrics::compute, src/lib.rs:149-194.  Written for the general thin shape
// (U m*k, Vt k*d); on square input it is the reference formula exactly.
int oracle_metrics(int64_t m, int64_t d, int64_t k, const double* A, const double* U,
                   const double* S, const double* Vt, const double* sigma_ref, double* out) {
    if (m <= 0 || d <= 0 || k <= 0 || !out) return -1;
    Mat a = Mat::from(m, d, A), u = Mat::from(m, k, U), vt = Mat::from(k, d, Vt);
    Mat us = u;
    for (int64_t i = 0; i < m; ++i)
        for (int64_t j = 0; j < k; ++j) us(i, j) *= S[j];
    Mat rec = matmul(us, vt);
    double num = 0.0;
    for (size_t i = 0; i < rec.a.size(); ++i) {
        const double dd = rec.a[i] - a.a[i];
        num += dd * dd;
    }
    out[0] = std::sqrt(num) / std::max(frob(a), 1e-300);
    out[1] = orth_err(u);
    out[2] = orth_err(vt.t());
    if (sigma_ref) {
        std::vector<double> got(S, S + k), want(sigma_ref, sigma_ref + k);
        auto desc = [](double x, double y) { return y < x; };
        std::stable_sort(got.begin(), got.end(), desc);
        std::stable_sort(want.begin(), want.end(), desc);
        double mx = 0.0, tail = 0.0;
        const int64_t tail_start = (k * 3) / 4;
        for (int64_t i = 0; i < k; ++i) {
            const double r = std::fabs(got[size_t(i)] - want[size_t(i)]) /
                             std::max(std::fabs(want[size_t(i)]), 1e-300);
            mx = std::max(mx, r);  // f64::max ignores NaN like fold(0, max)
            if (i >= tail_start) tail = std::max(tail, r);
        }
        out[3] = mx;
        out[4] = tail;
    } else {
        out[3] = NAN;
        out[4] = NAN;
    }
    return 0;
}

// HardwareSchedule::from_orthogonal_matrix, src/lie_svd_compiler.rs:144-198.
int64_t oracle_schedule_from_orthogonal(int64_t d, const double* V, int64_t cap, int64_t* ev_i,
                                        int64_t* ev_j, double* ev_theta, double* signs) {
    if (d < 0 || (d > 0 && !V)) return -1;
    Mat r = d ? Mat::from(d, d, V) : Mat(0, 0);
    int64_t count = 0;
    for (int64_t j = 0; j < d; ++j) {
        for (int64_t i = j + 1; i < d; ++i) {
            const double a = r(j, j), b = r(i, j);
            if (std::fabs(b) <= 1e-300) continue;
            const double nrm = std::sqrt(a * a + b * b);
            const double c = a / nrm, s = b / nrm;
            for (int64_t k = 0; k < d; ++k) {
                const double rj = r(j, k), ri = r(i, k);
                r(j, k) = c * rj + s * ri;
                r(i, k) = -s * rj + c * ri;
            }
            if (count < cap) {
                ev_i[count] = i;
                ev_j[count] = j;
                ev_theta[count] = std::atan2(s, c);
            }
            ++count;
        }
    }
    if (signs)
        for (int64_t k = 0; k < d; ++k) {
            const double x = r(k, k);  // f64::signum: +-1 by sign bit, NaN stays NaN
            signs[k] = std::isnan(x) ? NAN : (std::signbit(x) ? -1.0 : 1.0);
        }
    return count;
}

// Rust `{:.17e}`: 17 fractional digits, exponent without '+' or zero padding.
void oracle_set_dot_fma(int32_t on) { g_dot_fma = on != 0; }

// ndarray `a.dot(&b)` of row-major m x k and k x n operands (the product
// order of matmul above); used to rebuild inputs the reference constructs
// with dot products.
int oracle_dot(int64_t m, int64_t k, int64_t n, const double* A, const double* B, double* C) {
    if (m < 0 || k < 0 || n < 0 || (m * k > 0 && !A) || (k * n > 0 && !B) || (m * n > 0 && !C)) return -1;
    matmul(Mat::from(m, k, A), Mat::from(k, n, B)).store(C);
    return 0;
}

// One lagged covariance of Phase-BSS (src/lie_svd_bss.rs:172-190): for t
// ascending, then i, then j, C[i][j] += x[i][t + lag] * x[j][t] / (T - lag),
// each product divided before it is added; then C <- (C + C^T) / 2
// (src/lie_svd_bss.rs:187, ndarray's 0.5 * (&c + &c.t())).
int oracle_lagged_covariance(int64_t ch, int64_t samples, const double* x, int64_t lag, double* out) {
    if (ch < 1 || samples < 2 || lag < 1 || lag >= samples || !x || !out) return -1;
    const double denom = double(samples - lag);
    std::vector<double> c(size_t(ch * ch), 0.0);
    for (int64_t t = 0; t < samples - lag; ++t)
        for (int64_t i = 0; i < ch; ++i) {
            const double xi = x[i * samples + t + lag];
            double* ci = c.data() + i * ch;
            for (int64_t j = 0; j < ch; ++j) ci[j] += xi * x[j * samples + t] / denom;
        }
    for (int64_t i = 0; i < ch; ++i)
        for (int64_t j = 0; j < ch; ++j) out[i * ch + j] = 0.5 * (c[size_t(i * ch + j)] + c[size_t(j * ch + i)]);
    return 0;
}

int oracle_fmt_e17(double x, char* buf, int64_t cap) {
    char tmp[64];
    std::string s;
    if (std::isnan(x)) {
        s = "NaN";
    } else if (std::isinf(x)) {
        s = x < 0 ? "-inf" : "inf";
    } else {
        std::snprintf(tmp, sizeof(tmp), "%.17e", x);
        std::string t(tmp);
        const size_t e = t.find('e');
        std::string mant = t.substr(0, e);
        int ex = std::atoi(t.c_str() + e + 1);
        s = mant + "e" + std::to_string(ex);
    }
    if (cap > 0) {
        std::snprintf(buf, size_t(cap), "%s", s.c_str());
    }
    return int(s.size());
}

// Batch driver of the timed CPU baseline (no reference counterpart: the
// reference solves one matrix per call).  Matrices idx[0..count) of a packed
// uneven batch -- matrix t is n[t] x n[t] at element offset aoff[t], its
// singular values at soff[t] -- are solved by `threads` std::threads pulling
// positions from one atomic counter, each with the route of LieSvd::solve's
// exact tiers (LieSvdMicro for n <= 4, src/lie_svd_adaptive.rs:105-106,
// LieSvdSmall otherwise).  Outputs land at the same offsets.  Returns the
// number of matrices solved.
int64_t oracle_svd_batch(int64_t count, const int32_t* idx, const int32_t* n, const int64_t* aoff,
                         const int64_t* soff, const double* A, double* U, double* S, double* Vt,
                         int32_t threads) {
    std::atomic<int64_t> next{0};
    std::atomic<int64_t> done{0};
    auto worker = [&]() {
        oracle_small_info info;
        for (;;) {
            const int64_t k = next.fetch_add(1);
            if (k >= count) break;
            const int64_t t = idx[k];
            const int64_t nt = n[t];
            const int64_t ao = aoff[t], so = soff[t];
            const int rc = nt <= 4 ? oracle_micro_solve(nt, A + ao, U + ao, S + so, Vt + ao, &info)
                                   : oracle_small_solve(nt, A + ao, U + ao, S + so, Vt + ao, &info);
            if (rc == 0) done.fetch_add(1);
        }
    };
    const int nt = threads > 0 ? threads : 1;
    std::vector<std::thread> pool;
    pool.reserve(size_t(nt));
    for (int i = 0; i < nt; ++i) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
    return done.load();
}

}  // extern "C"

// ----------------------------------------------------------------- triage --
// Test infrastructure: restatement of the reference's triage statistics, the
// checker of lsvd_triage_batched_f64.

struct VecPhase {  // VectorPhaseHealth (src/lie_svd_phasehealth.rs:21-40)
    double scalar_mean, scalar_sq, vector_sq, delay_bivector_sq, gradient_sq, energy_entropy, twist_ratio, phase;
};

// analyze_vector_phase_by (src/lie_svd_phasehealth.rs:146-207) and
// normalized_energy_entropy_by (:313-329) over x(0..n-1).
template <class F>
static VecPhase vector_phase(int64_t n, F at) {
    VecPhase h{0, 0, 0, 0, 0, 0, 0, 0};
    if (n == 0) return h;
    const double nf = double(n);
    double sum = 0.0;
    for (int64_t i = 0; i < n; ++i) sum += at(i);
    const double mean = sum / nf;
    h.scalar_mean = mean;
    h.scalar_sq = nf * mean * mean;
    double vector_sq = 0.0, norm_sq = 0.0, delay = 0.0, grad = 0.0, energy = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double xi = at(i), xn = at((i + 1) % n);
        const double c = xi - mean;
        vector_sq += c * c;
        norm_sq += xi * xi;
        delay += xi * xn;
        const double d = xn - xi;
        grad += d * d;
        energy += xi * xi;
    }
    h.vector_sq = vector_sq;
    h.delay_bivector_sq = std::max(norm_sq * norm_sq - delay * delay, 0.0);
    h.gradient_sq = grad;
    double ent = 0.0;
    if (n > 1 && energy > 1e-300) {
        for (int64_t i = 0; i < n; ++i) {
            const double v = at(i);
            const double pr = (v * v) / energy;
            if (pr > 0.0) ent -= pr * std::log(pr);
        }
        ent /= std::log(nf);
    }
    h.energy_entropy = ent;
    h.twist_ratio = std::sqrt(h.delay_bivector_sq) / std::max(norm_sq, 1e-300);
    const double orient = delay >= 0.0 ? 1.0 : -1.0;
    h.phase = orient * std::atan2(std::sqrt(grad), std::fabs(mean) + std::sqrt(vector_sq) + 1e-300);
    return h;
}

struct PhaseSummary {  // PhaseHealthSummary via summarize (:274-311)
    double dbsq = 0.0, gsq = 0.0, max_twist = 0.0, mean_twist = 0.0, mean_entropy = 0.0;
    int64_t count = 0;
};

// global_phase_invariants' weighted phase sums (:219-232), rows then columns
struct PhaseSums {
    double sin_w = 0.0, cos_w = 0.0, w = 0.0;
};

static void add_item(PhaseSummary& s, PhaseSums& g, const VecPhase& h) {
    s.dbsq += h.delay_bivector_sq;
    s.gsq += h.gradient_sq;
    s.max_twist = std::max(s.max_twist, h.twist_ratio);
    s.mean_twist += h.twist_ratio;
    s.mean_entropy += h.energy_entropy;
    s.count += 1;
    const double w = std::sqrt(h.scalar_sq + h.vector_sq);
    g.sin_w += w * std::sin(h.phase);
    g.cos_w += w * std::cos(h.phase);
    g.w += w;
}

static void finish(PhaseSummary& s) {
    if (s.count) {
        s.mean_twist /= double(s.count);
        s.mean_entropy /= double(s.count);
    }
}

// analyze_block4_signature(..).dual_balance (src/lie_svd_block4.rs:210-262).
static double block4_dual_balance(int64_t rows, int64_t cols, const double* A) {
    const int64_t n = std::min(rows, cols), blocks = n / 4;
    if (blocks == 0) return 0.0;
    double sd2 = 0.0, asd2 = 0.0;
    auto w = [&](int64_t st, int a, int b) { return 0.5 * (A[(st + b) * cols + st + a] - A[(st + a) * cols + st + b]); };
    const double r = 0.70710678118654752440;  // 1/sqrt(2)
    for (int64_t blk = 0; blk < blocks; ++blk) {
        const int64_t st = blk * 4;
        const double w12 = w(st, 0, 1), w13 = w(st, 0, 2), w14 = w(st, 0, 3);
        const double w23 = w(st, 1, 2), w24 = w(st, 1, 3), w34 = w(st, 2, 3);
        const double sd[3] = {(w12 + w34) * r, (w13 - w24) * r, (w14 + w23) * r};
        const double asd[3] = {(w12 - w34) * r, (w13 + w24) * r, (w14 - w23) * r};
        sd2 += sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2];
        asd2 += asd[0] * asd[0] + asd[1] * asd[1] + asd[2] * asd[2];
    }
    const double a = std::sqrt(sd2), b = std::sqrt(asd2);
    return std::fabs(a - b) / std::max(a + b, 1e-300);
}

static double coeff_var(const std::vector<double>& v) {  // src/lie_svd_adaptive.rs:341-355
    double sum = 0.0;
    for (double x : v) sum += x;
    const double len = double(std::max<size_t>(v.size(), 1));
    const double mean = sum / len;
    if (std::fabs(mean) <= 1e-300) return 0.0;
    double var = 0.0;
    for (double x : v) var += (x - mean) * (x - mean);
    return std::sqrt(var / len) / std::fabs(mean);
}

static double rel_l2_mismatch(const std::vector<double>& a, const std::vector<double>& b) {  // :357-366
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < a.size(); ++i) {
        const double d = a[i] - b[i];
        num += d * d;
        den += a[i] * a[i] + b[i] * b[i];
    }
    return std::sqrt(num) / std::max(std::sqrt(den), 1e-300);
}

static double entropy01(const std::vector<double>& v) {  // :368-380
    double sum = 0.0;
    for (double x : v) sum += x;
    if (sum <= 1e-300 || v.size() <= 1) return 1.0;
    double h = 0.0;
    for (double x : v) {
        const double pr = x / sum;
        if (pr > 0.0) h -= pr * std::log(pr);
    }
    return h / std::max(std::log(double(v.size())), 1e-300);
}

extern "C" {

int oracle_triage(int64_t rows, int64_t cols, const double* A, double* out, int32_t* routes) {
    if (rows < 0 || cols < 0) return -1;
    const int64_t n = rows, m = cols;
    // phase signature (src/lie_svd_phasehealth.rs:100-140) and global invariants (:213-272)
    PhaseSummary R, Cs;
    PhaseSums g;
    for (int64_t i = 0; i < n; ++i) add_item(R, g, vector_phase(m, [&](int64_t j) { return A[i * m + j]; }));
    for (int64_t j = 0; j < m; ++j) add_item(Cs, g, vector_phase(n, [&](int64_t i) { return A[i * m + j]; }));
    finish(R);
    finish(Cs);
    const double count = double(std::max<int64_t>(R.count + Cs.count, 1));
    const double total_stress = std::sqrt(R.dbsq + Cs.dbsq) + std::sqrt(R.gsq + Cs.gsq);
    const double mean_stress = total_stress / count;
    const double max_twist = std::max(R.max_twist, Cs.max_twist);
    const double entropy_gap = std::fabs(R.mean_entropy - Cs.mean_entropy);
    const int64_t cor = std::min(n, m);
    double upper = 0.0, lower = 0.0, torsion = 0.0;
    for (int64_t i = 0; i < cor; ++i)
        for (int64_t j = i + 1; j < cor; ++j) {  // triangular_disbalance (:331-343)
            upper += A[i * m + j] * A[i * m + j];
            lower += A[j * m + i] * A[j * m + i];
        }
    const double causal = std::fabs(upper - lower) / std::max(upper + lower, 1e-300);
    for (int64_t i = 0; i < cor; ++i)
        for (int64_t j = i + 1; j < cor; ++j) {
            const double d = (A[i * m + j] - A[j * m + i]) * 0.5;
            torsion += 2.0 * d * d;
        }
    const double global_phase = g.w > 1e-300 ? std::atan2(g.sin_w, g.cos_w) : 0.0;
    double total_sq = 0.0;
    for (int64_t e = 0; e < n * m; ++e) total_sq += A[e] * A[e];
    double pent = 0.0;
    if (n * m > 1 && total_sq > 1e-300) {
        for (int64_t e = 0; e < n * m; ++e) {
            const double pr = (A[e] * A[e]) / total_sq;
            if (pr > 0.0) pent -= pr * std::log(pr);
        }
        pent /= std::log(double(n * m));
    }
    // PhaseEngine passport extras: real_chirality (src/lie_svd_engine.rs:277-292), golden_resonance_real (:310-326)
    double skew = 0.0, tot = 0.0;
    for (int64_t i = 0; i < cor; ++i)
        for (int64_t j = 0; j < cor; ++j) {
            const double x = A[i * m + j];
            tot += x * x;
            if (i < j) {
                const double d = A[i * m + j] - A[j * m + i];
                skew += d * d;
            }
        }
    const double chirality = std::sqrt(skew) / std::max(std::sqrt(tot), 1e-300);
    const double theta = 2.39996322972865332;
    double re = 0.0, im = 0.0, mass = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double ph = theta * double(i);
        double rm = 0.0;
        for (int64_t j = 0; j < m; ++j) rm += std::fabs(A[i * m + j]);
        re += rm * std::cos(ph);
        im += rm * std::sin(ph);
        mass += rm;
    }
    const double golden = std::sqrt(re * re + im * im) / std::max(mass, 1e-300);
    const double nan = std::nan("");
    for (int k = 0; k < 11; ++k) out[k] = nan;
    out[11] = mean_stress;
    out[12] = max_twist;
    out[13] = causal;
    out[14] = entropy_gap;
    out[15] = global_phase;
    out[16] = std::sqrt(torsion);
    out[17] = block4_dual_balance(n, m, A);
    out[18] = pent;
    out[19] = chirality;
    out[20] = golden;
    // passport route hint (src/lie_svd_engine.rs:75-82)
    routes[1] = (n == m && (max_twist > 0.8 || causal > 0.65 || entropy_gap > 0.2) && n <= 128) ? 1 : 0;
    routes[0] = -1;
    if (n != m) return 0;
    // analyze_matrix (src/lie_svd_adaptive.rs:186-274)
    double all_sq = 0.0, diag_sq = 0.0, off_sq = 0.0, sym_sq = 0.0, skew_sq = 0.0;
    std::vector<double> dabs(size_t(n), 0.0), rl1(size_t(n), 0.0), cl1(size_t(n), 0.0), rl2(size_t(n), 0.0),
        cl2(size_t(n), 0.0);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = 0; j < n; ++j) {
            const double v = A[i * n + j], av = std::fabs(v);
            all_sq += v * v;
            rl1[size_t(i)] += av;
            cl1[size_t(j)] += av;
            rl2[size_t(i)] += v * v;
            cl2[size_t(j)] += v * v;
            if (i == j) {
                diag_sq += v * v;
                dabs[size_t(i)] = av;
            } else {
                off_sq += v * v;
            }
        }
    for (int64_t i = 0; i < n; ++i) {
        rl2[size_t(i)] = std::sqrt(rl2[size_t(i)]);
        cl2[size_t(i)] = std::sqrt(cl2[size_t(i)]);
        for (int64_t j = i + 1; j < n; ++j) {
            const double a = A[i * n + j], b = A[j * n + i];
            const double sy = 0.5 * (a + b), sk = 0.5 * (a - b);
            sym_sq += 2.0 * sy * sy;
            skew_sq += 2.0 * sk * sk;
        }
    }
    const double norm = std::max(std::sqrt(all_sq), 1e-300);
    const double offdiag = std::sqrt(off_sq) / norm, dd = std::sqrt(diag_sq) / norm;
    const double rcv = coeff_var(rl2), ccv = coeff_var(cl2), mism = rel_l2_mismatch(rl1, cl1);
    const double symr = std::sqrt(sym_sq) / std::max(std::sqrt(sym_sq + skew_sq), 1e-300);
    const double torr = std::sqrt(skew_sq) / std::max(std::sqrt(sym_sq + skew_sq), 1e-300);
    const double dent = entropy01(dabs), rent = entropy01(rl1), cent = entropy01(cl1);
    // suspicious_score (:325-339)
    double score = 0.0;
    score += std::max(offdiag - 0.55, 0.0) * 0.9;
    score += std::max(0.35 - dd, 0.0) * 0.8;
    score += std::max(rcv, ccv) * 1.4;
    score += mism * 1.6;
    score += torr * 0.45;
    score += offdiag * std::max(symr - 0.82, 0.0) * 1.8;
    score += std::max(0.78 - dent, 0.0) * 1.2;
    const double vals[11] = {offdiag, dd, rcv, ccv, mism, symr, torr, dent, rent, cent, score};
    for (int k = 0; k < 11; ++k) out[k] = vals[k];
    // choose_route with LieSvdAdaptiveParams::default() (:55-65, :103-119, :121-184)
    const double thr = 1.15;
    const bool balanced_degenerate = score >= thr + 0.25 && offdiag > 0.90 && dd < 0.25 && rcv >= 0.20 &&
                                     ccv >= 0.20 && rcv < 0.45 && ccv < 0.45 && mism < 0.45;
    const bool phaseflow =
        balanced_degenerate || (causal > 0.88 && offdiag > 0.20 && mean_stress > 1.0) ||
        (mean_stress > 50.0 && max_twist > 0.92 && rcv < 0.42 && ccv < 0.42 && mism < 0.30 && offdiag > 0.85 &&
         dd < 0.35) ||
        (out[17] > 0.30 && offdiag > 0.20 && out[16] > 1.0 && dd < 0.5);
    const bool symmetric_topological = symr > 0.96 && offdiag > 0.35 && dd < 0.95;
    const bool coreflow = symmetric_topological || balanced_degenerate ||
                          (score >= thr && (rent < 0.92 || cent < 0.92) && mism < 0.22 &&
                           (torr < 0.62 || dent < 0.62) && rcv < 0.42 && ccv < 0.42);
    int route;
    if (n <= 4) route = 0;
    else if (offdiag <= 1e-5) route = 1;
    else if (n <= 64 && phaseflow) route = 2;
    else if (n <= 64 && coreflow) route = 3;
    else if (n <= 512) route = 1;
    else route = 4;
    routes[0] = route;
    return 0;
}

}  // extern "C"
