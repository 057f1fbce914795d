// C wrappers around the reference's own header-only PME math
// (include/atomiverse/cpu/longrange/pme_spline.h and pme_influence.h),
// compiled from the reference tree by oracle/ref_build.sh into
// oracle/_ref/libref_pme.so.  Test infrastructure: the oracle's PME
// restatement is checked against these functions.
#include <complex>
#include <vector>

#include "atomiverse/core/mat3.h"
#include "atomiverse/cpu/longrange/pme_influence.h"
#include "atomiverse/cpu/longrange/pme_spline.h"

namespace {
ATV::Mat3 diag_inv(const double L[3]) {
    ATV::Mat3 m;
    for (int d = 0; d < 3; ++d)
        m(d, d) = 1.0 / L[d];
    return m;
}
} // namespace

extern "C" {

void ref_bspline(double frac, int n, double* th, double* dth) {
    ATV::longrange::bspline(frac, n, th, dth);
}

int ref_good_fft_size(int n) { return ATV::longrange::good_fft_size(n); }

void ref_spline_moduli(int K, int n, double* out) {
    auto v = ATV::longrange::spline_moduli(K, n);
    for (int i = 0; i < K; ++i)
        out[i] = v[static_cast<std::size_t>(i)];
}

// Spread charges onto a complex grid (interleaved re/im), K0*K1*K2 points.
void ref_spread(int n, const double* x, const double* y, const double* z,
                const double* q, const double L[3], const int K[3], int order,
                double* grid_c) {
    std::vector<int> base(3 * static_cast<std::size_t>(n));
    std::vector<double> th(3 * static_cast<std::size_t>(order) * n),
        dth(3 * static_cast<std::size_t>(order) * n);
    ATV::longrange::pme_fill_atom_splines(x, y, z, n, diag_inv(L), K, order,
                                          base.data(), th.data(), dth.data());
    ATV::longrange::pme_spread_charges(
        q, n, order, K, base.data(), th.data(),
        reinterpret_cast<std::complex<double>*>(grid_c));
}

// Apply influence tables in place on a forward-transformed grid.
void ref_influence(double* grid_c, const double L[3], const int K[3], int order,
                   double alpha, double* energy, double* stress) {
    std::vector<double> m0 = ATV::longrange::spline_moduli(K[0], order);
    std::vector<double> m1 = ATV::longrange::spline_moduli(K[1], order);
    std::vector<double> m2 = ATV::longrange::spline_moduli(K[2], order);
    ATV::longrange::PmeInfluenceTables tab;
    ATV::longrange::pme_build_influence_tables(K, m0.data(), m1.data(),
                                               m2.data(), diag_inv(L), alpha,
                                               tab);
    ATV::longrange::pme_apply_influence_tables(
        reinterpret_cast<std::complex<double>*>(grid_c), K[0] * K[1] * K[2],
        tab, L[0] * L[1] * L[2], *energy, stress);
}

// Interpolate forces from a real-space (post inverse FFT) complex grid.
void ref_interpolate(int n, const double* x, const double* y, const double* z,
                     const double* q, const double L[3], const int K[3],
                     int order, const double* grid_c, double* fx, double* fy,
                     double* fz) {
    std::vector<int> base(3 * static_cast<std::size_t>(n));
    std::vector<double> th(3 * static_cast<std::size_t>(order) * n),
        dth(3 * static_cast<std::size_t>(order) * n);
    ATV::longrange::pme_fill_atom_splines(x, y, z, n, diag_inv(L), K, order,
                                          base.data(), th.data(), dth.data());
    ATV::longrange::pme_interpolate_forces(
        q, n, order, K, diag_inv(L), L[0] * L[1] * L[2], base.data(),
        th.data(), dth.data(),
        reinterpret_cast<const std::complex<double>*>(grid_c), fx, fy, fz);
}
}
