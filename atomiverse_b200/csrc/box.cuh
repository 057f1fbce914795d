// box.cuh -- every SysParams field that depends on the cell edges, computed
// in one place for the host (system setup) and the device (the MTK NPT cell
// update, committed once per step by k_sys_a).
//
// Depends on the cell: the fixed-point position scales, the minimum-image
// constants, the bin size (the bin COUNT is fixed when the system is
// planned), the FP32 screening bands of the neighbour build and of the mixed
// pair kernel (they bound rounding errors that grow with the coordinates),
// and the PME prefactors k_e/(pi V), k_e/(2 pi V) and the net-charge energy.
#pragma once

#include <math.h>

#include "atvb_common.cuh"

namespace atvb {

// |r2_fp32 - r2_fp64| of the mixed pair kernel: <= 10 2^-24 r2 (conversion,
// scale, product, squares and sums) + 2 sqrt(3) r q (32-bit fixed-point
// quantum q on both atoms); the band doubles it
__host__ __device__ inline double mixed_band(double rc2, double q) {
    return 2.0 * (10.0 / 16777216.0 * rc2 + 2.0 * sqrt(3.0) * sqrt(rc2) * q);
}

// P.nc, P.rlist, P.rlist2 and the physics flags must be set.  `npt_const`:
// also recompute the PME net-charge energy from the new volume.
__host__ __device__ inline void apply_box(SysParams& P, const double L[3], bool npt_const) {
    for (int k = 0; k < 3; ++k) {
        P.L[k] = L[k];
        P.invL[k] = 1.0 / L[k];
        P.halfL[k] = 0.5 * L[k];
        P.Lf_fix[k] = (float)(L[k] / 4294967296.0);
        P.fix_scale[k] = 4294967296.0 / L[k];
        P.fix64_scale[k] = 18446744073709551616.0 / L[k];
        P.Lfix64[k] = L[k] / 18446744073709551616.0;
        P.cs_inv[k] = (double)P.nc[k] / L[k];
    }
    // |r2_fp32 - r2_exact| of the list screen <= 5.4e-7 r2 (three FP32
    // roundings of each difference, three of the sum) + 3.6 r q (fixed-point
    // quantum q = L / 2^32 on both atoms); the band doubles both terms
    const double q = fmax(L[0], fmax(L[1], L[2])) / 4294967296.0;
    const double band = 2e-6 * P.rlist2 + 8.0 * P.rlist * q + 1e-12;
    P.lband_lo = nextafterf((float)(P.rlist2 - band), 0.0f);
    P.lband_hi = nextafterf((float)(P.rlist2 + band), 3.0e38f);
    // cell-local frame: coordinates up to R = rlist + 2 cell diagonals from
    // the origin, each carrying <= 3 FP32 roundings (2^-24 R) plus the
    // fixed-point quantum; the difference one more rounding
    double cs[3];
    for (int k = 0; k < 3; ++k)
        cs[k] = L[k] / (double)P.nc[k];
    const double cdiag = sqrt(cs[0] * cs[0] + cs[1] * cs[1] + cs[2] * cs[2]);
    const double R = P.rlist + 2.0 * cdiag;
    const double u = 1.0 / 16777216.0;
    const double ec = 3.0 * u * R + 2.0 * q;
    const double ed = 2.0 * ec + u * P.rlist;
    const double fband = 2.0 * (2.0 * sqrt(3.0) * P.rlist * ed + 3.0 * u * P.rlist2) + 1e-12;
    P.fband_lo = nextafterf((float)(P.rlist2 - fband), 0.0f);
    P.fband_hi = nextafterf((float)(P.rlist2 + fband), 3.0e38f);
    P.lframe_ok = 1;
    for (int k = 0; k < 3; ++k)
        if (!(0.5 * L[k] > R + 1e-9))
            P.lframe_ok = 0;
    // mixed pair kernel: bands around the LJ and Coulomb cutoffs (the LJ one
    // stays off where the settling was switched off)
    if (P.mix_band_lj > 0.0)
        P.mix_band_lj = mixed_band(P.lj_rc2, q);
    if (P.has_coul)
        P.mix_band_c = mixed_band(P.coul_rc2, q);
    if (P.has_pme) {
        const double vol = L[0] * L[1] * L[2];
        P.pme_fscale = kQqr2e / (kPi * vol);
        P.pme_escale = kQqr2e / (2.0 * kPi * vol);
        if (npt_const)
            P.e_const = P.pme_eself -
                        kQqr2e * kPi / (2.0 * vol * P.pme_alpha * P.pme_alpha) * P.pme_qsum2;
    }
}

} // namespace atvb
