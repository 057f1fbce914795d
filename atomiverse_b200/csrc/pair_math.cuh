// pair_math.cuh -- numerics shared by the pair kernels (pair.cu and
// pair_general.cu): approximate FP32 special functions, this library's FP64
// exp and reciprocal, the erfcx polynomial, per-row constants and sums, and
// the fixed-point flush of energies and virials.
#pragma once

#include "atvb_common.cuh"
#include "atvb_kernels.cuh"
#include "erfcx_coef.h"

namespace atvb {

constexpr double kMinPair2 = 1e-20; // lj_kernel.cuh:15 kMinPairDist^2

struct PairAcc {
    double fx, fy, fz, elj, ec;
    double v[6];
};

// ---- approximate FP32 special functions (PTX .approx instructions) -------
ATVB_DEV float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
ATVB_DEV float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
ATVB_DEV float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// exp(-z) for z >= 0 in FP64, table-driven (P. T. P. Tang, "Table-driven
// implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15 (1989) 144-157): n = rint(-z 64/ln2), r =
// -z - n ln2/64 (ln2/64 split into a head whose products with n are exact
// and a tail), |r| <= ln2/128, and exp(-z) = 2^(n div 64) 2^((n mod 64)/64)
// exp(r) with 2^(j/64) from a 64-entry table and exp(r) by its Taylor
// series to degree 5 (truncation < 4e-17).  z is clamped at 708 (the result
// is then ~1e-308, far below anything the callers keep).
// exp(w) for -708 <= w <= 0, no clamp (the pair kernels' arguments
// -alpha^2 r^2 stay above -(alpha rlist)^2 >= -676, checked at setup)
ATVB_DEV double exp_neg64_small(double w) {
    const double n = rint(w * kExp64ByLn2);
    double r = fma(-n, kExpLn2By64Hi, w);
    r = fma(-n, kExpLn2By64Lo, r);
    double p = 1.0 / 120.0;
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    const int ni = (int)n;
    const double t = __ldg(kExp2Tab + (ni & 63));
    const long long e = (long long)((ni >> 6) + 1023) << 52; // ni >> 6 >= -1022
    return (t * p) * __longlong_as_double(e);
}

ATVB_DEV double exp_neg64(double z) { return exp_neg64_small(-fmin(z, 708.0)); }

// 1 / v for 1 <= v <= 4 in FP64: FP32 estimate, two Newton steps
// (relative error 2^-22 -> 2^-44 -> below one FP64 ulp).
ATVB_DEV double rcp64(double v) {
    double t = (double)rcp_approx((float)v);
    t = fma(t, fma(-v, t, 1.0), t);
    return fma(t, fma(-v, t, 1.0), t);
}

// 1 / sqrt(v) in FP64 for v in the FP32 normal range: FP32 estimate
// (rsqrt.approx), then two Newton steps y <- y (3/2 - (v/2) y^2) (relative
// error 2^-22 -> 2^-45 -> rounding level).
ATVB_DEV double rsqrt64(double v) {
    double y = (double)rsqrt_approx((float)v);
    const double h = 0.5 * v;
    y = y * fma(-h, y * y, 1.5);
    return y * fma(-h, y * y, 1.5);
}

// erfcx(x) for 0 <= x <= 6 from the universal polynomial of erfcx_coef.h,
// given t = 1 / (1 + kErfcxP x).  Coefficients are compile-time constants.
// FP64: the even and odd coefficients as two Horner chains in u^2 (half
// the dependency depth of one chain, one more operation), p = E + u O
ATVB_DEV double erfcx_of_t(double t) {
    const double u = fma(kErfcxA, t, kErfcxB);
    const double v = u * u;
    constexpr int NE = (kErfcxD_N + 1) / 2, NO = kErfcxD_N / 2;
    double e = kErfcxD[2 * (NE - 1)];
    double o = kErfcxD[2 * (NO - 1) + 1];
#pragma unroll
    for (int k = NE - 2; k >= 0; --k)
        e = fma(e, v, kErfcxD[2 * k]);
#pragma unroll
    for (int k = NO - 2; k >= 0; --k)
        o = fma(o, v, kErfcxD[2 * k + 1]);
    return fma(u, o, e);
}
// the short-range FP64 set (systems with alpha * cutoff <= kErfcxSXmax):
// t = 1 / (1 + kErfcxSP x), five fewer terms
ATVB_DEV double erfcx_short_of_t(double t) {
    const double u = fma(kErfcxSA, t, kErfcxSB);
    const double v = u * u;
    constexpr int NE = (kErfcxS_N + 1) / 2, NO = kErfcxS_N / 2;
    double e = kErfcxS[2 * (NE - 1)];
    double o = kErfcxS[2 * (NO - 1) + 1];
#pragma unroll
    for (int k = NE - 2; k >= 0; --k)
        e = fma(e, v, kErfcxS[2 * k]);
#pragma unroll
    for (int k = NO - 2; k >= 0; --k)
        o = fma(o, v, kErfcxS[2 * k + 1]);
    return fma(u, o, e);
}
ATVB_DEV float erfcx_of_t(float t) {
    const float u = fmaf((float)kErfcxA, t, (float)kErfcxB);
    float p = kErfcxF[kErfcxF_N - 1];
#pragma unroll
    for (int k = kErfcxF_N - 2; k >= 0; --k)
        p = fmaf(p, u, kErfcxF[k]);
    return p;
}

// Per-row constants of one system, hoisted out of the pair loop.
template <typename T>
struct RowConst {
    // shifted LJ with folded constants (r6 = 1/r^6): F/r = r6 (lj1 r6 - lj2) / r^2,
    // E = r6 (lj3 r6 - lj4) - shift; lj1 = 48 eps sigma^12, lj2 = 24 eps sigma^6,
    // lj3 = 4 eps sigma^12, lj4 = 4 eps sigma^6
    T lj_rc2, lj1, lj2, lj3, lj4, shift;
    T sig6, eps4, eps24; // the unfolded form (FP32 build)
    T c_rc2, alpha, alpha2; // alpha2: alpha^2 (FP64) or alpha^2 log2(e) (FP32)
    T kqi;
    T band_lj, band_c; // FP32 only: error band of r^2 around each cutoff
};

template <typename T>
struct RowSums {
    T fx = 0, fy = 0, fz = 0, elj = 0, ec = 0;
    T v[6] = {0, 0, 0, 0, 0, 0};
    // mixed build: force components summed in 64-bit fixed point, units of
    // kForceFix^-1 eV/A (range +-2e9 eV/A), so the row sum is exact and
    // independent of summation order
    long long fq[3] = {0, 0, 0};
    // mixed build: the row's smallest r^2 (a pair closer than
    // SysParams::force_r2_safe may carry a force beyond the fixed point)
    T rmin = T(1e30);
};
constexpr float kForceFix = 4294967296.0f;  // 2^32
constexpr double kForceFixInv = 1.0 / 4294967296.0;

template <typename T>
ATVB_DEV void finish_row(const RowSums<T>& r, PairAcc& a, bool vir) {
    if constexpr (sizeof(T) == 4) {
        // multiples of 2^-32 below 2^21 in magnitude: every later FP64 sum of
        // the lanes' values is exact, so the force is order-independent
        a.fx = (double)r.fq[0] * kForceFixInv;
        a.fy = (double)r.fq[1] * kForceFixInv;
        a.fz = (double)r.fq[2] * kForceFixInv;
    } else {
        a.fx = (double)r.fx;
        a.fy = (double)r.fy;
        a.fz = (double)r.fz;
    }
    a.elj += (double)r.elj;
    a.ec += (double)r.ec;
    if (vir)
        for (int k = 0; k < 6; ++k)
            a.v[k] += (double)r.v[k];
}

template <typename T>
ATVB_DEV RowConst<T> row_const(const SysParams& P, double qi) {
    RowConst<T> c;
    c.lj_rc2 = (T)P.lj_rc2;
    c.lj1 = (T)(2.0 * P.lj_eps24 * P.lj_sig6 * P.lj_sig6);
    c.lj2 = (T)(P.lj_eps24 * P.lj_sig6);
    c.lj3 = (T)(P.lj_eps4 * P.lj_sig6 * P.lj_sig6);
    c.lj4 = (T)(P.lj_eps4 * P.lj_sig6);
    c.shift = (T)P.lj_shift;
    c.sig6 = (T)P.lj_sig6;
    c.eps4 = (T)P.lj_eps4;
    c.eps24 = (T)P.lj_eps24;
    c.c_rc2 = (T)P.coul_rc2;
    c.alpha = (T)P.coul_alpha;
    c.alpha2 = sizeof(T) == 4 ? (T)(P.coul_alpha2 * 1.4426950408889634) : (T)P.coul_alpha2;
    c.kqi = (T)(kQqr2e * qi);
    c.band_lj = (T)P.mix_band_lj;
    c.band_c = (T)P.mix_band_c;
    return c;
}

// Per-item flush: every item's energy/virial partial is rounded to fixed
// point on its own, so a system's sums do not depend on which other systems
// share the launch (results are identical alone and batched).
ATVB_DEV void flush_energy(const SysParams& P, PairAcc& a, double* sh) {
    if (P.need_virial) {
        double v[8] = {a.elj, a.ec, a.v[0], a.v[1], a.v[2], a.v[3], a.v[4], a.v[5]};
        block_sum_vec<8>(v, sh);
        if (threadIdx.x == 0) {
            if (P.has_lj)
                fix_add(&P.st->acc[kAccELJ], 0.5 * v[0]);
            if (P.has_coul)
                fix_add(&P.st->acc[kAccECoul], 0.5 * v[1]);
            for (int k = 0; k < 6; ++k)
                fix_add(&P.st->acc[kAccVir + k], 0.5 * v[2 + k]);
        }
    } else {
        double v[2] = {a.elj, a.ec};
        block_sum_vec<2>(v, sh);
        if (threadIdx.x == 0) {
            // 1/2: every pair is visited from both of its atoms
            if (P.has_lj)
                fix_add(&P.st->acc[kAccELJ], 0.5 * v[0]);
            if (P.has_coul)
                fix_add(&P.st->acc[kAccECoul], 0.5 * v[1]);
        }
    }
    a.elj = a.ec = 0.0;
    for (int k = 0; k < 6; ++k)
        a.v[k] = 0.0;
}

// Mixed: at least 3 resident blocks (80 registers); FP64: 2.
} // namespace atvb
