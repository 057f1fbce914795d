// pair.cu -- short-range pair force, energy and virial over the full list.
//
// Physics: shifted LJ 12-6 (src/cpu/potentials/pair_lj_cut.cpp:30-41 and
// :723-800; shift as include/atomiverse/cuda/potentials/lj_kernel.cuh:59-65)
// plus real-space Ewald Coulomb (src/cpu/potentials/coul_long.cpp:146-222):
//   E_ij = k_e q_i q_j erfc(a r)/r,
//   F_ij/r = k_e q_i q_j [erfc(a r) + 2/sqrt(pi) a r exp(-a^2 r^2)] / r^3.
// LJ and Coulomb are fused into ONE walk of the list (the reference CUDA
// backend walks it twice, pair_lj_cut.cu + coul_long.cu).
//
// Layout: G lanes share one sorted atom i; lane g takes row entries
// g, g+G, ...; the lanes' partial forces are combined with a fixed xor tree,
// so the force on every atom is summed in the same order on every run (no
// atomics on forces).  Because every pair appears in both rows, energy and
// virial carry a factor 1/2 (pair_lj_cut.cu:195 in the reference does the
// same on its full list).  Energy/virial block partials are added into the
// system's 64-bit fixed-point accumulators.
//
// erfc: erfc(x) = exp(-x^2) erfcx(x), with erfcx from ONE polynomial in
// t = 1/(1 + 0.4 x) valid for every system with alpha * cutoff <= 6
// (erfcx_coef.h, compile-time coefficients: no tables, no shared memory).
//
// FP64 build: positions as 64-bit fixed point (2^64 steps per box edge,
// so the wrapped integer difference is the exact minimum image) + FP64 q;
// all arithmetic in double;
// exp and the reciprocal of the erfcx variable are this library's own FP64
// routines (table-driven exp, Newton reciprocal), accurate to ~1 ulp;
// systems with alpha * cutoff <= 3.2 take a shorter erfcx polynomial.
// Mixed build: positions int4 {x, y, z fixed point with 2^32 steps per box
// edge, q as float}; the integer difference is the exact minimum-image
// separation, converted once to float; pair math in FP32 with the PTX
// approximate rsqrt / rcp / ex2; the next two row entries are gathered while
// the current two are computed; per-row sums are promoted to FP64 before the
// lanes are combined.
#include "pair_math.cuh"

namespace atvb {

// One pair (i, j) at separation (dx, dy, dz), charge product factor qj.
// Cutoffs are applied by selection, not branches: every lane of a warp runs
// the same instructions, and a value computed outside its range (including
// r^2 = 0) is never selected.
//
// FP32 only: the cutoff tests decide which pairs exist, and the shifted LJ
// force jumps at its cutoff, so a pair that FP32 rounding moves across a
// cutoff would cost a whole pair force.  `near` reports an r^2 within the
// FP32 error band of the LJ cutoff (a ~1e-6-thick shell, ~1e-5 of pairs);
// such pairs are queued and k_pair_fix settles them on the FP64 positions.
// `force` >= 0 overrides the decisions (bit 0 LJ, bit 1 Coulomb) and `neg`
// subtracts the term instead of adding it (k_pair_fix only).
template <bool LJ, bool CO, bool VIR, bool SHORT = false, typename T>
ATVB_DEV void pair_term(const RowConst<T>& c, T dx, T dy, T dz, T qj,
                        RowSums<T>& a, bool& near, int force = -1, bool neg = false) {
    constexpr bool F = sizeof(T) == 4;
    const T r2 = dx * dx + dy * dy + dz * dz;
    const bool ok = r2 >= (T)kMinPair2;
    bool in_lj = ok && r2 < c.lj_rc2, in_c = ok && r2 < c.c_rc2;
    if constexpr (F) {
        // only the LJ cutoff: the real-space Coulomb force at its cutoff is
        // damped by erfc(alpha rc) (~3e-5 eV/A per pair at alpha rc = 3),
        // so a flipped Coulomb pair moves the forces by ~1e-7 relative
        near = LJ && fabsf(r2 - c.lj_rc2) < c.band_lj;
        // (entries past a row's end are the atom itself, r^2 = 0: not pairs)
        a.rmin = ok ? fminf(a.rmin, r2) : a.rmin;
        if (force >= 0) {
            in_lj = force & 1;
            in_c = (force >> 1) & 1;
        }
    }
    T rinv;
    if constexpr (F)
        rinv = rsqrt_approx(r2);
    else
        rinv = rsqrt64(r2);
    const T r2inv = rinv * rinv;
    const T sg = neg ? T(-1) : T(1);
    T fpair = 0;
    if (LJ) {
        T flj, elj;
        if constexpr (F) {
            const T r6 = r2inv * r2inv * r2inv * c.sig6;
            flj = c.eps24 * r2inv * r6 * (T(2) * r6 - T(1));
            elj = c.eps4 * r6 * (r6 - T(1)) - c.shift;
        } else {
            // folded constants: four fewer FP64 operations
            const T r6 = r2inv * r2inv * r2inv;
            flj = (r2inv * r6) * fma(c.lj1, r6, -c.lj2);
            elj = fma(r6, fma(c.lj3, r6, -c.lj4), -c.shift);
        }
        fpair = in_lj ? flj : T(0);
        a.elj += in_lj ? sg * elj : T(0);
    }
    if (CO) {
        // erfc(x) = exp(-x^2) erfcx(x), x = alpha r
        const T qq = c.kqi * qj;
        const T x = c.alpha * (r2 * rinv);
        T t, e;
        if constexpr (F) {
            t = rcp_approx(fmaf((float)kErfcxP, x, 1.0f));
            e = ex2_approx(-c.alpha2 * r2);
        } else {
            t = rcp64(fma(SHORT ? kErfcxSP : kErfcxP, x, 1.0));
            e = exp_neg64_small(-(c.alpha2 * r2)); // alpha rlist <= 26 (checked at setup)
        }
        T p;
        if constexpr (!F && SHORT)
            p = erfcx_short_of_t(t);
        else
            p = erfcx_of_t(t);
        const T pref = qq * rinv * e;
        const T fc = pref * (p + (T)kEwaldF * x) * r2inv;
        // a plain rounded add: never fused with the product above, so every
        // instantiation (lane count) rounds each pair force the same way
        if constexpr (F)
            fpair = __fadd_rn(fpair, in_c ? fc : T(0));
        else
            fpair = __dadd_rn(fpair, in_c ? fc : T(0));
        a.ec += in_c ? sg * (pref * p) : T(0);
    }
    const T fxp = fpair * dx, fyp = fpair * dy, fzp = fpair * dz;
    if constexpr (F) {
        const long long qx = __float2ll_rn(fxp * kForceFix);
        const long long qy = __float2ll_rn(fyp * kForceFix);
        const long long qz = __float2ll_rn(fzp * kForceFix);
        a.fq[0] += neg ? -qx : qx;
        a.fq[1] += neg ? -qy : qy;
        a.fq[2] += neg ? -qz : qz;
    } else {
        a.fx += fxp;
        a.fy += fyp;
        a.fz += fzp;
    }
    if (VIR) {
        a.v[0] += sg * (dx * fxp);
        a.v[1] += sg * (dy * fyp);
        a.v[2] += sg * (dz * fzp);
        a.v[3] += sg * (dx * fyp);
        a.v[4] += sg * (dx * fzp);
        a.v[5] += sg * (dy * fzp);
    }
}

// Row of sorted atom s, lanes g, g+G, ...: two entries per iteration so that
// both index loads and both position gathers are in flight together.
template <bool LJ, bool CO, bool VIR, bool SHORT>
ATVB_DEV void row_fp64(const SysParams& P, int s, int g, int G, PairAcc& acc) {
    const double4* __restrict__ pos = reinterpret_cast<const double4*>(P.pos4);
    const double4 pi = pos[s];
    const int nn = P.nnbr[s];
    const int* __restrict__ row = P.nbr + (size_t)s * P.cap;
    const RowConst<double> c = row_const<double>(P, pi.w);
    RowSums<double> a;
    bool near;
    // the wrapped 64-bit difference is the exact minimum-image separation
    const double s0 = P.Lfix64[0], s1 = P.Lfix64[1], s2 = P.Lfix64[2];
    auto sep = [&](const double4& pj, double& dx, double& dy, double& dz) {
        dx = (double)(__double_as_longlong(pi.x) - __double_as_longlong(pj.x)) * s0;
        dy = (double)(__double_as_longlong(pi.y) - __double_as_longlong(pj.y)) * s1;
        dz = (double)(__double_as_longlong(pi.z) - __double_as_longlong(pj.z)) * s2;
    };
    // software pipeline: the positions of the next two entries and the row
    // indices of the two after them are in flight while the current pair
    // computes (the kernel waits on the gather, not on the FP64 pipe)
    int k = g;
    int ja = k < nn ? __ldg(row + k) : 0;
    int jb = k + G < nn ? __ldg(row + k + G) : 0;
    double4 pa = pos[ja], pb = pos[jb];
    {
        const int kn = k + 2 * G;
        ja = kn < nn ? __ldg(row + kn) : 0;
        jb = kn + G < nn ? __ldg(row + kn + G) : 0;
    }
    for (; k + G < nn; k += 2 * G) {
        const double4 ca = pa, cb = pb;
        pa = pos[ja];
        pb = pos[jb];
        const int kn = k + 4 * G;
        ja = kn < nn ? __ldg(row + kn) : 0;
        jb = kn + G < nn ? __ldg(row + kn + G) : 0;
        double dx, dy, dz;
        sep(ca, dx, dy, dz);
        pair_term<LJ, CO, VIR, SHORT>(c, dx, dy, dz, ca.w, a, near);
        sep(cb, dx, dy, dz);
        pair_term<LJ, CO, VIR, SHORT>(c, dx, dy, dz, cb.w, a, near);
    }
    if (k < nn) {
        double dx, dy, dz;
        sep(pa, dx, dy, dz);
        pair_term<LJ, CO, VIR, SHORT>(c, dx, dy, dz, pa.w, a, near);
    }
    finish_row(a, acc, VIR);
}

// Cutoff decisions of sorted pair (s, j) from the FP64 master positions,
// through the same 64-bit fixed-point minimum image as the FP64 build:
// bit 0 = inside the LJ cutoff, bit 1 = inside the Coulomb cutoff.  Out of
// line: it runs for ~1e-4 of the pairs and must not cost the hot loop
// registers.
__device__ __noinline__ unsigned exact_cutoffs(const SysParams& P, int s, int j) {
    const int io = P.perm[s], jo = P.perm[j];
    const double xi[3] = {P.x[io], P.y[io], P.z[io]};
    const double xj[3] = {P.x[jo], P.y[jo], P.z[jo]};
    double r2d = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const long long di = (long long)(pos_fix64(xi[d], P.fix64_scale[d]) -
                                         pos_fix64(xj[d], P.fix64_scale[d]));
        const double dd = (double)di * P.Lfix64[d];
        r2d += dd * dd;
    }
    if (!(r2d >= kMinPair2))
        return 0u;
    return (r2d < P.lj_rc2 ? 1u : 0u) | (r2d < P.coul_rc2 ? 2u : 0u);
}

// A lane's share of row s (entries g, g+G, ...) held a pair whose FP32 r^2
// fell in the LJ cutoff's error band: queued for k_pair_fix, which rescans
// that share and settles such pairs on the FP64 positions (rare: ~1e-5 of
// the pairs, one queue entry per affected lane).  code = g | (G << 6).
ATVB_DEV void queue_near(const SysParams& P, int s, int code) {
    const int q = atomicAdd(&P.st->nearq_n, 1);
    if (q < P.nearq_cap)
        P.nearq[q] = make_int2(s, code);
    else {
        // the share keeps its FP32 cutoff decisions: flagged, never silent
        atomicAdd(&P.st->nearq_lost, 1);
        atomicOr(&P.st->status, kStatusNearqLost);
    }
}

template <bool LJ, bool CO, bool VIR, bool NEAR>
ATVB_DEV void row_mixed(const SysParams& P, int s, int g, int G, PairAcc& acc) {
    const int4* __restrict__ pos = reinterpret_cast<const int4*>(P.pos4);
    const int4 pi = pos[s];
    const int nn = P.nnbr[s];
    const int* __restrict__ row = P.nbr + (size_t)s * P.cap;
    const float sx = P.Lf_fix[0], sy = P.Lf_fix[1], sz = P.Lf_fix[2];
    const RowConst<float> c = row_const<float>(P, (double)__int_as_float(pi.w));
    RowSums<float> a;
    // the wrapped integer difference is the exact minimum-image separation
    auto sep = [&](const int4& pj, float& dx, float& dy, float& dz) {
        dx = (float)(int)((unsigned)pi.x - (unsigned)pj.x) * sx;
        dy = (float)(int)((unsigned)pi.y - (unsigned)pj.y) * sy;
        dz = (float)(int)((unsigned)pi.z - (unsigned)pj.z) * sz;
    };
    // software pipeline: the positions of the next two entries and the row
    // indices of the two after them are loaded while the current two are
    // computed; an entry past the row end is the atom itself (r^2 = 0,
    // never selected)
    bool near;
    int n_near = 0;
    int k = g;
    int4 pa = pos[k < nn ? __ldg(row + k) : s];
    int4 pb = pos[k + G < nn ? __ldg(row + k + G) : s];
    int ia = k + 2 * G < nn ? __ldg(row + k + 2 * G) : s;
    int ib = k + 3 * G < nn ? __ldg(row + k + 3 * G) : s;
    for (; k < nn; k += 2 * G) {
        const int4 na = pos[ia];
        const int4 nb = pos[ib];
        const int kn = k + 4 * G;
        ia = kn < nn ? __ldg(row + kn) : s;
        ib = kn + G < nn ? __ldg(row + kn + G) : s;
        float dx, dy, dz;
        sep(pa, dx, dy, dz);
        pair_term<LJ, CO, VIR>(c, dx, dy, dz, __int_as_float(pa.w), a, near);
        if (NEAR)
            n_near += near;
        sep(pb, dx, dy, dz);
        pair_term<LJ, CO, VIR>(c, dx, dy, dz, __int_as_float(pb.w), a, near);
        if (NEAR)
            n_near += near;
        pa = na;
        pb = nb;
    }
    if (NEAR && n_near)
        queue_near(P, s, g | (G << 6));
    if (a.rmin < (float)P.force_r2_safe) // rare: a pair force may exceed the fixed point
        atomicOr(&P.st->status, kStatusForceRange);
    finish_row(a, acc, VIR);
}

template <bool MIXED, bool LJ, bool CO, bool VIR>
ATVB_DEV void row(const SysParams& P, int s, int g, int G, PairAcc& a) {
    if (MIXED) {
        // near-cutoff settling only where the LJ force jump matters
        if (LJ && P.mix_band_lj > 0.0)
            row_mixed<LJ, CO, VIR, true>(P, s, g, G, a);
        else
            row_mixed<LJ, CO, VIR, false>(P, s, g, G, a);
    } else if (CO && P.coul_short) {
        row_fp64<LJ, CO, VIR, true>(P, s, g, G, a);
    } else {
        row_fp64<LJ, CO, VIR, false>(P, s, g, G, a);
    }
}

template <bool MIXED, int G>
__global__ void __launch_bounds__(256, MIXED ? 3 : 2)
    k_pair(const Item* items, int nitems, const SysParams* sp) {
    __shared__ double sh[32 * 8];
    const int g = threadIdx.x % G;
    const int a_off = threadIdx.x / G;
    PairAcc acc;
    acc.elj = acc.ec = 0.0;
    for (int k = 0; k < 6; ++k)
        acc.v[k] = 0.0;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int s = item.begin + a_off;
        acc.fx = acc.fy = acc.fz = 0.0;
        if (s < P.n) {
            const bool lj = P.has_lj, co = P.has_coul, vr = P.need_virial;
            if (lj && co) {
                if (vr)
                    row<MIXED, true, true, true>(P, s, g, G, acc);
                else
                    row<MIXED, true, true, false>(P, s, g, G, acc);
            } else if (lj) {
                if (vr)
                    row<MIXED, true, false, true>(P, s, g, G, acc);
                else
                    row<MIXED, true, false, false>(P, s, g, G, acc);
            } else if (co) {
                if (vr)
                    row<MIXED, false, true, true>(P, s, g, G, acc);
                else
                    row<MIXED, false, true, false>(P, s, g, G, acc);
            }
        }
        double fx = acc.fx, fy = acc.fy, fz = acc.fz;
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
        }
        if (g == 0 && s < P.n)
            P.f4[s] = make_double4(fx, fy, fz, 0.0);
        flush_energy(P, acc, sh);
    }
}

// Settles the near-cutoff pairs of the queued lane shares (one warp per
// queue entry, kFixBlocks blocks per system): every entry of the share is
// recomputed exactly as the pair kernel computed it, and a pair inside the
// LJ band is subtracted and added back under the FP64 cutoff decisions.
// Force corrections are whole multiples of 2^-32 eV/A and so are the pair
// kernel's forces, so the additions are exact and their order does not
// matter; energy and virial corrections go to the fixed-point accumulators
// (x 1/2: each pair sits in both of its rows).  Runs after the pair kernel
// and before the PME gather adds to the same forces.  The queue is emptied
// at the start of the next step (k_sys_a) or force pass.
constexpr int kFixBlocks = 16;

template <bool LJ, bool CO, bool VIR>
ATVB_DEV void fix_share(const SysParams& P, int s, int code, int lane) {
    const int g = code & 63, G = code >> 6;
    const int4* __restrict__ pos = reinterpret_cast<const int4*>(P.pos4);
    const int4 pi = pos[s];
    const int nn = P.nnbr[s];
    const int* __restrict__ row = P.nbr + (size_t)s * P.cap;
    const RowConst<float> c = row_const<float>(P, (double)__int_as_float(pi.w));
    for (int k = g + G * lane; k < nn; k += 32 * G) {
        const int j = __ldg(row + k);
        const int4 pj = pos[j];
        const float dx = (float)(int)((unsigned)pi.x - (unsigned)pj.x) * P.Lf_fix[0];
        const float dy = (float)(int)((unsigned)pi.y - (unsigned)pj.y) * P.Lf_fix[1];
        const float dz = (float)(int)((unsigned)pi.z - (unsigned)pj.z) * P.Lf_fix[2];
        RowSums<float> d;
        bool near;
        pair_term<LJ, CO, VIR>(c, dx, dy, dz, __int_as_float(pj.w), d, near, -1, true);
        if (!near)
            continue;
        const int is = (int)exact_cutoffs(P, s, j);
        pair_term<LJ, CO, VIR>(c, dx, dy, dz, __int_as_float(pj.w), d, near, is, false);
        if (d.fq[0] | d.fq[1] | d.fq[2]) {
            double* f = reinterpret_cast<double*>(P.f4 + s);
            atomicAdd(f + 0, (double)d.fq[0] * kForceFixInv);
            atomicAdd(f + 1, (double)d.fq[1] * kForceFixInv);
            atomicAdd(f + 2, (double)d.fq[2] * kForceFixInv);
        }
        if (d.elj != 0.0f)
            fix_add(&P.st->acc[kAccELJ], 0.5 * (double)d.elj);
        if (d.ec != 0.0f)
            fix_add(&P.st->acc[kAccECoul], 0.5 * (double)d.ec);
        if (VIR)
            for (int q = 0; q < 6; ++q)
                if (d.v[q] != 0.0f)
                    fix_add(&P.st->acc[kAccVir + q], 0.5 * (double)d.v[q]);
    }
}

__global__ void __launch_bounds__(256)
    k_pair_fix(const int* sys_list, int nsys, const SysParams* sp) {
    const SysParams& P = sp[sys_list[blockIdx.x / kFixBlocks]];
    if (P.prec != kMixed || !P.has_lj || P.general || P.nearq == nullptr ||
        !(P.mix_band_lj > 0.0))
        return;
    const int nq = min(P.st->nearq_n, P.nearq_cap);
    const int lane = threadIdx.x & 31;
    const int w0 = (blockIdx.x % kFixBlocks) * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int nw = kFixBlocks * (blockDim.x / 32);
    const bool co = P.has_coul, vr = P.need_virial;
    for (int e = w0; e < nq; e += nw) {
        const int2 q = P.nearq[e];
        if (co) {
            if (vr)
                fix_share<true, true, true>(P, q.x, q.y, lane);
            else
                fix_share<true, true, false>(P, q.x, q.y, lane);
        } else {
            if (vr)
                fix_share<true, false, true>(P, q.x, q.y, lane);
            else
                fix_share<true, false, false>(P, q.x, q.y, lane);
        }
    }
}

template <bool MIXED>
static void launch_pair_prec(const LaunchCfg& lc, cudaStream_t s) {
    const ItemList* L = lc.pair[MIXED ? 1 : 0];
    if (L[0].n)
        k_pair<MIXED, 1><<<L[0].grid, kPairBlock, 0, s>>>(L[0].d, L[0].n, lc.sp);
    if (L[1].n)
        k_pair<MIXED, 2><<<L[1].grid, kPairBlock, 0, s>>>(L[1].d, L[1].n, lc.sp);
    if (L[2].n)
        k_pair<MIXED, 4><<<L[2].grid, kPairBlock, 0, s>>>(L[2].d, L[2].n, lc.sp);
    if (L[3].n)
        k_pair<MIXED, 8><<<L[3].grid, kPairBlock, 0, s>>>(L[3].d, L[3].n, lc.sp);
    if (L[4].n)
        k_pair<MIXED, 16><<<L[4].grid, kPairBlock, 0, s>>>(L[4].d, L[4].n, lc.sp);
    if (L[5].n)
        k_pair<MIXED, 32><<<L[5].grid, kPairBlock, 0, s>>>(L[5].d, L[5].n, lc.sp);
}

void launch_pair(const LaunchCfg& lc, cudaStream_t s) {
    launch_pair_prec<false>(lc, s);
    launch_pair_prec<true>(lc, s);
    launch_pair_general(lc, s);
}

void launch_pair_fix(const LaunchCfg& lc, cudaStream_t s) {
    if (lc.any_near && lc.nsys > 0)
        k_pair_fix<<<lc.nsys * kFixBlocks, 256, 0, s>>>(lc.sys_list, lc.nsys, lc.sp);
}

} // namespace atvb
