// pair_general.cu -- the pair kernel for systems with per-type LJ tables
// and/or special (bonded) pairs.
//
// Per-type LJ: each type pair has its own sigma^6, epsilon and shift at the
// common cutoff (src/cpu/potentials/pair_lj_cut.cpp:255-298 table,
// :755-800 use); an epsilon of 0 (a type without an LJ site) contributes
// nothing.  Special pairs (LAMMPS special_bonds, special_scale.h): the row
// entry carries the pair's class (1-2, 1-3, 1-4) in its top two bits, set by
// the list build; the LJ force and shifted energy are multiplied by the
// class's LJ scale (pair_lj_cut.cpp:770-800), and the real-space Coulomb term
// keeps erfc but subtracts (1 - f) k_e q_i q_j / r, the share the
// reciprocal sum added for the pair (coul_long.cpp:159-196).
//
// Same data layout, precision forms and determinism as pair.cu (FP64: 64-bit
// fixed-point positions, FP64 math; mixed: 32-bit fixed-point positions,
// FP32 math, per-pair 64-bit fixed-point force sums), kGenLanes lanes per
// atom, the physics flags read at run time (these systems are the minority,
// so one kernel serves every combination).
#include "pair_math.cuh"

namespace atvb {

template <typename T>
struct GenConst {
    T lj_rc2, sig6, eps4, eps24, shift; // single-type LJ (ntypes == 0)
    T c_rc2, alpha, alpha2, kqi;
};

template <bool MIXED>
ATVB_DEV void row_general(const SysParams& P, int s, int g, PairAcc& acc) {
    using T = typename std::conditional<MIXED, float, double>::type;
    const int nn = P.nnbr[s];
    const unsigned* __restrict__ row =
        reinterpret_cast<const unsigned*>(P.nbr) + (size_t)s * P.cap;
    const bool lj = P.has_lj, co = P.has_coul, vir = P.need_virial;
    const int nt = P.ntypes;
    const int ti = nt ? (int)P.stype[s] : 0;
    double qi;
    int4 qi4 = make_int4(0, 0, 0, 0);
    double4 pi8 = make_double4(0, 0, 0, 0);
    if (MIXED) {
        qi4 = reinterpret_cast<const int4*>(P.pos4)[s];
        qi = (double)__int_as_float(qi4.w);
    } else {
        pi8 = reinterpret_cast<const double4*>(P.pos4)[s];
        qi = pi8.w;
    }
    GenConst<T> c;
    c.lj_rc2 = (T)P.lj_rc2;
    c.sig6 = (T)P.lj_sig6;
    c.eps4 = (T)P.lj_eps4;
    c.eps24 = (T)P.lj_eps24;
    c.shift = (T)P.lj_shift;
    c.c_rc2 = (T)P.coul_rc2;
    c.alpha = (T)P.coul_alpha;
    c.alpha2 = MIXED ? (T)(P.coul_alpha2 * 1.4426950408889634) : (T)P.coul_alpha2;
    c.kqi = (T)(kQqr2e * qi);
    RowSums<T> a;
    // software pipeline: the position of the next entry and the row entry
    // after it are loaded while the current pair computes (an entry past
    // the row end is the atom itself, never computed)
    using Pos = typename std::conditional<MIXED, int4, double4>::type;
    const Pos* __restrict__ pos = reinterpret_cast<const Pos*>(P.pos4);
    int k = g;
    unsigned raw = k < nn ? __ldg(row + k) : (unsigned)s;
    unsigned rawn = k + kGenLanes < nn ? __ldg(row + k + kGenLanes) : (unsigned)s;
    Pos pj = pos[raw & kRowIdxMask];
    for (; k < nn; k += kGenLanes) {
        const Pos pn = pos[rawn & kRowIdxMask];
        const unsigned rawnn =
            k + 2 * kGenLanes < nn ? __ldg(row + k + 2 * kGenLanes) : (unsigned)s;
        const int j = (int)(raw & kRowIdxMask);
        const int cls = (int)(raw >> 30);
        T dx, dy, dz, qj;
        if constexpr (MIXED) {
            dx = (T)((float)(int)((unsigned)qi4.x - (unsigned)pj.x) * P.Lf_fix[0]);
            dy = (T)((float)(int)((unsigned)qi4.y - (unsigned)pj.y) * P.Lf_fix[1]);
            dz = (T)((float)(int)((unsigned)qi4.z - (unsigned)pj.z) * P.Lf_fix[2]);
            qj = (T)__int_as_float(pj.w);
        } else {
            dx = (T)((double)(__double_as_longlong(pi8.x) - __double_as_longlong(pj.x)) * P.Lfix64[0]);
            dy = (T)((double)(__double_as_longlong(pi8.y) - __double_as_longlong(pj.y)) * P.Lfix64[1]);
            dz = (T)((double)(__double_as_longlong(pi8.z) - __double_as_longlong(pj.z)) * P.Lfix64[2]);
            qj = (T)pj.w;
        }
        raw = rawn;
        rawn = rawnn;
        pj = pn;
        const T r2 = dx * dx + dy * dy + dz * dz;
        const bool ok = r2 >= (T)kMinPair2;
        T rinv;
        if (MIXED)
            rinv = (T)rsqrt_approx((float)r2);
        else
            rinv = (T)rsqrt64((double)r2);
        const T r2inv = rinv * rinv;
        T fpair = 0;
        const T sl = cls ? (T)P.sp_lj[cls] : T(1); // 0: excluded from LJ
        if (lj && ok && r2 < c.lj_rc2 && sl != T(0)) {
            T sig6 = c.sig6, eps4 = c.eps4, eps24 = c.eps24, shift = c.shift;
            if (nt) {
                const int t = ti * nt + (int)P.stype[j];
                if (MIXED) {
                    const float4 p = reinterpret_cast<const float4*>(P.lj_tabf)[t];
                    sig6 = (T)p.x;
                    eps4 = (T)p.y;
                    eps24 = (T)p.z;
                    shift = (T)p.w;
                } else {
                    const double* p = P.lj_tab + 4 * t;
                    sig6 = (T)p[0];
                    eps4 = (T)p[1];
                    eps24 = (T)p[2];
                    shift = (T)p[3];
                }
            }
            const T r6 = r2inv * r2inv * r2inv * sig6;
            fpair = sl * eps24 * r2inv * r6 * (T(2) * r6 - T(1));
            a.elj += sl * (eps4 * r6 * (r6 - T(1)) - shift);
        }
        if (co && ok && r2 < c.c_rc2) {
            const T qq = c.kqi * qj;
            if (qq != T(0)) {
                const T x = c.alpha * (r2 * rinv);
                T t, e;
                if (MIXED) {
                    t = (T)rcp_approx(fmaf((float)kErfcxP, (float)x, 1.0f));
                    e = (T)ex2_approx((float)(-c.alpha2 * r2));
                } else {
                    t = (T)rcp64(fma(kErfcxP, (double)x, 1.0));
                    e = (T)exp_neg64((double)(c.alpha2 * r2));
                }
                const T p = erfcx_of_t(t);
                const T pref = qq * rinv;
                T fc = pref * e * (p + (T)kEwaldF * x);
                T ec = pref * e * p;
                if (cls) {
                    const T w = T(1) - (T)P.sp_coul[cls];
                    fc -= w * pref;
                    ec -= w * pref;
                }
                fpair += fc * r2inv;
                a.ec += ec;
            }
        }
        const T fxp = fpair * dx, fyp = fpair * dy, fzp = fpair * dz;
        if (MIXED) {
            a.fq[0] += __float2ll_rn((float)fxp * kForceFix);
            a.fq[1] += __float2ll_rn((float)fyp * kForceFix);
            a.fq[2] += __float2ll_rn((float)fzp * kForceFix);
        } else {
            a.fx += fxp;
            a.fy += fyp;
            a.fz += fzp;
        }
        if (vir) {
            a.v[0] += dx * fxp;
            a.v[1] += dy * fyp;
            a.v[2] += dz * fzp;
            a.v[3] += dx * fyp;
            a.v[4] += dx * fzp;
            a.v[5] += dy * fzp;
        }
    }
    finish_row(a, acc, vir);
}

template <bool MIXED>
__global__ void __launch_bounds__(256)
    k_pair_general(const Item* items, int nitems, const SysParams* sp) {
    __shared__ double sh[32 * 8];
    const int g = threadIdx.x % kGenLanes;
    const int a_off = threadIdx.x / kGenLanes;
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
        if (s < P.n)
            row_general<MIXED>(P, s, g, acc);
        double fx = acc.fx, fy = acc.fy, fz = acc.fz;
#pragma unroll
        for (int o = kGenLanes / 2; o > 0; o >>= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
        }
        if (g == 0 && s < P.n)
            P.f4[s] = make_double4(fx, fy, fz, 0.0);
        flush_energy(P, acc, sh);
    }
}

void launch_pair_general(const LaunchCfg& lc, cudaStream_t s) {
    if (lc.pair_gen[0].n)
        k_pair_general<false><<<lc.pair_gen[0].grid, 256, 0, s>>>(lc.pair_gen[0].d,
                                                                  lc.pair_gen[0].n, lc.sp);
    if (lc.pair_gen[1].n)
        k_pair_general<true><<<lc.pair_gen[1].grid, 256, 0, s>>>(lc.pair_gen[1].d,
                                                                 lc.pair_gen[1].n, lc.sp);
}

} // namespace atvb
