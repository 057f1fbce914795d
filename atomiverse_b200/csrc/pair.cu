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
// FP64 build: positions double4 {x, y, z, q}, all arithmetic in double.
// Mixed build: positions int4 {x, y, z fixed point with 2^32 steps per box
// edge, q as float}; the integer difference is the exact minimum-image
// separation, converted once to float; pair math in FP32; per-row sums are
// promoted to FP64 before the lanes are combined.
#include "atvb_common.cuh"
#include "atvb_kernels.cuh"

namespace atvb {

constexpr double kMinPair2 = 1e-20; // lj_kernel.cuh:15 kMinPairDist^2

struct PairAcc {
    double fx, fy, fz, elj, ec;
    double v[6];
};

// erfcx(x) from the per-system piecewise polynomial held in shared memory
template <typename T, int NC>
ATVB_DEV T erfcx_poly(T x, T inv_h, int nint, const T* tab) {
    int k = (int)(x * inv_h);
    k = k < nint - 1 ? k : nint - 1;
    const T u = x * (T(2) * inv_h) - T(2 * k + 1);
    const T* c = tab + k * NC;
    T p = c[NC - 1];
#pragma unroll
    for (int d = NC - 2; d >= 0; --d)
        p = p * u + c[d];
    return p;
}

template <bool LJ, bool CO, bool VIR>
ATVB_DEV void row_fp64(const SysParams& P, int s, int g, int G, PairAcc& a,
                       const double* tab) {
    const double4* __restrict__ pos = reinterpret_cast<const double4*>(P.pos4);
    const double4 pi = pos[s];
    const int nn = P.nnbr[s];
    const int* __restrict__ row = P.nbr + (size_t)s * P.cap;
    const double L0 = P.L[0], L1 = P.L[1], L2 = P.L[2];
    const double i0 = P.invL[0], i1 = P.invL[1], i2 = P.invL[2];
    const double lj_rc2 = P.lj_rc2, sig6 = P.lj_sig6, eps4 = P.lj_eps4,
                 eps24 = P.lj_eps24, shift = P.lj_shift;
    const double c_rc2 = P.coul_rc2, alpha = P.coul_alpha,
                 alpha2 = P.coul_alpha2, inv_h = P.erfcx_inv_h;
    const int nint = P.erfcx_nint;
    const double kqi = kQqr2e * pi.w;
    double fx = 0, fy = 0, fz = 0, elj = 0, ec = 0;
    double v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
    for (int k = g; k < nn; k += G) {
        const int j = __ldg(row + k);
        const double4 pj = pos[j];
        const double dx = min_img(pi.x - pj.x, L0, i0);
        const double dy = min_img(pi.y - pj.y, L1, i1);
        const double dz = min_img(pi.z - pj.z, L2, i2);
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < kMinPair2)
            continue;
        const double rinv = rsqrt(r2);
        const double r2inv = rinv * rinv;
        double fpair = 0.0;
        if (LJ && r2 < lj_rc2) {
            const double r6inv = r2inv * r2inv * r2inv * sig6;
            fpair = eps24 * r2inv * (2.0 * r6inv * r6inv - r6inv);
            elj += eps4 * (r6inv * r6inv - r6inv) - shift;
        }
        if (CO && r2 < c_rc2) {
            const double qq = kqi * pj.w;
            if (qq != 0.0) {
                // erfc(x) = exp(-x^2) erfcx(x), x = alpha r
                const double x = alpha * (r2 * rinv);
                const double e = exp(-alpha2 * r2);
                const double ex = erfcx_poly<double, kErfcxNd>(x, inv_h, nint, tab);
                const double pref = qq * rinv;
                fpair += pref * e * (ex + kEwaldF * x) * r2inv;
                ec += pref * e * ex;
            }
        }
        const double fxp = fpair * dx, fyp = fpair * dy, fzp = fpair * dz;
        fx += fxp;
        fy += fyp;
        fz += fzp;
        if (VIR) {
            v0 += dx * fxp;
            v1 += dy * fyp;
            v2 += dz * fzp;
            v3 += dx * fyp;
            v4 += dx * fzp;
            v5 += dy * fzp;
        }
    }
    a.fx = fx;
    a.fy = fy;
    a.fz = fz;
    a.elj += elj;
    a.ec += ec;
    if (VIR) {
        a.v[0] += v0;
        a.v[1] += v1;
        a.v[2] += v2;
        a.v[3] += v3;
        a.v[4] += v4;
        a.v[5] += v5;
    }
}

template <bool LJ, bool CO, bool VIR>
ATVB_DEV void row_mixed(const SysParams& P, int s, int g, int G, PairAcc& a,
                        const float* tab) {
    const int4* __restrict__ pos = reinterpret_cast<const int4*>(P.pos4);
    const int4 pi = pos[s];
    const float qi = __int_as_float(pi.w);
    const int nn = P.nnbr[s];
    const int* __restrict__ row = P.nbr + (size_t)s * P.cap;
    const float sx = P.Lf_fix[0], sy = P.Lf_fix[1], sz = P.Lf_fix[2];
    const float lj_rc2 = (float)P.lj_rc2, sig6 = (float)P.lj_sig6,
                eps4 = (float)P.lj_eps4, eps24 = (float)P.lj_eps24,
                shift = (float)P.lj_shift;
    const float c_rc2 = (float)P.coul_rc2, alpha = (float)P.coul_alpha,
                alpha2 = (float)P.coul_alpha2, inv_h = (float)P.erfcx_inv_h;
    const int nint = P.erfcx_nint;
    const float kqi = (float)kQqr2e * qi, kf = (float)kEwaldF;
    float fx = 0, fy = 0, fz = 0, elj = 0, ec = 0;
    float v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
    for (int k = g; k < nn; k += G) {
        const int j = __ldg(row + k);
        const int4 pj = pos[j];
        const float dx = (float)(int)((unsigned)pi.x - (unsigned)pj.x) * sx;
        const float dy = (float)(int)((unsigned)pi.y - (unsigned)pj.y) * sy;
        const float dz = (float)(int)((unsigned)pi.z - (unsigned)pj.z) * sz;
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < 1e-20f)
            continue;
        const float r2inv = 1.0f / r2;
        float fpair = 0.0f;
        if (LJ && r2 < lj_rc2) {
            const float r6inv = r2inv * r2inv * r2inv * sig6;
            fpair = eps24 * r2inv * (2.0f * r6inv * r6inv - r6inv);
            elj += eps4 * (r6inv * r6inv - r6inv) - shift;
        }
        if (CO && r2 < c_rc2) {
            const float qq = kqi * __int_as_float(pj.w);
            if (qq != 0.0f) {
                const float rinv = rsqrtf(r2);
                const float x = alpha * (r2 * rinv);
                const float e = expf(-alpha2 * r2);
                const float ex = erfcx_poly<float, kErfcxNf>(x, inv_h, nint, tab);
                const float pref = qq * rinv;
                fpair += pref * e * (ex + kf * x) * r2inv;
                ec += pref * e * ex;
            }
        }
        const float fxp = fpair * dx, fyp = fpair * dy, fzp = fpair * dz;
        fx += fxp;
        fy += fyp;
        fz += fzp;
        if (VIR) {
            v0 += dx * fxp;
            v1 += dy * fyp;
            v2 += dz * fzp;
            v3 += dx * fyp;
            v4 += dx * fzp;
            v5 += dy * fzp;
        }
    }
    a.fx = fx;
    a.fy = fy;
    a.fz = fz;
    a.elj += elj;
    a.ec += ec;
    if (VIR) {
        a.v[0] += v0;
        a.v[1] += v1;
        a.v[2] += v2;
        a.v[3] += v3;
        a.v[4] += v4;
        a.v[5] += v5;
    }
}

template <bool MIXED, bool LJ, bool CO, bool VIR>
ATVB_DEV void row(const SysParams& P, int s, int g, int G, PairAcc& a,
                  const void* tab) {
    if (MIXED)
        row_mixed<LJ, CO, VIR>(P, s, g, G, a, (const float*)tab);
    else
        row_fp64<LJ, CO, VIR>(P, s, g, G, a, (const double*)tab);
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

template <bool MIXED, int G>
__global__ void __launch_bounds__(256)
    k_pair(const Item* items, int nitems, const SysParams* sp) {
    __shared__ double sh[32 * 8];
    __shared__ double tab[kErfcxMaxInt * kErfcxNd]; // erfcx of the current system
    int tab_sys = -1;
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
        if (P.has_coul && item.sys != tab_sys) { // block-uniform
            __syncthreads();
            const int nt = P.erfcx_nint * (MIXED ? kErfcxNf : kErfcxNd);
            if (MIXED) {
                float* tf = reinterpret_cast<float*>(tab);
                for (int k = threadIdx.x; k < nt; k += blockDim.x)
                    tf[k] = P.erfcx_f[k];
            } else {
                for (int k = threadIdx.x; k < nt; k += blockDim.x)
                    tab[k] = P.erfcx_d[k];
            }
            __syncthreads();
            tab_sys = item.sys;
        }
        const int s = item.begin + a_off;
        acc.fx = acc.fy = acc.fz = 0.0;
        if (s < P.n) {
            const bool lj = P.has_lj, co = P.has_coul, vr = P.need_virial;
            if (lj && co) {
                if (vr)
                    row<MIXED, true, true, true>(P, s, g, G, acc, tab);
                else
                    row<MIXED, true, true, false>(P, s, g, G, acc, tab);
            } else if (lj) {
                if (vr)
                    row<MIXED, true, false, true>(P, s, g, G, acc, tab);
                else
                    row<MIXED, true, false, false>(P, s, g, G, acc, tab);
            } else if (co) {
                if (vr)
                    row<MIXED, false, true, true>(P, s, g, G, acc, tab);
                else
                    row<MIXED, false, true, false>(P, s, g, G, acc, tab);
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

template <bool MIXED>
static void launch_pair_prec(const LaunchCfg& lc, cudaStream_t s) {
    const ItemList* L = lc.pair[MIXED ? 1 : 0];
    if (L[0].n)
        k_pair<MIXED, 1><<<L[0].grid, 256, 0, s>>>(L[0].d, L[0].n, lc.sp);
    if (L[1].n)
        k_pair<MIXED, 2><<<L[1].grid, 256, 0, s>>>(L[1].d, L[1].n, lc.sp);
    if (L[2].n)
        k_pair<MIXED, 4><<<L[2].grid, 256, 0, s>>>(L[2].d, L[2].n, lc.sp);
    if (L[3].n)
        k_pair<MIXED, 8><<<L[3].grid, 256, 0, s>>>(L[3].d, L[3].n, lc.sp);
    if (L[4].n)
        k_pair<MIXED, 16><<<L[4].grid, 256, 0, s>>>(L[4].d, L[4].n, lc.sp);
    if (L[5].n)
        k_pair<MIXED, 32><<<L[5].grid, 256, 0, s>>>(L[5].d, L[5].n, lc.sp);
}

void launch_pair(const LaunchCfg& lc, cudaStream_t s) {
    launch_pair_prec<false>(lc, s);
    launch_pair_prec<true>(lc, s);
}

} // namespace atvb
