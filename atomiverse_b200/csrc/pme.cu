// pme.cu -- smooth-PME reciprocal sum: B-spline spread and force gather
// (the transforms and the influence function are in fft.cu).
//
// Math follows the reference's header-only PME
// (include/atomiverse/cpu/longrange/pme_spline.h:32-58 B-spline recursion,
// :124-210 fractional coordinates and spreading;
// include/atomiverse/cpu/longrange/pme_influence.h:159-199 influence with
// energy and virial, :217-280 force interpolation; src/cpu/longrange/
// pme.cpp:152-253 driver).  Differences of layout, not of math:
//  * the charge grid is accumulated in 64-bit fixed point, so the spread is
//    order-independent and bit-reproducible;
//  * the transforms (fft.cu, hand-written) are real-to-complex /
//    complex-to-real on the half grid (K0 x K1 x (K2/2+1)), with the
//    conversion of the fixed-point grid folded into the first pass and the
//    influence function (in fft.cu's x pass) between the forward
//    and inverse x transforms; the half-grid energy and virial weight every
//    mode with 0 < m2 < K2/2 twice;
//  * H(m) is evaluated on the fly from the per-axis B-spline moduli and the
//    current cell (no 3D table: a changing NPT cell needs no rebuild), and
//    the virial that the reference CUDA PME omits is produced from the same
//    pass.
#include "atvb_common.cuh"
#include "atvb_kernels.cuh"
#include "pair_math.cuh"

namespace atvb {

// pme_spline.h:32-58 (Essmann et al. 1995 appendix recursion)
template <int N, typename T>
ATVB_DEV void bspline_dev(T frac, T* th, T* dth) {
    th[N - 1] = T(0);
    th[1] = frac;
    th[0] = T(1) - frac;
#pragma unroll
    for (int k = 3; k < N; ++k) {
        const T div = T(1) / T(k - 1);
        th[k - 1] = div * frac * th[k - 2];
#pragma unroll
        for (int j = 1; j < k - 1; ++j)
            th[k - 1 - j] = div * ((frac + T(j)) * th[k - 2 - j] +
                                   (T(k - j) - frac) * th[k - 1 - j]);
        th[0] = div * (T(1) - frac) * th[0];
    }
    dth[0] = -th[0];
#pragma unroll
    for (int j = 1; j < N; ++j)
        dth[j] = th[j - 1] - th[j];
    const T div = T(1) / T(N - 1);
    th[N - 1] = div * frac * th[N - 2];
#pragma unroll
    for (int j = 1; j < N - 1; ++j)
        th[N - 1 - j] = div * ((frac + T(j)) * th[N - 2 - j] +
                               (T(N - j) - frac) * th[N - 1 - j]);
    th[0] = div * (T(1) - frac) * th[0];
}

ATVB_DEV int gwrap(int g, int K) {
    if (g >= K)
        g -= K;
    if (g < 0)
        g += K;
    return g;
}

// Grid base point of a floored fractional coordinate.  The modulo above can
// round up to exactly K for a coordinate just below zero, and a non-finite
// position floors to NaN: both map to an in-range point so a corrupted
// state produces garbage energies, never an out-of-bounds grid access.
ATVB_DEV int base_index(double u0, int K) {
    if (!(u0 >= 0.0))
        return 0;
    if (u0 >= (double)K)
        return u0 < 2.0 * K ? (int)(u0 - K) : 0;
    return (int)u0;
}

// Fractional grid coordinate, base point and B-spline weights of one atom.
template <bool MIXED, int N, typename T>
ATVB_DEV void atom_splines(const SysParams& P, int s, T th[3][N], T dth[3][N],
                           int base[3], double& q) {
    if (MIXED) {
        const int4 p = reinterpret_cast<const int4*>(P.pos4)[s];
        q = (double)__int_as_float(p.w);
        const unsigned u[3] = {(unsigned)p.x, (unsigned)p.y, (unsigned)p.z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // fixed-point position is the fractional coordinate * 2^32
            const double uu = (double)u[d] * ((double)P.K[d] * kEFixInv);
            const double u0 = floor(uu);
            base[d] = (int)u0;
            if (base[d] >= P.K[d])
                base[d] -= P.K[d];
            bspline_dev<N, T>((T)(uu - u0), th[d], dth[d]);
        }
    } else {
        const double4 p = reinterpret_cast<const double4*>(P.pos4)[s];
        q = p.w;
        const unsigned long long u[3] = {(unsigned long long)__double_as_longlong(p.x),
                                         (unsigned long long)__double_as_longlong(p.y),
                                         (unsigned long long)__double_as_longlong(p.z)};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // fixed-point position is the fractional coordinate * 2^64
            const double uu = (double)u[d] * ((double)P.K[d] * 5.421010862427522e-20);
            const double u0 = floor(uu);
            base[d] = base_index(u0, P.K[d]);
            bspline_dev<N, T>((T)(uu - u0), th[d], dth[d]);
        }
    }
}

// Lanes of one atom: N consecutive lanes, lane c owning the grid points at
// z offset c (so the lanes of an atom touch N consecutive grid points and a
// warp instruction's accesses fall in a few 32-byte sectors); 32 / N atoms
// per warp, the leftover lanes idle.
template <int N>
struct AtomLanes {
    static constexpr int per_warp = 32 / N;
    static constexpr int per_block = per_warp * (kChunk / 32);
    int c, g;        // z offset, atom within the block's pass
    bool on;         // the lane belongs to an atom group
    ATVB_DEV AtomLanes() {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        const int gw = lane / N;
        c = lane - gw * N;
        on = gw < per_warp;
        g = w * per_warp + gw;
    }
};

// The weights of lane c along z (th[2][c], dth[2][c]) selected without
// indexing the arrays by a run-time value.
template <int N, typename T>
ATVB_DEV void lane_z(const T (&th)[3][N], const T (&dth)[3][N], int c, T& t, T& d) {
    t = th[2][0];
    d = dth[2][0];
#pragma unroll
    for (int k = 1; k < N; ++k) {
        t = c == k ? th[2][k] : t;
        d = c == k ? dth[2][k] : d;
    }
}

// pme_spline.h:176-210: q theta_x theta_y theta_z into the fixed-point grid.
// Every contribution is formed exactly as (q th0[a]) th1[b] th2[c] and added
// as an integer, so the grid does not depend on the lane layout or order.
template <bool MIXED, int N>
__global__ void __launch_bounds__(kChunk)
    k_pme_spread(const Item* items, int nitems, const SysParams* sp) {
    using T = typename std::conditional<MIXED, float, double>::type;
    const AtomLanes<N> L;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (P.prec != (MIXED ? kMixed : kFP64))
            continue;
        for (int a0 = 0; a0 < kChunk; a0 += AtomLanes<N>::per_block) {
            const int s = item.begin + a0 + L.g;
            if (!L.on || a0 + L.g >= kChunk || s >= P.n)
                continue;
            T th[3][N], dth[3][N];
            int base[3];
            double q;
            atom_splines<MIXED, N, T>(P, s, th, dth, base, q);
            if (q == 0.0)
                continue;
            T t2, d2;
            lane_z<N, T>(th, dth, L.c, t2, d2);
            const int K0 = P.K[0], K1 = P.K[1], K2 = P.K[2];
            const double gs = P.grid_scale;
            const int b0 = base[0] - (N - 1), b1 = base[1] - (N - 1);
            const int g2 = gwrap(base[2] - (N - 1) + L.c, K2);
            unsigned long long* __restrict__ grid = P.grid_fix + g2;
#pragma unroll
            for (int a = 0; a < N; ++a) {
                const int g0 = gwrap(b0 + a, K0);
                const T wa = (T)q * th[0][a];
#pragma unroll
                for (int b = 0; b < N; ++b) {
                    const int g1 = gwrap(b1 + b, K1);
                    const T wab = wa * th[1][b];
                    const size_t plane = (size_t)K2 * (g1 + (size_t)K1 * g0);
                    const double w = (double)(wab * t2);
                    red_add_u64(grid + plane, (unsigned long long)__double2ll_rn(w * gs));
                }
            }
        }
    }
}

// pme_influence.h:217-280 (orthorhombic: inv_cell is diagonal).  One
// thread per atom, its N^3 grid reads all in flight at once: measured on
// the 192^3 mesh at 44 us (FP64) / 28 us (FP32), against 48-77 us / 45-47
// us when the lanes of an atom split the reads by z offset as the spread
// does (fewer reads in flight per thread, the splines computed per lane).
template <bool MIXED, int N>
__global__ void __launch_bounds__(256)
    k_pme_gather(const Item* items, int nitems, const SysParams* sp) {
    using T = typename std::conditional<MIXED, float, double>::type;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int s = item.begin + threadIdx.x;
        if (s >= P.n)
            continue;
        T th[3][N], dth[3][N];
        int base[3];
        double q;
        atom_splines<MIXED, N, T>(P, s, th, dth, base, q);
        double fx = 0, fy = 0, fz = 0;
        if (q != 0.0) {
            const int K0 = P.K[0], K1 = P.K[1], K2 = P.K[2];
            const int b0 = base[0] - (N - 1), b1 = base[1] - (N - 1),
                      b2 = base[2] - (N - 1);
            const T* __restrict__ grid = reinterpret_cast<const T*>(P.grid_real);
            T g0s = 0, g1s = 0, g2s = 0;
#pragma unroll
            for (int a = 0; a < N; ++a) {
                const int g0 = gwrap(b0 + a, K0);
#pragma unroll
                for (int b = 0; b < N; ++b) {
                    const int g1 = gwrap(b1 + b, K1);
                    const size_t plane = (size_t)K2 * (g1 + (size_t)K1 * g0);
                    const T txy = th[0][a] * th[1][b];
                    const T dxy = dth[0][a] * th[1][b];
                    const T xdy = th[0][a] * dth[1][b];
#pragma unroll
                    for (int c = 0; c < N; ++c) {
                        const int g2 = gwrap(b2 + c, K2);
                        const T cv = __ldg(grid + plane + g2);
                        g0s += cv * dxy * th[2][c];
                        g1s += cv * xdy * th[2][c];
                        g2s += cv * txy * dth[2][c];
                    }
                }
            }
            const double pref = -P.pme_fscale * q;
            fx = pref * ((double)g0s * P.K[0] * P.invL[0]);
            fy = pref * ((double)g1s * P.K[1] * P.invL[1]);
            fz = pref * ((double)g2s * P.K[2] * P.invL[2]);
        }
        // reciprocal-space forces go to their own buffer, so this chain can
        // run beside the pair kernel; the next atom pass adds them
        P.fp4[s] = make_double4(fx, fy, fz, 0.0);
    }
}

template <bool MIXED>
static void spread_order(const LaunchCfg& lc, cudaStream_t s) {
    const ItemList& il = lc.pme_atoms;
    switch (lc.pme_order) {
    case 3: k_pme_spread<MIXED, 3><<<il.grid, kChunk, 0, s>>>(il.d, il.n, lc.sp); break;
    case 4: k_pme_spread<MIXED, 4><<<il.grid, kChunk, 0, s>>>(il.d, il.n, lc.sp); break;
    case 5: k_pme_spread<MIXED, 5><<<il.grid, kChunk, 0, s>>>(il.d, il.n, lc.sp); break;
    case 6: k_pme_spread<MIXED, 6><<<il.grid, kChunk, 0, s>>>(il.d, il.n, lc.sp); break;
    case 7: k_pme_spread<MIXED, 7><<<il.grid, kChunk, 0, s>>>(il.d, il.n, lc.sp); break;
    default: k_pme_spread<MIXED, 8><<<il.grid, kChunk, 0, s>>>(il.d, il.n, lc.sp); break;
    }
}

template <bool MIXED>
static void gather_order(const LaunchCfg& lc, cudaStream_t s) {
    const ItemList& il = lc.pme_atoms;
    constexpr int T = kChunk;
    switch (lc.pme_order) {
    case 3: k_pme_gather<MIXED, 3><<<il.grid, T, 0, s>>>(il.d, il.n, lc.sp); break;
    case 4: k_pme_gather<MIXED, 4><<<il.grid, T, 0, s>>>(il.d, il.n, lc.sp); break;
    case 5: k_pme_gather<MIXED, 5><<<il.grid, T, 0, s>>>(il.d, il.n, lc.sp); break;
    case 6: k_pme_gather<MIXED, 6><<<il.grid, T, 0, s>>>(il.d, il.n, lc.sp); break;
    case 7: k_pme_gather<MIXED, 7><<<il.grid, T, 0, s>>>(il.d, il.n, lc.sp); break;
    default: k_pme_gather<MIXED, 8><<<il.grid, T, 0, s>>>(il.d, il.n, lc.sp); break;
    }
}

void launch_pme_spread(const LaunchCfg& lc, cudaStream_t s) {
    if (lc.pme_mixed)
        spread_order<true>(lc, s);
    else
        spread_order<false>(lc, s);
}

void launch_pme_gather(const LaunchCfg& lc, cudaStream_t s) {
    if (lc.pme_mixed)
        gather_order<true>(lc, s);
    else
        gather_order<false>(lc, s);
}

} // namespace atvb
