// fft.cu -- the PME grid transforms, hand-written: a 3D real-to-complex
// FFT, the influence function, and the complex-to-real inverse, in five
// passes over the grid.
//
// The reference transforms with FFTW (src/cpu/longrange/pme.cpp:105-108,
// 203-210) or cuFFT (src/cuda/longrange/pme.cu:293,330,334), unnormalised
// in both directions, between its spread and its gather.  The same
// transform here, on the half-complex grid K0 x K1 x (K2/2 + 1) (index
// m2 + Khp (m1 + K1 m0), rows padded to Khp, a multiple of 16), with the
// stages of the PME step folded in:
//   1. z forward (one block per line group): the 64-bit fixed-point charge
//      grid read, converted and cleared, real-to-complex along z;
//   2. y forward: complex FFT along y (tiles of a few m2 columns, loaded
//      coalesced and transposed into shared memory);
//   3. x forward, the influence function H(m) with the reciprocal energy
//      and virial (pme_influence.h:159-199), x inverse: one kernel;
//   4. y inverse;
//   5. z inverse, complex-to-real into the real grid the gather reads.
// Each line is transformed in shared memory by a mixed-radix Stockham
// (self-sorting) FFT with radices 4, 2, 3, 5, 7 -- every PME mesh size is
// 2,3,5,7-smooth (good_fft_size, pme_spline.h:99-111) -- and twiddles from
// a per-axis table of the K-th roots of unity computed on the host.  Real
// lines of even length go through the half-length complex FFT with the
// standard even/odd split; odd lengths through the full complex one.
#include "atvb_common.cuh"
#include "atvb_kernels.cuh"
#include "pair_math.cuh"

namespace atvb {

template <typename T>
struct Cplx;
template <>
struct Cplx<double> {
    using type = double2;
};
template <>
struct Cplx<float> {
    using type = float2;
};

template <typename T2>
ATVB_DEV T2 cmul(T2 a, T2 b) {
    T2 r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <typename T2>
ATVB_DEV T2 cadd(T2 a, T2 b) {
    T2 r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}
template <typename T2>
ATVB_DEV T2 csub(T2 a, T2 b) {
    T2 r;
    r.x = a.x - b.x;
    r.y = a.y - b.y;
    return r;
}
template <typename T2>
ATVB_DEV T2 cconj(T2 a) {
    a.y = -a.y;
    return a;
}
// a times -i (forward) or +i (inverse)
template <typename T2>
ATVB_DEV T2 cmul_mi(T2 a, bool inv) {
    T2 r;
    r.x = inv ? -a.y : a.y;
    r.y = inv ? a.x : -a.x;
    return r;
}

// cos and sin of 2 pi k / p for the generic radices (mathematical constants)
__device__ const double kCos5[5] = {1.0, 0.30901699437494745, -0.8090169943749475,
                                   -0.8090169943749475, 0.30901699437494745};
__device__ const double kSin5[5] = {0.0, 0.9510565162951535, 0.5877852522924731,
                                   -0.5877852522924731, -0.9510565162951535};
__device__ const double kCos7[7] = {1.0, 0.6234898018587336, -0.22252093395631434,
                                   -0.900968867902419, -0.900968867902419,
                                   -0.22252093395631434, 0.6234898018587336};
__device__ const double kSin7[7] = {0.0, 0.7818314824680298, 0.9749279121818236,
                                   0.43388373911755823, -0.43388373911755823,
                                   -0.9749279121818236, -0.7818314824680298};

// In-place P-point DFT of x[0..P) (sign -1 forward, +1 inverse); P is a
// compile-time constant, so x stays in registers.
template <typename T, typename T2, int P>
ATVB_DEV void small_dft(T2 (&x)[P], bool inv) {
    constexpr int p = P;
    if constexpr (P == 2) {
        const T2 a = x[0], b = x[1];
        x[0] = cadd(a, b);
        x[1] = csub(a, b);
    } else if constexpr (P == 4) {
        const T2 a = cadd(x[0], x[2]), b = csub(x[0], x[2]);
        const T2 c = cadd(x[1], x[3]), d = cmul_mi(csub(x[1], x[3]), inv);
        x[0] = cadd(a, c);
        x[2] = csub(a, c);
        x[1] = cadd(b, d);
        x[3] = csub(b, d);
    } else if constexpr (P == 3) {
        const T s3 = (T)0.8660254037844386; // sqrt(3) / 2
        const T2 s = cadd(x[1], x[2]);
        const T2 d = cmul_mi(csub(x[1], x[2]), inv);
        T2 m;
        m.x = x[0].x - (T)0.5 * s.x;
        m.y = x[0].y - (T)0.5 * s.y;
        x[0] = cadd(x[0], s);
        T2 e;
        e.x = s3 * d.x;
        e.y = s3 * d.y;
        x[1] = cadd(m, e);
        x[2] = csub(m, e);
    } else {
        // 5 or 7: the direct sum with the constant roots
        const double* cs = p == 5 ? kCos5 : kCos7;
        const double* sn = p == 5 ? kSin5 : kSin7;
        T2 y[P];
#pragma unroll
        for (int u = 0; u < p; ++u) {
            T2 acc = x[0];
#pragma unroll
            for (int t = 1; t < p; ++t) {
                const int k = (u * t) % p;
                T2 w;
                w.x = (T)cs[k];
                w.y = inv ? (T)sn[k] : -(T)sn[k];
                acc = cadd(acc, cmul(x[t], w));
            }
            y[u] = acc;
        }
#pragma unroll
        for (int u = 0; u < p; ++u)
            x[u] = y[u];
    }
}

// A walk over the cells of a rows x cols grid by the threads of a block,
// q = threadIdx.x, threadIdx.x + blockDim.x, ...: row and column kept up to
// date by additions (one division at the start, none per step).
struct Walk2 {
    int r, c, dr, dc, cols;
    ATVB_DEV Walk2(int q0, int cols_, int stride) : cols(cols_) {
        r = q0 / cols;
        c = q0 - r * cols;
        dr = stride / cols;
        dc = stride - dr * cols;
    }
    ATVB_DEV void next() {
        c += dc;
        r += dr;
        if (c >= cols) {
            c -= cols;
            ++r;
        }
    }
};

// One radix-P Stockham stage of every line: butterfly i of a line reads
// x_t = src[i + t m] (m = n / P), twiddles it by w^(t k) (k = i mod T, w
// the (P T)-th root), transforms, and writes dst[(i - k) P + k + u T].
// T divides m, so k follows i by additions as the walk wraps.
template <typename T, typename T2, int P>
ATVB_DEV void fft_stage(const T2* __restrict__ a, T2* __restrict__ b, int nlines, int n, int ls,
                        int Tsz, const T2* __restrict__ roots, int rs, bool inv) {
    const int m = n / P;
    const int step = rs * (n / (P * Tsz)); // root index per t * k
    Walk2 w(threadIdx.x, m, blockDim.x);
    int k = w.c % Tsz;
    const int dk = w.dc % Tsz;
    for (; w.r < nlines; w.next()) {
        const int i = w.c;
        const T2* src = a + w.r * ls;
        T2* dst = b + w.r * ls;
        T2 x[P];
        x[0] = src[i];
#pragma unroll
        for (int t = 1; t < P; ++t) {
            T2 tw = roots[t * k * step];
            if (inv)
                tw = cconj(tw);
            x[t] = cmul(src[i + t * m], tw);
        }
        small_dft<T, T2, P>(x, inv);
        const int j = (i - k) * P + k;
#pragma unroll
        for (int u = 0; u < P; ++u)
            dst[j + u * Tsz] = x[u];
        k += dk;
        k -= k >= Tsz ? Tsz : 0;
    }
}

// One transform of `nlines` lines of length n held in shared memory (line l
// at a + l * ls), by the whole block: Stockham stages, ping-ponging between
// a and b.  fac: the radices (shared memory); roots: the table of
// e^{-2 pi i j / (n rs)}, read with stride rs.  Returns the buffer that
// holds the result.
template <typename T, typename T2>
ATVB_DEV T2* fft_lines(T2* a, T2* b, int nlines, int n, int ls, const int* fac, int nf,
                       const T2* __restrict__ roots, int rs, bool inv) {
    int Tsz = 1;
    for (int f = 0; f < nf; ++f) {
        const int p = fac[f];
        switch (p) {
        case 4: fft_stage<T, T2, 4>(a, b, nlines, n, ls, Tsz, roots, rs, inv); break;
        case 2: fft_stage<T, T2, 2>(a, b, nlines, n, ls, Tsz, roots, rs, inv); break;
        case 3: fft_stage<T, T2, 3>(a, b, nlines, n, ls, Tsz, roots, rs, inv); break;
        case 5: fft_stage<T, T2, 5>(a, b, nlines, n, ls, Tsz, roots, rs, inv); break;
        default: fft_stage<T, T2, 7>(a, b, nlines, n, ls, Tsz, roots, rs, inv); break;
        }
        __syncthreads();
        T2* t = a;
        a = b;
        b = t;
        Tsz *= p;
    }
    return a;
}

// Line length (with padding against bank conflicts) of a transform of n.
ATVB_DEV int line_stride(int n) { return n + 1; }

// The roots of unity of one axis (K entries) into shared memory after the
// two line buffers; visible after the block's next barrier.
template <typename T2>
ATVB_DEV T2* stage_roots(T2* base, const T2* __restrict__ roots, int K) {
    for (int j = threadIdx.x; j < K; j += blockDim.x)
        base[j] = roots[j];
    return base;
}

// The radices of one axis into shared memory (read by every stage).
ATVB_DEV void load_fac(const SysParams& P, int axis, int* s_fac, int& nf) {
    nf = P.fft_nf[axis];
    if (threadIdx.x < kFftMaxFac)
        s_fac[threadIdx.x] = P.fft_fac[axis][threadIdx.x];
}

// ---- pass 1: z forward, from the fixed-point charge grid -----------------
// Every SysParams field a loop needs is read into a register first: the
// loops write through pointers the compiler cannot prove apart from the
// parameter table.
template <bool MIXED>
__global__ void __launch_bounds__(kFftBlock, 3)
    k_fft_zf(const Item* items, int nitems, const SysParams* sp, int C) {
    using T = typename std::conditional<MIXED, float, double>::type;
    using T2 = typename Cplx<T>::type;
    extern __shared__ unsigned char fsh_raw[];
    __shared__ int s_fac[kFftMaxFac];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.has_pme || P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int K0 = P.K[0], K1 = P.K[1], K2 = P.K[2], Kh = P.Kh, Khp = P.Khp;
        const bool even = (K2 & 1) == 0;
        const int n = even ? K2 / 2 : K2, ls = line_stride(n);
        const int l0 = item.begin, nl = min(C, K0 * K1 - l0);
        const double gsi = P.grid_scale_inv;
        unsigned long long* __restrict__ gf = P.grid_fix + (size_t)l0 * K2;
        T2* __restrict__ out = reinterpret_cast<T2*>(P.grid_cplx) + (size_t)l0 * Khp;
        int nf;
        load_fac(P, 2, s_fac, nf);
        T2* a = reinterpret_cast<T2*>(fsh_raw);
        T2* b = a + C * ls;
        const T2* roots = stage_roots(b + C * ls, reinterpret_cast<const T2*>(P.fft_root[2]), K2);
        // the group's lines are contiguous in the grid: one flat walk
        // (streaming loads, and the clear as a separate loop below: storing
        // into each element right after loading it measured 4x slower)
        for (Walk2 w(threadIdx.x, K2, blockDim.x); w.r < nl; w.next()) {
            const int c = w.r, z = w.c, q = c * K2 + z;
            const long long v = (long long)__ldcs(gf + q);
            const T x = (T)((double)v * gsi);
            if (even) {
                // x[2n], x[2n+1] interleave as z[n] = x[2n] + i x[2n+1]
                reinterpret_cast<T*>(a + c * ls)[z] = x;
            } else {
                T2 v2;
                v2.x = x;
                v2.y = (T)0;
                a[c * ls + z] = v2;
            }
        }
        __syncthreads();
        for (int q = threadIdx.x; q < nl * K2; q += blockDim.x)
            __stcs(gf + q, 0ull); // ready for the next spread
        T2* r = fft_lines<T, T2>(a, b, nl, n, ls, s_fac, nf, roots, even ? 2 : 1, false);
        for (Walk2 w(threadIdx.x, Kh, blockDim.x); w.r < nl; w.next()) {
            const int c = w.r, k = w.c;
            T2 X;
            if (even) {
                // X[k] = E + e^{-2 pi i k / K2} O, E/O the spectra of the
                // even / odd samples, from Z[k] and conj(Z[n - k])
                const T2 Zk = r[c * ls + (k == n ? 0 : k)];
                const T2 Zc = cconj(r[c * ls + (k == 0 ? 0 : n - k)]);
                T2 E, O;
                E.x = (T)0.5 * (Zk.x + Zc.x);
                E.y = (T)0.5 * (Zk.y + Zc.y);
                O.x = (T)0.5 * (Zk.y - Zc.y);
                O.y = -(T)0.5 * (Zk.x - Zc.x);
                X = cadd(E, cmul(O, roots[k]));
            } else {
                X = r[c * ls + k];
            }
            out[(size_t)c * Khp + k] = X;
        }
        __syncthreads();
    }
}

// ---- passes 2 and 4: y forward / inverse ---------------------------------
template <bool MIXED, bool INV>
__global__ void __launch_bounds__(kFftBlock, 3)
    k_fft_y(const Item* items, int nitems, const SysParams* sp, int C) {
    using T = typename std::conditional<MIXED, float, double>::type;
    using T2 = typename Cplx<T>::type;
    extern __shared__ unsigned char fsh_raw[];
    __shared__ int s_fac[kFftMaxFac];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.has_pme || P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int K1 = P.K[1], Kh = P.Kh, Khp = P.Khp;
        const int nb2 = (Kh + C - 1) / C;
        const int k0 = item.begin / nb2, m2a = (item.begin - k0 * nb2) * C;
        const int nc = min(C, Kh - m2a);
        const int ls = line_stride(K1);
        T2* __restrict__ g = reinterpret_cast<T2*>(P.grid_cplx) + (size_t)k0 * K1 * Khp + m2a;
        int nf;
        load_fac(P, 1, s_fac, nf);
        T2* a = reinterpret_cast<T2*>(fsh_raw);
        T2* b = a + C * ls;
        const T2* roots = stage_roots(b + C * ls, reinterpret_cast<const T2*>(P.fft_root[1]), K1);
        for (Walk2 w(threadIdx.x, nc, blockDim.x); w.r < K1; w.next())
            a[w.c * ls + w.r] = g[(size_t)w.r * Khp + w.c];
        __syncthreads();
        T2* r = fft_lines<T, T2>(a, b, nc, K1, ls, s_fac, nf, roots, 1, INV);
        for (Walk2 w(threadIdx.x, nc, blockDim.x); w.r < K1; w.next())
            g[(size_t)w.r * Khp + w.c] = r[w.c * ls + w.r];
        __syncthreads();
    }
}

// ---- pass 3: x forward, influence with energy and virial, x inverse ------
template <bool MIXED>
__global__ void __launch_bounds__(kFftBlock, 3)
    k_fft_x_infl(const Item* items, int nitems, const SysParams* sp, int C) {
    using T = typename std::conditional<MIXED, float, double>::type;
    using T2 = typename Cplx<T>::type;
    extern __shared__ unsigned char fsh_raw[];
    __shared__ int s_fac[kFftMaxFac];
    __shared__ double sh[32 * 7];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.has_pme || P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int K0 = P.K[0], K1 = P.K[1], K2 = P.K[2], Kh = P.Kh;
        const int nb2 = (Kh + C - 1) / C;
        const int m1 = item.begin / nb2, m2a = (item.begin - m1 * nb2) * C;
        const int nc = min(C, Kh - m2a);
        const int ls = line_stride(K0);
        const size_t sx = (size_t)K1 * P.Khp; // stride along x
        T2* __restrict__ g = reinterpret_cast<T2*>(P.grid_cplx) + (size_t)m1 * P.Khp + m2a;
        const double* __restrict__ bm = P.bmod;
        const double ilx = P.invL[0], ily = P.invL[1], ilz = P.invL[2];
        const double a2pi2 = P.pme_alpha2_pi2, escale = P.pme_escale;
        const bool vir = P.need_virial;
        unsigned long long* acc_st = P.st->acc;
        int nf;
        load_fac(P, 0, s_fac, nf);
        T2* a = reinterpret_cast<T2*>(fsh_raw);
        T2* b = a + C * ls;
        const T2* roots = stage_roots(b + C * ls, reinterpret_cast<const T2*>(P.fft_root[0]), K0);
        for (Walk2 w(threadIdx.x, nc, blockDim.x); w.r < K0; w.next())
            a[w.c * ls + w.r] = g[(size_t)w.r * sx + w.c];
        __syncthreads();
        T2* r = fft_lines<T, T2>(a, b, nc, K0, ls, s_fac, nf, roots, 1, false);
        // H(m) = exp(-pi^2 m^2 / alpha^2) / m^2 * B(m) (zero mode cleared,
        // pme_influence.h:112-155) from the current cell; energy and virial
        // with the half-grid weights (modes 0 < m2 < K2/2 stand for two)
        double acc[7] = {0, 0, 0, 0, 0, 0, 0};
        const int h1 = m1 <= K1 / 2 ? m1 : m1 - K1;
        const double my = h1 * ily;
        const double bmy = bm[K0 + m1];
        for (Walk2 w(threadIdx.x, K0, blockDim.x); w.r < nc; w.next()) {
            const int c = w.r, m0 = w.c;
            const int m2 = m2a + c;
            const int h0 = m0 <= K0 / 2 ? m0 : m0 - K0;
            const int h2 = m2 <= K2 / 2 ? m2 : m2 - K2;
            const double mx = h0 * ilx, mz = h2 * ilz;
            const double msq = mx * mx + my * my + mz * mz;
            const bool zero = m0 == 0 && m1 == 0 && m2 == 0;
            const double imsq = zero ? 0.0 : rcp64(msq);
            const double H = zero ? 0.0
                                  : exp_neg64(a2pi2 * msq) * imsq * (bm[m0] * bmy) *
                                        bm[K0 + K1 + m2];
            T2 Qm = r[c * ls + m0];
            const double re = (double)Qm.x, im = (double)Qm.y;
            const double wt = (m2 == 0 || 2 * m2 == K2) ? 1.0 : 2.0;
            const double ug = wt * H * (re * re + im * im);
            acc[0] += ug;
            if (vir && H != 0.0) {
                const double vt = -2.0 * (imsq + a2pi2);
                acc[1] += ug * (1.0 + vt * mx * mx);
                acc[2] += ug * (1.0 + vt * my * my);
                acc[3] += ug * (1.0 + vt * mz * mz);
                acc[4] += ug * (vt * mx * my);
                acc[5] += ug * (vt * mx * mz);
                acc[6] += ug * (vt * my * mz);
            }
            Qm.x = (T)(H * re);
            Qm.y = (T)(H * im);
            r[c * ls + m0] = Qm;
        }
        __syncthreads();
        T2* o = r == a ? b : a;
        T2* r2 = fft_lines<T, T2>(r, o, nc, K0, ls, s_fac, nf, roots, 1, true);
        for (Walk2 w(threadIdx.x, nc, blockDim.x); w.r < K0; w.next())
            g[(size_t)w.r * sx + w.c] = r2[w.c * ls + w.r];
        // per-item fixed-point flush (independent of batch composition)
        if (vir) {
            block_sum_vec<7>(acc, sh);
            if (threadIdx.x == 0) {
                fix_add(&acc_st[kAccERecip], acc[0] * escale);
                for (int k = 0; k < 6; ++k)
                    fix_add(&acc_st[kAccVir + k], acc[1 + k] * escale);
            }
        } else {
            double e1[1] = {acc[0]};
            block_sum_vec<1>(e1, sh);
            if (threadIdx.x == 0)
                fix_add(&acc_st[kAccERecip], e1[0] * escale);
        }
        __syncthreads();
    }
}

// ---- pass 5: z inverse, complex-to-real into the real grid ---------------
template <bool MIXED>
__global__ void __launch_bounds__(kFftBlock, 3)
    k_fft_zi(const Item* items, int nitems, const SysParams* sp, int C) {
    using T = typename std::conditional<MIXED, float, double>::type;
    using T2 = typename Cplx<T>::type;
    extern __shared__ unsigned char fsh_raw[];
    __shared__ int s_fac[kFftMaxFac];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.has_pme || P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int K0 = P.K[0], K1 = P.K[1], K2 = P.K[2], Kh = P.Kh;
        const bool even = (K2 & 1) == 0;
        const int n = even ? K2 / 2 : K2, ls = line_stride(n);
        const int l0 = item.begin, nl = min(C, K0 * K1 - l0);
        const int Khp = P.Khp;
        const T2* __restrict__ in = reinterpret_cast<const T2*>(P.grid_cplx) + (size_t)l0 * Khp;
        T* __restrict__ out = reinterpret_cast<T*>(P.grid_real) + (size_t)l0 * K2;
        int nf;
        load_fac(P, 2, s_fac, nf);
        T2* a = reinterpret_cast<T2*>(fsh_raw);
        T2* b = a + C * ls;
        const T2* roots = stage_roots(b + C * ls, reinterpret_cast<const T2*>(P.fft_root[2]), K2);
        __syncthreads();
        if (even) {
            // Z'[k] = (X[k] + conj X[n-k]) + i (X[k] - conj X[n-k]) e^{2 pi i k / K2}
            for (Walk2 w(threadIdx.x, n, blockDim.x); w.r < nl; w.next()) {
                const int c = w.r, k = w.c;
                const size_t row = (size_t)c * Khp;
                const T2 Xk = in[row + k];
                const T2 Xc = cconj(in[row + (n - k)]);
                const T2 E = cadd(Xk, Xc);
                const T2 O = cmul(csub(Xk, Xc), cconj(roots[k]));
                T2 Z;
                Z.x = E.x - O.y;
                Z.y = E.y + O.x;
                a[c * ls + k] = Z;
            }
        } else {
            // the full Hermitian spectrum
            for (Walk2 w(threadIdx.x, K2, blockDim.x); w.r < nl; w.next()) {
                const int c = w.r, k = w.c;
                const size_t row = (size_t)c * Khp;
                a[c * ls + k] = k < Kh ? in[row + k] : cconj(in[row + (K2 - k)]);
            }
        }
        __syncthreads();
        T2* r = fft_lines<T, T2>(a, b, nl, n, ls, s_fac, nf, roots, even ? 2 : 1, true);
        for (Walk2 w(threadIdx.x, K2, blockDim.x); w.r < nl; w.next()) {
            const int c = w.r, z = w.c;
            T v;
            if (even) {
                const T2 zz = r[c * ls + (z >> 1)];
                v = (z & 1) ? zz.y : zz.x;
            } else {
                v = r[c * ls + z].x;
            }
            out[(size_t)c * K2 + z] = v;
        }
        __syncthreads();
    }
}

// Two buffers of C lines (n + 1 each) and the K roots of unity.
static size_t fft_smem(int C, int n, int K, bool mixed) {
    return ((size_t)2 * C * (n + 1) + K) * (mixed ? sizeof(float2) : sizeof(double2));
}

// Each pass runs, per line length, its register form (fft_reg.cuh) where
// there is one, else the generic Stockham kernel above.
template <bool MIXED>
static void fft_pass(int pass, const std::vector<FftGroup>& gs, const SysParams* sp,
                     cudaStream_t s) {
    for (const FftGroup& g : gs) {
        if (g.items.n == 0)
            continue;
        if (g.reg >= 0) {
            launch_fft_reg(pass, g.reg, MIXED, g.items, sp, s);
            continue;
        }
        const size_t sm = fft_smem(g.c, g.n, g.k, MIXED);
        const ItemList& il = g.items;
        switch (pass) {
        case 0: k_fft_zf<MIXED><<<il.grid, kFftBlock, sm, s>>>(il.d, il.n, sp, g.c); break;
        case 1: k_fft_y<MIXED, false><<<il.grid, kFftBlock, sm, s>>>(il.d, il.n, sp, g.c); break;
        case 2: k_fft_x_infl<MIXED><<<il.grid, kFftBlock, sm, s>>>(il.d, il.n, sp, g.c); break;
        case 3: k_fft_y<MIXED, true><<<il.grid, kFftBlock, sm, s>>>(il.d, il.n, sp, g.c); break;
        default: k_fft_zi<MIXED><<<il.grid, kFftBlock, sm, s>>>(il.d, il.n, sp, g.c); break;
        }
    }
}

template <bool MIXED>
static void fft_all(const LaunchCfg& lc, cudaStream_t s) {
    const FftCfg& f = lc.fft;
    fft_pass<MIXED>(0, f.z, lc.sp, s);
    fft_pass<MIXED>(1, f.y, lc.sp, s);
    fft_pass<MIXED>(2, f.x, lc.sp, s);
    fft_pass<MIXED>(3, f.y, lc.sp, s);
    fft_pass<MIXED>(4, f.z, lc.sp, s);
}

void launch_pme_fft(const LaunchCfg& lc, cudaStream_t s) {
    if (lc.pme_mixed)
        fft_all<true>(lc, s);
    else
        fft_all<false>(lc, s);
}

// The most dynamic shared memory an FFT launch may ask for, opted in once
// per device (outside any stream capture).
void fft_smem_optin(int bytes) {
    auto set = [&](const void* f) {
        cuda_check(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
                   "cudaFuncSetAttribute(fft)");
    };
    set((const void*)k_fft_zf<false>);
    set((const void*)k_fft_zf<true>);
    set((const void*)k_fft_y<false, false>);
    set((const void*)k_fft_y<false, true>);
    set((const void*)k_fft_y<true, false>);
    set((const void*)k_fft_y<true, true>);
    set((const void*)k_fft_x_infl<false>);
    set((const void*)k_fft_x_infl<true>);
    set((const void*)k_fft_zi<false>);
    set((const void*)k_fft_zi<true>);
}

// Lines per block for a transform of length n with K roots: as many as fit
// kFftSmem bytes of shared memory, at most kFftMaxLines.
int fft_lines_per_block(int n, int K, bool mixed) {
    const size_t per = fft_smem(1, n, 0, mixed);
    const size_t roots = fft_smem(0, 0, K, mixed);
    int C = (int)((kFftSmem - roots) / per);
    C = C > kFftMaxLines ? kFftMaxLines : C;
    return C < 1 ? 1 : C;
}

} // namespace atvb
