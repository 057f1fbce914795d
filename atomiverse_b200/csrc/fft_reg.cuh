// fft_reg.cuh -- register-resident PME line transforms for the common mesh
// sizes.  A line of n = N1 x N2 points is transformed four-step style:
//   X[k1 + N1 k2] = sum_s w_N2^(s k2) [ w_n^(s k1) sum_e x[s + N2 e] w_N1^(e k1) ],
// so N2 threads each load N1 points x[s + N2 e] straight from the grid into
// registers and transform them (DFT-N1 fully unrolled, compile-time
// twiddles), multiply by w_n^(s k1), and pass them through shared memory
// once; N1 threads then each hold N2 values and finish with a register
// DFT-N2.  One shared-memory exchange per line instead of one per radix
// stage, and no shared-memory staging of the loads and stores.  The
// inverse transforms use conj(DFT(conj x)).  Same passes and the same
// folded stages (fixed-point grid conversion and clear, influence function
// with energy and virial, real/complex splits) as the generic kernels in
// fft.cu, which cover the mesh sizes without a register form.
#pragma once
#include <type_traits>

#include "atvb_common.cuh"
#include "atvb_kernels.cuh"
#include "pair_math.cuh"

namespace atvb {
namespace fftr {

// ---- roots of unity as compile-time constants ------------------------------
constexpr double kTwoPi = 6.283185307179586476925286766559005768;

__host__ __device__ constexpr double taylor_sin(double x) {
    double t = x, s = x;
    for (int k = 1; k < 14; ++k) {
        t *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        s += t;
    }
    return s;
}
__host__ __device__ constexpr double taylor_cos(double x) {
    double t = 1.0, s = 1.0;
    for (int k = 1; k < 14; ++k) {
        t *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        s += t;
    }
    return s;
}
// cos (which = 0) or sin (which = 1) of 2 pi a / b: the angle reduced to
// [0, pi/4] in exact integer arithmetic (2 pi - t, pi - t, pi/2 - t), then
// the Taylor series.
__host__ __device__ constexpr double turn_trig(long long a, long long b, int which) {
    a %= b;
    if (a < 0)
        a += b;
    double sc = 1.0, ss = 1.0;
    if (2 * a > b) { // 2 pi - t
        a = b - a;
        ss = -ss;
    }
    if (4 * a > b) { // pi - t
        a = b - 2 * a;
        b = 2 * b;
        sc = -sc;
    }
    bool swap = false;
    if (8 * a > b) { // pi / 2 - t
        a = b - 4 * a;
        b = 4 * b;
        swap = true;
    }
    const double t = kTwoPi * (double)a / (double)b;
    double c = taylor_cos(t), s = taylor_sin(t);
    if (swap) {
        const double u = c;
        c = s;
        s = u;
    }
    return which == 0 ? sc * c : ss * s;
}
template <long long A, long long N>
struct Trig {
    static constexpr double c = turn_trig(A, N, 0);
    static constexpr double s = turn_trig(A, N, 1);
};

// ---- small helpers ---------------------------------------------------------
template <typename T>
struct C2;
template <>
struct C2<double> {
    using type = double2;
};
template <>
struct C2<float> {
    using type = float2;
};

template <typename T2>
ATVB_DEV T2 mk(decltype(T2::x) x, decltype(T2::x) y) {
    T2 r;
    r.x = x;
    r.y = y;
    return r;
}
template <typename T2>
ATVB_DEV T2 add(T2 a, T2 b) { return mk<T2>(a.x + b.x, a.y + b.y); }
template <typename T2>
ATVB_DEV T2 sub(T2 a, T2 b) { return mk<T2>(a.x - b.x, a.y - b.y); }
template <typename T2>
ATVB_DEV T2 mul(T2 a, T2 b) { return mk<T2>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename T2>
ATVB_DEV T2 conj(T2 a) { return mk<T2>(a.x, -a.y); }

// A compile-time index usable in device code (std::integral_constant's
// conversion is host-only).
template <int I>
struct Ic {
    static constexpr int value = I;
    __host__ __device__ constexpr operator int() const { return I; }
};

// compile-time loop: f(Ic<i>) for i in [B, E)
template <int B, int E, typename F>
ATVB_DEV void sfor(F&& f) {
    if constexpr (B < E) {
        f(Ic<B>());
        sfor<B + 1, E>(f);
    }
}

// v * e^{-2 pi i A / N}, the quarter turns without multiplications
template <typename T, int A, int N, typename T2>
ATVB_DEV T2 mul_root(T2 v) {
    constexpr int a = ((A % N) + N) % N;
    if constexpr (a == 0) {
        return v;
    } else if constexpr (2 * a == N) {
        return mk<T2>(-v.x, -v.y);
    } else if constexpr (4 * a == N) {
        return mk<T2>(v.y, -v.x);
    } else if constexpr (4 * a == 3 * N) {
        return mk<T2>(-v.y, v.x);
    } else {
        constexpr T c = (T)Trig<a, N>::c;
        constexpr T s = (T)-Trig<a, N>::s;
        return mk<T2>(v.x * c - v.y * s, v.x * s + v.y * c);
    }
}

template <int N>
__host__ __device__ constexpr int first_factor() {
    return (N % 4 == 0 && N != 4) ? 4 : N % 2 == 0 ? 2 : N % 3 == 0 ? 3 : N % 5 == 0 ? 5 : 7;
}

// ---- forward DFT of N points held in registers -----------------------------
// X[k] = sum_j x[j] e^{-2 pi i j k / N}, in place, N a 2,3,5,7-smooth
// compile-time size (2, 4 and the odd primes directly, others four-step).
template <typename T, int N, typename T2>
ATVB_DEV void rdft(T2 (&x)[N]) {
    if constexpr (N == 1) {
    } else if constexpr (N == 2) {
        const T2 a = x[0], b = x[1];
        x[0] = add(a, b);
        x[1] = sub(a, b);
    } else if constexpr (N == 4) {
        const T2 a = add(x[0], x[2]), b = sub(x[0], x[2]);
        const T2 c = add(x[1], x[3]), d0 = sub(x[1], x[3]);
        const T2 d = mk<T2>(d0.y, -d0.x); // -i (x1 - x3)
        x[0] = add(a, c);
        x[2] = sub(a, c);
        x[1] = add(b, d);
        x[3] = sub(b, d);
    } else if constexpr (N == 3 || N == 5 || N == 7) {
        // pairs t, N - t: X[u] = x0 + sum a_t cos - i sum b_t sin,
        // X[N - u] the same with + i (a_t = x_t + x_{N-t}, b_t = x_t - x_{N-t})
        constexpr int H = (N - 1) / 2;
        T2 a[H + 1], b[H + 1], y[N];
        sfor<1, H + 1>([&](auto t) {
            a[t] = add(x[t], x[N - t]);
            b[t] = sub(x[t], x[N - t]);
        });
        T2 X0 = x[0];
        sfor<1, H + 1>([&](auto t) { X0 = add(X0, a[t]); });
        y[0] = X0;
        sfor<1, H + 1>([&](auto u) {
            T2 R = x[0], S = mk<T2>((T)0, (T)0);
            sfor<1, H + 1>([&](auto t) {
                constexpr int ut = (decltype(u)::value * decltype(t)::value) % N;
                constexpr T c = (T)Trig<ut, N>::c, s = (T)Trig<ut, N>::s;
                R.x += a[t].x * c;
                R.y += a[t].y * c;
                S.x += b[t].x * s;
                S.y += b[t].y * s;
            });
            y[u] = mk<T2>(R.x + S.y, R.y - S.x);
            y[N - u] = mk<T2>(R.x - S.y, R.y + S.x);
        });
        sfor<0, N>([&](auto k) { x[k] = y[k]; });
    } else {
        constexpr int N1 = first_factor<N>(), N2 = N / N1;
        T2 y[N1][N2];
        sfor<0, N2>([&](auto s) {
            T2 v[N1];
            sfor<0, N1>([&](auto e) { v[e] = x[s + N2 * e]; });
            rdft<T, N1>(v);
            sfor<0, N1>([&](auto k1) {
                y[k1][s] = mul_root<T, decltype(s)::value * decltype(k1)::value, N>(v[k1]);
            });
        });
        sfor<0, N1>([&](auto k1) {
            rdft<T, N2>(y[k1]);
            sfor<0, N2>([&](auto k2) { x[k1 + N1 * k2] = y[k1][k2]; });
        });
    }
}

// v[k] *= roots[k * step] for k = 1 .. N-1 (roots: a shared table)
template <int N, typename T2>
ATVB_DEV void twiddle(T2 (&v)[N], const T2* roots, int step) {
    int j = step;
    sfor<1, N>([&](auto k) {
        v[k] = mul(v[k], roots[j]);
        j += step;
    });
}

// ---- launch shapes -----------------------------------------------------------
// Column tiles of the y and x passes: 128 bytes of a grid row.
template <bool MIXED>
__host__ __device__ constexpr int cols() { return MIXED ? 16 : 8; }

// Blocks per SM the compiler must fit: a register budget per thread
// (measured on the 192^3 mesh: 128 for the x pass, 96 for y (64 in FP32,
// where a looser budget only buys registers the pass does not need), 80
// for z; tighter budgets spill and run slower).
__host__ __device__ constexpr int min_blocks(int threads, int regs) {
    return 65536 / (threads * regs) < 1 ? 1 : 65536 / (threads * regs) > 16 ? 16
                                                                          : 65536 / (threads * regs);
}

template <int N1, int N2>
struct Shape {
    static constexpr int n = N1 * N2;
    static constexpr int TL = N1 > N2 ? N1 : N2; // threads per line
    // one line's exchange area: N1 rows of N2 + 1 (then N2 rows of N1 + 1
    // in the x pass's inverse, n + 1 for the z pass's natural order), odd
    // so that the lines of a quarter warp fall in distinct banks
    static constexpr int SL0 = N1 * (N2 + 1) > N2 * (N1 + 1) ? N1 * (N2 + 1) : N2 * (N1 + 1);
    static constexpr int SL = SL0 | 1;
    template <bool MIXED>
    __host__ __device__ static constexpr int col_threads() {
        return (cols<MIXED>() * TL + 31) / 32 * 32;
    }
    // z pass: lines per block, 16 unless that passes 40 KB of exchange
    template <bool MIXED>
    __host__ __device__ static constexpr int zlines() {
        return 16 * SL * (MIXED ? 8 : 16) <= 40 * 1024 ? 16 : 8;
    }
    template <bool MIXED>
    __host__ __device__ static constexpr int z_threads() {
        return (zlines<MIXED>() * TL + 31) / 32 * 32;
    }
};

// Stage one axis' K roots of unity into shared memory (every item of a
// register launch has the same mesh size and precision).
template <typename T2>
ATVB_DEV void stage_roots(T2* sr, const void* roots, int K) {
    const T2* r = reinterpret_cast<const T2*>(roots);
    for (int j = threadIdx.x; j < K; j += blockDim.x)
        sr[j] = r[j];
}

// ---- pass 1: z forward from the fixed-point charge grid ---------------------
// Lines of K2 = 2 n real points as n complex points; the real spectrum from
// the even/odd split X[k] = E[k] + e^{-2 pi i k / K2} O[k].
template <int N1, int N2, bool MIXED>
__global__ void __launch_bounds__(Shape<N1, N2>::template z_threads<MIXED>(),
                                  min_blocks(Shape<N1, N2>::template z_threads<MIXED>(), 80))
    k_fftr_zf(const Item* items, int nitems, const SysParams* sp) {
    using T = typename std::conditional<MIXED, float, double>::type;
    using T2 = typename C2<T>::type;
    using S = Shape<N1, N2>;
    constexpr int n = S::n, K2 = 2 * n, L = S::template zlines<MIXED>(), SL = S::SL;
    __shared__ T2 sb[L * SL];
    __shared__ T2 sr[K2];
    if (blockIdx.x >= nitems)
        return;
    stage_roots(sr, sp[items[blockIdx.x].sys].fft_root[2], K2);
    __syncthreads();
    const int tid = threadIdx.x;
    const int la = tid / N2, s = tid - la * N2;  // loading role
    const int lb = tid / N1, k1 = tid - lb * N1; // finishing role
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.has_pme || P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int l0 = item.begin, nl = min(L, P.K[0] * P.K[1] - l0);
        const int Khp = P.Khp;
        if (la < nl) {
            const double gsi = P.grid_scale_inv;
            ulonglong2* src = reinterpret_cast<ulonglong2*>(P.grid_fix + (size_t)(l0 + la) * K2) + s;
            ulonglong2 raw[N1];
            sfor<0, N1>([&](auto e) { raw[e] = __ldcs(src + N2 * e); });
            T2 v[N1];
            sfor<0, N1>([&](auto e) {
                // z[j] = x[2j] + i x[2j+1]
                v[e] = mk<T2>((T)((double)(long long)raw[e].x * gsi),
                              (T)((double)(long long)raw[e].y * gsi));
            });
            rdft<T, N1>(v);
            twiddle(v, sr, 2 * s);
            sfor<0, N1>([&](auto q) { sb[la * SL + q * (N2 + 1) + s] = v[q]; });
            ulonglong2 zero;
            zero.x = zero.y = 0ull;
            sfor<0, N1>([&](auto e) { __stcs(src + N2 * e, zero); }); // ready for the next spread
        }
        __syncthreads();
        T2 w[N2];
        const bool fin = lb < nl;
        if (fin) {
            sfor<0, N2>([&](auto q) { w[q] = sb[lb * SL + k1 * (N2 + 1) + q]; });
            rdft<T, N2>(w); // Z[k1 + N1 k2] = w[k2]
        }
        __syncthreads();
        if (fin)
            sfor<0, N2>([&](auto k2) { sb[lb * SL + k1 + N1 * k2] = w[k2]; });
        __syncthreads();
        if (fin) {
            const T2* z = sb + lb * SL;
            T2* out = reinterpret_cast<T2*>(P.grid_cplx) + (size_t)(l0 + lb) * Khp;
            auto split = [&](int k, T2 Zk) {
                const T2 Zc = conj(z[k == 0 || k == n ? 0 : n - k]);
                const T2 E = mk<T2>((T)0.5 * (Zk.x + Zc.x), (T)0.5 * (Zk.y + Zc.y));
                const T2 O = mk<T2>((T)0.5 * (Zk.y - Zc.y), -(T)0.5 * (Zk.x - Zc.x));
                out[k] = add(E, mul(O, sr[k]));
            };
            sfor<0, N2>([&](auto k2) { split(k1 + N1 * k2, w[k2]); });
            if (k1 == 0)
                split(n, w[0]);
        }
        __syncthreads();
    }
}

// ---- passes 2 and 4: y forward / inverse -------------------------------------
template <int N1, int N2, bool MIXED, bool INV>
__global__ void __launch_bounds__(Shape<N1, N2>::template col_threads<MIXED>(),
                                  min_blocks(Shape<N1, N2>::template col_threads<MIXED>(),
                                             MIXED ? 64 : 96))
    k_fftr_y(const Item* items, int nitems, const SysParams* sp) {
    using T = typename std::conditional<MIXED, float, double>::type;
    using T2 = typename C2<T>::type;
    using S = Shape<N1, N2>;
    constexpr int n = S::n, CW = cols<MIXED>(), SL = S::SL;
    __shared__ T2 sb[CW * SL];
    __shared__ T2 sr[n];
    if (blockIdx.x >= nitems)
        return;
    stage_roots(sr, sp[items[blockIdx.x].sys].fft_root[1], n);
    __syncthreads();
    const int c = threadIdx.x % CW, q = threadIdx.x / CW;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.has_pme || P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int Kh = P.Kh, Khp = P.Khp;
        const int nb2 = (Kh + CW - 1) / CW;
        const int k0 = item.begin / nb2, m2a = (item.begin - k0 * nb2) * CW;
        const bool col = c < Kh - m2a;
        T2* g = reinterpret_cast<T2*>(P.grid_cplx) + (size_t)k0 * n * Khp + m2a + c;
        if (col && q < N2) {
            T2 v[N1];
            sfor<0, N1>([&](auto e) { v[e] = g[(size_t)(q + N2 * e) * Khp]; });
            if (INV)
                sfor<0, N1>([&](auto e) { v[e].y = -v[e].y; });
            rdft<T, N1>(v);
            twiddle(v, sr, q);
            sfor<0, N1>([&](auto k) { sb[c * SL + k * (N2 + 1) + q] = v[k]; });
        }
        __syncthreads();
        if (col && q < N1) {
            T2 w[N2];
            sfor<0, N2>([&](auto s) { w[s] = sb[c * SL + q * (N2 + 1) + s]; });
            rdft<T, N2>(w);
            if (INV)
                sfor<0, N2>([&](auto k) { w[k].y = -w[k].y; });
            sfor<0, N2>([&](auto k2) { g[(size_t)(q + N1 * k2) * Khp] = w[k2]; });
        }
        __syncthreads();
    }
}

// ---- pass 3: x forward, influence with energy and virial, x inverse ---------
// The inverse takes the forward's output distribution as its input: thread
// k1 holds m0 = k1 + N1 e', which is the four-step load of the (N2, N1)
// split, so the second transform needs one more exchange and no reload.
template <int N1, int N2, bool MIXED>
__global__ void __launch_bounds__(Shape<N1, N2>::template col_threads<MIXED>(),
                                  min_blocks(Shape<N1, N2>::template col_threads<MIXED>(), 128))
    k_fftr_x(const Item* items, int nitems, const SysParams* sp) {
    using T = typename std::conditional<MIXED, float, double>::type;
    using T2 = typename C2<T>::type;
    using S = Shape<N1, N2>;
    constexpr int n = S::n, CW = cols<MIXED>(), SL = S::SL;
    __shared__ T2 sb[CW * SL];
    __shared__ T2 sr[n];
    __shared__ double sx_tab[n]; // bmod[m0] exp(-pi^2 mx^2 / alpha^2)
    __shared__ double sh[32 * 7];
    if (blockIdx.x >= nitems)
        return;
    stage_roots(sr, sp[items[blockIdx.x].sys].fft_root[0], n);
    __syncthreads();
    const int c = threadIdx.x % CW, q = threadIdx.x / CW;
    int tab_sys = -1; // the system sx_tab was made for (one cell per step)
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.has_pme || P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int K1 = P.K[1], K2 = P.K[2], Kh = P.Kh, Khp = P.Khp;
        const int nb2 = (Kh + CW - 1) / CW;
        const int m1 = item.begin / nb2, m2a = (item.begin - m1 * nb2) * CW;
        const int m2 = m2a + c;
        const bool col = m2 < Kh;
        const size_t sx = (size_t)K1 * Khp;
        T2* g = reinterpret_cast<T2*>(P.grid_cplx) + (size_t)m1 * Khp + m2;
        const double* __restrict__ bm = P.bmod;
        const double ilx = P.invL[0], ily = P.invL[1], ilz = P.invL[2];
        const double a2pi2 = P.pme_alpha2_pi2;
        const bool vir = P.need_virial;
        // H(m) = exp(-pi^2 m^2 / alpha^2) / m^2 B(m) (pme_influence.h:112-155),
        // the Gaussian and B(m) split per axis: a table along x, one factor
        // per thread for y and z
        if (item.sys != tab_sys) { // uniform across the block
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                const int h0 = j <= n / 2 ? j : j - n;
                const double mx = h0 * ilx;
                sx_tab[j] = bm[j] * exp_neg64(a2pi2 * mx * mx);
            }
            tab_sys = item.sys;
        }
        const int h1 = m1 <= K1 / 2 ? m1 : m1 - K1;
        const int h2 = m2 <= K2 / 2 ? m2 : m2 - K2;
        const double my = h1 * ily, mz = h2 * ilz;
        const double myz2 = my * my + mz * mz;
        const double fyz = col ? bm[n + m1] * bm[n + K1 + m2] * exp_neg64(a2pi2 * myz2) : 0.0;
        const double wt = (m2 == 0 || 2 * m2 == K2) ? 1.0 : 2.0; // half-grid weights
        if (col && q < N2) {
            T2 v[N1];
            sfor<0, N1>([&](auto e) { v[e] = g[(size_t)(q + N2 * e) * sx]; });
            rdft<T, N1>(v);
            twiddle(v, sr, q);
            sfor<0, N1>([&](auto k) { sb[c * SL + k * (N2 + 1) + q] = v[k]; });
        }
        __syncthreads();
        double acc[7] = {0, 0, 0, 0, 0, 0, 0};
        T2 w[N2];
        const bool mid = col && q < N1;
        if (mid) {
            sfor<0, N2>([&](auto s) { w[s] = sb[c * SL + q * (N2 + 1) + s]; });
            rdft<T, N2>(w); // X[q + N1 k2] = w[k2]
            sfor<0, N2>([&](auto k2) {
                const int m0 = q + N1 * k2;
                const int h0 = m0 <= n / 2 ? m0 : m0 - n;
                const double mx = h0 * ilx;
                const double msq = mx * mx + myz2;
                const bool zero = m0 == 0 && m1 == 0 && m2 == 0;
                const double imsq = zero ? 0.0 : rcp64(msq);
                const double H = zero ? 0.0 : sx_tab[m0] * fyz * imsq;
                const double re = (double)w[k2].x, im = (double)w[k2].y;
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
                // the inverse as conj(DFT(conj(H X)))
                w[k2] = mk<T2>((T)(H * re), (T)(-H * im));
            });
            rdft<T, N2>(w); // the (N2, N1) split: this thread is s' = q
            twiddle(w, sr, q);
        }
        __syncthreads();
        if (mid)
            sfor<0, N2>([&](auto k) { sb[c * SL + k * (N1 + 1) + q] = w[k]; });
        __syncthreads();
        if (col && q < N2) {
            T2 z[N1];
            sfor<0, N1>([&](auto s) { z[s] = sb[c * SL + q * (N1 + 1) + s]; });
            rdft<T, N1>(z);
            sfor<0, N1>([&](auto k2) { g[(size_t)(q + N2 * k2) * sx] = conj(z[k2]); });
        }
        // per-item fixed-point flush (independent of batch composition)
        unsigned long long* acc_st = P.st->acc;
        const double escale = P.pme_escale;
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

// ---- pass 5: z inverse, complex-to-real into the real grid ------------------
// Z'[j] = (X[j] + conj X[n-j]) + i (X[j] - conj X[n-j]) e^{2 pi i j / K2},
// then the complex inverse of length n; z[j] = x[2j] + i x[2j+1].
template <int N1, int N2, bool MIXED>
__global__ void __launch_bounds__(Shape<N1, N2>::template z_threads<MIXED>(),
                                  min_blocks(Shape<N1, N2>::template z_threads<MIXED>(), 80))
    k_fftr_zi(const Item* items, int nitems, const SysParams* sp) {
    using T = typename std::conditional<MIXED, float, double>::type;
    using T2 = typename C2<T>::type;
    using S = Shape<N1, N2>;
    constexpr int n = S::n, K2 = 2 * n, L = S::template zlines<MIXED>(), SL = S::SL;
    __shared__ T2 sb[L * SL];
    __shared__ T2 sr[K2];
    if (blockIdx.x >= nitems)
        return;
    stage_roots(sr, sp[items[blockIdx.x].sys].fft_root[2], K2);
    __syncthreads();
    const int tid = threadIdx.x;
    const int la = tid / N2, s = tid - la * N2;
    const int lb = tid / N1, k1 = tid - lb * N1;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.has_pme || P.prec != (MIXED ? kMixed : kFP64))
            continue;
        const int l0 = item.begin, nl = min(L, P.K[0] * P.K[1] - l0);
        const int Khp = P.Khp;
        if (la < nl) {
            const T2* in = reinterpret_cast<const T2*>(P.grid_cplx) + (size_t)(l0 + la) * Khp;
            T2 v[N1];
            sfor<0, N1>([&](auto e) {
                const int j = s + N2 * e;
                const T2 Xj = in[j];
                const T2 Xc = conj(in[n - j]);
                const T2 E = add(Xj, Xc);
                const T2 O = mul(sub(Xj, Xc), conj(sr[j]));
                v[e] = mk<T2>(E.x - O.y, -(E.y + O.x)); // conj(E + i O)
            });
            rdft<T, N1>(v);
            twiddle(v, sr, 2 * s);
            sfor<0, N1>([&](auto q) { sb[la * SL + q * (N2 + 1) + s] = v[q]; });
        }
        __syncthreads();
        if (lb < nl) {
            T2 w[N2];
            sfor<0, N2>([&](auto q) { w[q] = sb[lb * SL + k1 * (N2 + 1) + q]; });
            rdft<T, N2>(w);
            T2* out = reinterpret_cast<T2*>(P.grid_real) + (size_t)(l0 + lb) * n;
            sfor<0, N2>([&](auto k2) { out[k1 + N1 * k2] = conj(w[k2]); });
        }
        __syncthreads();
    }
}

// Line lengths with a register form, as (index, n, N1, N2): every
// 2,3,5,7-smooth n from 8 to 256 that splits into N1, N2 <= 16 (the most
// balanced split, N2 a power of two on ties), in two halves compiled by
// separate units.
#define ATVB_FFTR_SIZES_A(X) \
    X(0, 8, 2, 4) X(1, 9, 3, 3) X(2, 10, 5, 2) X(3, 12, 3, 4) X(4, 14, 7, 2)           \
    X(5, 15, 3, 5) X(6, 16, 4, 4) X(7, 18, 3, 6) X(8, 20, 5, 4) X(9, 21, 3, 7)         \
    X(10, 24, 6, 4) X(11, 25, 5, 5) X(12, 27, 3, 9) X(13, 28, 7, 4) X(14, 30, 5, 6)    \
    X(15, 32, 4, 8) X(16, 35, 5, 7) X(17, 36, 6, 6) X(18, 40, 5, 8) X(19, 42, 6, 7)    \
    X(20, 45, 5, 9) X(21, 48, 6, 8) X(22, 49, 7, 7) X(23, 50, 5, 10) X(24, 54, 6, 9)   \
    X(25, 56, 7, 8) X(26, 60, 6, 10) X(27, 63, 7, 9) X(28, 64, 8, 8)
#define ATVB_FFTR_SIZES_B(X) \
    X(29, 70, 7, 10) X(30, 72, 9, 8) X(31, 75, 5, 15) X(32, 80, 10, 8)                 \
    X(33, 81, 9, 9) X(34, 84, 7, 12) X(35, 90, 9, 10) X(36, 96, 12, 8)                 \
    X(37, 98, 7, 14) X(38, 100, 10, 10) X(39, 105, 7, 15) X(40, 108, 9, 12)            \
    X(41, 112, 14, 8) X(42, 120, 10, 12) X(43, 126, 9, 14) X(44, 128, 8, 16)           \
    X(45, 135, 9, 15) X(46, 140, 10, 14) X(47, 144, 12, 12) X(48, 150, 10, 15)         \
    X(49, 160, 10, 16) X(50, 168, 12, 14) X(51, 180, 12, 15) X(52, 192, 12, 16)        \
    X(53, 196, 14, 14) X(54, 210, 14, 15) X(55, 224, 14, 16) X(56, 225, 15, 15)        \
    X(57, 240, 15, 16) X(58, 256, 16, 16)
#define ATVB_FFTR_SIZES(X) ATVB_FFTR_SIZES_A(X) ATVB_FFTR_SIZES_B(X)

// One pass of the register form <N1, N2> over the items of `il`.
template <int N1, int N2, bool MIXED>
void launch_pass(int pass, const ItemList& il, const SysParams* sp, cudaStream_t s) {
    using S = Shape<N1, N2>;
    constexpr int zt = S::template z_threads<MIXED>(), ct = S::template col_threads<MIXED>();
    switch (pass) {
    case 0: k_fftr_zf<N1, N2, MIXED><<<il.grid, zt, 0, s>>>(il.d, il.n, sp); break;
    case 1: k_fftr_y<N1, N2, MIXED, false><<<il.grid, ct, 0, s>>>(il.d, il.n, sp); break;
    case 2: k_fftr_x<N1, N2, MIXED><<<il.grid, ct, 0, s>>>(il.d, il.n, sp); break;
    case 3: k_fftr_y<N1, N2, MIXED, true><<<il.grid, ct, 0, s>>>(il.d, il.n, sp); break;
    default: k_fftr_zi<N1, N2, MIXED><<<il.grid, zt, 0, s>>>(il.d, il.n, sp); break;
    }
}

#define ATVB_FFTR_CASE(i, len, a, b)                                                    \
    case i: launch_pass<a, b, MIXED>(pass, il, sp, s); return true;

// The launch of form `idx` if it is in the first (second) half of the table.
template <bool MIXED>
bool launch_half_a(int pass, int idx, const ItemList& il, const SysParams* sp, cudaStream_t s) {
    switch (idx) {
        ATVB_FFTR_SIZES_A(ATVB_FFTR_CASE)
    default: return false;
    }
}
template <bool MIXED>
bool launch_half_b(int pass, int idx, const ItemList& il, const SysParams* sp, cudaStream_t s) {
    switch (idx) {
        ATVB_FFTR_SIZES_B(ATVB_FFTR_CASE)
    default: return false;
    }
}
#undef ATVB_FFTR_CASE

} // namespace fftr
} // namespace atvb
