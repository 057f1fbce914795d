// engine.cu -- host side of the path: device allocation per system, the
// system table and work lists, the per-step CUDA graph, and the C ABI.
//
// The reference drives one system per cuda::md::MD through Backend::step
// (src/cuda/driver/driver.cu:123-157), which walks ten phases and launches
// every component kernel from the host each step.  Here a step is one CUDA
// graph launch: the phase order is fixed at capture time and the neighbour
// rebuild decision is taken on the device (k_sys_a), so the loop has no
// host synchronisation.  An Engine holds any number of systems; the
// single-system API is an Engine with one slot, the batch API an Engine
// with many, and the server an Engine whose slots come and go.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "atvb.h"
#include "atvb_common.cuh"
#include "atvb_engine.h"
#include "box.cuh"
#include "erfcx_coef.h"
#include "atvb_kernels.cuh"

namespace atvb {

thread_local std::string g_last_error;

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw Error(ATVB_ERR_CUDA, std::string(what) + ": " +
                                       cudaGetErrorString(e));
}
#define CK(x) cuda_check((x), #x)

// ---------------------------------------------------------------- helpers

static int round_up(long long v, int m) {
    return (int)(((v + m - 1) / m) * m);
}

// pme_spline.h:99-111
int good_fft_size(int n) {
    if (n < 4)
        n = 4;
    for (;; ++n) {
        int m = n;
        for (int p : {2, 3, 5, 7})
            while (m % p == 0)
                m /= p;
        if (m == 1)
            return n;
    }
}

// pme_spline.h:32-58 (host copy for the moduli)
static void bspline_host(double frac, int n, double* th, double* dth) {
    th[n - 1] = 0.0;
    th[1] = frac;
    th[0] = 1.0 - frac;
    for (int k = 3; k < n; ++k) {
        const double div = 1.0 / (k - 1);
        th[k - 1] = div * frac * th[k - 2];
        for (int j = 1; j < k - 1; ++j)
            th[k - 1 - j] = div * ((frac + j) * th[k - 2 - j] +
                                   (k - j - frac) * th[k - 1 - j]);
        th[0] = div * (1.0 - frac) * th[0];
    }
    dth[0] = -th[0];
    for (int j = 1; j < n; ++j)
        dth[j] = th[j - 1] - th[j];
    const double div = 1.0 / (n - 1);
    th[n - 1] = div * frac * th[n - 2];
    for (int j = 1; j < n - 1; ++j)
        th[n - 1 - j] = div * ((frac + j) * th[n - 2 - j] +
                               (n - j - frac) * th[n - 1 - j]);
    th[0] = div * (1.0 - frac) * th[0];
}

// pme_spline.h:67-94
static std::vector<double> spline_moduli(int K, int n) {
    std::vector<double> data(n), dd(n), mod(K);
    bspline_host(0.0, n, data.data(), dd.data());
    for (int i = 0; i < K; ++i) {
        double sr = 0, si = 0;
        for (int k = 0; k < n - 1; ++k) {
            const double arg = 2.0 * kPi * i * k / K;
            sr += data[k] * std::cos(arg);
            si += data[k] * std::sin(arg);
        }
        const double den = sr * sr + si * si;
        mod[i] = den > 1e-12 ? 1.0 / den : 0.0;
    }
    for (int i = 0; i < K; ++i)
        if (mod[i] == 0.0)
            mod[i] = 0.5 * (mod[(i - 1 + K) % K] + mod[(i + 1) % K]);
    return mod;
}


// ------------------------------------------------------------ geometry

// `shrink` > 0 (MTK NPT): plan the bins and stencil for every cell down to
// L (1 - shrink) per axis, so that the grid stays valid while the cell
// breathes; the bins then grow with the cell (bin count fixed).
Geometry make_geometry(const atvb_system_desc& d, double shrink) {
    Geometry g;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            if (r != c && d.box[3 * r + c] != 0.0)
                throw Error(ATVB_ERR_INVALID,
                            "only orthorhombic boxes are supported "
                            "(off-diagonal cell entries must be 0)");
    for (int k = 0; k < 3; ++k) {
        g.L[k] = d.box[4 * k];
        if (!(g.L[k] > 0.0))
            throw Error(ATVB_ERR_INVALID, "box edges must be positive");
    }
    if (d.n_atoms < 1)
        throw Error(ATVB_ERR_INVALID, "n_atoms must be >= 1");
    if (!(d.nl_cutoff > 0.0))
        throw Error(ATVB_ERR_INVALID, "NeighborList: cutoff must be > 0");
    // neighbor_list.cuh:98: skin < 0 means 0.3 * cutoff
    g.skin = d.nl_skin < 0.0 ? 0.3 * d.nl_cutoff : d.nl_skin;
    g.rlist = d.nl_cutoff + g.skin;
    for (int k = 0; k < 3; ++k)
        if (!(g.L[k] > 2.0 * g.rlist))
            throw Error(ATVB_ERR_INVALID,
                        "box edge must exceed 2*(cutoff+skin) so that each "
                        "pair has one minimum image");
    double Lp[3];
    for (int k = 0; k < 3; ++k) {
        Lp[k] = g.L[k] * (1.0 - shrink);
        g.Lmin[k] = Lp[k];
    }
    // Bins of at least rlist / reach.  Reach 3 (finer than the reference's
    // half-reach bins, cell_list.cpp:112-121, reach :186-191) gives the
    // fewest candidates per atom, but the list kernel spends a warp per bin
    // and resolves the stencil per bin, so bins must hold enough atoms to
    // amortise that: reach 3 from 5 atoms per bin, else reach 2 from 1.5,
    // else reach 1 (measured: the 262k-ion melt builds fastest at reach 2,
    // 12 ions per bin; reduced-unit LJ at reach 2, 2.3 atoms per bin).
    // The pair set does not depend on the bins.
    const double density = d.n_atoms / (Lp[0] * Lp[1] * Lp[2]);
    auto per_bin = [&](double reach) { return density * std::pow(g.rlist / reach, 3.0); };
    const double reach_t = per_bin(3.0) >= 5.0 ? 3.0 : (per_bin(2.0) >= 1.5 ? 2.0 : 1.0);
    for (int k = 0; k < 3; ++k) {
        int c = (int)std::floor(Lp[k] / (g.rlist / reach_t));
        g.nc[k] = c < 1 ? 1 : c;
        g.cs[k] = Lp[k] / g.nc[k];
        int r = (int)std::ceil(g.rlist / g.cs[k] - 1e-12);
        g.reach[k] = r < 1 ? 1 : r;
        g.alias[k] = g.nc[k] < 2 * g.reach[k] + 1;
    }
    // Stencil columns: every (dx, dy) whose prism can hold a pair, with the
    // z reach that the LAMMPS bin-distance rule (cell_list.cpp:199-209)
    // allows.  An aliased axis visits each of its cells exactly once.
    const double rl2 = g.rlist * g.rlist;
    auto axis_offsets = [&](int k) {
        std::vector<int> o;
        if (g.alias[k]) {
            for (int v = 0; v < g.nc[k]; ++v)
                o.push_back(v);
        } else {
            for (int v = -g.reach[k]; v <= g.reach[k]; ++v)
                o.push_back(v);
        }
        return o;
    };
    auto gap = [&](int k, int v) -> double {
        if (g.alias[k])
            return 0.0;
        const int a = v < 0 ? -v : v;
        return a == 0 ? 0.0 : (a - 1) * g.cs[k];
    };
    for (int dx : axis_offsets(0))
        for (int dy : axis_offsets(1)) {
            const double gx = gap(0, dx), gy = gap(1, dy);
            if (gx * gx + gy * gy > rl2)
                continue;
            int m;
            if (g.alias[2]) {
                m = -1;
            } else {
                m = 0;
                for (int dz = 1; dz <= g.reach[2]; ++dz) {
                    const double gz = gap(2, dz);
                    if (gx * gx + gy * gy + gz * gz <= rl2)
                        m = dz;
                }
            }
            g.cols.push_back(make_int4(dx, dy, m, 0));
        }
    return g;
}

static int pme_K(const atvb_system_desc& d, const Geometry& g, int k) {
    if (d.pme_grid[k] > 0)
        return d.pme_grid[k];
    if (!(d.pme_grid_spacing > 0.0))
        throw Error(ATVB_ERR_INVALID, "KSpacePME: grid_spacing must be > 0");
    // pme.cpp:69-76
    int K = good_fft_size((int)std::ceil(g.L[k] / d.pme_grid_spacing));
    if (K < d.pme_order + 1)
        K = good_fft_size(d.pme_order + 1);
    return K;
}

static int expected_row(const atvb_system_desc& d, const Geometry& g) {
    const double vol = g.L[0] * g.L[1] * g.L[2];
    const double rho = d.n_atoms / vol;
    const double nb = rho * 4.0 / 3.0 * kPi * g.rlist * g.rlist * g.rlist;
    int cap = round_up((long long)(1.5 * nb + 64.0), 32);
    const int nmax = round_up(d.n_atoms, 32);
    return std::min(cap, std::max(nmax, 32));
}

size_t estimate_bytes(const atvb_system_desc& d) {
    Geometry g = make_geometry(d);
    const size_t n = (size_t)d.n_atoms;
    const int cap = expected_row(d, g);
    size_t b = n * (14 * 8 + 8 + 32 + 32 + 6 * 4 + (size_t)cap * 4);
    if (d.precision == ATVB_MIXED)
        b += n * 16;
    b += (size_t)(g.nc[0] * g.nc[1] * g.nc[2] + 1) * 8;
    b += sizeof(SysState) + 3 * 8 * 4096;
    if (d.pme_enabled) {
        const size_t K0 = pme_K(d, g, 0), K1 = pme_K(d, g, 1),
                     K2 = pme_K(d, g, 2);
        const size_t nt = K0 * K1 * K2, nh = K0 * K1 * ((K2 / 2 + 1 + 15) / 16 * 16);
        const size_t rs = d.precision == ATVB_MIXED ? 4 : 8;
        b += nt * 8 + nt * rs + nh * 2 * rs + (K0 + K1 + K2) * 8;
        b += (K0 + K1 + K2) * 2 * rs; // roots of unity of the transforms
    }
    return b;
}

// --------------------------------------------------------------- Slot

// The smallest separation at which no pair force of a mixed-precision
// system can reach 2^21 eV/A (its row sums are 64-bit fixed point in units
// of 2^-32 eV/A, range 2^31 eV/A; 2^21 keeps any row of up to 1,024 such
// pairs in range), from the LJ parameters and the largest charge product
// (an upper bound of the real-space Coulomb force).  Bisection on the
// repulsive branch.  A closer pair raises kStatusForceRange.
static double force_safe_r2(const SysParams& hp, double qq_max) {
    if (hp.prec != kMixed)
        return 0.0;
    const double lim = 2097152.0;
    auto fmax = [&](double r) {
        double f = 0.0;
        if (hp.has_lj) {
            const double r2inv = 1.0 / (r * r);
            const double r6 = hp.lj_sig6 * r2inv * r2inv * r2inv;
            f += std::fabs(hp.lj_eps24 * r2inv * r6 * (2.0 * r6 - 1.0)) * r;
        }
        if (hp.has_coul)
            f += kQqr2e * qq_max * (1.0 / (r * r) + kEwaldF * hp.coul_alpha / r);
        return f;
    };
    double lo = 1e-9, hi = hp.rlist;
    if (!(fmax(hi) < lim))
        return hi * hi; // every listed pair may exceed it: all are flagged
    if (fmax(lo) < lim)
        return 0.0;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (fmax(mid) >= lim)
            lo = mid;
        else
            hi = mid;
    }
    return hi * hi;
}

void* DevMem::alloc(size_t b) const {
    void* p = nullptr;
    if (b == 0)
        b = 16;
    cudaError_t e = cudaMallocFromPoolAsync(&p, b, pool, stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(ATVB_ERR_NOMEM, "device allocation of " + std::to_string(b) +
                                        " bytes failed: " + cudaGetErrorString(e));
    }
    return p;
}

void DevMem::free(void* p) const {
    if (p)
        cudaFreeAsync(p, stream);
}

void* Slot::dalloc(size_t b) {
    void* p = mem_.alloc(b);
    allocs.push_back(p);
    bytes += b == 0 ? 16 : b;
    return p;
}

void Slot::free_alloc(void* p) {
    auto it = std::find(allocs.begin(), allocs.end(), p);
    if (it != allocs.end()) {
        allocs.erase(it);
        mem_.free(p);
    }
}

// Re-plan the bins and stencil for cells down to L (1 - shrink) per axis
// (MTK NPT): new bin arrays and columns, box-dependent fields recomputed.
void Slot::replan_cells(double shrink) {
    cudaStream_t stream = mem_.stream;
    geo = make_geometry(desc, shrink);
    free_alloc(hp.cell_count);
    free_alloc(hp.cell_start);
    free_alloc(hp.cols);
    for (int k = 0; k < 3; ++k) {
        hp.nc[k] = geo.nc[k];
        hp.alias[k] = geo.alias[k];
        hp.npt_Lmin[k] = geo.Lmin[k];
    }
    hp.ncell = geo.nc[0] * geo.nc[1] * geo.nc[2];
    hp.ncol = (int)geo.cols.size();
    hp.cell_count = (int*)dalloc(sizeof(int) * hp.ncell);
    hp.cell_start = (int*)dalloc(sizeof(int) * (hp.ncell + 1));
    CK(cudaMemsetAsync(hp.cell_count, 0, sizeof(int) * hp.ncell, stream));
    hp.cols = (int4*)dalloc(sizeof(int4) * geo.cols.size());
    CK(cudaMemcpyAsync(hp.cols, geo.cols.data(), sizeof(int4) * geo.cols.size(),
                       cudaMemcpyHostToDevice, stream));
    apply_box(hp, geo.L, false);
    CK(cudaStreamSynchronize(stream));
}

Slot::~Slot() {
    if (snap_host) {
        cudaStreamSynchronize(mem_.stream); // no snapshot kernel still writing
        cudaFreeHost(snap_host);
    }
    for (void* p : allocs)
        mem_.free(p);
    mem_.free(nbr_alloc);
}

void Slot::alloc_list(int new_cap) {
    mem_.free(nbr_alloc);
    nbr_alloc = nullptr;
    const size_t b = (size_t)hp.n * new_cap * sizeof(int);
    nbr_alloc = mem_.alloc(b);
    hp.nbr = (int*)nbr_alloc;
    hp.cap = new_cap;
}

void Slot::widen_list(int new_cap) {
    const int oc = hp.cap;
    if (new_cap <= oc)
        return;
    const size_t n = (size_t)hp.n;
    void* p = mem_.alloc(n * (size_t)new_cap * sizeof(int));
    CK(cudaMemcpy2DAsync(p, (size_t)new_cap * sizeof(int), hp.nbr, (size_t)oc * sizeof(int),
                         (size_t)oc * sizeof(int), n, cudaMemcpyDeviceToDevice, mem_.stream));
    mem_.free(nbr_alloc);
    nbr_alloc = p;
    hp.nbr = (int*)p;
    hp.cap = new_cap;
}

Slot::Slot(const atvb_system_desc& d, const DevMem& mem) : desc(d), mem_(mem) {
    cudaStream_t stream = mem.stream;
    geo = make_geometry(d);
    std::memset(&hp, 0, sizeof(hp));
    const int n = d.n_atoms;
    if (n > kMaxAtoms)
        throw Error(ATVB_ERR_INVALID, "at most 2^30 - 1 atoms per system");
    hp.n = n;
    hp.deform_axis = -1;
    hp.prec = d.precision == ATVB_MIXED ? kMixed : kFP64;
    if (d.precision != ATVB_FP64 && d.precision != ATVB_MIXED)
        throw Error(ATVB_ERR_INVALID, "unknown precision");
    for (int k = 0; k < 3; ++k) {
        hp.nc[k] = geo.nc[k];
        hp.alias[k] = geo.alias[k];
        hp.npt_Lmin[k] = geo.Lmin[k];
    }
    hp.ncell = geo.nc[0] * geo.nc[1] * geo.nc[2];
    hp.rlist = geo.rlist;
    hp.rlist2 = geo.rlist * geo.rlist;
    hp.nl_cut = d.nl_cutoff;
    hp.skin_half2 = 0.25 * geo.skin * geo.skin;
    hp.nl_every = d.nl_every < 1 ? 1 : d.nl_every;
    hp.nl_delay = d.nl_delay < 0 ? 0 : d.nl_delay;
    hp.nl_check = d.nl_check ? 1 : 0;
    hp.ncol = (int)geo.cols.size();
    // LJ (pair_lj_cut.cpp:30-41)
    hp.has_lj = d.lj_enabled ? 1 : 0;
    if (hp.has_lj) {
        if (!(d.lj_cutoff > 0.0))
            throw Error(ATVB_ERR_INVALID, "PairLJCut: cutoff must be positive");
        if (d.lj_cutoff > geo.rlist)
            throw Error(ATVB_ERR_INVALID,
                        "PairLJCut cutoff exceeds the neighbour list reach");
        const double s2 = d.lj_sigma * d.lj_sigma;
        hp.lj_sig6 = s2 * s2 * s2;
        hp.lj_rc2 = d.lj_cutoff * d.lj_cutoff;
        hp.lj_eps4 = 4.0 * d.lj_epsilon;
        hp.lj_eps24 = 24.0 * d.lj_epsilon;
        const double r2inv = 1.0 / hp.lj_rc2;
        const double r6inv = r2inv * r2inv * r2inv * hp.lj_sig6;
        hp.lj_shift = 4.0 * d.lj_epsilon * (r6inv * r6inv - r6inv);
    }
    // mixed build: settle pairs near the LJ cutoff (band set by apply_box).
    // A pair that FP32 rounding moves across the LJ cutoff changes the
    // forces by the force jump there (the energy is shifted, the force is
    // not); below 1e-5 eV/A that is negligible and the settling is off
    // (e.g. LJ cut at 4 sigma under Coulomb: 2.5e-6 eV/A)
    hp.mix_band_lj = d.lj_enabled ? 1.0 : 0.0;
    if (d.lj_enabled) {
        const double sr2 = d.lj_sigma * d.lj_sigma / (d.lj_cutoff * d.lj_cutoff);
        const double sr6 = sr2 * sr2 * sr2;
        const double jump = std::fabs(24.0 * d.lj_epsilon / d.lj_cutoff * (2.0 * sr6 * sr6 - sr6));
        if (jump < 1e-5)
            hp.mix_band_lj = 0.0;
    }
    hp.has_coul = d.coul_enabled ? 1 : 0;
    if (hp.has_coul) {
        if (!(d.coul_alpha > 0.0) || !(d.coul_cutoff > 0.0))
            throw Error(ATVB_ERR_INVALID,
                        "CoulLong: alpha and cutoff must be positive");
        if (d.coul_cutoff > geo.rlist)
            throw Error(ATVB_ERR_INVALID,
                        "CoulLong cutoff exceeds the neighbour list reach");
        hp.coul_rc2 = d.coul_cutoff * d.coul_cutoff;
        hp.coul_alpha = d.coul_alpha;
        hp.coul_alpha2 = d.coul_alpha * d.coul_alpha;
        hp.coul_short = d.coul_alpha * d.coul_cutoff <= kErfcxSXmax ? 1 : 0;
        // the pair kernels' erfcx polynomial covers alpha * r <= kErfcxXmax
        if (d.coul_alpha * d.coul_cutoff > kErfcxXmax)
            throw Error(ATVB_ERR_INVALID,
                        "CoulLong: alpha * cutoff must not exceed 6 "
                        "(erfc(6) = 2e-17 is below double precision)");
        if (d.coul_alpha * geo.rlist > 26.0)
            throw Error(ATVB_ERR_INVALID,
                        "CoulLong: alpha * (cutoff + skin) must not exceed 26");
    }
    // the largest interaction cutoff: the build-cell displacement rule of the
    // per-axis drift path (barostats, speed cap, deformation)
    hp.npt_cut = d.nl_cutoff;
    if (hp.has_lj)
        hp.npt_cut = std::max(hp.npt_cut, d.lj_cutoff);
    if (hp.has_coul)
        hp.npt_cut = std::max(hp.npt_cut, d.coul_cutoff);
    // integrator / thermostat
    if (!(d.dt > 0.0))
        throw Error(ATVB_ERR_INVALID, "VelocityVerlet: dt must be > 0");
    hp.dt = d.dt;
    hp.dtf = 0.5 * d.dt * kFtm2v;
    hp.thermostat = d.thermostat;
    hp.T = d.temperature;
    const int ndof = std::max(0, 3 * n - 3);
    hp.n_dof_kT = (double)ndof * kKB * d.temperature;
    if (d.thermostat == ATVB_NOSE_HOOVER) {
        if (!(d.tau > 0.0) || !(d.temperature > 0.0))
            throw Error(ATVB_ERR_INVALID,
                        "NoseHoover: temperature and tau must be > 0");
        hp.tau = d.tau;
        hp.Q = (double)ndof * kKB * d.temperature * d.tau * d.tau;
    } else if (d.thermostat == ATVB_LANGEVIN) {
        if (!(d.damp > 0.0) || d.temperature < 0.0)
            throw Error(ATVB_ERR_INVALID, "FixLangevin: damp must be > 0");
        hp.lang_g1 = 1.0 / (d.damp * kFtm2v);
        hp.lang_g2pre =
            std::sqrt(2.0 * kKB * d.temperature / (d.damp * d.dt * kMvv2e)) /
            kFtm2v;
        hp.lang_T0 = hp.lang_T1 = d.temperature;
        hp.lang_ddm = d.damp * d.dt * kMvv2e;
        hp.lang_nfirst = hp.lang_nlast = 0;
        hp.seed = d.seed;
    } else if (d.thermostat != ATVB_NVE) {
        throw Error(ATVB_ERR_INVALID, "unknown thermostat");
    }
    hp.need_virial = d.stress_required ? 1 : 0;
    // device memory
    auto dd = [&](size_t cnt) { return (double*)dalloc(cnt * sizeof(double)); };
    hp.x = dd(n);
    hp.y = dd(n);
    hp.z = dd(n);
    hp.vx = dd(n);
    hp.vy = dd(n);
    hp.vz = dd(n);
    hp.mass = dd(n);
    hp.q = dd(n);
    hp.xr = dd(n);
    hp.yr = dd(n);
    hp.zr = dd(n);
    hp.sx = dd(n);
    hp.sy = dd(n);
    hp.sz = dd(n);
    hp.tag = (long long*)dalloc((size_t)n * 8);
    hp.posd4 = (double4*)dalloc((size_t)n * sizeof(double4));
    hp.lpos = (int4*)dalloc((size_t)n * sizeof(int4));
    if (hp.prec == kMixed && d.lj_enabled) {
        hp.nearq_cap = std::max(4096, n / 16);
        hp.nearq = (int2*)dalloc((size_t)hp.nearq_cap * sizeof(int2));
    }
    hp.pos4 = hp.prec == kMixed ? dalloc((size_t)n * sizeof(int4))
                                : dalloc((size_t)n * sizeof(double4));
    hp.f4 = (double4*)dalloc((size_t)n * sizeof(double4));
    auto di = [&](size_t cnt) { return (int*)dalloc(cnt * sizeof(int)); };
    hp.perm = di(n);
    hp.rank = di(n);
    hp.cell_of = di(n);
    hp.slot = di(n);
    hp.cellS = di(n);
    hp.nnbr = di(n);
    hp.cell_count = di(hp.ncell);
    hp.cell_start = di(hp.ncell + 1);
    CK(cudaMemsetAsync(hp.cell_count, 0, sizeof(int) * hp.ncell, stream));
    hp.cols = (int4*)dalloc(sizeof(int4) * geo.cols.size());
    CK(cudaMemcpyAsync(hp.cols, geo.cols.data(), sizeof(int4) * geo.cols.size(),
                       cudaMemcpyHostToDevice, stream));
    hp.st = (SysState*)dalloc(sizeof(SysState));
    hp.ehist_cap = d.history_capacity > 0 ? d.history_capacity : 4096;
    hp.ehist = dd(3 * (size_t)hp.ehist_cap);
    alloc_list(expected_row(d, geo));
    // PME
    hp.has_pme = d.pme_enabled ? 1 : 0;
    if (hp.has_pme) {
        if (!(d.pme_alpha > 0.0))
            throw Error(ATVB_ERR_INVALID, "KSpacePME: alpha must be > 0");
        if (d.pme_order < 3 || d.pme_order > 8)
            throw Error(ATVB_ERR_INVALID, "KSpacePME: order must be in [3, 8]");
        hp.order = d.pme_order;
        for (int k = 0; k < 3; ++k)
            hp.K[k] = pme_K(d, geo, k);
        hp.Kh = hp.K[2] / 2 + 1;
        hp.Khp = (hp.Kh + 15) / 16 * 16;
        hp.pme_alpha = d.pme_alpha;
        hp.pme_alpha2_pi2 = kPi * kPi / (d.pme_alpha * d.pme_alpha);
        hp.grid_scale = hp.prec == kMixed ? 4294967296.0 : 1099511627776.0;
        hp.grid_scale_inv = 1.0 / hp.grid_scale;
        const size_t K0 = hp.K[0], K1 = hp.K[1], K2 = hp.K[2], Khp = hp.Khp;
        const size_t nt = K0 * K1 * K2, nh = K0 * K1 * Khp;
        const size_t rs = hp.prec == kMixed ? 4 : 8;
        hp.fp4 = (double4*)dalloc((size_t)n * sizeof(double4));
        hp.grid_fix = (unsigned long long*)dalloc(nt * 8);
        CK(cudaMemsetAsync(hp.grid_fix, 0, nt * 8, stream));
        hp.grid_real = dalloc(nt * rs);
        hp.grid_cplx = dalloc(nh * 2 * rs);
        // B-spline moduli per axis (pme_spline.h:67-94); the influence
        // function H(m) itself is evaluated on the fly from the current cell
        std::vector<double> bm;
        for (int k = 0; k < 3; ++k) {
            const std::vector<double> m = spline_moduli(hp.K[k], hp.order);
            bm.insert(bm.end(), m.begin(), m.end());
        }
        double* dbm = dd(bm.size());
        CK(cudaMemcpyAsync(dbm, bm.data(), bm.size() * 8, cudaMemcpyHostToDevice, stream));
        hp.bmod = dbm;
        // the transforms (fft.cu): radices per axis (z: the complex FFT of
        // K2 / 2 when K2 is even) and the K-th roots of unity per axis
        for (int k = 0; k < 3; ++k) {
            const int K = hp.K[k];
            int m = (k == 2 && K % 2 == 0) ? K / 2 : K;
            int nf = 0;
            for (int p : {4, 2, 3, 5, 7})
                while (m % p == 0 && nf < kFftMaxFac) {
                    hp.fft_fac[k][nf++] = p;
                    m /= p;
                }
            if (m != 1)
                throw Error(ATVB_ERR_INVALID, "KSpacePME: a mesh size must be 2,3,5,7-smooth "
                                              "(good_fft_size), got " + std::to_string(K));
            if (K > 2048) // a line and its roots must fit one block's shared memory
                throw Error(ATVB_ERR_INVALID, "KSpacePME: at most 2048 mesh points per axis, got " +
                                                  std::to_string(K));
            hp.fft_nf[k] = nf;
            std::vector<double> rt(2 * (size_t)K);
            for (int j = 0; j < K; ++j) {
                const long double a = -2.0L * 3.14159265358979323846264338327950288L * j / K;
                rt[2 * j] = (double)cosl(a);
                rt[2 * j + 1] = (double)sinl(a);
            }
            if (hp.prec == kMixed) {
                std::vector<float> rf(rt.begin(), rt.end());
                void* d = dalloc(rf.size() * sizeof(float));
                CK(cudaMemcpyAsync(d, rf.data(), rf.size() * sizeof(float),
                                   cudaMemcpyHostToDevice, stream));
                hp.fft_root[k] = d;
                CK(cudaStreamSynchronize(stream)); // rf is a local
            } else {
                void* d = dalloc(rt.size() * sizeof(double));
                CK(cudaMemcpyAsync(d, rt.data(), rt.size() * sizeof(double),
                                   cudaMemcpyHostToDevice, stream));
                hp.fft_root[k] = d;
                CK(cudaStreamSynchronize(stream));
            }
        }
        CK(cudaStreamSynchronize(stream));
    }
    apply_box(hp, geo.L, false);
    CK(cudaStreamSynchronize(stream));
}

// ------------------------------------------------------------- Engine

Engine::Engine(int device) : device_(device) {
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&cond_stream_, cudaStreamNonBlocking));
    CK(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount,
                              device));
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    CK(cudaMemPoolCreate(&mem_.pool, &props));
    // keep freed memory in the pool until the engine goes away
    uint64_t keep = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(mem_.pool, cudaMemPoolAttrReleaseThreshold, &keep));
    mem_.stream = stream_;
    // the PME branch (lane 0 and the FFT lanes) at the highest priority: its
    // short memory-bound kernels take SMs as pair blocks retire instead of
    // waiting for the whole pair grid
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    CK(cudaStreamCreateWithPriority(&pme_stream_, cudaStreamNonBlocking, prio_hi));
    CK(cudaEventCreateWithFlags(&pme_fork_, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&pme_join_, cudaEventDisableTiming));
    // the FFT blocks' line buffers live in dynamic shared memory above 48 KB
    fft_smem_optin(kFftSmem + 1024);
}

Engine::~Engine() {
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    for (auto it = comps_.rbegin(); it != comps_.rend(); ++it) // reverse plan order
        if (const UserComp& c = *it; c.built && c.destroy && has(c.slot)) {
            const atvb_launch_ctx ctx = comp_ctx(c, -1);
            c.destroy(c.user, &ctx); // errors cannot be reported from here
        }
    release_graph();
    slots_.clear();
    for (void* p : list_allocs_)
        mem_.free(p);
    mem_.free(d_sp_);
    cudaStreamSynchronize(stream_);
    if (row_hint_host_)
        cudaFreeHost(row_hint_host_);
    if (pme_stream_)
        cudaStreamDestroy(pme_stream_);
    if (pme_fork_)
        cudaEventDestroy(pme_fork_);
    if (pme_join_)
        cudaEventDestroy(pme_join_);
    if (mem_.pool)
        cudaMemPoolDestroy(mem_.pool);
    for (auto& e : prof_events_)
        cudaEventDestroy(e);
    if (cond_stream_)
        cudaStreamDestroy(cond_stream_);
    if (stream_)
        cudaStreamDestroy(stream_);
}

void Engine::release_graph() {
    if (gexec_)
        cudaGraphExecDestroy(gexec_);
    if (graph_)
        cudaGraphDestroy(graph_);
    gexec_ = nullptr;
    graph_ = nullptr;
}

int Engine::add(const atvb_system_desc& d) {
    CK(cudaSetDevice(device_));
    auto s = std::make_unique<Slot>(d, mem_);
    int id = -1;
    for (size_t k = 0; k < slots_.size(); ++k)
        if (!slots_[k]) {
            id = (int)k;
            break;
        }
    if (id < 0) {
        id = (int)slots_.size();
        slots_.emplace_back();
    }
    s->index = id;
    slots_[id] = std::move(s);
    ensure_table();
    row_hint_host_[id] = 0; // a reused entry may hold its last owner's hint
    row_hint_host_[sp_cap_ + id] = 0;
    push_params(id);
    dirty_ = true;
    return id;
}

void Engine::remove(int id) {
    Slot* s = slot(id);
    release_graph(); // the captured step references this system's memory
    slots_[id].reset(); // stream-ordered frees: no wait for the device
    dirty_ = true;
}

Slot* Engine::slot(int id) {
    if (id < 0 || id >= (int)slots_.size() || !slots_[id])
        throw Error(ATVB_ERR_NOTFOUND, "no system with id " + std::to_string(id));
    return slots_[id].get();
}

void Engine::ensure_table() {
    if ((int)slots_.size() <= sp_cap_)
        return;
    int cap = std::max(8, sp_cap_ * 2);
    while (cap < (int)slots_.size())
        cap *= 2;
    SysParams* nd = (SysParams*)mem_.alloc(sizeof(SysParams) * cap);
    if (d_sp_) {
        CK(cudaMemcpyAsync(nd, d_sp_, sizeof(SysParams) * sp_cap_,
                           cudaMemcpyDeviceToDevice, stream_));
        mem_.free(d_sp_);
    }
    release_graph(); // captured launches point at the old table
    // the row hints move with the table: nothing in flight may still write
    // the old array when it is freed, and every entry is re-pointed
    // one host-mapped array: row hints in [0, cap), status words in
    // [cap, 2 cap)
    void* h = nullptr;
    CK(cudaHostAlloc(&h, sizeof(int) * 2 * cap, cudaHostAllocMapped));
    std::memset(h, 0, sizeof(int) * 2 * cap);
    if (row_hint_host_) {
        CK(cudaDeviceSynchronize());
        std::memcpy(h, row_hint_host_, sizeof(int) * sp_cap_);
        std::memcpy((int*)h + cap, row_hint_host_ + sp_cap_, sizeof(int) * sp_cap_);
        CK(cudaFreeHost(row_hint_host_));
    }
    row_hint_host_ = (int*)h;
    void* hd = nullptr;
    CK(cudaHostGetDevicePointer(&hd, h, 0));
    row_hint_dev_ = (int*)hd;
    d_sp_ = nd;
    sp_cap_ = cap;
    for (int id = 0; id < (int)slots_.size(); ++id)
        if (slots_[id])
            push_params(id); // re-points row_hint at the new array
    dirty_ = true;
}

// Between step calls: a system whose last build filled more than 80 % of
// its row capacity gets rows 1.5 x that long.  The old rows are copied into
// the wider ones, stream-ordered behind the steps in flight, so the list
// and every later result stay exactly what they would have been; no build
// overflows unless a row grows by more than a quarter within one call.
void Engine::widen_rows() {
    if (!row_hint_host_)
        return;
    for (int id = 0; id < (int)slots_.size(); ++id) {
        Slot* s = slots_[id].get();
        if (!s || !s->uploaded || !s->hp.nbr)
            continue;
        const int m = ((volatile int*)row_hint_host_)[id];
        const int oc = s->hp.cap;
        if ((long long)m * 5 <= (long long)oc * 4)
            continue;
        if (s->row_cap_fixed > 0)
            continue; // pinned by atvb_system_set_capacity: reported, not grown
        s->widen_list(round_up((long long)(m * 1.5) + 32, 32));
        push_params(id);
        if (m > oc) {
            // a build within the last call cut a row (its forces missed
            // pairs, flagged in the status bits): build again at the next
            // step, into the wider rows, instead of waiting for the skin
            const int one = 1;
            CK(cudaMemcpyAsync(&s->hp.st->force_build, &one, sizeof(int),
                               cudaMemcpyHostToDevice, stream_));
            CK(cudaStreamSynchronize(stream_)); // `one` lives on this frame
        }
    }
}

void Engine::push_params(int id) {
    Slot* s = slot(id);
    s->hp.row_hint = (row_hint_dev_ && id < sp_cap_) ? row_hint_dev_ + id : nullptr;
    s->hp.status_hint =
        (row_hint_dev_ && id < sp_cap_) ? row_hint_dev_ + sp_cap_ + id : nullptr;
    if ((s->npt || s->baro || s->hp.deform_axis >= 0) && s->uploaded) {
        // the device owns an NPT system's cell: keep it
        SysParams dev;
        CK(cudaMemcpyAsync(&dev, d_sp_ + id, sizeof(SysParams), cudaMemcpyDeviceToHost,
                           stream_));
        CK(cudaStreamSynchronize(stream_));
        s->hp.e_const = dev.e_const;
        apply_box(s->hp, dev.L, true);
    }
    CK(cudaMemcpyAsync(d_sp_ + id, &s->hp, sizeof(SysParams),
                       cudaMemcpyHostToDevice, stream_));
}

static ItemList make_list(std::vector<void*>& allocs, const std::vector<Item>& v,
                          int max_grid, const DevMem& mem) {
    cudaStream_t stream = mem.stream;
    ItemList il;
    il.n = (int)v.size();
    if (v.empty())
        return il;
    void* p = mem.alloc(sizeof(Item) * v.size());
    allocs.push_back(p);
    CK(cudaMemcpyAsync(p, v.data(), sizeof(Item) * v.size(),
                       cudaMemcpyHostToDevice, stream));
    il.d = (const Item*)p;
    il.grid = std::min(il.n, max_grid);
    return il;
}

// Lanes per atom for one system, from that system alone: at least 4 (the
// lanes of an atom read consecutive row entries, so a warp's row loads
// coalesce; measured on 1M LJ atoms: 4 lanes 27 % (FP64) and 35 % (mixed)
// faster than 1), more while the GPU is not filled with this system's
// atoms, but no more than its rows can keep busy (at least 8 row entries
// per lane).
int Engine::lanes_for(const Slot& sl) const {
    if (lanes_fixed_ > 0)
        return lanes_fixed_;
    const long long n = sl.hp.n;
    const long long target = (long long)num_sms_ * 2048 * 2;
    int G = 4;
    while (G < 32 && n * G < target)
        G *= 2;
    int gmax = 1;
    while (gmax < 32 && gmax * 8 <= sl.mean_row)
        gmax *= 2;
    return std::max(1, std::min(G, gmax));
}

static int lane_class(int G) {
    int k = 0;
    while ((1 << k) < G)
        ++k;
    return k;
}

void Engine::build_lists() {
    release_graph();
    for (void* p : list_allocs_)
        mem_.free(p);
    list_allocs_.clear();
    std::vector<Item> atoms, list, cells, patoms;
    std::vector<int> sys;
    std::vector<Item> pair_by[2][kLaneClasses];
    std::vector<Item> pair_gen[2];
    lc_ = LaunchCfg{};
    int largest = -1;
    pme_slots_.clear();
    int pme_prec = -1, pme_order = -1;
    for (const auto& sp : slots_) {
        if (!sp || !sp->uploaded)
            continue;
        const SysParams& P = sp->hp;
        const int k = sp->index;
        sys.push_back(k);
        for (int b = 0; b < P.n; b += kChunk)
            atoms.push_back({k, b});
        for (int b = 0; b < P.ncell; b += kListChunk)
            list.push_back({k, b});
        sp->lanes = lanes_for(*sp);
        if (P.n > largest) {
            largest = P.n;
            lc_.pair_G = sp->lanes;
        }
        if (P.general) {
            // per-type LJ or special pairs: the general kernel
            for (int b = 0; b < P.n; b += kPairBlock / kGenLanes)
                pair_gen[P.prec == kMixed ? 1 : 0].push_back({k, b});
        } else {
            std::vector<Item>& pv = pair_by[P.prec == kMixed ? 1 : 0][lane_class(sp->lanes)];
            for (int b = 0; b < P.n; b += kPairBlock / sp->lanes)
                pv.push_back({k, b});
        }
        for (int b = 0; b < P.ncell; b += kChunk)
            cells.push_back({k, b});
        if (P.prec == kMixed)
            lc_.any_mixed = 1;
        else
            lc_.any_fp64 = 1;
        if (P.prec == kMixed && P.has_lj && !P.general && P.mix_band_lj > 0.0)
            lc_.any_near = 1;
        if (P.snap_ring)
            lc_.any_snap = 1;
        if (P.baro)
            lc_.any_baro = 1;
        if (P.has_pme) {
            if (pme_prec >= 0 && (pme_prec != P.prec || pme_order != P.order))
                throw Error(ATVB_ERR_INVALID,
                            "all PME systems of one engine must share "
                            "precision and spline order");
            pme_prec = P.prec;
            pme_order = P.order;
            pme_slots_.push_back(k);
            for (int b = 0; b < P.n; b += kChunk)
                patoms.push_back({k, b});
        }
    }
    const int g_light = num_sms_ * 16;
    lc_.sp = d_sp_;
    lc_.atoms = make_list(list_allocs_, atoms, g_light, mem_);
    lc_.list = make_list(list_allocs_, list, num_sms_ * 32, mem_);
    for (int p = 0; p < 2; ++p)
        for (int c = 0; c < kLaneClasses; ++c)
            lc_.pair[p][c] = make_list(list_allocs_, pair_by[p][c], num_sms_ * 16, mem_);
    for (int p = 0; p < 2; ++p)
        lc_.pair_gen[p] = make_list(list_allocs_, pair_gen[p], num_sms_ * 16, mem_);
    lc_.cells = make_list(list_allocs_, cells, g_light, mem_);
    lc_.pme_atoms = make_list(list_allocs_, patoms, g_light, mem_);
    lc_.nsys = (int)sys.size();
    if (!sys.empty()) {
        void* p = mem_.alloc(sizeof(int) * sys.size());
        list_allocs_.push_back(p);
        CK(cudaMemcpyAsync(p, sys.data(), sizeof(int) * sys.size(),
                           cudaMemcpyHostToDevice, stream_));
        lc_.sys_list = (const int*)p;
    }
    lc_.fft = fft_items(pme_slots_);
    lc_.pme_mixed = pme_prec == kMixed ? 1 : 0;
    lc_.pme_order = pme_order > 0 ? pme_order : 4;
    CK(cudaStreamSynchronize(stream_));
    release_graph();
    dirty_ = false;
    ++list_epoch_;
    single_.clear();
}

// The PME transforms' work items over the systems in `pme` (fft.cu): per
// pass one group per line length, in the register form of that length
// where there is one (fft_reg*.cu), else the generic kernels; the z items
// are groups of x-y lines, the y items k0 x a block of m2 columns and the x
// items m1 x a block of columns.
FftCfg Engine::fft_items(const std::vector<int>& pme) {
    FftCfg f;
    if (pme.empty())
        return f;
    const bool mixed = slots_[pme[0]]->hp.prec == kMixed;
    // register forms: 4 blocks per SM looping over their tiles (measured at
    // 192^3: 165 / 122 us FP64 / FP32 for the five passes, against 174 / 129
    // with 16 per SM and 220 / 142 with 2)
    const int g = num_sms_ * 8, gr = num_sms_ * 4;
    // axis 2: z, 1: y, 0: x
    for (int axis = 2; axis >= 0; --axis) {
        std::vector<FftGroup>& out = axis == 2 ? f.z : axis == 1 ? f.y : f.x;
        std::vector<std::vector<Item>> items;
        for (int id : pme) {
            const SysParams& P = slots_[id]->hp;
            const int K = P.K[axis];
            const int n = (axis == 2 && K % 2 == 0) ? K / 2 : K;
            size_t gi = 0;
            while (gi < out.size() && !(out[gi].n == n && out[gi].k == K))
                ++gi;
            if (gi == out.size()) {
                FftGroup grp;
                grp.n = n;
                grp.k = K;
                // the z register forms take an even K2 (lines of K2 / 2)
                grp.reg = (axis != 2 || K % 2 == 0) ? fft_reg_index(n) : -1;
                if (grp.reg >= 0)
                    grp.c = axis == 2 ? fft_reg_lines(grp.reg, mixed) : fft_reg_cols(mixed);
                else
                    grp.c = fft_lines_per_block(n, K, mixed);
                out.push_back(grp);
                items.emplace_back();
            }
            const int c = out[gi].c;
            std::vector<Item>& v = items[gi];
            if (axis == 2) {
                for (int l = 0; l < P.K[0] * P.K[1]; l += c)
                    v.push_back({id, l});
            } else {
                const int nb = (P.Kh + c - 1) / c;
                const int lines = axis == 1 ? P.K[0] : P.K[1];
                for (int q = 0; q < lines * nb; ++q)
                    v.push_back({id, q});
            }
        }
        for (size_t gi = 0; gi < out.size(); ++gi)
            out[gi].items = make_list(list_allocs_, items[gi], out[gi].reg >= 0 ? gr : g, mem_);
    }
    return f;
}

// ---- user components (atvb_system_add_component) ---------------------------

void Engine::add_component(int id, int phase, int order, atvb_component_fn build,
                           atvb_component_fn launch, atvb_component_fn destroy, void* user) {
    Slot* s = slot(id);
    if (phase < ATVB_PHASE_INITIAL_INTEGRATE || phase > ATVB_PHASE_END_OF_STEP)
        throw Error(ATVB_ERR_INVALID, "add_component: phase must be one of ATVB_PHASE_*");
    if (!launch)
        throw Error(ATVB_ERR_INVALID, "add_component: launch is required");
    CK(cudaSetDevice(device_));
    if (!s->hp.ext_f) {
        const size_t n = (size_t)s->hp.n;
        s->hp.ext_f = (double*)s->dalloc(3 * n * sizeof(double));
        s->hp.ext_ev = (double*)s->dalloc(7 * sizeof(double));
        CK(cudaMemsetAsync(s->hp.ext_f, 0, 3 * n * sizeof(double), stream_));
        CK(cudaMemsetAsync(s->hp.ext_ev, 0, 7 * sizeof(double), stream_));
        push_params(id);
        CK(cudaStreamSynchronize(stream_));
    }
    UserComp c{id, phase, order, (int)comps_.size(), build, launch, destroy, user, false};
    comps_.push_back(c);
    std::stable_sort(comps_.begin(), comps_.end(), [](const UserComp& a, const UserComp& b) {
        return a.phase != b.phase ? a.phase < b.phase
                                  : (a.order != b.order ? a.order < b.order : a.seq < b.seq);
    });
    release_graph(); // steps of a system with components run as launches
}

atvb_launch_ctx Engine::comp_ctx(const UserComp& c, int phase) const {
    const Slot& s = *slots_[c.slot];
    const SysParams& P = s.hp;
    atvb_launch_ctx x{};
    x.stream = (void*)stream_;
    x.phase = phase;
    x.step = comp_step_;
    atvb_device_frame& f = x.frame;
    f.n_atoms = P.n;
    f.x = P.x;
    f.y = P.y;
    f.z = P.z;
    f.vx = P.vx;
    f.vy = P.vy;
    f.vz = P.vz;
    f.mass = P.mass;
    f.charge = P.q;
    f.tag = reinterpret_cast<const int64_t*>(P.tag);
    f.fx = P.ext_f;
    f.fy = P.ext_f + P.n;
    f.fz = P.ext_f + 2 * (size_t)P.n;
    f.energy = P.ext_ev;
    f.virial = P.ext_ev + 1;
    // the device table entry's cell edges: the cell in force this step
    f.box = reinterpret_cast<const double*>(reinterpret_cast<const char*>(d_sp_ + c.slot) +
                                            offsetof(SysParams, L));
    return x;
}

// build() of every component not built yet (the frame is on the device),
// and the step index the next launches report.
void Engine::build_components() {
    CK(cudaStreamSynchronize(stream_));
    for (UserComp& c : comps_) {
        if (c.built)
            continue;
        if (c.build) {
            const atvb_launch_ctx ctx = comp_ctx(c, -1);
            const int rc = c.build(c.user, &ctx);
            if (rc != 0)
                throw Error(ATVB_ERR_STATE, "component build returned " + std::to_string(rc));
        }
        c.built = true;
    }
    SysState st;
    CK(cudaMemcpy(&st, slots_[comps_.front().slot]->hp.st, sizeof(st), cudaMemcpyDeviceToHost));
    comp_step_ = st.step;
}

void Engine::run_components(int phase, bool before) {
    for (const UserComp& c : comps_) {
        if (c.phase != phase || (c.order < 0) != before)
            continue;
        const atvb_launch_ctx ctx = comp_ctx(c, phase);
        const int rc = c.launch(c.user, &ctx);
        if (rc != 0)
            throw Error(ATVB_ERR_STATE, "component launch returned " + std::to_string(rc) +
                                            " at phase " + std::to_string(phase));
    }
}

void Engine::zero_component_sums() {
    for (const auto& up : slots_)
        if (up && up->hp.ext_f) {
            CK(cudaMemsetAsync(up->hp.ext_f, 0, 3 * (size_t)up->hp.n * sizeof(double), stream_));
            CK(cudaMemsetAsync(up->hp.ext_ev, 0, 7 * sizeof(double), stream_));
        }
}

// One step of a system with components: the kernels of enqueue_step as
// launches, with the components' callbacks at their phases (stage.h:24-36).
void Engine::enqueue_step_components() {
    auto phase = [&](int p, auto&& own) {
        run_components(p, true);
        own();
        run_components(p, false);
    };
    phase(ATVB_PHASE_INITIAL_INTEGRATE, [&] {
        launch_integrate_a(lc_, stream_);
        launch_sys_a(lc_, stream_);
    });
    phase(ATVB_PHASE_POST_INTEGRATE, [] {});
    phase(ATVB_PHASE_PRE_EXCHANGE, [] {});
    phase(ATVB_PHASE_PRE_NEIGHBOR, [] {});
    phase(ATVB_PHASE_NEIGHBOR, [&] {
        launch_sort_cells(lc_, stream_);
        launch_build_list(lc_, stream_);
    });
    phase(ATVB_PHASE_PRE_FORCE, [&] { zero_component_sums(); });
    phase(ATVB_PHASE_FORCE, [&] { enqueue_forces(lc_, pme_slots_, false, true, false); });
    phase(ATVB_PHASE_POST_FORCE, [] {});
    phase(ATVB_PHASE_FINAL_INTEGRATE, [&] { launch_integrate_b(lc_, stream_); });
    phase(ATVB_PHASE_END_OF_STEP, [&] {
        launch_sys_b(lc_, stream_);
        if (lc_.any_snap)
            launch_snapshots(lc_, stream_);
    });
    CK(cudaGetLastError());
    ++comp_step_;
}

// Kernel launches of one step.
int64_t Engine::kernels_per_step() const {
    int64_t k = 0;
    k += 2;                                   // integrate_a, sys_a
    k += kRebuildKernels;                     // list build (rebuild steps only)
    for (int p = 0; p < 2; ++p)                // pair: one per lane class used
        for (int c = 0; c < kLaneClasses; ++c)
            k += lc_.pair[p][c].n ? 1 : 0;
    k += lc_.any_near ? 1 : 0;                // near-cutoff fix-up (mixed LJ)
    k += (lc_.pair_gen[0].n ? 1 : 0) + (lc_.pair_gen[1].n ? 1 : 0); // general pair
    if (!pme_slots_.empty())
        k += 2 + lc_.fft.launches();          // spread, gather, the transform passes
    k += 2;                                   // integrate_b, sys_b
    k += lc_.any_snap ? 3 : 0;                // trajectory snapshots
    k += lc_.any_baro ? 1 : 0;                // Berendsen position scaling
    return k;
}

// Pair forces and the PME chain.  `overlap`: the PME chain (spread, FFTs,
// influence, gather into fp4) runs on lane 0 beside the pair kernel -- the
// pair kernel is arithmetic-bound, the PME kernels memory- and
// atomic-bound -- and joins before the next atom pass; otherwise (profiling,
// force passes) everything runs in order on the engine stream.
void Engine::enqueue_forces(const LaunchCfg& lc, const std::vector<int>& pme,
                            bool profile, bool overlap, bool build_list) {
    const bool side = overlap && !profile && !pme.empty();
    cudaStream_t ps = side ? pme_stream_ : stream_;
    if (side) {
        CK(cudaEventRecord(pme_fork_, stream_));
        CK(cudaStreamWaitEvent(ps, pme_fork_, 0));
    }
    // The PME chain reads only the sorted positions and charges, final once
    // the cells are sorted, so on a rebuild step it also runs beside the
    // list build (issue-bound at low occupancy), not only beside the pair
    // kernel.
    if (build_list) {
        if (capturing_)
            capture_if(cond_rows_, [&](cudaStream_t cs) { launch_build_list(lc, cs); });
        else
            launch_build_list(lc, stream_);
    }
    if (!pme.empty()) {
        prof_mark(profile, "pme_spread");
        launch_pme_spread(lc, ps);
        prof_mark(profile, "pme_fft");
        launch_pme_fft(lc, ps); // convert, transforms, influence, inverse
        prof_mark(profile, "pme_gather");
        launch_pme_gather(lc, ps);
    }
    prof_mark(profile, "pair");
    launch_pair(lc, stream_);
    if (lc.any_near) {
        prof_mark(profile, "pair_fix");
        launch_pair_fix(lc, stream_);
    }
    if (side) {
        CK(cudaEventRecord(pme_join_, ps));
        CK(cudaStreamWaitEvent(stream_, pme_join_, 0));
    }
}

// Inside the step graph being captured on stream_: an IF node on handle h
// (a handle serves one node) whose body is what `body` launches (captured
// on cond_stream_), with the capture continuing after the node.
template <typename F>
void Engine::capture_if(cudaGraphConditionalHandle h, F&& body) {
    cudaStreamCaptureStatus st;
    unsigned long long id = 0;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(stream_, &st, &id, &g, &deps, &nd));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeIf;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &p));
    CK(cudaStreamBeginCaptureToGraph(cond_stream_, p.conditional.phGraph_out[0], nullptr, nullptr,
                                     0, cudaStreamCaptureModeThreadLocal));
    body(cond_stream_);
    cudaGraph_t out = nullptr;
    CK(cudaStreamEndCapture(cond_stream_, &out));
    CK(cudaStreamUpdateCaptureDependencies(stream_, &node, 1, cudaStreamSetCaptureDependencies));
}

// One step.  In the captured graph of an engine with at least
// kCondMinAtoms atoms the list-build kernels sit in two IF nodes whose
// handles k_sys_a sets when any system builds its list (reset at every
// launch): the cell sort before the PME branch forks, the list build beside
// it; on other steps they do not launch.  Measured on the B200: 262,144
// ions +0.8 %, 1,000,188 LJ atoms +7 %; but 4,000 and 10,648 atoms -13 %
// and -15 % (the conditional nodes cost more than the early-exit launches
// of a small system), hence the threshold.
void Engine::enqueue_step(bool profile) {
    if (capturing_) {
        long long atoms = 0;
        for (const auto& up : slots_)
            if (up)
                atoms += up->hp.n;
        capturing_ = atoms >= kCondMinAtoms;
    }
    if (capturing_) {
        cudaStreamCaptureStatus st;
        unsigned long long id = 0;
        cudaGraph_t g = nullptr;
        CK(cudaStreamGetCaptureInfo(stream_, &st, &id, &g, nullptr, nullptr));
        CK(cudaGraphConditionalHandleCreate(&cond_sort_, g, 0, cudaGraphCondAssignDefault));
        CK(cudaGraphConditionalHandleCreate(&cond_rows_, g, 0, cudaGraphCondAssignDefault));
    }
    prof_mark(profile, "integrate_a");
    launch_integrate_a(lc_, stream_);
    launch_sys_a(lc_, stream_, cond_sort_, cond_rows_, capturing_);
    prof_mark(profile, "neighbor");
    if (capturing_)
        capture_if(cond_sort_, [&](cudaStream_t cs) { launch_sort_cells(lc_, cs); });
    else
        launch_sort_cells(lc_, stream_);
    enqueue_forces(lc_, pme_slots_, profile, true, true);
    prof_mark(profile, "integrate_b");
    launch_integrate_b(lc_, stream_);
    launch_sys_b(lc_, stream_);
    if (lc_.any_snap) {
        prof_mark(profile, "snapshot");
        launch_snapshots(lc_, stream_);
    }
    prof_mark(profile, nullptr);
}

void Engine::prof_mark(bool profile, const char* next) {
    if (!profile)
        return;
    cudaEvent_t e;
    if (prof_used_ < prof_events_.size()) {
        e = prof_events_[prof_used_];
    } else {
        CK(cudaEventCreate(&e));
        prof_events_.push_back(e);
    }
    prof_used_++;
    CK(cudaEventRecord(e, stream_));
    prof_seq_.push_back(next ? next : "");
}

void Engine::ensure_ready() {
    if (dirty_)
        build_lists();
    if (lc_.nsys == 0)
        throw Error(ATVB_ERR_STATE, "no uploaded system to advance");
}

// Steps every Deform system can take before its cell passes the smallest
// edge its bins were planned for (with the 2 % margin of the re-plan test):
// the edge of step k is L0 (1 + rate dt k), known in advance.  Reads the
// state after the stream has drained.
constexpr int kMaxPiece = 1000; // steps between host checks within one call

int Engine::deform_budget(int n) {
    long long k = n;
    for (auto& up : slots_) {
        if (!up || !up->uploaded || up->hp.deform_axis < 0)
            continue;
        const SysParams& P = up->hp;
        const double rdt = P.deform_rate * P.dt;
        if (!(rdt < 0.0))
            continue;
        long long step = 0;
        CK(cudaMemcpy(&step, &P.st->step, sizeof(step), cudaMemcpyDeviceToHost));
        const double lo = P.npt_Lmin[P.deform_axis] * 1.02;
        const double last = std::floor((lo / P.deform_L0 - 1.0) / rdt) - (double)step - 1.0;
        k = std::min<long long>(k, last < 1.0 ? 1 : (long long)std::min(last, 1e9));
    }
    return (int)k;
}

void Engine::step(int n) { run_pieces(n, nullptr, nullptr); }

// Systems stopped by StopOnNaN: every slot's host-mapped status word
// (bit 30), read after the stream has drained.
bool Engine::all_halted() const {
    bool any = false;
    for (const auto& up : slots_) {
        if (!up || !up->uploaded)
            continue;
        any = true;
        if (!(((volatile int*)row_hint_host_)[sp_cap_ + up->index] & (1 << 30)))
            return false;
    }
    return any;
}

void Engine::check_halted(int id) {
    CK(cudaSetDevice(device_));
    CK(cudaStreamSynchronize(stream_));
    Slot* s = slot(id);
    if (!row_hint_host_ || id >= sp_cap_)
        return;
    if (((volatile int*)row_hint_host_)[sp_cap_ + id] & (1 << 30)) {
        SysState st;
        CK(cudaMemcpy(&st, s->hp.st, sizeof(st), cudaMemcpyDeviceToHost));
        throw Error(ATVB_ERR_PHYSICS, "stopped by StopOnNaN at step " +
                                          std::to_string(st.step) +
                                          ": a position or velocity is not finite");
    }
}

// Steps in pieces of at most kMaxPiece, with the host checks between them
// (row widening, cell re-plan, Deform budget), outside any timed span.
// Timed (total_ms != null): a CUDA event before each piece and after every
// step on the engine stream; step_ms (may be null) gets each step's time,
// *total_ms the sum of the pieces' spans.
void Engine::run_pieces(int n, double* step_ms, double* total_ms) {
    CK(cudaSetDevice(device_));
    if (n < 0)
        throw Error(ATVB_ERR_INVALID, "n_steps must be >= 0");
    const bool timed = total_ms != nullptr;
    if (timed && profiling_)
        throw Error(ATVB_ERR_STATE, "step_timed is not available in profiling mode");
    std::vector<cudaEvent_t> ev;
    double tot = 0.0;
    int left = n, done = 0;
    do {
        // The cell re-plan and the row check read what the previous call
        // left (the engine stream is non-blocking, so a plain copy would not
        // wait for it): a piece starts once the one before has finished.
        CK(cudaStreamSynchronize(stream_));
        if (any_npt_)
            replan_npt();
        widen_rows();
        ensure_ready();
        if (done > 0 && all_halted())
            break; // every system stopped by StopOnNaN: nothing moves
        // Long calls run in pieces of at most kMaxPiece steps, so the row
        // check and the cell re-plan above also happen inside them; a Deform
        // cell is re-planned between pieces before it shrinks out of its bins
        const int piece = std::min(left, kMaxPiece);
        const int k = any_npt_ ? deform_budget(piece) : piece;
        if (!timed) {
            run_steps(k);
        } else {
            if (comps_.empty())
                ensure_graph();
            else
                build_components();
            while ((int)ev.size() < k + 1) {
                cudaEvent_t e;
                CK(cudaEventCreate(&e));
                ev.push_back(e);
            }
            CK(cudaEventRecord(ev[0], stream_));
            for (int j = 0; j < k; ++j) {
                if (comps_.empty())
                    CK(cudaGraphLaunch(gexec_, stream_));
                else
                    enqueue_step_components();
                CK(cudaEventRecord(ev[j + 1], stream_));
            }
            CK(cudaEventSynchronize(ev[k]));
            float ms = 0.f;
            if (step_ms)
                for (int j = 0; j < k; ++j) {
                    CK(cudaEventElapsedTime(&ms, ev[j], ev[j + 1]));
                    step_ms[done + j] = ms;
                }
            CK(cudaEventElapsedTime(&ms, ev[0], ev[k]));
            tot += ms;
        }
        left -= k;
        done += k;
    } while (left > 0);
    for (auto& e : ev)
        cudaEventDestroy(e);
    if (timed)
        *total_ms = tot;
    last_launches_ = kernels_per_step() * done;
    steps_since_check_ += done;
}

void Engine::ensure_graph() {
    if (gexec_)
        return;
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    capturing_ = true;
    try {
        enqueue_step(false);
    } catch (...) {
        capturing_ = false;
        cudaGraph_t g = nullptr;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(cond_stream_, &cs) == cudaSuccess &&
            cs != cudaStreamCaptureStatusNone) {
            cudaStreamEndCapture(cond_stream_, &g); // a body capture left open
            if (g)
                cudaGraphDestroy(g);
            g = nullptr;
        }
        cudaStreamEndCapture(stream_, &g);
        if (g)
            cudaGraphDestroy(g);
        throw;
    }
    capturing_ = false;
    CK(cudaStreamEndCapture(stream_, &graph_));
    CK(cudaGraphInstantiate(&gexec_, graph_, 0));
}

void Engine::run_steps(int n) {
    if (!comps_.empty()) {
        build_components();
        for (int k = 0; k < n; ++k)
            enqueue_step_components();
        return;
    }
    if (profiling_) {
        for (int k = 0; k < n; ++k) {
            enqueue_step(true);
            CK(cudaGetLastError());
        }
        collect_profile();
    } else {
        ensure_graph();
        for (int k = 0; k < n; ++k)
            CK(cudaGraphLaunch(gexec_, stream_));
    }
}

void Engine::step_timed(int n, double* step_ms, double* total_ms) {
    double tot = 0.0;
    run_pieces(n, step_ms, &tot);
    if (total_ms)
        *total_ms = tot;
}

void Engine::collect_profile() {
    CK(cudaStreamSynchronize(stream_));
    for (size_t k = 0; k + 1 < prof_used_; ++k) {
        const std::string& name = prof_seq_[k];
        if (name.empty())
            continue;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, prof_events_[k], prof_events_[k + 1]));
        auto it = std::find_if(prof_acc_.begin(), prof_acc_.end(),
                               [&](const ProfEntry& p) { return p.name == name; });
        if (it == prof_acc_.end()) {
            prof_acc_.push_back({name, 0.0, 0});
            it = prof_acc_.end() - 1;
        }
        it->ms += ms;
        it->launches += 1;
    }
    prof_used_ = 0;
    prof_seq_.clear();
}

void Engine::compute_forces() {
    CK(cudaSetDevice(device_));
    ensure_ready();
    sized_rebuild(lc_);
    if (!comps_.empty()) {
        // Verlet::setup: the force phases of the components too
        build_components();
        run_components(ATVB_PHASE_PRE_FORCE, true);
        zero_component_sums();
        run_components(ATVB_PHASE_PRE_FORCE, false);
        run_components(ATVB_PHASE_FORCE, true);
        enqueue_forces(lc_, pme_slots_, false, false);
        run_components(ATVB_PHASE_FORCE, false);
        run_components(ATVB_PHASE_POST_FORCE, true);
        run_components(ATVB_PHASE_POST_FORCE, false);
    } else {
        enqueue_forces(lc_, pme_slots_, false, false);
    }
    launch_force_combine(lc_, stream_);
    launch_sys_energy(lc_, stream_);
    launch_npt_prep(lc_, stream_);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
}

// Force pass of one system only (a request joining a running batch): the
// other systems' forces, which may carry this step's Langevin kicks, stay.
void Engine::compute_forces_one(int id) {
    CK(cudaSetDevice(device_));
    ensure_ready();
    const LaunchCfg one = restricted_cfg(id);
    sized_rebuild(one);
    std::vector<int> pme;
    if (slot(id)->hp.has_pme)
        pme.push_back(id);
    enqueue_forces(one, pme, false, false);
    launch_force_combine(one, stream_);
    launch_sys_energy(one, stream_);
    launch_npt_prep(one, stream_);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
}

// Forced neighbour build of the systems in `lc`, repeated with larger rows
// until no row overflows.  Outside the step loop only (upload, force pass).
void Engine::sized_rebuild(const LaunchCfg& lc) {
    // row-overflow bits raised by earlier steps stay; those of the attempts
    // below are dropped with the cut lists they describe
    std::vector<int> ids(lc.nsys);
    CK(cudaMemcpy(ids.data(), lc.sys_list, sizeof(int) * lc.nsys, cudaMemcpyDeviceToHost));
    std::vector<int> before(lc.nsys);
    for (int k = 0; k < lc.nsys; ++k) {
        SysState st;
        CK(cudaMemcpy(&st, slot(ids[k])->hp.st, sizeof(st), cudaMemcpyDeviceToHost));
        before[k] = st.status & kStatusRowOverflow;
    }
    for (int attempt = 0; attempt < 4; ++attempt) {
        launch_force_rebuild(lc, stream_);
        launch_rebuild(lc, stream_);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(stream_));
        if (!check_lists(lc)) {
            for (int k = 0; k < lc.nsys; ++k)
                if (before[k]) {
                    SysState* d = slot(ids[k])->hp.st;
                    int st = 0;
                    CK(cudaMemcpy(&st, &d->status, sizeof(int), cudaMemcpyDeviceToHost));
                    st |= kStatusRowOverflow;
                    CK(cudaMemcpy(&d->status, &st, sizeof(int), cudaMemcpyHostToDevice));
                }
            return;
        }
    }
    throw Error(ATVB_ERR_OVERFLOW, "neighbour rows kept overflowing");
}

// Read each system's largest row of the last build; grow the row capacity
// of any system that overflowed.  Returns true if a rebuild is needed.
bool Engine::check_lists(const LaunchCfg& lc) {
    std::vector<int> ids(lc.nsys);
    CK(cudaMemcpy(ids.data(), lc.sys_list, sizeof(int) * lc.nsys,
                  cudaMemcpyDeviceToHost));
    bool regrow = false;
    for (int id : ids) {
        Slot* sp = slot(id);
        SysState st;
        CK(cudaMemcpy(&st, sp->hp.st, sizeof(st), cudaMemcpyDeviceToHost));
        if (st.overflow || st.max_nnbr > sp->hp.cap) {
            if (sp->row_cap_fixed > 0)
                throw Error(ATVB_ERR_OVERFLOW,
                            "neighbour rows need " + std::to_string(st.max_nnbr) +
                                " entries, above the pinned capacity " +
                                std::to_string(sp->row_cap_fixed));
            const int cap = round_up((long long)(st.max_nnbr * 1.25) + 32, 32);
            sp->alloc_list(cap);
            // the cut list is rebuilt before any force kernel reads it: the
            // row-overflow bit this build raised does not stand (one that
            // an earlier step raised is put back by sized_rebuild)
            int zero = 0;
            CK(cudaMemcpy(&sp->hp.st->overflow, &zero, sizeof(int),
                          cudaMemcpyHostToDevice));
            const int status = st.status & ~kStatusRowOverflow;
            CK(cudaMemcpy(&sp->hp.st->status, &status, sizeof(int),
                          cudaMemcpyHostToDevice));
            push_params(sp->index);
            regrow = true;
        }
        sp->max_row = st.max_nnbr;
    }
    if (regrow) {
        CK(cudaStreamSynchronize(stream_));
        release_graph();
    }
    return regrow;
}

// Work lists restricted to one system (upload / download staging).
LaunchCfg Engine::restricted_cfg(int id) {
    auto it = single_.find(id);
    if (it != single_.end() && it->second.first == list_epoch_)
        return it->second.second;
    Slot* s = slot(id);
    const SysParams& P = s->hp;
    std::vector<Item> atoms, list, cells, pair, patoms;
    for (int b = 0; b < P.n; b += kChunk)
        atoms.push_back({id, b});
    for (int b = 0; b < P.ncell; b += kListChunk)
        list.push_back({id, b});
    for (int b = 0; b < P.ncell; b += kChunk)
        cells.push_back({id, b});
    const int pchunk = kPairBlock / (P.general ? kGenLanes : s->lanes);
    for (int b = 0; b < P.n; b += pchunk)
        pair.push_back({id, b});
    if (P.has_pme)
        for (int b = 0; b < P.n; b += kChunk)
            patoms.push_back({id, b});
    LaunchCfg c = lc_;
    c.sp = d_sp_;
    c.atoms = make_list(list_allocs_, atoms, num_sms_ * 16, mem_);
    c.list = make_list(list_allocs_, list, num_sms_ * 32, mem_);
    c.cells = make_list(list_allocs_, cells, num_sms_ * 16, mem_);
    for (int p = 0; p < 2; ++p) {
        for (int k = 0; k < kLaneClasses; ++k)
            c.pair[p][k] = ItemList{};
        c.pair_gen[p] = ItemList{};
    }
    if (P.general)
        c.pair_gen[P.prec == kMixed ? 1 : 0] = make_list(list_allocs_, pair, num_sms_ * 16, mem_);
    else
        c.pair[P.prec == kMixed ? 1 : 0][lane_class(s->lanes)] =
            make_list(list_allocs_, pair, num_sms_ * 16, mem_);
    c.pme_atoms = make_list(list_allocs_, patoms, num_sms_ * 16, mem_);
    c.fft = fft_items(P.has_pme ? std::vector<int>{id} : std::vector<int>{});
    c.any_mixed = P.prec == kMixed;
    c.any_fp64 = P.prec != kMixed;
    c.any_near = P.prec == kMixed && P.has_lj && !P.general && P.mix_band_lj > 0.0;
    c.any_baro = P.baro;
    if (P.has_pme) {
        c.pme_mixed = P.prec == kMixed;
        c.pme_order = P.order;
    }
    void* p = mem_.alloc(sizeof(int));
    list_allocs_.push_back(p);
    CK(cudaMemcpyAsync(p, &id, sizeof(int), cudaMemcpyHostToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
    c.sys_list = (const int*)p;
    c.nsys = 1;
    single_[id] = {list_epoch_, c};
    return c;
}

// md::NoseHooverNPT (nose_hoover_npt.cpp:76-172): parameters checked, the
// system switched from velocity Verlet to MTK NPT, the neighbour bins
// re-planned for a breathing cell (down to 90 % of each edge, or as far as
// the minimum-image limit 2 (cutoff + skin) allows).
void Engine::set_npt(int id, const atvb_npt_desc& p) {
    Slot* sl = slot(id);
    if (sl->uploaded)
        throw Error(ATVB_ERR_STATE, "NoseHooverNPT must be set before the first upload");
    if (sl->desc.thermostat != ATVB_NVE)
        throw Error(ATVB_ERR_INVALID,
                    "NoseHooverNPT replaces the thermostat: the system must be NVE");
    if (sl->baro)
        throw Error(ATVB_ERR_INVALID, "Barostat and NoseHooverNPT cannot be combined");
    if (sl->vlimit_xmax > 0.0)
        throw Error(ATVB_ERR_INVALID, "NoseHooverNPT replaces velocity Verlet, as NVELimit does");
    if (sl->hp.deform_axis >= 0)
        throw Error(ATVB_ERR_INVALID, "Deform cannot be combined with a barostat here");
    if (p.mtchain < 1 || p.mtchain > kMaxChain || p.mpchain < 1 || p.mpchain > kMaxChain)
        throw Error(ATVB_ERR_INVALID, "NoseHooverNPT: chain lengths must be in [1, 10]");
    if (!(p.tau_T > 0.0) || !(p.tau_P > 0.0) || !(p.T_start > 0.0))
        throw Error(ATVB_ERR_INVALID, "NoseHooverNPT: T, tau_T and tau_P must be > 0");
    if (!std::isfinite(p.P_target) || !(p.drag >= 0.0))
        throw Error(ATVB_ERR_INVALID, "NoseHooverNPT: bad P_target or drag");
    SysParams& h = sl->hp;
    double shrink = 0.1;
    for (int k = 0; k < 3; ++k)
        shrink = std::min(shrink, 1.0 - 2.0 * sl->geo.rlist * (1.0 + 1e-9) / sl->geo.L[k]);
    if (shrink < 0.0)
        shrink = 0.0;
    sl->replan_cells(shrink);
    h.thermostat = kNPT;
    h.need_virial = 1; // requires_system_stress (nose_hoover_npt.cuh:79-82)
    h.n_dof = std::max(0, 3 * h.n - 3);
    h.npt_T0 = p.T_start;
    h.npt_T1 = p.T_stop < 0.0 ? p.T_start : p.T_stop;
    h.npt_tauT = p.tau_T;
    h.npt_P = p.P_target;
    h.npt_mt = p.mtchain;
    h.npt_mp = p.mpchain;
    h.npt_pdim = 0;
    for (int a = 0; a < 3; ++a) {
        h.npt_couple[a] = p.couple[a] ? 1 : 0;
        h.npt_pdim += h.npt_couple[a];
    }
    h.npt_nfirst = p.nfirst;
    h.npt_nlast = p.nlast;
    const double kT = kKB * p.T_start;
    h.npt_Qb = kT * p.tau_P * p.tau_P;
    h.npt_W = ((double)h.n_dof + 3.0) * kT * p.tau_P * p.tau_P;
    h.npt_tdrag = 1.0 - p.drag * h.dt / p.tau_T;
    h.npt_pdrag = 1.0 - p.drag * h.dt / p.tau_P;
    double cut = sl->desc.nl_cutoff;
    if (h.has_lj)
        cut = std::max(cut, sl->desc.lj_cutoff);
    if (h.has_coul)
        cut = std::max(cut, sl->desc.coul_cutoff);
    h.npt_cut = cut;
    sl->npt = true;
    sl->npt_desc = p;
    any_npt_ = true;
    push_params(id);
    dirty_ = true;
}

// md::Barostat (Berendsen, src/cpu/dynamics/barostat.cpp:22-110): beside
// velocity Verlet and any thermostat, at end_of_step; the bins are planned
// for a breathing cell as for MTK NPT.
void Engine::set_barostat(int id, double P_target, double tau_P, double bulk_modulus) {
    Slot* sl = slot(id);
    if (sl->uploaded)
        throw Error(ATVB_ERR_STATE, "Barostat must be set before the first upload");
    if (sl->npt)
        throw Error(ATVB_ERR_INVALID, "Barostat and NoseHooverNPT cannot be combined");
    if (sl->hp.deform_axis >= 0)
        throw Error(ATVB_ERR_INVALID, "Deform cannot be combined with a barostat here");
    if (!(tau_P > 0.0) || !(bulk_modulus > 0.0) || !std::isfinite(P_target))
        throw Error(ATVB_ERR_INVALID, "Barostat: tau_P and bulk_modulus must be > 0");
    SysParams& h = sl->hp;
    double shrink = 0.1;
    for (int k = 0; k < 3; ++k)
        shrink = std::min(shrink, 1.0 - 2.0 * sl->geo.rlist * (1.0 + 1e-9) / sl->geo.L[k]);
    if (shrink < 0.0)
        shrink = 0.0;
    sl->replan_cells(shrink);
    h.baro = 1;
    h.generic_drift = 1;
    h.baro_P = P_target;
    h.baro_coef = h.dt / (tau_P * bulk_modulus);
    h.need_virial = 1;
    double cut = sl->desc.nl_cutoff;
    if (h.has_lj)
        cut = std::max(cut, sl->desc.lj_cutoff);
    if (h.has_coul)
        cut = std::max(cut, sl->desc.coul_cutoff);
    h.npt_cut = cut;
    sl->baro = true;
    sl->baro_args[0] = P_target;
    sl->baro_args[1] = tau_P;
    sl->baro_args[2] = bulk_modulus;
    any_npt_ = true;
    push_params(id);
    dirty_ = true;
}

// md::Deform(axis, strain_rate, dt) (cuda/dynamics/deform.cuh): constant
// engineering strain rate along one axis, from the cell at the first upload
// (L0 > 0: from that edge, as a re-planned system keeps its original L0).
void Engine::set_deform(int id, int axis, double rate, double L0) {
    Slot* sl = slot(id);
    if (sl->uploaded)
        throw Error(ATVB_ERR_STATE, "Deform must be set before the first upload");
    if (axis < 0 || axis > 2)
        throw Error(ATVB_ERR_INVALID, "Deform: axis must be 0, 1 or 2");
    if (!std::isfinite(rate))
        throw Error(ATVB_ERR_INVALID, "Deform: bad strain rate");
    if (sl->npt || sl->baro)
        throw Error(ATVB_ERR_INVALID, "Deform cannot be combined with a barostat here");
    SysParams& h = sl->hp;
    double shrink = 0.1;
    for (int k = 0; k < 3; ++k)
        shrink = std::min(shrink, 1.0 - 2.0 * sl->geo.rlist * (1.0 + 1e-9) / sl->geo.L[k]);
    if (shrink < 0.0)
        shrink = 0.0;
    sl->replan_cells(shrink);
    h.deform_axis = axis;
    h.deform_rate = rate;
    h.deform_L0 = L0 > 0.0 ? L0 : sl->geo.L[axis];
    h.generic_drift = 1;
    sl->deform_args[0] = axis;
    sl->deform_args[1] = rate;
    sl->deform_args[2] = h.deform_L0;
    any_npt_ = true;
    push_params(id);
    dirty_ = true;
}

// Sticky status bits and the StopOnNaN halt of one system, cleared (the
// caller has dealt with the cause, e.g. restored a checkpoint).
void Engine::clear_status(int id) {
    CK(cudaSetDevice(device_));
    Slot* s = slot(id);
    CK(cudaStreamSynchronize(stream_));
    if (s->uploaded) {
        SysState st;
        CK(cudaMemcpy(&st, s->hp.st, sizeof(st), cudaMemcpyDeviceToHost));
        st.status = 0;
        st.halted = 0;
        st.nearq_lost = 0;
        CK(cudaMemcpy(s->hp.st, &st, sizeof(st), cudaMemcpyHostToDevice));
    }
    if (row_hint_host_ && id < sp_cap_)
        ((volatile int*)row_hint_host_)[sp_cap_ + id] = 0;
}

// cuda::StopOnNaN attached to (or detached from) one system.
// FixLangevin(T_start, T_stop, ...).set_run_span(nfirst, nlast)
// (fix_langevin.cpp:94-104): the setpoint moves linearly from the
// descriptor's temperature to T_stop over the steps [nfirst, nlast] and holds
// outside it; T_stop < 0 or nlast <= nfirst: the constant setpoint.
void Engine::set_langevin_ramp(int id, double T_stop, long long nfirst, long long nlast) {
    Slot* s = slot(id);
    if (s->hp.thermostat != kLangevin)
        throw Error(ATVB_ERR_INVALID, "set_langevin_ramp: the system has no FixLangevin");
    if (T_stop >= 0.0 && nlast > nfirst) {
        s->hp.lang_T1 = T_stop;
        s->hp.lang_nfirst = nfirst;
        s->hp.lang_nlast = nlast;
    } else {
        s->hp.lang_T1 = s->hp.lang_T0;
        s->hp.lang_nfirst = s->hp.lang_nlast = 0;
    }
    push_params(id);
    CK(cudaStreamSynchronize(stream_));
}

void Engine::set_stop_on_nan(int id, bool on) {
    Slot* s = slot(id);
    s->hp.stop_on_nan = on ? 1 : 0;
    push_params(id);
    CK(cudaStreamSynchronize(stream_));
}

// Capacity overrides: a pinned row length (0: automatic) and the size of
// the mixed build's near-cutoff queue (0: automatic).
void Engine::set_capacity(int id, int row_cap, int nearq_cap) {
    CK(cudaSetDevice(device_));
    if (row_cap < 0 || nearq_cap < 0)
        throw Error(ATVB_ERR_INVALID, "capacities must be >= 0");
    Slot* s = slot(id);
    CK(cudaStreamSynchronize(stream_));
    release_graph();
    s->row_cap_fixed = row_cap;
    if (row_cap > 0 && row_cap != s->hp.cap)
        s->alloc_list(row_cap); // rows are rebuilt by the next upload or build
    if (nearq_cap > 0 && s->hp.nearq) {
        s->free_alloc(s->hp.nearq);
        s->hp.nearq = (int2*)s->dalloc((size_t)nearq_cap * sizeof(int2));
        s->hp.nearq_cap = nearq_cap;
    }
    push_params(id);
    CK(cudaStreamSynchronize(stream_));
    if (s->uploaded && row_cap > 0) {
        // the old rows are gone: build into the pinned ones now
        const LaunchCfg one = restricted_cfg(id);
        launch_force_rebuild(one, stream_);
        launch_rebuild(one, stream_);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(stream_));
    }
    dirty_ = true;
}

// md::NVELimit(dt, xmax) (cuda/dynamics/nve_limit.cuh): velocity Verlet
// with each half kick's speed capped at xmax / dt.
void Engine::set_nve_limit(int id, double xmax) {
    Slot* sl = slot(id);
    if (sl->uploaded)
        throw Error(ATVB_ERR_STATE, "NVELimit must be set before the first upload");
    if (sl->npt)
        throw Error(ATVB_ERR_INVALID, "NVELimit replaces velocity Verlet, as NoseHooverNPT does");
    if (!(xmax > 0.0))
        throw Error(ATVB_ERR_INVALID, "NVELimit: xmax must be > 0");
    SysParams& h = sl->hp;
    h.vlimit = xmax / h.dt;
    h.vlimit2 = h.vlimit * h.vlimit;
    h.generic_drift = 1;
    sl->vlimit_xmax = xmax;
    push_params(id);
    dirty_ = true;
}

// PairLJCut per-type coefficients (src/cpu/potentials/pair_lj_cut.cpp:44-112
// set_type_coeff): explicit symmetric (type_i, type_j, eps, sigma) entries,
// checked here, turned into tables at upload (build_lj_tables).
void Engine::set_lj_types(int id, int ncoef, const int32_t* ti, const int32_t* tj,
                          const double* eps, const double* sigma) {
    Slot* sl = slot(id);
    if (sl->uploaded)
        throw Error(ATVB_ERR_STATE, "LJ type coefficients must be set before the first upload");
    if (!sl->hp.has_lj)
        throw Error(ATVB_ERR_INVALID, "PairLJCut is not enabled for this system");
    if (ncoef < 1 || !ti || !tj || !eps || !sigma)
        throw Error(ATVB_ERR_INVALID,
                    "PairLJCut: the per-type form needs at least one coefficient");
    int nt = 0;
    for (int k = 0; k < ncoef; ++k) {
        if (ti[k] < 0 || tj[k] < 0)
            throw Error(ATVB_ERR_INVALID, "PairLJCut::set_type_coeff: types must be >= 0");
        if (!(sigma[k] > 0.0))
            throw Error(ATVB_ERR_INVALID, "PairLJCut::set_type_coeff: sigma must be > 0");
        nt = std::max(nt, std::max(ti[k], tj[k]) + 1);
    }
    if (nt > 255)
        throw Error(ATVB_ERR_INVALID, "at most 255 LJ types");
    sl->lj_ti.assign(ti, ti + ncoef);
    sl->lj_tj.assign(tj, tj + ncoef);
    sl->lj_eps.assign(eps, eps + ncoef);
    sl->lj_sig.assign(sigma, sigma + ncoef);
    sl->ntypes = nt;
    sl->hp.general = 1;
    push_params(id);
    dirty_ = true;
}

// The type tables (pair_lj_cut.cpp:255-298 finalize_type_table_), over every
// type named by a coefficient or carried by an atom: an unset cross term
// mixes by Lorentz-Berthelot from the two diagonals (sqrt(eps_ii eps_jj),
// (sigma_ii + sigma_jj) / 2); without both diagonals the pair does not
// interact (eps = 0), so a type with no coefficient has no LJ site; every
// type pair is shifted at the common cutoff.
void Slot::build_lj_tables(const std::vector<int>& types, cudaStream_t stream) {
    int nt = ntypes;
    for (int t : types) {
        if (t < 0 || t > 254)
            throw Error(ATVB_ERR_INVALID, "atom types must be in [0, 254]");
        nt = std::max(nt, t + 1);
    }
    std::vector<double> e((size_t)nt * nt, 0.0), sg((size_t)nt * nt, 0.0);
    std::vector<char> set((size_t)nt * nt, 0);
    for (size_t k = 0; k < lj_ti.size(); ++k) {
        const size_t ab = (size_t)lj_ti[k] * nt + lj_tj[k], ba = (size_t)lj_tj[k] * nt + lj_ti[k];
        e[ab] = e[ba] = lj_eps[k];
        sg[ab] = sg[ba] = lj_sig[k];
        set[ab] = set[ba] = 1;
    }
    const double rc = desc.lj_cutoff;
    std::vector<double> tab((size_t)nt * nt * 4);
    std::vector<float> tabf(tab.size());
    for (int a = 0; a < nt; ++a)
        for (int b = 0; b < nt; ++b) {
            const size_t ab = (size_t)a * nt + b;
            double ee = e[ab], ss = sg[ab];
            if (!set[ab]) {
                const size_t aa = (size_t)a * nt + a, bb = (size_t)b * nt + b;
                if (set[aa] && set[bb]) {
                    ee = std::sqrt(e[aa] * e[bb]);
                    ss = 0.5 * (sg[aa] + sg[bb]);
                } else {
                    ee = 0.0;
                    ss = 1.0;
                }
            }
            const double s2 = ss * ss, s6 = s2 * s2 * s2;
            const double r2inv = 1.0 / (rc * rc);
            const double r6inv = r2inv * r2inv * r2inv * s6;
            const double v[4] = {s6, 4.0 * ee, 24.0 * ee, 4.0 * ee * (r6inv * r6inv - r6inv)};
            for (int q = 0; q < 4; ++q) {
                tab[ab * 4 + q] = v[q];
                tabf[ab * 4 + q] = (float)v[q];
            }
        }
    double* dt = (double*)dalloc(tab.size() * sizeof(double));
    float* dtf = (float*)dalloc(tabf.size() * sizeof(float));
    int* dtype = (int*)dalloc((size_t)hp.n * sizeof(int));
    CK(cudaMemcpyAsync(dt, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice,
                       stream));
    CK(cudaMemcpyAsync(dtf, tabf.data(), tabf.size() * sizeof(float), cudaMemcpyHostToDevice,
                       stream));
    CK(cudaMemcpyAsync(dtype, types.data(), (size_t)hp.n * sizeof(int), cudaMemcpyHostToDevice,
                       stream));
    CK(cudaStreamSynchronize(stream));
    hp.lj_tab = dt;
    hp.lj_tabf = dtf;
    hp.type = dtype;
    hp.stype = (unsigned char*)dalloc((size_t)hp.n);
    hp.ntypes = nt;
}

// PairLJCut / CoulLong set_special_bonds(s12, s13, s14) with the bond
// topology: partners 1, 2 and 3 bonds away (the nearest distance wins) get
// the scales of their class; built at upload from the tags.
void Engine::set_special_bonds(int id, const double lj[3], const double coul[3],
                               int64_t nbonds, const int64_t* a, const int64_t* b) {
    Slot* sl = slot(id);
    if (sl->uploaded)
        throw Error(ATVB_ERR_STATE, "special bonds must be set before the first upload");
    if (nbonds < 0 || (nbonds > 0 && (!a || !b)))
        throw Error(ATVB_ERR_INVALID, "special bonds: bad bond list");
    for (int k = 0; k < 3; ++k) {
        if (!(lj[k] >= 0.0 && lj[k] <= 1.0) || !(coul[k] >= 0.0 && coul[k] <= 1.0))
            throw Error(ATVB_ERR_INVALID, "special bond scales must be in [0, 1]");
        sl->sp_lj[k] = lj[k];
        sl->sp_coul[k] = coul[k];
    }
    sl->bond_a.assign(a, a + nbonds);
    sl->bond_b.assign(b, b + nbonds);
    sl->special_set = true;
    sl->hp.general = 1;
    push_params(id);
    dirty_ = true;
}

void Slot::build_specials(const std::vector<long long>& tags, cudaStream_t stream) {
    const int n = hp.n;
    std::unordered_map<long long, int> idx;
    idx.reserve((size_t)n * 2);
    for (int i = 0; i < n; ++i)
        idx[tags[i]] = i;
    std::vector<std::vector<int>> adj(n);
    for (size_t k = 0; k < bond_a.size(); ++k) {
        auto ia = idx.find(bond_a[k]), ib = idx.find(bond_b[k]);
        if (ia == idx.end() || ib == idx.end() || ia->second == ib->second)
            throw Error(ATVB_ERR_INVALID, "special bonds: a bond names an unknown atom tag");
        adj[ia->second].push_back(ib->second);
        adj[ib->second].push_back(ia->second);
    }
    std::vector<int> first(n + 1, 0), js;
    std::vector<unsigned char> cls;
    std::vector<int> depth(n, -1), touched;
    for (int i = 0; i < n; ++i) {
        first[i] = (int)js.size();
        std::vector<int> frontier = {i};
        depth[i] = 0;
        touched.assign(1, i);
        std::vector<std::pair<int, int>> found;
        for (int d = 1; d <= 3; ++d) {
            std::vector<int> next;
            for (int u : frontier)
                for (int v : adj[u])
                    if (depth[v] < 0) {
                        depth[v] = d;
                        touched.push_back(v);
                        next.push_back(v);
                        if (sp_lj[d - 1] != 1.0 || sp_coul[d - 1] != 1.0)
                            found.push_back({v, d});
                    }
            frontier.swap(next);
        }
        for (int v : touched)
            depth[v] = -1;
        std::sort(found.begin(), found.end());
        for (auto& f : found) {
            js.push_back(f.first);
            cls.push_back((unsigned char)f.second);
        }
    }
    first[n] = (int)js.size();
    int* d_first = (int*)dalloc(first.size() * sizeof(int));
    int* d_j = (int*)dalloc(std::max<size_t>(js.size(), 1) * sizeof(int));
    unsigned char* d_c = (unsigned char*)dalloc(std::max<size_t>(cls.size(), 1));
    CK(cudaMemcpyAsync(d_first, first.data(), first.size() * sizeof(int),
                       cudaMemcpyHostToDevice, stream));
    if (!js.empty()) {
        CK(cudaMemcpyAsync(d_j, js.data(), js.size() * sizeof(int), cudaMemcpyHostToDevice,
                           stream));
        CK(cudaMemcpyAsync(d_c, cls.data(), cls.size(), cudaMemcpyHostToDevice, stream));
    }
    CK(cudaStreamSynchronize(stream));
    hp.sp_first = d_first;
    hp.sp_j = d_j;
    hp.sp_cls = d_c;
    hp.has_special = 1;
    hp.sp_lj[0] = hp.sp_coul[0] = 1.0;
    for (int k = 0; k < 3; ++k) {
        hp.sp_lj[k + 1] = sp_lj[k];
        hp.sp_coul[k + 1] = sp_coul[k];
    }
}

void Engine::upload(int id, const atvb_soa_view& f) {
    CK(cudaSetDevice(device_));
    Slot* s = slot(id);
    const int n = s->hp.n;
    const size_t b = sizeof(double) * n;
    std::vector<double> tmp;
    auto put = [&](double* dst, const double* src, double fill) {
        if (src) {
            CK(cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, stream_));
        } else {
            tmp.assign(n, fill);
            CK(cudaMemcpyAsync(dst, tmp.data(), b, cudaMemcpyHostToDevice,
                               stream_));
            CK(cudaStreamSynchronize(stream_));
        }
    };
    if (!f.x || !f.y || !f.z)
        throw Error(ATVB_ERR_INVALID, "upload needs positions");
    put(s->hp.x, f.x, 0.0);
    put(s->hp.y, f.y, 0.0);
    put(s->hp.z, f.z, 0.0);
    put(s->hp.vx, f.vx, 0.0);
    put(s->hp.vy, f.vy, 0.0);
    put(s->hp.vz, f.vz, 0.0);
    put(s->hp.mass, f.mass, 1.0);
    put(s->hp.q, f.charge, 0.0);
    put(s->hp.sx, f.fx, 0.0);
    put(s->hp.sy, f.fy, 0.0);
    put(s->hp.sz, f.fz, 0.0);
    if (f.mass)
        for (int i = 0; i < n; ++i)
            if (!(f.mass[i] > 0.0))
                throw Error(ATVB_ERR_INVALID, "masses must be positive");
    std::vector<long long> tag(n);
    for (int i = 0; i < n; ++i)
        tag[i] = f.tag ? f.tag[i] : (long long)(i + 1);
    CK(cudaMemcpyAsync(s->hp.tag, tag.data(), 8 * n, cudaMemcpyHostToDevice,
                       stream_));
    if (s->ntypes > 0) {
        std::vector<int> ty(n, 0);
        if (f.type)
            for (int i = 0; i < n; ++i)
                ty[i] = f.type[i];
        s->build_lj_tables(ty, stream_);
    }
    if (s->special_set)
        s->build_specials(tag, stream_);
    // charges: PME self + net-charge constants (pme.cpp:224-252)
    double qs = 0, q2 = 0;
    if (f.charge)
        for (int i = 0; i < n; ++i) {
            qs += f.charge[i];
            q2 += f.charge[i] * f.charge[i];
        }
    {
        double qm = 0.0;
        if (f.charge)
            for (int i = 0; i < n; ++i)
                qm = std::max(qm, std::fabs(f.charge[i]));
        s->hp.force_r2_safe = force_safe_r2(s->hp, qm * qm);
    }
    if (s->hp.has_pme) {
        const double vol = s->hp.L[0] * s->hp.L[1] * s->hp.L[2];
        const double a = s->desc.pme_alpha;
        s->hp.e_const = -kQqr2e * a / std::sqrt(kPi) * q2 -
                        kQqr2e * kPi / (2.0 * vol * a * a) * qs * qs;
        s->hp.pme_eself = -kQqr2e * a / std::sqrt(kPi) * q2;
        s->hp.pme_qsum2 = qs * qs;
    }
    SysState st0;
    std::memset(&st0, 0, sizeof(st0));
    st0.vscale = 1.0;
    st0.s_a = 1.0;
    for (int k = 0; k < 3; ++k) {
        st0.box[k] = s->hp.L[k];
        st0.Lb[k] = st0.Lnext[k] = s->hp.L[k];
        st0.Lb_inv[k] = 1.0 / s->hp.L[k];
        st0.vs[k] = st0.vs_out[k] = 1.0;
        // drift factors of a cell that does not move (the Berendsen
        // barostat's first step; MTK NPT prepares its own)
        st0.npt_a[k] = st0.npt_drift[k] = 1.0;
        st0.fixn_scale[k] = s->hp.fix_scale[k];
        st0.fixn64_scale[k] = s->hp.fix64_scale[k];
        st0.ub[k] = 1.0;
    }
    st0.mu = 1.0;
    {
        const double thr = 0.5 * (s->hp.rlist - s->hp.npt_cut);
        st0.disp_thr2 = thr > 0.0 ? thr * thr : -1.0;
    }
    CK(cudaMemcpyAsync(s->hp.st, &st0, sizeof(st0), cudaMemcpyHostToDevice,
                       stream_));
    push_params(id);
    CK(cudaStreamSynchronize(stream_));
    if (row_hint_host_ && id < sp_cap_)
        ((volatile int*)row_hint_host_)[sp_cap_ + id] = 0; // a fresh state: no status
    s->uploaded = true;
    s->snap_read = 0; // the published snapshot count restarts with the state
    dirty_ = true;
    build_lists();
    // wrap, first neighbour build, uploaded forces into sorted order, KE --
    // touching only this system
    const LaunchCfg one = restricted_cfg(id);
    launch_wrap_in(one, stream_);
    sized_rebuild(one);
    launch_state_in(one, stream_);
    launch_kinetic(one, stream_);
    launch_npt_prep(one, stream_);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    // the forced build counts as the setup build, not a step rebuild
    long long zero = 0;
    CK(cudaMemcpy(&s->hp.st->rebuilds, &zero, sizeof(zero),
                  cudaMemcpyHostToDevice));
    SysState st;
    CK(cudaMemcpy(&st, s->hp.st, sizeof(st), cudaMemcpyDeviceToHost));
    s->mean_row = st.max_nnbr;
    dirty_ = true; // lane choice may change with the measured row length
}

void Engine::scalars(int id, atvb_scalars* out) {
    CK(cudaSetDevice(device_));
    Slot* s = slot(id);
    SysState st;
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&st, s->hp.st, sizeof(st), cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    out->energy = st.energy;
    out->energy_pair = st.energy;
    out->energy_lj = st.e_lj;
    out->energy_coul = st.e_coul;
    out->energy_recip = st.e_recip;
    out->energy_const = st.e_const;
    out->kinetic = st.kinetic;
    out->conserved = st.conserved;
    for (int k = 0; k < 6; ++k)
        out->stress[k] = st.virial[k];
    out->nh_xi = st.xi;
    out->step = st.step;
    out->rebuilds = st.rebuilds;
    out->max_neighbors = st.max_nnbr;
    out->status_bits = (uint32_t)st.status;
    out->halted = st.halted;
    out->status = (st.status & kStatusRowOverflow)
                      ? ATVB_ERR_OVERFLOW
                      : ((st.status & kStatusBoxRange) ? ATVB_ERR_STATE
                                                        : (st.status ? ATVB_ERR_PHYSICS : 0));
    out->list_pairs = (int64_t)(st.list_entries / 2);
    for (int k = 0; k < 3; ++k)
        out->box[k] = st.box[k];
    out->pressure = st.pressure;
}

void Engine::download(int id, atvb_soa_view* f, atvb_scalars* sc) {
    CK(cudaSetDevice(device_));
    Slot* s = slot(id);
    if (!s->uploaded)
        throw Error(ATVB_ERR_STATE, "download before upload");
    const int n = s->hp.n;
    const size_t b = sizeof(double) * n;
    ensure_ready();
    const LaunchCfg one = restricted_cfg(id);
    if (f) {
        if (f->x)
            CK(cudaMemcpyAsync(f->x, s->hp.x, b, cudaMemcpyDeviceToHost, stream_));
        if (f->y)
            CK(cudaMemcpyAsync(f->y, s->hp.y, b, cudaMemcpyDeviceToHost, stream_));
        if (f->z)
            CK(cudaMemcpyAsync(f->z, s->hp.z, b, cudaMemcpyDeviceToHost, stream_));
        if (f->mass)
            CK(cudaMemcpyAsync(f->mass, s->hp.mass, b, cudaMemcpyDeviceToHost,
                               stream_));
        if (f->charge)
            CK(cudaMemcpyAsync(f->charge, s->hp.q, b, cudaMemcpyDeviceToHost,
                               stream_));
        if (f->fx || f->fy || f->fz) {
            launch_state_out(one, 0, stream_);
            if (f->fx)
                CK(cudaMemcpyAsync(f->fx, s->hp.sx, b, cudaMemcpyDeviceToHost,
                                   stream_));
            if (f->fy)
                CK(cudaMemcpyAsync(f->fy, s->hp.sy, b, cudaMemcpyDeviceToHost,
                                   stream_));
            if (f->fz)
                CK(cudaMemcpyAsync(f->fz, s->hp.sz, b, cudaMemcpyDeviceToHost,
                                   stream_));
        }
        if (f->vx || f->vy || f->vz) {
            launch_state_out(one, 1, stream_);
            if (f->vx)
                CK(cudaMemcpyAsync(f->vx, s->hp.sx, b, cudaMemcpyDeviceToHost,
                                   stream_));
            if (f->vy)
                CK(cudaMemcpyAsync(f->vy, s->hp.sy, b, cudaMemcpyDeviceToHost,
                                   stream_));
            if (f->vz)
                CK(cudaMemcpyAsync(f->vz, s->hp.sz, b, cudaMemcpyDeviceToHost,
                                   stream_));
        }
        if (f->tag) {
            std::vector<long long> t(n);
            CK(cudaMemcpyAsync(t.data(), s->hp.tag, 8 * n,
                               cudaMemcpyDeviceToHost, stream_));
            CK(cudaStreamSynchronize(stream_));
            for (int i = 0; i < n; ++i)
                f->tag[i] = t[i];
        }
    }
    CK(cudaStreamSynchronize(stream_));
    if (sc)
        scalars(id, sc);
}

int64_t Engine::pairs(int id, int32_t* pi, int32_t* pj, int64_t capacity) {
    CK(cudaSetDevice(device_));
    Slot* s = slot(id);
    const int n = s->hp.n, cap = s->hp.cap;
    std::vector<int> perm(n), nn(n), nbr((size_t)n * cap);
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(perm.data(), s->hp.perm, 4 * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(nn.data(), s->hp.nnbr, 4 * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(nbr.data(), s->hp.nbr, 4 * (size_t)n * cap,
                  cudaMemcpyDeviceToHost));
    int64_t cnt = 0;
    for (int a = 0; a < n; ++a)
        for (int k = 0; k < nn[a]; ++k) {
            const int i = perm[a], j = perm[nbr[(size_t)a * cap + k] & (int)kRowIdxMask];
            if (i < j) {
                if (pi && pj && cnt < capacity) {
                    pi[cnt] = i;
                    pj[cnt] = j;
                }
                ++cnt;
            }
        }
    return cnt;
}

int Engine::history(int id, double* out, int max_steps) {
    Slot* s = slot(id);
    SysState st;
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&st, s->hp.st, sizeof(st), cudaMemcpyDeviceToHost));
    const int cap = s->hp.ehist_cap;
    std::vector<double> ring(3 * (size_t)cap);
    CK(cudaMemcpy(ring.data(), s->hp.ehist, ring.size() * 8,
                  cudaMemcpyDeviceToHost));
    const long long total = st.step;
    const long long avail = std::min<long long>(total, cap);
    const long long cnt = std::min<long long>(avail, max_steps);
    for (long long k = 0; k < cnt; ++k) {
        const long long stepk = total - cnt + k;
        const long long slotk = stepk % cap;
        for (int c = 0; c < 3; ++c)
            out[3 * k + c] = ring[3 * slotk + c];
    }
    return (int)cnt;
}

void Engine::set_lanes(int lanes) {
    if (lanes != 0 && lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 &&
        lanes != 16 && lanes != 32)
        throw Error(ATVB_ERR_INVALID, "lanes must be 0 or a power of two <= 32");
    lanes_fixed_ = lanes;
    dirty_ = true;
}

// Project-written autotuner: time the pair kernel for every lane count on
// the engine's own systems and keep the fastest.
int Engine::autotune() {
    CK(cudaSetDevice(device_));
    ensure_ready();
    const int cands[6] = {1, 2, 4, 8, 16, 32};
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_g = 4;
    const int saved = lanes_fixed_;
    for (int g : cands) {
        lanes_fixed_ = g;
        build_lists();
        for (int w = 0; w < 2; ++w)
            launch_pair(lc_, stream_);
        CK(cudaEventRecord(e0, stream_));
        const int reps = 5;
        for (int r = 0; r < reps; ++r)
            launch_pair(lc_, stream_);
        CK(cudaEventRecord(e1, stream_));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            best_g = g;
        }
    }
    (void)saved;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    lanes_fixed_ = best_g;
    build_lists();
    // the timing runs polluted the energy accumulators: recompute
    compute_forces();
    return best_g;
}

} // namespace atvb

// ------------------------------------------------------------ checkpoints
//
// A checkpoint is the whole resumable state of one system: the master atom
// arrays (original order, raw velocities), the forces of the last force
// pass, the positions and cell of the last neighbour build, and the
// device-side SysState (thermostat / barostat chains, pending velocity
// scales, step and list counters).  Restoring rebuilds the neighbour list
// from the positions of the last build, so the rows, their order and the
// lane count are those of the saved run: continuing gives the same
// trajectory, bit for bit, as never stopping.

namespace atvb {

namespace {
constexpr char kCkptMagic[8] = {'A', 'T', 'V', 'B', 'C', 'K', 'P', '1'};
constexpr uint32_t kCkptVersion = 2;

struct CkptHeader {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    int32_t n;
    int32_t precision;
    int32_t thermostat;
    int32_t ntypes;
    int64_t state_bytes;
    double mean_row;
    double reserved[4];
};

// per-atom double arrays: x y z vx vy vz fx fy fz xr yr zr mass q
constexpr int kCkptArrays = 14;
} // namespace

size_t Engine::checkpoint_bytes(int id) {
    Slot* s = slot(id);
    const size_t n = (size_t)s->hp.n;
    return sizeof(CkptHeader) + sizeof(SysState) + n * (kCkptArrays * 8 + 8) +
           (s->ntypes > 0 ? n * 4 : 0);
}

void Engine::save(int id, void* buf, size_t cap) {
    CK(cudaSetDevice(device_));
    Slot* s = slot(id);
    if (!s->uploaded)
        throw Error(ATVB_ERR_STATE, "checkpoint before upload");
    const size_t need = checkpoint_bytes(id);
    if (!buf || cap < need)
        throw Error(ATVB_ERR_INVALID, "checkpoint buffer smaller than atvb_*_checkpoint_size");
    ensure_ready();
    const LaunchCfg one = restricted_cfg(id);
    const SysParams& P = s->hp;
    const size_t n = (size_t)P.n, b = n * 8;
    char* p = (char*)buf;
    CkptHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = kCkptVersion;
    h.header_bytes = sizeof(CkptHeader);
    h.n = P.n;
    h.precision = P.prec;
    h.thermostat = P.thermostat;
    h.ntypes = s->ntypes;
    h.state_bytes = sizeof(SysState);
    h.mean_row = s->mean_row;
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    CK(cudaMemcpyAsync(p, P.st, sizeof(SysState), cudaMemcpyDeviceToHost, stream_));
    p += sizeof(SysState);
    const double* src[6] = {P.x, P.y, P.z, P.vx, P.vy, P.vz};
    for (const double* a : src) {
        CK(cudaMemcpyAsync(p, a, b, cudaMemcpyDeviceToHost, stream_));
        p += b;
    }
    launch_state_out(one, 0, stream_); // forces, original order
    for (const double* a : {P.sx, P.sy, P.sz}) {
        CK(cudaMemcpyAsync(p, a, b, cudaMemcpyDeviceToHost, stream_));
        p += b;
    }
    for (const double* a : {P.xr, P.yr, P.zr, P.mass, P.q}) {
        CK(cudaMemcpyAsync(p, a, b, cudaMemcpyDeviceToHost, stream_));
        p += b;
    }
    CK(cudaMemcpyAsync(p, P.tag, b, cudaMemcpyDeviceToHost, stream_));
    p += b;
    if (s->ntypes > 0)
        CK(cudaMemcpyAsync(p, P.type, n * 4, cudaMemcpyDeviceToHost, stream_));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
}

void Engine::restore(int id, const void* buf, size_t size, bool fresh_list) {
    CK(cudaSetDevice(device_));
    Slot* s = slot(id);
    if (s->uploaded)
        throw Error(ATVB_ERR_STATE, "restore into a system that was already uploaded");
    if (!buf || size < sizeof(CkptHeader))
        throw Error(ATVB_ERR_INVALID, "checkpoint too short");
    CkptHeader h;
    std::memcpy(&h, buf, sizeof(h));
    if (std::memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != kCkptVersion ||
        h.header_bytes != sizeof(CkptHeader) || h.state_bytes != (int64_t)sizeof(SysState))
        throw Error(ATVB_ERR_INVALID, "not a checkpoint of this library version");
    SysParams& P = s->hp;
    if (h.n != P.n || h.precision != P.prec || h.thermostat != P.thermostat ||
        h.ntypes != s->ntypes)
        throw Error(ATVB_ERR_INVALID,
                    "checkpoint does not match the system (atoms, precision, "
                    "integrator or LJ types)");
    if (size < checkpoint_bytes(id))
        throw Error(ATVB_ERR_INVALID, "checkpoint too short");
    const size_t n = (size_t)P.n;
    const char* p = (const char*)buf + sizeof(CkptHeader);
    SysState st;
    std::memcpy(&st, p, sizeof(st));
    p += sizeof(SysState);
    if (!fresh_list)
        st.snap_count = 0; // snapshot rings belong to the running process
    st.snap_slot = -1;
    const double* a[kCkptArrays];
    for (int k = 0; k < kCkptArrays; ++k) {
        a[k] = (const double*)p;
        p += n * 8;
    }
    const int64_t* tag = (const int64_t*)p;
    p += n * 8;
    std::vector<int32_t> type;
    if (s->ntypes > 0) {
        type.resize(n);
        std::memcpy(type.data(), p, n * 4);
    }
    // 1. the positions and cell of the last neighbour build: the upload's
    //    list build then reproduces the saved run's list (fresh_list: a new
    //    list from the current positions in the current cell instead)
    if (s->npt || s->baro || P.deform_axis >= 0)
        apply_box(P, fresh_list ? st.box : st.Lb, true);
    const int bx = fresh_list ? 0 : 9;
    atvb_soa_view v;
    std::memset(&v, 0, sizeof(v));
    v.x = const_cast<double*>(a[bx]);
    v.y = const_cast<double*>(a[bx + 1]);
    v.z = const_cast<double*>(a[bx + 2]);
    v.vx = const_cast<double*>(a[3]);
    v.vy = const_cast<double*>(a[4]);
    v.vz = const_cast<double*>(a[5]);
    v.fx = const_cast<double*>(a[6]);
    v.fy = const_cast<double*>(a[7]);
    v.fz = const_cast<double*>(a[8]);
    v.mass = const_cast<double*>(a[12]);
    v.charge = const_cast<double*>(a[13]);
    v.tag = const_cast<int64_t*>(tag);
    v.type = type.empty() ? nullptr : type.data();
    upload(id, v);
    // 2. the current cell, positions and state
    if (s->npt || s->baro || P.deform_axis >= 0) {
        apply_box(P, st.box, true);
        CK(cudaMemcpyAsync(d_sp_ + id, &P, sizeof(SysParams), cudaMemcpyHostToDevice,
                           stream_));
    }
    const size_t b = n * 8;
    CK(cudaMemcpyAsync(P.x, a[0], b, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(P.y, a[1], b, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(P.z, a[2], b, cudaMemcpyHostToDevice, stream_));
    if (fresh_list) {
        // the list was built now, from the current positions and cell
        for (int d = 0; d < 3; ++d) {
            st.Lb[d] = st.box[d];
            st.Lb_inv[d] = 1.0 / st.box[d];
        }
        double lam = 1e300;
        for (int d = 0; d < 3; ++d) {
            st.ub[d] = st.Lb[d] / st.Lnext[d];
            lam = std::min(lam, st.Lnext[d] / st.Lb[d]);
        }
        const double thr = 0.5 * (P.rlist - P.npt_cut / lam);
        st.disp_thr2 = thr > 0.0 ? thr * thr : -1.0;
        st.need_rebuild = thr > 0.0 ? 0 : 1;
        st.ago = 0;
        st.held = 0; // the new bins cover the current cell (the sticky bit stays)
    } else {
        CK(cudaMemcpyAsync(P.xr, a[9], b, cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync(P.yr, a[10], b, cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync(P.zr, a[11], b, cudaMemcpyHostToDevice, stream_));
    }
    const LaunchCfg one = restricted_cfg(id);
    launch_repack(one, stream_);
    if (fresh_list) {
        // keep the list statistics of the build just made
        SysState cur;
        CK(cudaStreamSynchronize(stream_)); // the stream does not block a plain copy
        CK(cudaMemcpy(&cur, P.st, sizeof(cur), cudaMemcpyDeviceToHost));
        st.max_nnbr = cur.max_nnbr;
        st.list_entries = cur.list_entries;
        st.overflow = cur.overflow;
        st.rebuilds += 1;
    }
    CK(cudaMemcpyAsync(P.st, &st, sizeof(st), cudaMemcpyHostToDevice, stream_));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    if (!fresh_list)
        s->mean_row = h.mean_row;
    dirty_ = true;
}

// MTK NPT systems whose cell has moved close to the edge of the range their
// bins were planned for (or far beyond it, where the bins grow coarse) are
// re-planned between step calls, as the reference re-derives its grid and
// PME mesh when the cell changes (pme.cpp:64-131): checkpoint, a new slot
// for the current cell with the same configuration, restore with a new
// list.  The trajectory continues (not bit for bit: the new bins order the
// list differently).
void Engine::replan_npt() {
    for (auto& up : slots_) {
        if (!up || !(up->npt || up->baro || up->hp.deform_axis >= 0) || !up->uploaded)
            continue;
        Slot* old = up.get();
        SysState st;
        CK(cudaMemcpy(&st, old->hp.st, sizeof(st), cudaMemcpyDeviceToHost));
        bool need = st.held != 0;
        for (int k = 0; k < 3; ++k) {
            const double lo = old->hp.npt_Lmin[k], plan = old->geo.L[k];
            if (st.Lnext[k] < lo * 1.02 || st.Lnext[k] > plan * 1.25)
                need = true;
        }
        if (!need)
            continue;
        const int id = old->index;
        std::vector<char> blob(checkpoint_bytes(id));
        save(id, blob.data(), blob.size());
        atvb_system_desc d = old->desc;
        for (int k = 0; k < 9; ++k)
            d.box[k] = 0.0;
        for (int k = 0; k < 3; ++k)
            d.box[4 * k] = st.box[k];
        auto s = std::make_unique<Slot>(d, mem_);
        s->index = id;
        s->ntypes = old->ntypes;
        s->lj_ti = old->lj_ti;
        s->lj_tj = old->lj_tj;
        s->lj_eps = old->lj_eps;
        s->lj_sig = old->lj_sig;
        s->special_set = old->special_set;
        for (int k = 0; k < 3; ++k) {
            s->sp_lj[k] = old->sp_lj[k];
            s->sp_coul[k] = old->sp_coul[k];
        }
        s->bond_a = old->bond_a;
        s->bond_b = old->bond_b;
        s->hp.general = old->hp.general;
        // the snapshot ring moves over with its read position
        s->snap_host = old->snap_host;
        s->snap_read = old->snap_read;
        s->hp.snap_ring = old->hp.snap_ring;
        s->hp.snap_every = old->hp.snap_every;
        s->hp.snap_depth = old->hp.snap_depth;
        s->hp.snap_slot_bytes = old->hp.snap_slot_bytes;
        old->snap_host = nullptr;
        const atvb_npt_desc npt = old->npt_desc;
        const bool was_npt = old->npt, was_baro = old->baro;
        const double vx = old->vlimit_xmax;
        const bool was_def = old->hp.deform_axis >= 0;
        const double da[3] = {old->deform_args[0], old->deform_args[1], old->deform_args[2]};
        const double ba[3] = {old->baro_args[0], old->baro_args[1], old->baro_args[2]};
        CK(cudaStreamSynchronize(stream_));
        release_graph();
        up = std::move(s);
        push_params(id);
        if (was_npt)
            set_npt(id, npt);
        if (was_baro)
            set_barostat(id, ba[0], ba[1], ba[2]);
        if (vx > 0.0)
            set_nve_limit(id, vx);
        if (was_def)
            set_deform(id, (int)da[0], da[1], da[2]);
        restore(id, blob.data(), blob.size(), true);
    }
}

} // namespace atvb

// ------------------------------------------------------ trajectory snapshots

namespace atvb {

void Engine::set_snapshots(int id, int every, int depth) {
    CK(cudaSetDevice(device_));
    Slot* s = slot(id);
    if (every < 0 || (every > 0 && (depth < 1 || depth > 4096)))
        throw Error(ATVB_ERR_INVALID, "snapshots: every >= 0 and depth in [1, 4096]");
    CK(cudaStreamSynchronize(stream_));
    release_graph();
    if (s->snap_host) {
        CK(cudaFreeHost(s->snap_host));
        s->snap_host = nullptr;
    }
    SysParams& P = s->hp;
    P.snap_ring = nullptr;
    P.snap_every = 0;
    P.snap_depth = 0;
    if (every > 0) {
        const size_t slot_bytes = sizeof(SnapHeader) + (size_t)P.n * 6 * sizeof(double);
        void* h = nullptr;
        CK(cudaHostAlloc(&h, slot_bytes * depth, cudaHostAllocMapped));
        std::memset(h, 0, slot_bytes * depth);
        void* d = nullptr;
        CK(cudaHostGetDevicePointer(&d, h, 0));
        s->snap_host = (char*)h;
        P.snap_ring = (char*)d;
        P.snap_every = every;
        P.snap_depth = depth;
        P.snap_slot_bytes = (long long)slot_bytes;
    }
    // the published count restarts with the ring
    s->snap_read = 0;
    if (s->uploaded) {
        const long long zero = 0;
        CK(cudaMemcpy(&P.st->snap_count, &zero, sizeof(zero), cudaMemcpyHostToDevice));
    }
    push_params(id);
    dirty_ = true;
}

// Frames published since the last poll, oldest first, without waiting for
// the device: a slot is taken when its seqlock shows the expected sequence
// number before and after the copy; frames overwritten before they were
// read are counted as dropped.
int Engine::poll_snapshots(int id, int max_frames, int64_t* steps, double* box,
                           double* const out[6], int64_t* dropped) {
    Slot* s = slot(id);
    if (!s->snap_host)
        throw Error(ATVB_ERR_STATE, "snapshots are not enabled for this system");
    const SysParams& P = s->hp;
    const size_t n = (size_t)P.n, sb = (size_t)P.snap_slot_bytes;
    int got = 0;
    int64_t lost = 0;
    while (got < max_frames) {
        const long long want = s->snap_read + 1;
        const char* base = s->snap_host + (size_t)((want - 1) % P.snap_depth) * sb;
        const volatile SnapHeader* h = (const volatile SnapHeader*)base;
        const long long end = h->end;
        if (end < want)
            break; // not published yet
        if (end > want) {
            // overwritten: skip to the oldest frame the ring still holds
            const long long oldest = std::max(want + 1, end - P.snap_depth + 1);
            lost += oldest - want;
            s->snap_read = oldest - 1;
            continue;
        }
        std::atomic_thread_fence(std::memory_order_acquire);
        const int64_t step = h->step;
        double bx[3] = {h->box[0], h->box[1], h->box[2]};
        const double* d = (const double*)(base + sizeof(SnapHeader));
        for (int f = 0; f < 6; ++f)
            if (out[f])
                std::memcpy(out[f] + (size_t)got * n, d + (size_t)f * n, n * sizeof(double));
        std::atomic_thread_fence(std::memory_order_acquire);
        if (h->begin != want) {
            // overwritten while copying
            lost += 1;
            s->snap_read = want;
            continue;
        }
        if (steps)
            steps[got] = step;
        if (box)
            for (int a = 0; a < 3; ++a)
                box[3 * got + a] = bx[a];
        ++got;
        s->snap_read = want;
    }
    if (dropped)
        *dropped = lost;
    return got;
}

} // namespace atvb
