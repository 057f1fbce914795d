// atvb_common.cuh -- device-side data model shared by every kernel.
//
// One MD system lives in one slot of an Engine.  All per-system device
// pointers and constants sit in a SysParams record in device memory; every
// kernel walks a flat list of work items {system, first atom} so that one
// launch covers any number of systems (the single-system path is a batch of
// one).  Per-atom master state (x, v, mass, charge, tag) is kept in the
// caller's original order; the force kernels work on a cell-sorted copy of
// the positions (pos4) whose order is rebuilt with the neighbour list.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "atvb.h"

namespace atvb {

// units.h:138,165,166,173 of the reference (metal units)
constexpr double kKB = 8.617333262e-5;
constexpr double kFtm2v = 1.0 / 103.6427;
constexpr double kMvv2e = 103.6427;
constexpr double kQqr2e = 14.399645;
constexpr double kPi = 3.14159265358979323846;
constexpr double kEwaldF = 1.1283791670955126; // 2/sqrt(pi)

enum Precision : int { kFP64 = 0, kMixed = 1 };
enum Thermostat : int { kNVE = 0, kNoseHoover = 1, kLangevin = 2, kNPT = 3 };

// longest Nose-Hoover chain of the MTK NPT integrator
constexpr int kMaxChain = 10;
// most radices of one PME mesh axis (4, 2, 3, 5, 7)
constexpr int kFftMaxFac = 16;

// SysState::status bits (sticky; the ATVB_STATUS_* values of atvb.h)
constexpr int kStatusRowOverflow = ATVB_STATUS_ROW_OVERFLOW; // a step ran on cut rows
constexpr int kStatusBoxRange = ATVB_STATUS_BOX_RANGE; // cell left its planned range
constexpr int kStatusNearqLost = ATVB_STATUS_NEARQ_LOST; // settle queue overflowed
constexpr int kStatusNonFinite = ATVB_STATUS_NONFINITE;  // NaN / inf position or velocity
constexpr int kStatusForceRange = ATVB_STATUS_FORCE_RANGE; // pair force beyond fixed point

// Fixed-point scales.  Energies/virials/KE are accumulated per system as
// 64-bit integers in units of 2^-32 eV (range +-2.1e9 eV), so their sums are
// independent of block order; the PME charge grid uses 2^-40 e (FP64) or
// 2^-32 e (mixed).
constexpr double kEFix = 4294967296.0;          // 2^32
constexpr double kEFixInv = 1.0 / 4294967296.0;

// Indices into SysState::acc
enum Acc : int {
    kAccELJ = 0,
    kAccECoul = 1,
    kAccERecip = 2,
    kAccVir = 3, // 6 entries: xx yy zz xy xz yz
    kAccKEA = 9,
    kAccKEB = 10,
    kAccKEX = 12, // 3 entries: per-axis kinetic energy (NPT)
    kAccCount = 15
};

struct SysState {
    unsigned long long acc[kAccCount]; // fixed-point accumulators
    double xi;         // Nose-Hoover friction
    double vscale;     // deferred velocity scale (applied by next kick)
    double s_a;        // scale from the initial-half thermostat
    double energy, e_lj, e_coul, e_recip, e_const, kinetic, conserved;
    double virial[6];
    long long step;
    long long rebuilds;
    int ago;           // steps since the last neighbour build
    int need_rebuild;  // set by the displacement check
    int rebuild;       // decision for this step
    int overflow;      // neighbour row overflowed its capacity
    int max_nnbr;      // largest row seen at the last build
    int status;        // sticky error bits (kStatus*)
    int force_build;   // host request: build the list at the next step
    int halted;        // StopOnNaN: the system no longer integrates
    int held;          // the cell is held at the edge of its planned range
    unsigned long long list_entries; // row entries of the last build (2 x pairs)
    int nearq_n;       // mixed build: pairs queued this step for an exact LJ cutoff test
    int nearq_lost;    // pairs that did not fit the queue (decided in FP32)
    double box[3];     // current cell edges
    double pressure;   // (2 KE + trace W) / (3 V) [eV/A^3]
    // MTK NPT extended state (nose_hoover_npt.cpp): chains, strain rates and
    // the factors of the next initial half step, prepared at the end of the
    // previous step by k_sys_b (or by k_npt_prep before the first step)
    double eta_t[kMaxChain], eta_t_dot[kMaxChain];
    double eta_b[kMaxChain], eta_b_dot[kMaxChain];
    double eps_dot[3];
    double ke_global, kT, T_live, Qt0, Qt1;
    double vs[3];      // per-axis velocity scale applied by the next initial kick
    double vs_out[3];  // the part of vs that belongs to the finished step
    double npt_a[3], npt_drift[3]; // exp(eps_dot dt) and the drift factor
    double Lnext[3];   // cell after the next drift
    double fixn_scale[3], fixn64_scale[3]; // 2^32 / Lnext, 2^64 / Lnext
    double Lb[3], Lb_inv[3]; // cell at the last neighbour build
    double ub[3];      // Lb / Lnext: next positions mapped into the build cell
    double disp_thr2;  // squared displacement that forces a rebuild
    double mu;         // Berendsen dilation of this step's end
    // trajectory snapshots published so far, and the ring slot being
    // written this step (-1: none)
    long long snap_count;
    int snap_slot;
};

// Header of one trajectory snapshot slot in host-mapped memory (seqlock:
// `begin` is raised before the payload is written, `end` after it and a
// system-scope fence; a reader that sees begin == end == its sequence number
// around its copy has an untorn frame).
struct SnapHeader {
    long long begin, end, step, pad;
    double box[3], pad2;
};

struct SysParams {
    // geometry (orthorhombic)
    int n;
    int prec;
    double L[3], invL[3], halfL[3];
    float Lf_fix[3]; // L / 2^32 (mixed: fixed-point position step)
    double fix_scale[3]; // 2^32 / L
    double fix64_scale[3]; // 2^64 / L
    double Lfix64[3];      // L / 2^64
    // neighbour list
    double rlist2;     // (cutoff + skin)^2, the pair-set test
    // FP32 prefilter of the pair-set test on fixed-point positions: below
    // lband_lo a candidate is certainly listed, at or above lband_hi it is
    // certainly not; in between the exact FP64 test decides
    float lband_lo, lband_hi;
    // the same screen in a cell-local FP32 frame (coordinates relative to
    // the first atom of the home cell); usable when every box edge exceeds
    // 2 (cutoff + skin + 2 cell diagonals), so no fold is needed
    int lframe_ok;
    float fband_lo, fband_hi;
    double skin_half2; // (skin/2)^2
    double rlist;      // cutoff + skin
    double nl_cut;     // NeighborList cutoff (the largest interaction cutoff)
    int nl_every, nl_delay, nl_check;
    int nc[3], ncell;
    double cs_inv[3];
    int alias[3]; // axis has fewer than 2*reach+1 cells: visit every cell
    int ncol;     // stencil columns
    int4* cols;   // {dx, dy, zreach(-1 = whole column), 0}
    int cap;      // neighbour row capacity
    // LJ
    int has_lj;
    double lj_rc2, lj_sig6, lj_eps4, lj_eps24, lj_shift;
    // mixed build: FP32 error band of r^2 around the LJ and Coulomb cutoffs,
    // and the queue of (sorted i, sorted j) pairs found inside the LJ band
    double mix_band_lj, mix_band_c;
    int2* nearq;
    int nearq_cap;
    // real-space Coulomb
    int has_coul;
    double coul_rc2, coul_alpha, coul_alpha2;
    int coul_short; // alpha * cutoff <= kErfcxSXmax: the short FP64 erfcx set
    // per-type LJ and special pairs: such systems take k_pair_general
    int general;          // 1: pair forces from k_pair_general
    int ntypes;           // 0: one LJ type (lj_* above)
    const double* lj_tab; // ntypes^2 x {sig6, eps4, eps24, shift}
    const float* lj_tabf; // the same in FP32
    int* type;            // per atom, original order
    unsigned char* stype; // per atom, sorted order
    int has_special;
    const int* sp_first;  // n + 1 (original order): partners of each atom
    const int* sp_j;      // partner (original index)
    const unsigned char* sp_cls; // 1: 1-2, 2: 1-3, 3: 1-4
    double sp_lj[4], sp_coul[4]; // scale per class ([0] = 1: not special)
    // PME
    int has_pme;
    int K[3], Kh, order;
    int Khp; // row stride of the half-complex grid: Kh rounded up to 16
    double pme_fscale; // k_e / (pi V)
    double pme_escale; // k_e / (2 pi V)
    double pme_alpha2_pi2; // pi^2 / alpha^2
    double grid_scale, grid_scale_inv; // fixed-point charge scale
    const double* bmod;    // B-spline moduli |b(m)|^2 per axis: K0 + K1 + K2
    // the hand-written transforms (fft.cu): per axis the radices of the
    // complex FFT (z: of K2 / 2 when K2 is even, the real-to-complex split)
    // and the table of the K-th roots of unity e^{-2 pi i j / K}, j < K
    // (double2, float2 in the mixed build)
    int fft_nf[3];
    int fft_fac[3][kFftMaxFac];
    const void* fft_root[3];
    double pme_alpha, pme_eself, pme_qsum2; // e_const = eself - k_e pi qsum2 / (2 V alpha^2)
    // integrator / thermostat
    double dt, dtf; // dtf = dt/2 * ftm2v
    int thermostat;
    double T, Q, n_dof_kT, tau;
    double lang_g1, lang_g2pre; // -1/(damp ftm2v), sqrt(2 kT/(damp dt mvv2e))/ftm2v
    // setpoint ramp T0 -> T1 over steps [lang_nfirst, lang_nlast] (none when
    // lang_nlast <= lang_nfirst); lang_ddm = damp dt mvv2e
    double lang_T0, lang_T1, lang_ddm;
    long long lang_nfirst, lang_nlast;
    unsigned int seed;
    int need_virial;
    double e_const; // PME self + net-charge energy
    // MTK NPT (thermostat == kNPT; nose_hoover_npt.cpp)
    double npt_T0, npt_T1, npt_tauT, npt_P, npt_tdrag, npt_pdrag, npt_W, npt_Qb;
    int npt_mt, npt_mp, npt_pdim, n_dof;
    int npt_couple[3];
    long long npt_nfirst, npt_nlast;
    double npt_Lmin[3]; // smallest cell the neighbour grid is valid for
    double npt_cut;     // largest interaction cutoff (rebuild rule)
    // Berendsen barostat (beside velocity Verlet and the thermostat):
    // mu^3 = 1 - baro_coef (baro_P - P), baro_coef = dt / (tau_P bulk_modulus)
    int baro;
    double baro_P, baro_coef;
    // md::NVELimit: speed cap vlimit = xmax / dt after each half kick (0: off)
    double vlimit, vlimit2;
    // the initial half through npt_drift_atom's per-axis factors (barostat,
    // speed cap, deformation) instead of the plain kick-drift
    int generic_drift;
    // md::Deform: engineering strain along deform_axis (-1: off), the edge of
    // step k being deform_L0 (1 + deform_rate dt k)
    int deform_axis;
    double deform_rate, deform_L0;
    // trajectory snapshots: every `snap_every` steps positions and
    // velocities go to a ring of `snap_depth` slots in host-mapped memory
    char* snap_ring;    // device view of the ring (null: off)
    int snap_every, snap_depth;
    long long snap_slot_bytes;
    // host-mapped: the longest row of the last neighbour build, written at
    // the end of each step that built the list, so the host can widen the
    // rows between step calls before a build overflows them (null: off)
    int* row_hint;
    // host-mapped copy of SysState::status, written when a step ends with a
    // bit set (null: off), so the host sees errors without a device read
    int* status_hint;
    int stop_on_nan; // cuda::StopOnNaN attached: halt at a non-finite state
    // per-atom master state (original order)
    double *x, *y, *z, *vx, *vy, *vz, *mass, *q;
    long long* tag;
    // user components' accumulators (atvb_system_add_component), null when
    // the system has none: forces in the caller's order (x block, y block,
    // z block), energy + virial (7 doubles)
    double* ext_f;
    double* ext_ev;
    double *xr, *yr, *zr; // positions at the last neighbour build
    // sorted order
    void* pos4;      // FP64: 64-bit fixed-point x, y, z + q (pack_pos64); mixed: int4 fixed-point + float q
    double4* posd4;  // FP64 sorted positions used by the pair-set test
    int4* lpos;      // fixed-point sorted positions at the last build (prefilter)
    double4* f4;     // forces in sorted order
    // mixed build: pairs closer than this may carry a force beyond the range
    // of the 64-bit fixed-point sums (2^-32 eV/A units); set at upload from
    // the LJ parameters and the largest charge product (0 in FP64)
    double force_r2_safe;
    double4* fp4;    // PME reciprocal forces of this step (sorted; PME systems)
    int *perm, *rank, *cell_of, *slot, *cell_count, *cell_start, *cellS;
    int *nbr, *nnbr;
    // PME buffers
    unsigned long long* grid_fix;
    void* grid_real;  // double or float, K0*K1*K2
    void* grid_cplx;  // double2 or float2, K0*K1*Kh
    // staging for upload / download (original order)
    double *sx, *sy, *sz;
    // scalars
    SysState* st;
    double* ehist; // energy history ring: 3 doubles per step (E, KE, step)
    int ehist_cap;
};

// Row entries of the neighbour list: sorted index in the low 30 bits, the
// special class (0: none, 1: 1-2, 2: 1-3, 3: 1-4) in the top 2 bits.
constexpr unsigned kRowIdxMask = 0x3fffffffu;
constexpr int kMaxAtoms = (1 << 30) - 1;

// A unit of work: a chunk of atoms (or grid points) of one system.
struct Item {
    int sys;
    int begin;
};

#define ATVB_DEV __device__ __forceinline__

ATVB_DEV long long to_fix(double v) { return __double2ll_rn(v * kEFix); }

// Fire-and-forget 64-bit integer reduction (no value returned, so the
// issuing thread never waits for the L2 round trip).
ATVB_DEV void red_add_u64(unsigned long long* a, unsigned long long v) {
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(a), "l"(v) : "memory");
}

ATVB_DEV void fix_add(unsigned long long* a, double v) {
    red_add_u64(a, (unsigned long long)to_fix(v));
}

template <typename T>
ATVB_DEV T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide FP64 sum in a fixed order (deterministic for a fixed block
// shape); result valid in thread 0.  `sh` needs blockDim.x/32 doubles.
ATVB_DEV double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0)
        sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        t = l < nw ? sh[l] : 0.0;
        t = warp_sum(t);
    }
    return t;
}

// Block-wide sums of N values at once (one pair of barriers); results valid
// in thread 0.  `sh` needs 32*N doubles.  Fixed order, so deterministic for
// a fixed block shape.
template <int N>
ATVB_DEV void block_sum_vec(double (&v)[N], double* sh) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < N; ++k)
        v[k] = warp_sum(v[k]);
    __syncthreads();
    if (l == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k)
            sh[k * 32 + w] = v[k];
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double t = l < nw ? sh[k * 32 + l] : 0.0;
            v[k] = warp_sum(t);
        }
    }
}

// minimum image used by the force kernels (box.h:123-150 nearbyint form)
ATVB_DEV double min_img(double d, double L, double invL) {
    return d - L * rint(d * invL);
}

// orthorhombic wrap into [0, L) (pbc.h:48-50)
ATVB_DEV double wrap(double x, double L) { return x - L * floor(x / L); }

// x in [0, L] -> [0, 2^64) (L itself folds onto 0): the FP64 build's sorted
// positions, so that the minimum image is an exact integer difference
ATVB_DEV unsigned long long pos_fix64(double x, double scale) {
    double t = x * scale;
    if (t >= 18446744073709551616.0)
        t -= 18446744073709551616.0;
    return __double2ull_rn(t);
}

// FP64 sorted position record: three 64-bit fixed-point coordinates (stored
// as bit patterns in the x, y, z of a double4) and the charge in w
ATVB_DEV double4 pack_pos64(const double x[3], const double* scale, double q) {
    return make_double4(__longlong_as_double((long long)pos_fix64(x[0], scale[0])),
                        __longlong_as_double((long long)pos_fix64(x[1], scale[1])),
                        __longlong_as_double((long long)pos_fix64(x[2], scale[2])), q);
}

ATVB_DEV unsigned int pos_fix(double x, double scale) {
    // x in [0, L] -> [0, 2^32); L itself folds onto 0
    return (unsigned int)(unsigned long long)__double2ll_rn(x * scale);
}

} // namespace atvb
