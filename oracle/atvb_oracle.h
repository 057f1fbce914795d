/* atvb_oracle.h -- CPU FP64 restatement of the Atomiverse classical-MD hot
 * path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and the
 * CPU-baseline leg of bench.py call it as the checker.  The product path
 * (libatvb.so) never links, loads or calls anything in this directory.
 *
 * Each function names the reference file:line whose algorithm it restates
 * (paths are relative to the Atomiverse source tree).  Units are the
 * reference's "metal" set: Angstrom, eV, fs, amu, e, K.
 */
#ifndef ATVB_ORACLE_H
#define ATVB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/atomiverse/core/units.h:138,165,166,173 */
#define ORC_KB 8.617333262e-5
#define ORC_FTM2V (1.0 / 103.6427)
#define ORC_MVV2E 103.6427
#define ORC_QQR2E 14.399645
#define ORC_PI 3.14159265358979323846

enum { ORC_THERMO_NONE = 0, ORC_THERMO_NH = 1, ORC_THERMO_LANGEVIN = 2, ORC_THERMO_NPT = 3 };

#define ORC_MAXCHAIN 10

/* MTK NPT parameters: NoseHooverNPT(T_target, tau_T, P_target, tau_P, dt,
 * drag, mtchain, mpchain, couple_axis, T_stop) + set_run_span(nfirst, nlast)
 * (include/atomiverse/cpu/dynamics/nose_hoover_npt.h:180-215).  P_target in
 * eV/A^3 (positive compressive), T_stop < 0: no ramp. */
typedef struct orc_npt {
    double T_start, T_stop, tau_T, P_target, tau_P, drag;
    int mtchain, mpchain;
    int couple[3];
    int64_t nfirst, nlast;
} orc_npt;

typedef struct orc_desc {
    int n;                 /* atoms */
    double L[3];           /* orthorhombic box edges [A] */
    double nl_cutoff;      /* NeighborList cutoff [A] */
    double skin;           /* NeighborList skin [A] */
    int nl_every, nl_delay, nl_check; /* LAMMPS neigh_modify */
    int has_lj;
    double lj_eps, lj_sigma, lj_rc;
    int has_coul;
    double coul_alpha, coul_rc;
    int has_pme;
    double pme_alpha;
    int pme_K[3];
    int pme_order;
    double dt;             /* fs */
    int thermostat;        /* ORC_THERMO_* */
    double T, tau, damp;   /* K, fs (NH tau), fs (Langevin damp) */
    uint32_t seed;         /* Langevin seed */
    int need_virial;
    /* Langevin setpoint ramp T -> T_stop over steps [lang_nfirst,
     * lang_nlast] (fix_langevin.cpp:94-104; no ramp when nlast <= nfirst) */
    double T_stop;
    int64_t lang_nfirst, lang_nlast;
    /* test-only external term, the same one a user component adds on the
     * GPU: a harmonic wall E = k d^2, F = -2 k d along `wall_axis` for
     * d = coordinate - wall_pos > 0 (wall_axis < 0: none) */
    int wall_axis;
    double wall_pos, wall_k;
} orc_desc;

typedef struct orc_sys orc_sys;

/* Scalars layout returned by orc_scalars (all eV unless noted):
 * [0] energy (total potential)  [1] e_lj  [2] e_coul_real  [3] e_recip
 * [4] e_self+e_net              [5] kinetic
 * [6..11] virial xx yy zz xy xz yz   [12] NH xi  [13] step  [14] rebuilds */
#define ORC_NSCALARS 15

orc_sys* orc_create(const orc_desc* d);
void orc_destroy(orc_sys* s);
void orc_set_threads(int n);
int orc_get_threads(void);

/* Host arrays of length n. Positions are wrapped into [0, L) on entry. */
void orc_set_state(orc_sys* s, const double* x, const double* y,
                   const double* z, const double* vx, const double* vy,
                   const double* vz, const double* fx, const double* fy,
                   const double* fz, const double* mass, const double* q,
                   const int64_t* tag);
void orc_get_state(const orc_sys* s, double* x, double* y, double* z,
                   double* vx, double* vy, double* vz, double* fx, double* fy,
                   double* fz);
void orc_scalars(const orc_sys* s, double* out);

/* Half Verlet list at the current positions (cell_list.cpp:743-895
 * semantics): unordered pairs {i<j} with min-image r^2 < (cutoff+skin)^2.
 * Returns the pair count. */
int64_t orc_build_list(orc_sys* s);
void orc_get_pairs(const orc_sys* s, int32_t* pi, int32_t* pj);

/* Zero forces/energy/virial, then LJ + CoulLong + PME at current positions
 * over the current list (pre_force + force phases). */
void orc_compute_forces(orc_sys* s);

/* n MD steps in the LAMMPS Verlet order (runtime.cpp:452-501).  If hist is
 * non-NULL it receives 2 doubles per step: potential and kinetic energy at
 * end_of_step.  Returns the number of neighbour rebuilds. */
int orc_run(orc_sys* s, int n_steps, double* hist);

/* Per-type LJ (src/cpu/potentials/pair_lj_cut.cpp:44-112 per-type
 * constructor / set_type_coeff, :255-298 finalize_type_table_): ncoef
 * explicit (type_i, type_j, eps, sigma) entries, symmetric; an unset cross
 * term mixes by Lorentz-Berthelot (eps = sqrt(eps_ii eps_jj),
 * sigma = (sigma_ii + sigma_jj)/2, :246-252) when both diagonals are set,
 * else the pair does not interact (eps = 0).  Each type pair is shifted at
 * the common cutoff.  type[n] is the per-atom type; the table covers every
 * type named by a coefficient or carried by an atom (a type without
 * coefficients has no LJ site).  Returns the number of types, or -1 on a bad
 * coefficient (type < 0 or sigma <= 0) or a negative atom type. */
int orc_set_lj_types(orc_sys* s, int ncoef, const int32_t* ti, const int32_t* tj,
                     const double* eps, const double* sigma, const int32_t* type);
/* Special pairs (LAMMPS special_bonds; cpu/potentials/special_scale.h,
 * pair_lj_cut.cpp:770-800, coul_long.cpp:159-196): npairs unordered (i, j)
 * atom indices with an LJ scale (multiplies the LJ force and shifted
 * energy) and a Coulomb scale f (the real-space term keeps erfc and
 * subtracts (1 - f) k_e q_i q_j / r, the share the reciprocal sum added). */
void orc_set_special(orc_sys* s, int npairs, const int32_t* pi, const int32_t* pj,
                     const double* s_lj, const double* s_coul);

/* Switch the system's integrator to MTK NPT (replaces velocity Verlet and
 * the thermostat; nose_hoover_npt.cpp:87-172 build).  Returns 0, or -1 on a
 * bad parameter (chain length outside [1, ORC_MAXCHAIN], tau <= 0). */
int orc_set_npt(orc_sys* s, const orc_npt* p);
/* Berendsen barostat (cpu::md::Barostat(P_target, tau_P, dt, bulk_modulus),
 * src/cpu/dynamics/barostat.cpp:22-110) at end_of_step, beside velocity
 * Verlet and the thermostat; P_target in eV/A^3.  Returns 0 or -1. */
int orc_set_barostat(orc_sys* s, double P_target, double tau_P, double bulk_modulus);
/* NVELimit(dt, xmax) (cuda/dynamics/nve_limit.cu:20-130): speed cap xmax/dt
 * after each half kick.  Deform(axis, strain_rate, dt) (cuda/dynamics/
 * deform.cu:55-95): engineering strain along one axis after the drift.
 * Return 0 or -1 on a bad argument. */
int orc_set_nve_limit(orc_sys* s, double xmax);
int orc_set_deform(orc_sys* s, int axis, double rate);
/* NPT state: [0..2] box edges, [3] conserved extended Hamiltonian,
 * [4..6] eps_dot, [7] eta_t[0], [8] eta_t_dot[0], [9] eta_b[0],
 * [10] eta_b_dot[0], [11] live temperature setpoint, [12] KE_global. */
#define ORC_NPT_NSTATE 13
void orc_npt_state(const orc_sys* s, double* out);

/* ---- standalone pieces used by the known-answer tests ---- */
void orc_bspline(double frac, int n, double* theta, double* dtheta);
int orc_good_fft_size(int n);
void orc_spline_moduli(int K, int n, double* mod);
/* in-place 3D complex FFT, data interleaved re/im, layout k2 + K2*(k1+K1*k0);
 * sign -1 = forward (FFTW_FORWARD), +1 = backward (unnormalised). */
void orc_fft3d(int K0, int K1, int K2, double* data, int sign);
/* Reciprocal-space Ewald with self and net-charge terms (ewald_sum.h). */
void orc_ewald_recip(int n, const double* x, const double* y, const double* z,
                     const double* q, const double L[3], double alpha,
                     double accuracy, double* energy, double* fx, double* fy,
                     double* fz, double* virial);
/* PME reciprocal + self + net energy/forces/virial (pme.cpp:152-253). */
void orc_pme(int n, const double* x, const double* y, const double* z,
             const double* q, const double L[3], double alpha, const int K[3],
             int order, double* energy, double* fx, double* fy, double* fz,
             double* virial);
/* Langevin Gaussian triple for (seed, step, tag): fix_langevin.cpp:37-62,
 * 112-140. */
void orc_gauss3(uint32_t seed, int64_t step, int64_t tag, double* out3);

#ifdef __cplusplus
}
#endif
#endif
