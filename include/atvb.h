/* atvb.h -- C ABI of the B200 classical-MD hot path (libatvb.so).
 *
 * Plain C types only: pointers, sizes, POD structs.  Every function returns
 * ATVB_OK (0) or an ATVB_ERR_* code; the message of the last failure on the
 * calling thread is atvb_last_error().  No exception crosses the boundary.
 *
 * Each entry point names the reference interface it replaces (paths within
 * the Atomiverse source tree).  Units are the reference's metal units:
 * Angstrom, eV, fs, amu, elementary charge, K (include/atomiverse/core/units.h).
 */
#ifndef ATVB_H
#define ATVB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATVB_ABI_VERSION 1

#define ATVB_OK 0
#define ATVB_ERR_INVALID 1  /* bad argument (std::invalid_argument in the reference) */
#define ATVB_ERR_CUDA 2     /* CUDA runtime failure (ATV_CUDA_CHECK) */
#define ATVB_ERR_OVERFLOW 3 /* neighbour row capacity exceeded during a step */
#define ATVB_ERR_STATE 4    /* call out of order (e.g. step before upload) */
#define ATVB_ERR_NOMEM 5    /* device memory budget exceeded */
#define ATVB_ERR_NOTFOUND 6 /* unknown request / slot id */
#define ATVB_ERR_PHYSICS 7  /* a sticky status bit is set: some step ran on
                               wrong or non-finite physics (status_bits) */

/* atvb_scalars.status_bits: sticky until atvb_system_clear_status.  When any
 * is set, atvb_system_scalars / _download / _run and atvb_batch_download
 * still fill their outputs and then return ATVB_ERR_PHYSICS. */
#define ATVB_STATUS_ROW_OVERFLOW 1u  /* a step used a neighbour list whose row
                                        was cut at its capacity (pairs lost);
                                        the next step call widens the rows and
                                        rebuilds before stepping on */
#define ATVB_STATUS_BOX_RANGE 2u     /* an NPT / barostat / Deform cell left the
                                        range its bins were planned for within
                                        one call and was held */
#define ATVB_STATUS_NEARQ_LOST 4u    /* mixed: near-cutoff LJ pairs overflowed the
                                        settle queue and kept their FP32 cutoff
                                        decision */
#define ATVB_STATUS_NONFINITE 8u     /* a position or velocity became NaN or
                                        infinite (cuda::StopOnNaN's condition) */
#define ATVB_STATUS_FORCE_RANGE 16u  /* a pair force beyond the range of the
                                        fixed-point force accumulators */

enum atvb_precision {
    ATVB_FP64 = 0,  /* FP64 pair, PME and integrator (reference ATV_CUDA_PREC_MODE=double) */
    ATVB_MIXED = 1  /* FP32 pair/PME math, fixed-point grid, FP64 integrator and sums */
};

enum atvb_thermostat {
    ATVB_NVE = 0,
    ATVB_NOSE_HOOVER = 1, /* md::NoseHoover(T, tau, dt): src/cuda/dynamics/nose_hoover.cu:29 */
    ATVB_LANGEVIN = 2,    /* md::FixLangevin(T, T, damp, dt, seed): fix_langevin.cuh */
    ATVB_NPT = 3          /* md::NoseHooverNPT: set by atvb_system_set_npt */
};

typedef struct atvb_ctx atvb_ctx;
typedef struct atvb_system atvb_system;
typedef struct atvb_batch atvb_batch;
typedef struct atvb_server atvb_server;

typedef struct atvb_device_opts {
    int device;          /* CUDA ordinal */
    int reserved[7];
} atvb_device_opts;

/* One MD system: the constructor arguments of the reference components the
 * path binds (NeighborList, PairLJCut, CoulLong, KSpacePME, VelocityVerlet,
 * NoseHoover / FixLangevin) in one flat record. */
typedef struct atvb_system_desc {
    int32_t n_atoms;
    double box[9];          /* row-major cell [A]; orthorhombic only */
    int32_t precision;      /* atvb_precision */
    /* NeighborList(cutoff, skin, every, delay, check): neighbor_list.cuh:98,
     * cpu/neighbor/neighbor_list.h:79 */
    double nl_cutoff, nl_skin;
    int32_t nl_every, nl_delay, nl_check;
    /* PairLJCut(epsilon, sigma, cutoff): pair_lj_cut.cuh:25 */
    int32_t lj_enabled;
    double lj_epsilon, lj_sigma, lj_cutoff;
    /* CoulLong(alpha, cutoff): coul_long.cuh:24 */
    int32_t coul_enabled;
    double coul_alpha, coul_cutoff;
    /* KSpacePME(alpha, grid_spacing, order): pme.cuh:26; pme_grid[] > 0
     * overrides the spacing rule */
    int32_t pme_enabled;
    double pme_alpha, pme_grid_spacing;
    int32_t pme_order;
    int32_t pme_grid[3];
    /* VelocityVerlet(dt) + thermostat */
    double dt;
    int32_t thermostat;     /* atvb_thermostat */
    double temperature;     /* K */
    double tau;             /* Nose-Hoover tau [fs] */
    double damp;            /* Langevin damp [fs] */
    uint32_t seed;          /* Langevin seed */
    int32_t stress_required;   /* Component::set_stress_required (component.cuh:131) */
    int32_t history_capacity;  /* per-step energy ring length (0: default 4096) */
} atvb_system_desc;

/* md::NoseHooverNPT(T_target, tau_T, P_target, tau_P, dt, drag, mtchain,
 * mpchain, couple_axis, T_stop) + set_run_span(nfirst, nlast)
 * (include/atomiverse/cuda/dynamics/nose_hoover_npt.cuh:60-70,
 * src/cpu/dynamics/nose_hoover_npt.cpp:76-172): Martyna-Tobias-Klein NPT with
 * Nose-Hoover chains on the atoms and on the barostat.  P_target in eV/A^3
 * (LAMMPS sign: positive compresses); T_stop < 0: constant setpoint; dt is
 * the system's dt.  couple[a] != 0: axis a is barostatted (all three: the
 * axis pressures are averaged, isotropic cell). */
typedef struct atvb_npt_desc {
    double T_start, T_stop, tau_T;   /* K, K, fs */
    double P_target, tau_P, drag;    /* eV/A^3, fs, - */
    int32_t mtchain, mpchain;        /* chain lengths, 1..10 */
    int32_t couple[3];
    int64_t nfirst, nlast;           /* temperature ramp span (steps) */
} atvb_npt_desc;

/* Host SoA view of a frame (cuda::Frame::Atoms field names,
 * include/atomiverse/cuda/frame/frame.cuh:71-96).  Any pointer may be NULL on
 * upload (zeros / unit mass / tag = index+1) or on download (not copied). */
typedef struct atvb_soa_view {
    double *x, *y, *z;
    double *vx, *vy, *vz;
    double *fx, *fy, *fz;
    double *mass, *charge;
    int32_t* type;
    int64_t* tag;
} atvb_soa_view;

/* SystemScalars (include/atomiverse/core/system_scalars.h:17-95) plus the
 * per-term split of the path and the thermostat state. */
typedef struct atvb_scalars {
    double energy;        /* total potential [eV] */
    double energy_pair;   /* pair + long-range (the reference adds both to energy_pair) */
    double energy_lj, energy_coul, energy_recip, energy_const;
    double kinetic, conserved;
    double stress[6];     /* virial xx yy zz xy xz yz [eV] */
    double nh_xi;
    int64_t step;
    int64_t rebuilds;
    int32_t max_neighbors;
    int32_t status;       /* 0, or the ATVB_ERR_* code of the lowest status bit:
                             ATVB_ERR_OVERFLOW (row overflow), ATVB_ERR_STATE
                             (cell held), ATVB_ERR_PHYSICS (the others) */
    int64_t list_pairs;   /* unordered pairs in the current list (cutoff + skin) */
    double box[3];        /* current cell edges [A] (change under NPT) */
    double pressure;      /* (2 KE + W_xx + W_yy + W_zz) / (3 V) [eV/A^3] */
    uint32_t status_bits; /* ATVB_STATUS_* (sticky) */
    int32_t halted;       /* 1: stopped by StopOnNaN at step `step` */
} atvb_scalars;

/* Per-kernel-group device time from CUDA events (profiling mode). */
typedef struct atvb_kernel_time {
    char name[32];
    double total_ms;
    int64_t launches;
} atvb_kernel_time;

/* ---- library ---------------------------------------------------------- */
int atvb_abi_version(void);
/* Thread-local message of the last failing call ("" if none). */
const char* atvb_last_error(void);

/* ---- context: device + stream (cuda::Context, context.cuh:37-149) ------ */
int atvb_ctx_create(const atvb_device_opts* opts, atvb_ctx** out);
int atvb_ctx_destroy(atvb_ctx* ctx);

/* ---- one system: cuda::md::MD (include/atomiverse/cuda/dynamics/md.cuh) ----
 * create      ~ MD::set_* + MD::build()               (md.cuh:118-178, 285-318)
 * upload      ~ Backend::materialize, to_cuda          (driver.cu:34-86, transfer.cu:145)
 * step        ~ MD::run's loop of Backend::step        (driver.cu:123-157)
 * download    ~ Backend::retrieve, to_cpu              (driver.cu:177)
 * run         ~ MD::run(cpu::Frame&, n): upload on first use, step, download */
int atvb_system_create(atvb_ctx* ctx, const atvb_system_desc* desc,
                       atvb_system** out);
int atvb_system_destroy(atvb_system* sys);
int atvb_system_upload(atvb_system* sys, const atvb_soa_view* frame);
/* Force-only evaluation at the current positions (neighbour build, pair,
 * PME, energies): the LAMMPS Verlet::setup force pass. */
int atvb_system_compute_forces(atvb_system* sys);
int atvb_system_step(atvb_system* sys, int32_t n_steps);
/* atvb_system_step with a CUDA event on the system's stream before the
 * first step and after every step; step_ms (n_steps entries, may be NULL)
 * gets each step's device time, *total_ms the whole span.  Synchronises. */
int atvb_system_step_timed(atvb_system* sys, int32_t n_steps, double* step_ms,
                           double* total_ms);
int atvb_system_download(atvb_system* sys, atvb_soa_view* frame,
                         atvb_scalars* scalars);
int atvb_system_scalars(atvb_system* sys, atvb_scalars* scalars);
int atvb_system_run(atvb_system* sys, atvb_soa_view* frame, int32_t n_steps,
                    atvb_scalars* scalars);
/* ---- user components (include/atomiverse/cuda/component/component.cuh:94-203,
 * registration on(phase).add(c, order) of cuda/dynamics/md.cuh:115-126) ----
 * The phases of one step, in order (include/atomiverse/core/stage.h:24-36). */
#define ATVB_PHASE_INITIAL_INTEGRATE 0
#define ATVB_PHASE_POST_INTEGRATE 1
#define ATVB_PHASE_PRE_EXCHANGE 2
#define ATVB_PHASE_PRE_NEIGHBOR 3
#define ATVB_PHASE_NEIGHBOR 4
#define ATVB_PHASE_PRE_FORCE 5
#define ATVB_PHASE_FORCE 6
#define ATVB_PHASE_POST_FORCE 7
#define ATVB_PHASE_FINAL_INTEGRATE 8
#define ATVB_PHASE_END_OF_STEP 9

/* The system as a component sees it: device arrays in the caller's atom
 * order (the order of atvb_soa_view).  Positions are wrapped into [0, L).
 * fx/fy/fz, energy (1 double) and virial (6 doubles, xx yy zz xy xz yz, eV)
 * are the components' own accumulators: the library zeroes them before the
 * pre_force phase of every step (and of a force pass), adds the forces into
 * the step's forces at final_integrate and the energy and virial into the
 * step's scalars at end_of_step; downloads report the sums. */
typedef struct atvb_device_frame {
    int64_t n_atoms;
    const double* x;
    const double* y;
    const double* z;
    double* vx;
    double* vy;
    double* vz;
    const double* mass;
    const double* charge;
    const int64_t* tag;
    double* fx;
    double* fy;
    double* fz;
    double* energy;
    double* virial;
    const double* box; /* device: the 3 cell edges [A] in force this step */
} atvb_device_frame;

/* What a component's callbacks get: the library's stream (a cudaStream_t),
 * the phase (-1 for build and destroy), the cumulative step index of the
 * step being taken (0-based, continued across calls; a force pass reports
 * the index of the next step) and the frame. */
typedef struct atvb_launch_ctx {
    void* stream;
    int32_t phase;
    int32_t reserved;
    int64_t step;
    atvb_device_frame frame;
} atvb_launch_ctx;

/* A component callback; a non-zero return fails the library call that made
 * it (ATVB_ERR_STATE). */
typedef int (*atvb_component_fn)(void* user, const atvb_launch_ctx* ctx);

/* cuda::Component build / launch / destroy registered at `phase`, `order`.
 * build (may be NULL) runs once, on the first force pass or step call after
 * registration, when the frame is on the device: it may allocate and
 * synchronise.  launch runs at its phase of every step, and at the
 * pre_force, force and post_force phases of atvb_system_compute_forces
 * (Verlet::setup), on the calling thread; it must only enqueue device work
 * on ctx->stream (no allocation, no synchronisation).  Within a phase
 * components run by ascending order (ties: registration order); order < 0
 * runs before the library's own work of that phase, order >= 0 after it.
 * destroy (may be NULL) runs at atvb_system_destroy.  A system with
 * components runs its steps as individual launches instead of one CUDA
 * graph per step. */
int atvb_system_add_component(atvb_system* sys, int32_t phase, int32_t order,
                              atvb_component_fn build, atvb_component_fn launch,
                              atvb_component_fn destroy, void* user);

/* Energy history ring: 3 doubles per step (potential, kinetic, step).
 * Writes up to max_steps most recent entries, oldest first; *count gets the
 * number written. */
int atvb_system_energy_history(atvb_system* sys, double* out,
                               int32_t max_steps, int32_t* count);
/* Pair set of the current neighbour list as unordered pairs (i < j) of
 * original atom indices: the CSR half list of PairList
 * (include/atomiverse/core/pair_list.h) flattened.  Call with pi = pj = NULL
 * to get the count only. */
int atvb_system_pairs(atvb_system* sys, int32_t* pi, int32_t* pj,
                      int64_t capacity, int64_t* count);
/* Per-type LJ: PairLJCut(std::vector<LJTypeCoeff>, cutoff) / set_type_coeff
 * (src/cpu/potentials/pair_lj_cut.cpp:44-112; table :255-298).  ncoef
 * symmetric (type_i, type_j, epsilon, sigma) entries; an unset cross term
 * mixes by Lorentz-Berthelot from the two diagonals, or does not interact
 * (epsilon 0) when a diagonal is missing; every type pair is shifted at
 * lj_cutoff.  Per-atom types come from atvb_soa_view.type at upload.  Call
 * before the first upload (ATVB_ERR_STATE after); at most 255 types. */
int atvb_system_set_lj_types(atvb_system* sys, int32_t ncoef, const int32_t* type_i,
                             const int32_t* type_j, const double* epsilon,
                             const double* sigma);
/* Special bonds: PairLJCut::set_special_bonds / CoulLong::set_special_bonds
 * (s12, s13, s14) (pair_lj_cut.cpp:118-200, coul_long.cpp:34-99) with the
 * bond topology as pairs of atom tags.  Partners 1, 2 and 3 bonds away
 * (nearest wins) take the class scales: LJ force and shifted energy times
 * lj[c]; real-space Coulomb keeps erfc and subtracts (1 - coul[c]) k_e q q / r
 * (coul_long.cpp:159-196).  Scales in [0, 1].  Call before the first upload. */
int atvb_system_set_special_bonds(atvb_system* sys, const double lj[3],
                                  const double coul[3], int64_t nbonds,
                                  const int64_t* tag_a, const int64_t* tag_b);
/* MTK NPT in place of velocity Verlet + thermostat (NoseHooverNPT
 * "replaces VelocityVerlet + NoseHoover + Barostat", nose_hoover_npt.cuh:15):
 * desc.thermostat must be ATVB_NVE; stress is then always computed.  Before
 * the first upload.  The neighbour bins are planned for cells down to 90 %
 * of the initial edge (less when the box is barely larger than 2 (cutoff +
 * skin)); between step calls a system near that limit is re-planned for its
 * current cell (checkpoint, new bins and PME mesh, restore); a cell that
 * leaves the range within one call is held and flagged in
 * atvb_scalars.status. */
int atvb_system_set_npt(atvb_system* sys, const atvb_npt_desc* npt);
/* md::Barostat(P_target, tau_P, dt, bulk_modulus) (cuda/dynamics/barostat.cuh,
 * src/cpu/dynamics/barostat.cpp:22-110): Berendsen isotropic pressure
 * coupling at end_of_step beside velocity Verlet and any thermostat, with
 * the LAMMPS-standard scalar pressure (W_xx + W_yy + W_zz + 2 KE) / (3 V),
 * mu = cbrt(clamp(1 - dt/(tau_P bulk_modulus) (P_target - P), 0.5, 2)), cell
 * and positions scaled by mu.  P_target and bulk_modulus in eV/A^3; stress is
 * then always computed.  Before the first upload; not with set_npt. */
int atvb_system_set_barostat(atvb_system* sys, double P_target, double tau_P,
                             double bulk_modulus);
/* md::NVELimit(dt, xmax) (cuda/dynamics/nve_limit.cuh, nve_limit.cu:20-130):
 * velocity Verlet whose half kicks cap the speed at xmax / dt [A]. */
int atvb_system_set_nve_limit(atvb_system* sys, double xmax);
/* md::Deform(axis, strain_rate, dt) (cuda/dynamics/deform.cuh,
 * deform.cu:55-95): after the drift of step k the edge along `axis` is
 * L0 (1 + strain_rate dt k) (engineering strain, L0 the edge at upload) and
 * positions along it are scaled by the same ratio.  Not with a barostat. */
int atvb_system_set_deform(atvb_system* sys, int32_t axis, double strain_rate);
/* Checkpoints (state I/O; the reference's resumable record is
 * cpu/record/mrec.h MrecWriter::flush, a molrs Zarr store, and
 * cpu/io/frame_writer.h write_frame_zarr): the whole resumable state of a
 * system in one self-describing byte blob -- atom arrays, forces of the last
 * force pass, positions and cell of the last neighbour build, thermostat /
 * barostat chains, pending velocity scales, step and list counters.
 * Restore into a freshly created system with the same description and the
 * same set_lj_types / set_special_bonds / set_npt configuration, in place of
 * its first upload; stepping on gives the same trajectory, bit for bit, as
 * the saved run.  Layout: header (magic "ATVBCKP1", version, sizes), the
 * state record, 14 arrays of n doubles (x y z vx vy vz fx fy fz, positions
 * at the last build, mass, charge), n int64 tags, n int32 types if per-type
 * LJ. */
int atvb_system_checkpoint_size(atvb_system* sys, int64_t* bytes);
int atvb_system_save(atvb_system* sys, void* buf, int64_t capacity);
int atvb_system_restore(atvb_system* sys, const void* buf, int64_t size);
/* Trajectory snapshots (the async snapshot ring of
 * cuda/asynchronous/async_bridge.cuh; a recorder such as MrecRecorder or the
 * XYZ writer consumes the frames): every `every` steps (0: off) the step
 * graph writes positions and velocities (as a download reports them) into
 * a ring of `depth` frames in host-mapped memory, behind a per-slot seqlock;
 * the step stream never waits for the host.  atvb_system_snapshot_poll
 * returns the frames published since the last poll, oldest first, without
 * synchronising: each array holds max_frames x n doubles (frame-major, any
 * may be NULL), steps[max_frames], box[3 * max_frames]; frames overwritten
 * before they were polled are counted in *dropped. */
int atvb_system_set_snapshots(atvb_system* sys, int32_t every, int32_t depth);
int atvb_system_snapshot_poll(atvb_system* sys, int32_t max_frames, int64_t* steps,
                              double* box, double* x, double* y, double* z, double* vx,
                              double* vy, double* vz, int32_t* count, int64_t* dropped);
/* Sticky status bits (atvb_scalars.status_bits): clear them (and un-halt a
 * system stopped by StopOnNaN) once the caller has dealt with the cause. */
int atvb_system_clear_status(atvb_system* sys);
/* cuda::StopOnNaN (include/atomiverse/cuda/driver/criterion.cuh:166-178):
 * with on != 0, the step at which a position or velocity of the system
 * turns non-finite is its last: the device stops integrating it (positions,
 * velocities and the step counter stay as they were), later step calls
 * return ATVB_ERR_PHYSICS at once, and scalars report halted = 1.  Off by
 * default (the reference stops only with the criterion attached); the
 * ATVB_STATUS_NONFINITE bit is raised either way. */
int atvb_system_set_stop_on_nan(atvb_system* sys, int32_t on);
/* FixLangevin(T_start, T_stop, damp, dt, seed).set_run_span(nfirst, nlast)
 * (src/cpu/dynamics/fix_langevin.cpp:94-104,
 * include/atomiverse/cuda/dynamics/fix_langevin.cuh:69-80): the Langevin
 * setpoint moves linearly from the descriptor's temperature (T_start) to
 * T_stop over the cumulative steps [nfirst, nlast] and holds at either end
 * outside it.  T_stop < 0 or nlast <= nfirst: the constant setpoint.
 * ATVB_ERR_INVALID unless the system's thermostat is ATVB_LANGEVIN. */
int atvb_system_set_langevin_ramp(atvb_system* sys, double T_stop, int64_t nfirst,
                                  int64_t nlast);
/* Capacity overrides (0 = automatic sizing).  row_capacity pins the
 * neighbour row length (no automatic growth: a build that needs longer rows
 * fails with ATVB_ERR_OVERFLOW outside a step call, and raises
 * ATVB_STATUS_ROW_OVERFLOW within one); nearq_capacity sizes the mixed
 * build's near-cutoff settle queue.  For tuning and for tests. */
int atvb_system_set_capacity(atvb_system* sys, int32_t row_capacity,
                             int32_t nearq_capacity);
/* Profiling: enable per-kernel-group CUDA events on subsequent steps. */
int atvb_system_profile(atvb_system* sys, int32_t enable);
int atvb_system_profile_read(atvb_system* sys, atvb_kernel_time* out,
                             int32_t capacity, int32_t* count);
/* Lanes per atom in the pair kernel (1,2,4,8,16,32); 0 = autotune. */
int atvb_system_set_pair_lanes(atvb_system* sys, int32_t lanes);
/* Kernel launches of the last step() call, counting the six list-build
 * kernels on every step: in the step graph of a system (or batch) of at
 * least 100,000 atoms they launch only on steps where a system rebuilds
 * its list (conditional nodes), so the launches made there are this count
 * less 6 per step without a rebuild. */
int atvb_system_launch_count(atvb_system* sys, int64_t* launches);
/* The system's CUDA stream (cudaStream_t) for event timing by callers. */
void* atvb_system_stream(atvb_system* sys);

/* ---- batch: many independent systems in one launch per kernel ---------- */
int atvb_batch_create(atvb_ctx* ctx, const atvb_system_desc* descs,
                      int32_t n_systems, atvb_batch** out);
int atvb_batch_destroy(atvb_batch* b);
int atvb_batch_upload(atvb_batch* b, int32_t index, const atvb_soa_view* frame);
int atvb_batch_compute_forces(atvb_batch* b);
int atvb_batch_step(atvb_batch* b, int32_t n_steps);
int atvb_batch_download(atvb_batch* b, int32_t index, atvb_soa_view* frame,
                        atvb_scalars* scalars);
/* atvb_system_clear_status / _set_stop_on_nan for system `index`. */
int atvb_batch_clear_status(atvb_batch* b, int32_t index);
int atvb_batch_set_stop_on_nan(atvb_batch* b, int32_t index, int32_t on);
/* atvb_system_set_langevin_ramp for system `index`. */
int atvb_batch_set_langevin_ramp(atvb_batch* b, int32_t index, double T_stop,
                                 int64_t nfirst, int64_t nlast);
/* atvb_system_set_lj_types / _set_special_bonds for system `index` of a
 * batch, before that system's first upload. */
/* atvb_system_set_npt for system `index` of a batch, before its first upload. */
/* Checkpoints of system `index` of a batch (restore before its first upload). */
int atvb_batch_checkpoint_size(atvb_batch* b, int32_t index, int64_t* bytes);
int atvb_batch_save(atvb_batch* b, int32_t index, void* buf, int64_t capacity);
int atvb_batch_restore(atvb_batch* b, int32_t index, const void* buf, int64_t size);
int atvb_batch_set_npt(atvb_batch* b, int32_t index, const atvb_npt_desc* npt);
int atvb_batch_set_barostat(atvb_batch* b, int32_t index, double P_target, double tau_P,
                            double bulk_modulus);
int atvb_batch_set_nve_limit(atvb_batch* b, int32_t index, double xmax);
int atvb_batch_set_deform(atvb_batch* b, int32_t index, int32_t axis, double strain_rate);
int atvb_batch_set_lj_types(atvb_batch* b, int32_t index, int32_t ncoef,
                            const int32_t* type_i, const int32_t* type_j,
                            const double* epsilon, const double* sigma);
int atvb_batch_set_special_bonds(atvb_batch* b, int32_t index, const double lj[3],
                                 const double coul[3], int64_t nbonds,
                                 const int64_t* tag_a, const int64_t* tag_b);
/* Time candidate pair-kernel shapes on the batch's own size mix and keep
 * the fastest; *lanes receives the choice. */
int atvb_batch_autotune(atvb_batch* b, int32_t* lanes);
int atvb_batch_launch_count(atvb_batch* b, int64_t* launches);
/* Per-kernel-group CUDA-event times over every system of the batch, as
 * atvb_system_profile / atvb_system_profile_read. */
int atvb_batch_profile(atvb_batch* b, int32_t enable);
int atvb_batch_profile_read(atvb_batch* b, atvb_kernel_time* out,
                            int32_t capacity, int32_t* count);

/* ---- server: continuous batching of MD segments ------------------------ */
typedef struct atvb_request_result {
    int64_t id;
    int32_t state;        /* 0 queued, 1 running, 2 done, 3 cancelled, 4 failed
                             (not admitted, or finished with a sticky status
                             bit: the frame can still be collected),
                             5 suspended */
    int32_t steps_done;
    double t_submit, t_start, t_done; /* seconds on the server clock */
    atvb_scalars scalars;
} atvb_request_result;

int atvb_server_create(atvb_ctx* ctx, size_t hbm_budget_bytes,
                       int32_t max_active, atvb_server** out);
int atvb_server_destroy(atvb_server* srv);
/* Copies the frame; the request runs n_steps once admitted. */
int atvb_server_submit(atvb_server* srv, const atvb_system_desc* desc,
                       const atvb_soa_view* frame, int32_t n_steps,
                       int64_t* id);
int atvb_server_cancel(atvb_server* srv, int64_t id);
/* Admission limit besides the device-memory budget: requests are admitted
 * (in arrival order, smaller ones may pass a larger one that waited less
 * than half a second) only while the resident atoms stay within
 * max_resident_atoms; 0 = no limit.  At least one request is always
 * admitted.  Bounding the resident work keeps each step short, so requests
 * finish in arrival order instead of all together. */
int atvb_server_set_limits(atvb_server* srv, int64_t max_resident_atoms);
/* One scheduling round: admit what fits, advance every running segment by
 * `chunk` steps in one batched launch sequence, retire finished ones. */
int atvb_server_tick(atvb_server* srv, int32_t chunk);
int atvb_server_poll(atvb_server* srv, int64_t id, atvb_request_result* out);
/* Copy a finished request's frame out and release it. */
int atvb_server_collect(atvb_server* srv, int64_t id, atvb_soa_view* frame,
                        atvb_request_result* out);
int atvb_server_stats(atvb_server* srv, int64_t* queued, int64_t* running,
                      int64_t* done, size_t* bytes_in_use);
/* Resumable segments (checkpoints, see atvb_system_save).  suspend: stop a
 * running request, keep its state and frame (collect works), free its
 * device memory.  resume: queue a suspended request -- or a finished one
 * when keep_checkpoints is on -- for more_steps further steps; it continues
 * bit for bit where it stopped.  checkpoint: the blob of a running,
 * suspended or kept request (buf NULL: size only).  submit_checkpoint: a
 * new request that resumes from a blob, e.g. one taken on another GPU or
 * process (the desc must match the saved system). */
int atvb_server_keep_checkpoints(atvb_server* srv, int32_t on);
int atvb_server_suspend(atvb_server* srv, int64_t id);
int atvb_server_resume(atvb_server* srv, int64_t id, int32_t more_steps);
int atvb_server_checkpoint(atvb_server* srv, int64_t id, void* buf, int64_t capacity,
                           int64_t* size);
int atvb_server_submit_checkpoint(atvb_server* srv, const atvb_system_desc* desc,
                                  const void* buf, int64_t size, int32_t n_steps,
                                  int64_t* id);
/* Device bytes one request of this shape holds while resident. */
int atvb_request_bytes(const atvb_system_desc* desc, size_t* bytes);

/* ---- allocation-free pair forces -------------------------------------- *
 * No counterpart in the reference: a stand-alone evaluation of the
 * short-range pair term (shifted LJ + real-space Ewald erfc Coulomb, FP64)
 * that allocates nothing.  x, y, z, q (n_atoms each; q may be NULL without
 * Coulomb) are DEVICE pointers read on `stream` (a cudaStream_t, NULL = the
 * legacy default stream); fx, fy, fz (device, n_atoms) are overwritten with
 * the pair forces; energy (device, 2 doubles: LJ, Coulomb real space; may be
 * NULL) is overwritten.  Only n_atoms, box, precision (ATVB_FP64),
 * lj_* / coul_* and pme_enabled (must be 0) of the descriptor are read.
 * Limits: n_atoms <= 65536, at most 65536 cells of edge >= the cutoff,
 * orthorhombic box with every edge > 2 x cutoff; anything else returns
 * ATVB_ERR_INVALID before any launch.  Scratch is one fixed device array
 * per device: calls on the same device must not overlap in time (use one
 * stream or order the streams).  The first call on a device resolves the
 * scratch address; make it outside any stream capture.  Asynchronous: no
 * synchronisation, no host<->device copy. */
int atvb_pair_forces_static(const atvb_system_desc* desc, const double* x,
                            const double* y, const double* z, const double* q,
                            double* fx, double* fy, double* fz, double* energy,
                            void* stream);

#ifdef __cplusplus
}
#endif
#endif
