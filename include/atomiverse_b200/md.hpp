// md.hpp -- the reference's CUDA MD surface (cuda::md::MD and its
// components) as a header-only C++ layer over the C ABI in atvb.h.
//
// Component constructors keep the reference signatures:
//   NeighborList(cutoff, skin = -1, every = 1, delay = 0, check = true)
//       include/atomiverse/cuda/neighbor/neighbor_list.cuh:98
//   PairLJCut(epsilon, sigma, cutoff)       cuda/potentials/pair_lj_cut.cuh:25
//   PairLJCut({LJTypeCoeff...}, cutoff), set_type_coeff, set_special_bonds
//       (src/cpu/potentials/pair_lj_cut.cpp:44-200; CoulLong::set_special_bonds)
//   CoulLong(alpha, cutoff)                 cuda/potentials/coul_long.cuh:24
//   KSpacePME(alpha, grid_spacing = 1.0, order = 6)  cuda/longrange/pme.cuh:26
//   md::VelocityVerlet(dt), md::NoseHoover(T, tau, dt),
//   md::FixLangevin(T_start, T_stop, damp, dt, seed)
// and MD keeps set_neighbor / set_evaluator / set_integrator /
// set_thermostat and the continuable run(frame, n_steps)
// (include/atomiverse/cuda/dynamics/md.cuh:118-385).  Errors surface as
// std::invalid_argument (bad configuration) or std::runtime_error (CUDA),
// as in the reference.  The built-in components only record their
// parameters: the device step is one fused, graph-captured sequence built by
// the library.  User components (class Component, registered with
// MD::on(phase).add(c, order), include/atomiverse/cuda/component/
// component.cuh:94-203 and cuda/dynamics/md.cuh:115-126) run their own
// launches at their phase of every step on the library's stream.
#pragma once

#include <atvb.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <memory>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace atvb_cpp {

inline void check(int rc) {
    if (rc == ATVB_OK)
        return;
    const std::string msg = atvb_last_error();
    if (rc == ATVB_ERR_INVALID)
        throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

/// Host frame: SoA arrays named like cuda::Frame::Atoms plus the box.
struct Frame {
    std::vector<double> x, y, z, vx, vy, vz, fx, fy, fz, mass, charge;
    std::vector<int64_t> tag;
    std::vector<int32_t> type;                      // LJ type per atom (per-type PairLJCut)
    std::vector<std::pair<int64_t, int64_t>> bonds; // topology (tags) for special bonds
    double box[3] = {0, 0, 0};
    int n() const { return (int)x.size(); }
    void resize(int n) {
        for (auto* v : {&x, &y, &z, &vx, &vy, &vz, &fx, &fy, &fz, &mass, &charge})
            v->resize(n, 0.0);
        mass.assign(n, 1.0);
        tag.resize(n);
        for (int i = 0; i < n; ++i)
            tag[i] = i + 1;
    }
    atvb_soa_view view() {
        atvb_soa_view v{};
        v.x = x.data(); v.y = y.data(); v.z = z.data();
        v.vx = vx.data(); v.vy = vy.data(); v.vz = vz.data();
        v.fx = fx.data(); v.fy = fy.data(); v.fz = fz.data();
        v.mass = mass.data(); v.charge = charge.data(); v.tag = tag.data();
        v.type = type.empty() ? nullptr : type.data();
        return v;
    }
};

struct NeighborList {
    double cutoff, skin;
    int every, delay;
    bool check;
    explicit NeighborList(double cutoff_, double skin_ = -1.0, int every_ = 1,
                          int delay_ = 0, bool check_ = true)
        : cutoff(cutoff_), skin(skin_), every(every_), delay(delay_), check(check_) {}
};
/// One (type_i, type_j, epsilon, sigma) entry of a per-type PairLJCut.
struct LJTypeCoeff {
    int type_i, type_j;
    double epsilon, sigma;
};
/// LAMMPS special_bonds scales for 1-2, 1-3 and 1-4 partners.
struct SpecialScales {
    double s12 = 1.0, s13 = 1.0, s14 = 1.0;
    bool active() const { return s12 != 1.0 || s13 != 1.0 || s14 != 1.0; }
};
struct PairLJCut {
    double epsilon = 0.0, sigma = 0.0, cutoff;
    std::vector<LJTypeCoeff> coeffs; // non-empty: per-type form
    SpecialScales special;
    PairLJCut(double e, double s, double c) : epsilon(e), sigma(s), cutoff(c) {
        if (c <= 0.0)
            throw std::invalid_argument("PairLJCut: cutoff must be positive");
    }
    /// Per-type form (pair_lj_cut.cpp:44-66): unset cross terms mix by
    /// Lorentz-Berthelot; a type without coefficients has no LJ site.
    PairLJCut(std::vector<LJTypeCoeff> c, double rc) : cutoff(rc), coeffs(std::move(c)) {
        if (rc <= 0.0)
            throw std::invalid_argument("PairLJCut: cutoff must be positive");
        if (coeffs.empty())
            throw std::invalid_argument(
                "PairLJCut: the per-type constructor needs at least one coefficient");
        epsilon = coeffs[0].epsilon; // scalar fields only carry a valid description
        sigma = coeffs[0].sigma;
    }
    PairLJCut& set_type_coeff(int ti, int tj, double e, double s) {
        if (coeffs.empty())
            throw std::logic_error("PairLJCut::set_type_coeff: built with a single epsilon/sigma");
        if (ti < 0 || tj < 0)
            throw std::invalid_argument("PairLJCut::set_type_coeff: types must be >= 0");
        if (s <= 0.0)
            throw std::invalid_argument("PairLJCut::set_type_coeff: sigma must be > 0");
        coeffs.push_back({ti, tj, e, s});
        return *this;
    }
    PairLJCut& set_special_bonds(double s12, double s13, double s14) {
        special = {s12, s13, s14};
        return *this;
    }
};
struct CoulLong {
    double alpha, cutoff;
    SpecialScales special;
    CoulLong(double a, double c) : alpha(a), cutoff(c) {
        if (a <= 0.0 || c <= 0.0)
            throw std::invalid_argument("CoulLong: alpha and cutoff must be > 0");
    }
    CoulLong& set_special_bonds(double s12, double s13, double s14) {
        special = {s12, s13, s14};
        return *this;
    }
};
struct KSpacePME {
    double alpha, grid_spacing;
    int order;
    int grid[3] = {0, 0, 0};
    explicit KSpacePME(double a, double spacing = 1.0, int order_ = 6)
        : alpha(a), grid_spacing(spacing), order(order_) {
        if (a <= 0.0)
            throw std::invalid_argument("KSpacePME: alpha must be > 0");
        if (spacing <= 0.0)
            throw std::invalid_argument("KSpacePME: grid_spacing must be > 0");
        if (order_ < 3)
            throw std::invalid_argument("KSpacePME: order must be >= 3");
    }
};

// ---- user components --------------------------------------------------------

namespace md {
/// md::Phase (include/atomiverse/core/stage.h:24-36): the phases of a step.
enum class Phase {
    initial_integrate,
    post_integrate,
    pre_exchange,
    pre_neighbor,
    neighbor,
    pre_force,
    force,
    post_force,
    final_integrate,
    end_of_step,
    COUNT
};
} // namespace md

/// A component's default phase slot (include/atomiverse/core/binding.h).
struct DefaultBinding {
    md::Phase phase;
    int order;
};

/// What build / launch / destroy receive (component.cuh:22-49).  `stream` is
/// the library's cudaStream_t (the reference's cuda::Context streams);
/// `frame` the device arrays of the system (atvb_device_frame: positions,
/// velocities, masses, charges, tags in the caller's atom order, and the
/// components' own force / energy / virial accumulators).
struct BuildContext {
    void* stream;
    const atvb_device_frame& frame;
};
struct LaunchContext {
    void* stream;
    const atvb_device_frame& frame;
    int stage;    ///< the phase being walked (compare with at())
    int64_t step; ///< cumulative step index (0-based)
    template <typename PhaseEnum>
    bool at(PhaseEnum phase) const {
        return stage == static_cast<int>(phase);
    }
};
struct DestroyContext {
    void* stream;
    const atvb_device_frame& frame;
};

/// cuda::Component (include/atomiverse/cuda/component/component.cuh:94-203):
/// build once, launch every step at its phase (enqueue device work on
/// ctx.stream only: no allocation, no synchronisation), destroy at the end.
/// Forces, energy and virial a component adds to frame.fx / fy / fz /
/// energy / virial join the step's totals.
class Component {
  public:
    virtual ~Component() = default;
    virtual std::string name() const = 0;
    virtual bool requires_system_stress() const { return false; }
    virtual bool provides_system_stress() const { return false; }
    virtual bool provides_energy() const { return false; }
    virtual bool provides_force() const { return false; }
    /// Plan-level verdict, called once before the system is built: true iff
    /// some part of the simulation consumes the virial (component.cuh:131).
    virtual void set_stress_required(bool /*required*/) {}
    virtual std::vector<DefaultBinding> default_bindings() const { return {}; }
    virtual void build(const BuildContext& /*ctx*/) {}
    virtual void launch(const LaunchContext& ctx) = 0;
    virtual void destroy(const DestroyContext& /*ctx*/) {}
};

namespace md {
struct VelocityVerlet {
    double dt;
    explicit VelocityVerlet(double dt_) : dt(dt_) {}
};
struct NoseHoover {
    double T, tau, dt;
    NoseHoover(double T_, double tau_, double dt_) : T(T_), tau(tau_), dt(dt_) {}
};
/// FixLangevin (cuda/dynamics/fix_langevin.cuh:69-80): T_stop < 0 is the
/// constant setpoint; set_run_span(nfirst, nlast) ramps it linearly from
/// T_start to T_stop over those cumulative steps (fix_langevin.cpp:94-104).
struct FixLangevin {
    double T_start, T_stop, damp, dt;
    uint32_t seed;
    int64_t nfirst = 0, nlast = 0;
    FixLangevin(double t0, double t1, double damp_, double dt_, uint32_t seed_)
        : T_start(t0), T_stop(t1 < 0 ? t0 : t1), damp(damp_), dt(dt_), seed(seed_) {}
    FixLangevin& set_run_span(int64_t first, int64_t last) {
        nfirst = first;
        nlast = last;
        return *this;
    }
};
/// md::NVELimit(dt, xmax) (cuda/dynamics/nve_limit.cuh): velocity Verlet
/// with each half kick's speed capped at xmax / dt.  An integrator.
struct NVELimit {
    double dt, xmax;
    NVELimit(double dt_, double xmax_) : dt(dt_), xmax(xmax_) {
        if (!(xmax_ > 0.0))
            throw std::invalid_argument("NVELimit: xmax must be > 0");
    }
};
/// md::Deform(axis, strain_rate, dt) (cuda/dynamics/deform.cuh): constant
/// engineering strain rate along one axis after each drift.
struct Deform {
    int axis;
    double strain_rate, dt;
    Deform(int axis_, double rate, double dt_) : axis(axis_), strain_rate(rate), dt(dt_) {
        if (axis_ < 0 || axis_ > 2)
            throw std::invalid_argument("Deform: axis must be 0, 1 or 2");
    }
};
/// md::Barostat(P_target, tau_P, dt, bulk_modulus = 1) -- Berendsen pressure
/// coupling at end_of_step beside the thermostat (cpu/dynamics/barostat.h:86;
/// LAMMPS-standard pressure sign).  Bound with set_thermostat.
struct Barostat {
    double P_target, tau_P, dt, bulk_modulus;
    Barostat(double P, double tau, double dt_, double bulk = 1.0)
        : P_target(P), tau_P(tau), dt(dt_), bulk_modulus(bulk) {
        if (!(tau > 0.0) || !(bulk > 0.0))
            throw std::invalid_argument("Barostat: tau_P and bulk_modulus must be > 0");
    }
};
/// cuda::md::NoseHooverNPT(T_target, tau_T, P_target, tau_P, dt, drag,
/// mtchain, mpchain, couple_axis, T_stop) + set_run_span
/// (cuda/dynamics/nose_hoover_npt.cuh:60-70).  An integrator: it replaces
/// VelocityVerlet and the thermostat.  P_target in eV/A^3.
struct NoseHooverNPT {
    atvb_npt_desc p{};
    double dt;
    NoseHooverNPT(double T_target, double tau_T, double P_target, double tau_P, double dt_,
                  double drag = 0.0, int mtchain = 3, int mpchain = 3,
                  std::array<bool, 3> couple_axis = {true, true, true}, double T_stop = -1.0)
        : dt(dt_) {
        p.T_start = T_target;
        p.T_stop = T_stop;
        p.tau_T = tau_T;
        p.P_target = P_target;
        p.tau_P = tau_P;
        p.drag = drag;
        p.mtchain = mtchain;
        p.mpchain = mpchain;
        for (int a = 0; a < 3; ++a)
            p.couple[a] = couple_axis[a] ? 1 : 0;
    }
    NoseHooverNPT& set_run_span(int64_t nfirst, int64_t nlast) {
        p.nfirst = nfirst;
        p.nlast = nlast;
        return *this;
    }
    double T_target() const { return p.T_start; }
};

/// cuda::md::MD: categorical setters, then run(frame, n) -- continuable.
class MD {
  public:
    explicit MD(int device = 0, int precision = ATVB_FP64) : precision_(precision) {
        atvb_device_opts o{};
        o.device = device;
        check(atvb_ctx_create(&o, &ctx_));
        std::memset(&d_, 0, sizeof(d_));
        d_.nl_skin = -1.0;
        d_.nl_every = 1;
        d_.pme_order = 4;
    }
    ~MD() {
        if (sys_)
            atvb_system_destroy(sys_);
        if (ctx_)
            atvb_ctx_destroy(ctx_);
    }
    MD(const MD&) = delete;
    MD& operator=(const MD&) = delete;

    /// One phase of the plan: on(phase).add(component, order)
    /// (md.cuh:17,70,115-126).  Components of a phase run by ascending
    /// order; order < 0 before the library's own work of that phase.
    class PhaseSlot {
      public:
        template <typename C>
        MD& add(C&& c, int order = 0) {
            return md_.add_component(std::make_shared<std::decay_t<C>>(std::forward<C>(c)),
                                     {{phase_, order}});
        }

      private:
        friend class MD;
        PhaseSlot(MD& m, Phase p) : md_(m), phase_(p) {}
        MD& md_;
        Phase phase_;
    };
    PhaseSlot on(Phase p) { return PhaseSlot(*this, p); }

    /// add(component) at its default_bindings() (the path of set_observer).
    template <typename C>
    MD& add(C&& c) {
        auto sp = std::make_shared<std::decay_t<C>>(std::forward<C>(c));
        const std::vector<DefaultBinding> b = sp->default_bindings();
        if (b.empty())
            throw std::invalid_argument("MD::add: component " + sp->name() +
                                        " has no default binding; use on(phase).add");
        std::vector<std::pair<Phase, int>> at;
        for (const DefaultBinding& d : b)
            at.emplace_back(d.phase, d.order);
        return add_component(std::move(sp), at);
    }

    MD& set_neighbor(const NeighborList& nl) {
        d_.nl_cutoff = nl.cutoff;
        d_.nl_skin = nl.skin;
        d_.nl_every = nl.every;
        d_.nl_delay = nl.delay;
        d_.nl_check = nl.check ? 1 : 0;
        have_nl_ = true;
        return *this;
    }
    MD& set_evaluator(const PairLJCut& p) {
        d_.lj_enabled = 1;
        d_.lj_epsilon = p.epsilon;
        d_.lj_sigma = p.sigma;
        d_.lj_cutoff = p.cutoff;
        lj_coeffs_ = p.coeffs;
        lj_special_ = p.special;
        have_pair_ = true;
        return *this;
    }
    MD& set_evaluator(const CoulLong& c) {
        d_.coul_enabled = 1;
        d_.coul_alpha = c.alpha;
        d_.coul_cutoff = c.cutoff;
        coul_special_ = c.special;
        have_pair_ = true;
        return *this;
    }
    MD& set_evaluator(const KSpacePME& k) {
        d_.pme_enabled = 1;
        d_.pme_alpha = k.alpha;
        d_.pme_grid_spacing = k.grid_spacing;
        d_.pme_order = k.order;
        for (int i = 0; i < 3; ++i)
            d_.pme_grid[i] = k.grid[i];
        return *this;
    }
    MD& set_integrator(const VelocityVerlet& v) {
        if (have_integrator_ && v.dt != d_.dt)
            throw std::invalid_argument("set_integrator already configured");
        d_.dt = v.dt;
        have_integrator_ = true;
        return *this;
    }
    MD& set_integrator(const NoseHooverNPT& v) {
        if (have_integrator_)
            throw std::invalid_argument("set_integrator already configured");
        d_.dt = v.dt;
        npt_ = v.p;
        have_npt_ = true;
        have_integrator_ = true;
        return *this;
    }
    MD& set_integrator(const NVELimit& v) {
        if (have_integrator_)
            throw std::invalid_argument("set_integrator already configured");
        d_.dt = v.dt;
        vlimit_ = v.xmax;
        have_integrator_ = true;
        return *this;
    }
    /// Deform is a plain component: set_thermostat binds it at its default
    /// slot, initial_integrate +200 (md.cuh:229-233, deform.cu:40-46).
    MD& set_thermostat(const Deform& d) {
        deform_axis_ = d.axis;
        deform_rate_ = d.strain_rate;
        return *this;
    }
    MD& set_deform(const Deform& d) { return set_thermostat(d); }
    /// LAMMPS `fix press/berendsen` (md.cuh:239-243); set_thermostat takes
    /// it too, as the reference's bind_defaults does.
    MD& set_barostat(const Barostat& b) {
        baro_ = b;
        have_baro_ = true;
        return *this;
    }
    MD& set_thermostat(const Barostat& b) { return set_barostat(b); }
    MD& set_thermostat(const NoseHoover& t) {
        d_.thermostat = ATVB_NOSE_HOOVER;
        d_.temperature = t.T;
        d_.tau = t.tau;
        return *this;
    }
    MD& set_thermostat(const FixLangevin& t) {
        ramp_T_stop_ = t.T_stop;
        ramp_nfirst_ = t.nfirst;
        ramp_nlast_ = t.nlast;
        d_.thermostat = ATVB_LANGEVIN;
        d_.temperature = t.T_start;
        d_.damp = t.damp;
        d_.seed = t.seed;
        return *this;
    }
    MD& set_stress_required(bool on) {
        d_.stress_required = on ? 1 : 0;
        return *this;
    }

    /// Thermo output every `every` steps (MD::set_thermo, md.cuh:249-262;
    /// cuda::Thermo, record/thermo.cuh): Step, Temp (2 KE / (Ndof k_B),
    /// Ndof = 3N - 3), PotEng, KinEng, TotEng in the columns of
    /// cpu::thermo_print (record/thermo.cpp:56-81), read from the device's
    /// per-step energy ring after each run.  Step is the driver's zero-based
    /// iteration index, continued across run() calls (md.cuh:170), and a row
    /// is printed where it is a multiple of `every` (driver.cu:128).
    /// Singular: a different cadence on a second call throws.  `filename`
    /// also writes the rows there.
    MD& set_thermo(int every, const std::string& filename = "") {
        if (every <= 0)
            every = 1; // "0 is every step"
        if (thermo_every_ > 0) {
            if (thermo_every_ == every)
                return *this;
            throw std::invalid_argument("set_thermo already configured with " +
                                        std::to_string(thermo_every_) +
                                        ", rejected re-call with " + std::to_string(every));
        }
        thermo_every_ = every;
        if (!filename.empty()) {
            thermo_file_.open(filename);
            if (thermo_file_.is_open())
                thermo_file_ << "# Step Temp PotEng KinEng TotEng\n";
        }
        return *this;
    }

    /// Advance n_steps; the first call uploads `frame`, every call leaves the
    /// device state in `frame` (MD::run, md.cuh:155-178).
    atvb_scalars run(Frame& frame, int n_steps) {
        if (!have_integrator_)
            throw std::invalid_argument("MD: set_integrator is required");
        if (have_pair_ && !have_nl_)
            throw std::invalid_argument(
                "cuda::md::MD: Add `sim.set_neighbor(cuda::NeighborList{cutoff})`.");
        ensure_system(frame);
        atvb_soa_view v = frame.view();
        atvb_scalars s{};
        if (thermo_every_ <= 0) {
            check(atvb_system_run(sys_, &v, n_steps, &s));
        } else {
            // in pieces no longer than the energy ring, printing each piece
            const int cap = d_.history_capacity > 0 ? d_.history_capacity : 4096;
            std::vector<double> h((size_t)3 * cap);
            int left = n_steps;
            do {
                const int k = left < cap ? left : cap;
                check(atvb_system_run(sys_, &v, k, &s));
                int32_t cnt = 0;
                if (k > 0)
                    check(atvb_system_energy_history(sys_, h.data(), k, &cnt));
                for (int r = 0; r < cnt; ++r)
                    thermo_row((long long)h[3 * r + 2], h[3 * r], h[3 * r + 1]);
                left -= k;
            } while (left > 0);
        }
        for (int k = 0; k < 3; ++k) // the cell moves under NPT
            frame.box[k] = s.box[k];
        return s;
    }

    /// Checkpoint of the whole resumable state (atvb_system_save).
    std::vector<char> checkpoint() {
        if (!sys_)
            throw std::logic_error("MD::checkpoint: nothing has run yet");
        int64_t nb = 0;
        check(atvb_system_checkpoint_size(sys_, &nb));
        std::vector<char> blob((size_t)nb);
        check(atvb_system_save(sys_, blob.data(), nb));
        return blob;
    }

    /// Resume from checkpoint() bytes in place of the first run's upload;
    /// `frame` supplies the atom count and box (same as the saved system).
    /// The next run(frame, n) continues the saved trajectory bit for bit.
    void restore(Frame& frame, const std::vector<char>& blob) {
        if (sys_)
            throw std::logic_error("MD::restore: the system already exists");
        create_system(frame);
        check(atvb_system_restore(sys_, blob.data(), (int64_t)blob.size()));
    }

    /// Trajectory snapshots every `every` steps into a host ring of `depth`
    /// frames (atvb_system_set_snapshots); read them with poll_snapshots.
    MD& set_snapshots(int every, int depth) {
        snap_every_ = every;
        snap_depth_ = depth;
        if (sys_)
            check(atvb_system_set_snapshots(sys_, every, depth));
        return *this;
    }

    /// Frames published since the last poll, no device synchronisation:
    /// steps[f], and x, y, z of frame f at xyz[3 n f + {0, n, 2n} + i].
    int poll_snapshots(std::vector<int64_t>& steps, std::vector<double>& xyz, int max_frames = 16) {
        if (!sys_)
            return 0;
        const int n = d_.n_atoms;
        steps.assign(max_frames, 0);
        xyz.assign((size_t)3 * n * max_frames, 0.0);
        std::vector<double> x((size_t)n * max_frames), y(x.size()), z(x.size());
        int32_t cnt = 0;
        int64_t dropped = 0;
        check(atvb_system_snapshot_poll(sys_, max_frames, steps.data(), nullptr, x.data(),
                                        y.data(), z.data(), nullptr, nullptr, nullptr, &cnt,
                                        &dropped));
        for (int f = 0; f < cnt; ++f)
            for (int i = 0; i < n; ++i) {
                xyz[(size_t)3 * n * f + i] = x[(size_t)n * f + i];
                xyz[(size_t)3 * n * f + n + i] = y[(size_t)n * f + i];
                xyz[(size_t)3 * n * f + 2 * n + i] = z[(size_t)n * f + i];
            }
        steps.resize(cnt);
        xyz.resize((size_t)3 * n * cnt);
        return cnt;
    }

  private:
    void thermo_row(long long step, double pe, double ke) {
        if (step % thermo_every_ != 0)
            return;
        const int ndof = 3 * d_.n_atoms - 3;
        const double kB = 8.617333262e-5; // eV/K (units.h:138)
        const double temp = ndof > 0 ? 2.0 * ke / ((double)ndof * kB) : 0.0;
        if (!thermo_header_) {
            std::printf("%8s %12s %14s %14s %14s\n", "Step", "Temp", "PotEng", "KinEng",
                        "TotEng");
            thermo_header_ = true;
        }
        std::printf("%8lld %12.4f %14.6f %14.6f %14.6f\n", step, temp, pe, ke, pe + ke);
        if (thermo_file_.is_open()) {
            char line[160];
            std::snprintf(line, sizeof line, "%lld %.6f %.6f %.6f %.6f\n", step, temp, pe, ke,
                          pe + ke);
            thermo_file_ << line;
        }
    }

    // a component and its slots; the first slot carries build and destroy
    struct Bound {
        std::shared_ptr<Component> c;
        bool first;
    };

    static int comp_build(void* u, const atvb_launch_ctx* x) {
        try {
            static_cast<Bound*>(u)->c->build(BuildContext{x->stream, x->frame});
            return 0;
        } catch (...) {
            return 1;
        }
    }
    static int comp_launch(void* u, const atvb_launch_ctx* x) {
        try {
            static_cast<Bound*>(u)->c->launch(LaunchContext{x->stream, x->frame, x->phase, x->step});
            return 0;
        } catch (...) {
            return 1;
        }
    }
    static int comp_destroy(void* u, const atvb_launch_ctx* x) {
        try {
            static_cast<Bound*>(u)->c->destroy(DestroyContext{x->stream, x->frame});
            return 0;
        } catch (...) {
            return 1;
        }
    }

    MD& add_component(std::shared_ptr<Component> c, const std::vector<std::pair<Phase, int>>& at) {
        for (size_t k = 0; k < at.size(); ++k) {
            if (at[k].first == Phase::COUNT)
                throw std::invalid_argument("MD::on: not a phase");
            bound_.push_back(std::unique_ptr<Bound>(new Bound{c, k == 0}));
            slots_.emplace_back(bound_.back().get(), at[k]);
            if (sys_) // the system exists: the component joins from the next call
                register_slot(slots_.back());
        }
        return *this;
    }

    void register_slot(const std::pair<Bound*, std::pair<Phase, int>>& s) {
        check(atvb_system_add_component(sys_, (int32_t)s.second.first, s.second.second,
                                        s.first->first ? comp_build : nullptr, comp_launch,
                                        s.first->first ? comp_destroy : nullptr, s.first));
    }

    void ensure_system(Frame& frame) {
        if (!sys_)
            create_system(frame);
    }

    void create_system(Frame& frame) {
        if (!have_integrator_)
            throw std::invalid_argument("MD: set_integrator is required");
        if (have_pair_ && !have_nl_)
            throw std::invalid_argument(
                "cuda::md::MD: Add `sim.set_neighbor(cuda::NeighborList{cutoff})`.");
        {
            d_.n_atoms = frame.n();
            d_.precision = precision_;
            for (int k = 0; k < 9; ++k)
                d_.box[k] = 0.0;
            d_.box[0] = frame.box[0];
            d_.box[4] = frame.box[1];
            d_.box[8] = frame.box[2];
            // install_defaults: the plan-level stress verdict, to every
            // component and to the library's own evaluators
            bool needs = d_.stress_required != 0 || have_npt_ || have_baro_;
            for (const auto& b : bound_)
                needs = needs || b->c->requires_system_stress();
            for (const auto& b : bound_)
                if (b->first)
                    b->c->set_stress_required(needs);
            d_.stress_required = needs ? 1 : 0;
            check(atvb_system_create(ctx_, &d_, &sys_));
            if (have_npt_)
                check(atvb_system_set_npt(sys_, &npt_));
            if (have_baro_)
                check(atvb_system_set_barostat(sys_, baro_.P_target, baro_.tau_P,
                                               baro_.bulk_modulus));
            if (vlimit_ > 0.0)
                check(atvb_system_set_nve_limit(sys_, vlimit_));
            if (deform_axis_ >= 0)
                check(atvb_system_set_deform(sys_, deform_axis_, deform_rate_));
            if (d_.thermostat == ATVB_LANGEVIN && ramp_T_stop_ != d_.temperature)
                check(atvb_system_set_langevin_ramp(sys_, ramp_T_stop_, ramp_nfirst_,
                                                    ramp_nlast_));
            if (!lj_coeffs_.empty()) {
                std::vector<int32_t> ti, tj;
                std::vector<double> e, sg;
                for (const auto& c : lj_coeffs_) {
                    ti.push_back(c.type_i);
                    tj.push_back(c.type_j);
                    e.push_back(c.epsilon);
                    sg.push_back(c.sigma);
                }
                check(atvb_system_set_lj_types(sys_, (int32_t)ti.size(), ti.data(), tj.data(),
                                               e.data(), sg.data()));
            }
            if (lj_special_.active() || coul_special_.active()) {
                const double lj[3] = {lj_special_.s12, lj_special_.s13, lj_special_.s14};
                const double co[3] = {coul_special_.s12, coul_special_.s13, coul_special_.s14};
                std::vector<int64_t> a, b;
                for (const auto& bd : frame.bonds) {
                    a.push_back(bd.first);
                    b.push_back(bd.second);
                }
                check(atvb_system_set_special_bonds(sys_, lj, co, (int64_t)a.size(), a.data(),
                                                    b.data()));
            }
            if (snap_every_ > 0)
                check(atvb_system_set_snapshots(sys_, snap_every_, snap_depth_));
            for (const auto& s : slots_)
                register_slot(s);
        }
    }

    atvb_ctx* ctx_ = nullptr;
    atvb_system* sys_ = nullptr;
    atvb_system_desc d_;
    double ramp_T_stop_ = -1.0;
    int64_t ramp_nfirst_ = 0, ramp_nlast_ = 0;
    std::vector<std::unique_ptr<Bound>> bound_;
    std::vector<std::pair<Bound*, std::pair<Phase, int>>> slots_;
    int precision_;
    bool have_nl_ = false, have_pair_ = false, have_integrator_ = false;
    std::vector<LJTypeCoeff> lj_coeffs_;
    atvb_npt_desc npt_{};
    bool have_npt_ = false;
    int snap_every_ = 0, snap_depth_ = 0;
    Barostat baro_{0.0, 1.0, 1.0};
    bool have_baro_ = false;
    int thermo_every_ = 0;
    bool thermo_header_ = false;
    std::ofstream thermo_file_;
    double vlimit_ = 0.0;
    int deform_axis_ = -1;
    double deform_rate_ = 0.0;
    SpecialScales lj_special_, coul_special_;
};
} // namespace md
} // namespace atvb_cpp
