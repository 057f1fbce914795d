// atvb_engine.h -- host-side engine: systems (slots), work lists, graph.
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "atvb.h"
#include "atvb_common.cuh"
#include "atvb_kernels.cuh"

struct atvb_ctx {
    int device = 0;
};

namespace atvb {

extern thread_local std::string g_last_error;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what);
int good_fft_size(int n);
size_t estimate_bytes(const atvb_system_desc& d);

struct Geometry {
    double L[3];
    double Lmin[3]; // smallest cell the bins and stencil are valid for
    double skin, rlist;
    int nc[3];
    double cs[3];
    int reach[3];
    int alias[3];
    std::vector<int4> cols;
};
Geometry make_geometry(const atvb_system_desc& d, double shrink = 0.0);

// Stream-ordered device memory from an engine's own pool.  Frees go back to
// the pool in stream order (no device-wide synchronisation, no unmapping),
// so systems can join and leave a running engine without stalling it.
struct DevMem {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    void* alloc(size_t bytes) const; // throws Error(ATVB_ERR_NOMEM)
    void free(void* p) const;
};

// One system's device memory and host mirror of its SysParams.
class Slot {
  public:
    Slot(const atvb_system_desc& d, const DevMem& mem);
    ~Slot();
    Slot(const Slot&) = delete;
    Slot& operator=(const Slot&) = delete;
    void alloc_list(int cap);
    void widen_list(int cap); // wider rows, the current list copied in

    atvb_system_desc desc;
    Geometry geo;
    SysParams hp;
    int index = -1;
    bool uploaded = false;
    size_t bytes = 0;
    int max_row = 0;
    int lanes = 4;  // pair-kernel lanes per atom for this system
    double mean_row = 0.0;
    // per-type LJ and special bonds: configured before the first upload
    int ntypes = 0;          // > 0: per-type LJ (table built at upload)
    std::vector<int> lj_ti, lj_tj;
    std::vector<double> lj_eps, lj_sig;
    void build_lj_tables(const std::vector<int>& types, cudaStream_t stream);
    bool special_set = false;
    double sp_lj[3] = {1, 1, 1}, sp_coul[3] = {1, 1, 1};
    std::vector<long long> bond_a, bond_b;
    void build_specials(const std::vector<long long>& tags, cudaStream_t stream);

    void* dalloc(size_t b);
    void free_alloc(void* p);
    void replan_cells(double shrink);
    bool npt = false; // MTK NPT configured (atvb_system_set_npt)
    atvb_npt_desc npt_desc{};
    bool baro = false; // Berendsen barostat configured (atvb_system_set_barostat)
    double baro_args[3] = {0, 0, 0}; // P_target, tau_P, bulk_modulus
    double vlimit_xmax = 0.0;        // NVELimit xmax (0: plain velocity Verlet)
    double deform_args[3] = {0, 0, 0}; // Deform axis, strain rate, L0
    int row_cap_fixed = 0;     // atvb_system_set_capacity: pinned row length
    char* snap_host = nullptr; // trajectory snapshot ring (host-mapped)
    long long snap_read = 0;   // snapshots consumed by the host

  private:
    DevMem mem_;
    std::vector<void*> allocs;
    void* nbr_alloc = nullptr;
};

// A user component's callbacks at one phase (atvb_system_add_component).
struct UserComp {
    int slot, phase, order, seq;
    atvb_component_fn build, launch, destroy;
    void* user;
    bool built;
};

struct ProfEntry {
    std::string name;
    double ms;
    long long launches;
};

class Engine {
  public:
    explicit Engine(int device);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    int add(const atvb_system_desc& d);
    void remove(int id);
    Slot* slot(int id);
    void upload(int id, const atvb_soa_view& f);
    void set_lj_types(int id, int ncoef, const int32_t* ti, const int32_t* tj,
                      const double* eps, const double* sigma);
    void set_special_bonds(int id, const double lj[3], const double coul[3],
                           int64_t nbonds, const int64_t* a, const int64_t* b);
    void set_npt(int id, const atvb_npt_desc& p);
    void set_barostat(int id, double P_target, double tau_P, double bulk_modulus);
    void set_nve_limit(int id, double xmax);
    void set_deform(int id, int axis, double rate, double L0 = 0.0);
    void set_snapshots(int id, int every, int depth);
    int poll_snapshots(int id, int max_frames, int64_t* steps, double* box,
                       double* const out[6], int64_t* dropped);
    size_t checkpoint_bytes(int id);
    void save(int id, void* buf, size_t cap);
    void restore(int id, const void* buf, size_t size, bool fresh_list = false);
    void replan_npt();
    void compute_forces();
    void compute_forces_one(int id);
    void step(int n);
    void step_timed(int n, double* step_ms, double* total_ms);
    void check_halted(int id); // throws ATVB_ERR_PHYSICS if StopOnNaN stopped it
    void clear_status(int id);
    void set_stop_on_nan(int id, bool on);
    void set_langevin_ramp(int id, double T_stop, long long nfirst, long long nlast);
    void add_component(int id, int phase, int order, atvb_component_fn build,
                       atvb_component_fn launch, atvb_component_fn destroy, void* user);
    void set_capacity(int id, int row_cap, int nearq_cap);
    void download(int id, atvb_soa_view* f, atvb_scalars* sc);
    void scalars(int id, atvb_scalars* out);
    int64_t pairs(int id, int32_t* pi, int32_t* pj, int64_t capacity);
    int history(int id, double* out, int max_steps);
    void set_lanes(int lanes);
    int autotune();
    void set_profiling(bool on) { profiling_ = on; }
    const std::vector<ProfEntry>& profile() const { return prof_acc_; }
    void clear_profile() { prof_acc_.clear(); }
    int64_t last_launches() const { return last_launches_; }
    int64_t kernels_per_step() const;
    cudaStream_t stream() const { return stream_; }
    int device() const { return device_; }
    int lanes() const { return lc_.pair_G; }
    size_t slot_count() const { return slots_.size(); }
    bool has(int id) const {
        return id >= 0 && id < (int)slots_.size() && slots_[id] != nullptr;
    }

  private:
    FftCfg fft_items(const std::vector<int>& pme);
    void ensure_table();
    void push_params(int id);
    void build_lists();
    void ensure_ready();
    int lanes_for(const Slot& s) const;
    bool check_lists(const LaunchCfg& lc);
    void sized_rebuild(const LaunchCfg& lc);
    LaunchCfg restricted_cfg(int id);
    void enqueue_step(bool profile);
    void widen_rows();
    int deform_budget(int n);
    void run_steps(int n);
    void run_pieces(int n, double* step_ms, double* total_ms);
    void ensure_graph();
    bool all_halted() const;
    void enqueue_forces(const LaunchCfg& lc, const std::vector<int>& pme,
                        bool profile, bool overlap, bool build_list = false);
    void prof_mark(bool profile, const char* next);
    template <typename F>
    void capture_if(cudaGraphConditionalHandle h, F&& body);
    atvb_launch_ctx comp_ctx(const UserComp& c, int phase) const;
    void build_components();
    void run_components(int phase, bool before);
    void zero_component_sums();
    void enqueue_step_components();
    void collect_profile();
    void release_graph();

    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    DevMem mem_;
    cudaStream_t pme_stream_ = nullptr; // the PME chain beside the pair kernel
    // the list build as conditional nodes of the step graph: the handle of
    // the graph being captured and the stream their bodies are captured on
    cudaStream_t cond_stream_ = nullptr;
    cudaGraphConditionalHandle cond_sort_ = 0, cond_rows_ = 0; // one per node
    bool capturing_ = false;
    cudaEvent_t pme_fork_ = nullptr, pme_join_ = nullptr;
    bool any_npt_ = false; // an MTK NPT system exists (re-plan check per step call)
    int num_sms_ = 148;
    std::vector<std::unique_ptr<Slot>> slots_;
    SysParams* d_sp_ = nullptr;
    int sp_cap_ = 0;
    // host-mapped words, 2 per table entry: the longest-row hints
    // (SysParams::row_hint) in [0, sp_cap_), the status words
    // (SysParams::status_hint) in [sp_cap_, 2 sp_cap_)
    int* row_hint_host_ = nullptr;
    int* row_hint_dev_ = nullptr;
    std::vector<void*> list_allocs_;
    LaunchCfg lc_;
    std::vector<int> pme_slots_;
    bool dirty_ = true;
    int list_epoch_ = 0;
    std::map<int, std::pair<int, LaunchCfg>> single_;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t gexec_ = nullptr;
    int lanes_fixed_ = 0;
    int64_t last_launches_ = 0;
    int64_t steps_since_check_ = 0;
    bool profiling_ = false;
    std::vector<cudaEvent_t> prof_events_;
    size_t prof_used_ = 0;
    std::vector<std::string> prof_seq_;
    std::vector<ProfEntry> prof_acc_;
    std::vector<UserComp> comps_; // sorted by (phase, order, seq)
    long long comp_step_ = 0;     // cumulative index of the step being taken
};

} // namespace atvb
