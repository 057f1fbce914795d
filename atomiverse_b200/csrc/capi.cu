// capi.cu -- the extern "C" boundary (include/atvb.h).  Every entry point
// catches exceptions, records the message for atvb_last_error() and returns
// a status code; nothing C++ crosses the boundary.
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "atvb.h"
#include "atvb_engine.h"

using atvb::Engine;
using atvb::Error;

struct atvb_system {
    atvb_ctx* ctx = nullptr;
    std::unique_ptr<Engine> eng;
    int id = -1;
    bool uploaded = false;
};

struct atvb_batch {
    atvb_ctx* ctx = nullptr;
    std::unique_ptr<Engine> eng;
    std::vector<int> ids;
};

namespace {

template <typename F>
int guard(F&& f) {
    try {
        f();
        atvb::g_last_error.clear();
        return ATVB_OK;
    } catch (const Error& e) {
        atvb::g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        atvb::g_last_error = "host allocation failed";
        return ATVB_ERR_NOMEM;
    } catch (const std::exception& e) {
        atvb::g_last_error = e.what();
        return ATVB_ERR_INVALID;
    } catch (...) {
        atvb::g_last_error = "unknown error";
        return ATVB_ERR_INVALID;
    }
}

void need(const void* p, const char* what) {
    if (!p)
        throw Error(ATVB_ERR_INVALID, std::string(what) + " is NULL");
}

// After a call has filled its outputs: any sticky status bit of the system
// makes it return ATVB_ERR_PHYSICS, so wrong physics is never silent.
void raise_status(Engine& e, int id, const atvb_scalars* sc) {
    atvb_scalars local;
    if (!sc) {
        e.scalars(id, &local);
        sc = &local;
    }
    const uint32_t b = sc->status_bits;
    if (!b)
        return;
    std::string m = "system status:";
    if (b & ATVB_STATUS_ROW_OVERFLOW)
        m += " neighbour rows were cut at capacity (pairs lost);";
    if (b & ATVB_STATUS_BOX_RANGE)
        m += " the cell was held at the edge of its planned range;";
    if (b & ATVB_STATUS_NEARQ_LOST)
        m += " near-cutoff pairs overflowed the settle queue;";
    if (b & ATVB_STATUS_NONFINITE)
        m += " a position or velocity is not finite;";
    if (b & ATVB_STATUS_FORCE_RANGE)
        m += " a pair force exceeded the fixed-point range;";
    if (sc->halted)
        m += " stopped by StopOnNaN at step " + std::to_string(sc->step) + ";";
    m += " (atvb_system_clear_status resets the bits)";
    throw Error(ATVB_ERR_PHYSICS, m);
}

} // namespace

extern "C" {

int atvb_abi_version(void) { return ATVB_ABI_VERSION; }

const char* atvb_last_error(void) { return atvb::g_last_error.c_str(); }

int atvb_ctx_create(const atvb_device_opts* opts, atvb_ctx** out) {
    return guard([&] {
        need(out, "out");
        int dev = opts ? opts->device : 0;
        int count = 0;
        atvb::cuda_check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
        if (dev < 0 || dev >= count)
            throw Error(ATVB_ERR_INVALID, "no CUDA device " + std::to_string(dev));
        atvb::cuda_check(cudaSetDevice(dev), "cudaSetDevice");
        auto* c = new atvb_ctx;
        c->device = dev;
        *out = c;
    });
}

int atvb_ctx_destroy(atvb_ctx* ctx) {
    return guard([&] { delete ctx; });
}


// ---- single system ------------------------------------------------------

int atvb_system_create(atvb_ctx* ctx, const atvb_system_desc* desc,
                       atvb_system** out) {
    return guard([&] {
        need(ctx, "ctx");
        need(desc, "desc");
        need(out, "out");
        auto s = std::make_unique<atvb_system>();
        s->ctx = ctx;
        s->eng = std::make_unique<Engine>(ctx->device);
        s->id = s->eng->add(*desc);
        *out = s.release();
    });
}

int atvb_system_destroy(atvb_system* sys) {
    return guard([&] { delete sys; });
}

int atvb_system_upload(atvb_system* sys, const atvb_soa_view* frame) {
    return guard([&] {
        need(sys, "sys");
        need(frame, "frame");
        sys->eng->upload(sys->id, *frame);
        sys->uploaded = true;
    });
}

int atvb_system_compute_forces(atvb_system* sys) {
    return guard([&] {
        need(sys, "sys");
        if (!sys->uploaded)
            throw Error(ATVB_ERR_STATE, "compute_forces before upload");
        sys->eng->compute_forces();
    });
}

int atvb_system_step(atvb_system* sys, int32_t n_steps) {
    return guard([&] {
        need(sys, "sys");
        if (!sys->uploaded)
            throw Error(ATVB_ERR_STATE, "step before upload");
        sys->eng->check_halted(sys->id);
        sys->eng->step(n_steps);
    });
}

int atvb_system_step_timed(atvb_system* sys, int32_t n_steps, double* step_ms,
                           double* total_ms) {
    return guard([&] {
        need(sys, "sys");
        if (!sys->uploaded)
            throw Error(ATVB_ERR_STATE, "step before upload");
        if (n_steps < 1)
            throw Error(ATVB_ERR_INVALID, "n_steps must be >= 1");
        sys->eng->check_halted(sys->id);
        sys->eng->step_timed(n_steps, step_ms, total_ms);
    });
}

int atvb_system_download(atvb_system* sys, atvb_soa_view* frame,
                         atvb_scalars* scalars) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->download(sys->id, frame, scalars);
        raise_status(*sys->eng, sys->id, scalars);
    });
}

int atvb_system_scalars(atvb_system* sys, atvb_scalars* scalars) {
    return guard([&] {
        need(sys, "sys");
        need(scalars, "scalars");
        sys->eng->scalars(sys->id, scalars);
        raise_status(*sys->eng, sys->id, scalars);
    });
}

int atvb_system_clear_status(atvb_system* sys) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->clear_status(sys->id);
    });
}

int atvb_system_add_component(atvb_system* sys, int32_t phase, int32_t order,
                              atvb_component_fn build, atvb_component_fn launch,
                              atvb_component_fn destroy, void* user) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->add_component(sys->id, phase, order, build, launch, destroy, user);
    });
}

int atvb_system_set_langevin_ramp(atvb_system* sys, double T_stop, int64_t nfirst,
                                  int64_t nlast) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_langevin_ramp(sys->id, T_stop, nfirst, nlast);
    });
}

int atvb_system_set_stop_on_nan(atvb_system* sys, int32_t on) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_stop_on_nan(sys->id, on != 0);
    });
}

int atvb_system_set_capacity(atvb_system* sys, int32_t row_capacity,
                             int32_t nearq_capacity) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_capacity(sys->id, row_capacity, nearq_capacity);
    });
}

int atvb_system_run(atvb_system* sys, atvb_soa_view* frame, int32_t n_steps,
                    atvb_scalars* scalars) {
    return guard([&] {
        need(sys, "sys");
        need(frame, "frame");
        if (!sys->uploaded) {
            sys->eng->upload(sys->id, *frame);
            sys->uploaded = true;
        }
        sys->eng->check_halted(sys->id);
        sys->eng->step(n_steps);
        sys->eng->download(sys->id, frame, scalars);
        raise_status(*sys->eng, sys->id, scalars);
    });
}

int atvb_system_energy_history(atvb_system* sys, double* out,
                               int32_t max_steps, int32_t* count) {
    return guard([&] {
        need(sys, "sys");
        need(out, "out");
        int c = sys->eng->history(sys->id, out, max_steps);
        if (count)
            *count = c;
    });
}

int atvb_system_pairs(atvb_system* sys, int32_t* pi, int32_t* pj,
                      int64_t capacity, int64_t* count) {
    return guard([&] {
        need(sys, "sys");
        int64_t c = sys->eng->pairs(sys->id, pi, pj, capacity);
        if (count)
            *count = c;
    });
}

int atvb_system_set_snapshots(atvb_system* sys, int32_t every, int32_t depth) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_snapshots(sys->id, every, depth);
    });
}

int atvb_system_snapshot_poll(atvb_system* sys, int32_t max_frames, int64_t* steps,
                              double* box, double* x, double* y, double* z, double* vx,
                              double* vy, double* vz, int32_t* count, int64_t* dropped) {
    return guard([&] {
        need(sys, "sys");
        if (max_frames < 0)
            throw Error(ATVB_ERR_INVALID, "max_frames must be >= 0");
        double* const out[6] = {x, y, z, vx, vy, vz};
        const int c = sys->eng->poll_snapshots(sys->id, max_frames, steps, box, out, dropped);
        if (count)
            *count = c;
    });
}

int atvb_system_checkpoint_size(atvb_system* sys, int64_t* bytes) {
    return guard([&] {
        need(sys, "sys");
        need(bytes, "bytes");
        *bytes = (int64_t)sys->eng->checkpoint_bytes(sys->id);
    });
}

int atvb_system_save(atvb_system* sys, void* buf, int64_t capacity) {
    return guard([&] {
        need(sys, "sys");
        need(buf, "buf");
        sys->eng->save(sys->id, buf, capacity < 0 ? 0 : (size_t)capacity);
    });
}

int atvb_system_restore(atvb_system* sys, const void* buf, int64_t size) {
    return guard([&] {
        need(sys, "sys");
        need(buf, "buf");
        sys->eng->restore(sys->id, buf, size < 0 ? 0 : (size_t)size);
        sys->uploaded = true;
    });
}

int atvb_batch_checkpoint_size(atvb_batch* b, int32_t index, int64_t* bytes) {
    return guard([&] {
        need(b, "batch");
        need(bytes, "bytes");
        if (index < 0 || index >= (int)b->ids.size())
            throw Error(ATVB_ERR_NOTFOUND, "no system " + std::to_string(index) + " in batch");
        *bytes = (int64_t)b->eng->checkpoint_bytes(b->ids[index]);
    });
}

int atvb_batch_save(atvb_batch* b, int32_t index, void* buf, int64_t capacity) {
    return guard([&] {
        need(b, "batch");
        need(buf, "buf");
        if (index < 0 || index >= (int)b->ids.size())
            throw Error(ATVB_ERR_NOTFOUND, "no system " + std::to_string(index) + " in batch");
        b->eng->save(b->ids[index], buf, capacity < 0 ? 0 : (size_t)capacity);
    });
}

int atvb_batch_restore(atvb_batch* b, int32_t index, const void* buf, int64_t size) {
    return guard([&] {
        need(b, "batch");
        need(buf, "buf");
        if (index < 0 || index >= (int)b->ids.size())
            throw Error(ATVB_ERR_NOTFOUND, "no system " + std::to_string(index) + " in batch");
        b->eng->restore(b->ids[index], buf, size < 0 ? 0 : (size_t)size);
    });
}

int atvb_system_set_barostat(atvb_system* sys, double P_target, double tau_P,
                             double bulk_modulus) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_barostat(sys->id, P_target, tau_P, bulk_modulus);
    });
}

int atvb_batch_set_barostat(atvb_batch* b, int32_t index, double P_target, double tau_P,
                            double bulk_modulus) {
    return guard([&] {
        need(b, "batch");
        if (index < 0 || index >= (int)b->ids.size())
            throw Error(ATVB_ERR_NOTFOUND, "no system " + std::to_string(index) + " in batch");
        b->eng->set_barostat(b->ids[index], P_target, tau_P, bulk_modulus);
    });
}

int atvb_system_set_nve_limit(atvb_system* sys, double xmax) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_nve_limit(sys->id, xmax);
    });
}

int atvb_system_set_deform(atvb_system* sys, int32_t axis, double strain_rate) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_deform(sys->id, axis, strain_rate);
    });
}

int atvb_batch_set_nve_limit(atvb_batch* b, int32_t index, double xmax) {
    return guard([&] {
        need(b, "batch");
        if (index < 0 || index >= (int)b->ids.size())
            throw Error(ATVB_ERR_NOTFOUND, "no system " + std::to_string(index) + " in batch");
        b->eng->set_nve_limit(b->ids[index], xmax);
    });
}

int atvb_batch_set_deform(atvb_batch* b, int32_t index, int32_t axis, double strain_rate) {
    return guard([&] {
        need(b, "batch");
        if (index < 0 || index >= (int)b->ids.size())
            throw Error(ATVB_ERR_NOTFOUND, "no system " + std::to_string(index) + " in batch");
        b->eng->set_deform(b->ids[index], axis, strain_rate);
    });
}

int atvb_system_set_npt(atvb_system* sys, const atvb_npt_desc* npt) {
    return guard([&] {
        need(sys, "sys");
        need(npt, "npt");
        sys->eng->set_npt(sys->id, *npt);
    });
}

int atvb_system_set_lj_types(atvb_system* sys, int32_t ncoef, const int32_t* type_i,
                             const int32_t* type_j, const double* epsilon,
                             const double* sigma) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_lj_types(sys->id, ncoef, type_i, type_j, epsilon, sigma);
    });
}

int atvb_system_set_special_bonds(atvb_system* sys, const double lj[3], const double coul[3],
                                  int64_t nbonds, const int64_t* tag_a, const int64_t* tag_b) {
    return guard([&] {
        need(sys, "sys");
        need(lj, "lj");
        need(coul, "coul");
        sys->eng->set_special_bonds(sys->id, lj, coul, nbonds, tag_a, tag_b);
    });
}

int atvb_system_profile(atvb_system* sys, int32_t enable) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_profiling(enable != 0);
        if (enable)
            sys->eng->clear_profile();
    });
}

int atvb_system_profile_read(atvb_system* sys, atvb_kernel_time* out,
                             int32_t capacity, int32_t* count) {
    return guard([&] {
        need(sys, "sys");
        const auto& p = sys->eng->profile();
        int c = 0;
        for (const auto& e : p) {
            if (c >= capacity)
                break;
            if (out) {
                std::memset(&out[c], 0, sizeof(atvb_kernel_time));
                std::strncpy(out[c].name, e.name.c_str(), sizeof(out[c].name) - 1);
                out[c].total_ms = e.ms;
                out[c].launches = e.launches;
            }
            ++c;
        }
        if (count)
            *count = c;
    });
}

int atvb_system_set_pair_lanes(atvb_system* sys, int32_t lanes) {
    return guard([&] {
        need(sys, "sys");
        sys->eng->set_lanes(lanes);
    });
}

int atvb_system_launch_count(atvb_system* sys, int64_t* launches) {
    return guard([&] {
        need(sys, "sys");
        need(launches, "launches");
        *launches = sys->eng->last_launches();
    });
}

void* atvb_system_stream(atvb_system* sys) {
    return sys ? (void*)sys->eng->stream() : nullptr;
}

// ---- batch --------------------------------------------------------------

int atvb_batch_create(atvb_ctx* ctx, const atvb_system_desc* descs,
                      int32_t n_systems, atvb_batch** out) {
    return guard([&] {
        need(ctx, "ctx");
        need(descs, "descs");
        need(out, "out");
        if (n_systems < 1)
            throw Error(ATVB_ERR_INVALID, "n_systems must be >= 1");
        auto b = std::make_unique<atvb_batch>();
        b->ctx = ctx;
        b->eng = std::make_unique<Engine>(ctx->device);
        for (int k = 0; k < n_systems; ++k)
            b->ids.push_back(b->eng->add(descs[k]));
        *out = b.release();
    });
}

int atvb_batch_destroy(atvb_batch* b) {
    return guard([&] { delete b; });
}

static int batch_id(atvb_batch* b, int32_t index) {
    if (index < 0 || index >= (int)b->ids.size())
        throw Error(ATVB_ERR_NOTFOUND, "batch index out of range");
    return b->ids[index];
}

int atvb_batch_upload(atvb_batch* b, int32_t index, const atvb_soa_view* frame) {
    return guard([&] {
        need(b, "batch");
        need(frame, "frame");
        b->eng->upload(batch_id(b, index), *frame);
    });
}

int atvb_batch_compute_forces(atvb_batch* b) {
    return guard([&] {
        need(b, "batch");
        b->eng->compute_forces();
    });
}

int atvb_batch_step(atvb_batch* b, int32_t n_steps) {
    return guard([&] {
        need(b, "batch");
        b->eng->step(n_steps);
    });
}

int atvb_batch_download(atvb_batch* b, int32_t index, atvb_soa_view* frame,
                        atvb_scalars* scalars) {
    return guard([&] {
        need(b, "batch");
        b->eng->download(batch_id(b, index), frame, scalars);
        raise_status(*b->eng, batch_id(b, index), scalars);
    });
}

int atvb_batch_clear_status(atvb_batch* b, int32_t index) {
    return guard([&] {
        need(b, "batch");
        b->eng->clear_status(batch_id(b, index));
    });
}

int atvb_batch_set_langevin_ramp(atvb_batch* b, int32_t index, double T_stop,
                                 int64_t nfirst, int64_t nlast) {
    return guard([&] {
        need(b, "batch");
        b->eng->set_langevin_ramp(batch_id(b, index), T_stop, nfirst, nlast);
    });
}

int atvb_batch_set_stop_on_nan(atvb_batch* b, int32_t index, int32_t on) {
    return guard([&] {
        need(b, "batch");
        b->eng->set_stop_on_nan(batch_id(b, index), on != 0);
    });
}

int atvb_batch_autotune(atvb_batch* b, int32_t* lanes) {
    return guard([&] {
        need(b, "batch");
        const int g = b->eng->autotune();
        if (lanes)
            *lanes = g;
    });
}

int atvb_batch_set_lj_types(atvb_batch* b, int32_t index, int32_t ncoef,
                            const int32_t* type_i, const int32_t* type_j,
                            const double* epsilon, const double* sigma) {
    return guard([&] {
        need(b, "batch");
        if (index < 0 || index >= (int)b->ids.size())
            throw Error(ATVB_ERR_NOTFOUND, "no system " + std::to_string(index) + " in batch");
        b->eng->set_lj_types(b->ids[index], ncoef, type_i, type_j, epsilon, sigma);
    });
}

int atvb_batch_set_npt(atvb_batch* b, int32_t index, const atvb_npt_desc* npt) {
    return guard([&] {
        need(b, "batch");
        need(npt, "npt");
        if (index < 0 || index >= (int)b->ids.size())
            throw Error(ATVB_ERR_NOTFOUND, "no system " + std::to_string(index) + " in batch");
        b->eng->set_npt(b->ids[index], *npt);
    });
}

int atvb_batch_set_special_bonds(atvb_batch* b, int32_t index, const double lj[3],
                                 const double coul[3], int64_t nbonds, const int64_t* tag_a,
                                 const int64_t* tag_b) {
    return guard([&] {
        need(b, "batch");
        need(lj, "lj");
        need(coul, "coul");
        if (index < 0 || index >= (int)b->ids.size())
            throw Error(ATVB_ERR_NOTFOUND, "no system " + std::to_string(index) + " in batch");
        b->eng->set_special_bonds(b->ids[index], lj, coul, nbonds, tag_a, tag_b);
    });
}

int atvb_batch_profile(atvb_batch* b, int32_t enable) {
    return guard([&] {
        need(b, "batch");
        b->eng->set_profiling(enable != 0);
        if (enable)
            b->eng->clear_profile();
    });
}

int atvb_batch_profile_read(atvb_batch* b, atvb_kernel_time* out, int32_t capacity,
                            int32_t* count) {
    return guard([&] {
        need(b, "batch");
        const auto& p = b->eng->profile();
        int c = 0;
        for (const auto& e : p) {
            if (c >= capacity)
                break;
            if (out) {
                std::memset(&out[c], 0, sizeof(atvb_kernel_time));
                std::strncpy(out[c].name, e.name.c_str(), sizeof(out[c].name) - 1);
                out[c].total_ms = e.ms;
                out[c].launches = e.launches;
            }
            ++c;
        }
        if (count)
            *count = c;
    });
}

int atvb_batch_launch_count(atvb_batch* b, int64_t* launches) {
    return guard([&] {
        need(b, "batch");
        need(launches, "launches");
        *launches = b->eng->last_launches();
    });
}

int atvb_request_bytes(const atvb_system_desc* desc, size_t* bytes) {
    return guard([&] {
        need(desc, "desc");
        need(bytes, "bytes");
        *bytes = atvb::estimate_bytes(*desc);
    });
}

} // extern "C"
