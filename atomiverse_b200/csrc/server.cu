// server.cu -- continuous batching of MD segment requests on one device.
//
// A request is one system plus a step budget.  Each tick the server (1)
// admits queued requests while the device-memory budget and the slot limit
// allow (a request that does not fit is skipped over, unless it has waited
// longer than kMaxSkipWait, in which case admission stops behind it so it
// cannot starve), (2) advances every resident system together by one
// batched launch sequence of `chunk` steps (never past the nearest finish),
// and (3) retires finished requests: their frames are copied out and their
// device memory released.  Positions, velocities, neighbour lists and PME
// grids stay resident on the device between ticks.  A system's arithmetic
// does not depend on which other systems share the launch (per-atom work,
// fixed-point sums flushed per work item), so a request's result is the same
// alone and in the mix.
#include <algorithm>
#include <cstring>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "atvb.h"
#include "atvb_engine.h"

using atvb::Engine;
using atvb::Error;

namespace {

constexpr double kMaxSkipWait = 0.5; // seconds

struct Request {
    int64_t id = 0;
    atvb_system_desc desc{};
    std::vector<double> x, y, z, vx, vy, vz, fx, fy, fz, m, q;
    std::vector<int64_t> tag;
    int n_steps = 0;
    int steps_done = 0;
    int state = 0; // 0 queued, 1 running, 2 done, 3 cancelled, 4 failed, 5 suspended
    std::vector<char> ckpt; // resumable state (suspended, kept, or submitted)
    bool resume = false;    // admit from ckpt instead of the frame
    int slot = -1;
    size_t bytes = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    atvb_scalars sc{};

    atvb_soa_view view() {
        atvb_soa_view v{};
        v.x = x.data();
        v.y = y.data();
        v.z = z.data();
        v.vx = vx.data();
        v.vy = vy.data();
        v.vz = vz.data();
        v.fx = fx.data();
        v.fy = fy.data();
        v.fz = fz.data();
        v.mass = m.data();
        v.charge = q.data();
        v.tag = tag.data();
        return v;
    }
};

} // namespace

struct atvb_server {
    atvb_ctx* ctx = nullptr;
    std::unique_ptr<Engine> eng;
    size_t budget = 0;
    int max_active = 0;
    size_t in_use = 0;
    int64_t max_atoms = 0;   // resident-atom cap (0: none)
    bool keep_ckpt = false;  // finished requests keep a checkpoint (resumable)
    int64_t atoms_in_use = 0;
    int64_t next_id = 1;
    std::map<int64_t, Request> reqs;
    std::deque<int64_t> queue;
    std::vector<int64_t> running;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() -
                                             t0)
            .count();
    }

    Request& get(int64_t id) {
        auto it = reqs.find(id);
        if (it == reqs.end())
            throw Error(ATVB_ERR_NOTFOUND, "unknown request " + std::to_string(id));
        return it->second;
    }

    void admit() {
        const double t = now();
        for (auto it = queue.begin(); it != queue.end();) {
            if ((int)running.size() >= max_active)
                break;
            Request& r = get(*it);
            const bool over_atoms = max_atoms > 0 && !running.empty() &&
                                    atoms_in_use + r.desc.n_atoms > max_atoms;
            if (in_use + r.bytes > budget || over_atoms) {
                if (t - r.t_submit > kMaxSkipWait)
                    break; // hold the line for a request that waited long
                ++it;
                continue;
            }
            try {
                r.slot = eng->add(r.desc);
                if (r.resume) {
                    eng->restore(r.slot, r.ckpt.data(), r.ckpt.size());
                } else {
                    eng->upload(r.slot, r.view());
                    eng->compute_forces_one(r.slot);
                }
            } catch (const Error& e) {
                if (r.slot >= 0 && eng->has(r.slot))
                    eng->remove(r.slot);
                r.slot = -1;
                if (e.code == ATVB_ERR_NOMEM) {
                    ++it; // retry later when memory frees up
                    continue;
                }
                r.state = 4;
                r.t_done = now();
                it = queue.erase(it);
                continue;
            }
            r.state = 1;
            r.t_start = now();
            in_use += r.bytes;
            atoms_in_use += r.desc.n_atoms;
            running.push_back(r.id);
            it = queue.erase(it);
        }
    }

    void save(Request& r) {
        r.ckpt.resize(eng->checkpoint_bytes(r.slot));
        eng->save(r.slot, r.ckpt.data(), r.ckpt.size());
    }

    void retire(Request& r, bool keep_frame, bool keep_state = false) {
        if (keep_state)
            save(r);
        if (keep_frame) {
            atvb_soa_view v = r.view();
            eng->download(r.slot, &v, &r.sc);
        }
        eng->remove(r.slot);
        r.slot = -1;
        in_use -= r.bytes;
        atoms_in_use -= r.desc.n_atoms;
        running.erase(std::remove(running.begin(), running.end(), r.id),
                      running.end());
    }

    void tick(int chunk) {
        admit();
        if (running.empty())
            return;
        int n = chunk > 0 ? chunk : 1;
        for (int64_t id : running) {
            const Request& r = get(id);
            n = std::min(n, r.n_steps - r.steps_done);
        }
        if (n > 0)
            eng->step(n);
        std::vector<int64_t> done;
        for (int64_t id : running) {
            Request& r = get(id);
            r.steps_done += n;
            if (r.steps_done >= r.n_steps)
                done.push_back(id);
        }
        for (int64_t id : done) {
            Request& r = get(id);
            retire(r, true, keep_ckpt);
            // a segment that ran on wrong or non-finite physics (a sticky
            // status bit, atvb_scalars.status_bits) ends as failed; its frame
            // can still be collected
            r.state = r.sc.status_bits ? 4 : 2;
            r.t_done = now();
        }
    }
};

namespace {
template <typename F>
int sguard(F&& f) {
    try {
        f();
        atvb::g_last_error.clear();
        return ATVB_OK;
    } catch (const Error& e) {
        atvb::g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        atvb::g_last_error = e.what();
        return ATVB_ERR_INVALID;
    }
}
} // namespace

extern "C" {

int atvb_server_create(atvb_ctx* ctx, size_t hbm_budget_bytes,
                       int32_t max_active, atvb_server** out) {
    return sguard([&] {
        if (!ctx || !out)
            throw Error(ATVB_ERR_INVALID, "ctx/out is NULL");
        auto s = std::make_unique<atvb_server>();
        s->ctx = ctx;
        s->eng = std::make_unique<Engine>(ctx->device);
        s->budget = hbm_budget_bytes;
        s->max_active = max_active > 0 ? max_active : 1 << 20;
        *out = s.release();
    });
}

int atvb_server_destroy(atvb_server* srv) {
    return sguard([&] { delete srv; });
}

int atvb_server_submit(atvb_server* srv, const atvb_system_desc* desc,
                       const atvb_soa_view* frame, int32_t n_steps,
                       int64_t* id) {
    return sguard([&] {
        if (!srv || !desc || !frame || !frame->x || !frame->y || !frame->z)
            throw Error(ATVB_ERR_INVALID, "server/desc/frame is NULL");
        if (n_steps < 0)
            throw Error(ATVB_ERR_INVALID, "n_steps must be >= 0");
        atvb::make_geometry(*desc); // validate now, not at admission
        Request r;
        r.id = srv->next_id++;
        r.desc = *desc;
        const int n = desc->n_atoms;
        auto cp = [&](std::vector<double>& dst, const double* src, double fill) {
            dst.assign(n, fill);
            if (src)
                std::copy(src, src + n, dst.begin());
        };
        cp(r.x, frame->x, 0.0);
        cp(r.y, frame->y, 0.0);
        cp(r.z, frame->z, 0.0);
        cp(r.vx, frame->vx, 0.0);
        cp(r.vy, frame->vy, 0.0);
        cp(r.vz, frame->vz, 0.0);
        cp(r.fx, frame->fx, 0.0);
        cp(r.fy, frame->fy, 0.0);
        cp(r.fz, frame->fz, 0.0);
        cp(r.m, frame->mass, 1.0);
        cp(r.q, frame->charge, 0.0);
        r.tag.resize(n);
        for (int i = 0; i < n; ++i)
            r.tag[i] = frame->tag ? frame->tag[i] : i + 1;
        r.n_steps = n_steps;
        r.bytes = atvb::estimate_bytes(*desc);
        if (r.bytes > srv->budget)
            throw Error(ATVB_ERR_NOMEM,
                        "request needs " + std::to_string(r.bytes) +
                            " device bytes, more than the whole budget");
        r.t_submit = srv->now();
        const int64_t rid = r.id;
        srv->reqs.emplace(rid, std::move(r));
        srv->queue.push_back(rid);
        if (id)
            *id = rid;
    });
}

int atvb_server_set_limits(atvb_server* srv, int64_t max_resident_atoms) {
    return sguard([&] {
        if (!srv)
            throw Error(ATVB_ERR_INVALID, "server is NULL");
        if (max_resident_atoms < 0)
            throw Error(ATVB_ERR_INVALID, "max_resident_atoms must be >= 0");
        srv->max_atoms = max_resident_atoms;
    });
}

int atvb_server_cancel(atvb_server* srv, int64_t id) {
    return sguard([&] {
        if (!srv)
            throw Error(ATVB_ERR_INVALID, "server is NULL");
        Request& r = srv->get(id);
        if (r.state == 0) {
            srv->queue.erase(std::remove(srv->queue.begin(), srv->queue.end(), id),
                             srv->queue.end());
        } else if (r.state == 1) {
            srv->retire(r, false);
        } else {
            return;
        }
        r.state = 3;
        r.t_done = srv->now();
    });
}

int atvb_server_tick(atvb_server* srv, int32_t chunk) {
    return sguard([&] {
        if (!srv)
            throw Error(ATVB_ERR_INVALID, "server is NULL");
        srv->tick(chunk);
    });
}

static void fill_result(const Request& r, atvb_request_result* out) {
    out->id = r.id;
    out->state = r.state;
    out->steps_done = r.steps_done;
    out->t_submit = r.t_submit;
    out->t_start = r.t_start;
    out->t_done = r.t_done;
    out->scalars = r.sc;
}

int atvb_server_poll(atvb_server* srv, int64_t id, atvb_request_result* out) {
    return sguard([&] {
        if (!srv || !out)
            throw Error(ATVB_ERR_INVALID, "server/out is NULL");
        fill_result(srv->get(id), out);
    });
}

int atvb_server_collect(atvb_server* srv, int64_t id, atvb_soa_view* frame,
                        atvb_request_result* out) {
    return sguard([&] {
        if (!srv)
            throw Error(ATVB_ERR_INVALID, "server is NULL");
        Request& r = srv->get(id);
        if (r.state != 2 && r.state != 5)
            throw Error(ATVB_ERR_STATE, "request not finished or suspended");
        const size_t n = r.x.size();
        auto cp = [&](double* dst, const std::vector<double>& src) {
            if (dst)
                std::copy(src.begin(), src.begin() + n, dst);
        };
        if (frame) {
            cp(frame->x, r.x);
            cp(frame->y, r.y);
            cp(frame->z, r.z);
            cp(frame->vx, r.vx);
            cp(frame->vy, r.vy);
            cp(frame->vz, r.vz);
            cp(frame->fx, r.fx);
            cp(frame->fy, r.fy);
            cp(frame->fz, r.fz);
        }
        if (out)
            fill_result(r, out);
        srv->reqs.erase(id);
    });
}

int atvb_server_keep_checkpoints(atvb_server* srv, int32_t on) {
    return sguard([&] {
        if (!srv)
            throw Error(ATVB_ERR_INVALID, "server is NULL");
        srv->keep_ckpt = on != 0;
    });
}

int atvb_server_suspend(atvb_server* srv, int64_t id) {
    return sguard([&] {
        if (!srv)
            throw Error(ATVB_ERR_INVALID, "server is NULL");
        Request& r = srv->get(id);
        if (r.state != 1)
            throw Error(ATVB_ERR_STATE, "only a running request can be suspended");
        srv->retire(r, true, true);
        r.state = 5;
        r.t_done = srv->now();
    });
}

int atvb_server_resume(atvb_server* srv, int64_t id, int32_t more_steps) {
    return sguard([&] {
        if (!srv)
            throw Error(ATVB_ERR_INVALID, "server is NULL");
        if (more_steps < 0)
            throw Error(ATVB_ERR_INVALID, "more_steps must be >= 0");
        Request& r = srv->get(id);
        if (!((r.state == 5 || r.state == 2) && !r.ckpt.empty()))
            throw Error(ATVB_ERR_STATE,
                        "only a suspended request, or a finished one that kept its "
                        "checkpoint, can be resumed");
        r.n_steps = r.steps_done + more_steps;
        r.resume = true;
        r.state = 0;
        r.t_submit = srv->now();
        srv->queue.push_back(id);
    });
}

int atvb_server_checkpoint(atvb_server* srv, int64_t id, void* buf, int64_t capacity,
                           int64_t* size) {
    return sguard([&] {
        if (!srv)
            throw Error(ATVB_ERR_INVALID, "server is NULL");
        Request& r = srv->get(id);
        size_t need;
        if (r.state == 1)
            need = srv->eng->checkpoint_bytes(r.slot);
        else if (!r.ckpt.empty())
            need = r.ckpt.size();
        else
            throw Error(ATVB_ERR_STATE, "request holds no state to checkpoint");
        if (size)
            *size = (int64_t)need;
        if (!buf)
            return;
        if (capacity < (int64_t)need)
            throw Error(ATVB_ERR_INVALID, "checkpoint buffer too small");
        if (r.state == 1)
            srv->eng->save(r.slot, buf, need);
        else
            std::memcpy(buf, r.ckpt.data(), need);
    });
}

int atvb_server_submit_checkpoint(atvb_server* srv, const atvb_system_desc* desc,
                                  const void* buf, int64_t size, int32_t n_steps,
                                  int64_t* id) {
    return sguard([&] {
        if (!srv || !desc || !buf || size <= 0)
            throw Error(ATVB_ERR_INVALID, "server/desc/checkpoint is NULL");
        if (n_steps < 0)
            throw Error(ATVB_ERR_INVALID, "n_steps must be >= 0");
        atvb::make_geometry(*desc);
        Request r;
        r.id = srv->next_id++;
        r.desc = *desc;
        const int n = desc->n_atoms;
        for (auto* v : {&r.x, &r.y, &r.z, &r.vx, &r.vy, &r.vz, &r.fx, &r.fy, &r.fz, &r.m, &r.q})
            v->assign(n, 0.0);
        r.tag.assign(n, 0);
        r.ckpt.assign((const char*)buf, (const char*)buf + size);
        r.resume = true;
        r.n_steps = n_steps;
        r.bytes = atvb::estimate_bytes(*desc);
        if (r.bytes > srv->budget)
            throw Error(ATVB_ERR_NOMEM, "request needs more than the whole budget");
        r.t_submit = srv->now();
        const int64_t rid = r.id;
        srv->reqs.emplace(rid, std::move(r));
        srv->queue.push_back(rid);
        if (id)
            *id = rid;
    });
}

int atvb_server_stats(atvb_server* srv, int64_t* queued, int64_t* running,
                      int64_t* done, size_t* bytes_in_use) {
    return sguard([&] {
        if (!srv)
            throw Error(ATVB_ERR_INVALID, "server is NULL");
        int64_t d = 0;
        for (const auto& kv : srv->reqs)
            if (kv.second.state >= 2)
                ++d;
        if (queued)
            *queued = (int64_t)srv->queue.size();
        if (running)
            *running = (int64_t)srv->running.size();
        if (done)
            *done = d;
        if (bytes_in_use)
            *bytes_in_use = srv->in_use;
    });
}

} // extern "C"
