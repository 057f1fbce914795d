// integrate.cu -- velocity Verlet, Nose-Hoover, Langevin, kinetic energy and
// the per-system scalar updates, fused into two atom passes per step.
//
// Reference order (src/cpu/driver/runtime.cpp:452-501 with VelocityVerlet at
// order 0 and the thermostat at +100 in both integrate phases):
//   initial_integrate: v += dt/2 f/m * ftm2v; x += dt v; wrap   (velocity_verlet.cpp:40-55)
//                      NH: xi += dt/2 (2KE - Ndf kT)/Q; v *= exp(-dt/2 xi)  (nose_hoover.cpp:104-170)
//   neighbor decide (neighbor_list.h:128-141), force, post_force Langevin
//   (fix_langevin.cpp:79-155), final_integrate: v += dt/2 f/m; NH again;
//   end_of_step: KE (init.cpp:29-45).
// Fusion: the thermostat scale of each half is a per-system scalar produced
// by a one-thread-per-system kernel; it is applied to v by the NEXT atom
// pass (the initial-half scale by the final kick, the final-half scale by
// the next step's initial kick), so each half step reads and writes v once.
// The end-of-step kinetic energy is s_B^2 * KE(v) for the deferred scale.
#include "atvb_common.cuh"
#include "atvb_kernels.cuh"
#include "box.cuh"
#include "npt.cuh"

namespace atvb {

// splitmix64 stream + Box-Muller with a cached partner
// (fix_langevin.cpp:37-62); the key mixes seed, step and atom tag
// (fix_langevin.cpp:112-121).
struct GaussStream {
    unsigned long long s;
    bool has;
    double cached;
    ATVB_DEV double u01() {
        s += 0x9E3779B97F4A7C15ull;
        unsigned long long z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z = z ^ (z >> 31);
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    }
    ATVB_DEV double next() {
        if (has) {
            has = false;
            return cached;
        }
        const double u = u01();
        const double v = u01();
        const double r = sqrt(-2.0 * log(u > 1e-300 ? u : 1e-300));
        double sn, cs;
        sincos(2.0 * kPi * v, &sn, &cs);
        cached = r * sn;
        has = true;
        return r * cs;
    }
};

ATVB_DEV double fix_to_d(unsigned long long v) {
    return (double)(long long)v * kEFixInv;
}

// md::NVELimit (nve_limit.cu:20-30, LAMMPS fix nve/limit): after a half
// kick, a speed above vmax = xmax / dt is scaled back to vmax.
ATVB_DEV void speed_cap(double vlimit, double vlimit2, double v[3]) {
    if (!(vlimit2 > 0.0))
        return;
    const double vsq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (vsq > vlimit2) {
        const double s = vlimit / sqrt(vsq);
        v[0] *= s;
        v[1] *= s;
        v[2] *= s;
    }
}

// cuda::StopOnNaN's condition (criterion.cuh:166-178), per atom: a NaN or
// infinite position or velocity raises the sticky status bit.  Positions
// enter the force kernels as fixed point, where a NaN would become an
// ordinary coordinate, so the check sits here, on the FP64 master state of
// every drift (a non-finite force shows in the kicked velocity).
ATVB_DEV void check_finite(const SysParams& P, const double x[3], const double v[3]) {
    const double t = (x[0] + x[1]) + (x[2] + v[0]) + (v[1] + v[2]);
    if (!isfinite(t))
        atomicOr(&P.st->status, kStatusNonFinite);
}

// MTK NPT initial half for atom i (nose_hoover_npt.cpp:812-850 P2-P6): the
// pending per-axis velocity scale (end-of-step chain and barostat factors of
// the previous step, initial-half ones of this step), the force kick, the
// closed-form drift x e^{eps dt} + v dt drift into the next cell, wrap,
// sorted repack with the next cell's scales, displacement check in the
// build cell.
ATVB_DEV double npt_drift_atom(const SysParams& P, int i) {
    const SysState* st = P.st;
    const int r = P.rank[i];
    const double4 f = P.f4[r];
    const double dtfm = P.dtf / P.mass[i];
    double v[3] = {P.vx[i], P.vy[i], P.vz[i]};
    const double fa[3] = {f.x, f.y, f.z};
    double* const xs[3] = {P.x, P.y, P.z};
    double x[3];
    double d2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
        v[d] = __dadd_rn(__dmul_rn(v[d], st->vs[d]), __dmul_rn(dtfm, fa[d]));
    speed_cap(P.vlimit, P.vlimit2, v);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double Ln = st->Lnext[d];
        double xd = __dadd_rn(__dmul_rn(xs[d][i], st->npt_a[d]),
                              __dmul_rn(__dmul_rn(v[d], P.dt), st->npt_drift[d]));
        xd = __dadd_rn(xd, -__dmul_rn(Ln, floor(xd / Ln)));
        x[d] = xd;
        const double* xr = d == 0 ? P.xr : (d == 1 ? P.yr : P.zr);
        const double du = min_img(xd * st->ub[d] - xr[i], st->Lb[d], st->Lb_inv[d]);
        d2 += du * du;
    }
    P.vx[i] = v[0];
    P.vy[i] = v[1];
    P.vz[i] = v[2];
    P.x[i] = x[0];
    P.y[i] = x[1];
    P.z[i] = x[2];
    check_finite(P, x, v);
    const double q = P.q[i];
    if (P.prec == kMixed) {
        int4 p;
        p.x = (int)pos_fix(x[0], st->fixn_scale[0]);
        p.y = (int)pos_fix(x[1], st->fixn_scale[1]);
        p.z = (int)pos_fix(x[2], st->fixn_scale[2]);
        p.w = __float_as_int((float)q);
        reinterpret_cast<int4*>(P.pos4)[r] = p;
    } else {
        reinterpret_cast<double4*>(P.pos4)[r] = pack_pos64(x, st->fixn64_scale, q);
    }
    if (d2 > st->disp_thr2)
        P.st->need_rebuild = 1;
    return P.mass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

// Initial half: deferred scale, kick, drift, wrap, sorted repack,
// displacement check, KE of the kicked velocities (for Nose-Hoover).
__global__ void __launch_bounds__(kChunk, 3)
    k_integrate_a(const Item* items, int nitems, const SysParams* sp) {
    __shared__ double sh[32];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (P.st->halted)
            continue; // block-uniform: the item belongs to one system
        const int i = item.begin + threadIdx.x;
        double ke = 0.0;
        if (i < P.n && (P.thermostat == kNPT || P.generic_drift)) {
            ke = npt_drift_atom(P, i);
        } else if (i < P.n) {
            // every load first (atom data, then the system fields read after
            // the stores): a load placed after a store to global memory
            // cannot be hoisted above it, and would add a round trip
            const double sc = P.st->vscale;
            const int r = P.rank[i];
            const double4 f = P.f4[r];
            const double m = P.mass[i];
            const double q = P.q[i];
            const double x0[3] = {P.x[i], P.y[i], P.z[i]};
            const double xr[3] = {P.xr[i], P.yr[i], P.zr[i]};
            double v[3] = {P.vx[i], P.vy[i], P.vz[i]};
            const double L[3] = {P.L[0], P.L[1], P.L[2]};
            const double invL[3] = {P.invL[0], P.invL[1], P.invL[2]};
            const double dt = P.dt, skin_half2 = P.skin_half2;
            const bool mixed = P.prec == kMixed;
            const double fs[3] = {mixed ? P.fix_scale[0] : P.fix64_scale[0],
                                  mixed ? P.fix_scale[1] : P.fix64_scale[1],
                                  mixed ? P.fix_scale[2] : P.fix64_scale[2]};
            void* const pos4 = P.pos4;
            const double dtfm = P.dtf / m;
            const double fa[3] = {f.x, f.y, f.z};
            double x[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                v[d] = __dadd_rn(__dmul_rn(v[d], sc), __dmul_rn(dtfm, fa[d]));
                double xd = __dadd_rn(x0[d], __dmul_rn(dt, v[d]));
                xd = __dadd_rn(xd, -__dmul_rn(L[d], floor(xd / L[d])));
                x[d] = xd;
            }
            P.vx[i] = v[0];
            P.vy[i] = v[1];
            P.vz[i] = v[2];
            P.x[i] = x[0];
            P.y[i] = x[1];
            P.z[i] = x[2];
            check_finite(P, x, v);
            if (mixed) {
                int4 p;
                p.x = (int)pos_fix(x[0], fs[0]);
                p.y = (int)pos_fix(x[1], fs[1]);
                p.z = (int)pos_fix(x[2], fs[2]);
                p.w = __float_as_int((float)q);
                reinterpret_cast<int4*>(pos4)[r] = p;
            } else {
                reinterpret_cast<double4*>(pos4)[r] = pack_pos64(x, fs, q);
            }
            // cell_list.cpp:355-392 with min-image displacement
            const double ddx = min_img(x[0] - xr[0], L[0], invL[0]);
            const double ddy = min_img(x[1] - xr[1], L[1], invL[1]);
            const double ddz = min_img(x[2] - xr[2], L[2], invL[2]);
            if (ddx * ddx + ddy * ddy + ddz * ddz > skin_half2)
                P.st->need_rebuild = 1;
            ke = m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        }
        if (P.thermostat == kNoseHoover) {
            const double t = block_sum(ke, sh);
            if (threadIdx.x == 0)
                fix_add(&P.st->acc[kAccKEA], 0.5 * kMvv2e * t);
        }
    }
}

// One thread per system: thermostat scalar of the initial half, neighbour
// decision (every / delay / check), step accumulators reset.  Inside the
// step graph (use_cond), a system that builds its list sets the graph's
// two conditional handles (one per conditional node: the cell sort and the
// rows), which launch the list-build kernels of this step.
__global__ void k_sys_a(const int* sys_list, int nsys, const SysParams* sp,
                        cudaGraphConditionalHandle cond_sort,
                        cudaGraphConditionalHandle cond_rows, int use_cond) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsys)
        return;
    const SysParams& P = sp[sys_list[k]];
    SysState* gst = P.st;
    if (gst->halted) {
        gst->rebuild = 0; // nothing of this system moves: no list build either
        return;
    }
    // the state in local memory, written back once: each read below is then
    // an L1 hit instead of a global round trip ordered behind the previous
    // store (this thread is the state's only reader and writer meanwhile)
    SysState loc = *gst;
    SysState* st = &loc;
    if (P.thermostat == kNPT || P.deform_axis >= 0) {
        // commit the cell of this step's drift: every later kernel of the
        // step (neighbour build, forces, PME) reads it from SysParams
        apply_box(const_cast<SysParams&>(sp[sys_list[k]]), st->Lnext, true);
        for (int d = 0; d < 3; ++d)
            st->box[d] = st->Lnext[d];
    }
    st->vscale = 1.0;
    st->nearq_n = 0; // the previous step's near-cutoff queue has been settled
    if (P.thermostat == kNoseHoover) {
        const double ke = fix_to_d(st->acc[kAccKEA]);
        st->acc[kAccKEA] = 0ull;
        st->xi += (P.dt * 0.5) * (2.0 * ke - P.n_dof_kT) / P.Q;
        st->s_a = exp(-P.dt * 0.5 * st->xi);
    } else {
        st->s_a = 1.0;
    }
    st->ago += 1;
    const bool disp = st->need_rebuild != 0;
    st->need_rebuild = 0;
    // a build the host asked for (rows widened after one was cut) comes
    // first, whatever every/delay/check would say
    const bool forced = st->force_build != 0;
    st->force_build = 0;
    const bool rebuild = forced || (st->ago >= P.nl_delay && (st->ago % P.nl_every) == 0 &&
                                    (!P.nl_check || disp));
    st->rebuild = rebuild ? 1 : 0;
    if (rebuild && use_cond) {
        cudaGraphSetConditional(cond_sort, 1u);
        cudaGraphSetConditional(cond_rows, 1u);
    }
    if (rebuild) {
        st->overflow = 0; // set again by the build if a row is cut
        for (int d = 0; d < 3; ++d) {
            st->Lb[d] = P.L[d];
            st->Lb_inv[d] = 1.0 / P.L[d];
        }
        st->ago = 0;
        st->rebuilds += 1;
        st->max_nnbr = 0;
        st->list_entries = 0ull;
    }
    *gst = loc;
}

// sqrt(2 kB T / (damp dt mvv2e)) / ftm2v at the setpoint of `step`: the
// linear ramp of fix_langevin.cpp:94-104 (delta clamped to [0, 1]), each
// operation rounded separately, as the host and the reference compute it.
ATVB_DEV double lang_g2pre(const SysParams& P, long long step) {
    if (P.lang_nlast <= P.lang_nfirst)
        return P.lang_g2pre;
    double delta = __ddiv_rn((double)(step - P.lang_nfirst),
                             (double)(P.lang_nlast - P.lang_nfirst));
    delta = delta < 0.0 ? 0.0 : (delta > 1.0 ? 1.0 : delta);
    const double T = __dadd_rn(P.lang_T0, __dmul_rn(delta, __dsub_rn(P.lang_T1, P.lang_T0)));
    return __ddiv_rn(__dsqrt_rn(__ddiv_rn(__dmul_rn(2.0 * kKB, T), P.lang_ddm)), kFtm2v);
}

// Final half: initial-half thermostat scale, Langevin force, kick, KE.
__global__ void __launch_bounds__(kChunk)
    k_integrate_b(const Item* items, int nitems, const SysParams* sp) {
    __shared__ double sh[32];
    __shared__ double sh3[32 * 3];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (P.st->halted)
            continue;
        const int i = item.begin + threadIdx.x;
        double ke = 0.0;
        double kax[3] = {0.0, 0.0, 0.0};
        // system fields read after the force store below, read before it
        // (a load after a global store cannot be hoisted above it)
        const double dtf = P.dtf, vlimit = P.vlimit, vlimit2 = P.vlimit2;
        const int thermostat = P.thermostat;
        if (i < P.n) {
            const double sc = P.st->s_a;
            const int r = P.rank[i];
            double4 f = P.f4[r];
            const double m = P.mass[i];
            double v[3] = {__dmul_rn(P.vx[i], sc), __dmul_rn(P.vy[i], sc),
                           __dmul_rn(P.vz[i], sc)};
            if (P.has_pme) {
                // pair + reciprocal forces; the sum is the step's force
                const double4 g = P.fp4[r];
                f.x = __dadd_rn(f.x, g.x);
                f.y = __dadd_rn(f.y, g.y);
                f.z = __dadd_rn(f.z, g.z);
            }
            if (P.ext_f) {
                // the user components' forces (atvb_system_add_component)
                f.x = __dadd_rn(f.x, P.ext_f[i]);
                f.y = __dadd_rn(f.y, P.ext_f[P.n + i]);
                f.z = __dadd_rn(f.z, P.ext_f[2 * P.n + i]);
            }
            if ((P.has_pme || P.ext_f) && thermostat != kLangevin)
                P.f4[r] = f;
            if (thermostat == kLangevin) {
                const unsigned long long base =
                    (unsigned long long)P.seed * 0x9E3779B97F4A7C15ull +
                    (unsigned long long)P.st->step * 0xBF58476D1CE4E5B9ull;
                GaussStream g{base + (unsigned long long)P.tag[i] *
                                         0xD6E8FEB86659FD93ull,
                              false, 0.0};
                const double g1 = -m * P.lang_g1;
                const double g2 = lang_g2pre(P, P.st->step) * sqrt(m);
                const double rx = g.next(), ry = g.next(), rz = g.next();
                f.x += g1 * v[0] + g2 * rx;
                f.y += g1 * v[1] + g2 * ry;
                f.z += g1 * v[2] + g2 * rz;
                P.f4[r] = f;
            }
            const double dtfm = dtf / m;
            v[0] = __dadd_rn(v[0], __dmul_rn(dtfm, f.x));
            v[1] = __dadd_rn(v[1], __dmul_rn(dtfm, f.y));
            v[2] = __dadd_rn(v[2], __dmul_rn(dtfm, f.z));
            speed_cap(vlimit, vlimit2, v);
            P.vx[i] = v[0];
            P.vy[i] = v[1];
            P.vz[i] = v[2];
            ke = m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            kax[0] = m * v[0] * v[0];
            kax[1] = m * v[1] * v[1];
            kax[2] = m * v[2] * v[2];
        }
        if (thermostat == kNPT) {
            block_sum_vec<3>(kax, sh3);
            if (threadIdx.x == 0)
                for (int d = 0; d < 3; ++d)
                    fix_add(&P.st->acc[kAccKEX + d], 0.5 * kMvv2e * kax[d]);
        } else {
            const double t = block_sum(ke, sh);
            if (threadIdx.x == 0)
                fix_add(&P.st->acc[kAccKEB], 0.5 * kMvv2e * t);
        }
    }
}

ATVB_DEV void finish_energy(const SysParams& P, SysState* st) {
    st->e_lj = fix_to_d(st->acc[kAccELJ]);
    st->e_coul = fix_to_d(st->acc[kAccECoul]);
    st->e_recip = fix_to_d(st->acc[kAccERecip]);
    st->e_const = P.has_pme ? P.e_const : 0.0;
    st->energy = st->e_lj + st->e_coul + st->e_recip + st->e_const;
    for (int k = 0; k < 6; ++k)
        st->virial[k] = fix_to_d(st->acc[kAccVir + k]);
    if (P.ext_ev) { // the user components' energy and virial
        st->energy += P.ext_ev[0];
        for (int k = 0; k < 6; ++k)
            st->virial[k] += P.ext_ev[1 + k];
    }
    st->acc[kAccELJ] = st->acc[kAccECoul] = st->acc[kAccERecip] = 0ull;
    for (int k = 0; k < 6; ++k)
        st->acc[kAccVir + k] = 0ull;
}

// Cell edges and the scalar pressure (2 KE + W_xx + W_yy + W_zz) / (3 V)
ATVB_DEV void cell_scalars(const SysParams& P, SysState* st) {
    for (int d = 0; d < 3; ++d)
        st->box[d] = P.L[d];
    const double V = P.L[0] * P.L[1] * P.L[2];
    st->pressure =
        (2.0 * st->kinetic + st->virial[0] + st->virial[1] + st->virial[2]) / (3.0 * V);
}

// End of a step: StopOnNaN halts a system whose state went non-finite, and
// any sticky bit is published to the host-mapped status word.
ATVB_DEV void end_status(const SysParams& P, SysState* st) {
    if (P.stop_on_nan && (st->status & kStatusNonFinite))
        st->halted = 1;
    if (P.status_hint && st->status)
        *(volatile int*)P.status_hint = st->status | (st->halted ? (1 << 30) : 0);
}

ATVB_DEV void record_history(const SysParams& P, SysState* st) {
    if (P.ehist_cap > 0) {
        const long long slot = st->step % P.ehist_cap;
        P.ehist[3 * slot + 0] = st->energy;
        P.ehist[3 * slot + 1] = st->kinetic;
        P.ehist[3 * slot + 2] = (double)st->step;
    }
    if (P.row_hint && st->rebuild) // the longest row changes only at a build
        *(volatile int*)P.row_hint = st->max_nnbr;
    end_status(P, st);
}

// Berendsen barostat at end_of_step (barostat.cpp:27-110): from the scalar
// pressure of this step (st->pressure, virial + kinetic), the dilation
// mu = cbrt(clamp(1 - dt/(tau_P beta) (P_target - P), 0.5, 2)); the cell is
// committed here, k_baro_scale scales the positions, and the next initial
// half drifts in the new cell with the build-cell displacement rule.
ATVB_DEV void berendsen(const SysParams& P, SysState* st) {
    double mu3 = 1.0 - P.baro_coef * (P.baro_P - st->pressure);
    mu3 = mu3 < 0.5 ? 0.5 : (mu3 > 2.0 ? 2.0 : mu3);
    double mu = cbrt(mu3);
    double Ln[3];
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
        Ln[d] = P.L[d] * mu;
        if (!(Ln[d] >= P.npt_Lmin[d]))
            ok = false;
    }
    if (!ok) {
        st->status |= kStatusBoxRange;
        st->held = 1;
        mu = 1.0;
        for (int d = 0; d < 3; ++d)
            Ln[d] = P.L[d];
    }
    st->mu = mu;
    SysParams& W = const_cast<SysParams&>(P);
    apply_box(W, Ln, true);
    double lam = 1e300;
    for (int d = 0; d < 3; ++d) {
        st->box[d] = Ln[d];
        st->vs[d] = st->vscale;
        st->vs_out[d] = st->vscale;
        st->npt_a[d] = 1.0;
        st->npt_drift[d] = 1.0;
        st->Lnext[d] = Ln[d];
        st->fixn_scale[d] = W.fix_scale[d];
        st->fixn64_scale[d] = W.fix64_scale[d];
        st->ub[d] = st->Lb[d] / Ln[d];
        lam = fmin(lam, Ln[d] / st->Lb[d]);
    }
    const double thr = 0.5 * (P.rlist - P.npt_cut / lam);
    st->disp_thr2 = thr > 0.0 ? thr * thr : -1.0;
    if (thr <= 0.0)
        st->need_rebuild = 1;
}

// md::Deform (deform.cu:55-95, initial_integrate +200: after the drift):
// the k-th deformation step takes the axis edge from L0 (1 + r dt (k-1)) to
// L0 (1 + r dt k) (engineering strain, linear in time) and scales positions
// along it by the same ratio.  Folded into the next initial half's drift
// (x s + v dt s along the axis, in the new cell); k_sys_a commits the cell.
ATVB_DEV void deform_prepare(const SysParams& P, SysState* st, long long k) {
    const int ax = P.deform_axis;
    const double rdt = P.deform_rate * P.dt;
    const double Lp = P.deform_L0 * (1.0 + rdt * (double)(k - 1));
    const double Lc = P.deform_L0 * (1.0 + rdt * (double)k);
    const double sc = Lc / Lp;
    double lam = 1e300;
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
        const double f = d == ax ? sc : 1.0;
        st->vs[d] = st->vscale;
        st->vs_out[d] = st->vscale;
        st->npt_a[d] = f;
        st->npt_drift[d] = f;
        st->Lnext[d] = P.L[d] * f;
        if (!(st->Lnext[d] >= P.npt_Lmin[d]))
            ok = false;
    }
    if (!ok) {
        st->status |= kStatusBoxRange;
        st->held = 1;
    }
    for (int d = 0; d < 3; ++d) {
        st->fixn_scale[d] = 4294967296.0 / st->Lnext[d];
        st->fixn64_scale[d] = 18446744073709551616.0 / st->Lnext[d];
        st->ub[d] = st->Lb[d] / st->Lnext[d];
        lam = fmin(lam, st->Lnext[d] / st->Lb[d]);
    }
    const double thr = 0.5 * (P.rlist - P.npt_cut / lam);
    st->disp_thr2 = thr > 0.0 ? thr * thr : -1.0;
    if (thr <= 0.0)
        st->need_rebuild = 1;
}

// Positions scaled by this step's Berendsen dilation (original order).
__global__ void k_baro_scale(const Item* items, int nitems, const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        const int i = item.begin + threadIdx.x;
        if (!P.baro || i >= P.n)
            continue;
        const double mu = P.st->mu;
        P.x[i] *= mu;
        P.y[i] *= mu;
        P.z[i] *= mu;
    }
}

// MTK NPT end of step (nose_hoover_npt.cpp:855-885, P8-P11) from the
// per-axis kinetic energies of the kicked velocities, then the scalars of
// the next step's initial half (npt_prepare).
ATVB_DEV void npt_end_of_step(const SysParams& P, SysState* st) {
    const double hdt = 0.5 * P.dt;
    double ke[3];
    for (int d = 0; d < 3; ++d) {
        ke[d] = fix_to_d(st->acc[kAccKEX + d]);
        st->acc[kAccKEX + d] = 0ull;
    }
    finish_energy(P, st); // energies and the virial of this step's forces
    st->ke_global = ke[0] + ke[1] + ke[2];
    double s8[3];
    npt_scale_baro(P, st, hdt, ke, s8);                 // P8
    npt_update_eps(P, st, hdt, ke);                     // P9
    const double s10 = npt_nhc_atoms(P, st, hdt, ke);   // P10
    npt_nhc_baro(P, st, hdt);                           // P11
    st->kinetic = st->ke_global;
    st->conserved = npt_hamiltonian(P, st);
    st->vscale = 1.0;
    cell_scalars(P, st);
    record_history(P, st);
    st->step += 1;
    const double vs_out[3] = {s8[0] * s10, s8[1] * s10, s8[2] * s10};
    npt_prepare(P, st, ke, vs_out);
}

// One thread per system: final-half thermostat, end-of-step scalars,
// energy history, step counter.
__global__ void k_sys_b(const int* sys_list, int nsys, const SysParams* sp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsys)
        return;
    const SysParams& P = sp[sys_list[k]];
    SysState* gst = P.st;
    if (gst->halted)
        return;
    // the state in local memory, written back once (as in k_sys_a)
    SysState loc = *gst;
    SysState* st = &loc;
    if (P.thermostat == kNPT) {
        npt_end_of_step(P, st);
        *gst = loc;
        return;
    }
    const double ke = fix_to_d(st->acc[kAccKEB]);
    st->acc[kAccKEB] = 0ull;
    if (P.thermostat == kNoseHoover) {
        st->xi += (P.dt * 0.5) * (2.0 * ke - P.n_dof_kT) / P.Q;
        const double s = exp(-P.dt * 0.5 * st->xi);
        st->vscale = s;
        st->kinetic = s * s * ke;
    } else {
        st->vscale = 1.0;
        st->kinetic = ke;
    }
    finish_energy(P, st);
    st->conserved = st->energy + st->kinetic;
    cell_scalars(P, st);
    if (P.baro)
        berendsen(P, st);
    else if (P.deform_axis >= 0)
        deform_prepare(P, st, st->step + 2); // st->step counts this step only below
    else if (P.generic_drift)
        for (int d = 0; d < 3; ++d)
            st->vs[d] = st->vscale; // fixed cell: the identity drift factors stay
    if (P.ehist_cap > 0) {
        const long long slot = st->step % P.ehist_cap;
        P.ehist[3 * slot + 0] = st->energy;
        P.ehist[3 * slot + 1] = st->kinetic;
        P.ehist[3 * slot + 2] = (double)st->step;
    }
    if (P.row_hint && st->rebuild) // the longest row changes only at a build
        *(volatile int*)P.row_hint = st->max_nnbr;
    end_status(P, st);
    st->step += 1;
    *gst = loc;
}

// Energies of a force-only evaluation (no step, no thermostat update).
__global__ void k_sys_energy(const int* sys_list, int nsys,
                             const SysParams* sp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsys)
        return;
    const SysParams& P = sp[sys_list[k]];
    finish_energy(P, P.st);
    P.st->conserved = P.st->energy + P.st->kinetic;
    cell_scalars(P, P.st);
}

__global__ void k_force_rebuild(const int* sys_list, int nsys,
                                const SysParams* sp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsys)
        return;
    SysState* st = sp[sys_list[k]].st;
    st->rebuild = 1;
    st->ago = 0;
    st->max_nnbr = 0;
    st->list_entries = 0ull;
    // a force pass outside the step loop starts its energy and virial sums
    // from zero, whatever ran before it (e.g. autotuning launches)
    st->acc[kAccELJ] = st->acc[kAccECoul] = st->acc[kAccERecip] = 0ull;
    for (int v = 0; v < 6; ++v)
        st->acc[kAccVir + v] = 0ull;
    st->nearq_n = 0; // nothing queued by launches outside a force pass counts
    st->nearq_lost = 0;
}

// After an upload: wrap positions into [0, L) (pbc.h:48-50) and keep the
// uploaded forces (staged in sx/sy/sz) in sorted order.  Runs after a
// forced rebuild, so rank is valid.
__global__ void k_state_in(const Item* items, int nitems, const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        const int i = item.begin + threadIdx.x;
        if (i >= P.n)
            continue;
        P.f4[P.rank[i]] = make_double4(P.sx[i], P.sy[i], P.sz[i], 0.0);
    }
}

__global__ void k_wrap_in(const Item* items, int nitems, const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        const int i = item.begin + threadIdx.x;
        if (i >= P.n)
            continue;
        P.x[i] = wrap(P.x[i], P.L[0]);
        P.y[i] = wrap(P.y[i], P.L[1]);
        P.z[i] = wrap(P.z[i], P.L[2]);
    }
}

// what = 0: forces (original order) into sx/sy/sz;
// what = 1: velocities with the pending scale applied into sx/sy/sz.
__global__ void k_state_out(const Item* items, int nitems, const SysParams* sp,
                            int what) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        const int i = item.begin + threadIdx.x;
        if (i >= P.n)
            continue;
        if (what == 0) {
            const double4 f = P.f4[P.rank[i]];
            P.sx[i] = f.x;
            P.sy[i] = f.y;
            P.sz[i] = f.z;
        } else if (P.thermostat == kNPT) {
            const double* s = P.st->vs_out;
            P.sx[i] = P.vx[i] * s[0];
            P.sy[i] = P.vy[i] * s[1];
            P.sz[i] = P.vz[i] * s[2];
        } else {
            const double s = P.st->vscale;
            P.sx[i] = P.vx[i] * s;
            P.sy[i] = P.vy[i] * s;
            P.sz[i] = P.vz[i] * s;
        }
    }
}

__global__ void k_kinetic(const Item* items, int nitems, const SysParams* sp) {
    __shared__ double sh[32];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        const int i = item.begin + threadIdx.x;
        double ke = 0.0;
        if (i < P.n)
            ke = P.mass[i] *
                 (P.vx[i] * P.vx[i] + P.vy[i] * P.vy[i] + P.vz[i] * P.vz[i]);
        const double t = block_sum(ke, sh);
        if (threadIdx.x == 0)
            fix_add(&P.st->acc[kAccKEB], 0.5 * kMvv2e * t);
    }
}

__global__ void k_kinetic_finish(const int* sys_list, int nsys,
                                 const SysParams* sp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsys)
        return;
    SysState* st = sp[sys_list[k]].st;
    st->kinetic = fix_to_d(st->acc[kAccKEB]);
    st->acc[kAccKEB] = 0ull;
}

// Per-axis kinetic energy of MTK NPT systems that have not stepped yet (the
// input of their first initial half).
__global__ void k_npt_kinetic(const Item* items, int nitems, const SysParams* sp) {
    __shared__ double sh[32 * 3];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (P.thermostat != kNPT || P.st->step != 0)
            continue;
        const int i = item.begin + threadIdx.x;
        double k[3] = {0.0, 0.0, 0.0};
        if (i < P.n) {
            const double m = P.mass[i];
            k[0] = m * P.vx[i] * P.vx[i];
            k[1] = m * P.vy[i] * P.vy[i];
            k[2] = m * P.vz[i] * P.vz[i];
        }
        block_sum_vec<3>(k, sh);
        if (threadIdx.x == 0)
            for (int d = 0; d < 3; ++d)
                fix_add(&P.st->acc[kAccKEX + d], 0.5 * kMvv2e * k[d]);
    }
}

// Before the first step of an MTK NPT system: the extended state of the
// reference's build() (chains and strain rates at rest, KE_global at
// equipartition, nose_hoover_npt.cpp:87-172), then the scalars of step 0's
// initial half from the virial of the last force evaluation (zero before
// any).  Idempotent while no step has run.
__global__ void k_npt_prep(const int* sys_list, int nsys, const SysParams* sp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsys)
        return;
    const SysParams& P = sp[sys_list[k]];
    SysState* st = P.st;
    if (P.deform_axis >= 0 && st->step == 0) {
        deform_prepare(P, st, 1);
        return;
    }
    if (P.thermostat != kNPT || st->step != 0)
        return;
    double ke[3];
    for (int d = 0; d < 3; ++d) {
        ke[d] = fix_to_d(st->acc[kAccKEX + d]);
        st->acc[kAccKEX + d] = 0ull;
    }
    for (int c = 0; c < kMaxChain; ++c)
        st->eta_t[c] = st->eta_t_dot[c] = st->eta_b[c] = st->eta_b_dot[c] = 0.0;
    for (int d = 0; d < 3; ++d)
        st->eps_dot[d] = 0.0;
    st->ke_global = 0.5 * (double)P.n_dof * kKB * P.npt_T0;
    const double one[3] = {1.0, 1.0, 1.0};
    npt_prepare(P, st, ke, one);
}

// Sorted position records from the master positions with the committed
// cell's scales (a restored checkpoint: the list was rebuilt from the
// positions of the last build, the atoms have moved on since).
__global__ void k_repack(const Item* items, int nitems, const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        const int i = item.begin + threadIdx.x;
        if (i >= P.n)
            continue;
        const int r = P.rank[i];
        const double x[3] = {P.x[i], P.y[i], P.z[i]};
        const double q = P.q[i];
        if (P.prec == kMixed) {
            int4 p;
            p.x = (int)pos_fix(x[0], P.fix_scale[0]);
            p.y = (int)pos_fix(x[1], P.fix_scale[1]);
            p.z = (int)pos_fix(x[2], P.fix_scale[2]);
            p.w = __float_as_int((float)q);
            reinterpret_cast<int4*>(P.pos4)[r] = p;
        } else {
            reinterpret_cast<double4*>(P.pos4)[r] = pack_pos64(x, P.fix64_scale, q);
        }
    }
}

// Trajectory snapshots (the device-ordered freeze of
// cuda/asynchronous/async_bridge.cuh, written straight into host-mapped
// memory): after a step whose count is a multiple of snap_every, open a
// ring slot, copy positions and velocities (with the pending scale, as a
// download sees them), close the slot.  Kernel boundaries order the three
// phases; the fences make each phase visible to the host before the next.
__global__ void k_snap_open(const int* sys_list, int nsys, const SysParams* sp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsys)
        return;
    const SysParams& P = sp[sys_list[k]];
    SysState* st = P.st;
    st->snap_slot = -1;
    if (!P.snap_ring || st->step % P.snap_every != 0)
        return;
    const int slot = (int)(st->snap_count % P.snap_depth);
    SnapHeader* h = reinterpret_cast<SnapHeader*>(P.snap_ring + (size_t)slot * P.snap_slot_bytes);
    *(volatile long long*)&h->begin = st->snap_count + 1;
    __threadfence_system();
    st->snap_slot = slot;
}

__global__ void k_snap_data(const Item* items, int nitems, const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.snap_ring)
            continue;
        const SysState* st = P.st;
        const int slot = st->snap_slot;
        const int i = item.begin + threadIdx.x;
        if (slot < 0 || i >= P.n)
            continue;
        double* d = reinterpret_cast<double*>(P.snap_ring + (size_t)slot * P.snap_slot_bytes +
                                              sizeof(SnapHeader));
        const size_t n = (size_t)P.n;
        double s[3];
        for (int a = 0; a < 3; ++a)
            s[a] = P.thermostat == kNPT ? st->vs_out[a] : st->vscale;
        d[i] = P.x[i];
        d[n + i] = P.y[i];
        d[2 * n + i] = P.z[i];
        d[3 * n + i] = P.vx[i] * s[0];
        d[4 * n + i] = P.vy[i] * s[1];
        d[5 * n + i] = P.vz[i] * s[2];
        __threadfence_system(); // payload visible to the host before the close
    }
}

__global__ void k_snap_close(const int* sys_list, int nsys, const SysParams* sp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsys)
        return;
    const SysParams& P = sp[sys_list[k]];
    SysState* st = P.st;
    if (!P.snap_ring || st->snap_slot < 0)
        return;
    SnapHeader* h =
        reinterpret_cast<SnapHeader*>(P.snap_ring + (size_t)st->snap_slot * P.snap_slot_bytes);
    h->step = st->step;
    for (int a = 0; a < 3; ++a)
        h->box[a] = P.L[a];
    __threadfence_system();
    *(volatile long long*)&h->end = st->snap_count + 1;
    __threadfence_system();
    st->snap_count += 1;
    st->snap_slot = -1;
}

// After a force pass outside the step: pair + reciprocal forces into f4.
__global__ void k_force_combine(const Item* items, int nitems, const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        const int i = item.begin + threadIdx.x;
        if (!(P.has_pme || P.ext_f) || i >= P.n)
            continue;
        const int r = P.rank[i];
        double4 f = P.f4[r];
        if (P.has_pme) {
            const double4 g = P.fp4[r];
            f.x = __dadd_rn(f.x, g.x);
            f.y = __dadd_rn(f.y, g.y);
            f.z = __dadd_rn(f.z, g.z);
        }
        if (P.ext_f) {
            f.x = __dadd_rn(f.x, P.ext_f[i]);
            f.y = __dadd_rn(f.y, P.ext_f[P.n + i]);
            f.z = __dadd_rn(f.z, P.ext_f[2 * P.n + i]);
        }
        P.f4[r] = f;
    }
}

static int sys_blocks(int nsys) { return (nsys + 127) / 128; }

void launch_force_combine(const LaunchCfg& lc, cudaStream_t s) {
    k_force_combine<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp);
}

void launch_snapshots(const LaunchCfg& lc, cudaStream_t s) {
    k_snap_open<<<sys_blocks(lc.nsys), 128, 0, s>>>(lc.sys_list, lc.nsys, lc.sp);
    k_snap_data<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp);
    k_snap_close<<<sys_blocks(lc.nsys), 128, 0, s>>>(lc.sys_list, lc.nsys, lc.sp);
}

void launch_repack(const LaunchCfg& lc, cudaStream_t s) {
    k_repack<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp);
}

void launch_npt_prep(const LaunchCfg& lc, cudaStream_t s) {
    k_npt_kinetic<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp);
    k_npt_prep<<<sys_blocks(lc.nsys), 128, 0, s>>>(lc.sys_list, lc.nsys, lc.sp);
}

void launch_integrate_a(const LaunchCfg& lc, cudaStream_t s) {
    k_integrate_a<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n,
                                                    lc.sp);
}
void launch_sys_a(const LaunchCfg& lc, cudaStream_t s, cudaGraphConditionalHandle cond_sort,
                  cudaGraphConditionalHandle cond_rows, bool use_cond) {
    k_sys_a<<<sys_blocks(lc.nsys), 128, 0, s>>>(lc.sys_list, lc.nsys, lc.sp, cond_sort,
                                                 cond_rows, use_cond ? 1 : 0);
}
void launch_integrate_b(const LaunchCfg& lc, cudaStream_t s) {
    k_integrate_b<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n,
                                                    lc.sp);
}
void launch_sys_b(const LaunchCfg& lc, cudaStream_t s) {
    k_sys_b<<<sys_blocks(lc.nsys), 128, 0, s>>>(lc.sys_list, lc.nsys, lc.sp);
    if (lc.any_baro)
        k_baro_scale<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp);
}
void launch_sys_energy(const LaunchCfg& lc, cudaStream_t s) {
    k_sys_energy<<<sys_blocks(lc.nsys), 128, 0, s>>>(lc.sys_list, lc.nsys,
                                                     lc.sp);
}
void launch_force_rebuild(const LaunchCfg& lc, cudaStream_t s) {
    k_force_rebuild<<<sys_blocks(lc.nsys), 128, 0, s>>>(lc.sys_list, lc.nsys,
                                                        lc.sp);
}
void launch_state_in(const LaunchCfg& lc, cudaStream_t s) {
    k_state_in<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp);
}
void launch_wrap_in(const LaunchCfg& lc, cudaStream_t s) {
    k_wrap_in<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp);
}
void launch_state_out(const LaunchCfg& lc, int what, cudaStream_t s) {
    k_state_out<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp,
                                                 what);
}
void launch_kinetic(const LaunchCfg& lc, cudaStream_t s) {
    k_kinetic<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp);
    k_kinetic_finish<<<sys_blocks(lc.nsys), 128, 0, s>>>(lc.sys_list, lc.nsys,
                                                         lc.sp);
}

} // namespace atvb
