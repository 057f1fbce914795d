// npt.cuh -- the scalar half of the MTK NPT integrator
// (src/cpu/dynamics/nose_hoover_npt.cpp), run by one thread per system.
//
// The atom side of every Trotter factor is a per-axis velocity scale or the
// closed-form drift; those are applied by the atom passes of the step
// (k_integrate_a / k_integrate_b).  Everything else -- both Nose-Hoover
// chains, the strain rates eps_dot, the cell -- lives in SysState and is
// advanced here.  The per-axis kinetic energies that the reference
// recomputes from the velocities after each scaling are carried analytically
// (a scale s on axis a multiplies KE_a by s^2), so one reduction per step
// suffices.
#pragma once

#include "atvb_common.cuh"

namespace atvb {

// |eps_dot dt| clamp of the cell update (nose_hoover_npt.cpp:44)
constexpr double kEpsDtMax = 0.005;

// (e^{2x} - 1) / (2x) with the Taylor branch near 0 (nose_hoover_npt.cpp:66-73)
ATVB_DEV double npt_expm1c(double x) {
    if (fabs(x) < 1e-6)
        return 1.0 + x + (2.0 / 3.0) * x * x;
    return expm1(2.0 * x) / (2.0 * x);
}

// compute_temp_target + the atom-chain masses recomputed from it
// (nose_hoover_npt.cpp:192-203, 830-840)
ATVB_DEV void npt_temp_target(const SysParams& P, SysState* st, long long step) {
    double delta = 0.0;
    if (P.npt_nlast > P.npt_nfirst) {
        delta = (double)(step - P.npt_nfirst) / (double)(P.npt_nlast - P.npt_nfirst);
        delta = delta < 0.0 ? 0.0 : (delta > 1.0 ? 1.0 : delta);
    }
    st->T_live = P.npt_T0 + delta * (P.npt_T1 - P.npt_T0);
    st->kT = kKB * st->T_live;
    const double t2 = P.npt_tauT * P.npt_tauT;
    st->Qt0 = (double)P.n_dof * st->kT * t2;
    st->Qt1 = st->kT * t2;
}

// nhc_atoms_half (nose_hoover_npt.cpp:267-340); returns the velocity scale,
// KE_global and ke[] scaled by its square
ATVB_DEV double npt_nhc_atoms(const SysParams& P, SysState* st, double hdt, double ke[3]) {
    const double qdt = 0.5 * hdt, edt = 0.5 * qdt;
    const int M = P.npt_mt;
    double sc = 1.0;
    for (int pass = 0; pass < 2; ++pass) {
        for (int j = 0; j < M; ++j) {
            const int k = pass == 0 ? M - 1 - j : j;
            const double expfac = k < M - 1 ? exp(-st->eta_t_dot[k + 1] * edt) : 1.0;
            const double G =
                k == 0 ? (2.0 * st->ke_global - P.n_dof * st->kT) / st->Qt0
                       : ((k == 1 ? st->Qt0 : st->Qt1) * st->eta_t_dot[k - 1] * st->eta_t_dot[k - 1] -
                          st->kT) / st->Qt1;
            st->eta_t_dot[k] *= expfac;
            st->eta_t_dot[k] += G * qdt;
            if (pass == 0)
                st->eta_t_dot[k] *= P.npt_tdrag;
            st->eta_t_dot[k] *= expfac;
        }
        if (pass == 0) {
            sc = exp(-st->eta_t_dot[0] * hdt);
            st->ke_global *= sc * sc;
            for (int a = 0; a < 3; ++a)
                ke[a] *= sc * sc;
            for (int k = 0; k < M; ++k)
                st->eta_t[k] += st->eta_t_dot[k] * hdt;
        }
    }
    return sc;
}

// nhc_baro_half (nose_hoover_npt.cpp:347-420)
ATVB_DEV void npt_nhc_baro(const SysParams& P, SysState* st, double hdt) {
    const double qdt = 0.5 * hdt, edt = 0.5 * qdt;
    const int M = P.npt_mp;
    const double Wa = P.npt_W / 3.0;
    for (int pass = 0; pass < 2; ++pass) {
        for (int j = 0; j < M; ++j) {
            const int k = pass == 0 ? M - 1 - j : j;
            const double expfac = k < M - 1 ? exp(-st->eta_b_dot[k + 1] * edt) : 1.0;
            double G;
            if (k == 0) {
                double ke2 = 0.0;
                for (int a = 0; a < 3; ++a)
                    if (P.npt_couple[a])
                        ke2 += Wa * st->eps_dot[a] * st->eps_dot[a];
                G = (ke2 - st->kT) / P.npt_Qb;
            } else {
                G = (P.npt_Qb * st->eta_b_dot[k - 1] * st->eta_b_dot[k - 1] - st->kT) / P.npt_Qb;
            }
            st->eta_b_dot[k] *= expfac;
            st->eta_b_dot[k] += G * qdt;
            if (pass == 0)
                st->eta_b_dot[k] *= P.npt_pdrag;
            st->eta_b_dot[k] *= expfac;
        }
        if (pass == 0) {
            const double bs = exp(-st->eta_b_dot[0] * hdt);
            for (int a = 0; a < 3; ++a)
                if (P.npt_couple[a])
                    st->eps_dot[a] *= bs;
            for (int k = 0; k < M; ++k)
                st->eta_b[k] += st->eta_b_dot[k] * hdt;
        }
    }
}

// update_eps_dot (nose_hoover_npt.cpp:422-560): driving pressure per axis
// from the virial diagonal and 2 KE_a, averaged over the axes when all
// three are barostatted (couple())
ATVB_DEV void npt_update_eps(const SysParams& P, SysState* st, double hdt, const double ke[3]) {
    const double V = P.L[0] * P.L[1] * P.L[2];
    if (V <= 0.0)
        return;
    double diag[3] = {st->virial[0] + 2.0 * ke[0], st->virial[1] + 2.0 * ke[1],
                      st->virial[2] + 2.0 * ke[2]};
    if (P.npt_pdim == 3) {
        const double ave = (1.0 / 3.0) * (diag[0] + diag[1] + diag[2]);
        diag[0] = diag[1] = diag[2] = ave;
    }
    double mtk_ke = 0.0;
    for (int a = 0; a < 3; ++a)
        if (P.npt_couple[a])
            mtk_ke += ke[a];
    const int n_atoms = (P.n_dof + 3) / 3;
    const double mtk = P.npt_pdim > 0 ? 6.0 * mtk_ke / ((double)P.npt_pdim * n_atoms) : 0.0;
    for (int a = 0; a < 3; ++a) {
        if (!P.npt_couple[a])
            continue;
        const double Pa = diag[a] / V;
        const double G = (3.0 * V * (Pa - P.npt_P) + mtk) / P.npt_W;
        st->eps_dot[a] += G * hdt;
    }
}

// scale_v_by_baro factors (nose_hoover_npt.cpp:580-630); KE_global follows
// the reference's rule (isotropic: times s^2, else the per-axis sum)
ATVB_DEV void npt_scale_baro(const SysParams& P, SysState* st, double hdt, double ke[3],
                             double s[3]) {
    double sum = 0.0;
    for (int a = 0; a < 3; ++a)
        if (P.npt_couple[a])
            sum += st->eps_dot[a];
    const int n_atoms = (P.n_dof + 3) / 3;
    const double mtk2 = P.npt_pdim > 0 ? sum / ((double)P.npt_pdim * n_atoms) : 0.0;
    for (int a = 0; a < 3; ++a) {
        s[a] = exp(-(st->eps_dot[a] + mtk2) * hdt);
        ke[a] *= s[a] * s[a];
    }
    if (s[0] == s[1] && s[1] == s[2])
        st->ke_global *= s[0] * s[0];
    else
        st->ke_global = ke[0] + ke[1] + ke[2];
}

// extended_hamiltonian (nose_hoover_npt.cpp:770-805); st->kinetic and
// st->energy hold the end-of-step values
ATVB_DEV double npt_hamiltonian(const SysParams& P, const SysState* st) {
    double H = st->kinetic + st->energy;
    const double Wa = P.npt_W / 3.0;
    for (int a = 0; a < 3; ++a)
        if (P.npt_couple[a])
            H += 0.5 * Wa * st->eps_dot[a] * st->eps_dot[a];
    for (int k = 0; k < P.npt_mt; ++k)
        H += 0.5 * (k == 0 ? st->Qt0 : st->Qt1) * st->eta_t_dot[k] * st->eta_t_dot[k];
    for (int k = 0; k < P.npt_mp; ++k)
        H += 0.5 * P.npt_Qb * st->eta_b_dot[k] * st->eta_b_dot[k];
    H += (double)P.n_dof * st->kT * st->eta_t[0];
    for (int k = 1; k < P.npt_mt; ++k)
        H += st->kT * st->eta_t[k];
    for (int k = 0; k < P.npt_mp; ++k)
        H += st->kT * st->eta_b[k];
    H += P.npt_P * P.L[0] * P.L[1] * P.L[2];
    return H;
}

// The scalars of the next step's initial half (P1-P4: baro chain, atom
// chain, eps_dot from the virial of the last force evaluation, barostat
// velocity scale) and its drift factors (P6), from the state after a step.
// st->step is the index of the step to come; ke[] are the per-axis kinetic
// energies of the current velocities, vs_out[] the scale still pending on
// them.  The cell after the drift must stay above the smallest cell the
// neighbour grid was planned for; otherwise it is held (status bit set).
ATVB_DEV void npt_prepare(const SysParams& P, SysState* st, double ke[3], const double vs_out[3]) {
    const double hdt = 0.5 * P.dt;
    npt_temp_target(P, st, st->step);
    npt_nhc_baro(P, st, hdt);                            // P1
    const double s2 = npt_nhc_atoms(P, st, hdt, ke);     // P2
    npt_update_eps(P, st, hdt, ke);                      // P3
    double s4[3];
    npt_scale_baro(P, st, hdt, ke, s4);                  // P4
    for (int a = 0; a < 3; ++a) {
        st->vs_out[a] = vs_out[a];
        st->vs[a] = vs_out[a] * s2 * s4[a];
    }
    // P6: x <- x e^{eps dt} + v dt (e^{eps dt} - 1)/(eps dt), cell edge
    // times e^{eps dt} (nose_hoover_npt.cpp:650-700)
    double a[3], dr[3], Ln[3];
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
        double e = st->eps_dot[d] * P.dt;
        e = e < -kEpsDtMax ? -kEpsDtMax : (e > kEpsDtMax ? kEpsDtMax : e);
        a[d] = exp(e);
        dr[d] = npt_expm1c(e * 0.5);
        Ln[d] = P.L[d] * a[d];
        if (!(Ln[d] >= P.npt_Lmin[d]))
            ok = false;
    }
    if (!ok) {
        st->status |= kStatusBoxRange;
        st->held = 1;
        for (int d = 0; d < 3; ++d) {
            a[d] = 1.0;
            dr[d] = 1.0;
            Ln[d] = P.L[d];
        }
    }
    double lam = 1e300;
    for (int d = 0; d < 3; ++d) {
        st->npt_a[d] = a[d];
        st->npt_drift[d] = dr[d];
        st->Lnext[d] = Ln[d];
        st->fixn_scale[d] = 4294967296.0 / Ln[d];
        st->fixn64_scale[d] = 18446744073709551616.0 / Ln[d];
        st->ub[d] = st->Lb[d] / Ln[d];
        lam = fmin(lam, Ln[d] / st->Lb[d]);
    }
    // Rebuild rule under a changing cell: with u = x Lb / L the positions
    // mapped into the build cell, a pair left out of the list had
    // |u_j - u_i| >= rlist - 2 max|du|, so |r_ij| >= lam (rlist - 2 max|du|)
    // with lam the smallest edge ratio; it stays beyond the cutoff while
    // max|du| <= (rlist - cut / lam) / 2
    const double thr = 0.5 * (P.rlist - P.npt_cut / lam);
    st->disp_thr2 = thr > 0.0 ? thr * thr : -1.0;
    if (thr <= 0.0)
        st->need_rebuild = 1;
}

} // namespace atvb
