/* atvb_oracle.c -- CPU FP64 restatement of the Atomiverse classical-MD hot
 * path.  TEST INFRASTRUCTURE ONLY (the checker for the CUDA path and the CPU
 * baseline of bench.py); the product library never links or calls it.
 *
 * Built with -ffp-contract=off so that every product and sum is rounded on
 * its own, which is the rounding the CUDA neighbour build reproduces with
 * __dmul_rn/__dadd_rn: the pair sets of the two sides are then equal bit for
 * bit on the same coordinates.
 *
 * Reference algorithms restated here (paths in the Atomiverse tree):
 *   cell grid / stencil / binning  src/cpu/neighbor/cell_list.cpp:83-314
 *   half list (OpenMP path)        src/cpu/neighbor/cell_list.cpp:743-895
 *   neighbour decide               include/atomiverse/cpu/neighbor/neighbor_list.h:128-141
 *   LJ 12-6 shifted                src/cpu/potentials/pair_lj_cut.cpp:30-41,723-800
 *   real-space Ewald Coulomb       src/cpu/potentials/coul_long.cpp:146-222
 *   PME splines/moduli/spread      include/atomiverse/cpu/longrange/pme_spline.h:32-210
 *   PME influence/virial/gather    include/atomiverse/cpu/longrange/pme_influence.h:112-280
 *   PME driver, self + net terms   src/cpu/longrange/pme.cpp:64-131,152-253
 *   Ewald k-space sum              include/atomiverse/cpu/longrange/ewald_sum.h:58-140
 *   velocity Verlet                src/cpu/dynamics/velocity_verlet.cpp:24-68
 *   orthorhombic wrap              include/atomiverse/cpu/frame/pbc.h:37-52
 *   Nose-Hoover                    src/cpu/dynamics/nose_hoover.cpp:104-170
 *   Langevin + GaussStream         src/cpu/dynamics/fix_langevin.cpp:37-155
 *   kinetic energy                 src/cpu/dynamics/init.cpp:29-45
 *   Verlet step order              src/cpu/driver/runtime.cpp:452-501
 */
#include "atvb_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 0;

void orc_set_threads(int n) {
    g_threads = n;
#ifdef _OPENMP
    if (n > 0)
        omp_set_num_threads(n);
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* geometry helpers                                                    */
/* ------------------------------------------------------------------ */

/* pbc.h:48-50 */
static inline double wrap_coord(double x, double L) {
    return x - L * floor(x / L);
}

/* cell_list.h:214-227 (branchy min image used by the neighbour build) */
static inline double min_image_branchy(double d, double L, double half) {
    while (d > half)
        d -= L;
    while (d < -half)
        d += L;
    return d;
}

/* box.h:123-150 (nearbyint min image used by the force kernels) */
static inline double min_image_round(double d, double L) {
    return d - L * nearbyint(d / L);
}

/* ------------------------------------------------------------------ */
/* system object                                                       */
/* ------------------------------------------------------------------ */

struct orc_sys {
    orc_desc d;
    int n;
    double *x, *y, *z, *vx, *vy, *vz, *fx, *fy, *fz, *m, *q;
    int64_t* tag;
    /* neighbour state */
    double *xs, *ys, *zs; /* positions at last build */
    int ago;
    int rebuilds;
    int64_t npairs;
    int32_t* first; /* CSR over i */
    int32_t* num;
    int32_t* nbr;
    int64_t nbr_cap;
    /* scalars */
    double e_lj, e_coul, e_recip, e_const, e_ext, ke, vir[6];
    double xi, Q;
    int64_t step;
    int n_dof;
    /* PME persistent tables (pme.cpp:64-131) */
    int K[3];
    double* grid;    /* complex, interleaved */
    double* infl_H;  /* influence tables */
    double *infl_mx, *infl_my, *infl_mz, *infl_inv_msq;
    double inv_pi2_a2;
    double infl_L[3]; /* box the influence tables were built for */
    /* per-type LJ tables (ntypes x ntypes) and per-atom types */
    int ntypes;
    double *t_sig6, *t_eps, *t_shift;
    int32_t* type;
    /* special pairs: per atom, partners sorted by index with scales */
    int32_t* sp_first; /* n + 1 */
    int32_t* sp_j;
    double *sp_lj, *sp_coul;
    /* MTK NPT (nose_hoover_npt.cpp): parameters and extended state */
    int npt_on;
    orc_npt np;
    int pdim;
    double kT, T_live, W, tdrag, pdrag, KE_global, conserved;
    double Qt[ORC_MAXCHAIN], Qb[ORC_MAXCHAIN];
    double eta_t[ORC_MAXCHAIN], eta_t_dot[ORC_MAXCHAIN];
    double eta_b[ORC_MAXCHAIN], eta_b_dot[ORC_MAXCHAIN];
    double eps_dot[3];
    /* Berendsen barostat (barostat.cpp) */
    int baro_on;
    double baro_P, baro_tau, baro_bulk;
    /* NVELimit speed cap (0: off) and Deform (axis -1: off) */
    double vmax;
    int def_axis;
    double def_rate, def_L0;
    int64_t def_count;
};

orc_sys* orc_create(const orc_desc* d) {
    orc_sys* s = (orc_sys*)calloc(1, sizeof(orc_sys));
    s->d = *d;
    s->n = d->n;
    size_t n = (size_t)(d->n > 0 ? d->n : 1);
    double** arrs[] = {&s->x,  &s->y,  &s->z,  &s->vx, &s->vy, &s->vz, &s->fx,
                       &s->fy, &s->fz, &s->m,  &s->q,  &s->xs, &s->ys, &s->zs};
    for (size_t k = 0; k < sizeof(arrs) / sizeof(arrs[0]); ++k)
        *arrs[k] = (double*)calloc(n, sizeof(double));
    s->tag = (int64_t*)calloc(n, sizeof(int64_t));
    s->first = (int32_t*)calloc(n, sizeof(int32_t));
    s->num = (int32_t*)calloc(n, sizeof(int32_t));
    s->nbr = NULL;
    s->nbr_cap = 0;
    s->def_axis = -1;
    s->n_dof = 3 * d->n - 3;
    if (s->n_dof < 0)
        s->n_dof = 0;
    s->ago = 0;
    return s;
}

void orc_destroy(orc_sys* s) {
    if (!s)
        return;
    double* arrs[] = {s->x,  s->y,  s->z, s->vx, s->vy, s->vz, s->fx,
                      s->fy, s->fz, s->m, s->q,  s->xs, s->ys, s->zs};
    for (size_t k = 0; k < sizeof(arrs) / sizeof(arrs[0]); ++k)
        free(arrs[k]);
    free(s->tag);
    free(s->first);
    free(s->num);
    free(s->nbr);
    free(s->t_sig6);
    free(s->t_eps);
    free(s->t_shift);
    free(s->type);
    free(s->sp_first);
    free(s->sp_j);
    free(s->sp_lj);
    free(s->sp_coul);
    free(s->grid);
    free(s->infl_H);
    free(s->infl_mx);
    free(s->infl_my);
    free(s->infl_mz);
    free(s->infl_inv_msq);
    free(s);
}

void orc_set_state(orc_sys* s, const double* x, const double* y,
                   const double* z, const double* vx, const double* vy,
                   const double* vz, const double* fx, const double* fy,
                   const double* fz, const double* mass, const double* q,
                   const int64_t* tag) {
    const int n = s->n;
    for (int i = 0; i < n; ++i) {
        s->x[i] = wrap_coord(x[i], s->d.L[0]);
        s->y[i] = wrap_coord(y[i], s->d.L[1]);
        s->z[i] = wrap_coord(z[i], s->d.L[2]);
        s->vx[i] = vx ? vx[i] : 0.0;
        s->vy[i] = vy ? vy[i] : 0.0;
        s->vz[i] = vz ? vz[i] : 0.0;
        s->fx[i] = fx ? fx[i] : 0.0;
        s->fy[i] = fy ? fy[i] : 0.0;
        s->fz[i] = fz ? fz[i] : 0.0;
        s->m[i] = mass ? mass[i] : 1.0;
        s->q[i] = q ? q[i] : 0.0;
        s->tag[i] = tag ? tag[i] : (int64_t)(i + 1);
    }
}

void orc_get_state(const orc_sys* s, double* x, double* y, double* z,
                   double* vx, double* vy, double* vz, double* fx, double* fy,
                   double* fz) {
    const size_t b = (size_t)s->n * sizeof(double);
    if (x)
        memcpy(x, s->x, b);
    if (y)
        memcpy(y, s->y, b);
    if (z)
        memcpy(z, s->z, b);
    if (vx)
        memcpy(vx, s->vx, b);
    if (vy)
        memcpy(vy, s->vy, b);
    if (vz)
        memcpy(vz, s->vz, b);
    if (fx)
        memcpy(fx, s->fx, b);
    if (fy)
        memcpy(fy, s->fy, b);
    if (fz)
        memcpy(fz, s->fz, b);
}

void orc_scalars(const orc_sys* s, double* out) {
    out[0] = s->e_lj + s->e_coul + s->e_recip + s->e_const + s->e_ext;
    out[1] = s->e_lj;
    out[2] = s->e_coul;
    out[3] = s->e_recip;
    out[4] = s->e_const;
    out[5] = s->ke;
    for (int k = 0; k < 6; ++k)
        out[6 + k] = s->vir[k];
    out[12] = s->xi;
    out[13] = (double)s->step;
    out[14] = (double)s->rebuilds;
}

/* ------------------------------------------------------------------ */
/* neighbour list: cell grid, stencil, binning, half list              */
/* ------------------------------------------------------------------ */

typedef struct {
    int di, dj, dk;
} stencil_off;

/* cell_list.cpp:83-154 (grid), :179-232 (stencil), :234-314 (binning),
 * :743-895 (OpenMP full-stencil half list with j > i and min image). */
int64_t orc_build_list(orc_sys* s) {
    const int n = s->n;
    const double rl = s->d.nl_cutoff + s->d.skin;
    const double rl2 = rl * rl;
    int nc[3];
    double cs[3];
    for (int d = 0; d < 3; ++d) {
        int c = (int)floor(s->d.L[d] / (0.5 * rl));
        nc[d] = c < 1 ? 1 : c;
        cs[d] = s->d.L[d] / nc[d];
    }
    int reach[3];
    for (int d = 0; d < 3; ++d) {
        int r = (int)ceil(rl / cs[d] - 1e-12);
        reach[d] = r < 1 ? 1 : r;
    }
    /* full stencil with LAMMPS bin_distance pruning */
    int nmax = (2 * reach[0] + 1) * (2 * reach[1] + 1) * (2 * reach[2] + 1);
    stencil_off* st = (stencil_off*)malloc(sizeof(stencil_off) * nmax);
    int nst = 0;
    for (int di = -reach[0]; di <= reach[0]; ++di)
        for (int dj = -reach[1]; dj <= reach[1]; ++dj)
            for (int dk = -reach[2]; dk <= reach[2]; ++dk) {
                double ddx = di > 0 ? (di - 1) * cs[0]
                                    : (di < 0 ? (di + 1) * cs[0] : 0.0);
                double ddy = dj > 0 ? (dj - 1) * cs[1]
                                    : (dj < 0 ? (dj + 1) * cs[1] : 0.0);
                double ddz = dk > 0 ? (dk - 1) * cs[2]
                                    : (dk < 0 ? (dk + 1) * cs[2] : 0.0);
                if (ddx * ddx + ddy * ddy + ddz * ddz > rl2)
                    continue;
                st[nst].di = di;
                st[nst].dj = dj;
                st[nst].dk = dk;
                ++nst;
            }
    const int ncell = nc[0] * nc[1] * nc[2];
    int* cell_of = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
    int* count = (int*)calloc((size_t)ncell, sizeof(int));
    int* offset = (int*)malloc(sizeof(int) * (size_t)(ncell + 1));
    int* binned = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        double p[3] = {wrap_coord(s->x[i], s->d.L[0]),
                       wrap_coord(s->y[i], s->d.L[1]),
                       wrap_coord(s->z[i], s->d.L[2])};
        int c[3];
        for (int d = 0; d < 3; ++d) {
            c[d] = (int)floor(p[d] / cs[d]);
            if (c[d] < 0)
                c[d] = 0;
            if (c[d] > nc[d] - 1)
                c[d] = nc[d] - 1;
        }
        cell_of[i] = c[0] * nc[1] * nc[2] + c[1] * nc[2] + c[2];
        count[cell_of[i]]++;
    }
    offset[0] = 0;
    for (int c = 0; c < ncell; ++c)
        offset[c + 1] = offset[c] + count[c];
    {
        int* wp = (int*)malloc(sizeof(int) * (size_t)ncell);
        memcpy(wp, offset, sizeof(int) * (size_t)ncell);
        for (int i = 0; i < n; ++i)
            binned[wp[cell_of[i]]++] = i;
        free(wp);
    }

    const double hx = 0.5 * s->d.L[0], hy = 0.5 * s->d.L[1],
                 hz = 0.5 * s->d.L[2];
    /* pass 1: counts */
    int32_t* num = s->num;
#pragma omp parallel
    {
        int* visited = (int*)malloc(sizeof(int) * (size_t)(nst > 0 ? nst : 1));
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < n; ++i) {
            const int ci = cell_of[i];
            const int cz0 = ci % nc[2];
            const int cy0 = (ci / nc[2]) % nc[1];
            const int cx0 = ci / (nc[1] * nc[2]);
            int nv = 0, cnt = 0;
            for (int t = 0; t < nst; ++t) {
                int cx = cx0 + st[t].di, cy = cy0 + st[t].dj,
                    cz = cz0 + st[t].dk;
                cx = ((cx % nc[0]) + nc[0]) % nc[0];
                cy = ((cy % nc[1]) + nc[1]) % nc[1];
                cz = ((cz % nc[2]) + nc[2]) % nc[2];
                const int cj = cx * nc[1] * nc[2] + cy * nc[2] + cz;
                int seen = 0;
                for (int v = 0; v < nv; ++v)
                    if (visited[v] == cj) {
                        seen = 1;
                        break;
                    }
                if (seen)
                    continue;
                visited[nv++] = cj;
                for (int idx = offset[cj]; idx < offset[cj + 1]; ++idx) {
                    const int j = binned[idx];
                    if (j <= i)
                        continue;
                    double dx = min_image_branchy(s->x[i] - s->x[j],
                                                  s->d.L[0], hx);
                    double dy = min_image_branchy(s->y[i] - s->y[j],
                                                  s->d.L[1], hy);
                    double dz = min_image_branchy(s->z[i] - s->z[j],
                                                  s->d.L[2], hz);
                    double r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 < rl2)
                        ++cnt;
                }
            }
            num[i] = cnt;
        }
        free(visited);
    }
    int64_t tot = 0;
    for (int i = 0; i < n; ++i) {
        s->first[i] = (int32_t)tot;
        tot += num[i];
    }
    if (tot > s->nbr_cap) {
        free(s->nbr);
        s->nbr_cap = tot + tot / 4 + 16;
        s->nbr = (int32_t*)malloc(sizeof(int32_t) * (size_t)s->nbr_cap);
    }
    /* pass 2: fill (each i writes its own contiguous slice) */
#pragma omp parallel
    {
        int* visited = (int*)malloc(sizeof(int) * (size_t)(nst > 0 ? nst : 1));
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < n; ++i) {
            const int ci = cell_of[i];
            const int cz0 = ci % nc[2];
            const int cy0 = (ci / nc[2]) % nc[1];
            const int cx0 = ci / (nc[1] * nc[2]);
            int nv = 0;
            int64_t w = s->first[i];
            for (int t = 0; t < nst; ++t) {
                int cx = cx0 + st[t].di, cy = cy0 + st[t].dj,
                    cz = cz0 + st[t].dk;
                cx = ((cx % nc[0]) + nc[0]) % nc[0];
                cy = ((cy % nc[1]) + nc[1]) % nc[1];
                cz = ((cz % nc[2]) + nc[2]) % nc[2];
                const int cj = cx * nc[1] * nc[2] + cy * nc[2] + cz;
                int seen = 0;
                for (int v = 0; v < nv; ++v)
                    if (visited[v] == cj) {
                        seen = 1;
                        break;
                    }
                if (seen)
                    continue;
                visited[nv++] = cj;
                for (int idx = offset[cj]; idx < offset[cj + 1]; ++idx) {
                    const int j = binned[idx];
                    if (j <= i)
                        continue;
                    double dx = min_image_branchy(s->x[i] - s->x[j],
                                                  s->d.L[0], hx);
                    double dy = min_image_branchy(s->y[i] - s->y[j],
                                                  s->d.L[1], hy);
                    double dz = min_image_branchy(s->z[i] - s->z[j],
                                                  s->d.L[2], hz);
                    double r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 < rl2)
                        s->nbr[w++] = j;
                }
            }
        }
        free(visited);
    }
    s->npairs = tot;
    /* cell_list.cpp:316-327 save_positions */
    memcpy(s->xs, s->x, sizeof(double) * (size_t)n);
    memcpy(s->ys, s->y, sizeof(double) * (size_t)n);
    memcpy(s->zs, s->z, sizeof(double) * (size_t)n);
    s->ago = 0;
    free(st);
    free(cell_of);
    free(count);
    free(offset);
    free(binned);
    return tot;
}

void orc_get_pairs(const orc_sys* s, int32_t* pi, int32_t* pj) {
    int64_t w = 0;
    for (int i = 0; i < s->n; ++i)
        for (int k = 0; k < s->num[i]; ++k) {
            pi[w] = i;
            pj[w] = s->nbr[s->first[i] + k];
            ++w;
        }
}

/* cell_list.cpp:355-392: rebuild when 4 * max_disp^2 > skin^2 */
static int needs_rebuild(const orc_sys* s) {
    double mx = 0.0;
    const double L0 = s->d.L[0], L1 = s->d.L[1], L2 = s->d.L[2];
#pragma omp parallel for reduction(max : mx) schedule(static)
    for (int i = 0; i < s->n; ++i) {
        double dx = min_image_round(s->x[i] - s->xs[i], L0);
        double dy = min_image_round(s->y[i] - s->ys[i], L1);
        double dz = min_image_round(s->z[i] - s->zs[i], L2);
        double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 > mx)
            mx = d2;
    }
    return mx * 4.0 > s->d.skin * s->d.skin;
}

/* ------------------------------------------------------------------ */
/* per-type LJ tables and special pairs                                */
/* ------------------------------------------------------------------ */

int orc_set_lj_types(orc_sys* s, int ncoef, const int32_t* ti, const int32_t* tj,
                     const double* eps, const double* sigma, const int32_t* type) {
    int nt = 0;
    for (int k = 0; k < ncoef; ++k) {
        if (ti[k] < 0 || tj[k] < 0 || !(sigma[k] > 0.0))
            return -1;
        if (ti[k] + 1 > nt)
            nt = ti[k] + 1;
        if (tj[k] + 1 > nt)
            nt = tj[k] + 1;
    }
    /* atom types without coefficients have no LJ site (eps = 0) */
    for (int i = 0; type && i < s->n; ++i) {
        if (type[i] < 0)
            return -1;
        if (type[i] + 1 > nt)
            nt = type[i] + 1;
    }
    const size_t nn = (size_t)nt * nt;
    double* e = (double*)calloc(nn, sizeof(double));
    double* sg = (double*)calloc(nn, sizeof(double));
    char* set = (char*)calloc(nn, 1);
    for (int k = 0; k < ncoef; ++k) { /* set_type_coeff: symmetric, last wins */
        const size_t ab = (size_t)ti[k] * nt + tj[k], ba = (size_t)tj[k] * nt + ti[k];
        e[ab] = e[ba] = eps[k];
        sg[ab] = sg[ba] = sigma[k];
        set[ab] = set[ba] = 1;
    }
    free(s->t_sig6);
    free(s->t_eps);
    free(s->t_shift);
    s->t_sig6 = (double*)calloc(nn, sizeof(double));
    s->t_eps = (double*)calloc(nn, sizeof(double));
    s->t_shift = (double*)calloc(nn, sizeof(double));
    const double rc = s->d.lj_rc;
    for (int a = 0; a < nt; ++a)
        for (int b = 0; b < nt; ++b) {
            const size_t ab = (size_t)a * nt + b;
            double ee = e[ab], ss = sg[ab];
            if (!set[ab]) {
                const size_t aa = (size_t)a * nt + a, bb = (size_t)b * nt + b;
                if (set[aa] && set[bb]) {
                    ee = sqrt(e[aa] * e[bb]);
                    ss = 0.5 * (sg[aa] + sg[bb]);
                } else {
                    ee = 0.0;
                    ss = 1.0;
                }
            }
            const double s2 = ss * ss, s6 = s2 * s2 * s2;
            s->t_sig6[ab] = s6;
            s->t_eps[ab] = ee;
            const double r2inv = 1.0 / (rc * rc);
            const double r6inv = r2inv * r2inv * r2inv * s6;
            s->t_shift[ab] = 4.0 * ee * (r6inv * r6inv - r6inv);
        }
    free(e);
    free(sg);
    free(set);
    free(s->type);
    s->type = (int32_t*)calloc((size_t)(s->n > 0 ? s->n : 1), sizeof(int32_t));
    for (int i = 0; i < s->n; ++i)
        s->type[i] = type ? type[i] : 0;
    s->ntypes = nt;
    return nt;
}

void orc_set_special(orc_sys* s, int npairs, const int32_t* pi, const int32_t* pj,
                     const double* s_lj, const double* s_coul) {
    const int n = s->n;
    free(s->sp_first);
    free(s->sp_j);
    free(s->sp_lj);
    free(s->sp_coul);
    s->sp_first = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    for (int k = 0; k < npairs; ++k) {
        s->sp_first[pi[k] + 1]++;
        s->sp_first[pj[k] + 1]++;
    }
    for (int i = 0; i < n; ++i)
        s->sp_first[i + 1] += s->sp_first[i];
    const size_t m = (size_t)s->sp_first[n];
    s->sp_j = (int32_t*)calloc(m ? m : 1, sizeof(int32_t));
    s->sp_lj = (double*)calloc(m ? m : 1, sizeof(double));
    s->sp_coul = (double*)calloc(m ? m : 1, sizeof(double));
    int32_t* fill = (int32_t*)calloc((size_t)n, sizeof(int32_t));
    for (int k = 0; k < npairs; ++k) {
        const int a = pi[k], b = pj[k];
        size_t q = (size_t)s->sp_first[a] + fill[a]++;
        s->sp_j[q] = b;
        s->sp_lj[q] = s_lj[k];
        s->sp_coul[q] = s_coul[k];
        q = (size_t)s->sp_first[b] + fill[b]++;
        s->sp_j[q] = a;
        s->sp_lj[q] = s_lj[k];
        s->sp_coul[q] = s_coul[k];
    }
    free(fill);
}

/* LJ and Coulomb scale of pair (i, j): 1, 1 unless listed as special */
static void special_scale(const orc_sys* s, int i, int j, double* sl, double* sc) {
    *sl = 1.0;
    *sc = 1.0;
    if (!s->sp_first)
        return;
    for (int q = s->sp_first[i]; q < s->sp_first[i + 1]; ++q)
        if (s->sp_j[q] == j) {
            *sl = s->sp_lj[q];
            *sc = s->sp_coul[q];
            return;
        }
}

/* ------------------------------------------------------------------ */
/* pair forces: LJ (pair_lj_cut.cpp:723-800) + CoulLong (coul_long.cpp)  */
/* ------------------------------------------------------------------ */

static void pair_forces(orc_sys* s) {
    const int n = s->n;
    const double L0 = s->d.L[0], L1 = s->d.L[1], L2 = s->d.L[2];
    const double iL0 = 1.0 / L0, iL1 = 1.0 / L1, iL2 = 1.0 / L2;
    const int do_lj = s->d.has_lj, do_coul = s->d.has_coul;
    const double lj_rc2 = s->d.lj_rc * s->d.lj_rc;
    const double sig2 = s->d.lj_sigma * s->d.lj_sigma;
    const double sig6 = sig2 * sig2 * sig2;
    const double eps24 = 24.0 * s->d.lj_eps, eps4 = 4.0 * s->d.lj_eps;
    double vshift;
    {
        /* pair_lj_cut.cpp:37-40 */
        double r2inv = 1.0 / lj_rc2;
        double r6inv = r2inv * r2inv * r2inv * sig6;
        vshift = 4.0 * s->d.lj_eps * (r6inv * r6inv - r6inv);
    }
    const double c_rc2 = s->d.coul_rc * s->d.coul_rc;
    const double alpha = s->d.coul_alpha;
    const double kEwaldF = 1.1283791670955126; /* 2/sqrt(pi) */
    const int nt = orc_get_threads();
    double* fbuf = (double*)calloc((size_t)nt * 3 * (size_t)n, sizeof(double));
    double e_lj = 0, e_c = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
#pragma omp parallel reduction(+ : e_lj, e_c, v0, v1, v2, v3, v4, v5)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* fxt = fbuf + (size_t)tid * 3 * (size_t)n;
        double* fyt = fxt + n;
        double* fzt = fyt + n;
#pragma omp for schedule(dynamic, 32)
        for (int i = 0; i < n; ++i) {
            const double xi = s->x[i], yi = s->y[i], zi = s->z[i];
            const double qi = s->q[i];
            double fix = 0, fiy = 0, fiz = 0;
            const int off = s->first[i];
            for (int k = 0; k < s->num[i]; ++k) {
                const int j = s->nbr[off + k];
                double dx = min_image_round(xi - s->x[j], L0);
                double dy = min_image_round(yi - s->y[j], L1);
                double dz = min_image_round(zi - s->z[j], L2);
                (void)iL0;
                (void)iL1;
                (void)iL2;
                const double r2 = dx * dx + dy * dy + dz * dz;
                double fpair = 0.0;
                double sl = 1.0, sc = 1.0;
                special_scale(s, i, j, &sl, &sc);
                if (do_lj && r2 < lj_rc2 && sl != 0.0) {
                    double p_sig6 = sig6, p_eps24 = eps24, p_eps4 = eps4, p_shift = vshift;
                    if (s->ntypes) { /* pair_lj_cut.cpp:760-770 */
                        const size_t ab = (size_t)s->type[i] * s->ntypes + s->type[j];
                        p_sig6 = s->t_sig6[ab];
                        p_eps24 = 24.0 * s->t_eps[ab];
                        p_eps4 = 4.0 * s->t_eps[ab];
                        p_shift = s->t_shift[ab];
                    }
                    const double r2inv = 1.0 / r2;
                    const double r6inv = r2inv * r2inv * r2inv * p_sig6;
                    fpair += sl * p_eps24 * r2inv * (2.0 * r6inv * r6inv - r6inv);
                    e_lj += sl * (p_eps4 * (r6inv * r6inv - r6inv) - p_shift);
                }
                if (do_coul && r2 < c_rc2 && r2 != 0.0) {
                    const double qj = s->q[j];
                    if (qi != 0.0 && qj != 0.0) {
                        const double r = sqrt(r2);
                        const double r2inv = 1.0 / r2;
                        const double grij = alpha * r;
                        const double expm2 = exp(-grij * grij);
                        const double erfcv = erfc(grij);
                        const double prefactor = ORC_QQR2E * qi * qj / r;
                        double forcecoul =
                            prefactor * (erfcv + kEwaldF * grij * expm2);
                        if (sc != 1.0)
                            forcecoul -= (1.0 - sc) * prefactor;
                        fpair += forcecoul * r2inv;
                        e_c += sc != 1.0 ? prefactor * erfcv - (1.0 - sc) * prefactor
                                         : prefactor * erfcv;
                    }
                }
                if (fpair != 0.0) {
                    const double fxp = fpair * dx, fyp = fpair * dy,
                                 fzp = fpair * dz;
                    fix += fxp;
                    fiy += fyp;
                    fiz += fzp;
                    fxt[j] -= fxp;
                    fyt[j] -= fyp;
                    fzt[j] -= fzp;
                    v0 += dx * fxp;
                    v1 += dy * fyp;
                    v2 += dz * fzp;
                    v3 += dx * fyp;
                    v4 += dx * fzp;
                    v5 += dy * fzp;
                }
            }
            fxt[i] += fix;
            fyt[i] += fiy;
            fzt[i] += fiz;
        }
#pragma omp barrier
#pragma omp for schedule(static)
        for (int i = 0; i < n; ++i) {
            double ax = 0, ay = 0, az = 0;
            for (int t = 0; t < nt; ++t) {
                const double* b = fbuf + (size_t)t * 3 * (size_t)n;
                ax += b[i];
                ay += b[n + i];
                az += b[2 * n + i];
            }
            s->fx[i] += ax;
            s->fy[i] += ay;
            s->fz[i] += az;
        }
    }
    free(fbuf);
    s->e_lj += e_lj;
    s->e_coul += e_c;
    s->vir[0] += v0;
    s->vir[1] += v1;
    s->vir[2] += v2;
    s->vir[3] += v3;
    s->vir[4] += v4;
    s->vir[5] += v5;
}

/* ------------------------------------------------------------------ */
/* PME math (pme_spline.h / pme_influence.h)                           */
/* ------------------------------------------------------------------ */

/* pme_spline.h:32-58: Essmann cardinal B-spline recursion */
void orc_bspline(double frac, int n, double* theta, double* dtheta) {
    theta[n - 1] = 0.0;
    theta[1] = frac;
    theta[0] = 1.0 - frac;
    for (int k = 3; k < n; ++k) {
        const double div = 1.0 / (k - 1);
        theta[k - 1] = div * frac * theta[k - 2];
        for (int j = 1; j < k - 1; ++j)
            theta[k - 1 - j] = div * ((frac + j) * theta[k - 2 - j] +
                                      (k - j - frac) * theta[k - 1 - j]);
        theta[0] = div * (1.0 - frac) * theta[0];
    }
    dtheta[0] = -theta[0];
    for (int j = 1; j < n; ++j)
        dtheta[j] = theta[j - 1] - theta[j];
    const double div = 1.0 / (n - 1);
    theta[n - 1] = div * frac * theta[n - 2];
    for (int j = 1; j < n - 1; ++j)
        theta[n - 1 - j] = div * ((frac + j) * theta[n - 2 - j] +
                                  (n - j - frac) * theta[n - 1 - j]);
    theta[0] = div * (1.0 - frac) * theta[0];
}

/* pme_spline.h:67-94: Euler spline moduli with zero repair */
void orc_spline_moduli(int K, int n, double* mod) {
    double data[32], dd[32];
    orc_bspline(0.0, n, data, dd);
    for (int i = 0; i < K; ++i) {
        double sr = 0, si = 0;
        for (int k = 0; k < n - 1; ++k) {
            const double arg = 2.0 * ORC_PI * i * k / K;
            sr += data[k] * cos(arg);
            si += data[k] * sin(arg);
        }
        const double den = sr * sr + si * si;
        mod[i] = den > 1e-12 ? 1.0 / den : 0.0;
    }
    for (int i = 0; i < K; ++i)
        if (mod[i] == 0.0)
            mod[i] = 0.5 * (mod[(i - 1 + K) % K] + mod[(i + 1) % K]);
}

/* pme_spline.h:99-111 */
int orc_good_fft_size(int n) {
    if (n < 4)
        n = 4;
    for (;; ++n) {
        int m = n;
        const int ps[4] = {2, 3, 5, 7};
        for (int k = 0; k < 4; ++k)
            while (m % ps[k] == 0)
                m /= ps[k];
        if (m == 1)
            return n;
    }
}

/* ---- own mixed-radix (2,3,4,5,7) Stockham FFT; FFTW3 is not available --- */

typedef struct {
    int n, nst, radix[64];
    double complex* tw[64]; /* per stage: Ns*R twiddles */
    int sign;
} fft_plan1;

static void plan1_init(fft_plan1* p, int n, int sign) {
    p->n = n;
    p->sign = sign;
    p->nst = 0;
    int m = n;
    while (m % 4 == 0) {
        p->radix[p->nst++] = 4;
        m /= 4;
    }
    const int ps[4] = {2, 3, 5, 7};
    for (int k = 0; k < 4; ++k)
        while (m % ps[k] == 0) {
            p->radix[p->nst++] = ps[k];
            m /= ps[k];
        }
    if (m != 1) { /* not smooth: treat the rest as one radix (direct DFT) */
        p->radix[p->nst++] = m;
    }
    int Ns = 1;
    for (int st = 0; st < p->nst; ++st) {
        const int R = p->radix[st];
        p->tw[st] = (double complex*)malloc(sizeof(double complex) *
                                            (size_t)(Ns * R));
        for (int j = 0; j < Ns; ++j)
            for (int r = 0; r < R; ++r) {
                const double ang = sign * 2.0 * ORC_PI * (double)(j * r) /
                                   (double)(Ns * R);
                p->tw[st][j * R + r] = cos(ang) + I * sin(ang);
            }
        Ns *= R;
    }
}

static void plan1_free(fft_plan1* p) {
    for (int st = 0; st < p->nst; ++st)
        free(p->tw[st]);
}

/* Stockham autosort FFT (Govindaraju et al. formulation): out-of-place
 * ping-pong between a and b; result returned pointer. */
static double complex* fft1(const fft_plan1* p, double complex* a,
                            double complex* b) {
    const int N = p->n;
    int Ns = 1;
    double complex v[64];
    double complex wR[64];
    for (int st = 0; st < p->nst; ++st) {
        const int R = p->radix[st];
        for (int r = 0; r < R; ++r) {
            const double ang = p->sign * 2.0 * ORC_PI * r / R;
            wR[r] = cos(ang) + I * sin(ang);
        }
        const int NR = N / R;
        for (int j = 0; j < NR; ++j) {
            const int jm = j % Ns;
            const double complex* tw = p->tw[st] + jm * R;
            for (int r = 0; r < R; ++r)
                v[r] = a[j + r * NR] * tw[r];
            double complex o[64];
            if (R == 2) {
                o[0] = v[0] + v[1];
                o[1] = v[0] - v[1];
            } else if (R == 4) {
                const double complex t0 = v[0] + v[2], t1 = v[0] - v[2];
                const double complex t2 = v[1] + v[3];
                double complex t3 = v[1] - v[3];
                /* multiply by sign*i */
                t3 = (p->sign < 0) ? (cimag(t3) - I * creal(t3))
                                   : (-cimag(t3) + I * creal(t3));
                o[0] = t0 + t2;
                o[2] = t0 - t2;
                o[1] = t1 + t3;
                o[3] = t1 - t3;
            } else {
                for (int k = 0; k < R; ++k) {
                    double complex acc = 0;
                    for (int r = 0; r < R; ++r)
                        acc += v[r] * wR[(k * r) % R];
                    o[k] = acc;
                }
            }
            const int idxD = (j / Ns) * Ns * R + jm;
            for (int r = 0; r < R; ++r)
                b[idxD + r * Ns] = o[r];
        }
        double complex* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

void orc_fft3d(int K0, int K1, int K2, double* data, int sign) {
    double complex* g = (double complex*)data;
    const int Ks[3] = {K0, K1, K2};
    for (int dim = 2; dim >= 0; --dim) {
        const int n = Ks[dim];
        fft_plan1 p;
        plan1_init(&p, n, sign);
        const long stride = dim == 2 ? 1 : (dim == 1 ? K2 : (long)K1 * K2);
        const long nlines = (long)K0 * K1 * K2 / n;
#pragma omp parallel
        {
            double complex* a =
                (double complex*)malloc(sizeof(double complex) * (size_t)n);
            double complex* b =
                (double complex*)malloc(sizeof(double complex) * (size_t)n);
#pragma omp for schedule(static)
            for (long line = 0; line < nlines; ++line) {
                long base;
                if (dim == 2)
                    base = line * K2;
                else if (dim == 1)
                    base = (line / K2) * (long)K1 * K2 + (line % K2);
                else
                    base = line;
                for (int k = 0; k < n; ++k)
                    a[k] = g[base + k * stride];
                const double complex* r = fft1(&p, a, b);
                for (int k = 0; k < n; ++k)
                    g[base + k * stride] = r[k];
            }
            free(a);
            free(b);
        }
        plan1_free(&p);
    }
}

static inline int pme_wrap(int g, int K) {
    if (g >= K)
        g -= K;
    if (g < 0)
        g += K;
    if (g >= K)
        g -= K;
    if (g < 0)
        g += K;
    return g;
}

/* pme.cpp:64-131 ensure_grid + pme_influence.h:112-155 tables */
static void pme_setup(orc_sys* s) {
    /* the tables depend on the cell: rebuilt whenever it changed (NPT) */
    if (s->grid && s->infl_L[0] == s->d.L[0] && s->infl_L[1] == s->d.L[1] &&
        s->infl_L[2] == s->d.L[2])
        return;
    for (int d = 0; d < 3; ++d)
        s->K[d] = s->d.pme_K[d];
    const long ntot = (long)s->K[0] * s->K[1] * s->K[2];
    if (!s->grid) {
        s->grid = (double*)calloc((size_t)(2 * ntot), sizeof(double));
        s->infl_H = (double*)calloc((size_t)ntot, sizeof(double));
        s->infl_mx = (double*)calloc((size_t)ntot, sizeof(double));
        s->infl_my = (double*)calloc((size_t)ntot, sizeof(double));
        s->infl_mz = (double*)calloc((size_t)ntot, sizeof(double));
        s->infl_inv_msq = (double*)calloc((size_t)ntot, sizeof(double));
    }
    for (int d = 0; d < 3; ++d)
        s->infl_L[d] = s->d.L[d];
    const int order = s->d.pme_order;
    double* bm[3];
    for (int d = 0; d < 3; ++d) {
        bm[d] = (double*)malloc(sizeof(double) * (size_t)s->K[d]);
        orc_spline_moduli(s->K[d], order, bm[d]);
    }
    const double alpha = s->d.pme_alpha;
    s->inv_pi2_a2 = ORC_PI * ORC_PI / (alpha * alpha);
    const double ic[3] = {1.0 / s->d.L[0], 1.0 / s->d.L[1], 1.0 / s->d.L[2]};
    const int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2];
#pragma omp parallel for schedule(static)
    for (int m0 = 0; m0 < K0; ++m0) {
        const int h0 = (m0 <= K0 / 2) ? m0 : m0 - K0;
        for (int m1 = 0; m1 < K1; ++m1) {
            const int h1 = (m1 <= K1 / 2) ? m1 : m1 - K1;
            const double bm01 = bm[0][m0] * bm[1][m1];
            for (int m2 = 0; m2 < K2; ++m2) {
                const long idx = m2 + (long)K2 * (m1 + (long)K1 * m0);
                if (m0 == 0 && m1 == 0 && m2 == 0)
                    continue;
                const int h2 = (m2 <= K2 / 2) ? m2 : m2 - K2;
                const double mx = h0 * ic[0], my = h1 * ic[1], mz = h2 * ic[2];
                const double msq = mx * mx + my * my + mz * mz;
                const double inv_msq = 1.0 / msq;
                const double B = bm01 * bm[2][m2];
                s->infl_H[idx] = exp(-s->inv_pi2_a2 * msq) * inv_msq * B;
                s->infl_mx[idx] = mx;
                s->infl_my[idx] = my;
                s->infl_mz[idx] = mz;
                s->infl_inv_msq[idx] = inv_msq;
            }
        }
    }
    for (int d = 0; d < 3; ++d)
        free(bm[d]);
}

/* pme.cpp:152-253: spread, FFT, influence (+virial), inverse FFT, gather,
 * self and net-charge energies. */
static void pme_forces(orc_sys* s) {
    pme_setup(s);
    const int n = s->n, order = s->d.pme_order, nm1 = order - 1;
    const int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2];
    const long ntot = (long)K0 * K1 * K2;
    const double ic[3] = {1.0 / s->d.L[0], 1.0 / s->d.L[1], 1.0 / s->d.L[2]};
    const double vol = s->d.L[0] * s->d.L[1] * s->d.L[2];
    int* base = (int*)malloc(sizeof(int) * 3 * (size_t)(n > 0 ? n : 1));
    double* th =
        (double*)malloc(sizeof(double) * 3 * (size_t)order * (n > 0 ? n : 1));
    double* dth =
        (double*)malloc(sizeof(double) * 3 * (size_t)order * (n > 0 ? n : 1));
    /* pme_spline.h:124-144 */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const double p[3] = {s->x[i], s->y[i], s->z[i]};
        for (int d = 0; d < 3; ++d) {
            const double sd = ic[d] * p[d];
            double u = sd * s->K[d];
            u -= floor(u / s->K[d]) * s->K[d];
            const int u0 = (int)floor(u);
            const double frac = u - u0;
            orc_bspline(frac, order, &th[(3 * i + d) * order],
                        &dth[(3 * i + d) * order]);
            base[3 * i + d] = u0;
        }
    }
    memset(s->grid, 0, sizeof(double) * 2 * (size_t)ntot);
    /* pme_spline.h:176-210 (serial: the oracle keeps the reference's
     * summation order) */
    for (int i = 0; i < n; ++i) {
        const double qi = s->q[i];
        if (qi == 0.0)
            continue;
        const double* thx = &th[(3 * i + 0) * order];
        const double* thy = &th[(3 * i + 1) * order];
        const double* thz = &th[(3 * i + 2) * order];
        const int b0 = base[3 * i + 0] - nm1;
        const int b1 = base[3 * i + 1] - nm1;
        const int b2 = base[3 * i + 2] - nm1;
        for (int a = 0; a < order; ++a) {
            const int g0 = pme_wrap(b0 + a, K0);
            const double wa = qi * thx[a];
            for (int b = 0; b < order; ++b) {
                const int g1 = pme_wrap(b1 + b, K1);
                const double wab = wa * thy[b];
                const long plane = (long)K2 * (g1 + (long)K1 * g0);
                for (int c = 0; c < order; ++c) {
                    const int g2 = pme_wrap(b2 + c, K2);
                    s->grid[2 * (plane + g2)] += wab * thz[c];
                }
            }
        }
    }
    orc_fft3d(K0, K1, K2, s->grid, -1);
    /* pme_influence.h:159-199 */
    double e = 0, w0 = 0, w1 = 0, w2 = 0, w3 = 0, w4 = 0, w5 = 0;
    const double vt_const = s->inv_pi2_a2;
#pragma omp parallel for reduction(+ : e, w0, w1, w2, w3, w4, w5) \
    schedule(static)
    for (long idx = 0; idx < ntot; ++idx) {
        const double h = s->infl_H[idx];
        if (h == 0.0) {
            s->grid[2 * idx] = 0;
            s->grid[2 * idx + 1] = 0;
            continue;
        }
        const double re = s->grid[2 * idx], im = s->grid[2 * idx + 1];
        const double q2 = re * re + im * im;
        e += h * q2;
        const double vt = -2.0 * (s->infl_inv_msq[idx] + vt_const);
        const double ug = h * q2;
        const double mx = s->infl_mx[idx], my = s->infl_my[idx],
                     mz = s->infl_mz[idx];
        w0 += ug * (1.0 + vt * mx * mx);
        w1 += ug * (1.0 + vt * my * my);
        w2 += ug * (1.0 + vt * mz * mz);
        w3 += ug * (vt * mx * my);
        w4 += ug * (vt * mx * mz);
        w5 += ug * (vt * my * mz);
        s->grid[2 * idx] = h * re;
        s->grid[2 * idx + 1] = h * im;
    }
    const double escale = ORC_QQR2E / (2.0 * ORC_PI * vol);
    s->e_recip += e * escale;
    s->vir[0] += w0 * escale;
    s->vir[1] += w1 * escale;
    s->vir[2] += w2 * escale;
    s->vir[3] += w3 * escale;
    s->vir[4] += w4 * escale;
    s->vir[5] += w5 * escale;
    orc_fft3d(K0, K1, K2, s->grid, +1);
    /* pme_influence.h:217-280 */
    const double fscale = ORC_QQR2E / (ORC_PI * vol);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const double qi = s->q[i];
        if (qi == 0.0)
            continue;
        const double* thx = &th[(3 * i + 0) * order];
        const double* thy = &th[(3 * i + 1) * order];
        const double* thz = &th[(3 * i + 2) * order];
        const double* dthx = &dth[(3 * i + 0) * order];
        const double* dthy = &dth[(3 * i + 1) * order];
        const double* dthz = &dth[(3 * i + 2) * order];
        const int b0 = base[3 * i + 0] - nm1;
        const int b1 = base[3 * i + 1] - nm1;
        const int b2 = base[3 * i + 2] - nm1;
        double g[3] = {0, 0, 0};
        for (int a = 0; a < order; ++a) {
            const int g0 = pme_wrap(b0 + a, K0);
            for (int b = 0; b < order; ++b) {
                const int g1 = pme_wrap(b1 + b, K1);
                const long plane = (long)K2 * (g1 + (long)K1 * g0);
                for (int c = 0; c < order; ++c) {
                    const int g2 = pme_wrap(b2 + c, K2);
                    const double cv = s->grid[2 * (plane + g2)];
                    g[0] += cv * dthx[a] * thy[b] * thz[c];
                    g[1] += cv * thx[a] * dthy[b] * thz[c];
                    g[2] += cv * thx[a] * thy[b] * dthz[c];
                }
            }
        }
        /* orthorhombic inv_cell: only the diagonal contributes */
        s->fx[i] += -fscale * qi * (g[0] * s->K[0] * ic[0]);
        s->fy[i] += -fscale * qi * (g[1] * s->K[1] * ic[1]);
        s->fz[i] += -fscale * qi * (g[2] * s->K[2] * ic[2]);
    }
    double qsq = 0, qt = 0;
    for (int i = 0; i < n; ++i) {
        qsq += s->q[i] * s->q[i];
        qt += s->q[i];
    }
    const double alpha = s->d.pme_alpha;
    const double e_self = -ORC_QQR2E * alpha / sqrt(ORC_PI) * qsq;
    const double e_net =
        -ORC_QQR2E * ORC_PI / (2.0 * vol * alpha * alpha) * qt * qt;
    s->e_const += e_self + e_net;
    free(base);
    free(th);
    free(dth);
}

void orc_pme(int n, const double* x, const double* y, const double* z,
             const double* q, const double L[3], double alpha, const int K[3],
             int order, double* energy, double* fx, double* fy, double* fz,
             double* virial) {
    orc_desc d;
    memset(&d, 0, sizeof(d));
    d.n = n;
    for (int k = 0; k < 3; ++k) {
        d.L[k] = L[k];
        d.pme_K[k] = K[k];
    }
    d.has_pme = 1;
    d.pme_alpha = alpha;
    d.pme_order = order;
    orc_sys* s = orc_create(&d);
    orc_set_state(s, x, y, z, NULL, NULL, NULL, NULL, NULL, NULL, NULL, q,
                  NULL);
    pme_forces(s);
    *energy = s->e_recip + s->e_const;
    for (int i = 0; i < n; ++i) {
        fx[i] = s->fx[i];
        fy[i] = s->fy[i];
        fz[i] = s->fz[i];
    }
    for (int k = 0; k < 6; ++k)
        virial[k] = s->vir[k];
    orc_destroy(s);
}

/* ewald_sum.h:58-140 (positive hemisphere, prefactor 4*pi/V) */
void orc_ewald_recip(int n, const double* x, const double* y, const double* z,
                     const double* q, const double L[3], double alpha,
                     double accuracy, double* energy, double* fx, double* fy,
                     double* fz, double* virial) {
    const double tp = 2.0 * ORC_PI;
    const double b[3] = {tp / L[0], tp / L[1], tp / L[2]};
    const double gcut = 2.0 * alpha * sqrt(-log(accuracy));
    const double gcut2 = gcut * gcut;
    int kmax[3];
    for (int i = 0; i < 3; ++i) {
        kmax[i] = (int)ceil(gcut / b[i]);
        if (kmax[i] < 1)
            kmax[i] = 1;
    }
    const double vol = L[0] * L[1] * L[2];
    const double inv4a2 = 1.0 / (4.0 * alpha * alpha);
    const double pref = ORC_QQR2E * 4.0 * ORC_PI / vol;
    double e = 0, w[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < n; ++i)
        fx[i] = fy[i] = fz[i] = 0.0;
    for (int mx = -kmax[0]; mx <= kmax[0]; ++mx)
        for (int my = -kmax[1]; my <= kmax[1]; ++my)
            for (int mz = -kmax[2]; mz <= kmax[2]; ++mz) {
                if (mx == 0 && my == 0 && mz == 0)
                    continue;
                if (mz < 0)
                    continue;
                if (mz == 0 && my < 0)
                    continue;
                if (mz == 0 && my == 0 && mx < 0)
                    continue;
                const double gx = mx * b[0], gy = my * b[1], gz = mz * b[2];
                const double g2 = gx * gx + gy * gy + gz * gz;
                if (g2 > gcut2)
                    continue;
                const double kw = exp(-g2 * inv4a2) / g2;
                const double kv = -2.0 * (1.0 / g2 + inv4a2);
                double sr = 0, si = 0;
                for (int i = 0; i < n; ++i) {
                    const double th = gx * x[i] + gy * y[i] + gz * z[i];
                    sr += q[i] * cos(th);
                    si += q[i] * sin(th);
                }
                const double s2 = sr * sr + si * si;
                e += kw * s2;
                w[0] += kw * s2 * (1.0 + kv * gx * gx);
                w[1] += kw * s2 * (1.0 + kv * gy * gy);
                w[2] += kw * s2 * (1.0 + kv * gz * gz);
                w[3] += kw * s2 * (kv * gx * gy);
                w[4] += kw * s2 * (kv * gx * gz);
                w[5] += kw * s2 * (kv * gy * gz);
                for (int i = 0; i < n; ++i) {
                    const double th = gx * x[i] + gy * y[i] + gz * z[i];
                    const double im = sr * sin(th) - si * cos(th);
                    const double f = 2.0 * pref * kw * q[i] * im;
                    fx[i] += f * gx;
                    fy[i] += f * gy;
                    fz[i] += f * gz;
                }
            }
    double qsq = 0, qt = 0;
    for (int i = 0; i < n; ++i) {
        qsq += q[i] * q[i];
        qt += q[i];
    }
    *energy = pref * e - ORC_QQR2E * alpha / sqrt(ORC_PI) * qsq -
              ORC_QQR2E * ORC_PI / (2.0 * vol * alpha * alpha) * qt * qt;
    for (int k = 0; k < 6; ++k)
        virial[k] = pref * w[k];
}

/* ------------------------------------------------------------------ */
/* integrators and thermostats                                         */
/* ------------------------------------------------------------------ */

/* the test-only harmonic wall (orc_desc.wall_*) */
static void wall_forces(orc_sys* s) {
    double* c = s->d.wall_axis == 0 ? s->x : s->d.wall_axis == 1 ? s->y : s->z;
    double* f = s->d.wall_axis == 0 ? s->fx : s->d.wall_axis == 1 ? s->fy : s->fz;
    double e = 0.0;
    for (int i = 0; i < s->n; ++i) {
        const double d = c[i] - s->d.wall_pos;
        if (d > 0.0) {
            f[i] += -2.0 * s->d.wall_k * d;
            e += s->d.wall_k * d * d;
        }
    }
    s->e_ext = e;
}

void orc_compute_forces(orc_sys* s) {
    const int n = s->n;
    memset(s->fx, 0, sizeof(double) * (size_t)n);
    memset(s->fy, 0, sizeof(double) * (size_t)n);
    memset(s->fz, 0, sizeof(double) * (size_t)n);
    s->e_lj = s->e_coul = s->e_recip = s->e_const = s->e_ext = 0.0;
    for (int k = 0; k < 6; ++k)
        s->vir[k] = 0.0;
    if (s->d.has_lj || s->d.has_coul)
        pair_forces(s);
    if (s->d.has_pme)
        pme_forces(s);
    if (s->d.wall_axis >= 0 && s->d.wall_axis < 3)
        wall_forces(s);
}

/* init.cpp:29-45 */
static double kinetic(const orc_sys* s) {
    double ke = 0;
#pragma omp parallel for reduction(+ : ke) schedule(static)
    for (int i = 0; i < s->n; ++i)
        ke += s->m[i] *
              (s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i]);
    return 0.5 * ORC_MVV2E * ke;
}

/* nose_hoover.cpp:104-170 */
static void nose_hoover(orc_sys* s) {
    const double T = s->d.T;
    s->Q = (double)s->n_dof * ORC_KB * T * s->d.tau * s->d.tau;
    double ke = 0;
    for (int i = 0; i < s->n; ++i)
        ke += s->m[i] *
              (s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i]);
    ke *= 0.5 * ORC_MVV2E;
    s->xi += (s->d.dt * 0.5) * (2.0 * ke - (double)s->n_dof * ORC_KB * T) /
             s->Q;
    const double scale = exp(-s->d.dt * 0.5 * s->xi);
    for (int i = 0; i < s->n; ++i) {
        s->vx[i] *= scale;
        s->vy[i] *= scale;
        s->vz[i] *= scale;
    }
}

/* fix_langevin.cpp:37-62 GaussStream (splitmix64 + Box-Muller) */
typedef struct {
    uint64_t s;
    int has;
    double cached;
} gauss_stream;

static double gs_u01(gauss_stream* g) {
    g->s += 0x9E3779B97F4A7C15ULL;
    uint64_t z = g->s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

static double gs_next(gauss_stream* g) {
    if (g->has) {
        g->has = 0;
        return g->cached;
    }
    const double u = gs_u01(g);
    const double v = gs_u01(g);
    const double r = sqrt(-2.0 * log(u > 1e-300 ? u : 1e-300));
    const double th = 2.0 * ORC_PI * v;
    g->cached = r * sin(th);
    g->has = 1;
    return r * cos(th);
}

void orc_gauss3(uint32_t seed, int64_t step, int64_t tag, double* out3) {
    const uint64_t base = (uint64_t)seed * 0x9E3779B97F4A7C15ULL +
                          (uint64_t)step * 0xBF58476D1CE4E5B9ULL;
    gauss_stream g = {base + (uint64_t)tag * 0xD6E8FEB86659FD93ULL, 0, 0.0};
    out3[0] = gs_next(&g);
    out3[1] = gs_next(&g);
    out3[2] = gs_next(&g);
}

/* fix_langevin.cpp:79-155; the setpoint follows the linear ramp of
 * :94-104, delta = (step - nfirst) / (nlast - nfirst) clamped to [0, 1] */
static void langevin(orc_sys* s) {
    double T = s->d.T;
    if (s->d.lang_nlast > s->d.lang_nfirst) {
        double delta = (double)(s->step - s->d.lang_nfirst) /
                       (double)(s->d.lang_nlast - s->d.lang_nfirst);
        delta = delta < 0.0 ? 0.0 : (delta > 1.0 ? 1.0 : delta);
        T = s->d.T + delta * (s->d.T_stop - s->d.T);
    }
    const double inv_damp_ftm2v = 1.0 / (s->d.damp * ORC_FTM2V);
    const double g2pre =
        sqrt(2.0 * ORC_KB * T / (s->d.damp * s->d.dt * ORC_MVV2E)) /
        ORC_FTM2V;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; ++i) {
        double r[3];
        orc_gauss3(s->d.seed, s->step, s->tag[i], r);
        const double m = s->m[i];
        const double g1 = -m * inv_damp_ftm2v;
        const double g2 = g2pre * sqrt(m);
        s->fx[i] += g1 * s->vx[i] + g2 * r[0];
        s->fy[i] += g1 * s->vy[i] + g2 * r[1];
        s->fz[i] += g1 * s->vz[i] + g2 * r[2];
    }
}

/* ------------------------------------------------------------------ */
/* MTK NPT (src/cpu/dynamics/nose_hoover_npt.cpp)                      */
/* ------------------------------------------------------------------ */

/* |eps_dot dt| clamp of the box update (nose_hoover_npt.cpp:44) */
#define ORC_EPS_DT_MAX 0.005

/* (e^{2x} - 1) / (2x) with the Taylor branch near 0 (nose_hoover_npt.cpp:66-73) */
static double npt_expm1c(double x) {
    if (fabs(x) < 1e-6)
        return 1.0 + x + (2.0 / 3.0) * x * x;
    return expm1(2.0 * x) / (2.0 * x);
}

/* build(): chain, barostat masses, drag factors, equipartition KE
 * (nose_hoover_npt.cpp:87-172) */
int orc_set_npt(orc_sys* s, const orc_npt* p) {
    if (p->mtchain < 1 || p->mtchain > ORC_MAXCHAIN || p->mpchain < 1 ||
        p->mpchain > ORC_MAXCHAIN || !(p->tau_T > 0.0) || !(p->tau_P > 0.0) ||
        !(p->T_start > 0.0))
        return -1;
    s->np = *p;
    if (s->np.T_stop < 0.0)
        s->np.T_stop = s->np.T_start;
    s->npt_on = 1;
    s->d.thermostat = ORC_THERMO_NPT;
    s->d.need_virial = 1;
    s->pdim = (p->couple[0] ? 1 : 0) + (p->couple[1] ? 1 : 0) + (p->couple[2] ? 1 : 0);
    s->T_live = s->np.T_start;
    s->kT = ORC_KB * s->np.T_start;
    const double tT2 = p->tau_T * p->tau_T, tP2 = p->tau_P * p->tau_P;
    for (int k = 0; k < ORC_MAXCHAIN; ++k) {
        s->Qt[k] = s->kT * tT2;
        s->Qb[k] = s->kT * tP2;
        s->eta_t[k] = s->eta_t_dot[k] = s->eta_b[k] = s->eta_b_dot[k] = 0.0;
    }
    s->Qt[0] = (double)s->n_dof * s->kT * tT2;
    s->W = ((double)s->n_dof + 3.0) * s->kT * tP2;
    s->tdrag = 1.0 - p->drag * s->d.dt / p->tau_T;
    s->pdrag = 1.0 - p->drag * s->d.dt / p->tau_P;
    s->eps_dot[0] = s->eps_dot[1] = s->eps_dot[2] = 0.0;
    s->KE_global = 0.5 * (double)s->n_dof * s->kT;
    s->conserved = 0.0;
    return 0;
}

void orc_npt_state(const orc_sys* s, double* out) {
    out[0] = s->d.L[0];
    out[1] = s->d.L[1];
    out[2] = s->d.L[2];
    out[3] = s->conserved;
    out[4] = s->eps_dot[0];
    out[5] = s->eps_dot[1];
    out[6] = s->eps_dot[2];
    out[7] = s->eta_t[0];
    out[8] = s->eta_t_dot[0];
    out[9] = s->eta_b[0];
    out[10] = s->eta_b_dot[0];
    out[11] = s->T_live;
    out[12] = s->KE_global;
}

/* compute_temp_target (nose_hoover_npt.cpp:192-203) */
static void npt_temp_target(orc_sys* s, int64_t step) {
    double delta = 0.0;
    if (s->np.nlast > s->np.nfirst) {
        delta = (double)(step - s->np.nfirst) / (double)(s->np.nlast - s->np.nfirst);
        delta = delta < 0.0 ? 0.0 : (delta > 1.0 ? 1.0 : delta);
    }
    s->T_live = s->np.T_start + delta * (s->np.T_stop - s->np.T_start);
    s->kT = ORC_KB * s->T_live;
}

static double npt_ke(const orc_sys* s) { return kinetic(s); }

/* compute_axis_KE (nose_hoover_npt.cpp:236-265) */
static void npt_axis_ke(const orc_sys* s, double ke[3]) {
    double kx = 0, ky = 0, kz = 0;
#pragma omp parallel for reduction(+ : kx, ky, kz) schedule(static)
    for (int i = 0; i < s->n; ++i) {
        const double m = s->m[i];
        kx += m * s->vx[i] * s->vx[i];
        ky += m * s->vy[i] * s->vy[i];
        kz += m * s->vz[i] * s->vz[i];
    }
    ke[0] = 0.5 * ORC_MVV2E * kx;
    ke[1] = 0.5 * ORC_MVV2E * ky;
    ke[2] = 0.5 * ORC_MVV2E * kz;
}

static void npt_scale_v(orc_sys* s, double sx, double sy, double sz) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; ++i) {
        s->vx[i] *= sx;
        s->vy[i] *= sy;
        s->vz[i] *= sz;
    }
}

/* nhc_atoms_half (nose_hoover_npt.cpp:267-340): backward sweep with drag at
 * every link, velocity scale, chain positions, forward sweep without drag */
static void npt_nhc_atoms(orc_sys* s, double hdt) {
    const double qdt = 0.5 * hdt, edt = 0.5 * qdt;
    const int M = s->np.mtchain;
    for (int pass = 0; pass < 2; ++pass) {
        for (int j = 0; j < M; ++j) {
            const int k = pass == 0 ? M - 1 - j : j;
            const double expfac = k < M - 1 ? exp(-s->eta_t_dot[k + 1] * edt) : 1.0;
            const double G = k == 0 ? (2.0 * s->KE_global - s->n_dof * s->kT) / s->Qt[0]
                                    : (s->Qt[k - 1] * s->eta_t_dot[k - 1] * s->eta_t_dot[k - 1] - s->kT) /
                                          s->Qt[k];
            s->eta_t_dot[k] *= expfac;
            s->eta_t_dot[k] += G * qdt;
            if (pass == 0)
                s->eta_t_dot[k] *= s->tdrag;
            s->eta_t_dot[k] *= expfac;
        }
        if (pass == 0) {
            const double sc = exp(-s->eta_t_dot[0] * hdt);
            npt_scale_v(s, sc, sc, sc);
            s->KE_global *= sc * sc;
            for (int k = 0; k < M; ++k)
                s->eta_t[k] += s->eta_t_dot[k] * hdt;
        }
    }
}

/* nhc_baro_half (nose_hoover_npt.cpp:347-420) */
static void npt_nhc_baro(orc_sys* s, double hdt) {
    const double qdt = 0.5 * hdt, edt = 0.5 * qdt;
    const int M = s->np.mpchain;
    const double Wa = s->W / 3.0;
    for (int pass = 0; pass < 2; ++pass) {
        for (int j = 0; j < M; ++j) {
            const int k = pass == 0 ? M - 1 - j : j;
            const double expfac = k < M - 1 ? exp(-s->eta_b_dot[k + 1] * edt) : 1.0;
            double G;
            if (k == 0) {
                double ke2 = 0.0;
                for (int a = 0; a < 3; ++a)
                    if (s->np.couple[a])
                        ke2 += Wa * s->eps_dot[a] * s->eps_dot[a];
                G = (ke2 - s->kT) / s->Qb[0];
            } else {
                G = (s->Qb[k - 1] * s->eta_b_dot[k - 1] * s->eta_b_dot[k - 1] - s->kT) / s->Qb[k];
            }
            s->eta_b_dot[k] *= expfac;
            s->eta_b_dot[k] += G * qdt;
            if (pass == 0)
                s->eta_b_dot[k] *= s->pdrag;
            s->eta_b_dot[k] *= expfac;
        }
        if (pass == 0) {
            const double bs = exp(-s->eta_b_dot[0] * hdt);
            for (int a = 0; a < 3; ++a)
                if (s->np.couple[a])
                    s->eps_dot[a] *= bs;
            for (int k = 0; k < M; ++k)
                s->eta_b[k] += s->eta_b_dot[k] * hdt;
        }
    }
}

/* update_eps_dot (nose_hoover_npt.cpp:422-560) with the isotropic couple()
 * average when all three axes are barostatted */
static void npt_update_eps(orc_sys* s, double hdt) {
    const double V = s->d.L[0] * s->d.L[1] * s->d.L[2];
    if (V <= 0.0)
        return;
    double ke[3];
    npt_axis_ke(s, ke);
    double diag[3] = {s->vir[0] + 2.0 * ke[0], s->vir[1] + 2.0 * ke[1],
                      s->vir[2] + 2.0 * ke[2]};
    if (s->pdim == 3) {
        const double ave = (1.0 / 3.0) * (diag[0] + diag[1] + diag[2]);
        diag[0] = diag[1] = diag[2] = ave;
    }
    double mtk_ke = 0.0;
    for (int a = 0; a < 3; ++a)
        if (s->np.couple[a])
            mtk_ke += ke[a];
    const int n_atoms = (s->n_dof + 3) / 3;
    const double mtk = s->pdim > 0 ? 6.0 * mtk_ke / ((double)s->pdim * n_atoms) : 0.0;
    for (int a = 0; a < 3; ++a) {
        if (!s->np.couple[a])
            continue;
        const double Pa = diag[a] / V;
        const double G = (3.0 * V * (Pa - s->np.P_target) + mtk) / s->W;
        s->eps_dot[a] += G * hdt;
    }
}

/* scale_v_by_baro (nose_hoover_npt.cpp:580-630) */
static void npt_scale_baro(orc_sys* s, double hdt) {
    double sum = 0.0;
    for (int a = 0; a < 3; ++a)
        if (s->np.couple[a])
            sum += s->eps_dot[a];
    const int n_atoms = (s->n_dof + 3) / 3;
    const double mtk2 = s->pdim > 0 ? sum / ((double)s->pdim * n_atoms) : 0.0;
    const double sx = exp(-(s->eps_dot[0] + mtk2) * hdt);
    const double sy = exp(-(s->eps_dot[1] + mtk2) * hdt);
    const double sz = exp(-(s->eps_dot[2] + mtk2) * hdt);
    npt_scale_v(s, sx, sy, sz);
    if (sx == sy && sy == sz)
        s->KE_global *= sx * sx;
    else
        s->KE_global = npt_ke(s);
}

static void npt_kick(orc_sys* s) {
    const double dtf = 0.5 * s->d.dt * ORC_FTM2V;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; ++i) {
        const double dtfm = dtf / s->m[i];
        s->vx[i] += dtfm * s->fx[i];
        s->vy[i] += dtfm * s->fy[i];
        s->vz[i] += dtfm * s->fz[i];
    }
}

/* propagate_x_and_box (nose_hoover_npt.cpp:650-760): closed-form drift,
 * box scaled per axis, wrap */
static void npt_propagate(orc_sys* s) {
    const double dt = s->d.dt;
    double a[3], dr[3];
    for (int d = 0; d < 3; ++d) {
        double e = s->eps_dot[d] * dt;
        e = e < -ORC_EPS_DT_MAX ? -ORC_EPS_DT_MAX : (e > ORC_EPS_DT_MAX ? ORC_EPS_DT_MAX : e);
        a[d] = exp(e);
        dr[d] = npt_expm1c(e * 0.5);
    }
    for (int d = 0; d < 3; ++d)
        s->d.L[d] *= a[d];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; ++i) {
        s->x[i] = wrap_coord(s->x[i] * a[0] + s->vx[i] * dt * dr[0], s->d.L[0]);
        s->y[i] = wrap_coord(s->y[i] * a[1] + s->vy[i] * dt * dr[1], s->d.L[1]);
        s->z[i] = wrap_coord(s->z[i] * a[2] + s->vz[i] * dt * dr[2], s->d.L[2]);
    }
}

/* extended_hamiltonian (nose_hoover_npt.cpp:770-805) */
static double npt_hamiltonian(const orc_sys* s) {
    double H = s->ke + (s->e_lj + s->e_coul + s->e_recip + s->e_const + s->e_ext);
    const double Wa = s->W / 3.0;
    for (int a = 0; a < 3; ++a)
        if (s->np.couple[a])
            H += 0.5 * Wa * s->eps_dot[a] * s->eps_dot[a];
    for (int k = 0; k < s->np.mtchain; ++k)
        H += 0.5 * s->Qt[k] * s->eta_t_dot[k] * s->eta_t_dot[k];
    for (int k = 0; k < s->np.mpchain; ++k)
        H += 0.5 * s->Qb[k] * s->eta_b_dot[k] * s->eta_b_dot[k];
    H += (double)s->n_dof * s->kT * s->eta_t[0];
    for (int k = 1; k < s->np.mtchain; ++k)
        H += s->kT * s->eta_t[k];
    for (int k = 0; k < s->np.mpchain; ++k)
        H += s->kT * s->eta_b[k];
    H += s->np.P_target * s->d.L[0] * s->d.L[1] * s->d.L[2];
    return H;
}

/* One MTK step (nose_hoover_npt.cpp:812-885 launch: P1-P6 at
 * initial_integrate, P7 at final_integrate, P8-P11 at end_of_step).  The
 * list is rebuilt every step: the cell changes every step. */
static void npt_step(orc_sys* s) {
    const double hdt = 0.5 * s->d.dt;
    npt_temp_target(s, s->step);
    const double tT2 = s->np.tau_T * s->np.tau_T;
    s->Qt[0] = (double)s->n_dof * s->kT * tT2;
    for (int k = 1; k < s->np.mtchain; ++k)
        s->Qt[k] = s->kT * tT2;
    npt_nhc_baro(s, hdt);   /* P1 */
    npt_nhc_atoms(s, hdt);  /* P2 */
    npt_update_eps(s, hdt); /* P3: the virial of the last force evaluation */
    npt_scale_baro(s, hdt); /* P4 */
    npt_kick(s);            /* P5 */
    npt_propagate(s);       /* P6 */
    orc_build_list(s);
    ++s->rebuilds;
    orc_compute_forces(s);
    npt_kick(s); /* P7 */
    s->KE_global = npt_ke(s);
    npt_scale_baro(s, hdt); /* P8 */
    npt_update_eps(s, hdt); /* P9 */
    npt_nhc_atoms(s, hdt);  /* P10 */
    npt_nhc_baro(s, hdt);   /* P11 */
    s->ke = s->KE_global;
    s->conserved = npt_hamiltonian(s);
}

/* Berendsen barostat at end_of_step (barostat.cpp:27-110): scalar pressure
 * P = (W_xx + W_yy + W_zz + 2 KE) / (3 V), dilation
 * mu = cbrt(clamp(1 - dt / (tau_P beta) (P_target - P), 0.5, 2)), cell and
 * positions scaled by mu. */
static void berendsen(orc_sys* s) {
    const double V = s->d.L[0] * s->d.L[1] * s->d.L[2];
    if (V <= 0.0)
        return;
    const double P = (s->vir[0] + s->vir[1] + s->vir[2] + 2.0 * s->ke) / (3.0 * V);
    double mu3 = 1.0 - (s->d.dt / (s->baro_tau * s->baro_bulk)) * (s->baro_P - P);
    mu3 = mu3 < 0.5 ? 0.5 : (mu3 > 2.0 ? 2.0 : mu3);
    const double mu = cbrt(mu3);
    for (int d = 0; d < 3; ++d)
        s->d.L[d] *= mu;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; ++i) {
        s->x[i] *= mu;
        s->y[i] *= mu;
        s->z[i] *= mu;
    }
}

/* NVELimit (nve_limit.cu:20-30, LAMMPS fix nve/limit): after a half kick a
 * speed above xmax / dt is scaled back to it. */
static inline void speed_cap(const orc_sys* s, int i) {
    if (!(s->vmax > 0.0))
        return;
    const double vsq = s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i];
    if (vsq > s->vmax * s->vmax) {
        const double f = s->vmax / sqrt(vsq);
        s->vx[i] *= f;
        s->vy[i] *= f;
        s->vz[i] *= f;
    }
}

/* Deform (deform.cu:55-95, initial_integrate +200): the k-th step takes the
 * axis edge from L0 (1 + r dt (k-1)) to L0 (1 + r dt k) and scales positions
 * along the axis by the ratio. */
static void deform(orc_sys* s) {
    s->def_count += 1;
    const double rdt = s->def_rate * s->d.dt;
    const double Lp = s->def_L0 * (1.0 + rdt * (double)(s->def_count - 1));
    const double Lc = s->def_L0 * (1.0 + rdt * (double)s->def_count);
    const double f = Lc / Lp;
    double* p = s->def_axis == 0 ? s->x : (s->def_axis == 1 ? s->y : s->z);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; ++i)
        p[i] *= f;
    s->d.L[s->def_axis] *= f;
}

int orc_set_nve_limit(orc_sys* s, double xmax) {
    if (!(xmax > 0.0))
        return -1;
    s->vmax = xmax / s->d.dt;
    return 0;
}

int orc_set_deform(orc_sys* s, int axis, double rate) {
    if (axis < 0 || axis > 2)
        return -1;
    s->def_axis = axis;
    s->def_rate = rate;
    s->def_L0 = s->d.L[axis];
    s->def_count = 0;
    return 0;
}

int orc_set_barostat(orc_sys* s, double P_target, double tau_P, double bulk_modulus) {
    if (!(tau_P > 0.0) || !(bulk_modulus > 0.0) || s->npt_on)
        return -1;
    s->baro_on = 1;
    s->baro_P = P_target;
    s->baro_tau = tau_P;
    s->baro_bulk = bulk_modulus;
    s->d.need_virial = 1;
    return 0;
}

/* runtime.cpp:452-501 step order with VelocityVerlet (velocity_verlet.cpp)
 * at order 0 and the thermostat at +100 in both integrate phases. */
int orc_run(orc_sys* s, int n_steps, double* hist) {
    const int n = s->n;
    const double dt = s->d.dt;
    const double dtf = 0.5 * dt * ORC_FTM2V;
    int rebuilds = 0;
    if (s->npairs == 0 && s->nbr == NULL)
        orc_build_list(s);
    if (s->npt_on) {
        for (int st = 0; st < n_steps; ++st) {
            npt_step(s);
            ++rebuilds;
            if (hist) {
                hist[2 * st] = s->e_lj + s->e_coul + s->e_recip + s->e_const + s->e_ext;
                hist[2 * st + 1] = s->ke;
            }
            s->step++;
        }
        return rebuilds;
    }
    for (int st = 0; st < n_steps; ++st) {
        /* initial_integrate */
        const double L0 = s->d.L[0], L1 = s->d.L[1], L2 = s->d.L[2];
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            const double dtfm = dtf / s->m[i];
            s->vx[i] += dtfm * s->fx[i];
            s->vy[i] += dtfm * s->fy[i];
            s->vz[i] += dtfm * s->fz[i];
            speed_cap(s, i);
            s->x[i] += dt * s->vx[i];
            s->y[i] += dt * s->vy[i];
            s->z[i] += dt * s->vz[i];
            s->x[i] = wrap_coord(s->x[i], L0);
            s->y[i] = wrap_coord(s->y[i], L1);
            s->z[i] = wrap_coord(s->z[i], L2);
        }
        if (s->d.thermostat == ORC_THERMO_NH)
            nose_hoover(s);
        if (s->def_axis >= 0)
            deform(s);
        /* neighbor decide (neighbor_list.h:128-141) */
        s->ago++;
        const int every = s->d.nl_every < 1 ? 1 : s->d.nl_every;
        const int delay = s->d.nl_delay < 0 ? 0 : s->d.nl_delay;
        /* the cell changes every step under the barostat: rebuild every step */
        if (s->baro_on || s->def_axis >= 0 || (s->ago >= delay && (s->ago % every) == 0 &&
                           (!s->d.nl_check || needs_rebuild(s)))) {
            orc_build_list(s);
            ++rebuilds;
            ++s->rebuilds;
        }
        /* pre_force + force */
        orc_compute_forces(s);
        /* post_force */
        if (s->d.thermostat == ORC_THERMO_LANGEVIN)
            langevin(s);
        /* final_integrate */
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            const double dtfm = dtf / s->m[i];
            s->vx[i] += dtfm * s->fx[i];
            s->vy[i] += dtfm * s->fy[i];
            s->vz[i] += dtfm * s->fz[i];
            speed_cap(s, i);
        }
        if (s->d.thermostat == ORC_THERMO_NH)
            nose_hoover(s);
        /* end_of_step */
        s->ke = kinetic(s);
        if (s->baro_on)
            berendsen(s);
        if (hist) {
            hist[2 * st] = s->e_lj + s->e_coul + s->e_recip + s->e_const + s->e_ext;
            hist[2 * st + 1] = s->ke;
        }
        s->step++;
    }
    return rebuilds;
}
