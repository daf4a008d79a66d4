/*
 * sph_oracle.c — CPU ORACLE, TEST INFRASTRUCTURE ONLY.
 *
 * A serial FP64 restatement, in plain C, of the reference's step for this
 * path (cwang2015/sources, the `nthreads == 1`, `nnps == 1` branch):
 *   pair search    direct_find      m_particles.f90:938-1001
 *                  direct_find_2    m_particles.f90:1004-1062
 *   kernel         kernel           m_particles.f90:1469-1602
 *   physics        m_particles.f90:1605-1642, 1711-1991, 1996-2037,
 *                  2105-2500, 2504-2564, 2658-2695, 2761-2793, 2855-2932,
 *                  3047-3119, 3323-3505, 3700-3762, 3832-3988
 *   step drivers   declarations_sph.f90:1131-1435, 1439-1526, 1530-1655
 *   integrators    declarations_sph.f90:525-791, 794-886, 978-1127
 * Pair loops run in the reference's pair-list order and scatter to both ends
 * exactly as the Fortran does; single-precision literals inside the FP64 code
 * are reproduced with F32() (e.g. `2./3.`, `pi`, `0.000005`).
 *
 * PARITY UNPINNED: the reference ships no tests, fixtures or golden vectors
 * for this path and cannot be compiled here (no Fortran compiler; missing
 * modules `constants`/`declarations`).  The restatement is pinned instead by
 * known-answer checks in tests/ (kernel normalisation, finite-difference
 * gradients, partition of unity, momentum conservation, DP return, pair set
 * against brute force), and by a second restatement in numpy, written
 * separately from the same Fortran, that agrees with this one bit for bit on
 * the three right-hand sides and integrators (tests/test_oracle_numpy.py).
 *
 * Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
 * use this file, as the checker.  The product (libsphg) never links it.
 *
 * Build: oracle/build_oracle.sh (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "../include/sphg.h"

#define F32(v) ((double)(float)(v))
/* m_particles.f90:1483: pi is a double parameter set from a default-real
 * literal, so it carries single precision. */
static const double PI_REF = (double)3.14159265358979323846f;

/* ------------------------------------------------------------------ */
typedef struct {
    int ntotal, nvirt, n, material;
    double dspp;
    double *x, *vx, *dvx, *av, *v_min;                 /* 2n */
    double *rho, *rho_min, *drho, *p, *c, *mass, *hsml;
    double *vof, *vof_min, *dvof, *vof2;
    double *sxx, *sxy, *syy, *dsxx, *dsxy, *dsyy, *dp;
    double *sxx_min, *sxy_min, *syy_min, *p_min;
    double *epsilon_p, *vcc;
    double *txx, *tyy, *txy, *wxy;                     /* aliases, see below */
    int *itype, *fail, nfail;
    int *countiac;
    int64_t niac;
} or_phase;

typedef struct {
    sphg_params prm;
    int nphase;
    or_phase ph[2];
    int maxn;
    /* shared working arrays, declarations_sph.f90:52,368-377,414-415 */
    double *wtxx, *wtyy, *wtxy;
    /* the pair arrays (soil shares water's, declarations_sph.f90:403-406) */
    int64_t cap;
    int *pair_i, *pair_j;
    double *w, *dwdx;            /* dwdx(2,cap) */
    int64_t niac;
    /* copies of each list of the last step, for export */
    int *save_i[3], *save_j[3];
    int64_t save_n[3];
    int search_mode;             /* 0: brute force; 1: cell list, same order */
    int status;
} or_ctx;

/* ------------------------------------------------------------------ */
/* get_scale_k, m_particles.f90:916-935 */
static int scale_k_of(int skf) {
    switch (skf) { case 1: return 2; case 2: return 3; case 3: return 3; case 4: return 2; }
    return -1;
}

static double ipow(double x, int n) {  /* Fortran integer power */
    double r = 1.0;
    for (int i = 0; i < n; ++i) r = r * x;
    return r;
}

/* kernel, m_particles.f90:1469-1602 (dim = 2). */
void or_kernel(int skf, double r, const double* dx, double hsml, double* w, double* dwdx) {
    double q = r / hsml, factor;
    *w = 0.0; dwdx[0] = 0.0; dwdx[1] = 0.0;
    if (skf == 1) {
        factor = 15.0 / (7.0 * PI_REF * hsml * hsml);
        if (q >= 0 && q <= 1.0) {
            *w = factor * (F32(2.0f / 3.0f) - q * q + ipow(q, 3) / 2.0);
            for (int d = 0; d < 2; ++d) dwdx[d] = factor * (-2.0 + 3.0 / 2.0 * q) / (hsml * hsml) * dx[d];
        } else if (q > 1.0 && q <= 2) {
            *w = factor * 1.0 / 6.0 * ipow(2.0 - q, 3);
            for (int d = 0; d < 2; ++d)
                dwdx[d] = -(factor * 1.0 / 6.0 * 3.0 * ipow(2.0 - q, 2) / hsml * (dx[d] / r));
        }
    } else if (skf == 2) {
        factor = 1.0 / ((hsml * hsml) * pow(PI_REF, 2 / 2.0));
        if (q >= 0 && q <= 3) {
            *w = factor * exp(-q * q);
            for (int d = 0; d < 2; ++d) dwdx[d] = *w * (-2.0 * dx[d] / hsml / hsml);
        }
    } else if (skf == 3) {
        factor = 7.0 / (478.0 * PI_REF * hsml * hsml);
        if (q >= 0 && q <= 1) {
            *w = factor * (ipow(3 - q, 5) - 6 * ipow(2 - q, 5) + 15 * ipow(1 - q, 5));
            for (int d = 0; d < 2; ++d)
                dwdx[d] = factor * ((-120 + 120 * q - 50 * ipow(q, 2)) / (hsml * hsml) * dx[d]);
        } else if (q > 1 && q <= 2) {
            *w = factor * (ipow(3 - q, 5) - 6 * ipow(2 - q, 5));
            for (int d = 0; d < 2; ++d)
                dwdx[d] = factor * (-5 * ipow(3 - q, 4) + 30 * ipow(2 - q, 4)) / hsml * (dx[d] / r);
        } else if (q > 2 && q <= 3) {
            *w = factor * ipow(3 - q, 5);
            for (int d = 0; d < 2; ++d) dwdx[d] = factor * (-5 * ipow(3 - q, 4)) / hsml * (dx[d] / r);
        }
    } else if (skf == 4) {
        factor = 7.0 / (4.0 * PI_REF * hsml * hsml);
        if (q >= 0 && q <= 2) {
            *w = factor * (ipow(1 - q / 2, 4) * (1 + 2 * q));
            for (int d = 0; d < 2; ++d)
                dwdx[d] = factor * (-5 + 15 * q / 2 - 15 * ipow(q, 2) / 4 + 5 * ipow(q, 3) / 8) / (hsml * hsml) * dx[d];
        }
    }
}

/* ------------------------------------------------------------------ */
static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }
static int* ialloc(size_t n) { return (int*)calloc(n ? n : 1, sizeof(int)); }

static int push_pair(or_ctx* C, int i, int j, const double* dxv, double r, double mhsml) {
    if (C->niac >= C->cap) { C->status = SPHG_ERR_PAIR_OVERFLOW; return -1; }
    int64_t k = C->niac++;
    C->pair_i[k] = i; C->pair_j[k] = j;
    double tdw[2];
    or_kernel(C->prm.skf, r, dxv, mhsml, &C->w[k], tdw);
    C->dwdx[2 * k] = tdw[0]; C->dwdx[2 * k + 1] = tdw[1];
    return 0;
}

/* --- cell list that visits candidates in direct_find order ------------ */
typedef struct { int ncx, ncy; double x0, y0, inv; int* start; int* idx; } or_grid;

static void grid_build(or_grid* g, const or_phase* P, double cell, const sphg_params* prm) {
    g->x0 = prm->x_min; g->y0 = prm->y_min; g->inv = 1.0 / cell;
    g->ncx = (int)ceil((prm->x_max - prm->x_min) * g->inv) + 1;
    g->ncy = (int)ceil((prm->y_max - prm->y_min) * g->inv) + 1;
    int nc = g->ncx * g->ncy;
    g->start = ialloc((size_t)nc + 1);
    g->idx = ialloc((size_t)P->n);
    int* cid = ialloc((size_t)P->n);
    for (int i = 0; i < P->n; ++i) {
        double fx = floor((P->x[2 * i] - g->x0) * g->inv), fy = floor((P->x[2 * i + 1] - g->y0) * g->inv);
        if (!(fx >= 0)) fx = 0; if (fx > g->ncx - 1) fx = g->ncx - 1;
        if (!(fy >= 0)) fy = 0; if (fy > g->ncy - 1) fy = g->ncy - 1;
        cid[i] = (int)fy * g->ncx + (int)fx;
        g->start[cid[i] + 1]++;
    }
    for (int c = 0; c < nc; ++c) g->start[c + 1] += g->start[c];
    int* fill = ialloc((size_t)nc);
    for (int i = 0; i < P->n; ++i) g->idx[g->start[cid[i]] + fill[cid[i]]++] = i;  /* ascending i per cell */
    free(fill); free(cid);
}
static void grid_free(or_grid* g) { free(g->start); free(g->idx); }

static int cmp_int(const void* a, const void* b) { int x = *(const int*)a, y = *(const int*)b; return (x > y) - (x < y); }

/* candidates of particle i (of phase owning g) around position (px,py) with
 * index > jmin, sorted ascending. */
static int grid_candidates(const or_grid* g, double px, double py, int jmin, int* out) {
    double fx = floor((px - g->x0) * g->inv), fy = floor((py - g->y0) * g->inv);
    if (!(fx >= 0)) fx = 0; if (fx > g->ncx - 1) fx = g->ncx - 1;
    if (!(fy >= 0)) fy = 0; if (fy > g->ncy - 1) fy = g->ncy - 1;
    int cx = (int)fx, cy = (int)fy, m = 0;
    for (int yy = cy - 1; yy <= cy + 1; ++yy) {
        if (yy < 0 || yy >= g->ncy) continue;
        int x0 = cx - 1 < 0 ? 0 : cx - 1, x1 = cx + 1 >= g->ncx ? g->ncx - 1 : cx + 1;
        for (int k = g->start[yy * g->ncx + x0]; k < g->start[yy * g->ncx + x1 + 1]; ++k)
            if (g->idx[k] > jmin) out[m++] = g->idx[k];
    }
    qsort(out, (size_t)m, sizeof(int), cmp_int);
    return m;
}

static double max_h(const or_phase* a, const or_phase* b) {
    double h = 0;
    for (int i = 0; i < a->n; ++i) if (a->hsml[i] > h) h = a->hsml[i];
    if (b) for (int i = 0; i < b->n; ++i) if (b->hsml[i] > h) h = b->hsml[i];
    return h;
}

/* direct_find, m_particles.f90:938-1001 (i < j, sqrt(r^2) < k*(hi+hj)/2) */
static int direct_find(or_ctx* C, or_phase* P) {
    int n = P->n, scale_k = scale_k_of(C->prm.skf);
    if (scale_k < 0) { C->status = SPHG_ERR_BAD_KERNEL; return -1; }
    for (int i = 0; i < n; ++i) P->countiac[i] = 0;
    C->niac = 0;
    or_grid g; int* cand = NULL;
    if (C->search_mode == 1) {
        grid_build(&g, P, scale_k * max_h(P, NULL) * (1.0 + 1e-6), &C->prm);
        cand = ialloc((size_t)n);
    }
    for (int i = 0; i < n - 1; ++i) {
        int m = n - 1 - i, *list = NULL;
        if (C->search_mode == 1) { m = grid_candidates(&g, P->x[2 * i], P->x[2 * i + 1], i, cand); list = cand; }
        for (int t = 0; t < m; ++t) {
            int j = list ? list[t] : i + 1 + t;
            double dxv[2];
            dxv[0] = P->x[2 * i] - P->x[2 * j];
            double driac = dxv[0] * dxv[0];
            dxv[1] = P->x[2 * i + 1] - P->x[2 * j + 1];
            driac = driac + dxv[1] * dxv[1];
            double mhsml = (P->hsml[i] + P->hsml[j]) / 2.0;
            if (sqrt(driac) < scale_k * mhsml) {
                if (push_pair(C, i, j, dxv, sqrt(driac), mhsml)) goto out;
                P->countiac[i]++; P->countiac[j]++;
            }
        }
    }
out:
    if (C->search_mode == 1) { grid_free(&g); free(cand); }
    P->niac = C->niac;
    return C->status ? -1 : 0;
}

/* direct_find_2, m_particles.f90:1004-1062: water i x soil j, r = 0 kept */
static int direct_find_2(or_ctx* C, or_phase* W, or_phase* S) {
    int scale_k = scale_k_of(C->prm.skf);
    if (scale_k < 0) { C->status = SPHG_ERR_BAD_KERNEL; return -1; }
    for (int i = 0; i < W->n; ++i) W->countiac[i] = 0;
    for (int j = 0; j < S->n; ++j) S->countiac[j] = 0;
    C->niac = 0;
    or_grid g; int* cand = NULL;
    if (C->search_mode == 1) {
        grid_build(&g, S, scale_k * max_h(W, S) * (1.0 + 1e-6), &C->prm);
        cand = ialloc((size_t)S->n);
    }
    for (int i = 0; i < W->n; ++i) {
        int m = S->n, *list = NULL;
        if (C->search_mode == 1) { m = grid_candidates(&g, W->x[2 * i], W->x[2 * i + 1], -1, cand); list = cand; }
        for (int t = 0; t < m; ++t) {
            int j = list ? list[t] : t;
            double dxv[2];
            dxv[0] = W->x[2 * i] - S->x[2 * j];
            double driac = dxv[0] * dxv[0];
            dxv[1] = W->x[2 * i + 1] - S->x[2 * j + 1];
            driac = driac + dxv[1] * dxv[1];
            double mhsml = (W->hsml[i] + S->hsml[j]) / 2.0;
            if (sqrt(driac) < scale_k * mhsml) {
                if (push_pair(C, i, j, dxv, sqrt(driac), mhsml)) goto out;
                W->countiac[i]++; S->countiac[j]++;
            }
        }
    }
out:
    if (C->search_mode == 1) { grid_free(&g); free(cand); }
    W->niac = C->niac;
    return C->status ? -1 : 0;
}

static void save_pairs(or_ctx* C, int which) {
    free(C->save_i[which]); free(C->save_j[which]);
    C->save_i[which] = ialloc((size_t)C->niac);
    C->save_j[which] = ialloc((size_t)C->niac);
    memcpy(C->save_i[which], C->pair_i, sizeof(int) * (size_t)C->niac);
    memcpy(C->save_j[which], C->pair_j, sizeof(int) * (size_t)C->niac);
    C->save_n[which] = C->niac;
}

/* ------------------------------------------------------------------ */
/* con_density, m_particles.f90:2402-2431 */
static void con_density(or_ctx* C, or_phase* P) {
    for (int i = 0; i < P->n; ++i) P->drho[i] = 0.0;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double dv0 = P->vx[2 * i] - P->vx[2 * j], dv1 = P->vx[2 * i + 1] - P->vx[2 * j + 1];
        double vcc = dv0 * C->dwdx[2 * k];
        vcc = vcc + dv1 * C->dwdx[2 * k + 1];
        P->drho[i] = P->drho[i] + P->mass[j] * vcc;
        P->drho[j] = P->drho[j] + P->mass[i] * vcc;
    }
}

/* sum_density, m_particles.f90:2243-2298 */
static void sum_density(or_ctx* C, or_phase* P) {
    int n = P->n;
    double* wi = dalloc((size_t)n);
    double hv[2] = {0, 0}, hv2[2], selfdens;
    for (int i = 0; i < n; ++i) {
        or_kernel(C->prm.skf, 0.0, hv, P->hsml[i], &selfdens, hv2);
        wi[i] = selfdens * P->mass[i] / P->rho[i];
    }
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        wi[i] = wi[i] + P->mass[j] / P->rho[j] * C->w[k];
        wi[j] = wi[j] + P->mass[i] / P->rho[i] * C->w[k];
    }
    for (int i = 0; i < n; ++i) {
        or_kernel(C->prm.skf, 0.0, hv, P->hsml[i], &selfdens, hv2);
        P->rho[i] = selfdens * P->mass[i];
    }
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        P->rho[i] = P->rho[i] + P->mass[j] * C->w[k];
        P->rho[j] = P->rho[j] + P->mass[i] * C->w[k];
    }
    for (int i = 0; i < n; ++i) P->rho[i] = P->rho[i] / wi[i];
    free(wi);
}

/* delta_sph, m_particles.f90:2658-2695 */
static void delta_sph(or_ctx* C, or_phase* P, const double* f, double* df) {
    double delta = C->prm.delta;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double dx0 = P->x[2 * i] - P->x[2 * j], dx1 = P->x[2 * i + 1] - P->x[2 * j + 1];
        double rr = 0.0;
        rr = rr + dx0 * dx0;
        rr = rr + dx1 * dx1;
        double muv = 2.0 * (f[i] - f[j]) / rr;
        double h = 0.0;
        h = h + dx0 * muv * C->dwdx[2 * k];
        h = h + dx1 * muv * C->dwdx[2 * k + 1];
        df[i] = df[i] + delta * P->hsml[i] * P->c[i] * P->mass[j] * h / P->rho[j];
        df[j] = df[j] - delta * P->hsml[j] * P->c[j] * P->mass[i] * h / P->rho[i];
    }
}

/* shear_strain_rate, m_particles.f90:2855-2932 */
static void shear_strain_rate(or_ctx* C, or_phase* P) {
    const double c23 = F32(2.0f / 3.0f);  /* 2.e0/3.e0 is a default-real constant */
    for (int i = 0; i < P->n; ++i) { P->txx[i] = 0.0; P->tyy[i] = 0.0; P->txy[i] = 0.0; }
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double d0 = P->vx[2 * j] - P->vx[2 * i], d1 = P->vx[2 * j + 1] - P->vx[2 * i + 1];
        double w0 = C->dwdx[2 * k], w1 = C->dwdx[2 * k + 1];
        double hxx = 2.0 * d0 * w0 - d1 * w1;
        double hxy = d0 * w1 + d1 * w0;
        double hyy = 2.0 * d1 * w1 - d0 * w0;
        hxx = c23 * hxx;
        hyy = c23 * hyy;
        P->txx[i] = P->txx[i] + P->mass[j] * hxx / P->rho[j];
        P->txx[j] = P->txx[j] + P->mass[i] * hxx / P->rho[i];
        P->txy[i] = P->txy[i] + P->mass[j] * hxy / P->rho[j];
        P->txy[j] = P->txy[j] + P->mass[i] * hxy / P->rho[i];
        P->tyy[i] = P->tyy[i] + P->mass[j] * hyy / P->rho[j];
        P->tyy[j] = P->tyy[j] + P->mass[i] * hyy / P->rho[i];
    }
}

/* velocity_divergence, m_particles.f90:1996-2037 */
static void velocity_divergence(or_ctx* C, or_phase* P) {
    for (int i = 0; i < P->n; ++i) P->vcc[i] = 0.0;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double d0 = P->vx[2 * j] - P->vx[2 * i], d1 = P->vx[2 * j + 1] - P->vx[2 * i + 1];
        double hvcc = d0 * C->dwdx[2 * k];
        hvcc = hvcc + d1 * C->dwdx[2 * k + 1];
        P->vcc[i] = P->vcc[i] + P->mass[j] * hvcc / P->rho[j];
        P->vcc[j] = P->vcc[j] + P->mass[i] * hvcc / P->rho[i];
    }
}

/* pressure, m_particles.f90:2133-2175 */
static void pressure(or_ctx* C, or_phase* P) {
    if (P->material == SPHG_WATER) {
        const sphg_material* m = &C->prm.water;
        for (int i = 0; i < P->n; ++i)
            P->p[i] = m->b * (pow(P->rho[i] / (m->rho0 * P->vof[i]), m->gamma) - 1);
        for (int i = 0; i < P->n; ++i)
            P->c[i] = m->c * pow(P->rho[i] / (m->rho0 * P->vof[i]), 3.0);
    } else {
        for (int i = 0; i < P->n; ++i) P->c[i] = C->prm.soil.c;
    }
}

/* newtonian_fluid, m_particles.f90:2484-2500 (sxx is txx: in place) */
static void newtonian_fluid(or_ctx* C, or_phase* P) {
    double mu = C->prm.water.viscosity;
    for (int i = 0; i < P->n; ++i) {
        P->sxx[i] = mu * P->txx[i];
        P->syy[i] = mu * P->tyy[i];
        P->sxy[i] = mu * P->txy[i];
    }
}

/* art_visc, m_particles.f90:2504-2564 */
static void art_visc(or_ctx* C, or_phase* P) {
    double alpha = C->prm.alpha, beta = C->prm.beta, etq = C->prm.etq;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double mhsml = (P->hsml[i] + P->hsml[j]) / 2.0;
        double vr = 0.0, rr = 0.0;
        for (int d = 0; d < 2; ++d) {
            double dv = P->vx[2 * i + d] - P->vx[2 * j + d];
            double dx = P->x[2 * i + d] - P->x[2 * j + d];
            vr = vr + dv * dx;
            rr = rr + dx * dx;
        }
        if (vr < 0.0) {
            double muv = mhsml * vr / (rr + mhsml * mhsml * etq * etq);
            double mc = 0.5 * (P->c[i] + P->c[j]);
            double mrho = 0.5 * (P->rho[i] + P->rho[j]);
            double piv = (beta * muv - alpha * mc) * muv / mrho;
            for (int d = 0; d < 2; ++d) {
                double h = -piv * C->dwdx[2 * k + d];
                P->dvx[2 * i + d] = P->dvx[2 * i + d] + P->mass[j] * h;
                P->dvx[2 * j + d] = P->dvx[2 * j + d] - P->mass[i] * h;
            }
        }
    }
}

/* av_vel, m_particles.f90:2761-2793 (only real particles are scaled) */
static void av_vel(or_ctx* C, or_phase* P) {
    double eps = C->prm.epsilon;
    for (int i = 0; i < 2 * P->n; ++i) P->av[i] = 0.0;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double mrho = (P->rho[i] + P->rho[j]) / 2.0;
        for (int d = 0; d < 2; ++d) {
            double dv = P->vx[2 * i + d] - P->vx[2 * j + d];
            P->av[2 * i + d] = P->av[2 * i + d] - P->mass[j] * dv / mrho * C->w[k];
            P->av[2 * j + d] = P->av[2 * j + d] + P->mass[i] * dv / mrho * C->w[k];
        }
    }
    for (int i = 0; i < P->ntotal; ++i)
        for (int d = 0; d < 2; ++d) P->av[2 * i + d] = eps * P->av[2 * i + d];
}

/* repulsive_force, m_particles.f90:1605-1642 */
static void repulsive_force(or_ctx* C, or_phase* P) {
    double rr0 = P->dspp, dd = C->prm.dd, p1 = C->prm.p1, p2 = C->prm.p2;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        if (P->itype[i] * P->itype[j] > 0) continue;
        double dx[2], rr = 0.0;
        for (int d = 0; d < 2; ++d) { dx[d] = P->x[2 * i + d] - P->x[2 * j + d]; rr = rr + dx[d] * dx[d]; }
        rr = sqrt(rr);
        if (rr > rr0) continue;
        double f = (pow(rr0 / rr, p1) - pow(rr0 / rr, p2)) / (rr * rr);
        int ii = i;
        if (P->itype[i] < 0) ii = j;
        for (int d = 0; d < 2; ++d) P->dvx[2 * ii + d] = P->dvx[2 * ii + d] + dd * dx[d] * f;
    }
}

/* df / df2 / df3, m_particles.f90:1711-1736, 1802-1831, 1898-1927.
 * comp selects dwdx(1,:) or dwdx(2,:). */
static void op_df(or_ctx* C, or_phase* P, const double* f, int comp, double* out) {
    for (int i = 0; i < P->n; ++i) out[i] = 0.0;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double fwx = (f[i] + f[j]) * C->dwdx[2 * k + comp];
        out[i] = out[i] + P->mass[j] / P->rho[j] * fwx;
        out[j] = out[j] - P->mass[i] / P->rho[i] * fwx;
    }
}
static void op_df2(or_ctx* C, or_phase* P, const double* f, int stride, int comp, double* out) {
    for (int i = 0; i < P->n; ++i) out[i] = 0.0;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double fwx = (f[stride * j] - f[stride * i]) * C->dwdx[2 * k + comp];
        out[i] = out[i] + P->mass[j] * fwx;
        out[j] = out[j] + P->mass[i] * fwx;
    }
    for (int i = 0; i < P->n; ++i) out[i] = out[i] / P->rho[i];
}
static void op_df3(or_ctx* C, or_phase* P, const double* f, int comp, double* out) {
    for (int i = 0; i < P->n; ++i) out[i] = 0.0;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double fwx = ((f[i] / (P->rho[i] * P->rho[i])) + (f[j] / (P->rho[j] * P->rho[j]))) * C->dwdx[2 * k + comp];
        out[i] = out[i] + P->mass[j] * fwx;
        out[j] = out[j] - P->mass[i] * fwx;
    }
    for (int i = 0; i < P->n; ++i) out[i] = out[i] * P->rho[i];
}
/* df of a strided field (velocity component) */
static void op_df_s(or_ctx* C, or_phase* P, const double* f, int stride, int comp, double* out) {
    for (int i = 0; i < P->n; ++i) out[i] = 0.0;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double fwx = (f[stride * i] + f[stride * j]) * C->dwdx[2 * k + comp];
        out[i] = out[i] + P->mass[j] / P->rho[j] * fwx;
        out[j] = out[j] - P->mass[i] / P->rho[i] * fwx;
    }
}

/* alpha1 of the Drucker-Prager cone: tan(phi)/sqrt(9.+12.*tan(phi)**2.) */
static double dp_alpha(double phi) { double t = tan(phi); return t / sqrt(9.0 + 12.0 * (t * t)); }

/* drucker_prager_failure_criterion, m_particles.f90:3323-3381 */
static void drucker_prager(or_ctx* C, or_phase* P) {
    double alpha1 = dp_alpha(C->prm.soil.phi);
    int k = 0;
    for (int i = 0; i < P->n; ++i) P->fail[i] = 0;
    for (int i = 0; i < P->n; ++i) {
        if (P->p[i] < 0.0) P->p[i] = 0.0;
        double I1 = 3.0 * P->p[i];
        double s0 = P->sxx[i], s1 = P->sxy[i], s2 = P->syy[i];
        double J2 = s0 * s0 + 2.0 * (s1 * s1) + s2 * s2 + (s0 + s2) * (s0 + s2);
        J2 = sqrt(J2 / 2.0) + 1.0e-6;
        if (J2 > alpha1 * I1) {
            k = k + 1;
            P->fail[i] = 1;
            double skale = alpha1 * I1 / J2;
            P->sxx[i] = skale * P->sxx[i];
            P->sxy[i] = skale * P->sxy[i];
            P->syy[i] = skale * P->syy[i];
        }
    }
    P->nfail = k;
}

/* plastic_or_not, m_particles.f90:3447-3505 */
static void plastic_or_not(or_ctx* C, or_phase* P) {
    double alpha1 = dp_alpha(C->prm.soil.phi);
    int k = 0;
    for (int i = 0; i < P->n; ++i) P->fail[i] = 0;
    for (int i = 0; i < P->n; ++i) {
        double I1 = 3.0 * P->p[i];
        double s0 = P->sxx[i], s1 = P->sxy[i], s2 = P->syy[i];
        double J2 = s0 * s0 + 2.0 * (s1 * s1) + s2 * s2 + (s0 + s2) * (s0 + s2);
        J2 = sqrt(J2 / 2.0) + 1.0e-6;
        if (fabs(J2 - alpha1 * I1) < F32(1.0e-5f)) { k = k + 1; P->fail[i] = 1; }
    }
    P->nfail = k;
}

/* plastic_flow_rule3, m_particles.f90:3700-3762 */
static void plastic_flow_rule3(or_ctx* C, or_phase* P) {
    const sphg_material* m = &C->prm.soil;
    double phi = m->phi, K = m->k, e = m->E, niu = m->niu;
    double alpha = dp_alpha(phi);
    double G = e / (2.0 * (1 + niu));
    const double small_value = 1.0e-10;
    for (int i = 0; i < P->n; ++i) {
        if (P->fail[i] != 1) continue;
        double exx = P->txx[i] / 2.0 + P->vcc[i] / 3.0;
        double exy = P->txy[i] / 2.0;
        double eyy = P->tyy[i] / 2.0 + P->vcc[i] / 3.0;
        double s0 = P->sxx[i], s1 = P->sxy[i], s2 = P->syy[i];
        double sde = s0 * exx + 2.0 * s1 * exy + s2 * eyy;
        double J2 = (s0 * s0 + 2.0 * (s1 * s1) + s2 * s2 + (s0 + s2) * (s0 + s2)) / 2.0;
        J2 = J2 + small_value;
        double dlambda = (3.0 * alpha * K * P->vcc[i] + G / sqrt(J2) * sde) / (9.0 * (alpha * alpha) * K + G);
        if (dlambda < 0) continue;
        P->dsxx[i] = P->dsxx[i] - dlambda * (G / sqrt(J2) * s0);
        P->dsxy[i] = P->dsxy[i] - dlambda * (G / sqrt(J2) * s1);
        P->dsyy[i] = P->dsyy[i] - dlambda * (G / sqrt(J2) * s2);
        P->dp[i] = P->dp[i] + 3.0 * K * alpha * dlambda;
        P->epsilon_p[i] = P->epsilon_p[i] + dlambda * s1 / (2 * sqrt(J2)) * F32(0.000005f);
    }
}

/* Jaumann_rate, m_particles.f90:3047-3119.  wxy is txy (alias): the spin
 * sum overwrites the shear strain rate after it was used. */
static void jaumann_rate(or_ctx* C, or_phase* P) {
    const sphg_material* m = &C->prm.soil;
    double G = m->E / (2.0 * (1 + m->niu));
    for (int i = 0; i < P->n; ++i) {
        P->dsxx[i] = P->dsxx[i] + G * P->txx[i];
        P->dsxy[i] = P->dsxy[i] + G * P->txy[i];
        P->dsyy[i] = P->dsyy[i] + G * P->tyy[i];
    }
    for (int i = 0; i < P->n; ++i) P->dp[i] = P->dp[i] - m->k * P->vcc[i];
    for (int i = 0; i < C->maxn; ++i) P->wxy[i] = 0.0;  /* parts%wxy = 0.d0 (whole array) */
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double d0 = P->vx[2 * j] - P->vx[2 * i], d1 = P->vx[2 * j + 1] - P->vx[2 * i + 1];
        double hxy = 0.5 * (d0 * C->dwdx[2 * k + 1] - d1 * C->dwdx[2 * k]);
        P->wxy[i] = P->wxy[i] + P->mass[j] * hxy / P->rho[j];
        P->wxy[j] = P->wxy[j] + P->mass[i] * hxy / P->rho[i];
    }
    for (int i = 0; i < P->n; ++i) {
        P->dsxx[i] = P->dsxx[i] + 2.0 * P->sxy[i] * P->wxy[i];
        P->dsxy[i] = P->dsxy[i] - (P->sxx[i] - P->syy[i]) * P->wxy[i];
        P->dsyy[i] = P->dsyy[i] - 2.0 * P->sxy[i] * P->wxy[i];
    }
}

/* darcy_law, m_particles.f90:3832-3874.  With forchheimer_b > 0 (not in the
 * reference) the pair's coefficient cf is scaled by 1 + ks*b*|v_w - v_s|, the
 * Forchheimer law i = u/ks + b|u|u in the reference's hydraulic-gradient form. */
static void darcy_law(or_ctx* C, or_phase* W, or_phase* S) {
    double gravity = C->prm.numeric_gravity, ks = C->prm.soil.permeability;
    double kb = ks * C->prm.forchheimer_b;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double rrw = C->w[k] / (W->rho[i] * S->rho[j]);
        double cf = W->vof[i] * S->vof[j] * W->rho[i] * (-gravity) / ks;
        if (kb != 0.0) {
            double u0 = W->vx[2 * i] - S->vx[2 * j], u1 = W->vx[2 * i + 1] - S->vx[2 * j + 1];
            cf = cf * (1.0 + kb * sqrt(u0 * u0 + u1 * u1));
        }
        for (int d = 0; d < 2; ++d) {
            double sp = cf * (W->vx[2 * i + d] - S->vx[2 * j + d]) * rrw;
            W->dvx[2 * i + d] = W->dvx[2 * i + d] - S->mass[j] * sp;
            S->dvx[2 * j + d] = S->dvx[2 * j + d] + W->mass[i] * sp;
        }
    }
}

/* pore_water_pressure, m_particles.f90:3877-3909 */
static void pore_water_pressure(or_ctx* C, or_phase* W, or_phase* S) {
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double mprr = W->mass[i] * W->p[i] / (W->rho[i] * S->rho[j]);
        for (int d = 0; d < 2; ++d)
            S->dvx[2 * j + d] = S->dvx[2 * j + d] + mprr * C->dwdx[2 * k + d] * S->vof[j];
    }
}

/* volume_fraction_water, m_particles.f90:3912-3937 */
static void volume_fraction_water(or_ctx* C, or_phase* W, or_phase* S) {
    for (int i = 0; i < C->maxn && i < W->n; ++i) W->vof2[i] = 0.0;
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        W->vof2[i] = W->vof2[i] + S->mass[j] * C->w[k];
    }
    for (int k = 0; k < W->n; ++k) W->vof2[k] = 1.0 - W->vof2[k] / C->prm.soil.rho0;
}

/* volume_fraction_water2, m_particles.f90:3940-3967 */
static void volume_fraction_water2(or_ctx* C, or_phase* W, or_phase* S) {
    for (int64_t k = 0; k < C->niac; ++k) {
        int i = C->pair_i[k], j = C->pair_j[k];
        double d0 = W->vx[2 * i] - S->vx[2 * j], d1 = W->vx[2 * i + 1] - S->vx[2 * j + 1];
        double tmp = d0 * C->dwdx[2 * k] + d1 * C->dwdx[2 * k + 1];
        W->dvof[i] = W->dvof[i] - S->mass[j] * tmp / C->prm.soil.rho0;
    }
}

/* volume_fraction_soil, m_particles.f90:3970-3988 */
static void volume_fraction_soil(or_ctx* C, or_phase* S) {
    for (int i = 0; i < S->n; ++i) S->vof[i] = S->rho[i] / C->prm.soil.rho0;
}

/* ------------------------------------------------------------------ */
/* single_step, declarations_sph.f90:1131-1435 */
static int single_step_two_phase(or_ctx* C, int itimestep) {
    const sphg_params* prm = &C->prm;
    int nphase = prm->single_phase ? 1 : 2;
    for (int iphase = 0; iphase < nphase; ++iphase) {
        or_phase* pl = &C->ph[iphase];
        int n = pl->n;
        memset(pl->dvx, 0, sizeof(double) * 2 * (size_t)n);
        memset(pl->drho, 0, sizeof(double) * (size_t)n);
        if (pl->material == SPHG_WATER) memset(pl->dvof, 0, sizeof(double) * (size_t)n);
        if (pl->material == SPHG_SOIL) {
            memset(pl->dsxx, 0, sizeof(double) * (size_t)n); memset(pl->dsxy, 0, sizeof(double) * (size_t)n);
            memset(pl->dsyy, 0, sizeof(double) * (size_t)n); memset(pl->dp, 0, sizeof(double) * (size_t)n);
        }
        if (direct_find(C, pl)) return C->status;
        save_pairs(C, iphase);
        con_density(C, pl);
        if (prm->artificial_density) delta_sph(C, pl, pl->rho, pl->drho);
        shear_strain_rate(C, pl);
        if (pl->material == SPHG_SOIL) velocity_divergence(C, pl);
        pressure(C, pl);
        if (pl->material == SPHG_WATER) newtonian_fluid(C, pl);
        else if (prm->yield_criterion == 2) drucker_prager(C, pl);

        double *t1 = dalloc((size_t)n), *t2 = dalloc((size_t)n), *t3 = dalloc((size_t)n), *f = dalloc((size_t)n);
        if (pl->material == SPHG_WATER) {
            for (int comp = 0; comp < 2; ++comp) {
                const double* sa = comp == 0 ? pl->sxx : pl->sxy;   /* df(vof*sxx,'x') | df(vof*sxy,'x') */
                const double* sb = comp == 0 ? pl->sxy : pl->syy;   /* df(vof*sxy,'y') | df(vof*syy,'y') */
                op_df(C, pl, pl->p, comp, t1);
                for (int i = 0; i < n; ++i) f[i] = pl->vof[i] * sa[i];
                op_df(C, pl, f, 0, t2);
                for (int i = 0; i < n; ++i) f[i] = pl->vof[i] * sb[i];
                op_df(C, pl, f, 1, t3);
                for (int i = 0; i < n; ++i) pl->dvx[2 * i + comp] = -(pl->vof[i] * t1[i]) + t2[i] + t3[i];
            }
        } else {
            for (int comp = 0; comp < 2; ++comp) {
                const double* sa = comp == 0 ? pl->sxx : pl->sxy;
                const double* sb = comp == 0 ? pl->sxy : pl->syy;
                for (int i = 0; i < n; ++i) f[i] = pl->vof[i] * pl->p[i];
                op_df3(C, pl, f, comp, t1);
                for (int i = 0; i < n; ++i) f[i] = pl->vof[i] * sa[i];
                op_df3(C, pl, f, 0, t2);
                for (int i = 0; i < n; ++i) f[i] = pl->vof[i] * sb[i];
                op_df3(C, pl, f, 1, t3);
                for (int i = 0; i < n; ++i) pl->dvx[2 * i + comp] = -t1[i] + t2[i] + t3[i];
            }
        }
        free(t1); free(t2); free(t3); free(f);
        for (int i = 0; i < n; ++i)
            if (pl->rho[i] > 0.0) { pl->dvx[2 * i] = pl->dvx[2 * i] / pl->rho[i]; }
        for (int i = 0; i < n; ++i)
            if (pl->rho[i] > 0.0) { pl->dvx[2 * i + 1] = pl->dvx[2 * i + 1] / pl->rho[i]; }

        if (pl->material == SPHG_SOIL && prm->plasticity == 3) {
            plastic_or_not(C, pl);
            plastic_flow_rule3(C, pl);
        }
        if (pl->material == SPHG_SOIL) jaumann_rate(C, pl);
        if (prm->visc_artificial) art_visc(C, pl);
        if (pl->material == SPHG_SOIL && prm->soil_artificial_stress) {
            delta_sph(C, pl, pl->p, pl->dp);
            delta_sph(C, pl, pl->sxx, pl->dsxx);
            delta_sph(C, pl, pl->sxy, pl->dsxy);
            delta_sph(C, pl, pl->syy, pl->dsyy);
        }
        if (pl->material == SPHG_WATER && prm->water_artificial_volume) delta_sph(C, pl, pl->vof, pl->dvof);
        repulsive_force(C, pl);
        for (int i = 0; i < n; ++i) pl->dvx[2 * i + 1] = pl->dvx[2 * i + 1] + prm->gravity;
        if (prm->average_velocity) av_vel(C, pl);
    }
    if (!prm->single_phase) {
        or_phase *W = &C->ph[0], *S = &C->ph[1];
        if (direct_find_2(C, W, S)) return C->status;
        save_pairs(C, 2);
        darcy_law(C, W, S);
        pore_water_pressure(C, W, S);
        if (prm->volume_fraction) {
            volume_fraction_soil(C, S);
            volume_fraction_water2(C, W, S);
            volume_fraction_water(C, W, S);
            if (prm->volume_fraction_renorm && prm->renorm_interval > 0 && itimestep % prm->renorm_interval == 0) {
                for (int i = 0; i < W->n; ++i) W->rho[i] = W->rho[i] / W->vof[i];
                for (int i = 0; i < W->n; ++i) W->vof[i] = W->vof2[i];
                for (int i = 0; i < W->n; ++i) W->rho[i] = W->rho[i] * W->vof[i];
            }
        }
    }
    return 0;
}

/* single_step_for_water, declarations_sph.f90:1439-1526 */
static int single_step_water(or_ctx* C) {
    const sphg_params* prm = &C->prm;
    or_phase* pl = &C->ph[0];
    const sphg_material* m = &prm->water;
    int n = pl->n;
    memset(pl->dvx, 0, sizeof(double) * 2 * (size_t)n);
    memset(pl->drho, 0, sizeof(double) * (size_t)n);
    if (direct_find(C, pl)) return C->status;
    save_pairs(C, 0);
    sum_density(C, pl);
    double *a = dalloc((size_t)n), *b = dalloc((size_t)n), *c = dalloc((size_t)n), *d = dalloc((size_t)n);
    op_df2(C, pl, pl->vx, 2, 0, a);
    op_df2(C, pl, pl->vx + 1, 2, 1, b);
    for (int i = 0; i < n; ++i) pl->drho[i] = -pl->rho[i] * (a[i] + b[i]);
    if (prm->artificial_density) delta_sph(C, pl, pl->rho, pl->drho);
    for (int i = 0; i < n; ++i)
        if (pl->rho[i] > 0.0) pl->p[i] = m->b * (pow(pl->rho[i] / m->rho0, m->gamma) - 1);
    const double c23 = F32(2.0f / 3.0f);
    /* df(vx,'x'), df(vy,'y'), df(vx,'y'), df(vy,'x') */
    op_df_s(C, pl, pl->vx, 2, 0, a);
    op_df_s(C, pl, pl->vx + 1, 2, 1, b);
    op_df_s(C, pl, pl->vx, 2, 1, c);
    op_df_s(C, pl, pl->vx + 1, 2, 0, d);
    for (int i = 0; i < n; ++i) {
        pl->txx[i] = c23 * (2.0 * a[i] - b[i]);
        pl->txy[i] = c[i] + d[i];
        pl->tyy[i] = c23 * (2.0 * b[i] - a[i]);
    }
    for (int i = 0; i < n; ++i) {  /* sxx => txx etc.: in place */
        pl->sxx[i] = m->viscosity * pl->txx[i];
        pl->syy[i] = m->viscosity * pl->tyy[i];
        pl->sxy[i] = m->viscosity * pl->txy[i];
    }
    for (int comp = 0; comp < 2; ++comp) {
        const double* sa = comp == 0 ? pl->sxx : pl->sxy;
        const double* sb = comp == 0 ? pl->sxy : pl->syy;
        op_df(C, pl, pl->p, comp, a);
        op_df(C, pl, sa, 0, b);
        op_df(C, pl, sb, 1, c);
        for (int i = 0; i < n; ++i) pl->dvx[2 * i + comp] = -a[i] + b[i] + c[i];
    }
    free(a); free(b); free(c); free(d);
    for (int i = 0; i < n; ++i) if (pl->rho[i] > 0.0) pl->dvx[2 * i] = pl->dvx[2 * i] / pl->rho[i];
    for (int i = 0; i < n; ++i) if (pl->rho[i] > 0.0) pl->dvx[2 * i + 1] = pl->dvx[2 * i + 1] / pl->rho[i];
    if (prm->visc_artificial) art_visc(C, pl);
    for (int i = 0; i < n; ++i) pl->dvx[2 * i + 1] = pl->dvx[2 * i + 1] + prm->gravity;
    if (prm->average_velocity) av_vel(C, pl);
    return 0;
}

/* single_step_for_soil, declarations_sph.f90:1530-1655 */
static int single_step_soil(or_ctx* C) {
    const sphg_params* prm = &C->prm;
    or_phase* pl = &C->ph[0];
    int n = pl->n;
    memset(pl->dvx, 0, sizeof(double) * 2 * (size_t)n);
    memset(pl->drho, 0, sizeof(double) * (size_t)n);
    memset(pl->dsxx, 0, sizeof(double) * (size_t)n); memset(pl->dsxy, 0, sizeof(double) * (size_t)n);
    memset(pl->dsyy, 0, sizeof(double) * (size_t)n); memset(pl->dp, 0, sizeof(double) * (size_t)n);
    if (direct_find(C, pl)) return C->status;
    save_pairs(C, 0);
    if (prm->summation_density) sum_density(C, pl); else con_density(C, pl);
    if (prm->artificial_density) delta_sph(C, pl, pl->rho, pl->drho);
    shear_strain_rate(C, pl);
    velocity_divergence(C, pl);
    pressure(C, pl);
    if (prm->yield_criterion == 2) drucker_prager(C, pl);
    double *a = dalloc((size_t)n), *b = dalloc((size_t)n), *c = dalloc((size_t)n);
    for (int comp = 0; comp < 2; ++comp) {
        const double* sa = comp == 0 ? pl->sxx : pl->sxy;
        const double* sb = comp == 0 ? pl->sxy : pl->syy;
        op_df(C, pl, pl->p, comp, a);
        op_df(C, pl, sa, 0, b);
        op_df(C, pl, sb, 1, c);
        for (int i = 0; i < n; ++i) pl->dvx[2 * i + comp] = -a[i] + b[i] + c[i];
    }
    free(a); free(b); free(c);
    for (int i = 0; i < n; ++i) if (pl->rho[i] > 0.0) pl->dvx[2 * i] = pl->dvx[2 * i] / pl->rho[i];
    for (int i = 0; i < n; ++i) if (pl->rho[i] > 0.0) pl->dvx[2 * i + 1] = pl->dvx[2 * i + 1] / pl->rho[i];
    if (prm->plasticity == 3) { plastic_or_not(C, pl); plastic_flow_rule3(C, pl); }
    jaumann_rate(C, pl);
    if (prm->visc_artificial) art_visc(C, pl);
    if (prm->soil_artificial_stress) {
        delta_sph(C, pl, pl->p, pl->dp);
        delta_sph(C, pl, pl->sxx, pl->dsxx);
        delta_sph(C, pl, pl->sxy, pl->dsxy);
        delta_sph(C, pl, pl->syy, pl->dsyy);
    }
    for (int i = 0; i < n; ++i) pl->dvx[2 * i + 1] = pl->dvx[2 * i + 1] + prm->gravity;
    if (prm->average_velocity) av_vel(C, pl);
    return 0;
}

int or_single_step(or_ctx* C, int itimestep) {
    if (!C) return SPHG_ERR_BAD_ARG;
    C->status = 0;
    int rc;
    if (C->prm.single_phase)
        rc = C->ph[0].material == SPHG_WATER ? single_step_water(C) : single_step_soil(C);
    else
        rc = single_step_two_phase(C, itimestep);
    return rc ? (C->status ? C->status : rc) : 0;
}

/* ------------------------------------------------------------------ */
/* integrator pieces: first_half / first_step / second_half,
 * declarations_sph.f90:643-762 (two-phase) and the single-phase copies
 * :812-866 (water) and :998-1100 (soil). */
static void first_half(or_ctx* C, or_phase* pl, int with_vof) {
    const sphg_params* prm = &C->prm; double dt = prm->dt;
    for (int i = 0; i < pl->n; ++i) {
        if (!prm->summation_density) { pl->rho_min[i] = pl->rho[i]; pl->rho[i] = pl->rho[i] + (dt / 2.0) * pl->drho[i]; }
        if (with_vof && pl->material == SPHG_WATER && prm->volume_fraction) {
            pl->vof_min[i] = pl->vof[i]; pl->vof[i] = pl->vof[i] + (dt / 2.0) * pl->dvof[i];
        }
        if (pl->material == SPHG_SOIL && prm->stress_integration == 2) {
            pl->sxx_min[i] = pl->sxx[i]; pl->sxy_min[i] = pl->sxy[i]; pl->syy_min[i] = pl->syy[i]; pl->p_min[i] = pl->p[i];
            pl->sxx[i] = pl->sxx[i] + (dt / 2.0) * pl->dsxx[i];
            pl->sxy[i] = pl->sxy[i] + (dt / 2.0) * pl->dsxy[i];
            pl->syy[i] = pl->syy[i] + (dt / 2.0) * pl->dsyy[i];
            pl->p[i] = pl->p[i] + (dt / 2.0) * pl->dp[i];
        }
        if (pl->itype[i] < 0) continue;
        for (int d = 0; d < 2; ++d) { pl->v_min[2 * i + d] = pl->vx[2 * i + d]; pl->vx[2 * i + d] = pl->vx[2 * i + d] + (dt / 2.0) * pl->dvx[2 * i + d]; }
    }
}
static void first_step(or_ctx* C, or_phase* pl, int with_vof) {
    const sphg_params* prm = &C->prm; double dt = prm->dt;
    for (int i = 0; i < pl->n; ++i) {
        if (!prm->summation_density) pl->rho[i] = pl->rho[i] + (dt / 2.0) * pl->drho[i];
        if (with_vof && pl->material == SPHG_WATER && prm->volume_fraction) pl->vof[i] = pl->vof[i] + (dt / 2.0) * pl->dvof[i];
        if (pl->material == SPHG_SOIL) {
            if (prm->stress_integration == 1) {
                pl->sxx[i] = pl->sxx[i] + dt * pl->dsxx[i]; pl->sxy[i] = pl->sxy[i] + dt * pl->dsxy[i];
                pl->syy[i] = pl->syy[i] + dt * pl->dsyy[i]; pl->p[i] = pl->p[i] + dt * pl->dp[i];
            } else if (prm->stress_integration == 2) {
                pl->sxx[i] = pl->sxx[i] + (dt / 2.0) * pl->dsxx[i]; pl->sxy[i] = pl->sxy[i] + (dt / 2.0) * pl->dsxy[i];
                pl->syy[i] = pl->syy[i] + (dt / 2.0) * pl->dsyy[i]; pl->p[i] = pl->p[i] + (dt / 2.0) * pl->dp[i];
            }
        }
        if (pl->itype[i] < 0) continue;
        for (int d = 0; d < 2; ++d) {
            pl->vx[2 * i + d] = pl->vx[2 * i + d] + (dt / 2.0) * pl->dvx[2 * i + d] + pl->av[2 * i + d];
            pl->x[2 * i + d] = pl->x[2 * i + d] + dt * pl->vx[2 * i + d];
        }
    }
}
static void second_half(or_ctx* C, or_phase* pl, int with_vof) {
    const sphg_params* prm = &C->prm; double dt = prm->dt;
    for (int i = 0; i < pl->n; ++i) {
        if (!prm->summation_density) pl->rho[i] = pl->rho_min[i] + dt * pl->drho[i];
        if (with_vof && pl->material == SPHG_WATER && prm->volume_fraction) pl->vof[i] = pl->vof_min[i] + dt * pl->dvof[i];
        if (pl->material == SPHG_SOIL) {
            if (prm->stress_integration == 1) {
                pl->sxx[i] = pl->sxx[i] + dt * pl->dsxx[i]; pl->sxy[i] = pl->sxy[i] + dt * pl->dsxy[i];
                pl->syy[i] = pl->syy[i] + dt * pl->dsyy[i]; pl->p[i] = pl->p[i] + dt * pl->dp[i];
            } else if (prm->stress_integration == 2) {
                pl->sxx[i] = pl->sxx_min[i] + dt * pl->dsxx[i]; pl->sxy[i] = pl->sxy_min[i] + dt * pl->dsxy[i];
                pl->syy[i] = pl->syy_min[i] + dt * pl->dsyy[i]; pl->p[i] = pl->p_min[i] + dt * pl->dp[i];
            }
        }
        if (pl->itype[i] < 0) continue;
        for (int d = 0; d < 2; ++d) {
            pl->vx[2 * i + d] = pl->v_min[2 * i + d] + dt * pl->dvx[2 * i + d] + pl->av[2 * i + d];
            pl->x[2 * i + d] = pl->x[2 * i + d] + dt * pl->vx[2 * i + d];
        }
    }
}

/* time_integration (:525), time_integration_for_water (:794),
 * time_integration_for_soil (:978) */
int or_time_integration(or_ctx* C, int maxtimestep, int* itimestep, double* time) {
    if (!C || !itimestep || !time) return SPHG_ERR_BAD_ARG;
    const sphg_params* prm = &C->prm;
    for (int it = 0; it < maxtimestep; ++it) {
        *itimestep = *itimestep + 1;
        int ts = *itimestep;
        if (prm->single_phase) {
            or_phase* pl = &C->ph[0];
            int soil = pl->material == SPHG_SOIL;
            if (ts != 1) { first_half(C, pl, 0); if (soil) drucker_prager(C, pl); }
            int rc = or_single_step(C, ts);
            if (rc) return rc;
            if (ts == 1) first_step(C, pl, 0); else second_half(C, pl, 0);
            if (soil) drucker_prager(C, pl);
        } else {
            or_phase *W = &C->ph[0], *S = &C->ph[1];
            if (ts != 1) { first_half(C, W, 1); first_half(C, S, 1); drucker_prager(C, S); }
            int rc = or_single_step(C, ts);
            if (rc) return rc;
            if (ts == 1) { first_step(C, W, 1); first_step(C, S, 1); }
            else { second_half(C, W, 1); second_half(C, S, 1); }
            drucker_prager(C, S);
        }
        *time = *time + prm->dt;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
static void phase_alloc(or_ctx* C, or_phase* P, int n) {
    size_t N = (size_t)n;
    P->n = n;
    P->x = dalloc(2 * N); P->vx = dalloc(2 * N); P->dvx = dalloc(2 * N); P->av = dalloc(2 * N); P->v_min = dalloc(2 * N);
    P->rho = dalloc(N); P->rho_min = dalloc(N); P->drho = dalloc(N); P->p = dalloc(N); P->c = dalloc(N);
    P->mass = dalloc(N); P->hsml = dalloc(N);
    P->vof = dalloc(N); P->vof_min = dalloc(N); P->dvof = dalloc(N); P->vof2 = dalloc(N);
    P->dsxx = dalloc(N); P->dsxy = dalloc(N); P->dsyy = dalloc(N); P->dp = dalloc(N);
    P->sxx_min = dalloc(N); P->sxy_min = dalloc(N); P->syy_min = dalloc(N); P->p_min = dalloc(N);
    P->epsilon_p = dalloc(N); P->vcc = dalloc(N);
    P->itype = ialloc(N); P->fail = ialloc(N); P->countiac = ialloc(N);
    (void)C;
}

static void phase_free(or_phase* P) {
    void* ptrs[] = {P->x, P->vx, P->dvx, P->av, P->v_min, P->rho, P->rho_min, P->drho, P->p, P->c, P->mass, P->hsml,
                    P->vof, P->vof_min, P->dvof, P->vof2, P->dsxx, P->dsxy, P->dsyy, P->dp, P->sxx_min, P->sxy_min,
                    P->syy_min, P->p_min, P->epsilon_p, P->vcc, P->itype, P->fail, P->countiac};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
    if (P->material == SPHG_SOIL) { free(P->sxx); free(P->sxy); free(P->syy); }
}

or_ctx* or_create(const sphg_params* p, int nphase) {
    if (!p || (nphase != 1 && nphase != 2)) return NULL;
    or_ctx* C = (or_ctx*)calloc(1, sizeof(or_ctx));
    C->prm = *p;
    C->nphase = nphase;
    C->search_mode = 0;
    return C;
}

void or_set_search_mode(or_ctx* C, int mode) { if (C) C->search_mode = mode; }

/* Wire the aliases of allocate_sph (declarations_sph.f90:368-377,414-415)
 * once both phases are known. */
static void wire_aliases(or_ctx* C) {
    int maxn = 0;
    for (int k = 0; k < C->nphase; ++k) if (C->ph[k].n > maxn) maxn = C->ph[k].n;
    if (maxn > C->maxn) {  /* grow, keeping what an earlier upload stored */
        double* a[3] = {C->wtxx, C->wtyy, C->wtxy};
        double* b[3];
        for (int t = 0; t < 3; ++t) {
            b[t] = dalloc((size_t)maxn);
            if (a[t]) memcpy(b[t], a[t], sizeof(double) * (size_t)C->maxn);
            free(a[t]);
        }
        C->wtxx = b[0]; C->wtyy = b[1]; C->wtxy = b[2];
        C->maxn = maxn;
    }
    for (int k = 0; k < C->nphase; ++k) {
        or_phase* P = &C->ph[k];
        if (!P->x) continue;
        P->txx = C->wtxx; P->tyy = C->wtyy; P->txy = C->wtxy;
        if (P->material == SPHG_WATER) { P->sxx = C->wtxx; P->syy = C->wtyy; P->sxy = C->wtxy; P->wxy = NULL; }
        else P->wxy = C->wtxy;
    }
    int64_t cap = C->prm.max_interaction > 0 ? C->prm.max_interaction : 1;
    if (cap != C->cap) {
        free(C->pair_i); free(C->pair_j); free(C->w); free(C->dwdx);
        C->cap = cap;
        C->pair_i = ialloc((size_t)cap); C->pair_j = ialloc((size_t)cap);
        C->w = dalloc((size_t)cap); C->dwdx = dalloc(2 * (size_t)cap);
    }
}

static void cp_in(double* dst, const double* src, size_t n) { if (src) memcpy(dst, src, n * sizeof(double)); else memset(dst, 0, n * sizeof(double)); }
static void cp_out(double* dst, const double* src, size_t n) { if (dst && src) memcpy(dst, src, n * sizeof(double)); }

int or_upload_phase(or_ctx* C, int phase, const sphg_phase_host* h) {
    if (!C || !h || phase < 1 || phase > C->nphase) return SPHG_ERR_BAD_ARG;
    if (!h->x || !h->vx || !h->rho || !h->p || !h->c || !h->mass || !h->hsml || !h->itype) return SPHG_ERR_BAD_ARG;
    or_phase* P = &C->ph[phase - 1];
    int n = h->ntotal + h->nvirt;
    if (P->x) phase_free(P);
    memset(P, 0, sizeof(*P));
    phase_alloc(C, P, n);
    P->ntotal = h->ntotal; P->nvirt = h->nvirt; P->material = h->material; P->dspp = h->dspp;
    size_t N = (size_t)n;
    cp_in(P->x, h->x, 2 * N); cp_in(P->vx, h->vx, 2 * N); cp_in(P->dvx, h->dvx, 2 * N);
    cp_in(P->av, h->av, 2 * N); cp_in(P->v_min, h->v_min, 2 * N);
    cp_in(P->rho, h->rho, N); cp_in(P->rho_min, h->rho_min, N); cp_in(P->drho, h->drho, N);
    cp_in(P->p, h->p, N); cp_in(P->c, h->c, N); cp_in(P->mass, h->mass, N); cp_in(P->hsml, h->hsml, N);
    cp_in(P->vof, h->vof, N); cp_in(P->vof_min, h->vof_min, N); cp_in(P->dvof, h->dvof, N); cp_in(P->vof2, h->vof2, N);
    cp_in(P->dsxx, h->dsxx, N); cp_in(P->dsxy, h->dsxy, N); cp_in(P->dsyy, h->dsyy, N); cp_in(P->dp, h->dp, N);
    cp_in(P->sxx_min, h->sxx_min, N); cp_in(P->sxy_min, h->sxy_min, N); cp_in(P->syy_min, h->syy_min, N);
    cp_in(P->p_min, h->p_min, N); cp_in(P->epsilon_p, h->epsilon_p, N); cp_in(P->vcc, h->vcc, N);
    for (int i = 0; i < n; ++i) P->itype[i] = h->itype[i];
    if (P->material == SPHG_SOIL) {
        P->sxx = dalloc(N); P->sxy = dalloc(N); P->syy = dalloc(N);
        cp_in(P->sxx, h->sxx, N); cp_in(P->sxy, h->sxy, N); cp_in(P->syy, h->syy, N);
    }
    wire_aliases(C);
    /* water stress lives in the shared working arrays */
    if (P->material == SPHG_WATER) {
        if (h->sxx) memcpy(P->sxx, h->sxx, N * sizeof(double));
        if (h->syy) memcpy(P->syy, h->syy, N * sizeof(double));
        if (h->sxy) memcpy(P->sxy, h->sxy, N * sizeof(double));
    }
    return 0;
}

int or_download_phase(or_ctx* C, int phase, sphg_phase_host* h) {
    if (!C || !h || phase < 1 || phase > C->nphase) return SPHG_ERR_BAD_ARG;
    or_phase* P = &C->ph[phase - 1];
    size_t N = (size_t)P->n;
    h->ntotal = P->ntotal; h->nvirt = P->nvirt; h->material = P->material; h->nfail = P->nfail;
    cp_out(h->x, P->x, 2 * N); cp_out(h->vx, P->vx, 2 * N); cp_out(h->dvx, P->dvx, 2 * N);
    cp_out(h->av, P->av, 2 * N); cp_out(h->v_min, P->v_min, 2 * N);
    cp_out(h->rho, P->rho, N); cp_out(h->rho_min, P->rho_min, N); cp_out(h->drho, P->drho, N);
    cp_out(h->p, P->p, N); cp_out(h->c, P->c, N); cp_out(h->mass, P->mass, N); cp_out(h->hsml, P->hsml, N);
    cp_out(h->vof, P->vof, N); cp_out(h->vof_min, P->vof_min, N); cp_out(h->dvof, P->dvof, N); cp_out(h->vof2, P->vof2, N);
    cp_out(h->sxx, P->sxx, N); cp_out(h->sxy, P->sxy, N); cp_out(h->syy, P->syy, N);
    cp_out(h->dsxx, P->dsxx, N); cp_out(h->dsxy, P->dsxy, N); cp_out(h->dsyy, P->dsyy, N); cp_out(h->dp, P->dp, N);
    cp_out(h->sxx_min, P->sxx_min, N); cp_out(h->sxy_min, P->sxy_min, N); cp_out(h->syy_min, P->syy_min, N);
    cp_out(h->p_min, P->p_min, N); cp_out(h->epsilon_p, P->epsilon_p, N); cp_out(h->vcc, P->vcc, N);
    cp_out(h->txx, P->txx, N); cp_out(h->tyy, P->tyy, N); cp_out(h->txy, P->txy, N);
    if (h->itype) for (size_t i = 0; i < N; ++i) h->itype[i] = P->itype[i];
    if (h->fail) for (size_t i = 0; i < N; ++i) h->fail[i] = P->fail[i];
    return 0;
}

/* 1-based (i,j) of the last step's lists, in the reference's own order
 * (which for direct_find / direct_find_2 is sorted by i then j). */
int64_t or_export_pairs(or_ctx* C, int which, int32_t* pi, int32_t* pj, int64_t cap) {
    if (!C || which < 0 || which > 2) return -1;
    int64_t n = C->save_n[which];
    for (int64_t k = 0; k < n && k < cap; ++k) { pi[k] = C->save_i[which][k] + 1; pj[k] = C->save_j[which][k] + 1; }
    return n;
}

int or_nfail(or_ctx* C, int phase) { return (C && phase >= 1 && phase <= C->nphase) ? C->ph[phase - 1].nfail : -1; }

void or_destroy(or_ctx* C) {
    if (!C) return;
    for (int k = 0; k < 2; ++k) if (C->ph[k].x) phase_free(&C->ph[k]);
    free(C->wtxx); free(C->wtyy); free(C->wtxy);
    free(C->pair_i); free(C->pair_j); free(C->w); free(C->dwdx);
    for (int k = 0; k < 3; ++k) { free(C->save_i[k]); free(C->save_j[k]); }
    free(C);
}
