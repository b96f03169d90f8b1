/*
 * jv_oracle.c -- CPU restatement of the jarvis elastic FDTD modelling and
 * VOWR RTM path.  TEST INFRASTRUCTURE ONLY (see jv_oracle.h): the CUDA
 * product never links or calls this file.
 *
 * The arithmetic follows the reference kernels term by term; the only
 * intended differences are the working precision (JVO_REAL) and the data
 * layout (dense x-fastest extended grid, memory variables held on the full
 * extended grid and used only where the reference allocates them).
 *
 * Reference paths below are relative to the reference project root, with
 *   FD  = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/
 *         elastic_1_fdtd3d_model_mpi
 *   RTM = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/
 *         elastic_1_rtm3d_model_mpi
 */
#include "jv_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef JVO_REAL
#define JVO_REAL double
#endif
typedef JVO_REAL real;

#define PHY_HALF 4 /* GeoConst::phy_fdorder_half, FD/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp:13 */
#define PML_HALF 2 /* GeoConst::pml_fdorder_half, :14 */

enum { M_FWD = 0, M_RTMF = 1, M_BWD = 2, M_REV = 3 };
enum { VX, VY, VZ, SXX, SYY, SZZ, SXY, SXZ, SYZ, SAU, VXP, VYP, VZP, NFLD };
/* velocity memory variables (one per stress derivative feeding v) */
enum { PV_SXX_X, PV_SXY_Y, PV_SXZ_Z, PV_SXY_X, PV_SYY_Y, PV_SYZ_Z, PV_SXZ_X, PV_SYZ_Y, PV_SZZ_Z, NPV };
/* stress memory variables (one per velocity derivative) */
enum { PS_VX_X, PS_VY_Y, PS_VZ_Z, PS_VY_X, PS_VX_Y, PS_VZ_X, PS_VX_Z, PS_VZ_Y, PS_VY_Z, NPS };

typedef struct {
    int nx, ny, nz; /* extended */
    int m;          /* margin */
    int px, py, pz; /* physical */
    size_t sy, sz, n;
    real dx, dy, dz, dt;
    float fdx, fdy, fdz, fdt, ffm;
    float lx, ly, lz; /* gridext l_rows/l_cols/l_slices (float, as Frame) */
} grid_t;

typedef struct {
    real *f[NFLD];
    real *pv[NPV];
    real *ps[NPS];
} wave_t;

typedef struct {
    real *rho, *lam, *mu;
    float *vp;
} model_t;

typedef struct {
    real dc4[4], dc2[2];
    real list[5][4]; /* list[o] = coefficients of half-order o (1..4) */
} coef_t;

/* ------------------------------------------------------------------ */
/* small helpers                                                      */
/* ------------------------------------------------------------------ */

int jvo_ntime(float T, float dt)
{
    /* ntime = ceil(T / dt) in float: fdtd3d_base_4_seisrecord_meat.hpp:278 */
    float q = T / dt;
    return (int)ceilf(q);
}

void jvo_diff_coeff(int order, double *c)
{
    /* jarvis_device_geometry_bones.hpp:29-49 */
    for (int n = 0; n < order; n++) {
        double a1 = 1, a2 = 1, a3 = 1;
        for (int i = 0; i < order; i++) {
            if (i != n) a1 = a1 * (2 * i + 1) * (2 * i + 1);
            if (i < n) a2 = a2 * ((2 * n + 1) * (2 * n + 1) - (2 * i + 1) * (2 * i + 1));
            if (i > n) a3 = a3 * ((2 * i + 1) * (2 * i + 1) - (2 * n + 1) * (2 * n + 1));
        }
        a1 = a1 * ((n % 2) ? -1.0 : 1.0);
        c[n] = a1 / ((2 * n + 1) * a2 * a3);
    }
}

void jvo_ricker(int nt, float fm, float dt, float *w)
{
    /* fdtd3d_base_4_seisrecord_meat.hpp:279-285: the time argument is a
     * float product, pi is double, the value is stored as float. */
    const double pi = 3.14159265358979323846;
    float dura = 1.3f / fm;
    int n0 = (int)floorf(dura / dt + 0.5f);
    for (int i = 0; i < nt; i++) {
        float t = (float)(i - n0) * dt;
        double a = pi * (double)fm * (double)t;
        double a2 = a * a;
        w[i] = (float)(1.0e4 * (1.0 - 2.0 * a2) * exp(-a2));
    }
}

int jvo_gap_num(float l, float r, float d)
{
    /* jarvis_3_device_field_meat.hpp:9-22 */
    int n_l, n_r;
    float v = 1.0f / d;
    if (l > 0) n_l = (int)(l * v + 0.125f);
    else n_l = (int)(l * v - 0.125f);
    if (r > 0) n_r = (int)(r * v + 0.125f);
    else n_r = (int)(r * v - 0.125f);
    return n_r - n_l;
}

int jvo_cpml_ab(int c, int n, int m, float vp, float delta, float fm, float dt, double *out)
{
    /* fdtd3d_cpml_mpi_1_host_meat.hpp:147-620 (one axis, one cell).
     * Low side (top/front/right):  s = m - c,            s_half = m - c - 0.5
     * High side (bottom/back/left): s = c-(n-m-1) - 0.5, s_half = c-(n-m-1)  */
    const double pi = 3.14159265358979323846;
    double s, sh;
    out[0] = 0.0; out[1] = 1.0; out[2] = 0.0; out[3] = 1.0;
    if (c >= PML_HALF && c < m) {
        s = (double)(m - c);
        sh = (double)(m - c) - 0.5;
    } else if (c >= n - m && c < n - PML_HALF) {
        s = (double)(c - (n - m - 1)) - 0.5;
        sh = (double)(c - (n - m - 1));
    } else {
        return 0;
    }
    double N = (double)(m - PML_HALF);
    double R = (double)0.001f;
    double l10 = (double)log10f(1.0f / (float)R);
    double temp = l10 * 7.0 * (double)vp / (2.0 * N * (double)delta);
    double d = temp * (s / N) * (s / N);
    double dh = temp * (sh / N) * (sh / N);
    double al = pi * (double)fm * (1.0 - s / N);
    double alh = pi * (double)fm * (1.0 - sh / N);
    if (al < 0) al = 0;
    if (alh < 0) alh = 0;
    double b = exp(-(d + al) * (double)dt);
    double bh = exp(-(dh + alh) * (double)dt);
    double a = 0.0, ah = 0.0;
    if (fabs(d) >= 1e-8) {
        a = d * (b - 1.0) / (d + al);
        ah = dh * (bh - 1.0) / (dh + alh);
    }
    out[0] = a; out[1] = b; out[2] = ah; out[3] = bh;
    return 1;
}

static int inside_phy(const jvo_problem *p, const float *q)
{
    /* gridphy: l = 0, r = (n-1)*d (Frame::Frame, jarvis_0_frame_meat.hpp:28-67) */
    float rx = (float)(p->nx - 1) * p->dx, ry = (float)(p->ny - 1) * p->dy, rz = (float)(p->nz - 1) * p->dz;
    return q[0] >= 0.0f && q[0] <= rx && q[1] >= 0.0f && q[1] <= ry && q[2] >= 0.0f && q[2] <= rz;
}

int jvo_select_inside(const jvo_problem *p, const float *xyz, int n, int *idx)
{
    int c = 0;
    for (int i = 0; i < n; i++)
        if (inside_phy(p, xyz + 3 * i)) {
            if (idx) idx[c] = i;
            c++;
        }
    return c;
}

static void make_grid(const jvo_problem *p, grid_t *g)
{
    g->m = p->pml;
    g->px = p->nx; g->py = p->ny; g->pz = p->nz;
    g->nx = p->nx + 2 * p->pml; g->ny = p->ny + 2 * p->pml; g->nz = p->nz + 2 * p->pml;
    g->sy = (size_t)g->nx;
    g->sz = (size_t)g->nx * (size_t)g->ny;
    g->n = g->sz * (size_t)g->nz;
    g->fdx = p->dx; g->fdy = p->dy; g->fdz = p->dz; g->fdt = p->dt; g->ffm = p->fm;
    g->dx = p->dx; g->dy = p->dy; g->dz = p->dz; g->dt = p->dt;
    g->lx = -(float)p->pml * p->dx;
    g->ly = -(float)p->pml * p->dy;
    g->lz = -(float)p->pml * p->dz;
}

static void make_coef(coef_t *c)
{
    double t[4];
    jvo_diff_coeff(4, t);
    for (int i = 0; i < 4; i++) c->dc4[i] = (real)t[i];
    jvo_diff_coeff(2, t);
    c->dc2[0] = (real)t[0]; c->dc2[1] = (real)t[1];
    memset(c->list, 0, sizeof(c->list));
    for (int o = 1; o <= 4; o++) {
        jvo_diff_coeff(o, t);
        for (int i = 0; i < o; i++) c->list[o][i] = (real)t[i];
    }
}

/* Extension into the PML by nearest-cell copy (the 26 regions of
 * fdtd3d_base_3_geomodel_meat.hpp:101-364 reduce to index clamping). */
static void extend(const grid_t *g, const float *phy, float *ext)
{
    for (int k = 0; k < g->nz; k++) {
        int pk = k - g->m; if (pk < 0) pk = 0; if (pk > g->pz - 1) pk = g->pz - 1;
        for (int j = 0; j < g->ny; j++) {
            int pj = j - g->m; if (pj < 0) pj = 0; if (pj > g->py - 1) pj = g->py - 1;
            for (int i = 0; i < g->nx; i++) {
                int pi_ = i - g->m; if (pi_ < 0) pi_ = 0; if (pi_ > g->px - 1) pi_ = g->px - 1;
                ext[(size_t)i + g->sy * j + g->sz * k] =
                    phy[(size_t)pi_ + (size_t)g->px * ((size_t)pj + (size_t)g->py * pk)];
            }
        }
    }
}

static int make_model(const grid_t *g, const float *vp, const float *vs, const float *rho, model_t *md)
{
    float *evp = (float *)malloc(g->n * sizeof(float));
    float *evs = (float *)malloc(g->n * sizeof(float));
    float *erho = (float *)malloc(g->n * sizeof(float));
    md->rho = (real *)malloc(g->n * sizeof(real));
    md->lam = (real *)malloc(g->n * sizeof(real));
    md->mu = (real *)malloc(g->n * sizeof(real));
    if (!evp || !evs || !erho || !md->rho || !md->lam || !md->mu) return -1;
    extend(g, vp, evp);
    extend(g, vs, evs);
    extend(g, rho, erho);
    /* lambda = rho (vp^2 - 2 vs^2), mu = rho vs^2 (geomodel_meat.hpp:454-460) */
    for (size_t i = 0; i < g->n; i++) {
        real r = erho[i], a = evp[i], b = evs[i];
        md->rho[i] = r;
        md->lam[i] = r * (a * a - (real)2 * b * b);
        md->mu[i] = r * (b * b);
    }
    md->vp = evp;
    free(evs);
    free(erho);
    return 0;
}

static void free_model(model_t *md)
{
    free(md->rho); free(md->lam); free(md->mu); free(md->vp);
}

static int alloc_wave(const grid_t *g, wave_t *w, int with_psi)
{
    memset(w, 0, sizeof(*w));
    for (int f = 0; f < NFLD; f++) {
        w->f[f] = (real *)calloc(g->n, sizeof(real));
        if (!w->f[f]) return -1;
    }
    if (with_psi) {
        for (int f = 0; f < NPV; f++) {
            w->pv[f] = (real *)calloc(g->n, sizeof(real));
            if (!w->pv[f]) return -1;
        }
        for (int f = 0; f < NPS; f++) {
            w->ps[f] = (real *)calloc(g->n, sizeof(real));
            if (!w->ps[f]) return -1;
        }
    }
    return 0;
}

static void free_wave(wave_t *w)
{
    for (int f = 0; f < NFLD; f++) free(w->f[f]);
    for (int f = 0; f < NPV; f++) free(w->pv[f]);
    for (int f = 0; f < NPS; f++) free(w->ps[f]);
}

/* staggered differences: Dp = sum c_r (f[i+(r+1)s] - f[i-rs]),
 *                        Dm = sum c_r (f[i+rs]     - f[i-(r+1)s]) */
static inline real Dp(const real *f, size_t i, size_t s, const real *c, int o)
{
    real t = 0;
    for (int r = 0; r < o; r++) t += c[r] * (f[i + (size_t)(r + 1) * s] - f[i - (size_t)r * s]);
    return t;
}
static inline real Dm(const real *f, size_t i, size_t s, const real *c, int o)
{
    real t = 0;
    for (int r = 0; r < o; r++) t += c[r] * (f[i + (size_t)r * s] - f[i - (size_t)(r + 1) * s]);
    return t;
}

/* Order of one axis of the interior update.  Full 8th order except in the
 * rtm_backward rim, where the order drops so that the stencil reaches at
 * most rec_width layers outside gridphy
 * (FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_2_vel_kernel.hpp:132-152,
 * 240-261; the same selection in every edge kernel). */
static inline void axis_order(const coef_t *cf, int mode, int w, int p, int np, const real **c, int *o)
{
    *c = cf->dc4;
    *o = PHY_HALF;
    if (mode != M_BWD) return;
    int e;
    if (p < PHY_HALF) e = p;
    else if (np - 1 - p < PHY_HALF) e = np - 1 - p;
    else return;
    int ord = (e < w) ? w : e + 1;
    *c = cf->list[ord];
    *o = ord;
}

/* ------------------------------------------------------------------ */
/* interior (gridphy) updates                                          */
/* ------------------------------------------------------------------ */

/* sub_update_vel_phy_domain_inside + edge kernels
 * (FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_2_vel_kernel.hpp:7-80) */
static void vel_interior(const grid_t *g, const coef_t *cf, const model_t *md, wave_t *w, int mode, int rec_w, real dt)
{
    real *vx = w->f[VX], *vy = w->f[VY], *vz = w->f[VZ];
    const real *sxx = w->f[SXX], *syy = w->f[SYY], *szz = w->f[SZZ];
    const real *sxy = w->f[SXY], *sxz = w->f[SXZ], *syz = w->f[SYZ], *sau = w->f[SAU];
    real *vxp = w->f[VXP], *vyp = w->f[VYP], *vzp = w->f[VZP];
    const size_t sy = g->sy, sz = g->sz;
    const int with_p = (mode == M_BWD || mode == M_REV);
#pragma omp parallel for schedule(static)
    for (int pk = 0; pk < g->pz; pk++) {
        const real *cz; int oz;
        axis_order(cf, mode, rec_w, pk, g->pz, &cz, &oz);
        for (int pj = 0; pj < g->py; pj++) {
            const real *cy; int oy;
            axis_order(cf, mode, rec_w, pj, g->py, &cy, &oy);
            for (int pi_ = 0; pi_ < g->px; pi_++) {
                const real *cx; int ox;
                axis_order(cf, mode, rec_w, pi_, g->px, &cx, &ox);
                size_t i = (size_t)(pi_ + g->m) + sy * (pj + g->m) + sz * (pk + g->m);
                real dtr = dt / md->rho[i];
                real a = dtr / g->dx, b = dtr / g->dy, c = dtr / g->dz;
                real sxx_x = Dp(sxx, i, 1, cx, ox);
                real syx_x = Dm(sxy, i, 1, cx, ox);
                real szx_x = Dm(sxz, i, 1, cx, ox);
                real sxy_y = Dm(sxy, i, sy, cy, oy);
                real syy_y = Dp(syy, i, sy, cy, oy);
                real szy_y = Dm(syz, i, sy, cy, oy);
                real sxz_z = Dm(sxz, i, sz, cz, oz);
                real syz_z = Dm(syz, i, sz, cz, oz);
                real szz_z = Dp(szz, i, sz, cz, oz);
                vx[i] += a * sxx_x + b * sxy_y + c * sxz_z;
                vy[i] += a * syx_x + b * syy_y + c * syz_z;
                vz[i] += a * szx_x + b * szy_y + c * szz_z;
                if (with_p) {
                    vxp[i] += a * Dp(sau, i, 1, cx, ox);
                    vyp[i] += b * Dp(sau, i, sy, cy, oy);
                    vzp[i] += c * Dp(sau, i, sz, cz, oz);
                }
            }
        }
    }
}

/* sub_update_stress_phy_domain_inside + edge kernels
 * (FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_3_stress_kernel.hpp:7-60) */
static void stress_interior(const grid_t *g, const coef_t *cf, const model_t *md, wave_t *w, int mode, int rec_w, real dt)
{
    const real *vx = w->f[VX], *vy = w->f[VY], *vz = w->f[VZ];
    real *sxx = w->f[SXX], *syy = w->f[SYY], *szz = w->f[SZZ];
    real *sxy = w->f[SXY], *sxz = w->f[SXZ], *syz = w->f[SYZ], *sau = w->f[SAU];
    const size_t sy = g->sy, sz = g->sz;
    const int with_sau = (mode != M_FWD);
#pragma omp parallel for schedule(static)
    for (int pk = 0; pk < g->pz; pk++) {
        const real *cz; int oz;
        axis_order(cf, mode, rec_w, pk, g->pz, &cz, &oz);
        for (int pj = 0; pj < g->py; pj++) {
            const real *cy; int oy;
            axis_order(cf, mode, rec_w, pj, g->py, &cy, &oy);
            for (int pi_ = 0; pi_ < g->px; pi_++) {
                const real *cx; int ox;
                axis_order(cf, mode, rec_w, pi_, g->px, &cx, &ox);
                size_t i = (size_t)(pi_ + g->m) + sy * (pj + g->m) + sz * (pk + g->m);
                real a = dt / g->dx, b = dt / g->dy, c = dt / g->dz;
                real l = md->lam[i], mu = md->mu[i];
                real l2m = l + (real)2 * mu;
                real vx_x = Dm(vx, i, 1, cx, ox);
                real vy_x = Dp(vy, i, 1, cx, ox);
                real vz_x = Dp(vz, i, 1, cx, ox);
                real vx_y = Dp(vx, i, sy, cy, oy);
                real vy_y = Dm(vy, i, sy, cy, oy);
                real vz_y = Dp(vz, i, sy, cy, oy);
                real vx_z = Dp(vx, i, sz, cz, oz);
                real vy_z = Dp(vy, i, sz, cz, oz);
                real vz_z = Dm(vz, i, sz, cz, oz);
                sxx[i] += a * l2m * vx_x + b * l * vy_y + c * l * vz_z;
                syy[i] += a * l * vx_x + b * l2m * vy_y + c * l * vz_z;
                szz[i] += a * l * vx_x + b * l * vy_y + c * l2m * vz_z;
                sxy[i] += a * mu * vy_x + b * mu * vx_y;
                sxz[i] += a * mu * vz_x + c * mu * vx_z;
                syz[i] += b * mu * vz_y + c * mu * vy_z;
                if (with_sau) sau[i] += a * l2m * vx_x + b * l2m * vy_y + c * l2m * vz_z;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* CPML (absorbing layer) updates                                     */
/* ------------------------------------------------------------------ */

static inline int in_pml_cell(const grid_t *g, int i, int j, int k)
{
    if (i < PML_HALF || i >= g->nx - PML_HALF) return 0;
    if (j < PML_HALF || j >= g->ny - PML_HALF) return 0;
    if (k < PML_HALF || k >= g->nz - PML_HALF) return 0;
    int phy = (i >= g->m && i < g->nx - g->m) && (j >= g->m && j < g->ny - g->m) && (k >= g->m && k < g->nz - g->m);
    return !phy;
}

/* The six slab kernels of FD/fdtd3d_1_cpml_mpi_module cover every cell of
 * the extended grid outside gridphy and outside the 2-cell outer rim; each
 * applies a memory variable to the derivatives along the axes on which
 * the cell lies inside that axis' absorbing range (z-slabs: x,y,z;
 * y-slabs: x,y; x-slabs: x; coefficients are a=0, b=1 elsewhere). */
static void vel_pml(const grid_t *g, const coef_t *cf, const model_t *md, wave_t *w)
{
    real *vx = w->f[VX], *vy = w->f[VY], *vz = w->f[VZ];
    const real *sxx = w->f[SXX], *syy = w->f[SYY], *szz = w->f[SZZ];
    const real *sxy = w->f[SXY], *sxz = w->f[SXZ], *syz = w->f[SYZ];
    const size_t sy = g->sy, sz = g->sz;
    const real *c2 = cf->dc2;
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = PML_HALF; k < g->nz - PML_HALF; k++) {
        for (int j = PML_HALF; j < g->ny - PML_HALF; j++) {
            for (int i = PML_HALF; i < g->nx - PML_HALF; i++) {
                if (!in_pml_cell(g, i, j, k)) continue;
                size_t idx = (size_t)i + sy * j + sz * k;
                float vp = md->vp[idx];
                double ax[4], ay[4], az[4];
                int xa = jvo_cpml_ab(i, g->nx, g->m, vp, g->fdx, g->ffm, g->fdt, ax);
                int ya = jvo_cpml_ab(j, g->ny, g->m, vp, g->fdy, g->ffm, g->fdt, ay);
                int za = jvo_cpml_ab(k, g->nz, g->m, vp, g->fdz, g->ffm, g->fdt, az);
                /* FD/fdtd3d_1_cpml_mpi_module/fdtd3d_cpml_mpi_2_kernel_device_z_meat.hpp:9-196 */
                real sxx_x = Dp(sxx, idx, 1, c2, 2) / g->dx;
                real syx_x = Dm(sxy, idx, 1, c2, 2) / g->dx;
                real szx_x = Dm(sxz, idx, 1, c2, 2) / g->dx;
                real sxy_y = Dm(sxy, idx, sy, c2, 2) / g->dy;
                real syy_y = Dp(syy, idx, sy, c2, 2) / g->dy;
                real szy_y = Dm(syz, idx, sy, c2, 2) / g->dy;
                real sxz_z = Dm(sxz, idx, sz, c2, 2) / g->dz;
                real syz_z = Dm(syz, idx, sz, c2, 2) / g->dz;
                real szz_z = Dp(szz, idx, sz, c2, 2) / g->dz;
                if (xa) {
                    real *p0 = &w->pv[PV_SXX_X][idx], *p1 = &w->pv[PV_SXY_X][idx], *p2 = &w->pv[PV_SXZ_X][idx];
                    *p0 = (real)ax[3] * *p0 + (real)ax[2] * sxx_x; sxx_x += *p0;
                    *p1 = (real)ax[1] * *p1 + (real)ax[0] * syx_x; syx_x += *p1;
                    *p2 = (real)ax[1] * *p2 + (real)ax[0] * szx_x; szx_x += *p2;
                }
                if (ya) {
                    real *p0 = &w->pv[PV_SXY_Y][idx], *p1 = &w->pv[PV_SYY_Y][idx], *p2 = &w->pv[PV_SYZ_Y][idx];
                    *p0 = (real)ay[1] * *p0 + (real)ay[0] * sxy_y; sxy_y += *p0;
                    *p1 = (real)ay[3] * *p1 + (real)ay[2] * syy_y; syy_y += *p1;
                    *p2 = (real)ay[1] * *p2 + (real)ay[0] * szy_y; szy_y += *p2;
                }
                if (za) {
                    real *p0 = &w->pv[PV_SXZ_Z][idx], *p1 = &w->pv[PV_SYZ_Z][idx], *p2 = &w->pv[PV_SZZ_Z][idx];
                    *p0 = (real)az[1] * *p0 + (real)az[0] * sxz_z; sxz_z += *p0;
                    *p1 = (real)az[1] * *p1 + (real)az[0] * syz_z; syz_z += *p1;
                    *p2 = (real)az[3] * *p2 + (real)az[2] * szz_z; szz_z += *p2;
                }
                real dtr = g->dt / md->rho[idx];
                vx[idx] += dtr * (sxx_x + sxy_y + sxz_z);
                vy[idx] += dtr * (syx_x + syy_y + syz_z);
                vz[idx] += dtr * (szx_x + szy_y + szz_z);
            }
        }
    }
}

static void stress_pml(const grid_t *g, const coef_t *cf, const model_t *md, wave_t *w)
{
    const real *vx = w->f[VX], *vy = w->f[VY], *vz = w->f[VZ];
    real *sxx = w->f[SXX], *syy = w->f[SYY], *szz = w->f[SZZ];
    real *sxy = w->f[SXY], *sxz = w->f[SXZ], *syz = w->f[SYZ], *sau = w->f[SAU];
    const size_t sy = g->sy, sz = g->sz;
    const real *c2 = cf->dc2;
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = PML_HALF; k < g->nz - PML_HALF; k++) {
        for (int j = PML_HALF; j < g->ny - PML_HALF; j++) {
            for (int i = PML_HALF; i < g->nx - PML_HALF; i++) {
                if (!in_pml_cell(g, i, j, k)) continue;
                size_t idx = (size_t)i + sy * j + sz * k;
                float vp = md->vp[idx];
                double ax[4], ay[4], az[4];
                int xa = jvo_cpml_ab(i, g->nx, g->m, vp, g->fdx, g->ffm, g->fdt, ax);
                int ya = jvo_cpml_ab(j, g->ny, g->m, vp, g->fdy, g->ffm, g->fdt, ay);
                int za = jvo_cpml_ab(k, g->nz, g->m, vp, g->fdz, g->ffm, g->fdt, az);
                /* FD/fdtd3d_1_cpml_mpi_module/fdtd3d_cpml_mpi_2_kernel_device_z_meat.hpp:198-391 */
                real vx_x = Dm(vx, idx, 1, c2, 2) / g->dx;
                real vy_x = Dp(vy, idx, 1, c2, 2) / g->dx;
                real vz_x = Dp(vz, idx, 1, c2, 2) / g->dx;
                real vx_y = Dp(vx, idx, sy, c2, 2) / g->dy;
                real vy_y = Dm(vy, idx, sy, c2, 2) / g->dy;
                real vz_y = Dp(vz, idx, sy, c2, 2) / g->dy;
                real vx_z = Dp(vx, idx, sz, c2, 2) / g->dz;
                real vy_z = Dp(vy, idx, sz, c2, 2) / g->dz;
                real vz_z = Dm(vz, idx, sz, c2, 2) / g->dz;
                if (xa) {
                    real *p0 = &w->ps[PS_VX_X][idx], *p1 = &w->ps[PS_VY_X][idx], *p2 = &w->ps[PS_VZ_X][idx];
                    *p0 = (real)ax[1] * *p0 + (real)ax[0] * vx_x; vx_x += *p0;
                    *p1 = (real)ax[3] * *p1 + (real)ax[2] * vy_x; vy_x += *p1;
                    *p2 = (real)ax[3] * *p2 + (real)ax[2] * vz_x; vz_x += *p2;
                }
                if (ya) {
                    real *p0 = &w->ps[PS_VY_Y][idx], *p1 = &w->ps[PS_VX_Y][idx], *p2 = &w->ps[PS_VZ_Y][idx];
                    *p0 = (real)ay[1] * *p0 + (real)ay[0] * vy_y; vy_y += *p0;
                    *p1 = (real)ay[3] * *p1 + (real)ay[2] * vx_y; vx_y += *p1;
                    *p2 = (real)ay[3] * *p2 + (real)ay[2] * vz_y; vz_y += *p2;
                }
                if (za) {
                    real *p0 = &w->ps[PS_VZ_Z][idx], *p1 = &w->ps[PS_VX_Z][idx], *p2 = &w->ps[PS_VY_Z][idx];
                    *p0 = (real)az[1] * *p0 + (real)az[0] * vz_z; vz_z += *p0;
                    *p1 = (real)az[3] * *p1 + (real)az[2] * vx_z; vx_z += *p1;
                    *p2 = (real)az[3] * *p2 + (real)az[2] * vy_z; vy_z += *p2;
                }
                real l = md->lam[idx], mu = md->mu[idx];
                real l2m = l + (real)2 * mu;
                real dt = g->dt;
                sxx[idx] += dt * (l2m * vx_x + l * vy_y + l * vz_z);
                syy[idx] += dt * (l * vx_x + l2m * vy_y + l * vz_z);
                szz[idx] += dt * (l * vx_x + l * vy_y + l2m * vz_z);
                sau[idx] += dt * (l2m * vx_x + l2m * vy_y + l2m * vz_z);
                sxy[idx] += dt * mu * (vy_x + vx_y);
                sxz[idx] += dt * mu * (vz_x + vx_z);
                syz[idx] += dt * mu * (vz_y + vy_z);
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* VOWR boundary store                                                 */
/* ------------------------------------------------------------------ */

/* Face widths per field (top, bottom, front, back, right, left) for
 * rec_width w: FD/fdtd3d_0_base_module/fdtd3d_base_5_wave_recon_meat.hpp:19-30 */
typedef struct { int fld; int x0, x1, y0, y1, z0, z1; } box_t;

static int vowr_boxes(const grid_t *g, int w, box_t *out)
{
    static const int flds[10] = {VX, VY, VZ, SXX, SYY, SZZ, SAU, SXY, SXZ, SYZ};
    int W[10][6] = {
        {w - 1, w, w - 1, w, w, w - 1}, /* vx  */
        {w - 1, w, w, w - 1, w - 1, w}, /* vy  */
        {w, w - 1, w - 1, w, w - 1, w}, /* vz  */
        {0, 0, 0, 0, w - 1, w},         /* sxx */
        {0, 0, w - 1, w, 0, 0},         /* syy */
        {w - 1, w, 0, 0, 0, 0},         /* szz */
        {w - 1, w, w - 1, w, w - 1, w}, /* sau */
        {0, 0, w, w - 1, w, w - 1},     /* sxy */
        {w, w - 1, 0, 0, w, w - 1},     /* sxz */
        {w, w - 1, w, w - 1, 0, 0},     /* syz */
    };
    int nb = 0;
    int X0 = g->m, X1 = g->m + g->px, Y0 = g->m, Y1 = g->m + g->py, Z0 = g->m, Z1 = g->m + g->pz;
    for (int f = 0; f < 10; f++) {
        for (int face = 0; face < 6; face++) {
            int wd = W[f][face];
            if (wd <= 0) continue;
            box_t b = {flds[f], X0, X1, Y0, Y1, Z0, Z1};
            /* jarvis_1_mpicu_halo_store_operator_meat.hpp:129-134 */
            switch (face) {
            case 0: b.z0 = Z0 - wd; b.z1 = Z0; break;
            case 1: b.z0 = Z1; b.z1 = Z1 + wd; break;
            case 2: b.y0 = Y0 - wd; b.y1 = Y0; break;
            case 3: b.y0 = Y1; b.y1 = Y1 + wd; break;
            case 4: b.x0 = X0 - wd; b.x1 = X0; break;
            default: b.x0 = X1; b.x1 = X1 + wd; break;
            }
            if (out) out[nb] = b;
            nb++;
        }
    }
    return nb;
}

static size_t boxes_size(const box_t *b, int nb)
{
    size_t s = 0;
    for (int i = 0; i < nb; i++) s += (size_t)(b[i].x1 - b[i].x0) * (b[i].y1 - b[i].y0) * (b[i].z1 - b[i].z0);
    return s;
}

static void box_copy(const grid_t *g, wave_t *w, const box_t *b, int nb, real *buf, int pack, int only_vel, int only_stress)
{
    size_t o = 0;
    for (int q = 0; q < nb; q++) {
        const box_t *x = &b[q];
        size_t cnt = (size_t)(x->x1 - x->x0) * (x->y1 - x->y0) * (x->z1 - x->z0);
        int isvel = (x->fld == VX || x->fld == VY || x->fld == VZ);
        if ((only_vel && !isvel) || (only_stress && isvel)) { o += cnt; continue; }
        real *f = w->f[x->fld];
        for (int k = x->z0; k < x->z1; k++)
            for (int j = x->y0; j < x->y1; j++)
                for (int i = x->x0; i < x->x1; i++) {
                    size_t idx = (size_t)i + g->sy * j + g->sz * k;
                    if (pack) buf[o] = f[idx];
                    else f[idx] = buf[o];
                    o++;
                }
    }
}

/* ------------------------------------------------------------------ */
/* shot geometry                                                       */
/* ------------------------------------------------------------------ */

static size_t ext_index_of(const grid_t *g, const float *q)
{
    /* get_gap_num against gridext (seisrecord_meat.hpp:67-70,
     * stress_kernel.hpp:1328-1331) */
    int i = jvo_gap_num(g->lx, q[0], g->fdx);
    int j = jvo_gap_num(g->ly, q[1], g->fdy);
    int k = jvo_gap_num(g->lz, q[2], g->fdz);
    return (size_t)i + g->sy * j + g->sz * k;
}

static void set_threads(const jvo_problem *p)
{
#ifdef _OPENMP
    if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#else
    (void)p;
#endif
}

typedef struct {
    grid_t g;
    coef_t cf;
    model_t md;
    int nt;
    float *wl;
    int nrec;
    size_t *rec_idx;
    size_t src_idx;
} ctx_t;

static int ctx_init(ctx_t *c, const jvo_problem *p, const float *vp, const float *vs, const float *rho, int shot)
{
    memset(c, 0, sizeof(*c));
    if (p->nx < 8 || p->ny < 8 || p->nz < 8 || p->pml < PHY_HALF) return -2;
    if (shot < 0 || shot >= p->n_shot) return -3;
    if (!inside_phy(p, p->shot_xyz + 3 * shot)) return -3;
    set_threads(p);
    make_grid(p, &c->g);
    make_coef(&c->cf);
    if (make_model(&c->g, vp, vs, rho, &c->md)) return -1;
    c->nt = jvo_ntime(p->T, p->dt);
    c->wl = (float *)malloc(sizeof(float) * (size_t)(c->nt > 0 ? c->nt : 1));
    jvo_ricker(c->nt, p->fm, p->dt, c->wl);
    int *sel = (int *)malloc(sizeof(int) * (size_t)(p->n_recv > 0 ? p->n_recv : 1));
    c->nrec = jvo_select_inside(p, p->recv_xyz, p->n_recv, sel);
    c->rec_idx = (size_t *)malloc(sizeof(size_t) * (size_t)(c->nrec > 0 ? c->nrec : 1));
    for (int r = 0; r < c->nrec; r++) c->rec_idx[r] = ext_index_of(&c->g, p->recv_xyz + 3 * sel[r]);
    free(sel);
    c->src_idx = ext_index_of(&c->g, p->shot_xyz + 3 * shot);
    return 0;
}

static void ctx_free(ctx_t *c)
{
    free_model(&c->md);
    free(c->wl);
    free(c->rec_idx);
}

/* ------------------------------------------------------------------ */
/* storage-precision study (jvo_set_store16; off by default)          */
/* ------------------------------------------------------------------ */

static int g_store16 = 0;

void jvo_set_store16(int mode) { g_store16 = (mode == 1 || mode == 2) ? mode : 0; }

/* x rounded to 16 bits: FP16 by the compiler's round-to-nearest-even
 * conversion, BF16 by round-to-nearest-even on the upper half of the
 * FP32 bit pattern */
static inline float round16(float x)
{
    if (g_store16 == 1) return (float)(_Float16)x;
    uint32_t u;
    memcpy(&u, &x, 4);
    u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    memcpy(&x, &u, 4);
    return x;
}

/* fields f0..f1 of w as 16-bit storage would hold them: per z plane of
 * gridext a power-of-two scale s (FP16: largest magnitude / s in
 * (2^11, 2^12]; BF16: in (1/2, 1]), values v -> s * round16(v / s) */
static void store16(const grid_t *g, wave_t *w, int f0, int f1)
{
    if (!g_store16) return;
    for (int f = f0; f <= f1; f++) {
        real *a = w->f[f];
#pragma omp parallel for schedule(static)
        for (int k = 0; k < g->nz; k++) {
            real *p = a + g->sz * (size_t)k;
            double amax = 0;
            for (size_t i = 0; i < g->sz; i++) amax = fmax(amax, fabs((double)p[i]));
            if (amax == 0) continue;
            int e;
            frexp(amax, &e);
            if (e < -100) e = -100;  /* keep 1/s finite for subnormal planes */
            const float s = ldexpf(1.0f, g_store16 == 1 ? e - 12 : e), inv = 1.0f / s;
            for (size_t i = 0; i < g->sz; i++) p[i] = (real)(s * round16((float)p[i] * inv));
        }
    }
}

static void add_source(wave_t *w, size_t s, real a)
{
    /* sub_add_stress_source / sub_subtract_stress_source
     * (FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_3_stress_kernel.hpp:1308-1364) */
    w->f[SXX][s] += a;
    w->f[SYY][s] += a;
    w->f[SZZ][s] += a;
}

/* One forward time step, mode FWD (pure_forward) or RTMF (rtm_forward):
 * FD/fdtd3d_3_model_mpi_blend/fdtd3d_blend_elastic_model_mpi_meat.hpp:51-79
 * and :130-146.  store != NULL packs the VOWR layers after the CPML
 * stress update (:141-142). */
static void step_forward(ctx_t *c, wave_t *w, int it, int mode, const box_t *bx, int nb, real *store)
{
    vel_pml(&c->g, &c->cf, &c->md, w);
    vel_interior(&c->g, &c->cf, &c->md, w, mode, PHY_HALF, c->g.dt);
    store16(&c->g, w, VX, VZ);
    add_source(w, c->src_idx, (real)c->wl[it]);
    stress_pml(&c->g, &c->cf, &c->md, w);
    if (store) box_copy(&c->g, w, bx, nb, store, 1, 0, 0);
    stress_interior(&c->g, &c->cf, &c->md, w, mode, PHY_HALF, c->g.dt);
    store16(&c->g, w, SXX, SAU);
}

int jvo_forward(const jvo_problem *p, const float *vp, const float *vs, const float *rho, int shot,
                double *tr_vx, double *tr_vy, double *tr_vz)
{
    ctx_t c;
    int rc = ctx_init(&c, p, vp, vs, rho, shot);
    if (rc) return rc;
    wave_t w;
    if (alloc_wave(&c.g, &w, 1)) { ctx_free(&c); return -1; }
    for (int it = 0; it < c.nt; it++) {
        step_forward(&c, &w, it, M_FWD, NULL, 0, NULL);
        /* sub_cal_seis_data_base (seisrecord_meat.hpp:57-77) after the
         * stress update: samples the velocities of step it */
        for (int r = 0; r < c.nrec; r++) {
            size_t s = c.rec_idx[r], o = (size_t)it + (size_t)r * c.nt;
            tr_vx[o] = w.f[VX][s];
            tr_vy[o] = w.f[VY][s];
            tr_vz[o] = w.f[VZ][s];
        }
    }
    free_wave(&w);
    ctx_free(&c);
    return 0;
}

static double rel_l2_vel(const grid_t *g, wave_t *a, real *snap)
{
    double num = 0, den = 0;
    size_t o = 0;
    for (int k = g->m; k < g->m + g->pz; k++)
        for (int j = g->m; j < g->m + g->py; j++)
            for (int i = g->m; i < g->m + g->px; i++) {
                size_t idx = (size_t)i + g->sy * j + g->sz * k;
                for (int f = 0; f < 3; f++) {
                    double d = (double)a->f[VX + f][idx] - (double)snap[o];
                    num += d * d;
                    den += (double)snap[o] * (double)snap[o];
                    o++;
                }
            }
    return den > 0 ? sqrt(num / den) : sqrt(num);
}

static void snap_vel(const grid_t *g, wave_t *a, real *snap)
{
    size_t o = 0;
    for (int k = g->m; k < g->m + g->pz; k++)
        for (int j = g->m; j < g->m + g->py; j++)
            for (int i = g->m; i < g->m + g->px; i++) {
                size_t idx = (size_t)i + g->sy * j + g->sz * k;
                for (int f = 0; f < 3; f++) snap[o++] = a->f[VX + f][idx];
            }
}

/* Imaging condition, cal_correlation_from_wave
 * (RTM/rtm3d_0_image_module/rtm3d_iamge_kernel.hpp:6-51): s = the
 * reconstructed source wavefield (rtm_backward), r = the receiver
 * wavefield (rtm_reverse). */
static void image_accumulate(const grid_t *g, wave_t *s, wave_t *r, double *ip, double *pp, double *ps,
                             double *sp, double *ss)
{
#pragma omp parallel for schedule(static)
    for (int pk = 0; pk < g->pz; pk++)
        for (int pj = 0; pj < g->py; pj++)
            for (int pi_ = 0; pi_ < g->px; pi_++) {
                size_t i = (size_t)(pi_ + g->m) + g->sy * (pj + g->m) + g->sz * (pk + g->m);
                size_t o = (size_t)pi_ + (size_t)g->px * ((size_t)pj + (size_t)g->py * pk);
                real psx = s->f[VXP][i], psy = s->f[VYP][i], psz = s->f[VZP][i];
                real ssx = s->f[VX][i] - psx, ssy = s->f[VY][i] - psy, ssz = s->f[VZ][i] - psz;
                real prx = r->f[VXP][i], pry = r->f[VYP][i], prz = r->f[VZP][i];
                real srx = r->f[VX][i] - prx, sry = r->f[VY][i] - pry, srz = r->f[VZ][i] - prz;
                ip[o] += (double)(psx * psx + psy * psy + psz * psz);
                pp[o] += (double)(psx * prx + psy * pry + psz * prz);
                ps[o] += (double)(psx * srx + psy * sry + psz * srz);
                sp[o] += (double)(ssx * prx + ssy * pry + ssz * prz);
                ss[o] += (double)(ssx * srx + ssy * sry + ssz * srz);
            }
}

/* Core of one RTM shot; nsteps_limit > 0 runs only that many time steps
 * of each phase (bounded CPU-baseline sample, no imaging output kept). */
static int rtm_core(const jvo_problem *p, const float *vp, const float *vs, const float *rho, int shot,
                    const double *obs_vx, const double *obs_vy, const double *obs_vz, double *ip, double *pp,
                    double *ps, double *sp, double *ss, double *recon_err, int nsteps_limit)
{
    ctx_t c;
    int rc = ctx_init(&c, p, vp, vs, rho, shot);
    if (rc) return rc;
    const int nt = c.nt;
    const int nrun = (nsteps_limit > 0 && nsteps_limit < nt) ? nsteps_limit : nt;
    int w = p->rec_width;
    if (w < 1 || w > PHY_HALF || w > p->pml) { ctx_free(&c); return -2; }
    int nb = vowr_boxes(&c.g, w, NULL);
    box_t *bx = (box_t *)malloc(sizeof(box_t) * (size_t)(nb > 0 ? nb : 1));
    vowr_boxes(&c.g, w, bx);
    size_t per = boxes_size(bx, nb);
    /* store slices it = 0 .. nt-2 (halo_store slice_num = ntime-1) */
    int nslice = nrun < nt ? nrun : nt - 1;
    if (nslice < 1) nslice = 1;
    real *store = (real *)malloc(sizeof(real) * per * (size_t)nslice + 1);
    wave_t F, R;
    if (!store || alloc_wave(&c.g, &F, 1) || alloc_wave(&c.g, &R, 1)) { ctx_free(&c); return -1; }
    int it_chk = nt / 2;
    size_t nphy = (size_t)c.g.px * c.g.py * c.g.pz;
    real *snap = recon_err ? (real *)malloc(sizeof(real) * 3 * nphy) : NULL;

    /* forward for reconstruction: fdtd3d_blend_elastic_model_mpi_meat.hpp:125-146 */
    for (int it = 0; it < nrun; it++) {
        real *slot = NULL;
        if (it <= nt - 2 && it < nslice) slot = store + per * (size_t)it;
        step_forward(&c, &F, it, M_RTMF, bx, nb, slot);
        if (snap && it == it_chk - 1) snap_vel(&c.g, &F, snap);
    }

    /* time-reverse loop: RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:64-113 */
    int it_end = (nrun < nt) ? nt - nrun : 0;
    double *tip = ip, *tpp = pp, *tps = ps, *tsp = sp, *tss = ss;
    double *scratch = NULL;
    if (!ip) {
        scratch = (double *)calloc(5 * nphy, sizeof(double));
        tip = scratch; tpp = scratch + nphy; tps = scratch + 2 * nphy; tsp = scratch + 3 * nphy; tss = scratch + 4 * nphy;
    }
    for (int it = nt - 1; it >= it_end; it--) {
        /* UPDATE 1 */
        add_source(&F, c.src_idx, -(real)c.wl[it]);
        for (int r = 0; r < c.nrec; r++) {
            size_t s = c.rec_idx[r], o = (size_t)it + (size_t)r * nt;
            /* sub_rtm_reverse_add_vel_source (seisrecord_meat.hpp:79-107) */
            R.f[VX][s] += (real)obs_vx[o];
            R.f[VY][s] += (real)obs_vy[o];
            R.f[VZ][s] += (real)obs_vz[o];
        }
        store16(&c.g, &R, VX, VZ);
        stress_interior(&c.g, &c.cf, &c.md, &F, M_BWD, w, -c.g.dt);
        store16(&c.g, &F, SXX, SAU);
        vel_pml(&c.g, &c.cf, &c.md, &R);
        vel_interior(&c.g, &c.cf, &c.md, &R, M_REV, PHY_HALF, c.g.dt);
        store16(&c.g, &R, VX, VZ);
        store16(&c.g, &R, VXP, VZP);
        int sl = it - 1;
        int have = (sl >= 0 && sl <= nt - 2);
        /* a bounded sample keeps only nslice slots and cycles through them */
        real *slot = have ? store + per * (size_t)(nrun < nt ? sl % nslice : sl) : NULL;
        if (have) box_copy(&c.g, &F, bx, nb, slot, 0, 0, 1);
        store16(&c.g, &F, SXX, SAU);
        /* UPDATE 2 */
        vel_interior(&c.g, &c.cf, &c.md, &F, M_BWD, w, -c.g.dt);
        store16(&c.g, &F, VX, VZ);
        stress_pml(&c.g, &c.cf, &c.md, &R);
        stress_interior(&c.g, &c.cf, &c.md, &R, M_REV, PHY_HALF, c.g.dt);
        store16(&c.g, &R, SXX, SAU);
        if (have) box_copy(&c.g, &F, bx, nb, slot, 0, 1, 0);
        store16(&c.g, &F, VX, VZ);
        image_accumulate(&c.g, &F, &R, tip, tpp, tps, tsp, tss);
        if (snap && it == it_chk) *recon_err = rel_l2_vel(&c.g, &F, snap);
    }
    free(scratch);
    free(snap);
    free(store);
    free(bx);
    free_wave(&F);
    free_wave(&R);
    ctx_free(&c);
    return 0;
}

int jvo_rtm_shot(const jvo_problem *p, const float *vp, const float *vs, const float *rho, int shot,
                 const double *obs_vx, const double *obs_vy, const double *obs_vz, double *ip, double *pp,
                 double *ps, double *sp, double *ss, double *recon_err)
{
    if (!ip || !pp || !ps || !sp || !ss) return -4;
    return rtm_core(p, vp, vs, rho, shot, obs_vx, obs_vy, obs_vz, ip, pp, ps, sp, ss, recon_err, 0);
}

void jvo_finalize_image(int nx, int ny, int nz, const double *ip, double *pp, double *ps, double *sp, double *ss,
                        double *lap_pp, double *lap_ps, double *lap_sp, double *lap_ss)
{
    /* laplace_filter_cal_for_image (RTM/rtm3d_0_image_module/rtm3d_iamge_kernel.hpp:184-200) */
    size_t sy = (size_t)nx, sz = (size_t)nx * ny, n = sz * nz;
    double *src[4] = {pp, ps, sp, ss};
    double *dst[4] = {lap_pp, lap_ps, lap_sp, lap_ss};
    for (int q = 0; q < 4; q++) {
        if (!dst[q]) continue;
        memset(dst[q], 0, n * sizeof(double));
        for (int k = 2; k <= nz - 3; k++)
            for (int j = 2; j <= ny - 3; j++)
                for (int i = 2; i <= nx - 3; i++) {
                    size_t x = (size_t)i + sy * j + sz * k;
                    const double *f = src[q];
                    dst[q][x] = f[x + 1] + f[x - 1] + f[x + sy] + f[x - sy] + f[x + sz] + f[x - sz] - 6.0 * f[x];
                }
    }
    /* source_compensation (rtm3d_iamge_kernel.hpp:118-135) */
    for (size_t x = 0; x < n; x++) {
        double d = ip[x];
        if (d > 3.4e-38) {
            pp[x] /= d; ps[x] /= d; sp[x] /= d; ss[x] /= d;
        }
    }
}

double jvo_rtm_sample(const jvo_problem *p, const float *vp, const float *vs, const float *rho, int shot,
                      int steps)
{
    /* One RTM shot's propagations (forward with boundary store, then the
     * reverse loop with reconstruction, receiver propagation and imaging),
     * `steps` time steps of each, on zero data of the right size. */
    ctx_t c;
    if (ctx_init(&c, p, vp, vs, rho, shot)) return -1.0;
    int nt = c.nt;
    int nrun = steps < nt ? steps : nt;
    double n_ext = (double)c.g.n, n_phy = (double)c.g.px * c.g.py * c.g.pz;
    int nrec = c.nrec;
    ctx_free(&c);
    size_t tr = (size_t)(nrec > 0 ? nrec : 1) * (size_t)nt;
    double *z = (double *)calloc(3 * tr, sizeof(double));
    if (!z) return -1.0;
    int rc = rtm_core(p, vp, vs, rho, shot, z, z + tr, z + 2 * tr, NULL, NULL, NULL, NULL, NULL, NULL, nrun);
    free(z);
    if (rc) return -1.0;
    return (double)nrun * (n_ext + n_phy + n_ext);
}
