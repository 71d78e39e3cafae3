/*
 * sp_oracle.c — TEST INFRASTRUCTURE.  A sequential C restatement of SW2D's native
 * single-porosity (SP) time step, used only to check the CUDA path (tests/, the smoke check
 * and bench.py's CPU-baseline leg).  The product never links or calls it.
 *
 * Every routine cites the reference routine it restates (paths relative to the reference
 * project).  Expressions keep the reference's operand order so that, compiled without FP
 * contraction (-ffp-contract=off), the results are bit-identical to the reference built with
 * g++ on x86-64.  Ternaries restate std::max(a,b) == (a < b ? b : a) and
 * std::min(a,b) == (b < a ? b : a) literally, including their NaN behaviour.
 *
 * Pinned against the reference compiled from its own sources (oracle/_ref/libsw2d_ref.so):
 * tests/test_oracle_pin.py runs both on the shipped sp_toce case and on synthetic cases.
 */
#include "sp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../inria-internship-project-sw2d-enzyme_b200/csrc/portable_math.h"

#define SMALL_REAL 1e-16 /* src/common/param.h:2 */
#define GRAVITY 9.81     /* src/common/param.h:3 */

/* exp/log used by the step: the host libm (as the reference built with g++), or the portable
 * versions the CUDA build uses (spo_set_portable_math) */
typedef double (*math_fn)(double);
static double pm_exp(double x) { return sw2d_exp(x); }
static double pm_log(double x) { return sw2d_log(x); }

static inline double smax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static inline double smin(double a, double b) { return (b < a) ? b : a; } /* std::min */

struct sp_oracle {
    /* sizes */
    long nc, ni, nb;
    /* mesh (reference numbering) */
    double *area, *cx, *cy, *zb;
    long *L, *R;
    double *li, *nxi, *nyi, *mxi, *myi;
    long* bcell;
    double *lb, *nxb, *nyb;
    int* bbc;
    /* per-cell lists built like swParent::setMeshTables (swParent.cpp:469-486) */
    long *cb_off, *cb_idx; /* boundary edges of each cell, increasing index */
    long *ci_off, *ci_idx; /* internal edges of each cell, increasing index */
    long* cn_idx;          /* neighbour cell across ci_idx[k] */
    /* parameters */
    sw2d_params p;
    double *phi, *bous, *fr1, *fr2, *fcos, *fsin, *hs, *hk1, *hk2, *hcos, *hsin;
    /* boundary series */
    int nbc;
    int* bctype;
    long* bcoff;
    double *bctimes, *bcvals, *bcval;
    /* state */
    double *h, *q, *r;
    double t, dt;
    /* edge factors, swSp::computeEdgeFactors (swSp.cpp:338-444) */
    double *cL, *cR, *cB;
    /* Riemann states and fluxes (persistent, as the reference's member vectors) */
    double *zRb, *qRb, *rRb, *lpb, *lmb, *lxb;
    double *zL, *zR, *qL, *qR, *rL, *rR, *lmL, *lmR, *lpL, *lpR, *lx;
    double *F1b, *F2b, *F3b, *S2b;
    double *F1, *F2, *F3, *S2L, *S2R;
    double *sx, *sy, *zc, *swept;
    math_fn fexp, flog;
};

static double* dup_or(const double* src, long n, double fill)
{
    double* d = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
    for (long i = 0; i < n; i++) d[i] = src ? src[i] : fill;
    return d;
}
static double* zeros(long n) { return (double*)calloc(n > 0 ? n : 1, sizeof(double)); }

sp_oracle* spo_create(const sw2d_mesh* m, const sw2d_params* p, const sw2d_cell_fields* f,
                      const sw2d_bc_table* bc, const double* h0, const double* q0, const double* r0)
{
    sp_oracle* o = (sp_oracle*)calloc(1, sizeof(sp_oracle));
    long nc = o->nc = m->cell_nb, ni = o->ni = m->edge_int_nb, nb = o->nb = m->edge_bnd_nb;
    o->p = *p;
    o->area = dup_or(m->cell_area, nc, 0);
    o->cx = dup_or(m->cell_x, nc, 0);
    o->cy = dup_or(m->cell_y, nc, 0);
    o->zb = dup_or(m->cell_z_b, nc, 0);
    o->L = (long*)malloc(sizeof(long) * (ni + 1));
    o->R = (long*)malloc(sizeof(long) * (ni + 1));
    for (long e = 0; e < ni; e++) { o->L[e] = m->edge_int_cells[2 * e]; o->R[e] = m->edge_int_cells[2 * e + 1]; }
    o->li = dup_or(m->edge_int_length, ni, 0);
    o->nxi = dup_or(m->edge_int_nx, ni, 0);
    o->nyi = dup_or(m->edge_int_ny, ni, 0);
    o->mxi = dup_or(m->edge_int_mx, ni, 0);
    o->myi = dup_or(m->edge_int_my, ni, 0);
    o->bcell = (long*)malloc(sizeof(long) * (nb + 1));
    o->bbc = (int*)malloc(sizeof(int) * (nb + 1));
    for (long e = 0; e < nb; e++) { o->bcell[e] = m->edge_bnd_cell[e]; o->bbc[e] = m->edge_bnd_bc[e]; }
    o->lb = dup_or(m->edge_bnd_length, nb, 0);
    o->nxb = dup_or(m->edge_bnd_nx, nb, 0);
    o->nyb = dup_or(m->edge_bnd_ny, nb, 0);

    /* cell -> edge lists in increasing edge order (swParent.cpp:469-486) */
    o->cb_off = (long*)calloc(nc + 1, sizeof(long));
    o->ci_off = (long*)calloc(nc + 1, sizeof(long));
    for (long e = 0; e < nb; e++) o->cb_off[o->bcell[e] + 1]++;
    for (long e = 0; e < ni; e++) { o->ci_off[o->L[e] + 1]++; o->ci_off[o->R[e] + 1]++; }
    for (long c = 0; c < nc; c++) { o->cb_off[c + 1] += o->cb_off[c]; o->ci_off[c + 1] += o->ci_off[c]; }
    o->cb_idx = (long*)malloc(sizeof(long) * (nb + 1));
    o->ci_idx = (long*)malloc(sizeof(long) * (2 * ni + 1));
    o->cn_idx = (long*)malloc(sizeof(long) * (2 * ni + 1));
    long* fillb = (long*)calloc(nc + 1, sizeof(long));
    long* filli = (long*)calloc(nc + 1, sizeof(long));
    for (long e = 0; e < nb; e++) { long c = o->bcell[e]; o->cb_idx[o->cb_off[c] + fillb[c]++] = e; }
    for (long e = 0; e < ni; e++) {
        long a = o->L[e], b = o->R[e];
        o->ci_idx[o->ci_off[a] + filli[a]] = e; o->cn_idx[o->ci_off[a] + filli[a]++] = b;
        o->ci_idx[o->ci_off[b] + filli[b]] = e; o->cn_idx[o->ci_off[b] + filli[b]++] = a;
    }
    free(fillb); free(filli);

    /* per-cell parameters; angles degrees -> radians as swSp::setFrictionParameters
     * (swSp.cpp:1063-1068) and setSingularHeadLossParameters (swSp.cpp:1363) */
    o->phi = dup_or(f->phi, nc, 1.0);
    o->bous = dup_or(f->boussinesq, nc, 1.0);
    o->fr1 = dup_or(f->friction_1, nc, 0);
    o->fr2 = dup_or(f->friction_2, nc, 0);
    o->fcos = zeros(nc); o->fsin = zeros(nc);
    o->hs = dup_or(f->hl_h_sing, nc, 0);
    o->hk1 = dup_or(f->hl_coeff_1, nc, 0);
    o->hk2 = dup_or(f->hl_coeff_2, nc, 0);
    o->hcos = zeros(nc); o->hsin = zeros(nc);
    for (long c = 0; c < nc; c++) {
        double a = (f->friction_alpha ? f->friction_alpha[c] : 0.0) * atan(1.0) / 45.0;
        o->fcos[c] = cos(a); o->fsin[c] = sin(a);
        double b = (f->hl_alpha ? f->hl_alpha[c] : 0.0) * atan(1.0) / 45.0;
        o->hcos[c] = cos(b); o->hsin[c] = sin(b);
    }

    o->nbc = bc->bc_nb;
    o->bctype = (int*)malloc(sizeof(int) * (o->nbc + 1));
    o->bcoff = (long*)malloc(sizeof(long) * (o->nbc + 1));
    for (int k = 0; k < o->nbc; k++) o->bctype[k] = bc->type[k];
    for (int k = 0; k <= o->nbc; k++) o->bcoff[k] = bc->offset[k];
    long nrec = bc->offset[o->nbc];
    o->bctimes = dup_or(bc->times, nrec, 0);
    o->bcvals = dup_or(bc->values, nrec, 0);
    o->bcval = zeros(o->nbc);

    o->h = dup_or(h0, nc, 0); o->q = dup_or(q0, nc, 0); o->r = dup_or(r0, nc, 0);
    o->t = p->t_0;
    o->dt = 0.0; /* swSp.h:155 */

    /* swSp::computeEdgeFactors (swSp.cpp:338-444): coeff = w / area / phi when phi > phi_min */
    o->cB = zeros(nb); o->cL = zeros(ni); o->cR = zeros(ni);
    for (long e = 0; e < nb; e++) {
        long c = o->bcell[e];
        o->cB[e] = (o->phi[c] > p->phi_min) ? o->lb[e] / o->area[c] / o->phi[c] : 0.0;
    }
    for (long e = 0; e < ni; e++) {
        long a = o->L[e], b = o->R[e];
        o->cL[e] = (o->phi[a] > p->phi_min) ? o->li[e] / o->area[a] / o->phi[a] : 0.0;
        o->cR[e] = (o->phi[b] > p->phi_min) ? o->li[e] / o->area[b] / o->phi[b] : 0.0;
    }

    o->zRb = zeros(nb); o->qRb = zeros(nb); o->rRb = zeros(nb);
    o->lpb = zeros(nb); o->lmb = zeros(nb); o->lxb = zeros(nb);
    o->zL = zeros(ni); o->zR = zeros(ni); o->qL = zeros(ni); o->qR = zeros(ni);
    o->rL = zeros(ni); o->rR = zeros(ni); o->lmL = zeros(ni); o->lmR = zeros(ni);
    o->lpL = zeros(ni); o->lpR = zeros(ni); o->lx = zeros(ni);
    o->F1b = zeros(nb); o->F2b = zeros(nb); o->F3b = zeros(nb); o->S2b = zeros(nb);
    o->F1 = zeros(ni); o->F2 = zeros(ni); o->F3 = zeros(ni); o->S2L = zeros(ni); o->S2R = zeros(ni);
    o->sx = zeros(nc); o->sy = zeros(nc); o->zc = zeros(nc); o->swept = zeros(nc);
    o->fexp = exp;
    o->flog = log;
    return o;
}

void spo_set_portable_math(sp_oracle* o, int on)
{
    o->fexp = on ? pm_exp : exp;
    o->flog = on ? pm_log : log;
}

/* swSp::lambdaMinus / lambdaPlus (swSp.cpp:972-995) */
static inline double lam_minus(double b, double c, double u) { return b * u - sqrt((b - 1.0) * b * u * u + c * c); }
static inline double lam_plus(double b, double c, double u) { return b * u + sqrt((b - 1.0) * b * u * u + c * c); }
/* swSp::specificForce (swSp.cpp:1388-1399) */
static inline double spec_force(double b, double phi, double h, double u) { return phi * (b * h * u * u + 0.5 * GRAVITY * h * h); }

/* First-order state of a cell seen from an edge, shared by the boundary loops of both
 * schemes and the internal loop of Godunov (swSpHypGodunov.cpp:17-35,44-76). */
static void godunov_side(const sp_oracle* o, long c, double nx, double ny, double* z, double* qn, double* rn,
                         double* lm, double* lp)
{
    double b = o->bous[c], q = o->q[c], r = o->r[c];
    double hh = o->h[c];
    *z = o->h[c] + o->zb[c];
    *qn = q * nx + r * ny;
    *rn = -q * ny + r * nx;
    double u = *qn / smax(hh, SMALL_REAL);
    double cc = sqrt(GRAVITY * hh);
    *lm = lam_minus(b, cc, u);
    *lp = lam_plus(b, cc, u);
}

static void boundary_states(sp_oracle* o)
{
    for (long e = 0; e < o->nb; e++) {
        godunov_side(o, o->bcell[e], o->nxb[e], o->nyb[e], &o->zRb[e], &o->qRb[e], &o->rRb[e], &o->lmb[e], &o->lpb[e]);
        /* Godunov: max(|l+|,|l-|) (swSpHypGodunov.cpp:34); MUSCL: max(|l-|,|l+|) (swSpHypMusclEvr.cpp:158) */
        if (o->p.scheme == SW2D_SCHEME_GODUNOV) o->lxb[e] = smax(fabs(o->lpb[e]), fabs(o->lmb[e]));
        else o->lxb[e] = smax(fabs(o->lmb[e]), fabs(o->lpb[e]));
    }
}

static double max4(double a, double b, double c, double d)
{ /* std::max({a,b,c,d}): first largest by operator< */
    double m = a;
    if (m < b) m = b;
    if (m < c) m = c;
    if (m < d) m = d;
    return m;
}

/* swSp::hypGodunovComputeLRStates (swSpHypGodunov.cpp:9-84) */
static void godunov_states(sp_oracle* o)
{
    boundary_states(o);
    for (long e = 0; e < o->ni; e++) {
        double nx = o->nxi[e], ny = o->nyi[e];
        godunov_side(o, o->L[e], nx, ny, &o->zL[e], &o->qL[e], &o->rL[e], &o->lmL[e], &o->lpL[e]);
        godunov_side(o, o->R[e], nx, ny, &o->zR[e], &o->qR[e], &o->rR[e], &o->lmR[e], &o->lpR[e]);
        o->lx[e] = max4(fabs(o->lmL[e]), fabs(o->lpL[e]), fabs(o->lmR[e]), fabs(o->lpR[e]));
    }
}

/* swSp::computeMusclSlopes (swSpHypMusclEvr.cpp:11-115) restated per cell: step 1 sums over
 * the neighbours in increasing internal-edge order; step 2 applies, for each internal edge in
 * increasing order, the under/overshoot scaling of the slopes of L then R.  The scaling of a
 * cell's slope only reads that cell's slope, so the edge-ordered loop is the reference's own. */
static void muscl_slopes(sp_oracle* o)
{
    for (long c = 0; c < o->nc; c++) o->zc[c] = o->h[c] + o->zb[c];
    for (long c = 0; c < o->nc; c++) {
        o->sx[c] = 0.0;
        o->sy[c] = 0.0;
        double wsum = 0.0;
        long k0 = o->ci_off[c], k1 = o->ci_off[c + 1];
        if (k1 - k0 > 1) {
            for (long k = k0; k < k1; k++) {
                long j = o->cn_idx[k];
                double dx = o->cx[j] - o->cx[c];
                double dy = o->cy[j] - o->cy[c];
                double dist = sqrt(dx * dx + dy * dy);
                double w = 1.0 / dist;
                o->sx[c] += (o->zc[j] - o->zc[c]) * dx / dist / dist * w;
                o->sy[c] += (o->zc[j] - o->zc[c]) * dy / dist / dist * w;
                wsum += w;
            }
            o->sx[c] /= wsum;
            o->sy[c] /= wsum;
        }
    }
    for (long e = 0; e < o->ni; e++) {
        long a = o->L[e], b = o->R[e];
        double fmx = smax(o->zc[a], o->zc[b]);
        double fmn = smin(o->zc[a], o->zc[b]);
        for (int side = 0; side < 2; side++) {
            long c = side == 0 ? a : b;
            double rec = o->zc[c] + (o->mxi[e] - o->cx[c]) * o->sx[c] + (o->myi[e] - o->cy[c]) * o->sy[c];
            if (rec < fmn) {
                double fac = (fmn - o->zc[c]) / (rec - o->zc[c]);
                o->sx[c] *= fac;
                o->sy[c] *= fac;
            }
            if (rec > fmx) {
                double fac = (fmx - o->zc[c]) / (rec - o->zc[c]);
                o->sx[c] *= fac;
                o->sy[c] *= fac;
            }
        }
    }
}

/* One side of swSp::hypMusclEvrComputeLRStates (swSpHypMusclEvr.cpp:162-272).  side 0 = L
 * (wave speeds clipped with max(0,.)), side 1 = R (min(0,.)). */
static void evr_side(const sp_oracle* o, long c, long e, int side, double* z, double* qn, double* rn, double* lm,
                     double* lp)
{
    double nx = o->nxi[e], ny = o->nyi[e];
    double b = o->bous[c], zbc = o->zb[c];
    double q = o->q[c], r = o->r[c], hl = o->h[c];
    double ql = q * nx + r * ny;
    double rl = r * nx - q * ny;
    double cl = sqrt(GRAVITY * smax(SMALL_REAL, hl));
    double ul = ql / smax(SMALL_REAL, hl);
    double vl = rl / smax(SMALL_REAL, hl);
    double l1 = side == 0 ? smax(0.0, lam_minus(b, cl, ul)) : smin(0.0, lam_minus(b, cl, ul));
    double dx1 = o->mxi[e] - o->cx[c] - 0.5 * l1 * o->dt * nx;
    double dy1 = o->myi[e] - o->cy[c] - 0.5 * l1 * o->dt * ny;
    double z1 = o->zc[c] + dx1 * o->sx[c] + dy1 * o->sy[c];
    double h1 = smax(0.0, z1 - zbc);
    double l2 = side == 0 ? smax(0.0, lam_plus(b, cl, ul)) : smin(0.0, lam_plus(b, cl, ul));
    double dx2 = o->mxi[e] - o->cx[c] - 0.5 * l2 * o->dt * nx;
    double dy2 = o->myi[e] - o->cy[c] - 0.5 * l2 * o->dt * ny;
    double z2 = o->zc[c] + dx2 * o->sx[c] + dy2 * o->sy[c];
    double h2 = smax(0.0, z2 - zbc);
    double hr = 0.5 * (h1 + h2);
    *z = 0.5 * (h1 + h2) + zbc;
    *qn = 0.5 * (h1 + h2) * ul;
    *rn = 0.5 * (h1 + h2) * vl;
    double u = *qn / smax(hr, SMALL_REAL);
    double cc = sqrt(GRAVITY * hr);
    *lm = lam_minus(b, cc, u);
    *lp = lam_plus(b, cc, u);
}

/* swSp::hypMusclEvrComputeLRStates (swSpHypMusclEvr.cpp:119-277); uses the member dt, i.e. the
 * time step of the previous step (0 at the first step). */
static void muscl_states(sp_oracle* o)
{
    muscl_slopes(o);
    boundary_states(o);
    for (long e = 0; e < o->ni; e++) {
        evr_side(o, o->L[e], e, 0, &o->zL[e], &o->qL[e], &o->rL[e], &o->lmL[e], &o->lpL[e]);
        evr_side(o, o->R[e], e, 1, &o->zR[e], &o->qR[e], &o->rR[e], &o->lmR[e], &o->lpR[e]);
        o->lx[e] = max4(fabs(o->lmL[e]), fabs(o->lpL[e]), fabs(o->lmR[e]), fabs(o->lpR[e]));
    }
}

/* swSp::hypComputeTimeStep (swSpHyp.cpp:430-512), including the carry-over of `lambda` from the
 * L side to the R side of an internal edge (:456-476) and the dt_map snap (:496-504). */
static double time_step(sp_oracle* o)
{
    double dt = o->p.dt_max;
    double* sw = o->swept;
    for (long c = 0; c < o->nc; c++) sw[c] = 0.0;
    for (long e = 0; e < o->nb; e++) {
        long c = o->bcell[e];
        if (o->h[c] > o->p.h_min) sw[c] += o->lxb[e] * o->lb[e];
    }
    for (long e = 0; e < o->ni; e++) {
        double lam = 0.0;
        long a = o->L[e], b = o->R[e];
        if (o->h[a] > o->p.h_min) lam = o->lx[e];
        sw[a] += lam * o->li[e];
        if (o->h[b] > o->p.h_min) lam = o->lx[e];
        sw[b] += lam * o->li[e];
    }
    for (long c = 0; c < o->nc; c++) {
        double x = o->p.cfl_max * (o->area[c] / smax(sw[c], SMALL_REAL));
        if (x < dt) dt = x;
    }
    if (o->p.dt_map > SMALL_REAL) {
        int now = (int)(o->t / o->p.dt_map);
        int later = (int)((o->t + dt) / o->p.dt_map);
        if (later > now) dt = later * o->p.dt_map - o->t;
    }
    if ((o->t + dt) > o->p.t_max) dt = o->p.t_max - o->t;
    return dt;
}

/* swBoundaryConditionTimeSeries::initialise + computeValBC
 * (models/common/swBoundaryConditionTimeSeries.cpp:17-96), walked from the initial cursor;
 * time only increases, so this equals the reference's incremental cursor. */
static double bc_value(const sp_oracle* o, int k, double time)
{
    const double* tv = o->bctimes + o->bcoff[k];
    const double* vv = o->bcvals + o->bcoff[k];
    long n = o->bcoff[k + 1] - o->bcoff[k];
    double v_inf = vv[0], t_inf = tv[0], v_sup, t_sup;
    int at_end = 0;
    if (n > 1) { v_sup = vv[1]; t_sup = tv[1]; }
    else { v_sup = v_inf; t_sup = t_inf; at_end = 1; }
    long rank = 1;
    while ((time > t_sup) && !at_end) {
        v_inf = v_sup;
        t_inf = t_sup;
        t_sup = tv[rank];
        v_sup = vv[rank];
        ++rank;
        if (rank == n) at_end = 1;
    }
    if (time > t_sup) return v_sup;
    if (time < t_inf) return v_inf;
    double d = (time - t_inf) / (t_sup - t_inf);
    return v_inf + (v_sup - v_inf) * d;
}

/* swSp::hypHCritical (swSpHyp.cpp:651-661) */
static double h_critical(const sp_oracle* o, double phi, double q)
{
    return o->fexp((1. / 3.) * o->flog((q / smax(phi, SMALL_REAL)) / GRAVITY));
}

/* swSp::hypBoundaryFlux (swSpHyp.cpp:13-135); source_right stays 0. */
static int boundary_flux(const sp_oracle* o, double bR, double phiR, double zbR, double zR, double qR, double rR,
                         double lpR, int type, double bcv, double* f1, double* f2, double* f3)
{
    double hR = zR - zbR;
    double q1 = qR, r1 = rR;
    if (hR < o->p.h_min) { q1 = 0.; r1 = 0.; hR = 0.; }
    double cR = sqrt(GRAVITY * smax(hR, SMALL_REAL));
    double uR = q1 / smax(hR, SMALL_REAL);
    double L1 = smax(0.0, lpR);
    double flux2R = spec_force(bR, phiR, hR, uR);
    double flux1 = 0.0, flux2 = 0.0;
    if (type == SW2D_BC_FR) {
        if ((bcv < 0.) | (bcv > 1.)) return SW2D_E_BC_FR;
        double c = (uR - 2. * cR) / (-bcv - 2.);
        c = smax(c, 0.);
        double u = -bcv * c;
        double h = c * c / GRAVITY;
        flux1 = phiR * u * h;
        flux2 = flux2R + (flux1 - q1 * phiR) * L1;
    } else if (type == SW2D_BC_H || type == SW2D_BC_Z) {
        double h_bc = type == SW2D_BC_H ? smax(bcv, 0.) : smax(bcv - zbR, 0.);
        if (hR > o->p.h_min) {
            flux1 = phiR * (q1 + L1 * (h_bc - hR));
            flux2 = flux2R + (flux1 - q1 * phiR) * L1;
        } else {
            double c = sqrt(GRAVITY * h_bc);
            flux1 = phiR * h_bc * c;
            flux2 = spec_force(bR, phiR, h_bc, c);
        }
    } else if (type == SW2D_BC_Q) {
        flux1 = bcv;
        double hc = h_critical(o, phiR, bcv);
        if (hc >= hR) flux1 = phiR * 1.5 * sqrt(GRAVITY * hc) * hc;
        flux2 = flux2R + (flux1 - q1 * phiR) * L1;
    } else {
        return SW2D_E_BC_TYPE;
    }
    double flux3;
    if (flux1 > 0) flux3 = 0;
    else {
        double vR = r1 / smax(hR, SMALL_REAL);
        flux3 = flux1 * vR;
    }
    *f1 = flux1; *f2 = flux2; *f3 = flux3;
    return 0;
}

/* Wet/dry configuration shared by swSp::hypHllc (swSpHyp.cpp:688-739) and hypHllcBlending
 * (:852-903).  Returns 0 both, 1 lhs alone, 2 rhs alone, 3 nowhere, -1 impossible. */
static int hllc_config(double hL, double hR, double zL, double zR, double zbL, double zbR, double phiL, double phiR,
                       double h_min, double phi_min)
{
    int both = 0, lhs = 0, rhs = 0, none = 0;
    if (((hL <= h_min) && (hR <= h_min)) || ((phiL <= phi_min) && (phiR <= phi_min))) none = 1;
    else {
        both = 1;
        if ((phiR <= phi_min) || ((phiR > phi_min) && (hR <= h_min) && (zL <= zbR + h_min))) { lhs = 1; both = 0; }
        if ((phiL <= phi_min) || ((phiL > phi_min) && (hL <= h_min) && (zR <= zbL + h_min))) { rhs = 1; both = 0; }
    }
    if (both + lhs + rhs + none != 1) return -1;
    return both ? 0 : lhs ? 1 : rhs ? 2 : 3;
}

/* swSp::hypHllc (swSpHyp.cpp:664-821) and swSp::hypHllcBlending (:824-998). */
static int hllc(const sp_oracle* o, int blending, double bL, double bR, double phiL, double phiR, double zbL, double zbR,
                double zL, double qL, double rL, double zR, double qR, double rR, double lmL, double lmR, double lpL,
                double lpR, double* f1, double* f2, double* f3, double* sl, double* sr)
{
    double hL, hR;
    if (blending) { hL = zL - zbL; hR = zR - zbR; }
    else { hL = smax(0.0, zL - zbL); hR = smax(0.0, zR - zbR); }
    int cfg = hllc_config(hL, hR, zL, zR, zbL, zbR, phiL, phiR, o->p.h_min, o->p.phi_min);
    if (cfg < 0) return SW2D_E_HLLC_CONFIG;
    if (cfg == 0) {
        double uL, uR;
        if (blending) { uL = qL / smax(hL, SMALL_REAL); uR = qR / smax(hR, SMALL_REAL); }
        else { uL = qL / smax(SMALL_REAL, hL); uR = qR / smax(SMALL_REAL, hR); }
        double L1 = smin(lmL, smin(lmR, 0.));
        double L2 = smax(lpL, smax(lpR, 0.));
        double phiLR = smin(phiL, phiR);
        double flux1, s2;
        if (blending) {
            double alpha_h = 0.0;
            if (fabs(zbL - zbR) > SMALL_REAL) alpha_h = smax(0.0, smin(1.0, (zL - zR) / (zbL - zbR)));
            double F1h = phiLR * (L2 * qL - L1 * qR + L1 * L2 * (hR - hL)) / smax(L2 - L1, SMALL_REAL);
            double F1z = phiLR * (L2 * qL - L1 * qR + L1 * L2 * (zR - zL)) / smax(L2 - L1, SMALL_REAL);
            flux1 = alpha_h * F1h + (1.0 - alpha_h) * F1z;
            double fact = 0.5 * smin(phiL, phiR) * (hL + hR);
            double s2z = (phiR * hR * hR - phiL * hL * hL) * 0.5 + fact * (zL - zR);
            double s2h;
            if (zbL > zbR) s2h = phiR * hR * (zbL - zbR);
            else s2h = phiL * hL * (zbL - zbR);
            s2 = alpha_h * s2h + (1.0 - alpha_h) * s2z;
        } else {
            flux1 = phiLR * (L2 * qL - L1 * qR + L1 * L2 * (zR - zL)) / smax(L2 - L1, SMALL_REAL);
            double fact = 0.5 * smin(phiL, phiR) * (hL + hR);
            s2 = (phiR * hR * hR - phiL * hL * hL) * 0.5 + fact * (zL - zR);
        }
        s2 = s2 * GRAVITY / smax(L2 - L1, SMALL_REAL);
        double source_left = -L1 * s2;
        double source_right = L2 * s2;
        double FL = spec_force(bL, phiL, hL, uL);
        double FR = spec_force(bR, phiR, hR, uR);
        double flux2 = (L2 * (FL + source_left) - L1 * (FR - source_right) + L1 * L2 * (phiR * qR - phiL * qL)) /
                       smax(L2 - L1, SMALL_REAL);
        double vL = rL / smax(hL, SMALL_REAL);
        double vR = rR / smax(hR, SMALL_REAL);
        double flux3 = (flux1 >= 0) ? bL * flux1 * vL : bR * flux1 * vR;
        *f1 = flux1; *f2 = flux2; *f3 = flux3; *sl = source_left; *sr = source_right;
    } else if (cfg == 2) {
        *f1 = 0.; *f2 = 0.; *sl = 0.; *sr = phiR * 0.5 * GRAVITY * hR * hR; *f3 = 0.;
    } else if (cfg == 1) {
        *f1 = 0.; *f2 = 0.; *sl = -phiL * 0.5 * GRAVITY * hL * hL; *sr = 0.; *f3 = 0.;
    } else {
        *f1 = 0.; *f2 = 0.; *sl = 0.; *sr = 0.; *f3 = 0.;
    }
    return 0;
}

/* swSp::hypComputeFluxes (swSpHyp.cpp:276-402).  Internal fluxes are computed only when one
 * side is wet (:339); otherwise the previous values stay in the arrays. */
static int fluxes(sp_oracle* o)
{
    for (int k = 0; k < o->nbc; k++) o->bcval[k] = bc_value(o, k, o->t);
    for (long e = 0; e < o->nb; e++) {
        long c = o->bcell[e];
        int k = o->bbc[e];
        double f1 = 0, f2 = 0, f3 = 0;
        int st = boundary_flux(o, o->bous[c], o->phi[c], o->zb[c], o->zRb[e], o->qRb[e], o->rRb[e], o->lpb[e],
                               o->bctype[k], o->bcval[k], &f1, &f2, &f3);
        if (st) return st;
        o->F1b[e] = f1; o->F2b[e] = f2; o->F3b[e] = f3; o->S2b[e] = 0.0;
    }
    int blending = o->p.topo == SW2D_TOPO_BLENDING;
    for (long e = 0; e < o->ni; e++) {
        long a = o->L[e], b = o->R[e];
        double zbL = o->zb[a], zbR = o->zb[b];
        double hL = o->zL[e] - zbL, hR = o->zR[e] - zbR;
        if ((hL > o->p.h_min) || (hR > o->p.h_min)) {
            double f1 = 0, f2 = 0, f3 = 0, sl = 0, sr = 0;
            int st = hllc(o, blending, o->bous[a], o->bous[b], o->phi[a], o->phi[b], zbL, zbR, o->zL[e], o->qL[e],
                          o->rL[e], o->zR[e], o->qR[e], o->rR[e], o->lmL[e], o->lmR[e], o->lpL[e], o->lpR[e], &f1,
                          &f2, &f3, &sl, &sr);
            if (st) return st;
            if (isnan(f1)) return SW2D_E_NAN_FLUX;
            o->F1[e] = f1; o->F2[e] = f2; o->F3[e] = f3; o->S2L[e] = sl; o->S2R[e] = sr;
        }
    }
    return 0;
}

/* swSp::hypComputeBalance (swSpHyp.cpp:214-273) with the factors of computeEdgeFactors. */
static void balance(sp_oracle* o, double dt)
{
    double *h = o->h, *q = o->q, *r = o->r;
    for (long e = 0; e < o->nb; e++) {
        long c = o->bcell[e];
        double cf = o->cB[e], nx = o->nxb[e], ny = o->nyb[e];
        double f1 = +cf, f2F2 = +cf * nx, f2F3 = -cf * ny, f2S2 = +cf * nx, f3F2 = +cf * ny, f3F3 = +cf * nx,
               f3S2 = +cf * ny;
        h[c] += f1 * o->F1b[e] * dt;
        q[c] += (f2F2 * o->F2b[e] + f2S2 * o->S2b[e] + f2F3 * o->F3b[e]) * dt;
        r[c] += (f3F2 * o->F2b[e] + f3S2 * o->S2b[e] + f3F3 * o->F3b[e]) * dt;
    }
    for (long e = 0; e < o->ni; e++) {
        long a = o->L[e], b = o->R[e];
        double cl = o->cL[e], cr = o->cR[e], nx = o->nxi[e], ny = o->nyi[e];
        double f1L = -cl, f1R = +cr;
        double f2F2L = -cl * nx, f2F2R = +cr * nx, f2F3L = +cl * ny, f2F3R = -cr * ny, f2S2L = +cl * nx,
               f2S2R = +cr * nx;
        double f3F2L = -cl * ny, f3F2R = +cr * ny, f3F3L = -cl * nx, f3F3R = +cr * nx, f3S2L = +cl * ny,
               f3S2R = +cr * ny;
        h[a] += f1L * o->F1[e] * dt;
        h[b] += f1R * o->F1[e] * dt;
        q[a] += (f2F2L * o->F2[e] + f2S2L * o->S2L[e] + f2F3L * o->F3[e]) * dt;
        q[b] += (f2F2R * o->F2[e] + f2S2R * o->S2R[e] + f2F3R * o->F3[e]) * dt;
        r[a] += (f3F2L * o->F2[e] + f3S2L * o->S2L[e] + f3F3L * o->F3[e]) * dt;
        r[b] += (f3F2R * o->F2[e] + f3S2R * o->S2R[e] + f3F3R * o->F3[e]) * dt;
    }
    for (long c = 0; c < o->nc; c++) {
        if (fabs(h[c]) < SMALL_REAL) h[c] = 0.;
        if (fabs(q[c]) < SMALL_REAL) q[c] = 0.;
        if (fabs(r[c]) < SMALL_REAL) r[c] = 0.;
    }
}

/* swSource::frictionChezy1D / frictionManning1D / frictionStrickler1D
 * (models/common/swSourceFriction.cpp:7-79) */
static double friction_factor(const sp_oracle* o, int model, double k, double h, double un, double dt)
{
    math_fn exp = o->fexp, log = o->flog;
    double factor = 1.0;
    if (model == SW2D_FRICTION_CHEZY) {
        if ((h > SMALL_REAL) && (k > SMALL_REAL)) factor = exp(-GRAVITY * un / k / k / h * dt);
        else factor = 0.0;
    } else if (model == SW2D_FRICTION_MANNING) {
        if (h > SMALL_REAL) factor = exp(-GRAVITY * un * k * k * exp(-4.0 / 3.0 * log(h)) * dt);
        else factor = 0.0;
    } else {
        if ((h > SMALL_REAL) && (k > SMALL_REAL)) factor = exp(-GRAVITY * un / k / k * exp(-4.0 / 3.0 * log(h)) * dt);
        else factor = 0.0;
    }
    return factor;
}

/* swSp::sourceFrictionChezy/Manning/Strickler (swSpSourceFriction.cpp:39-171) */
static void friction(sp_oracle* o, double dt)
{
    double hthr = smax(o->p.h_min, SMALL_REAL);
    for (long c = 0; c < o->nc; c++) {
        double h = o->h[c];
        if (h > hthr) {
            double u = o->q[c] / h;
            double v = o->r[c] / h;
            double ca = o->fcos[c], sa = o->fsin[c];
            double ul = u * ca + v * sa;
            double vl = -u * sa + v * ca;
            double un = sqrt(u * u + v * v);
            double f1 = friction_factor(o, o->p.friction, o->fr1[c], h, un, dt);
            double f2 = friction_factor(o, o->p.friction, o->fr2[c], h, un, dt);
            ul *= f1;
            vl *= f2;
            o->q[c] = (ul * ca - vl * sa) * h;
            o->r[c] = (ul * sa + vl * ca) * h;
        } else {
            o->q[c] = 0.;
            o->r[c] = 0.;
        }
    }
}

/* swSp::sourceSingularHeadLoss (swSpSourceFriction.cpp:174-219) */
static void head_loss(sp_oracle* o, double dt)
{
    double hthr = smax(o->p.h_min, SMALL_REAL);
    for (long c = 0; c < o->nc; c++) {
        double ca = o->hcos[c], sa = o->hsin[c];
        double qx = o->q[c] * ca + o->r[c] * sa;
        double qy = -o->q[c] * sa + o->r[c] * ca;
        double h = o->h[c];
        if (h > hthr) {
            double ax = 0, ay = 0;
            if (h > o->hs[c]) {
                ax = sqrt(qx * qx + qy * qy) * o->hk1[c] / h;
                ay = sqrt(qx * qx + qy * qy) * o->hk2[c] / h;
            }
            qx = qx * o->fexp(-ax * dt);
            qy = qy * o->fexp(-ay * dt);
        } else {
            qx = 0.;
            qy = 0.;
        }
        o->q[c] = qx * ca - qy * sa;
        o->r[c] = qx * sa + qy * ca;
    }
}

/* swSp::correctVelocity (swSp.cpp:447-479) */
static void correct_velocity(sp_oracle* o)
{
    for (long c = 0; c < o->nc; c++) {
        double h = o->h[c];
        if (h > o->p.h_min) {
            double q = o->q[c], r = o->r[c];
            double qn = sqrt(q * q + r * r);
            double cc = sqrt(GRAVITY * h);
            double Fr = qn / cc / h;
            double fact = smax(qn / (h * o->p.v_max), Fr / o->p.fr_max);
            if (fact > 1.0) {
                o->q[c] = q / fact;
                o->r[c] = r / fact;
            }
        }
    }
}

/* One pass of the body of swSp::execute's loop (swSp.cpp:522-589) through hypCompute
 * (swSpHyp.cpp:137-211). */
static int step_once(sp_oracle* o)
{
    if (o->p.scheme == SW2D_SCHEME_GODUNOV) godunov_states(o);
    else muscl_states(o);
    o->dt = time_step(o);
    int st = fluxes(o);
    if (st) return st;
    balance(o, o->dt);
    for (long c = 0; c < o->nc; c++) {
        if (o->p.negative_depth_detection) {
            if (o->h[c] < 0) return SW2D_E_NEG_DEPTH;
        } else if (o->h[c] < 0.) {
            o->h[c] = 0.; o->q[c] = 0.; o->r[c] = 0.;
        }
    }
    if (o->p.friction != SW2D_FRICTION_NONE) friction(o, o->dt);
    if (o->p.singular_head_loss) head_loss(o, o->dt);
    correct_velocity(o);
    o->t += o->dt;
    return 0;
}

int spo_step(sp_oracle* o, int n)
{
    int done = 0;
    for (int i = 0; i < n; i++) {
        if (!(o->t < o->p.t_max)) break;
        int st = step_once(o);
        if (st) return st;
        done++;
    }
    return done;
}

void spo_get_state(const sp_oracle* o, double* h, double* q, double* r)
{
    memcpy(h, o->h, sizeof(double) * o->nc);
    memcpy(q, o->q, sizeof(double) * o->nc);
    memcpy(r, o->r, sizeof(double) * o->nc);
}

void spo_set_state(sp_oracle* o, const double* h, const double* q, const double* r)
{
    memcpy(o->h, h, sizeof(double) * o->nc);
    memcpy(o->q, q, sizeof(double) * o->nc);
    memcpy(o->r, r, sizeof(double) * o->nc);
}

double spo_time(const sp_oracle* o) { return o->t; }
double spo_dt(const sp_oracle* o) { return o->dt; }
void spo_set_time(sp_oracle* o, double t, double dt) { o->t = t; o->dt = dt; }

long spo_get_array(const sp_oracle* o, const char* name, double* out)
{
    struct { const char* n; const double* a; long len; } tab[] = {
        {"F1_int", o->F1, o->ni}, {"F2_int", o->F2, o->ni}, {"F3_int", o->F3, o->ni},
        {"s2L_int", o->S2L, o->ni}, {"s2R_int", o->S2R, o->ni},
        {"F1_bnd", o->F1b, o->nb}, {"F2_bnd", o->F2b, o->nb}, {"F3_bnd", o->F3b, o->nb}, {"s2R_bnd", o->S2b, o->nb},
        {"lambda_max_int", o->lx, o->ni}, {"lambda_max_bnd", o->lxb, o->nb},
        {"z_riemann_L", o->zL, o->ni}, {"z_riemann_R", o->zR, o->ni},
        {"q_riemann_L", o->qL, o->ni}, {"q_riemann_R", o->qR, o->ni},
        {"r_riemann_L", o->rL, o->ni}, {"r_riemann_R", o->rR, o->ni},
        {"lambda_minus_L", o->lmL, o->ni}, {"lambda_minus_R", o->lmR, o->ni},
        {"lambda_plus_L", o->lpL, o->ni}, {"lambda_plus_R", o->lpR, o->ni},
        {"slope_x", o->sx, o->nc}, {"slope_y", o->sy, o->nc}, {"swept", o->swept, o->nc},
        {"h", o->h, o->nc}, {"q", o->q, o->nc}, {"r", o->r, o->nc},
    };
    for (size_t i = 0; i < sizeof(tab) / sizeof(tab[0]); i++) {
        if (strcmp(tab[i].n, name) == 0) {
            memcpy(out, tab[i].a, sizeof(double) * tab[i].len);
            return tab[i].len;
        }
    }
    return -1;
}

void spo_destroy(sp_oracle* o)
{
    if (!o) return;
    double* dbl[] = {o->area, o->cx, o->cy, o->zb, o->li, o->nxi, o->nyi, o->mxi, o->myi, o->lb, o->nxb, o->nyb,
                     o->phi, o->bous, o->fr1, o->fr2, o->fcos, o->fsin, o->hs, o->hk1, o->hk2, o->hcos, o->hsin,
                     o->bctimes, o->bcvals, o->bcval, o->h, o->q, o->r, o->cL, o->cR, o->cB,
                     o->zRb, o->qRb, o->rRb, o->lpb, o->lmb, o->lxb, o->zL, o->zR, o->qL, o->qR, o->rL, o->rR,
                     o->lmL, o->lmR, o->lpL, o->lpR, o->lx, o->F1b, o->F2b, o->F3b, o->S2b, o->F1, o->F2, o->F3,
                     o->S2L, o->S2R, o->sx, o->sy, o->zc, o->swept};
    for (size_t i = 0; i < sizeof(dbl) / sizeof(dbl[0]); i++) free(dbl[i]);
    free(o->L); free(o->R); free(o->bcell); free(o->bbc); free(o->cb_off); free(o->cb_idx);
    free(o->ci_off); free(o->ci_idx); free(o->cn_idx); free(o->bctype); free(o->bcoff);
    free(o);
}
