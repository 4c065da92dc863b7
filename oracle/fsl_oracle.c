/*
 * fsl_oracle.c -- CPU restatement of freeShearLayer's explicit time step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see fsl_oracle.h).  Every function
 * cites the reference file:line it restates.  FP64, reference evaluation
 * order, compile with -ffp-contract=off.
 */
#include "fsl_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* gas constants and scheme constants, src/def.h:25-45 */
#define K 1.4
#define K_1 0.4
#define NK_1 (-0.4)
#define K05 0.7
#define K_K_1 3.5
#define K_1_2 0.2
#define H_K_1 1.25
#define CV 717.75
#define R_VOZD 287.10
#define C1 0.333333333333333
#define C2 0.166666666666667
#define SMALL 1e-30
#define TWO_THIRDS 0.666666666666667

struct orc_ctx {
    orc_params p;
    int L, H, D;
    size_t pj, pi, ncell;
    /* derived constants, src/initialize.c:67-94 */
    double dt, dtx, dty, dtz, rdx, rdy, rdz, r2dx, r2dy, r2dz, r4dx, r4dy, r4dz;
    double lambda_L, cp_Pr_T, DD;
    /* disturbance block state, src/layer2.c:95-101,120 */
    unsigned k_min, k_max;
    double Ud, Vd, Wd, X;
    int counter;
    unsigned step;
    double last_maxco;
    /* fields */
    double *U[5], *Up[5], *mu;
    double **cur; /* U*_: either U or Up */
    double *fs[3][2][5]; /* face arrays [dir][side][var] */
};

#define IC(o, i, j, k) ((size_t)(i) * (o)->pi + (size_t)(j) * (o)->pj + (size_t)(k))
#define IX(o, i, j, k) (((size_t)(i) * (o)->H + (size_t)(j)) * (o)->D + (size_t)(k))
#define IY(o, i, j, k) (((size_t)(i) * ((o)->H + 1) + (size_t)(j)) * (o)->D + (size_t)(k))
#define IZ(o, i, j, k) (((size_t)(i) * (o)->H + (size_t)(j)) * ((o)->D + 1) + (size_t)(k))

static size_t face_count(const orc_ctx *o, int dir)
{
    return (size_t)(o->L + (dir == 0)) * (o->H + (dir == 1)) * (o->D + (dir == 2));
}

orc_ctx *orc_create(const orc_params *p)
{
    orc_ctx *o = calloc(1, sizeof *o);
    int v, d, s;
    if (!o) return NULL;
    o->p = *p;
    o->L = p->LEN; o->H = p->HIG; o->D = p->DEP;
    o->pj = (size_t)o->D + 2;
    o->pi = o->pj * ((size_t)o->H + 2);
    o->ncell = o->pi * ((size_t)o->L + 2);
    /* src/initialize.c:67-94 */
    o->dt = p->deltaT;
    o->dtx = o->dt / p->deltaX; o->dty = o->dt / p->deltaY; o->dtz = o->dt / p->deltaZ;
    o->rdx = 1. / p->deltaX; o->rdy = 1. / p->deltaY; o->rdz = 1. / p->deltaZ;
    o->r4dx = 1. / (4 * p->deltaX); o->r4dy = 1. / (4 * p->deltaY); o->r4dz = 1. / (4 * p->deltaZ);
    o->r2dx = o->r4dx + o->r4dx; o->r2dy = o->r4dy + o->r4dy; o->r2dz = o->r4dz + o->r4dz;
    o->lambda_L = p->mu_L * CV * K / p->Pr_L;
    o->cp_Pr_T = CV * K / p->Pr_T;
    o->DD = pow(p->deltaX * p->deltaY * p->deltaZ, TWO_THIRDS);
    o->X = p->seed_X;
    for (v = 0; v < 5; v++) {
        o->U[v] = calloc(o->ncell, sizeof(double));
        o->Up[v] = calloc(o->ncell, sizeof(double));
        for (d = 0; d < 3; d++)
            for (s = 0; s < 2; s++) o->fs[d][s][v] = calloc(face_count(o, d), sizeof(double));
    }
    o->mu = calloc(o->ncell, sizeof(double));
    o->cur = o->U;
    return o;
}

void orc_destroy(orc_ctx *o)
{
    int v, d, s;
    if (!o) return;
    for (v = 0; v < 5; v++) {
        free(o->U[v]); free(o->Up[v]);
        for (d = 0; d < 3; d++)
            for (s = 0; s < 2; s++) free(o->fs[d][s][v]);
    }
    free(o->mu);
    free(o);
}

int orc_cells(orc_ctx *o, int which, int var, double *buf, int write)
{
    double *a;
    if (var < 0 || var > 4) return -1;
    switch (which) {
    case 0: a = o->U[var]; break;
    case 1: a = o->Up[var]; break;
    case 2: a = o->cur[var]; break;
    case 3: a = o->mu; break;
    default: return -1;
    }
    if (write) memcpy(a, buf, o->ncell * sizeof(double));
    else memcpy(buf, a, o->ncell * sizeof(double));
    return 0;
}

int orc_faces(orc_ctx *o, int dir, int side, int var, double *buf, int write)
{
    size_t n;
    if (dir < 0 || dir > 2 || side < 0 || side > 1 || var < 0 || var > 4) return -1;
    n = face_count(o, dir) * sizeof(double);
    if (write) memcpy(o->fs[dir][side][var], buf, n);
    else memcpy(buf, o->fs[dir][side][var], n);
    return 0;
}

/* backup.dat row layout, src/finalize.c:22-29 / src/initialize.c:134-148 */
int orc_state(orc_ctx *o, double *buf, int write)
{
    int i, j, v;
    size_t n = 0;
    for (i = 1; i <= o->L; i++)
        for (j = 1; j <= o->H; j++)
            for (v = 0; v < 5; v++, n += o->D) {
                double *row = o->U[v] + IC(o, i, j, 1);
                if (write) memcpy(row, buf + n, o->D * sizeof(double));
                else memcpy(buf + n, row, o->D * sizeof(double));
            }
    return 0;
}

void orc_set_cur(orc_ctx *o, int which) { o->cur = which ? o->Up : o->U; }
int orc_get_cur(orc_ctx *o) { return o->cur == o->U ? 0 : 1; }

void orc_get_scalars(orc_ctx *o, double *out)
{
    out[0] = o->dt; out[1] = o->dtx; out[2] = o->dty; out[3] = o->dtz;
    out[4] = o->X; out[5] = o->k_min; out[6] = o->k_max;
    out[7] = o->Ud; out[8] = o->Vd; out[9] = o->Wd; out[10] = o->step;
    out[11] = o->DD; out[12] = o->lambda_L; out[13] = o->cp_Pr_T;
    out[14] = o->p.maxCoNum; out[15] = o->counter; out[16] = o->last_maxco;
}

/* src/helpers.c:47-50 */
void orc_set_dt(orc_ctx *o, double dt)
{
    o->dt = dt;
    o->dtx = o->dt / o->p.deltaX; o->dty = o->dt / o->p.deltaY; o->dtz = o->dt / o->p.deltaZ;
}

void orc_set_disturbance(orc_ctx *o, unsigned kmin, unsigned kmax, double ud, double vd, double wd)
{
    o->k_min = kmin; o->k_max = kmax; o->Ud = ud; o->Vd = vd; o->Wd = wd;
}

/* ------------------------------------------------------------------------
 * A1: ghost cells, src/boundCondInGhostCells.c:10-96.
 * Spatial (reference): x inflow step profile / outflow with E rebuilt at
 * P = 1e5, then z periodic over i in [0,LEN+1], then y slip over all i, k.
 * Temporal (project extension): x periodic, z periodic, y zero-gradient, in
 * the same x -> z -> y order so that edges and corners are filled alike.
 * ------------------------------------------------------------------------ */
void orc_ghost_bc(orc_ctx *o)
{
    const int L = o->L, H = o->H, D = o->D;
    double **u = o->cur;
    int i, j, k, v;
    if (o->p.setup == ORC_SETUP_SPATIAL) {
        double P = 100000., R = 1.0, U;
        U = 76.4; /* :17-28 */
        for (j = 1; j <= H / 2; j++)
            for (k = 1; k < D + 1; k++) {
                size_t c = IC(o, 0, j, k);
                u[0][c] = R; u[1][c] = R * U; u[2][c] = 0.; u[3][c] = 0.;
                u[4][c] = P / K_1 + 0.5 * R * (U * U);
            }
        U = 200; /* :31-40 */
        for (j = H / 2 + 1; j < H + 1; j++)
            for (k = 1; k < D + 1; k++) {
                size_t c = IC(o, 0, j, k);
                u[0][c] = R; u[1][c] = R * U; u[2][c] = 0.; u[3][c] = 0.;
                u[4][c] = P / K_1 + 0.5 * R * (U * U);
            }
        /* :44-52, outflow; the momenta are held in R,U,V,W */
        for (j = 1; j < H + 1; j++)
            for (k = 1; k < D + 1; k++) {
                size_t c = IC(o, L + 1, j, k), s = IC(o, L, j, k);
                double r = u[0][s], mu_ = u[1][s], mv = u[2][s], mw = u[3][s];
                u[0][c] = r; u[1][c] = mu_; u[2][c] = mv; u[3][c] = mw;
                u[4][c] = P / K_1 + 0.5 * (mu_ * mu_ + mv * mv + mw * mw) / r;
            }
    } else {
        for (j = 1; j < H + 1; j++)
            for (k = 1; k < D + 1; k++)
                for (v = 0; v < 5; v++) {
                    u[v][IC(o, 0, j, k)] = u[v][IC(o, L, j, k)];
                    u[v][IC(o, L + 1, j, k)] = u[v][IC(o, 1, j, k)];
                }
    }
    /* :58-73, z periodic */
    for (i = 0; i <= L + 1; i++)
        for (j = 1; j < H + 1; j++)
            for (v = 0; v < 5; v++) {
                u[v][IC(o, i, j, 0)] = u[v][IC(o, i, j, D)];
                u[v][IC(o, i, j, D + 1)] = u[v][IC(o, i, j, 1)];
            }
    /* :79-94, y slip (reference) or zero-gradient (temporal) */
    for (i = 0; i <= L + 1; i++)
        for (k = 0; k <= D + 1; k++)
            for (v = 0; v < 5; v++) {
                double sgn = (v == 2 && o->p.setup == ORC_SETUP_SPATIAL) ? -1.0 : 1.0;
                if (sgn < 0) {
                    u[v][IC(o, i, 0, k)] = -u[v][IC(o, i, 1, k)];
                    u[v][IC(o, i, H + 1, k)] = -u[v][IC(o, i, H, k)];
                } else {
                    u[v][IC(o, i, 0, k)] = u[v][IC(o, i, 1, k)];
                    u[v][IC(o, i, H + 1, k)] = u[v][IC(o, i, H, k)];
                }
            }
}

/* ------------------------------------------------------------------------
 * A2: characteristic reconstruction, src/reconstruction.c:17-345.
 * ------------------------------------------------------------------------ */

/* Chakravarthy-Osher minmod with compression 4, src/reconstruction.c:17-24 */
double orc_minmod(double x, double y)
{
    double ay;
    if (x * y <= 0) return 0;
    ay = ((y *= 4.0) > 0) ? y : -y;
    if (x > 0) return (x < ay) ? x : ay;
    return ((-x < ay) ? x : -ay);
}

/* Per-cell constants shared by the three directions, :63-88 */
typedef struct {
    double u[5];        /* u1..u5 */
    double U, V, W, C;  /* primitives */
    double aa, ll, ee, gg, hh, nn, S11;
    double u_hh, v_hh, w_hh, u_ee, v_ee, w_ee;
} cellc;

/* One direction of :90-170 (x), :173-256 (y), :258-341 (z).
 * n  = index (1..4) of the normal momentum in u[]; t1, t2 = the tangential
 * momenta in the order the reference permutes them (x: 2 3 4, y: 3 4 2,
 * z: 4 2 3).  vn, vt1, vt2 = the matching velocities; bn, bt1, bt2 = -(K-1)
 * times them; n_hh/t1_hh/t2_hh, n_ee/t1_ee/t2_ee = U*hh etc.; t2_ee is the
 * coefficient the reference applies to the t2 momentum (src/reconstruction.c:328
 * uses w_ee for rho v in the z sweep; it is passed as given).
 * fw[5], bw[5] = conserved values of the forward and backward neighbours in
 * the order (rho, n, t1, t2, E).  hi[5] receives the state on the face towards
 * the forward neighbour, lo[5] the state on the face towards the backward one,
 * both in natural variable order. */
static void recon_dir(const cellc *c, int n, int t1, int t2, double vn, double vt1, double vt2,
                      double bn, double bt1, double bt2, double n_hh, double t1_hh, double t2_hh,
                      double n_ee, double t1_ee, double t2_ee, const double *fw, const double *bw,
                      double *hi, double *lo)
{
    double m1, m2, m3, m4, m5, w1, w2, w3, w4, w5;
    double M1, M2, M3, M4, M5, W1, W2, W3, W4, W5;
    double _M1, _M2, _M3, _M4, _M5, _W1, _W2, _W3, _W4, _W5;
    double S12, S41, S42, S51, S52, _S24, _S25, _S54, _S55;
    double k1, k2, k3, k4, k5, kk, mm;
    const double *u = c->u;
    const double C = c->C;
    mm = vn * c->ll;
    m1 = fw[0] - u[0]; m2 = fw[1] - u[n]; m3 = fw[2] - u[t1]; m4 = fw[3] - u[t2]; m5 = fw[4] - u[4];
    w1 = u[0] - bw[0]; w2 = u[n] - bw[1]; w3 = u[t1] - bw[2]; w4 = u[t2] - bw[3]; w5 = u[4] - bw[4];
    S41 = c->aa - (kk = C * vn);
    S51 = c->aa + kk;
    S12 = S42 = S52 = bn;
    S42 += C;
    S52 -= C;
    kk = K_1 * m5; k2 = bt1 * m3; k3 = bt2 * m4;
    M1 = c->S11 * m1 + S12 * m2 + k2 + k3 + kk;
    M2 = -vt1 * m1 + m3;
    M3 = -vt2 * m1 + m4;
    M4 = S41 * m1 + S42 * m2 + k2 + k3 + kk;
    M5 = S51 * m1 + S52 * m2 + k2 + k3 + kk;
    kk = K_1 * w5; k2 = bt1 * w3; k3 = bt2 * w4;
    W1 = c->S11 * w1 + S12 * w2 + k2 + k3 + kk;
    W2 = -vt1 * w1 + w3;
    W3 = -vt2 * w1 + w4;
    W4 = S41 * w1 + S42 * w2 + k2 + k3 + kk;
    W5 = S51 * w1 + S52 * w2 + k2 + k3 + kk;
    _M1 = orc_minmod(M1, W1); _M2 = orc_minmod(M2, W2); _M3 = orc_minmod(M3, W3);
    _M4 = orc_minmod(M4, W4); _M5 = orc_minmod(M5, W5);
    _W1 = orc_minmod(W1, M1); _W2 = orc_minmod(W2, M2); _W3 = orc_minmod(W3, M3);
    _W4 = orc_minmod(W4, M4); _W5 = orc_minmod(W5, M5);
    _S24 = n_ee + c->ll; _S25 = n_ee - c->ll;
    _S54 = _S55 = c->nn + H_K_1;
    _S54 += mm; _S55 -= mm;
    /* face towards the forward neighbour, :148-158 */
    k1 = _M1 * C1 + _W1 * C2; k2 = _M2 * C1 + _W2 * C2; k3 = _M3 * C1 + _W3 * C2;
    k4 = _M4 * C1 + _W4 * C2; k5 = _M5 * C1 + _W5 * C2;
    kk = k4 + k5;
    hi[0] = u[0] + c->hh * k1 + c->ee * kk;
    hi[n] = u[n] + n_hh * k1 + _S24 * k4 + _S25 * k5;
    hi[t1] = u[t1] + t1_hh * k1 + k2 + t1_ee * kk;
    hi[t2] = u[t2] + t2_hh * k1 + k3 + t2_ee * kk;
    hi[4] = u[4] + c->gg * k1 + vt1 * k2 + vt2 * k3 + _S54 * k4 + _S55 * k5;
    /* face towards the backward neighbour, :160-170 */
    k1 = _M1 * C2 + _W1 * C1; k2 = _M2 * C2 + _W2 * C1; k3 = _M3 * C2 + _W3 * C1;
    k4 = _M4 * C2 + _W4 * C1; k5 = _M5 * C2 + _W5 * C1;
    kk = k4 + k5;
    lo[0] = u[0] - c->hh * k1 - c->ee * kk;
    lo[n] = u[n] - n_hh * k1 - _S24 * k4 - _S25 * k5;
    lo[t1] = u[t1] - t1_hh * k1 - k2 - t1_ee * kk;
    lo[t2] = u[t2] - t2_hh * k1 - k3 - t2_ee * kk;
    lo[4] = u[4] - c->gg * k1 - vt1 * k2 - vt2 * k3 - _S54 * k4 - _S55 * k5;
}

/* ------------------------------------------------------------------------
 * PPM reconstruction (project extension; the reference has none): Colella &
 * Woodward (1984) on the characteristic variables of the reference's
 * reconstruction (the transform of src/reconstruction.c:104-129 and its
 * inverse, :148-158, with cell i's constants).  Per characteristic field:
 * monotonised-central slopes (CW84 eq. 1.8) of cells i-1, i, i+1 from the
 * four differences around cell i, edge values a_{i+1/2} - a_i =
 * 1/2 d_{i+1/2} - (da_{i+1} - da_i)/6 and a_{i-1/2} - a_i =
 * -1/2 d_{i-1/2} - (da_i - da_{i-1})/6 (eq. 1.6), the monotonicity limiter
 * (eq. 1.10), and the two face states.  Cells next to a domain boundary in
 * the sweep direction (one ghost layer: no second neighbour) use the
 * reference's reconstruction in that direction.
 * ------------------------------------------------------------------------ */
static double orc_mc(double a, double b)
{
    double m, t;
    if (a * b <= 0.0) return 0.0;
    m = 0.5 * fabs(a + b);
    t = 2.0 * fabs(a);
    if (t < m) m = t;
    t = 2.0 * fabs(b);
    if (t < m) m = t;
    return a > 0.0 ? m : -m;
}

/* d: a difference in the sweep's order (rho, normal, t1, t2, E) -> M */
static void char_fwd(const cellc *c, double vn, double vt1, double vt2, double bn, double bt1, double bt2,
                     const double *d, double *M)
{
    double S12, S41, S42, S51, S52, kk, k2, k3;
    const double C = c->C;
    S41 = c->aa - (kk = C * vn);
    S51 = c->aa + kk;
    S12 = S42 = S52 = bn;
    S42 += C;
    S52 -= C;
    kk = K_1 * d[4]; k2 = bt1 * d[2]; k3 = bt2 * d[3];
    M[0] = c->S11 * d[0] + S12 * d[1] + k2 + k3 + kk;
    M[1] = -vt1 * d[0] + d[2];
    M[2] = -vt2 * d[0] + d[3];
    M[3] = S41 * d[0] + S42 * d[1] + k2 + k3 + kk;
    M[4] = S51 * d[0] + S52 * d[1] + k2 + k3 + kk;
}

/* out = u + R q (natural variable order) */
static void char_inv(const cellc *c, int n, int t1, int t2, double vn, double vt1, double vt2, double n_hh,
                     double t1_hh, double t2_hh, double n_ee, double t1_ee, double t2_ee, const double *q, double *out)
{
    const double *u = c->u;
    const double mm = vn * c->ll;
    double _S24, _S25, _S54, _S55, kk;
    _S24 = n_ee + c->ll; _S25 = n_ee - c->ll;
    _S54 = _S55 = c->nn + H_K_1;
    _S54 += mm; _S55 -= mm;
    kk = q[3] + q[4];
    out[0] = u[0] + c->hh * q[0] + c->ee * kk;
    out[n] = u[n] + n_hh * q[0] + _S24 * q[3] + _S25 * q[4];
    out[t1] = u[t1] + t1_hh * q[0] + q[1] + t1_ee * kk;
    out[t2] = u[t2] + t2_hh * q[0] + q[2] + t2_ee * kk;
    out[4] = u[4] + c->gg * q[0] + vt1 * q[1] + vt2 * q[2] + _S54 * q[3] + _S55 * q[4];
}

/* m2, m1, p1, p2: neighbours at -2, -1, +1, +2 in the sweep's order */
static void recon_dir_ppm(const cellc *c, int n, int t1, int t2, double vn, double vt1, double vt2, double bn,
                          double bt1, double bt2, double n_hh, double t1_hh, double t2_hh, double n_ee, double t1_ee,
                          double t2_ee, const double *m2, const double *m1, const double *p1, const double *p2,
                          double *hi, double *lo)
{
    const double *u = c->u;
    const double uc[5] = {u[0], u[n], u[t1], u[t2], u[4]};
    double d[4][5], W[4][5], qR[5], qL[5];
    int v;
    for (v = 0; v < 5; v++) {
        d[0][v] = m1[v] - m2[v];
        d[1][v] = uc[v] - m1[v];
        d[2][v] = p1[v] - uc[v];
        d[3][v] = p2[v] - p1[v];
    }
    for (v = 0; v < 4; v++) char_fwd(c, vn, vt1, vt2, bn, bt1, bt2, d[v], W[v]);
    for (v = 0; v < 5; v++) {
        const double dm = orc_mc(W[0][v], W[1][v]), d0 = orc_mc(W[1][v], W[2][v]), dp = orc_mc(W[2][v], W[3][v]);
        double r = 0.5 * W[2][v] - (dp - d0) / 6.0, l = -0.5 * W[1][v] - (d0 - dm) / 6.0;
        if (r * l >= 0.0) {
            r = 0.0;
            l = 0.0;
        } else if (fabs(r) > 2.0 * fabs(l)) {
            r = -2.0 * l;
        } else if (fabs(l) > 2.0 * fabs(r)) {
            l = -2.0 * r;
        }
        qR[v] = r;
        qL[v] = l;
    }
    char_inv(c, n, t1, t2, vn, vt1, vt2, n_hh, t1_hh, t2_hh, n_ee, t1_ee, t2_ee, qR, hi);
    char_inv(c, n, t1, t2, vn, vt1, vt2, n_hh, t1_hh, t2_hh, n_ee, t1_ee, t2_ee, qL, lo);
}

void orc_reconstruct(orc_ctx *o)
{
    const int L = o->L, H = o->H, D = o->D;
    double **u = o->cur;
    int i, j, k, v;
    for (i = 1; i < L + 1; i++)
        for (j = 1; j < H + 1; j++)
            for (k = 1; k < D + 1; k++) {
                cellc c;
                double R, P, ff, bb, cc, dd;
                double fw[5], bw[5], hi[5], lo[5];
                size_t ic = IC(o, i, j, k), f, b;
                for (v = 0; v < 5; v++) c.u[v] = u[v][ic];
                /* :71-76 */
                R = 1. / c.u[0];
                c.U = c.u[1] * R; c.V = c.u[2] * R; c.W = c.u[3] * R;
                P = (c.u[4] - 0.5 * (c.u[1] * c.u[1] + c.u[2] * c.u[2] + c.u[3] * c.u[3]) * R) * K_1;
                c.C = sqrt(K * P * R);
                /* :79-88 */
                ff = c.U * c.U + c.V * c.V + c.W * c.W;
                c.aa = K_1_2 * ff;
                bb = NK_1 * c.U; cc = NK_1 * c.V; dd = NK_1 * c.W;
                c.ll = 1. / (c.C + c.C);
                c.ee = c.ll / c.C;
                c.gg = -ff * c.ee;
                c.hh = -(c.ee + c.ee);
                c.S11 = c.aa - c.C * c.C; /* :104 */
                /* :142-145 */
                c.u_hh = c.U * c.hh; c.v_hh = c.V * c.hh; c.w_hh = c.W * c.hh;
                c.u_ee = c.U * c.ee; c.v_ee = c.V * c.ee; c.w_ee = c.W * c.ee;
                c.nn = -0.5 * c.gg;
                /* x sweep, :90-170: (rho, rho u, rho v, rho w, E) */
                f = IC(o, i + 1, j, k); b = IC(o, i - 1, j, k);
                fw[0] = u[0][f]; fw[1] = u[1][f]; fw[2] = u[2][f]; fw[3] = u[3][f]; fw[4] = u[4][f];
                bw[0] = u[0][b]; bw[1] = u[1][b]; bw[2] = u[2][b]; bw[3] = u[3][b]; bw[4] = u[4][b];
                if (o->p.recon == 1 && i >= 2 && i <= L - 1) {
                    double m2[5], p2[5];
                    size_t a2 = IC(o, i + 2, j, k), b2 = IC(o, i - 2, j, k);
                    for (v = 0; v < 5; v++) { p2[v] = u[v][a2]; m2[v] = u[v][b2]; }
                    recon_dir_ppm(&c, 1, 2, 3, c.U, c.V, c.W, bb, cc, dd, c.u_hh, c.v_hh, c.w_hh,
                                  c.u_ee, c.v_ee, c.w_ee, m2, bw, fw, p2, hi, lo);
                } else {
                    recon_dir(&c, 1, 2, 3, c.U, c.V, c.W, bb, cc, dd, c.u_hh, c.v_hh, c.w_hh,
                              c.u_ee, c.v_ee, c.w_ee, fw, bw, hi, lo);
                }
                for (v = 0; v < 5; v++) {
                    o->fs[0][0][v][IX(o, i, j - 1, k - 1)] = hi[v];
                    o->fs[0][1][v][IX(o, i - 1, j - 1, k - 1)] = lo[v];
                }
                /* y sweep, :173-256: momenta permuted 3-4-2 */
                f = IC(o, i, j + 1, k); b = IC(o, i, j - 1, k);
                fw[0] = u[0][f]; fw[1] = u[2][f]; fw[2] = u[3][f]; fw[3] = u[1][f]; fw[4] = u[4][f];
                bw[0] = u[0][b]; bw[1] = u[2][b]; bw[2] = u[3][b]; bw[3] = u[1][b]; bw[4] = u[4][b];
                if (o->p.recon == 1 && j >= 2 && j <= H - 1) {
                    double m2[5], p2[5];
                    size_t a2 = IC(o, i, j + 2, k), b2 = IC(o, i, j - 2, k);
                    p2[0] = u[0][a2]; p2[1] = u[2][a2]; p2[2] = u[3][a2]; p2[3] = u[1][a2]; p2[4] = u[4][a2];
                    m2[0] = u[0][b2]; m2[1] = u[2][b2]; m2[2] = u[3][b2]; m2[3] = u[1][b2]; m2[4] = u[4][b2];
                    recon_dir_ppm(&c, 2, 3, 1, c.V, c.W, c.U, cc, dd, bb, c.v_hh, c.w_hh, c.u_hh,
                                  c.v_ee, c.w_ee, c.u_ee, m2, bw, fw, p2, hi, lo);
                } else {
                    recon_dir(&c, 2, 3, 1, c.V, c.W, c.U, cc, dd, bb, c.v_hh, c.w_hh, c.u_hh,
                              c.v_ee, c.w_ee, c.u_ee, fw, bw, hi, lo);
                }
                for (v = 0; v < 5; v++) {
                    o->fs[1][0][v][IY(o, i - 1, j, k - 1)] = hi[v];
                    o->fs[1][1][v][IY(o, i - 1, j - 1, k - 1)] = lo[v];
                }
                /* z sweep, :258-341: momenta permuted 4-2-3; :328,:340 apply
                 * w_ee to rho v */
                f = IC(o, i, j, k + 1); b = IC(o, i, j, k - 1);
                fw[0] = u[0][f]; fw[1] = u[3][f]; fw[2] = u[1][f]; fw[3] = u[2][f]; fw[4] = u[4][f];
                bw[0] = u[0][b]; bw[1] = u[3][b]; bw[2] = u[1][b]; bw[3] = u[2][b]; bw[4] = u[4][b];
                if (o->p.recon == 1 && k >= 2 && k <= D - 1) {
                    double m2[5], p2[5];
                    size_t a2 = IC(o, i, j, k + 2), b2 = IC(o, i, j, k - 2);
                    p2[0] = u[0][a2]; p2[1] = u[3][a2]; p2[2] = u[1][a2]; p2[3] = u[2][a2]; p2[4] = u[4][a2];
                    m2[0] = u[0][b2]; m2[1] = u[3][b2]; m2[2] = u[1][b2]; m2[3] = u[2][b2]; m2[4] = u[4][b2];
                    recon_dir_ppm(&c, 3, 1, 2, c.W, c.U, c.V, dd, bb, cc, c.w_hh, c.u_hh, c.v_hh,
                                  c.w_ee, c.u_ee, c.w_ee, m2, bw, fw, p2, hi, lo);
                } else {
                    recon_dir(&c, 3, 1, 2, c.W, c.U, c.V, dd, bb, cc, c.w_hh, c.u_hh, c.v_hh,
                              c.w_ee, c.u_ee, c.w_ee, fw, bw, hi, lo);
                }
                for (v = 0; v < 5; v++) {
                    o->fs[2][0][v][IZ(o, i - 1, j - 1, k)] = hi[v];
                    o->fs[2][1][v][IZ(o, i - 1, j - 1, k - 1)] = lo[v];
                }
            }
}

/* ------------------------------------------------------------------------
 * A3: boundary face states, src/bounCondOnInterfaces.c:11-110 (spatial);
 * temporal: x periodic like the reference's z rule (:94-109), y zero-gradient.
 * ------------------------------------------------------------------------ */
void orc_interface_bc(orc_ctx *o)
{
    const int L = o->L, H = o->H, D = o->D;
    double *(*xl) = o->fs[0][0], *(*xr) = o->fs[0][1];
    double *(*yl) = o->fs[1][0], *(*yr) = o->fs[1][1];
    double *(*zl) = o->fs[2][0], *(*zr) = o->fs[2][1];
    int i, j, k, v;
    if (o->p.setup == ORC_SETUP_SPATIAL) {
        double P = 100000., U = 76.4, V = 0., W = 0., R = 1.0;
        /* :17-29 */
        for (j = 0; j < H / 2; j++)
            for (k = 0; k < D; k++) {
                size_t f = IX(o, 0, j, k);
                xl[0][f] = R; xl[1][f] = R * U; xl[2][f] = 0.; xl[3][f] = 0.;
                xl[4][f] = P / K_1 + 0.5 * R * (U * U);
            }
        /* :31-49, the disturbance block */
        for (j = H / 2; j < H / 2 + o->p.BL_HIG; j++)
            for (k = 0; k < D; k++) {
                size_t f = IX(o, 0, j, k);
                unsigned ku = (unsigned)k;
                if (o->k_max > o->k_min) {
                    if (ku >= o->k_min && ku < o->k_max) { U = 200. + o->Ud; V = o->Vd; W = o->Wd; }
                    else { U = 200.; V = W = 0.; }
                } else {
                    if (ku >= o->k_max && ku < o->k_min) { U = 200.; V = W = 0.; }
                    else { U = 200. + o->Ud; V = o->Vd; W = o->Wd; }
                }
                xl[0][f] = R; xl[1][f] = R * U; xl[2][f] = R * V; xl[3][f] = R * W;
                xl[4][f] = P / K_1 + 0.5 * R * (U * U + V * V + W * W);
            }
        /* :51-60 */
        U = 200.;
        for (j = H / 2 + o->p.BL_HIG; j < H; j++)
            for (k = 0; k < D; k++) {
                size_t f = IX(o, 0, j, k);
                xl[0][f] = R; xl[1][f] = R * U; xl[2][f] = 0.; xl[3][f] = 0.;
                xl[4][f] = P / K_1 + 0.5 * R * (U * U);
            }
        /* :62-71 outflow: plus-side state = minus-side momenta, E at P = 1e5 */
        P = 100000.;
        for (j = 0; j < H; j++)
            for (k = 0; k < D; k++) {
                size_t f = IX(o, L, j, k);
                double r = xl[0][f], mu_ = xl[1][f], mv = xl[2][f], mw = xl[3][f];
                xr[0][f] = r; xr[1][f] = mu_; xr[2][f] = mv; xr[3][f] = mw;
                xr[4][f] = P / K_1 + 0.5 * (mu_ * mu_ + mv * mv + mw * mw) / r;
            }
        /* :75-90, y slip */
        for (i = 0; i < L; i++)
            for (k = 0; k < D; k++)
                for (v = 0; v < 5; v++) {
                    size_t f0 = IY(o, i, 0, k), fH = IY(o, i, H, k);
                    if (v == 2) { yl[v][f0] = -yr[v][f0]; yr[v][fH] = -yl[v][fH]; }
                    else { yl[v][f0] = yr[v][f0]; yr[v][fH] = yl[v][fH]; }
                }
    } else {
        for (j = 0; j < H; j++)
            for (k = 0; k < D; k++)
                for (v = 0; v < 5; v++) {
                    xl[v][IX(o, 0, j, k)] = xl[v][IX(o, L, j, k)];
                    xr[v][IX(o, L, j, k)] = xr[v][IX(o, 0, j, k)];
                }
        for (i = 0; i < L; i++)
            for (k = 0; k < D; k++)
                for (v = 0; v < 5; v++) {
                    yl[v][IY(o, i, 0, k)] = yr[v][IY(o, i, 0, k)];
                    yr[v][IY(o, i, H, k)] = yl[v][IY(o, i, H, k)];
                }
    }
    /* :94-109, z periodic */
    for (i = 0; i < L; i++)
        for (j = 0; j < H; j++)
            for (v = 0; v < 5; v++) {
                zl[v][IZ(o, i, j, 0)] = zl[v][IZ(o, i, j, D)];
                zr[v][IZ(o, i, j, D)] = zr[v][IZ(o, i, j, 0)];
            }
}

/* ------------------------------------------------------------------------
 * A5: test filter, src/turbulence.c:17-100, box kernel {1/3,1/3,1/3} (:113),
 * with the zero-initialised temporaries of the oracle convention.
 * ------------------------------------------------------------------------ */
static void filter_ctx(int L, int H, int D, const double *U, double *out, double *T2)
{
    const double h0 = 1. / 3., h1 = 1. / 3., h2 = 1. / 3.;
    const size_t pj = (size_t)D + 2, pi = pj * ((size_t)H + 2), n = pi * ((size_t)L + 2);
    double *T1 = out; /* pass 3 writes back into pass 1's buffer, :80-95 */
    int i, j, k;
    memset(T1, 0, n * sizeof(double));
    memset(T2, 0, n * sizeof(double));
    /* :47-61 y pass: i in [0,LEN], j in [1,HIG], k in [0,DEP] */
    for (i = 0; i < L + 1; i++)
        for (j = 1; j < H + 1; j++)
            for (k = 0; k < D + 1; k++) {
                size_t c = i * pi + j * pj + k;
                double t = 0.;
                t += U[c - pj] * h0; t += U[c] * h1; t += U[c + pj] * h2;
                T1[c] = t;
            }
    /* :63-77 z pass: i in [0,LEN], j in [0,HIG], k in [1,DEP] */
    for (i = 0; i < L + 1; i++)
        for (j = 0; j < H + 1; j++)
            for (k = 1; k < D + 1; k++) {
                size_t c = i * pi + j * pj + k;
                double t = 0.;
                t += T1[c - 1] * h0; t += T1[c] * h1; t += T1[c + 1] * h2;
                T2[c] = t;
            }
    /* :80-95 x pass: i in [1,LEN], j in [0,HIG], k in [0,DEP] */
    for (i = 1; i < L + 1; i++)
        for (j = 0; j < H + 1; j++)
            for (k = 0; k < D + 1; k++) {
                size_t c = i * pi + j * pj + k;
                double t = 0.;
                t += T2[c - pi] * h0; t += T2[c] * h1; t += T2[c + pi] * h2;
                T1[c] = t;
            }
}

void orc_filter(const orc_params *p, const double *in, double *out)
{
    size_t n = ((size_t)p->LEN + 2) * ((size_t)p->HIG + 2) * ((size_t)p->DEP + 2);
    double *t2 = malloc(n * sizeof(double));
    filter_ctx(p->LEN, p->HIG, p->DEP, in, out, t2);
    free(t2);
}

/* ------------------------------------------------------------------------
 * A6: dynamic Smagorinsky (Germano-Lilly), src/turbulence.c:103-507, on U^n.
 * The reference filters all nine u_i u_j products; the symmetric pairs are
 * bitwise equal (v*u == u*v), so six filters give the same nine fields.
 * ------------------------------------------------------------------------ */
void orc_dynamic_smagorinsky(orc_ctx *o)
{
    const int L = o->L, H = o->H, D = o->D;
    const size_t n = o->ncell, pj = o->pj, pi = o->pi;
    double *rho = o->U[0], *ru = o->U[1], *rv = o->U[2], *rw = o->U[3];
    double *u = malloc(n * sizeof(double)), *v = malloc(n * sizeof(double)), *w = malloc(n * sizeof(double));
    double *prod[6], *fprod[6], *fu, *fv, *fw, *A[6], *fA[6], *mag, *tmp;
    int a, i, j, k;
    size_t c;
    for (a = 0; a < 6; a++) {
        prod[a] = malloc(n * sizeof(double));
        fprod[a] = malloc(n * sizeof(double));
        A[a] = calloc(n, sizeof(double)); /* ghost layer never written: 0 */
        fA[a] = malloc(n * sizeof(double));
    }
    fu = malloc(n * sizeof(double)); fv = malloc(n * sizeof(double)); fw = malloc(n * sizeof(double));
    mag = calloc(n, sizeof(double));
    tmp = malloc(n * sizeof(double));
    double *B[6];
    for (a = 0; a < 6; a++) B[a] = calloc(n, sizeof(double));
    /* :197-209 */
    for (c = 0; c < n; c++) {
        double rr = 1. / rho[c];
        u[c] = ru[c] * rr; v[c] = rv[c] * rr; w[c] = rw[c] * rr;
    }
    /* :213-230; order 11 12 13 22 23 33 */
    for (c = 0; c < n; c++) {
        prod[0][c] = u[c] * u[c]; prod[1][c] = u[c] * v[c]; prod[2][c] = u[c] * w[c];
        prod[3][c] = v[c] * v[c]; prod[4][c] = v[c] * w[c]; prod[5][c] = w[c] * w[c];
    }
    /* :233-248 */
    filter_ctx(L, H, D, u, fu, tmp);
    filter_ctx(L, H, D, v, fv, tmp);
    filter_ctx(L, H, D, w, fw, tmp);
    for (a = 0; a < 6; a++) filter_ctx(L, H, D, prod[a], fprod[a], tmp);
    /* :250-382 interior: Leonard stress into prod[], |S|, A, B */
    for (i = 1; i < L + 1; i++)
        for (j = 1; j < H + 1; j++)
            for (k = 1; k < D + 1; k++) {
                double du_dx, du_dy, du_dz, dv_dx, dv_dy, dv_dz, dw_dx, dw_dy, dw_dz;
                double S11, S12, S13, S21, S22, S23, S31, S32, S33, S, S_;
                c = i * pi + j * pj + k;
                prod[0][c] = fprod[0][c] - fu[c] * fu[c];
                prod[1][c] = fprod[1][c] - fu[c] * fv[c];
                prod[2][c] = fprod[2][c] - fu[c] * fw[c];
                prod[3][c] = fprod[3][c] - fv[c] * fv[c];
                prod[4][c] = fprod[4][c] - fv[c] * fw[c];
                prod[5][c] = fprod[5][c] - fw[c] * fw[c];
                /* :273-311 */
                du_dx = (u[c + pi] - u[c - pi]) * o->r2dx;
                du_dy = (u[c + pj] - u[c - pj]) * o->r2dy;
                du_dz = (u[c + 1] - u[c - 1]) * o->r2dz;
                dv_dx = (v[c + pi] - v[c - pi]) * o->r2dx;
                dv_dy = (v[c + pj] - v[c - pj]) * o->r2dy;
                dv_dz = (v[c + 1] - v[c - 1]) * o->r2dz;
                dw_dx = (w[c + pi] - w[c - pi]) * o->r2dx;
                dw_dy = (w[c + pj] - w[c - pj]) * o->r2dy;
                dw_dz = (w[c + 1] - w[c - 1]) * o->r2dz;
                S11 = du_dx; S12 = 0.5 * (du_dy + dv_dx); S13 = 0.5 * (du_dz + dw_dx);
                S21 = S12; S22 = dv_dy; S23 = 0.5 * (dv_dz + dw_dy);
                S31 = S13; S32 = S23; S33 = dw_dz;
                S = sqrt(2 * (S11 * S11 + S12 * S12 + S13 * S13 + S21 * S21 + S22 * S22 + S23 * S23 +
                              S31 * S31 + S32 * S32 + S33 * S33));
                mag[c] = S;
                A[0][c] = S * S11; A[1][c] = S * S12; A[2][c] = S * S13;
                A[3][c] = S * S22; A[4][c] = S * S23; A[5][c] = S * S33;
                /* :316-366 */
                du_dx = (fu[c + pi] - fu[c - pi]) * o->r2dx;
                du_dy = (fu[c + pj] - fu[c - pj]) * o->r2dy;
                du_dz = (fu[c + 1] - fu[c - 1]) * o->r2dz;
                dv_dx = (fv[c + pi] - fv[c - pi]) * o->r2dx;
                dv_dy = (fv[c + pj] - fv[c - pj]) * o->r2dy;
                dv_dz = (fv[c + 1] - fv[c - 1]) * o->r2dz;
                dw_dx = (fw[c + pi] - fw[c - pi]) * o->r2dx;
                dw_dy = (fw[c + pj] - fw[c - pj]) * o->r2dy;
                dw_dz = (fw[c + 1] - fw[c - 1]) * o->r2dz;
                S11 = du_dx; S12 = 0.5 * (du_dy + dv_dx); S13 = 0.5 * (du_dz + dw_dx);
                S21 = S12; S22 = dv_dy; S23 = 0.5 * (dv_dz + dw_dy);
                S31 = S13; S32 = S23; S33 = dw_dz;
                S_ = sqrt(2 * (S11 * S11 + S12 * S12 + S13 * S13 + S21 * S21 + S22 * S22 + S23 * S23 +
                               S31 * S31 + S32 * S32 + S33 * S33));
                B[0][c] = S_ * S11; B[1][c] = S_ * S12; B[2][c] = S_ * S13;
                B[3][c] = S_ * S22; B[4][c] = S_ * S23; B[5][c] = S_ * S33;
            }
    /* :386-396 */
    for (a = 0; a < 6; a++) filter_ctx(L, H, D, A[a], fA[a], tmp);
    /* :398-445 */
    for (i = 1; i < L + 1; i++)
        for (j = 1; j < H + 1; j++)
            for (k = 1; k < D + 1; k++) {
                double M11, M12, M13, M22, M23, M33, L11, L12, L13, L22, L23, L33;
                double tr, LLMM, MMMM, Cd;
                c = i * pi + j * pj + k;
                M11 = o->DD * (4 * B[0][c] - fA[0][c]);
                M12 = o->DD * (4 * B[1][c] - fA[1][c]);
                M13 = o->DD * (4 * B[2][c] - fA[2][c]);
                M22 = o->DD * (4 * B[3][c] - fA[3][c]);
                M23 = o->DD * (4 * B[4][c] - fA[4][c]);
                M33 = o->DD * (4 * B[5][c] - fA[5][c]);
                L11 = prod[0][c]; L12 = prod[1][c]; L13 = prod[2][c];
                L22 = prod[3][c]; L23 = prod[4][c]; L33 = prod[5][c];
                tr = -(1.0 / 3.0) * (L11 + L22 + L33);
                L11 += tr; L22 += tr; L33 += tr;
                LLMM = (L11 * M11 + L12 * M12 + L13 * M13 + L12 * M12 + L22 * M22 + L23 * M23 +
                        L13 * M13 + L23 * M23 + L33 * M33);
                MMMM = (M11 * M11 + M12 * M12 + M13 * M13 + M12 * M12 + M22 * M22 + M23 * M23 +
                        M13 * M13 + M23 * M23 + M33 * M33);
                Cd = -0.5 * (LLMM / (MMMM + SMALL));
                if (Cd > 0.15) Cd = 0.15;
                else if (Cd < 0.0) Cd = 0.0;
                o->mu[c] = rho[c] * Cd * o->DD * mag[c];
            }
    free(u); free(v); free(w); free(fu); free(fv); free(fw); free(mag); free(tmp);
    for (a = 0; a < 6; a++) { free(prod[a]); free(fprod[a]); free(A[a]); free(fA[a]); free(B[a]); }
}

/* ------------------------------------------------------------------------
 * A4: fluxes, src/fluxes.c:12-573.
 * ------------------------------------------------------------------------ */

/* Linearised characteristic Riemann solve of one face, :61-113 (x),
 * :230-282 (y), :401-453 (z).  L[5], Rt[5]: minus/plus conserved states in
 * natural order; n = index of the normal momentum (1..3).  Outputs the
 * interface density, normal velocity, pressure and the two upwinded
 * tangential velocities in natural order (vel[3]). */
static void riemann(const double *Lm, const double *Rp, int n, double *Rho, double *Pr, double *vel)
{
    double _R, _U, _V, _W, _P, _C, _jo, _jp, _jm, RU;
    double R_, U_, V_, W_, P_, C_, jo_, jp_, jm_;
    double Un, C, C_p, C_m, C_o, al_p, al_m, al_o, J_p, J_m, J_o, P;
    double lv[3], rv[3];
    _R = Lm[0]; _U = Lm[1] / _R; _V = Lm[2] / _R; _W = Lm[3] / _R;
    _P = (Lm[4] - 0.5 * _R * (_U * _U + _V * _V + _W * _W)) * K_1;
    _C = sqrt(K * _P / _R);
    lv[0] = _U; lv[1] = _V; lv[2] = _W;
    _jo = NK_1 * _P;
    _jp = lv[n - 1] + (RU = _P / (_R * _C));
    _jm = lv[n - 1] - RU;
    R_ = Rp[0]; U_ = Rp[1] / R_; V_ = Rp[2] / R_; W_ = Rp[3] / R_;
    P_ = (Rp[4] - 0.5 * R_ * (U_ * U_ + V_ * V_ + W_ * W_)) * K_1;
    C_ = sqrt(K * P_ / R_);
    rv[0] = U_; rv[1] = V_; rv[2] = W_;
    jo_ = NK_1 * P_;
    jp_ = rv[n - 1] + (RU = P_ / (R_ * C_));
    jm_ = rv[n - 1] - RU;
    Un = 0.5 * (lv[n - 1] + rv[n - 1]);
    C = 0.5 * (_C + C_);
    C_p = Un + C; C_m = Un - C; C_o = Un;
    if (C_p > 0.) { al_p = K_1_2 * (_jm - _jp) / _jo; J_p = _jp; }
    else { al_p = K_1_2 * (jm_ - jp_) / jo_; J_p = jp_; }
    if (C_m > 0.) { al_m = K_1_2 * (_jp - _jm) / _jo; J_m = _jm; }
    else { al_m = K_1_2 * (jp_ - jm_) / jo_; J_m = jm_; }
    if (C_o > 0.) { al_o = K05 * (_jp - _jm); al_o = -al_o * al_o; J_o = _jo; }
    else { al_o = K05 * (jp_ - jm_); al_o = -al_o * al_o; J_o = jo_; }
    P = (J_p - J_m) / (al_p - al_m);
    Un = J_p - al_p * P;
    *Rho = (J_o - P) / al_o;
    *Pr = P;
    if (Un > 0) { vel[0] = lv[0]; vel[1] = lv[1]; vel[2] = lv[2]; }
    else { vel[0] = rv[0]; vel[1] = rv[1]; vel[2] = rv[2]; }
    vel[n - 1] = Un;
}

/* velocities by reciprocal (RU = 1./rho; u = rho u * RU), :124-142 */
static void vel_rcp(double **u, size_t c, double *out)
{
    double RU = 1. / u[0][c];
    out[0] = u[1][c] * RU; out[1] = u[2][c] * RU; out[2] = u[3][c] * RU;
}

/* velocities and temperature by division, :117-122 */
static void vel_div(double **u, size_t c, double *out, double *T)
{
    double R_ = u[0][c], U_, V_, W_, P_;
    U_ = u[1][c] / R_; V_ = u[2][c] / R_; W_ = u[3][c] / R_;
    P_ = (u[4][c] - 0.5 * R_ * (U_ * U_ + V_ * V_ + W_ * W_)) * K_1;
    *T = P_ / (R_VOZD * R_);
    out[0] = U_; out[1] = V_; out[2] = W_;
}

/* The dynamic procedure computes mu_SGS unless the static model or none is
 * selected (any other value, the learned closure's included, is the dynamic
 * procedure here: the oracle has no learned closure). */
static int sgs_dynamic(const orc_ctx *o) { return o->p.sgs != ORC_SGS_STATIC && o->p.sgs != ORC_SGS_NONE; }

/* SGS viscosity of one face.  Dynamic: the average of mu_SGS over the plus
 * cell and its x-neighbour (:191, and the reference's x-average on the y and
 * z faces, :360, :531).  Static (the reference's DynamicSmagorinskySGS 0
 * branch, src/fluxes.c:193-205 x, :362-374 y, :533-545 z): the mean density
 * of the two cells beside the face times CsDD times |S| from the face
 * velocity gradients. */
static double face_mu_t(const orc_ctx *o, const double *mu, size_t plus, size_t xnb, double rp, double rm,
                        double du_dx, double dv_dx, double dw_dx, double du_dy, double dv_dy, double dw_dy,
                        double du_dz, double dv_dz, double dw_dz)
{
    double rr, S12, S13, S23, S;
    if (o->p.sgs == ORC_SGS_NONE) return 0.0;
    if (o->p.sgs != ORC_SGS_STATIC) return 0.5 * (mu[plus] + mu[xnb]);
    rr = 0.5 * (rp + rm);
    S12 = 0.5 * (du_dy + dv_dx);
    S13 = 0.5 * (du_dz + dw_dx);
    S23 = 0.5 * (dv_dz + dw_dy);
    S = sqrt(2 * (du_dx * du_dx + dv_dy * dv_dy + dw_dz * dw_dz + 2 * (S12 * S12 + S13 * S13 + S23 * S23)));
    return rr * (o->p.Cs * o->DD) * S;
}

void orc_fluxes_only(orc_ctx *o)
{
    const int L = o->L, H = o->H, D = o->D;
    double **u = o->cur;
    double *mu = o->mu;
    int i, j, k, v;
    /* :57-223, x faces */
    for (i = 0; i < L + 1; i++)
        for (j = 0; j < H; j++)
            for (k = 0; k < D; k++) {
                size_t f = IX(o, i, j, k);
                double Lm[5], Rp[5], Rho, P, vel[3], fw[3], bw[3], T_, _T;
                double Uj[3], jU[3], Uk[3], kU[3], uj[3], ju[3], uk[3], ku[3];
                double du_dx, dv_dx, dw_dx, du_dy, dv_dy, dw_dy, du_dz, dv_dz, dw_dz;
                double uu, vv, ww, mu_T, mu_E, sxx, sxy, sxz, lambda_E, q, RU;
                for (v = 0; v < 5; v++) { Lm[v] = o->fs[0][0][v][f]; Rp[v] = o->fs[0][1][v][f]; }
                riemann(Lm, Rp, 1, &Rho, &P, vel);
                vel_div(u, IC(o, i + 1, j + 1, k + 1), fw, &T_);
                vel_rcp(u, IC(o, i + 1, j + 2, k + 1), Uj);
                vel_rcp(u, IC(o, i + 1, j, k + 1), jU);
                vel_rcp(u, IC(o, i + 1, j + 1, k + 2), Uk);
                vel_rcp(u, IC(o, i + 1, j + 1, k), kU);
                vel_div(u, IC(o, i, j + 1, k + 1), bw, &_T);
                vel_rcp(u, IC(o, i, j + 2, k + 1), uj);
                vel_rcp(u, IC(o, i, j, k + 1), ju);
                vel_rcp(u, IC(o, i, j + 1, k + 2), uk);
                vel_rcp(u, IC(o, i, j + 1, k), ku);
                du_dx = (fw[0] - bw[0]) * o->rdx;
                dv_dx = (fw[1] - bw[1]) * o->rdx;
                dw_dx = (fw[2] - bw[2]) * o->rdx;
                du_dy = (Uj[0] + uj[0] - jU[0] - ju[0]) * o->r4dy;
                dv_dy = (Uj[1] + uj[1] - jU[1] - ju[1]) * o->r4dy;
                dw_dy = (Uj[2] + uj[2] - jU[2] - ju[2]) * o->r4dy;
                du_dz = (Uk[0] + uk[0] - kU[0] - ku[0]) * o->r4dz;
                dv_dz = (Uk[1] + uk[1] - kU[1] - ku[1]) * o->r4dz;
                dw_dz = (Uk[2] + uk[2] - kU[2] - ku[2]) * o->r4dz;
                uu = 0.5 * (fw[0] + bw[0]); vv = 0.5 * (fw[1] + bw[1]); ww = 0.5 * (fw[2] + bw[2]);
                mu_T = face_mu_t(o, mu, IC(o, i + 1, j + 1, k + 1), IC(o, i, j + 1, k + 1), u[0][IC(o, i + 1, j + 1, k + 1)],
                                 u[0][IC(o, i, j + 1, k + 1)], du_dx, dv_dx, dw_dx, du_dy, dv_dy, dw_dy, du_dz, dv_dz,
                                 dw_dz); /* :189-205 */
                mu_E = o->p.mu_L + mu_T;
                sxx = TWO_THIRDS * mu_E * (du_dx + du_dx - dv_dy - dw_dz);
                sxy = mu_E * (du_dy + dv_dx);
                sxz = mu_E * (du_dz + dw_dx);
                lambda_E = o->lambda_L + mu_T * o->cp_Pr_T;
                q = -lambda_E * (T_ - _T) * o->rdx;
                /* :215-220 */
                o->fs[0][0][0][f] = RU = Rho * vel[0];
                o->fs[0][0][1][f] = RU * vel[0] + P - sxx;
                o->fs[0][0][2][f] = RU * vel[1] - sxy;
                o->fs[0][0][3][f] = RU * vel[2] - sxz;
                o->fs[0][0][4][f] = vel[0] * (K_K_1 * P + 0.5 * Rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2])) -
                                    uu * sxx - vv * sxy - ww * sxz + q;
            }
    /* :226-394, y faces */
    for (i = 0; i < L; i++)
        for (j = 0; j < H + 1; j++)
            for (k = 0; k < D; k++) {
                size_t f = IY(o, i, j, k);
                double Lm[5], Rp[5], Rho, P, vel[3], up[3], lw[3], T_, _T;
                double Uk[3], kU[3], Ui[3], iU[3], uk[3], ku[3], ui[3], iu[3];
                double du_dx, dv_dx, dw_dx, du_dy, dv_dy, dw_dy, du_dz, dv_dz, dw_dz;
                double uu, vv, ww, mu_T, mu_E, syx, syy, syz, lambda_E, q, RU;
                for (v = 0; v < 5; v++) { Lm[v] = o->fs[1][0][v][f]; Rp[v] = o->fs[1][1][v][f]; }
                riemann(Lm, Rp, 2, &Rho, &P, vel);
                vel_div(u, IC(o, i + 1, j + 1, k + 1), up, &T_);
                vel_rcp(u, IC(o, i + 1, j + 1, k + 2), Uk);
                vel_rcp(u, IC(o, i + 1, j + 1, k), kU);
                vel_rcp(u, IC(o, i + 2, j + 1, k + 1), Ui);
                vel_rcp(u, IC(o, i, j + 1, k + 1), iU);
                vel_div(u, IC(o, i + 1, j, k + 1), lw, &_T);
                vel_rcp(u, IC(o, i + 1, j, k + 2), uk);
                vel_rcp(u, IC(o, i + 1, j, k), ku);
                vel_rcp(u, IC(o, i + 2, j, k + 1), ui);
                vel_rcp(u, IC(o, i, j, k + 1), iu);
                du_dx = (Ui[0] + ui[0] - iU[0] - iu[0]) * o->r4dx;
                dv_dx = (Ui[1] + ui[1] - iU[1] - iu[1]) * o->r4dx;
                dw_dx = (Ui[2] + ui[2] - iU[2] - iu[2]) * o->r4dx;
                du_dy = (up[0] - lw[0]) * o->rdy;
                dv_dy = (up[1] - lw[1]) * o->rdy;
                dw_dy = (up[2] - lw[2]) * o->rdy;
                du_dz = (Uk[0] + uk[0] - kU[0] - ku[0]) * o->r4dz;
                dv_dz = (Uk[1] + uk[1] - kU[1] - ku[1]) * o->r4dz;
                dw_dz = (Uk[2] + uk[2] - kU[2] - ku[2]) * o->r4dz;
                uu = 0.5 * (up[0] + lw[0]); vv = 0.5 * (up[1] + lw[1]); ww = 0.5 * (up[2] + lw[2]);
                mu_T = face_mu_t(o, mu, IC(o, i + 1, j + 1, k + 1), IC(o, i, j + 1, k + 1), u[0][IC(o, i + 1, j + 1, k + 1)],
                                 u[0][IC(o, i + 1, j, k + 1)], du_dx, dv_dx, dw_dx, du_dy, dv_dy, dw_dy, du_dz, dv_dz,
                                 dw_dz); /* :358-374 */
                mu_E = o->p.mu_L + mu_T;
                syx = mu_E * (dv_dx + du_dy);
                syy = TWO_THIRDS * mu_E * (dv_dy + dv_dy - du_dx - dw_dz);
                syz = mu_E * (dv_dz + dw_dy);
                lambda_E = o->lambda_L + mu_T * o->cp_Pr_T;
                q = -lambda_E * (T_ - _T) * o->rdy;
                /* :386-391 */
                o->fs[1][0][0][f] = RU = Rho * vel[1];
                o->fs[1][0][1][f] = RU * vel[0] - syx;
                o->fs[1][0][2][f] = RU * vel[1] + P - syy;
                o->fs[1][0][3][f] = RU * vel[2] - syz;
                o->fs[1][0][4][f] = vel[1] * (K_K_1 * P + 0.5 * Rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2])) -
                                    uu * syx - vv * syy - ww * syz + q;
            }
    /* :397-571, z faces */
    for (i = 0; i < L; i++)
        for (j = 0; j < H; j++)
            for (k = 0; k < D + 1; k++) {
                size_t f = IZ(o, i, j, k);
                double Lm[5], Rp[5], Rho, P, vel[3], nr[3], fr[3], T_, _T;
                double Ui[3], iU[3], Uj[3], jU[3], ui[3], iu[3], uj[3], ju[3];
                double du_dx, dv_dx, dw_dx, du_dy, dv_dy, dw_dy, du_dz, dv_dz, dw_dz;
                double uu, vv, ww, mu_T, mu_E, szx, szy, szz, lambda_E, q, RU;
                for (v = 0; v < 5; v++) { Lm[v] = o->fs[2][0][v][f]; Rp[v] = o->fs[2][1][v][f]; }
                riemann(Lm, Rp, 3, &Rho, &P, vel);
                vel_div(u, IC(o, i + 1, j + 1, k + 1), nr, &T_);
                vel_rcp(u, IC(o, i + 2, j + 1, k + 1), Ui);
                vel_rcp(u, IC(o, i, j + 1, k + 1), iU);
                vel_rcp(u, IC(o, i + 1, j + 2, k + 1), Uj);
                vel_rcp(u, IC(o, i + 1, j, k + 1), jU);
                vel_div(u, IC(o, i + 1, j + 1, k), fr, &_T);
                vel_rcp(u, IC(o, i + 2, j + 1, k), ui);
                vel_rcp(u, IC(o, i, j + 1, k), iu);
                vel_rcp(u, IC(o, i + 1, j + 2, k), uj);
                vel_rcp(u, IC(o, i + 1, j, k), ju);
                du_dx = (Ui[0] + ui[0] - iU[0] - iu[0]) * o->r4dx;
                dv_dx = (Ui[1] + ui[1] - iU[1] - iu[1]) * o->r4dx;
                dw_dx = (Ui[2] + ui[2] - iU[2] - iu[2]) * o->r4dx;
                du_dy = (Uj[0] + uj[0] - jU[0] - ju[0]) * o->r4dy;
                dv_dy = (Uj[1] + uj[1] - jU[1] - ju[1]) * o->r4dy;
                dw_dy = (Uj[2] + uj[2] - jU[2] - ju[2]) * o->r4dy;
                du_dz = (nr[0] - fr[0]) * o->rdz;
                dv_dz = (nr[1] - fr[1]) * o->rdz;
                dw_dz = (nr[2] - fr[2]) * o->rdz;
                uu = 0.5 * (nr[0] + fr[0]); vv = 0.5 * (nr[1] + fr[1]); ww = 0.5 * (nr[2] + fr[2]);
                mu_T = face_mu_t(o, mu, IC(o, i + 1, j + 1, k + 1), IC(o, i, j + 1, k + 1), u[0][IC(o, i + 1, j + 1, k + 1)],
                                 u[0][IC(o, i + 1, j + 1, k)], du_dx, dv_dx, dw_dx, du_dy, dv_dy, dw_dy, du_dz, dv_dz,
                                 dw_dz); /* :529-545 */
                mu_E = o->p.mu_L + mu_T;
                szx = mu_E * (dw_dx + du_dz);
                szy = mu_E * (dw_dy + dv_dz);
                szz = TWO_THIRDS * mu_E * (dw_dz + dw_dz - du_dx - dv_dy);
                lambda_E = o->lambda_L + mu_T * o->cp_Pr_T;
                q = -lambda_E * (T_ - _T) * o->rdz;
                /* :563-568 */
                o->fs[2][0][0][f] = RU = Rho * vel[2];
                o->fs[2][0][1][f] = RU * vel[0] - szx;
                o->fs[2][0][2][f] = RU * vel[1] - szy;
                o->fs[2][0][3][f] = RU * vel[2] + P - szz;
                o->fs[2][0][4][f] = vel[2] * (K_K_1 * P + 0.5 * Rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2])) -
                                    uu * szx - vv * szy - ww * szz + q;
            }
}

void orc_fluxes(orc_ctx *o)
{
    if (sgs_dynamic(o)) orc_dynamic_smagorinsky(o); /* src/fluxes.c:52-54 */
    orc_fluxes_only(o);
}

/* ------------------------------------------------------------------------
 * A7: TVD Runge-Kutta, src/evolution.c:15-245.
 * ------------------------------------------------------------------------ */
static double divx(const orc_ctx *o, const double *F, int i, int j, int k)
{
    return o->dtx * (F[IX(o, i - 1, j - 1, k - 1)] - F[IX(o, i, j - 1, k - 1)]);
}
static double divy(const orc_ctx *o, const double *F, int i, int j, int k)
{
    return o->dty * (F[IY(o, i - 1, j - 1, k - 1)] - F[IY(o, i - 1, j, k - 1)]);
}
static double divz(const orc_ctx *o, const double *F, int i, int j, int k)
{
    return o->dtz * (F[IZ(o, i - 1, j - 1, k - 1)] - F[IZ(o, i - 1, j - 1, k)]);
}

static void rk3(orc_ctx *o, int stage)
{
    const double one_third = 1. / 3., two_thirds = 2. / 3.;
    int i, j, k, v;
    for (v = 0; v < 5; v++) {
        double *U = o->U[v], *Up = o->Up[v];
        const double *Fx = o->fs[0][0][v], *Fy = o->fs[1][0][v], *Fz = o->fs[2][0][v];
        for (i = 1; i < o->L + 1; i++)
            for (j = 1; j < o->H + 1; j++)
                for (k = 1; k < o->D + 1; k++) {
                    size_t c = IC(o, i, j, k);
                    if (stage == 1) /* :44-63 */
                        Up[c] = U[c] + divx(o, Fx, i, j, k) + divy(o, Fy, i, j, k) + divz(o, Fz, i, j, k);
                    else if (stage == 2) /* :81-105 */
                        Up[c] = 0.75 * U[c] + 0.25 * (Up[c] + divx(o, Fx, i, j, k) + divy(o, Fy, i, j, k) +
                                                      divz(o, Fz, i, j, k));
                    else /* :123-147 */
                        U[c] = one_third * U[c] + two_thirds * (Up[c] + divx(o, Fx, i, j, k) +
                                                                divy(o, Fy, i, j, k) + divz(o, Fz, i, j, k));
                }
    }
    o->cur = (stage == 1 || stage == 2) ? o->Up : o->U;
}

static void rk2(orc_ctx *o, int stage)
{
    int i, j, k, v;
    for (v = 0; v < 5; v++) {
        double *U = o->U[v], *Up = o->Up[v];
        const double *Fx = o->fs[0][0][v], *Fy = o->fs[1][0][v], *Fz = o->fs[2][0][v];
        for (i = 1; i < o->L + 1; i++)
            for (j = 1; j < o->H + 1; j++)
                for (k = 1; k < o->D + 1; k++) {
                    size_t c = IC(o, i, j, k);
                    if (stage == 1) /* :172-195 */
                        Up[c] = U[c] + divx(o, Fx, i, j, k) + divy(o, Fy, i, j, k) + divz(o, Fz, i, j, k);
                    else /* :208-231 */
                        U[c] = 0.5 * (U[c] + Up[c] + divx(o, Fx, i, j, k) + divy(o, Fy, i, j, k) +
                                      divz(o, Fz, i, j, k));
                }
    }
    o->cur = (stage == 1) ? o->Up : o->U;
}

/* src/evolution.c:15-27: nStages == 2 falls through into the RK3 update */
void orc_evolution(orc_ctx *o, int nstages, int stage)
{
    if (nstages == 2) rk2(o, stage);
    rk3(o, stage);
}

/* ------------------------------------------------------------------------
 * A8: CFL, src/helpers.c:23-52 (streamwise u only, signed); acoustic mode is
 * a project extension: max over cells of dt*((|u|+c)/dx+(|v|+c)/dy+(|w|+c)/dz).
 * ------------------------------------------------------------------------ */
double orc_check_courant(orc_ctx *o)
{
    double maxCo = 0.0, CoNum;
    int i, j, k;
    for (k = 1; k < o->D + 1; k++)
        for (j = 1; j < o->H + 1; j++)
            for (i = 1; i < o->L + 1; i++) {
                size_t c = IC(o, i, j, k);
                double R = o->U[0][c];
                if (o->p.cfl_mode == ORC_CFL_ACOUSTIC) {
                    /* the extension's own form: the reciprocal of rho once */
                    double ir = 1.0 / R;
                    double U = o->U[1][c] * ir, V = o->U[2][c] * ir, W = o->U[3][c] * ir;
                    double P = (o->U[4][c] - 0.5 * R * (U * U + V * V + W * W)) * K_1;
                    double Cs = sqrt(K * P * ir);
                    CoNum = (fabs(U) + Cs) * o->dtx + (fabs(V) + Cs) * o->dty + (fabs(W) + Cs) * o->dtz;
                } else {
                    CoNum = o->U[1][c] / R * o->dtx;
                }
                maxCo = (CoNum > maxCo) ? CoNum : maxCo;
            }
    o->dt *= (o->p.maxCoNum / maxCo);
    o->dtx = o->dt / o->p.deltaX; o->dty = o->dt / o->p.deltaY; o->dtz = o->dt / o->p.deltaZ;
    o->last_maxco = maxCo;
    return maxCo;
}

/* ------------------------------------------------------------------------
 * A9: disturbance RNG, src/helpers.c:13-17 and src/layer2.c:152-162.
 * ------------------------------------------------------------------------ */
double orc_random(double x)
{
    x = 11. * x + 3.14159265358979323846;
    return x - (double)((int)x);
}

void orc_disturb(orc_ctx *o)
{
    const unsigned DEP = (unsigned)o->D;
    double X = o->X;
    if (o->counter > 0) o->counter--;
    else {
        o->counter = (int)(o->p.Ns_min + o->p.Nst * (X = orc_random(X)));
        o->k_min = (unsigned)(DEP * (X = orc_random(X)));
        o->k_max = (unsigned)(o->k_min + DEP * (X = orc_random(X)));
        if (o->k_max > DEP) o->k_max -= DEP;
        X = orc_random(X); o->Ud = o->p.Ua * (1 - X - X);
        X = orc_random(X); o->Vd = o->p.Va * (1 - X - X);
        X = orc_random(X); o->Wd = o->p.Wa * (1 - X - X);
    }
    o->X = X;
}

/* Driver loop body, src/layer2.c:141-185.  The SGS viscosity depends only on
 * U^n (src/fluxes.c:53), which no stage changes before the last evolution, so
 * computing it once at stage 1 gives the reference's values in every stage. */
static void step_impl(orc_ctx *o, int nsteps, int every_stage)
{
    int s;
    while (nsteps-- > 0) {
        orc_check_courant(o);
        ++o->step;
        orc_disturb(o);
        for (s = 1; s <= o->p.nStages; s++) {
            orc_ghost_bc(o);
            orc_reconstruct(o);
            orc_interface_bc(o);
            if ((s == 1 || every_stage) && sgs_dynamic(o)) orc_dynamic_smagorinsky(o);
            orc_fluxes_only(o);
            orc_evolution(o, o->p.nStages, s);
        }
    }
}

void orc_step(orc_ctx *o, int nsteps) { step_impl(o, nsteps, 0); }
void orc_step_ref_sgs(orc_ctx *o, int nsteps) { step_impl(o, nsteps, 1); }

/* ------------------------------------------------------------------------
 * Temporal shear layer (project extension; no reference counterpart).
 * u(y) = dU/2 tanh(2 y / delta_w0), y measured from the domain centre,
 * uniform pressure p0 = 1e5 Pa, free-stream density 1 kg/m^3 on both sides,
 * Crocco-Busemann temperature T = T_inf + (dU^2/4 - u^2) / (2 cp), dU from
 * the convective Mach number with equal free-stream sound speeds,
 * dU = 2 Mc c_inf.  Velocity perturbations: independent uniform draws in
 * [-amp dU, amp dU) for u, v, w of every cell, from splitmix64(seed), in
 * i, j, k order, three draws per cell.
 * ------------------------------------------------------------------------ */
static uint64_t splitmix64(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static double unif_pm1(uint64_t *s)
{
    return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

int orc_temporal_state(const orc_params *p, double Mc, double delta_w0, double amp,
                       unsigned long long seed, double *state, double *dU_out)
{
    const double p0 = 100000., rho0 = 1.0, cp = CV * K;
    const double Tinf = p0 / (R_VOZD * rho0);
    const double cinf = sqrt(K * p0 / rho0);
    const double dU = 2.0 * Mc * cinf;
    const double Ly = p->HIG * p->deltaY;
    uint64_t s = seed;
    size_t n = 0;
    int i, j, k;
    double *row = malloc(sizeof(double) * 5 * p->DEP);
    if (!row) return -1;
    for (i = 1; i <= p->LEN; i++)
        for (j = 1; j <= p->HIG; j++) {
            double y = (j - 0.5) * p->deltaY - 0.5 * Ly;
            double um = 0.5 * dU * tanh(2.0 * y / delta_w0);
            double T = Tinf + (0.25 * dU * dU - um * um) / (2.0 * cp);
            double rho = p0 / (R_VOZD * T);
            for (k = 0; k < p->DEP; k++) {
                double du = amp * dU * unif_pm1(&s);
                double dv = amp * dU * unif_pm1(&s);
                double dw = amp * dU * unif_pm1(&s);
                double uu = um + du;
                row[k] = rho;
                row[p->DEP + k] = rho * uu;
                row[2 * p->DEP + k] = rho * dv;
                row[3 * p->DEP + k] = rho * dw;
                row[4 * p->DEP + k] = p0 / K_1 + 0.5 * rho * (uu * uu + dv * dv + dw * dw);
            }
            memcpy(state + n, row, sizeof(double) * 5 * p->DEP);
            n += 5 * (size_t)p->DEP;
        }
    free(row);
    if (dU_out) *dU_out = dU;
    return 0;
}

/* Volume integrals of the conserved variables over the interior of U^n. */
void orc_sums(orc_ctx *o, double *sums)
{
    const double vol = o->p.deltaX * o->p.deltaY * o->p.deltaZ;
    int i, j, k, v;
    for (v = 0; v < 5; v++) {
        long double acc = 0;
        for (i = 1; i <= o->L; i++)
            for (j = 1; j <= o->H; j++)
                for (k = 1; k <= o->D; k++) acc += o->U[v][IC(o, i, j, k)];
        sums[v] = (double)acc * vol;
    }
}

/* Per y-row plane sums used for Favre averages (momentum thickness, Reynolds
 * stresses): rho, rho u, rho v, rho w, rho u u, rho v v, rho w w, rho u v. */
void orc_plane_sums(orc_ctx *o, double *rows)
{
    int i, j, k, q;
    for (j = 1; j <= o->H; j++) {
        long double acc[8] = {0};
        for (i = 1; i <= o->L; i++)
            for (k = 1; k <= o->D; k++) {
                size_t c = IC(o, i, j, k);
                double r = o->U[0][c], u = o->U[1][c] / r, v = o->U[2][c] / r, w = o->U[3][c] / r;
                acc[0] += r; acc[1] += r * u; acc[2] += r * v; acc[3] += r * w;
                acc[4] += r * u * u; acc[5] += r * v * v; acc[6] += r * w * w; acc[7] += r * u * v;
            }
        for (q = 0; q < 8; q++) rows[8 * (j - 1) + q] = (double)acc[q];
    }
}

/* The per-cell values Output() writes to <step>.plt (src/output.c:66-139), in
 * its loop order (k, then j, then i fastest), 12 per cell: the cell centre,
 * rho, u, v, w, p, T, vorticity magnitude, Q criterion and the static
 * Smagorinsky viscosity ratio rho Cs DD |S| / mu_L.  It reads U^n with the
 * ghost layer the last stage left, as Output() does. */
void orc_output_fields(orc_ctx *o, double *out)
{
    const double *U1 = o->U[0], *U2 = o->U[1], *U3 = o->U[2], *U4 = o->U[3], *U5 = o->U[4];
    const double dX = o->p.deltaX, dY = o->p.deltaY, dZ = o->p.deltaZ;
    const double CsDD = o->p.Cs * o->DD, mu_L = o->p.mu_L;
    size_t n = 0;
    int i, j, k;
    for (k = 1; k <= o->D; k++)
        for (j = 1; j <= o->H; j++)
            for (i = 1; i <= o->L; i++) {
                const size_t c = IC(o, i, j, k), xi = o->pi, yj = o->pj;
                double R, Uu, V, W, P, T, du_dx, du_dy, du_dz, dv_dx, dv_dy, dv_dz, dw_dx, dw_dy, dw_dz;
                double ox, oy, oz, Om, S12, S13, S23, St, *q = out + 12 * n++;
                q[0] = (i - 1) * dX + 0.5 * dX;
                q[1] = (j - 1) * dY + 0.5 * dY;
                q[2] = (k - 1) * dZ + 0.5 * dZ;
                R = U1[c];
                Uu = U2[c] / R;
                V = U3[c] / R;
                W = U4[c] / R;
                P = (U5[c] - 0.5 * R * (Uu * Uu + V * V + W * W)) * 0.4;
                T = P / (287.10 * R);
                du_dx = (U2[c + xi] / U1[c + xi] - U2[c - xi] / U1[c - xi]) * o->r2dx;
                du_dy = (U2[c + yj] / U1[c + yj] - U2[c - yj] / U1[c - yj]) * o->r2dy;
                du_dz = (U2[c + 1] / U1[c + 1] - U2[c - 1] / U1[c - 1]) * o->r2dz;
                dv_dx = (U3[c + xi] / U1[c + xi] - U3[c - xi] / U1[c - xi]) * o->r2dx;
                dv_dy = (U3[c + yj] / U1[c + yj] - U3[c - yj] / U1[c - yj]) * o->r2dy;
                dv_dz = (U3[c + 1] / U1[c + 1] - U3[c - 1] / U1[c - 1]) * o->r2dz;
                dw_dx = (U4[c + xi] / U1[c + xi] - U4[c - xi] / U1[c - xi]) * o->r2dx;
                dw_dy = (U4[c + yj] / U1[c + yj] - U4[c - yj] / U1[c - yj]) * o->r2dy;
                dw_dz = (U4[c + 1] / U1[c + 1] - U4[c - 1] / U1[c - 1]) * o->r2dz;
                ox = dw_dy - dv_dz;
                oy = du_dz - dw_dx;
                oz = dv_dx - du_dy;
                Om = sqrt(ox * ox + oy * oy + oz * oz);
                S12 = 0.5 * (du_dy + dv_dx);
                S13 = 0.5 * (du_dz + dw_dx);
                S23 = 0.5 * (dv_dz + dw_dy);
                St = sqrt(2 * (du_dx * du_dx + dv_dy * dv_dy + dw_dz * dw_dz + 2 * (S12 * S12 + S13 * S13 + S23 * S23)));
                q[3] = R; q[4] = Uu; q[5] = V; q[6] = W; q[7] = P; q[8] = T;
                q[9] = Om;
                q[10] = 0.5 * (Om * Om - St * St);
                q[11] = R * CsDD * St / mu_L;
            }
}
