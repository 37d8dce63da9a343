/*
 * CPU oracle -- plain-C restatement of the reference solver's time-marching
 * path (azhang22/3D_MPI_TEST) for a single MPI rank.
 *
 * TEST INFRASTRUCTURE ONLY. Tests, smoke() and bench.py's cpu_baseline use it
 * as the checker; the product (the B200 library) never links or calls it.
 *
 * Every function names the reference lines it restates. Floating-point
 * expressions keep the reference's association order so that, compiled
 * without FMA contraction, the restatement reproduces the compiled
 * reference bit for bit; that is checked in tests/test_oracle_pin.py
 * against oracle/_ref/ref_harness.
 *
 * Arrays are flat, [i][j][k] with k fastest (the reference's double***
 * layout, calculation_2D.cpp:107-123).
 */
#include "fdtd_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* boundary_type, mygeneral.h:49 */
enum { BT_RIGID = 0, BT_ABSORBING, BT_POROUS, BT_RADIATION, BT_TDBC };
/* scheme_list, mygeneral.h:48 */
enum { S_FB_P_V = 0, S_FB_V_P, S_FB_VP, S_LEAPTRAP, S_ABM, S_RK4, S_RK2 };

typedef struct { int Judge, JMAX, lead_DJ, trail_DJ; double ratio; } mframe;

/* ---------------------------------------------------------------- grid */
/* calculation_2D members, calculation_2D.h:24-74 (single rank: mpi_*MAX == whole) */
typedef struct {
    int I, J, K;
    int IMAX, IMAX1, IMAX2, JMAX, JMAX1, JMAX2, JMAX3, KMAX, KMAX1, KMAX2, IJKMAX;
    double dt, rdx, rdy, rdz, dx1, dy1, dz1, gcoef;
    double *X, *Y, *Z, *axX, *axY, *axZ, *Xx, *Yy, *Zz, *Jac;
    /* terrain-following grid (extension; NULL on flat ground): ground
     * elevation zg[j], physical height Zt[j][k] of every node, and the
     * metric derivatives Z_over_z = Zz2[j][k], Z_over_y = Zy2[j][k] that
     * replace the reference's 1D Zz[k] and fixed-zero Z_over_y */
    double *zg, *Zt, *Zz2, *Zy2;
    double *un, *vn, *wn, *pn, *unn, *vnn, *wnn, *pnn;
    double *psi; /* [i][k][6], calculation_2D.cpp:125-135 */
    mframe mf;
    /* porous medium constants, porous.cpp:40-51 */
    double eff, Beta, Gama, invBeta;
} grid;

/* TDBC poles, calculation_2D.h:73-75 */
static const double TD_A[6] = {8.226223820e-01, 3.732304064e-01, 9.106232372e-02,
                               4.819445335e-02, 4.225250937e-01, 1.837970986e-01};
static const double TD_R[6] = {8.681310138e-01, 1.953722814e-01, 1.108067950e-02,
                               2.566498621e-03, 1.457297589e-04, 4.648583789e-02};

typedef struct { int n0, n1, n2; double *q[4]; } slab; /* q: u v w p */

/* air members, air.h:27-71 */
typedef struct {
    grid g;
    double *Uav, *Vav, *Wav;
    int vmethod;
    double vb, vc, valpha; /* SpeedProfile, air.cpp:40-43 */
    double vkappa, vz0;    /* log law (extension, method 7): V = (vb / vkappa) ln(z / vz0) */
    int upwind;            /* extension: backward-difference velocity advection (advection.dat) */
    double gamma, P0, Aav, c0;
    int jx, jy, jz;
    double sxmax, ax, symax, ay, szmax, az;
    double x1, x2, w1, w2, y1, y2, l1, l2, z1, z2, h1, h2;
    int pml_count, pml_time;
    slab s[6]; /* x1 x2 y1 y2 z1 z2 */
    int cr_judge, istar, istop, jstar, jstop, kstar, kstop;
    int *cr_uc;
    double eff1, gama1, invb1, eff2, gama2, invb2;
} airm;

struct orc {
    /* parsed input.txt (airpore.cpp:17-316) */
    double gauss_width;
    mframe mf;
    int scheme;
    int bc_n, bc_s, bc_e, bc_w, bc_f, bc_b;
    int case_no;
    int time_domain;
    double vcoef;
    int vmethod;
    double gamma, P0, c0, Aav;
    double pxa, pxs, pya, pys, pza, pzs;
    int pyt, jx, jy, jz;
    double pq, pporo, psig, peff, pKp, Zinf, tau;
    double src[3], rcv[3];
    double dt, dx, dy, dz, pdx, pdy, pdz;
    int cjudge, cpoints;
    double cc[12];
    double hq[3], hpor[3], hsig[3], heff[3], hKp[3];
    double box[6];
    /* media */
    airm air;
    grid pore;
    int has_pore;
    /* receivers */
    int nrec;
    int *ri, *rj, *rk;
    /* extension: impedance ground, a 6-pole TDBC on the rigid south face
     * (case_dir/tdbc_ground.dat: Zinf tau a0..a5 r0..r5) */
    int gtdbc;
    double gZ, gtau, ga[6], gr[6];
    double *gpsi; /* [i][j][6] */
};

#define IX(g, i, j, k) ((((size_t)(i)) * (size_t)(g)->J + (size_t)(j)) * (size_t)(g)->K + (size_t)(k))
#define SX(s, a, b, c) ((((size_t)(a)) * (size_t)(s)->n1 + (size_t)(b)) * (size_t)(s)->n2 + (size_t)(c))

static double *zalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

static void seterr(char *err, int errlen, const char *fmt, ...)
{
    if (!err || errlen <= 0) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, (size_t)errlen, fmt, ap);
    va_end(ap);
}

/* ------------------------------------------------ stream-like text reader */
typedef struct { const char *s; size_t n, pos; int fail; } rdr;

static void rd_ws(rdr *r)
{
    while (r->pos < r->n && isspace((unsigned char)r->s[r->pos])) r->pos++;
}
static double rd_d(rdr *r)
{
    rd_ws(r);
    char *end;
    double v = strtod(r->s + r->pos, &end);
    if (end == r->s + r->pos) { r->fail = 1; return 0.0; }
    r->pos = (size_t)(end - r->s);
    return v;
}
static int rd_i(rdr *r)
{
    rd_ws(r);
    char *end;
    long v = strtol(r->s + r->pos, &end, 10);
    if (end == r->s + r->pos) { r->fail = 1; return 0; }
    r->pos = (size_t)(end - r->s);
    return (int)v;
}
static void rd_word(rdr *r)
{
    rd_ws(r);
    while (r->pos < r->n && !isspace((unsigned char)r->s[r->pos])) r->pos++;
}
/* istream::ignore(100, '\n') */
static void rd_ignore(rdr *r)
{
    for (int c = 0; c < 100 && r->pos < r->n; ++c) {
        if (r->s[r->pos++] == '\n') break;
    }
}

static char *slurp(const char *path, size_t *n)
{
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long len = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *b = (char *)malloc((size_t)len + 1);
    if (fread(b, 1, (size_t)len, f) != (size_t)len) { free(b); fclose(f); return NULL; }
    b[len] = 0;
    fclose(f);
    *n = (size_t)len;
    return b;
}

/* ------------------------------------------- airpore::airpore (parse) */
static int parse_input(orc *o, const char *dir, char *err, int errlen)
{
    char path[4096];
    snprintf(path, sizeof path, "%s/input.txt", dir);
    size_t n;
    char *txt = slurp(path, &n);
    if (!txt) { seterr(err, errlen, "cannot open %s", path); return -1; }
    rdr R = {txt, n, 0, 0}, *r = &R;
    int num_pml[3] = {0, 0, 0};
    o->gauss_width = rd_d(r); rd_ignore(r);
    o->mf.JMAX = rd_i(r); o->mf.lead_DJ = rd_i(r); o->mf.trail_DJ = rd_i(r);
    o->mf.Judge = rd_i(r); o->mf.ratio = rd_d(r); rd_ignore(r);
    int st = rd_i(r); rd_ignore(r);
    switch (st) { /* airpore.cpp:25-43 */
    case 1: o->scheme = S_FB_V_P; break;
    case 2: o->scheme = S_FB_P_V; break;
    case 3: o->scheme = S_FB_VP; break;
    case 4: o->scheme = S_LEAPTRAP; break;
    case 5: o->scheme = S_RK4; break;
    case 6: o->scheme = S_RK2; break;
    case 7: o->scheme = S_ABM; break;
    default: o->scheme = S_FB_P_V;
    }
    int bch[6];
    for (int i = 0; i < 6; ++i) bch[i] = rd_i(r);
    rd_ignore(r); rd_ignore(r);
    o->bc_n = o->bc_s = o->bc_e = o->bc_w = o->bc_f = o->bc_b = BT_RIGID;
    int *slot_direct[6] = {&o->bc_n, &o->bc_s, &o->bc_e, &o->bc_w, &o->bc_f, &o->bc_b};
    /* radiation codes swap E/W and F/B (airpore.cpp:126-144) */
    int *slot_rad[6] = {&o->bc_n, &o->bc_s, &o->bc_w, &o->bc_e, &o->bc_b, &o->bc_f};
    for (int i = 0; i < 6; ++i) { /* airpore.cpp:52-159 */
        switch (bch[i]) {
        case 1: *slot_direct[i] = BT_RIGID; break;
        case 2:
            *slot_direct[i] = BT_ABSORBING;
            num_pml[i / 2] += (i % 2 == 0) ? 1 : 10;
            break;
        case 3: *slot_direct[i] = BT_POROUS; break;
        case 4: *slot_rad[i] = BT_RADIATION; break;
        case 5: if (i == 2) o->bc_e = BT_TDBC; break;
        default: break;
        }
    }
    switch (o->bc_n) { /* airpore.cpp:160-169 */
    case BT_ABSORBING: case BT_RIGID: o->case_no = 1; break;
    case BT_POROUS: o->case_no = 2; break;
    case BT_RADIATION: o->case_no = 3; break;
    default: o->case_no = 0;
    }
    o->time_domain = rd_i(r); rd_i(r); rd_i(r); rd_d(r); rd_ignore(r);
    o->vcoef = rd_d(r); o->vmethod = rd_i(r); rd_ignore(r);
    o->gamma = rd_d(r); o->P0 = rd_d(r); o->c0 = rd_d(r); rd_ignore(r);
    o->Aav = pow(o->c0, 2) / o->gamma / o->P0;
    o->pxa = rd_d(r); o->pxs = rd_d(r); rd_ignore(r);
    o->pya = rd_d(r); o->pys = rd_d(r); o->pyt = rd_i(r); rd_ignore(r);
    o->pza = rd_d(r); o->pzs = rd_d(r); rd_ignore(r);
    int *judges[3] = {&o->jz, &o->jy, &o->jx};
    for (int i = 0; i < 3; ++i) { /* airpore.cpp:182-247 */
        switch (num_pml[i]) {
        case 0: *judges[i] = 0; break;
        case 1: *judges[i] = 2; break;
        case 10: *judges[i] = 1; break;
        case 11: *judges[i] = 3; break;
        default: *judges[i] = 0;
        }
    }
    /* porous parameters, airpore.cpp:249-254 */
    o->pq = rd_d(r); o->pporo = rd_d(r); o->psig = rd_d(r); rd_ignore(r);
    o->peff = o->pq * o->pq / o->pporo / o->Aav;
    o->pKp = 1.0 / o->gamma / o->P0;
    double rho = o->gamma * o->P0 / 340.29 / 340.29;
    o->Zinf = rho * 340.29 * o->pq / o->pporo;
    o->tau = o->gamma * rho * o->pq * o->pq / o->psig / o->pporo;
    for (int i = 0; i < 3; ++i) o->src[i] = rd_d(r);
    for (int i = 0; i < 3; ++i) o->rcv[i] = rd_d(r);
    rd_ignore(r);
    o->dt = rd_d(r); rd_ignore(r);
    o->dx = rd_d(r); o->dy = rd_d(r); o->dz = rd_d(r); rd_ignore(r);
    rd_i(r); rd_i(r); rd_i(r); rd_ignore(r);
    rd_ignore(r); rd_ignore(r);
    rd_i(r); rd_i(r); rd_word(r);
    rd_ignore(r); rd_ignore(r);
    o->cjudge = rd_i(r);
    for (int i = 0; i < 12; ++i) o->cc[i] = rd_d(r);
    o->cpoints = rd_i(r); rd_ignore(r);
    for (int h = 0; h < 3; ++h) { /* hill, canopy, trunk: airpore.cpp:285-295 */
        o->hq[h] = rd_d(r); o->hpor[h] = rd_d(r); o->hsig[h] = rd_d(r); rd_ignore(r);
        o->heff[h] = o->hq[h] * o->hq[h] / o->hpor[h] / o->Aav;
        o->hKp[h] = 1.0 / o->gamma / o->P0;
    }
    for (int i = 0; i < 6; ++i) o->box[i] = rd_d(r);
    rd_ignore(r);
    rd_ignore(r); rd_ignore(r);
    if (o->bc_s == BT_POROUS) {
        o->pdx = rd_d(r); o->pdy = rd_d(r); o->pdz = rd_d(r); rd_ignore(r);
    }
    int fail = r->fail;
    free(txt);
    if (fail) { seterr(err, errlen, "malformed %s", path); return -1; }
    return 0;
}

/* ------------------------------------ calculation_2D::calculation_2D */
static int grid_init(grid *g, const char *dir, const char *prefix, double dt, double dx, double dy,
                     double dz, mframe mf, double gauss_width, int judge_porous, char *err, int errlen)
{
    char path[4096];
    size_t n;
    g->dt = dt;
    g->rdx = 1.0 / dx; g->rdy = 1.0 / dy; g->rdz = 1.0 / dz;
    g->dx1 = dx; g->dy1 = dy; g->dz1 = dz;
    g->gcoef = 4.0 * log(2.0) / pow(gauss_width, 2); /* calculation_2D.cpp:26 */
    g->mf = mf;
    snprintf(path, sizeof path, "%s/%s1.dat", dir, prefix);
    char *t1 = slurp(path, &n);
    if (!t1) { seterr(err, errlen, "cannot open %s", path); return -1; }
    rdr R1 = {t1, n, 0, 0};
    g->IMAX = rd_i(&R1); g->IMAX1 = rd_i(&R1); g->IMAX2 = rd_i(&R1);
    g->JMAX = rd_i(&R1); g->JMAX1 = rd_i(&R1); g->JMAX2 = rd_i(&R1);
    g->KMAX = rd_i(&R1); g->KMAX1 = rd_i(&R1); g->KMAX2 = rd_i(&R1);
    g->IJKMAX = rd_i(&R1);
    g->JMAX3 = g->JMAX1;
    if (g->mf.Judge == 1) { /* calculation_2D.cpp:58-68 */
        if ((g->IJKMAX - g->mf.JMAX) % (g->mf.lead_DJ - 1) != 0) {
            int N_limit = (g->IJKMAX - g->mf.JMAX) / (g->mf.lead_DJ - 1);
            g->IJKMAX = g->mf.JMAX + (N_limit + 1) * (g->mf.lead_DJ - 1);
        }
        g->JMAX = g->mf.JMAX;
    } else {
        g->mf.JMAX = g->JMAX;
        g->IJKMAX = g->JMAX;
    }
    (void)judge_porous; /* one rank: every grid spans 0..KMAX-1 */
    g->I = g->IMAX; g->J = g->JMAX; g->K = g->KMAX;
    if (g->I < 3 || g->J < 5 || g->K < 3) { free(t1); seterr(err, errlen, "grid too small"); return -1; }
    size_t N = (size_t)g->I * g->J * g->K;
    g->X = zalloc(g->I); g->Y = zalloc(g->J); g->Z = zalloc(g->K);
    g->axX = zalloc(g->IMAX); g->axY = zalloc(g->JMAX); g->axZ = zalloc(g->KMAX);
    g->Xx = zalloc(g->I); g->Yy = zalloc(g->J); g->Zz = zalloc(g->K);
    g->Jac = zalloc(N);
    g->un = zalloc(N); g->vn = zalloc(N); g->wn = zalloc(N); g->pn = zalloc(N);
    g->unn = zalloc(N); g->vnn = zalloc(N); g->wnn = zalloc(N); g->pnn = zalloc(N);
    g->psi = zalloc((size_t)g->I * g->K * 6);
    for (int i = 0; i < g->IMAX; ++i) { double v = rd_d(&R1); g->X[i] = v; g->axX[i] = v; }
    int fail = R1.fail;
    free(t1);
    snprintf(path, sizeof path, "%s/%s2.dat", dir, prefix);
    char *t2 = slurp(path, &n);
    if (!t2) { seterr(err, errlen, "cannot open %s", path); return -1; }
    rdr R2 = {t2, n, 0, 0};
    for (int j = 0; j < g->JMAX; ++j) { double v = rd_d(&R2); g->Y[j] = v; g->axY[j] = v; }
    fail |= R2.fail;
    free(t2);
    snprintf(path, sizeof path, "%s/%s3.dat", dir, prefix);
    char *t3 = slurp(path, &n);
    if (!t3) { seterr(err, errlen, "cannot open %s", path); return -1; }
    rdr R3 = {t3, n, 0, 0};
    for (int k = 0; k < g->KMAX; ++k) { double v = rd_d(&R3); g->Z[k] = v; g->axZ[k] = v; }
    fail |= R3.fail;
    free(t3);
    if (fail) { seterr(err, errlen, "malformed %s axis files", prefix); return -1; }
    return 0;
}

static void grid_free(grid *g)
{
    double **ps[] = {&g->X, &g->Y, &g->Z, &g->axX, &g->axY, &g->axZ, &g->Xx, &g->Yy, &g->Zz, &g->Jac,
                     &g->un, &g->vn, &g->wn, &g->pn, &g->unn, &g->vnn, &g->wnn, &g->pnn, &g->psi,
                     &g->zg, &g->Zt, &g->Zz2, &g->Zy2};
    for (size_t i = 0; i < sizeof ps / sizeof ps[0]; ++i) { free(*ps[i]); *ps[i] = NULL; }
}

/* calculation_2D::Set_InitialCond + cal_InitialPressure, calculation_2D.cpp:292-314 */
static void grid_set_initial(grid *g, const double *src, int judge)
{
    for (int i = 0; i < g->I; i++)
        for (int j = 0; j < g->J; j++)
            for (int k = 0; k < g->K; k++) {
                size_t c = IX(g, i, j, k);
                g->un[c] = 0; g->vn[c] = 0; g->wn[c] = 0;
                if (judge == 1) {
                    double zk = g->Zt ? g->Zt[(size_t)j * g->K + k] : g->Z[k];
                    double x = g->X[i] - src[0], y = g->Y[j] - src[1], z = zk - src[2];
                    double rr = sqrt(pow(x, 2) + pow(y, 2) + pow(z, 2));
                    g->pn[c] = 1.0 * exp(-g->gcoef * rr * rr);
                } else {
                    g->pn[c] = 0;
                }
            }
}

/* calculation_2D::SetMovingFrame, calculation_2D.cpp:405-496 (one rank:
 * the leading block receives nothing, MPI_PROC_NULL). */
static void grid_set_moving_frame(grid *g, int N)
{
    const double X_over_y = 0.0, X_over_z = 0.0, Y_over_x = 0.0, Y_over_z = 0.0, Z_over_x = 0.0,
                 Z_over_y = 0.0;
    if (N != 0)
        for (int j = 0; j < g->J; j++) g->Y[j] = g->axY[j] + N * (g->mf.trail_DJ - 1) * g->dy1;
    for (int i = 1; i < g->I - 1; i++) g->Xx[i] = (g->X[i + 1] - g->X[i - 1]) * g->rdx * 0.5;
    for (int j = 1; j < g->J - 1; j++) g->Yy[j] = (g->Y[j + 1] - g->Y[j - 1]) * g->rdy * 0.5;
    for (int k = 1; k < g->K - 1; k++) g->Zz[k] = (g->Z[k + 1] - g->Z[k - 1]) * g->rdz * 0.5;
    if (g->Zt) { /* terrain: the same central differences of the node heights */
        const int K = g->K;
        for (int j = 0; j < g->J; j++)
            for (int k = 1; k < K - 1; k++)
                g->Zz2[(size_t)j * K + k] = (g->Zt[(size_t)j * K + k + 1] - g->Zt[(size_t)j * K + k - 1]) * g->rdz * 0.5;
        for (int j = 1; j < g->J - 1; j++)
            for (int k = 0; k < K; k++)
                g->Zy2[(size_t)j * K + k] =
                    (g->Zt[(size_t)(j + 1) * K + k] - g->Zt[(size_t)(j - 1) * K + k]) * g->rdy * 0.5;
    }
    for (int i = 1; i < g->I - 1; i++)
        for (int j = 1; j < g->J - 1; j++)
            for (int k = 1; k < g->K - 1; k++) {
                const double Zz = g->Zt ? g->Zz2[(size_t)j * g->K + k] : g->Zz[k];
                const double Zy = g->Zt ? g->Zy2[(size_t)j * g->K + k] : Z_over_y;
                double jac = g->Xx[i] * g->Yy[j] * Zz + Z_over_x * X_over_y * Y_over_z + Y_over_x * Zy * X_over_z;
                jac += -g->Xx[i] * Zy * Y_over_z - Y_over_x * X_over_y * Zz - Z_over_x * g->Yy[j] * X_over_z;
                g->Jac[IX(g, i, j, k)] = 1.0 / jac;
            }
    int temp_J = (N == 0) ? 0 : g->mf.JMAX - g->mf.lead_DJ;
    if (temp_J != 0) {
        const int sh = g->mf.trail_DJ - 1;
        for (int k = 0; k < g->K; k++)
            for (int i = 0; i < g->I; i++) {
                for (int j = 0; j < g->J; j++) {
                    size_t c = IX(g, i, j, k);
                    if (j < temp_J + 1 && j + g->mf.lead_DJ - 1 < g->J - 1) {
                        size_t s = IX(g, i, j + sh, k);
                        g->un[c] = g->un[s]; g->vn[c] = g->vn[s]; g->wn[c] = g->wn[s]; g->pn[c] = g->pn[s];
                    } else if (j >= temp_J + 1) {
                        g->un[c] = 0.0; g->vn[c] = 0.0; g->wn[c] = 0.0; g->pn[c] = 0.0;
                    }
                }
                g->pn[IX(g, i, 0, k)] = g->pn[IX(g, i, 1, k)];
            }
    }
}

/* calculation_2D::UpdateInitialCond, calculation_2D.cpp:354-369 */
static void grid_update_initial(grid *g)
{
    size_t N = (size_t)g->I * g->J * g->K;
    memcpy(g->un, g->unn, N * sizeof(double));
    memcpy(g->vn, g->vnn, N * sizeof(double));
    memcpy(g->wn, g->wnn, N * sizeof(double));
    memcpy(g->pn, g->pnn, N * sizeof(double));
}

/* Geo_over_var, df_over_var.cpp:5-9 */
static inline double gov(double a, double b, double c, double d, double jac) { return (a * b - c * d) * jac; }

/* The nine inverse metrics with the reference's fixed-zero cross terms
 * (calculation_2D.cpp:102-104; use sites air.cpp:1497-1514). On a
 * terrain-following grid (extension) Z_over_z and Z_over_y are the node's
 * own (j, k) values; the other cross terms stay zero. */
typedef struct { double xX, xY, xZ, yX, yY, yZ, zX, zY, zZ; } metr;
static inline metr metrics_at(const grid *g, int i, int j, int k)
{
    const double X_over_y = 0.0, X_over_z = 0.0, Y_over_x = 0.0, Y_over_z = 0.0, Z_over_x = 0.0;
    const double Z_over_y = g->Zt ? g->Zy2[(size_t)j * g->K + k] : 0.0;
    const double Zz = g->Zt ? g->Zz2[(size_t)j * g->K + k] : g->Zz[k];
    double jac = g->Jac[IX(g, i, j, k)];
    metr m;
    m.xX = gov(g->Yy[j], Zz, Y_over_z, Z_over_y, jac);
    m.xY = gov(X_over_z, Z_over_y, X_over_y, Zz, jac);
    m.xZ = gov(X_over_y, Y_over_z, X_over_z, g->Yy[j], jac);
    m.yX = gov(Y_over_z, Z_over_x, Y_over_x, Zz, jac);
    m.yY = gov(g->Xx[i], Zz, X_over_z, Z_over_x, jac);
    m.yZ = gov(X_over_z, Y_over_x, g->Xx[i], Y_over_z, jac);
    m.zX = gov(Y_over_x, Z_over_y, g->Yy[j], Z_over_x, jac);
    m.zY = gov(X_over_y, Z_over_x, g->Xx[i], Z_over_y, jac);
    m.zZ = gov(g->Xx[i], g->Yy[j], X_over_y, Y_over_x, jac);
    return m;
}

/* ---------------------------------------------------------- wind profile */
/* SpeedProfile::Uav/Vav/Wav, air.cpp:71-253 (methods whose parameters the
 * reference initialises: 1, 2, 4, 5; others return 0 here). */
static double sp_U(airm *a, double x, double y, double z)
{
    (void)x; (void)z;
    switch (a->vmethod) {
    case 5: return a->vb * y;
    default: return 0;
    }
}
static double sp_V(airm *a, double x, double y, double z)
{
    (void)x;
    switch (a->vmethod) {
    case 1:
        if (z >= 2.8) return a->vb * 2.8;
        else if (z >= 0.0) return a->vb * z;
        else return 0.0;
    case 2: {
        double Rr = sqrt(pow(y - 5.0, 2) + pow(z - 2.0, 2));
        if (fabs(y - 5.0) <= 1.0e-6 && fabs(z - 2.0) <= 1.0e-6) a->valpha = 0.0;
        else if (y - 5.0 >= 0.0) a->valpha = asin((y - 5.0) / Rr);
        else if (y - 5.0 <= 0.0) a->valpha = asin((y - 5.0) / Rr) + 3.1415926;
        return -1.0 * 2.0 / (Rr + 2.0) * sin(a->valpha);
    }
    case 5: return a->vb * log(fabs(z) / 0.1 + 1);
    /* extension: the surface-layer log law (u_star / kappa) ln(z / z0), calm below z0 */
    case 7: return z > a->vz0 ? a->vb / a->vkappa * log(z / a->vz0) : 0.0;
    default: return 0;
    }
}
static double sp_W(airm *a, double x, double y, double z)
{
    (void)x;
    switch (a->vmethod) {
    case 2: {
        double Rr = sqrt(pow(y - 5.0, 2) + pow(z - 2.0, 2));
        if (fabs(y - 5.0) <= 1.0e-6 && fabs(z - 2.0) <= 1.0e-6) a->valpha = 0.0;
        else if (y - 5.0 >= 0.0) a->valpha = asin((y - 5.0) / Rr);
        else if (y - 5.0 <= 0.0) a->valpha = asin((y - 5.0) / Rr) + 3.1415926;
        return 1.0 * 2.0 / (Rr + 2.0) * cos(a->valpha);
    }
    case 5: return a->vb * y;
    default: return 0;
    }
}

/* air::SetWindProfile, air.cpp:1286-1304 */
static void air_set_wind(airm *a, int N)
{
    grid *g = &a->g;
    if (N != 0) {
        if (g->JMAX1 - 1 >= 0) a->y1 = g->axY[g->JMAX1 - 1] + N * (g->mf.trail_DJ - 1) * g->dy1;
        if (g->JMAX - g->JMAX2 < g->JMAX) a->y2 = g->axY[g->JMAX - g->JMAX2] + N * (g->mf.trail_DJ - 1) * g->dy1;
    }
    for (int i = 0; i < g->I; i++)
        for (int j = 0; j < g->J; j++)
            for (int k = 0; k < g->K; k++) {
                double Z0 = 0.0;
                /* terrain: height above the local ground */
                double zk = g->Zt ? g->Zt[(size_t)j * g->K + k] : g->Z[k];
                if (g->Zt) Z0 = g->zg[j];
                size_t c = IX(g, i, j, k);
                a->Uav[c] = sp_U(a, g->X[i], g->Y[j], zk - Z0);
                a->Vav[c] = sp_V(a, g->X[i], g->Y[j], zk - Z0);
                a->Wav[c] = sp_W(a, g->X[i], g->Y[j], zk - Z0);
            }
}

/* ------------------------------------------------------------- PML setup */
static void slab_alloc(slab *s, int n0, int n1, int n2)
{
    s->n0 = n0; s->n1 = n1; s->n2 = n2;
    for (int c = 0; c < 4; ++c) s->q[c] = zalloc((size_t)n0 * n1 * n2);
}

/* air::cal_PML_var, air.cpp:509-937 (single rank) */
static void air_pml_setup(orc *o)
{
    airm *a = &o->air;
    grid *g = &a->g;
    a->jx = o->jx; a->jy = o->jy; a->jz = o->jz;
    memset(a->s, 0, sizeof a->s);
    a->x1 = a->x2 = a->y1 = a->y2 = a->z1 = a->z2 = 0;
    a->w1 = a->w2 = a->l1 = a->l2 = a->h1 = a->h2 = 0;
    if (a->jx != 0) {
        a->sxmax = o->pxs; a->ax = o->pxa;
        if (a->jx == 1 || a->jx == 3) {
            a->w1 = 1.0 / fabs(g->axX[g->IMAX1 - 1] - g->axX[0]);
            a->x1 = g->axX[g->IMAX1 - 1];
        }
        if (a->jx == 2 || a->jx == 3) {
            a->w2 = 1.0 / fabs(g->axX[g->IMAX - 1] - g->axX[g->IMAX - g->IMAX2]);
            a->x2 = g->axX[g->IMAX - g->IMAX2];
        }
        if (a->jx == 1) g->IMAX2 = 0;
        if (a->jx == 2) g->IMAX1 = 0;
        if (g->IMAX1 > 0 && (a->jx == 1 || a->jx == 3)) slab_alloc(&a->s[0], g->IMAX1 + 1, g->J, g->K);
        if (g->IMAX2 > 0 && (a->jx == 2 || a->jx == 3)) slab_alloc(&a->s[1], g->IMAX2 + 1, g->J, g->K);
    } else {
        g->IMAX1 = 0; g->IMAX2 = 0;
    }
    if (a->jy != 0) {
        a->symax = o->pys; a->ay = o->pya;
        if (a->jy == 1 || a->jy == 3) {
            a->l1 = 1.0 / fabs(g->axY[g->JMAX1 - 1] - g->axY[0]);
            a->y1 = g->axY[g->JMAX1 - 1];
            a->pml_time = o->pyt;
            a->pml_count = 0;
        }
        if (a->jy == 2 || a->jy == 3) {
            a->l2 = 1.0 / fabs(g->axY[g->JMAX - 1] - g->axY[g->JMAX - g->JMAX2]);
            a->y2 = g->axY[g->JMAX - g->JMAX2];
        }
        if (a->jy == 1) g->JMAX2 = 0;
        if (a->jy == 2) g->JMAX1 = 0;
        if (g->JMAX1 > 0 && (a->jy == 1 || a->jy == 3)) slab_alloc(&a->s[2], g->I, g->JMAX1 + 1, g->K);
        if (g->JMAX2 > 0 && (a->jy == 2 || a->jy == 3)) slab_alloc(&a->s[3], g->I, g->JMAX2 + 1, g->K);
    } else {
        g->JMAX1 = 0; g->JMAX2 = 0;
    }
    if (a->jz != 0) {
        a->szmax = o->pzs; a->az = o->pza;
        if (a->jz == 1 || a->jz == 3) {
            a->h1 = 1.0 / fabs(g->axZ[g->KMAX1 - 1] - g->axZ[0]);
            a->z1 = g->axZ[g->KMAX1 - 1];
        }
        if (a->jz == 2 || a->jz == 3) {
            a->h2 = 1.0 / fabs(g->axZ[g->KMAX - 1] - g->axZ[g->KMAX - g->KMAX2]);
            a->z2 = g->axZ[g->KMAX - g->KMAX2];
        }
        if (a->jz == 1) g->KMAX2 = 0;
        if (a->jz == 2) g->KMAX1 = 0;
        if (g->KMAX1 > 0 && (a->jz == 1 || a->jz == 3)) slab_alloc(&a->s[4], g->I, g->J, g->KMAX1 + 1);
        if (g->KMAX2 > 0 && (a->jz == 2 || a->jz == 3)) slab_alloc(&a->s[5], g->I, g->J, g->KMAX2 + 1);
    } else {
        g->KMAX1 = 0; g->KMAX2 = 0;
    }
}

/* ------------------------------------------------------------ hill mask */
static inline int *crp(airm *a, int i, int j, int k)
{
    int nj = a->jstop - a->jstar + 1, nk = a->kstop - a->kstar + 1;
    return &a->cr_uc[((size_t)(i - a->istar) * nj + (j - a->jstar)) * nk + (k - a->kstar)];
}

/* air::cal_hill_var, air.cpp:938-1122 */
static void air_hill_setup(orc *o)
{
    airm *a = &o->air;
    grid *g = &a->g;
    a->cr_judge = o->cjudge;
    if (a->cr_judge == 0) return;
    const double *c = o->cc; /* a..l */
    double cr_a = c[0], cr_b = c[1], cr_c = c[2], cr_d = c[3], cr_e = c[4], cr_f = c[5], cr_g = c[6],
           cr_h = c[7], cr_i = c[8], cr_j = c[9], cr_k = c[10];
    /* mask 1 uses the canopy parameters, mask 2 the trunk ones (air.cpp:966-980,1910-1944) */
    a->eff1 = 1.0 / o->heff[1];
    a->invb1 = 1.0 / (1.0 + o->hsig[1] * g->dt * a->eff1);
    a->gama1 = g->dt / o->hKp[1] / o->hpor[1];
    a->eff2 = 1.0 / o->heff[2];
    a->invb2 = 1.0 / (1.0 + o->hsig[2] * g->dt * a->eff2);
    a->gama2 = g->dt / o->hKp[2] / o->hpor[2];
    a->istar = a->istop = a->jstar = a->jstop = a->kstar = a->kstop = 0;
    for (int i = 0; i < g->IMAX; i++) {
        if (fabs(g->axX[i] - o->box[0]) <= g->dx1 / 8.0) a->istar = i;
        if (fabs(g->axX[i] - o->box[1]) <= g->dx1 / 8.0) { a->istop = i; break; }
    }
    for (int j = 0; j < g->JMAX; j++) {
        if (fabs(g->axY[j] - o->box[2]) <= g->dy1 / 8.0) a->jstar = j;
        if (fabs(g->axY[j] - o->box[3]) <= g->dy1 / 8.0) { a->jstop = j; break; }
    }
    for (int k = 0; k < g->KMAX; k++) {
        if (fabs(g->axZ[k] - o->box[4]) <= g->dz1 / 8.0) a->kstar = k;
        if (fabs(g->axZ[k] - o->box[5]) <= g->dz1 / 8.0) { a->kstop = k; break; }
    }
    int ni = a->istop - a->istar + 1, nj = a->jstop - a->jstar + 1, nk = a->kstop - a->kstar + 1;
    if (ni <= 0 || nj <= 0 || nk <= 0) { a->cr_judge = 0; return; }
    a->cr_uc = (int *)calloc((size_t)ni * nj * nk, sizeof(int));
    const double *X = g->axX, *Y = g->axY, *Z = g->axZ;
    int ii = 0, jj = 0;
    for (int i = a->istar; i < a->istop + 1; i++)
        for (int j = a->jstar; j < a->jstop + 1; j++)
            for (int k = a->kstar; k < a->kstop + 1; k++) {
                int *m = crp(a, i, j, k);
                double len;
                *m = 0;
                switch (a->cr_judge) {
                case 1: /* sphere */
                    len = pow((X[i] - cr_c), 2) + pow((Y[j] - cr_d), 2) + pow((Z[k] - cr_e), 2);
                    if (sqrt(len) <= cr_b) *m = 1;
                    break;
                case 2: /* box */
                    if (X[i] >= cr_a && X[i] <= cr_b && Y[j] >= cr_c && Y[j] <= cr_d && Z[k] >= cr_e && Z[k] <= cr_f)
                        *m = 1;
                    break;
                case 3: /* three rows of cylinders */
                    for (jj = 0; jj < o->cpoints; jj++) {
                        len = pow((X[i] - cr_c), 2) + pow((Y[j] - (cr_d + jj * cr_b)), 2);
                        if (sqrt(len) <= cr_a && Z[k] <= cr_e) *m = 1;
                        len = pow((X[i] - cr_f), 2) + pow((Y[j] - (cr_g + jj * cr_b)), 2);
                        if (sqrt(len) <= cr_a && Z[k] <= cr_h) *m = 1;
                        len = pow((X[i] - cr_i), 2) + pow((Y[j] - (cr_j + jj * cr_b)), 2);
                        if (sqrt(len) <= cr_a && Z[k] <= cr_k) *m = 1;
                    }
                    break;
                case 4: /* cylinder array */
                    for (ii = 0; ii < cr_g; ii++)
                        for (jj = 0; jj < cr_f; jj++) {
                            len = pow((X[i] - (cr_b + ii * cr_e)), 2) + pow((Y[j] - (cr_c + jj * cr_d)), 2);
                            if (sqrt(len) <= cr_a) *m = 1;
                        }
                    break;
                case 5: /* tree: canopy cone + trunk */
                    for (ii = 0; ii < 1; ii++)
                        for (jj = 0; jj < 1; jj++) {
                            len = pow((X[i] - (0.0 + ii * 2.0)), 2) + pow((Y[j] - (3.0 + jj * 2.0)), 2);
                            double hgt = -25 / (9 - 1e-50) * sqrt(len) + 3.0;
                            if (sqrt(len) <= 0.9 && Z[k] <= hgt && Z[k] >= 0.5) *m = 1;
                            if (sqrt(len) <= 0.1 && Z[k] <= 1.5) *m = 2;
                        }
                    break;
                default: break;
                }
            }
    if (a->cr_judge == 5) {
        /* second sweep reuses the finished loop counters (ii = jj = 1), air.cpp:1108-1118 */
        for (int i = a->istar; i < a->istop + 1; i++)
            for (int j = a->jstar; j < a->jstop + 1; j++)
                for (int k = a->kstar; k < a->kstop + 1; k++) {
                    double len = pow((X[i] - (0.0 + ii * 2.0)), 2) + pow((Y[j] - (3.0 + jj * 2.0)), 2);
                    if (sqrt(len) <= 0.1 && Z[k] <= 1.5) *crp(a, i, j, k) = 2;
                }
    }
    (void)cr_h;
}

static inline int hill_mask(const airm *a, int in, int jn, int kn)
{
    if (a->cr_judge == 0) return 0;
    if (in < a->istar || in > a->istop || jn < a->jstar || jn > a->jstop || kn < a->kstar || kn > a->kstop)
        return 0;
    return *crp((airm *)a, in, jn, kn);
}

/* -------------------------------------------------- air::SetQMove */
static void slab_shift_j(slab *s, int jdim_is_1, const grid *g, int temp_J)
{
    /* shift along j by trail_DJ-1, zero the leading region (air.cpp:2522-2729) */
    (void)jdim_is_1;
    const int sh = g->mf.trail_DJ - 1;
    for (int c = 0; c < 4; ++c) {
        double *q = s->q[c];
        for (int a = 0; a < s->n0; a++)
            for (int j = 0; j < s->n1; j++)
                for (int k = 0; k < s->n2; k++) {
                    size_t d = SX(s, a, j, k);
                    if (j < temp_J + 1 && j + g->mf.lead_DJ - 1 < g->J - 1) q[d] = q[SX(s, a, j + sh, k)];
                    else if (j >= temp_J + 1) q[d] = 0.0;
                }
    }
}

static void air_set_q_move(airm *a, int N)
{
    grid *g = &a->g;
    int temp_J;
    if (N == 0) {
        temp_J = 0;
        for (int s = 0; s < 6; ++s)
            if (a->s[s].n0)
                for (int c = 0; c < 4; ++c)
                    memset(a->s[s].q[c], 0, sizeof(double) * a->s[s].n0 * a->s[s].n1 * a->s[s].n2);
    } else {
        temp_J = g->mf.JMAX - g->mf.lead_DJ;
    }
    if (temp_J != 0) {
        /* x1, x2 (j is dim 1) and z1, z2 (j is dim 1 too); y slabs are not moved */
        if (a->s[0].n0) slab_shift_j(&a->s[0], 1, g, temp_J);
        if (a->s[1].n0) slab_shift_j(&a->s[1], 1, g, temp_J);
        if (a->s[4].n0) slab_shift_j(&a->s[4], 1, g, temp_J);
        if (a->s[5].n0) slab_shift_j(&a->s[5], 1, g, temp_J);
    }
}

/* ---------------------------------------------------- stencil helpers */
/* forward first differences of a field at (i,j,k) */
#define FDI(A, g, i, j, k) ((A)[IX(g, (i) + 1, j, k)] - (A)[IX(g, i, j, k)])
#define FDJ(A, g, i, j, k) ((A)[IX(g, i, (j) + 1, k)] - (A)[IX(g, i, j, k)])
#define FDK(A, g, i, j, k) ((A)[IX(g, i, j, (k) + 1)] - (A)[IX(g, i, j, k)])
#define BDI(A, g, i, j, k) ((A)[IX(g, i, j, k)] - (A)[IX(g, (i) - 1, j, k)])
#define BDJ(A, g, i, j, k) ((A)[IX(g, i, j, k)] - (A)[IX(g, i, (j) - 1, k)])
#define BDK(A, g, i, j, k) ((A)[IX(g, i, j, k)] - (A)[IX(g, i, j, (k) - 1)])

/* Slab accessors: slab s at slab-local (a,b,c) */
#define QV(s, c, a, b, cc) ((s)->q[c][SX(s, a, b, cc)])

/* forward gradient of slab component along a metric row (xM,yM,zM), as
 * "xM*(Q[a+1]-Q[a])*rdx + yM*(..)*rdy + zM*(..)*rdz" */
static inline double sgrad_f(const slab *s, int c, int a, int b, int d, double xM, double yM, double zM,
                             double rdx, double rdy, double rdz)
{
    return xM * (QV(s, c, a + 1, b, d) - QV(s, c, a, b, d)) * rdx +
           yM * (QV(s, c, a, b + 1, d) - QV(s, c, a, b, d)) * rdy +
           zM * (QV(s, c, a, b, d + 1) - QV(s, c, a, b, d)) * rdz;
}
/* six-term forward sum of two slab components, left-to-right like the reference */
static inline double sgrad_f6(const slab *s, int c1, double x1, double y1, double z1, int c2, double x2,
                              double y2, double z2, int a, int b, int d, double rdx, double rdy, double rdz)
{
    return x1 * (QV(s, c1, a + 1, b, d) - QV(s, c1, a, b, d)) * rdx +
           y1 * (QV(s, c1, a, b + 1, d) - QV(s, c1, a, b, d)) * rdy +
           z1 * (QV(s, c1, a, b, d + 1) - QV(s, c1, a, b, d)) * rdz +
           x2 * (QV(s, c2, a + 1, b, d) - QV(s, c2, a, b, d)) * rdx +
           y2 * (QV(s, c2, a, b + 1, d) - QV(s, c2, a, b, d)) * rdy +
           z2 * (QV(s, c2, a, b, d + 1) - QV(s, c2, a, b, d)) * rdz;
}
/* backward gradient of slab component p (c=3) along a metric row */
static inline double sgrad_b(const slab *s, int a, int b, int d, double xM, double yM, double zM, double rdx,
                             double rdy, double rdz)
{
    return xM * (QV(s, 3, a, b, d) - QV(s, 3, a - 1, b, d)) * rdx +
           yM * (QV(s, 3, a, b, d) - QV(s, 3, a, b - 1, d)) * rdy +
           zM * (QV(s, 3, a, b, d) - QV(s, 3, a, b, d - 1)) * rdz;
}

/* PML profile sigma = smax*(d*W)^alpha, beta = 1 + 25*(d*W)^alpha (air.cpp:1580-1581) */
#define SIG(smax, dist, W, al) ((smax) * pow((dist) * (W), (al)))
#define BET(dist, W, al) (1.0 + 25.0 * pow((dist) * (W), (al)))

/* ------------------------------------------------------ air::cal_fp */
/* air.cpp:1953-2322: writes the pressure increment into p_nn (interior) */
static void air_cal_fp(airm *a, const double *tu, const double *tv, const double *tw, const double *tp, int scheme)
{
    grid *g = &a->g;
    const double dt = g->dt, rdx = g->rdx, rdy = g->rdy, rdz = g->rdz;
    const double gam = a->gamma, Pav = a->P0;
    if (scheme == S_FB_P_V && (a->jy == 1 || a->jy == 3)) { /* air.cpp:1965-1969 */
        a->pml_count = a->pml_count + 1;
        if (a->pml_count >= a->pml_time) g->JMAX1 = g->JMAX3;
        else g->JMAX1 = 0;
    }
    const int I = g->I, J = g->J, K = g->K;
    const slab *sx1 = &a->s[0], *sx2 = &a->s[1], *sy1 = &a->s[2], *sy2 = &a->s[3], *sz1 = &a->s[4],
               *sz2 = &a->s[5];
    for (int i = 1; i < I - 1; i++)
        for (int j = 1; j < J - 1; j++)
            for (int k = 1; k < K - 1; k++) {
                const int in = i, jn = j, kn = k;
                const size_t c = IX(g, i, j, k);
                metr m = metrics_at(g, i, j, k);
                const double *U = a->Uav, *V = a->Vav, *W = a->Wav;
                double coef1 = (U[c] * m.xX + V[c] * m.xY + W[c] * m.xZ) * rdx * dt;
                double coef2 = (U[c] * m.yX + V[c] * m.yY + W[c] * m.yZ) * rdy * dt;
                double coef3 = (U[c] * m.zX + V[c] * m.zY + W[c] * m.zZ) * rdz * dt;
#define CDIFF3(F, r1, r2, r3)                                                                                 \
    (r1 * ((F)[IX(g, i + 1, j, k)] - (F)[IX(g, i - 1, j, k)]) * rdx * 0.5 +                                   \
     r2 * ((F)[IX(g, i, j + 1, k)] - (F)[IX(g, i, j - 1, k)]) * rdy * 0.5 +                                   \
     r3 * ((F)[IX(g, i, j, k + 1)] - (F)[IX(g, i, j, k - 1)]) * rdz * 0.5)
                double U_X = CDIFF3(U, m.xX, m.yX, m.zX);
                double V_Y = CDIFF3(V, m.xY, m.yY, m.zY);
                double W_Z = CDIFF3(W, m.xZ, m.yZ, m.zZ);
                double P = tp[c];
                double pn = -coef1 * BDI(tp, g, i, j, k) - coef2 * BDJ(tp, g, i, j, k) - coef3 * BDK(tp, g, i, j, k);
                pn += -gam * P * dt * (U_X + V_Y + W_Z);
                double du_i = FDI(tu, g, i, j, k), du_j = FDJ(tu, g, i, j, k), du_k = FDK(tu, g, i, j, k);
                double dv_i = FDI(tv, g, i, j, k), dv_j = FDJ(tv, g, i, j, k), dv_k = FDK(tv, g, i, j, k);
                double dw_i = FDI(tw, g, i, j, k), dw_j = FDJ(tw, g, i, j, k), dw_k = FDK(tw, g, i, j, k);
                double div9 = m.xX * du_i * rdx + m.yX * du_j * rdy + m.zX * du_k * rdz + m.xY * dv_i * rdx +
                              m.yY * dv_j * rdy + m.zY * dv_k * rdz + m.xZ * dw_i * rdx + m.yZ * dw_j * rdy +
                              m.zZ * dw_k * rdz;
                pn += -gam * Pav * dt * (div9);
                double gu = m.xX * du_i * rdx + m.yX * du_j * rdy + m.zX * du_k * rdz;
                double gv = m.xY * dv_i * rdx + m.yY * dv_j * rdy + m.zY * dv_k * rdz;
                double gw = m.xZ * dw_i * rdx + m.yZ * dw_j * rdy + m.zZ * dw_k * rdz;
                double sx1v = 0, bx1 = 0, sx2v = 0, bx2 = 0;
                int ii = 0;
                const int inx1 = in < g->IMAX1, inx2 = in >= g->IMAX - g->IMAX2;
                if (inx1) {
                    sx1v = SIG(a->sxmax, a->x1 - g->X[i], a->w1, a->ax);
                    bx1 = BET(a->x1 - g->X[i], a->w1, a->ax);
                }
                if (inx2) {
                    ii = i - (I - sx2->n0);
                    sx2v = SIG(a->sxmax, g->X[i] - a->x2, a->w2, a->ax);
                    bx2 = BET(g->X[i] - a->x2, a->w2, a->ax);
                }
                /* PML X1 / X2 (air.cpp:2044-2074) */
                if (inx1) {
                    pn += (1.0 - 1.0 / bx1) * (gam * Pav * (gu)) * dt -
                          (sx1v * (P + gam * Pav * sgrad_f6(sx1, 1, m.xY, m.yY, m.zY, 2, m.xZ, m.yZ, m.zZ, i, j, k,
                                                              rdx, rdy, rdz))) *
                              dt;
                }
                if (inx2) {
                    pn += (1.0 - 1.0 / bx2) * (gam * Pav * (gu)) * dt -
                          (sx2v * (P + gam * Pav * sgrad_f6(sx2, 1, m.xY, m.yY, m.zY, 2, m.xZ, m.yZ, m.zZ, ii, j, k,
                                                              rdx, rdy, rdz))) *
                              dt;
                }
                /* PML Y1 / Y2 with X corners (air.cpp:2076-2158) */
                for (int side = 0; side < 2; ++side) {
                    int iny = side == 0 ? (jn < g->JMAX1) : (jn >= g->JMAX - g->JMAX2);
                    if (!iny) continue;
                    const slab *sy = side == 0 ? sy1 : sy2;
                    int jj = side == 0 ? j : j - (J - sy2->n1);
                    double dist = side == 0 ? (a->y1 - g->Y[j]) : (g->Y[j] - a->y2);
                    double Wd = side == 0 ? a->l1 : a->l2;
                    double syv = SIG(a->symax, dist, Wd, a->ay);
                    double by = BET(dist, Wd, a->ay);
                    pn += (1.0 - 1.0 / by) * (gam * Pav * (gv)) * dt -
                          syv * (P + gam * Pav * sgrad_f6(sy, 0, m.xX, m.yX, m.zX, 2, m.xZ, m.yZ, m.zZ, i, jj, k, rdx,
                                                          rdy, rdz)) *
                              dt;
                    if (inx1) {
                        pn += -(QV(sx1, 3, i, j, k) * sx1v * syv +
                                gam * Pav *
                                    ((1 / bx1 - 1) * syv * sgrad_f(sx1, 0, i, j, k, m.xX, m.yX, m.zX, rdx, rdy, rdz) +
                                     (1 / by - 1) * sx1v * sgrad_f(sx1, 1, i, j, k, m.xY, m.yY, m.zY, rdx, rdy, rdz))) *
                              dt;
                    } else if (inx2) {
                        pn += -(QV(sx2, 3, ii, j, k) * sx2v * syv +
                                gam * Pav *
                                    ((1 / bx2 - 1) * syv * sgrad_f(sx2, 0, ii, j, k, m.xX, m.yX, m.zX, rdx, rdy, rdz) +
                                     (1 / by - 1) * sx2v * sgrad_f(sx2, 1, ii, j, k, m.xY, m.yY, m.zY, rdx, rdy, rdz))) *
                              dt;
                    }
                }
                /* PML Z1 / Z2 with X and Y corners (air.cpp:2160-2292) */
                for (int side = 0; side < 2; ++side) {
                    int inz = side == 0 ? (kn < g->KMAX1) : (kn >= g->KMAX - g->KMAX2);
                    if (!inz) continue;
                    const slab *sz = side == 0 ? sz1 : sz2;
                    int kk = side == 0 ? k : k - (K - sz2->n2);
                    double dist = side == 0 ? (a->z1 - g->Z[k]) : (g->Z[k] - a->z2);
                    double Wd = side == 0 ? a->h1 : a->h2;
                    double szv = SIG(a->szmax, dist, Wd, a->az);
                    double bz = BET(dist, Wd, a->az);
                    pn += (1.0 - 1.0 / bz) * gam * Pav * (gw) * dt -
                          szv * (P + gam * Pav * sgrad_f6(sz, 0, m.xX, m.yX, m.zX, 1, m.xY, m.yY, m.zY, i, j, kk, rdx,
                                                          rdy, rdz)) *
                              dt;
                    if (inx1) {
                        pn += -(QV(sx1, 3, i, j, k) * sx1v * szv +
                                gam * Pav *
                                    ((1 / bx1 - 1) * szv * sgrad_f(sx1, 0, i, j, k, m.xX, m.yX, m.zX, rdx, rdy, rdz) +
                                     (1 / bz - 1) * sx1v * sgrad_f(sx1, 2, i, j, k, m.xZ, m.yZ, m.zZ, rdx, rdy, rdz))) *
                              dt;
                    } else if (inx2) {
                        pn += -(QV(sx2, 3, ii, j, k) * sx2v * szv +
                                gam * Pav *
                                    ((1 / bx2 - 1) * szv * sgrad_f(sx2, 0, ii, j, k, m.xX, m.yX, m.zX, rdx, rdy, rdz) +
                                     (1 / bz - 1) * sx2v * sgrad_f(sx2, 2, ii, j, k, m.xZ, m.yZ, m.zZ, rdx, rdy, rdz))) *
                              dt;
                    }
                    for (int ys = 0; ys < 2; ++ys) {
                        int iny = ys == 0 ? (jn < g->JMAX1) : (jn >= g->JMAX - g->JMAX2);
                        if (!iny) continue;
                        const slab *sy = ys == 0 ? sy1 : sy2;
                        int jj = ys == 0 ? j : j - (J - sy2->n1);
                        double distv = ys == 0 ? (a->y1 - g->Y[j]) : (g->Y[j] - a->y2);
                        double Wy = ys == 0 ? a->l1 : a->l2;
                        double syv = SIG(a->symax, distv, Wy, a->ay);
                        double by = BET(distv, Wy, a->ay);
                        pn += -(QV(sy, 3, i, jj, k) * syv * szv +
                                gam * Pav *
                                    ((1 / by - 1) * szv * sgrad_f(sy, 1, i, jj, k, m.xY, m.yY, m.zY, rdx, rdy, rdz) +
                                     (1 / bz - 1) * syv * sgrad_f(sy, 2, i, jj, k, m.xZ, m.yZ, m.zZ, rdx, rdy, rdz))) *
                              dt;
                        break; /* y1 and y2 are exclusive ("else if") */
                    }
                }
                /* porous inclusions (air.cpp:2295-2318) */
                int msk = hill_mask(a, in, jn, kn);
                if (msk == 1) pn = -a->gama1 * (div9);
                if (msk == 2) pn = -a->gama2 * (div9);
                g->pnn[c] = pn;
            }
#undef CDIFF3
}

/* ---------------------------------------------------- air::cal_fuvw */
/* air.cpp:1476-1949: writes the velocity increments into u/v/w_nn (interior) */
static void air_cal_fuvw(airm *a, const double *tu, const double *tv, const double *tw, const double *tp, int scheme)
{
    grid *g = &a->g;
    const double dt = g->dt, rdx = g->rdx, rdy = g->rdy, rdz = g->rdz;
    const double Aav = a->Aav;
    if (scheme == S_FB_V_P && (a->jy == 1 || a->jy == 3)) { /* air.cpp:1488-1492 */
        a->pml_count = a->pml_count + 1;
        if (a->pml_count >= a->pml_time) g->JMAX1 = g->JMAX3;
        else g->JMAX1 = 0;
    }
    const int I = g->I, J = g->J, K = g->K;
    const slab *sx1 = &a->s[0], *sx2 = &a->s[1], *sy1 = &a->s[2], *sy2 = &a->s[3], *sz1 = &a->s[4],
               *sz2 = &a->s[5];
    for (int i = 1; i < I - 1; i++)
        for (int j = 1; j < J - 1; j++)
            for (int k = 1; k < K - 1; k++) {
                const int in = i, jn = j, kn = k;
                const size_t c = IX(g, i, j, k);
                metr m = metrics_at(g, i, j, k);
                const double *U = a->Uav, *V = a->Vav, *W = a->Wav;
                double coef1 = (U[c] * m.xX + V[c] * m.xY + W[c] * m.xZ) * rdx * dt;
                double coef2 = (U[c] * m.yX + V[c] * m.yY + W[c] * m.yZ) * rdy * dt;
                double coef3 = (U[c] * m.zX + V[c] * m.zY + W[c] * m.zZ) * rdz * dt;
#define CDIFF3(F, r1, r2, r3)                                                                                 \
    (r1 * ((F)[IX(g, i + 1, j, k)] - (F)[IX(g, i - 1, j, k)]) * rdx * 0.5 +                                   \
     r2 * ((F)[IX(g, i, j + 1, k)] - (F)[IX(g, i, j - 1, k)]) * rdy * 0.5 +                                   \
     r3 * ((F)[IX(g, i, j, k + 1)] - (F)[IX(g, i, j, k - 1)]) * rdz * 0.5)
                double U_X = CDIFF3(U, m.xX, m.yX, m.zX), U_Y = CDIFF3(U, m.xY, m.yY, m.zY),
                       U_Z = CDIFF3(U, m.xZ, m.yZ, m.zZ);
                double V_X = CDIFF3(V, m.xX, m.yX, m.zX), V_Y = CDIFF3(V, m.xY, m.yY, m.zY),
                       V_Z = CDIFF3(V, m.xZ, m.yZ, m.zZ);
                double W_X = CDIFF3(W, m.xX, m.yX, m.zX), W_Y = CDIFF3(W, m.xY, m.yY, m.zY),
                       W_Z = CDIFF3(W, m.xZ, m.yZ, m.zZ);
#undef CDIFF3
                const double u = tu[c], v = tv[c], w = tw[c];
                double gpX = m.xX * BDI(tp, g, i, j, k) * rdx + m.yX * BDJ(tp, g, i, j, k) * rdy +
                             m.zX * BDK(tp, g, i, j, k) * rdz;
                double gpY = m.xY * BDI(tp, g, i, j, k) * rdx + m.yY * BDJ(tp, g, i, j, k) * rdy +
                             m.zY * BDK(tp, g, i, j, k) * rdz;
                double gpZ = m.xZ * BDI(tp, g, i, j, k) * rdx + m.yZ * BDJ(tp, g, i, j, k) * rdy +
                             m.zZ * BDK(tp, g, i, j, k) * rdz;
                double un = (a->upwind ? -coef1 * BDI(tu, g, i, j, k) - coef2 * BDJ(tu, g, i, j, k) - coef3 * BDK(tu, g, i, j, k)
                                     : -coef1 * FDI(tu, g, i, j, k) - coef2 * FDJ(tu, g, i, j, k) - coef3 * FDK(tu, g, i, j, k));
                un += -u * U_X * dt - v * U_Y * dt - w * U_Z * dt;
                un += -Aav * dt * (gpX);
                double vn = (a->upwind ? -coef1 * BDI(tv, g, i, j, k) - coef2 * BDJ(tv, g, i, j, k) - coef3 * BDK(tv, g, i, j, k)
                                     : -coef1 * FDI(tv, g, i, j, k) - coef2 * FDJ(tv, g, i, j, k) - coef3 * FDK(tv, g, i, j, k));
                vn += -u * V_X * dt - v * V_Y * dt - w * V_Z * dt;
                vn += -Aav * dt * (gpY);
                double wn = (a->upwind ? -coef1 * BDI(tw, g, i, j, k) - coef2 * BDJ(tw, g, i, j, k) - coef3 * BDK(tw, g, i, j, k)
                                     : -coef1 * FDI(tw, g, i, j, k) - coef2 * FDJ(tw, g, i, j, k) - coef3 * FDK(tw, g, i, j, k));
                wn += -u * W_X * dt - v * W_Y * dt - w * W_Z * dt;
                wn += -Aav * dt * (gpZ);
                double sx1v = 0, bx1 = 0, sx2v = 0, bx2 = 0;
                int ii = 0;
                const int inx1 = in < g->IMAX1, inx2 = in >= g->IMAX - g->IMAX2;
                if (inx1) {
                    sx1v = SIG(a->sxmax, a->x1 - g->X[i], a->w1, a->ax);
                    bx1 = BET(a->x1 - g->X[i], a->w1, a->ax);
                }
                if (inx2) {
                    ii = i - (I - sx2->n0);
                    sx2v = SIG(a->sxmax, g->X[i] - a->x2, a->w2, a->ax);
                    bx2 = BET(g->X[i] - a->x2, a->w2, a->ax);
                }
                /* PML X1 / X2 (air.cpp:1579-1619) */
                for (int xs = 0; xs < 2; ++xs) {
                    int inx = xs == 0 ? inx1 : inx2;
                    if (!inx) continue;
                    const slab *sx = xs == 0 ? sx1 : sx2;
                    int ia = xs == 0 ? i : ii;
                    double sxv = xs == 0 ? sx1v : sx2v, bx = xs == 0 ? bx1 : bx2;
                    un += -sxv * (u) * dt + (1.0 - 1.0 / bx) * (Aav * (gpX)) * dt;
                    vn += -sxv * (v + Aav * sgrad_b(sx, ia, j, k, m.xY, m.yY, m.zY, rdx, rdy, rdz)) * dt;
                    wn += -sxv * (w + Aav * sgrad_b(sx, ia, j, k, m.xZ, m.yZ, m.zZ, rdx, rdy, rdz)) * dt;
                }
                /* PML Y1 / Y2 with X corners (air.cpp:1621-1728) */
                for (int ys = 0; ys < 2; ++ys) {
                    int iny = ys == 0 ? (jn < g->JMAX1) : (jn >= g->JMAX - g->JMAX2);
                    if (!iny) continue;
                    const slab *sy = ys == 0 ? sy1 : sy2;
                    int jj = ys == 0 ? j : j - (J - sy2->n1);
                    double dist = ys == 0 ? (a->y1 - g->Y[j]) : (g->Y[j] - a->y2);
                    double Wd = ys == 0 ? a->l1 : a->l2;
                    double syv = SIG(a->symax, dist, Wd, a->ay);
                    double by = BET(dist, Wd, a->ay);
                    un += -syv * (u + Aav * sgrad_b(sy, i, jj, k, m.xX, m.yX, m.zX, rdx, rdy, rdz)) * dt;
                    vn += (1.0 - 1.0 / by) * Aav * (gpY) * dt - syv * v * dt;
                    wn += -syv * (w + Aav * sgrad_b(sy, i, jj, k, m.xZ, m.yZ, m.zZ, rdx, rdy, rdz)) * dt;
                    if (inx1 || inx2) {
                        const slab *sx = inx1 ? sx1 : sx2;
                        int ia = inx1 ? i : ii;
                        double sxv = inx1 ? sx1v : sx2v, bx = inx1 ? bx1 : bx2;
                        un += -(QV(sx, 0, ia, j, k) * sxv * syv +
                                (1 / bx - 1) * syv * Aav * sgrad_b(sx, ia, j, k, m.xX, m.yX, m.zX, rdx, rdy, rdz)) *
                              dt;
                        vn += -(QV(sx, 1, ia, j, k) * sxv * syv +
                                (1 / by - 1) * sxv * Aav * sgrad_b(sx, ia, j, k, m.xY, m.yY, m.zY, rdx, rdy, rdz)) *
                              dt;
                        wn += -QV(sx, 2, ia, j, k) * sxv * syv * dt;
                    }
                }
                /* PML Z1 / Z2 with X and Y corners (air.cpp:1730-1905) */
                for (int zs = 0; zs < 2; ++zs) {
                    int inz = zs == 0 ? (kn < g->KMAX1) : (kn >= g->KMAX - g->KMAX2);
                    if (!inz) continue;
                    const slab *sz = zs == 0 ? sz1 : sz2;
                    int kk = zs == 0 ? k : k - (K - sz2->n2);
                    double dist = zs == 0 ? (a->z1 - g->Z[k]) : (g->Z[k] - a->z2);
                    double Wd = zs == 0 ? a->h1 : a->h2;
                    double szv = SIG(a->szmax, dist, Wd, a->az);
                    double bz = BET(dist, Wd, a->az);
                    un += -szv * (u + Aav * sgrad_b(sz, i, j, kk, m.xX, m.yX, m.zX, rdx, rdy, rdz)) * dt;
                    vn += -szv * (v + Aav * sgrad_b(sz, i, j, kk, m.xY, m.yY, m.zY, rdx, rdy, rdz)) * dt;
                    wn += (1.0 - 1.0 / bz) * Aav * (gpZ) * dt - szv * w * dt;
                    if (inx1 || inx2) {
                        const slab *sx = inx1 ? sx1 : sx2;
                        int ia = inx1 ? i : ii;
                        double sxv = inx1 ? sx1v : sx2v, bx = inx1 ? bx1 : bx2;
                        un += -(QV(sx, 0, ia, j, k) * sxv * szv +
                                (1.0 / bx - 1.0) * szv * Aav * sgrad_b(sx, ia, j, k, m.xX, m.yX, m.zX, rdx, rdy, rdz)) *
                              dt;
                        vn += -QV(sx, 1, ia, j, k) * sxv * szv * dt;
                        wn += -(QV(sx, 2, ia, j, k) * sxv * szv +
                                (1.0 / bz - 1.0) * sxv * Aav * sgrad_b(sx, ia, j, k, m.xZ, m.yZ, m.zZ, rdx, rdy, rdz)) *
                              dt;
                    }
                    int iny1 = jn < g->JMAX1, iny2 = jn >= g->JMAX - g->JMAX2;
                    if (iny1 || iny2) {
                        const slab *sy = iny1 ? sy1 : sy2;
                        int jj = iny1 ? j : j - (J - sy2->n1);
                        double distv = iny1 ? (a->y1 - g->Y[j]) : (g->Y[j] - a->y2);
                        double Wy = iny1 ? a->l1 : a->l2;
                        double syv = SIG(a->symax, distv, Wy, a->ay);
                        double by = BET(distv, Wy, a->ay);
                        un += -QV(sy, 0, i, jj, k) * syv * szv * dt;
                        vn += -(QV(sy, 1, i, jj, k) * syv * szv +
                                (1.0 / by - 1.0) * szv * Aav * sgrad_b(sy, i, jj, k, m.xY, m.yY, m.zY, rdx, rdy, rdz)) *
                              dt;
                        wn += -(QV(sy, 2, i, jj, k) * syv * szv +
                                (1.0 / bz - 1.0) * syv * Aav * sgrad_b(sy, i, jj, k, m.xZ, m.yZ, m.zZ, rdx, rdy, rdz)) *
                              dt;
                    }
                }
                /* porous inclusions (air.cpp:1908-1945) */
                int msk = hill_mask(a, in, jn, kn);
                if (msk == 1) {
                    un = -1.0 * a->invb1 * dt * a->eff1 * (gpX) + u * a->invb1 - u;
                    vn = -1.0 * a->invb1 * dt * a->eff1 * (gpY) + v * a->invb1 - v;
                    wn = -1.0 * a->invb1 * dt * a->eff1 * (gpZ) + w * a->invb1 - w;
                }
                if (msk == 2) {
                    un = -1.0 * a->invb2 * dt * a->eff2 * (gpX) + u * a->invb2 - u;
                    vn = -1.0 * a->invb2 * dt * a->eff2 * (gpY) + v * a->invb2 - v;
                    wn = -1.0 * a->invb2 * dt * a->eff2 * (gpZ) + w * a->invb2 - w;
                }
                g->unn[c] = un; g->vnn[c] = vn; g->wnn[c] = wn;
            }
}

/* ------------------------------------------------- porous::cal_fuvw/fp */
/* porous.cpp:58-104 */
static void pore_cal_fuvw(grid *g, const double *tu, const double *tv, const double *tw, const double *tp)
{
    const double dt = g->dt, rdx = g->rdx, rdy = g->rdy, rdz = g->rdz;
    for (int k = 1; k < g->K - 1; k++)
        for (int j = 1; j < g->J - 1; j++)
            for (int i = 1; i < g->I - 1; i++) {
                metr m = metrics_at(g, i, j, k);
                size_t c = IX(g, i, j, k);
                double bi = BDI(tp, g, i, j, k), bj = BDJ(tp, g, i, j, k), bk = BDK(tp, g, i, j, k);
                g->unn[c] = -1.0 * g->invBeta * dt * g->eff * (m.xX * bi * rdx + m.yX * bj * rdy + m.zX * bk * rdz) +
                            tu[c] * g->invBeta - tu[c];
                g->vnn[c] = -1.0 * g->invBeta * dt * g->eff * (m.xY * bi * rdx + m.yY * bj * rdy + m.zY * bk * rdz) +
                            tv[c] * g->invBeta - tv[c];
                g->wnn[c] = -1.0 * g->invBeta * dt * g->eff * (m.xZ * bi * rdx + m.yZ * bj * rdy + m.zZ * bk * rdz) +
                            tw[c] * g->invBeta - tw[c];
            }
}

/* porous.cpp:107-143 */
static void pore_cal_fp(grid *g, const double *tu, const double *tv, const double *tw)
{
    const double rdx = g->rdx, rdy = g->rdy, rdz = g->rdz;
    for (int k = 1; k < g->K - 1; k++)
        for (int j = 1; j < g->J - 1; j++)
            for (int i = 1; i < g->I - 1; i++) {
                metr m = metrics_at(g, i, j, k);
                size_t c = IX(g, i, j, k);
                g->pnn[c] = -g->Gama * (m.xX * rdx * FDI(tu, g, i, j, k) + m.yX * rdy * FDJ(tu, g, i, j, k) +
                                        m.zX * rdz * FDK(tu, g, i, j, k) + m.xY * rdx * FDI(tv, g, i, j, k) +
                                        m.yY * rdy * FDJ(tv, g, i, j, k) + m.zY * rdz * FDK(tv, g, i, j, k) +
                                        m.xZ * rdx * FDI(tw, g, i, j, k) + m.yZ * rdy * FDJ(tw, g, i, j, k) +
                                        m.zZ * rdz * FDK(tw, g, i, j, k));
            }
}

/* ----------------------------------------- calculation_2D::Cal_* */
/* calculation_2D.cpp:581-613 (pressure) and 548-579 (velocity): add the
 * increments to the old state on the interior. */
static void grid_accumulate_p(grid *g)
{
    for (int i = 1; i < g->I - 1; i++)
        for (int j = 1; j < g->J - 1; j++)
            for (int k = 1; k < g->K - 1; k++) {
                size_t c = IX(g, i, j, k);
                g->pnn[c] = g->pn[c] + g->pnn[c];
            }
}
static void grid_accumulate_v(grid *g)
{
    for (int i = 1; i < g->I - 1; i++)
        for (int j = 1; j < g->J - 1; j++)
            for (int k = 1; k < g->K - 1; k++) {
                size_t c = IX(g, i, j, k);
                g->unn[c] = g->un[c] + g->unn[c];
                g->vnn[c] = g->vn[c] + g->vnn[c];
                g->wnn[c] = g->wn[c] + g->wnn[c];
            }
}

/* ------------------------------------------------------ face BCs */
enum { F_NORTH, F_SOUTH, F_WEST, F_EAST, F_FRONT, F_BACK };

/* calculation_2D::UpdateBC_pressure, calculation_2D.cpp:646-721 */
static void bc_pressure(grid *g, int face)
{
    double *p = g->pnn;
    const int I = g->I, J = g->J, K = g->K;
    switch (face) {
    case F_WEST:
        for (int i = 0; i < I; i++) for (int k = 0; k < K; k++) p[IX(g, i, 0, k)] = p[IX(g, i, 1, k)];
        break;
    case F_EAST:
        for (int i = 0; i < I; i++)
            for (int k = 0; k < K; k++) {
                int jn = J - 1;
                p[IX(g, i, jn, k)] = 15.0 / 8.0 * p[IX(g, i, jn - 1, k)] - 5.0 / 4.0 * p[IX(g, i, jn - 2, k)] +
                                     3.0 / 8.0 * p[IX(g, i, jn - 3, k)];
            }
        break;
    case F_SOUTH:
        for (int i = 0; i < I; i++) for (int j = 0; j < J; j++) p[IX(g, i, j, 0)] = p[IX(g, i, j, 1)];
        break;
    case F_NORTH:
        for (int i = 0; i < I; i++) for (int j = 0; j < J; j++) p[IX(g, i, j, K - 1)] = p[IX(g, i, j, K - 2)];
        break;
    case F_FRONT:
        for (int j = 0; j < J; j++) for (int k = 0; k < K; k++) p[IX(g, 0, j, k)] = p[IX(g, 1, j, k)];
        break;
    case F_BACK:
        for (int j = 0; j < J; j++) for (int k = 0; k < K; k++) p[IX(g, I - 1, j, k)] = p[IX(g, I - 2, j, k)];
        break;
    }
}

/* calculation_2D::UpdateBC_velocity, calculation_2D.cpp:777-864 */
static void bc_velocity(grid *g, int face)
{
    double *u = g->unn, *v = g->vnn, *w = g->wnn;
    const int I = g->I, J = g->J, K = g->K;
    switch (face) {
    case F_WEST:
        for (int i = 0; i < I; i++)
            for (int k = 0; k < K; k++) {
                u[IX(g, i, 0, k)] = u[IX(g, i, 1, k)]; v[IX(g, i, 0, k)] = 0.0; w[IX(g, i, 0, k)] = w[IX(g, i, 1, k)];
            }
        break;
    case F_EAST:
        for (int i = 0; i < I; i++)
            for (int k = 0; k < K; k++) {
                u[IX(g, i, J - 1, k)] = u[IX(g, i, J - 2, k)];
                v[IX(g, i, J - 1, k)] = 0.0;
                w[IX(g, i, J - 1, k)] = w[IX(g, i, J - 2, k)];
            }
        break;
    case F_SOUTH:
        for (int i = 0; i < I; i++)
            for (int j = 0; j < J; j++) {
                u[IX(g, i, j, 0)] = u[IX(g, i, j, 1)]; v[IX(g, i, j, 0)] = v[IX(g, i, j, 1)]; w[IX(g, i, j, 0)] = 0.0;
            }
        break;
    case F_NORTH:
        for (int i = 0; i < I; i++)
            for (int j = 0; j < J; j++) {
                u[IX(g, i, j, K - 1)] = u[IX(g, i, j, K - 2)];
                v[IX(g, i, j, K - 1)] = v[IX(g, i, j, K - 2)];
                w[IX(g, i, j, K - 1)] = 0.0;
            }
        break;
    case F_FRONT:
        for (int j = 0; j < J; j++)
            for (int k = 0; k < K; k++) {
                u[IX(g, 0, j, k)] = 0.0; v[IX(g, 0, j, k)] = v[IX(g, 1, j, k)]; w[IX(g, 0, j, k)] = w[IX(g, 1, j, k)];
            }
        break;
    case F_BACK:
        for (int j = 0; j < J; j++)
            for (int k = 0; k < K; k++) {
                u[IX(g, I - 1, j, k)] = 0.0;
                v[IX(g, I - 1, j, k)] = v[IX(g, I - 2, j, k)];
                w[IX(g, I - 1, j, k)] = w[IX(g, I - 2, j, k)];
            }
        break;
    }
}

/* TDBC on the east face: calculation_2D.cpp:986-1028 */
static double cal_tdbc(const double *psi, double p, double Z, double dt)
{
    double temp_at = 0, temp_psi = 0;
    for (int k = 0; k < 6; k++) {
        temp_at += TD_A[k] * dt;
        temp_psi += exp(-1 * TD_R[k] * dt) * psi[k];
    }
    return 1.0 / (1 + temp_at) * (p / Z - temp_psi);
}
static void update_psi(double *psi, double w, double dt)
{
    for (int k = 0; k < 6; k++) psi[k] = exp(-1 * TD_R[k] * dt) * psi[k] + TD_A[k] * w * dt;
}
/* Impedance ground (extension; the reference's TDBC acts on the east face
 * only). The face between the south nodes k = 0 and k = 1 is where w(k = 1)
 * sits: the pressure update at k = 1 takes w(2) - w(1), and the rigid face
 * holds it by the copy p(0) = p(1). The impedance face sets w(1) at every
 * interior node from the new pressure p(1) with the east face's recursive
 * convolution (calculation_2D.cpp:986-1017) and its own poles: the normal
 * velocity into the ground is v_n = -w, p / Z = v_n + sum psi_q, and
 * psi_q <- exp(-r_q dt') psi_q + a_q dt' v_n with dt' = dt / tau, i.e.
 * Z(w) = Z_inf (1 + sum a_q / (r_q + i w tau)) for small dt'. Runs before
 * the face copies, which then carry w(1) to the edge nodes. */
static void bc_velocity_tdbc_ground(orc *o)
{
    grid *g = &o->air.g;
    const double dtp = g->dt / o->gtau;
    double e[6], adt = 0;
    for (int q = 0; q < 6; q++) {
        e[q] = exp(-1 * o->gr[q] * dtp);
        adt += o->ga[q] * dtp;
    }
    for (int i = 1; i < g->I - 1; i++)
        for (int j = 1; j < g->J - 1; j++) {
            double *psi = &o->gpsi[((size_t)i * g->J + j) * 6];
            double mem = 0;
            for (int q = 0; q < 6; q++) mem += e[q] * psi[q];
            const double vn = 1.0 / (1 + adt) * (g->pnn[IX(g, i, j, 1)] / o->gZ - mem);
            g->wnn[IX(g, i, j, 1)] = -vn;
            for (int q = 0; q < 6; q++) psi[q] = e[q] * psi[q] + o->ga[q] * dtp * vn;
        }
}

static void bc_velocity_tdbc_east(grid *g, double Z, double tau)
{
    const int I = g->I, J = g->J, K = g->K;
    for (int i = 0; i < I; i++)
        for (int k = 0; k < K; k++) {
            size_t c = IX(g, i, J - 1, k);
            g->unn[c] = g->unn[IX(g, i, J - 2, k)];
            g->vnn[c] = 0.0;
            g->wnn[c] = g->wnn[IX(g, i, J - 2, k)];
            double *psi = &g->psi[((size_t)i * K + k) * 6];
            g->vnn[c] = cal_tdbc(psi, g->pnn[c], Z, g->dt / tau);
            update_psi(psi, g->vnn[c], g->dt / tau);
        }
}

/* air-porous interface, calculation_2D.cpp:865-985 (ratio < 5 branch) */
static int coupling_ratio_ok(const grid *air, const grid *pore)
{
    int r = (int)(air->dz1 / pore->dz1);
    return r < 5.0;
}
static void interface_velocity(grid *air, grid *pore)
{
    if (!coupling_ratio_ok(air, pore)) return;
    for (int i = 0; i < air->I; i++)
        for (int j = 0; j < air->J; j++) {
            air->unn[IX(air, i, j, 0)] = pore->unn[IX(pore, i, j, pore->K - 2)];
            pore->unn[IX(pore, i, j, pore->K - 1)] = air->unn[IX(air, i, j, 1)];
            air->vnn[IX(air, i, j, 0)] = pore->vnn[IX(pore, i, j, pore->K - 2)];
            pore->vnn[IX(pore, i, j, pore->K - 1)] = air->vnn[IX(air, i, j, 1)];
            air->wnn[IX(air, i, j, 0)] = pore->wnn[IX(pore, i, j, pore->K - 2)];
            pore->wnn[IX(pore, i, j, pore->K - 1)] = air->wnn[IX(air, i, j, 1)];
        }
}
static void interface_pressure(grid *air, grid *pore)
{
    if (!coupling_ratio_ok(air, pore)) return;
    for (int i = 0; i < air->I; i++)
        for (int j = 0; j < air->J; j++) {
            air->pnn[IX(air, i, j, 0)] = pore->pnn[IX(pore, i, j, pore->K - 2)];
            pore->pnn[IX(pore, i, j, pore->K - 1)] = air->pnn[IX(air, i, j, 1)];
        }
}

/* ---------------------------------------------- PML integral updates */
/* air::Update_PML_Qvw / Update_PML_Qp, air.cpp:2323-2439 */
static void slab_accumulate(airm *a, int sid, int comp, const double *f)
{
    slab *s = &a->s[sid];
    grid *g = &a->g;
    if (!s->n0) return;
    const double dt = g->dt;
    int i0 = 0, j0 = 0, k0 = 0;
    if (sid == 1) i0 = g->I - s->n0;
    if (sid == 3) j0 = g->J - s->n1;
    if (sid == 5) k0 = g->K - s->n2;
    double *q = s->q[comp];
    for (int x = 0; x < s->n0; x++)
        for (int y = 0; y < s->n1; y++)
            for (int z = 0; z < s->n2; z++) q[SX(s, x, y, z)] += dt * f[IX(g, x + i0, y + j0, z + k0)];
}
static void air_update_qvw(airm *a)
{
    for (int sid = 0; sid < 6; ++sid) {
        if (sid == 2 && !(a->pml_count >= a->pml_time)) continue;
        slab_accumulate(a, sid, 0, a->g.unn);
        slab_accumulate(a, sid, 1, a->g.vnn);
        slab_accumulate(a, sid, 2, a->g.wnn);
    }
}
static void air_update_qp(airm *a)
{
    for (int sid = 0; sid < 6; ++sid) {
        if (sid == 2 && !(a->pml_count >= a->pml_time)) continue;
        slab_accumulate(a, sid, 3, a->g.pnn);
    }
}

/* ---------------------------------------------- airpore half steps */
/* airpore::Cal_pressure, airpore.cpp:366-398 */
static void airpore_cal_pressure(orc *o)
{
    airm *a = &o->air;
    grid *g = &a->g;
    if (o->scheme == S_FB_V_P) air_cal_fp(a, g->unn, g->vnn, g->wnn, g->pn, o->scheme);
    else if (o->scheme == S_FB_P_V) air_cal_fp(a, g->un, g->vn, g->wn, g->pn, o->scheme);
    if (o->scheme == S_FB_V_P || o->scheme == S_FB_P_V) grid_accumulate_p(g);
    if (o->case_no != 1) return;
    bc_pressure(g, F_NORTH);
    bc_pressure(g, F_EAST);
    bc_pressure(g, F_WEST);
    bc_pressure(g, F_FRONT);
    bc_pressure(g, F_BACK);
    if (o->bc_s == BT_RIGID || o->bc_s == BT_ABSORBING) {
        bc_pressure(g, F_SOUTH);
    } else {
        grid *pg = &o->pore;
        if (o->scheme == S_FB_V_P) pore_cal_fp(pg, pg->unn, pg->vnn, pg->wnn);
        else if (o->scheme == S_FB_P_V) pore_cal_fp(pg, pg->un, pg->vn, pg->wn);
        if (o->scheme == S_FB_V_P || o->scheme == S_FB_P_V) grid_accumulate_p(pg);
        bc_pressure(pg, F_SOUTH);
        bc_pressure(pg, F_EAST);
        bc_pressure(pg, F_WEST);
        bc_pressure(pg, F_FRONT);
        bc_pressure(pg, F_BACK);
        interface_pressure(g, pg);
    }
    air_update_qp(a);
}

/* airpore::Cal_velocity, airpore.cpp:324-364 */
static void airpore_cal_velocity(orc *o)
{
    airm *a = &o->air;
    grid *g = &a->g;
    if (o->scheme == S_FB_V_P) air_cal_fuvw(a, g->un, g->vn, g->wn, g->pn, o->scheme);
    else if (o->scheme == S_FB_P_V) air_cal_fuvw(a, g->un, g->vn, g->wn, g->pnn, o->scheme);
    if (o->scheme == S_FB_V_P || o->scheme == S_FB_P_V) grid_accumulate_v(g);
    if (o->case_no != 1) return;
    if (o->gtdbc) bc_velocity_tdbc_ground(o);
    bc_velocity(g, F_NORTH);
    if (o->bc_e == BT_TDBC) bc_velocity_tdbc_east(g, o->Zinf, o->tau);
    else bc_velocity(g, F_EAST);
    bc_velocity(g, F_WEST);
    bc_velocity(g, F_FRONT);
    bc_velocity(g, F_BACK);
    if (o->bc_s == BT_RIGID || o->bc_s == BT_ABSORBING) {
        bc_velocity(g, F_SOUTH);
    } else {
        grid *pg = &o->pore;
        if (o->scheme == S_FB_V_P) pore_cal_fuvw(pg, pg->un, pg->vn, pg->wn, pg->pn);
        else if (o->scheme == S_FB_P_V) pore_cal_fuvw(pg, pg->un, pg->vn, pg->wn, pg->pnn);
        if (o->scheme == S_FB_V_P || o->scheme == S_FB_P_V) grid_accumulate_v(pg);
        bc_velocity(pg, F_SOUTH);
        bc_velocity(pg, F_EAST);
        bc_velocity(pg, F_WEST);
        bc_velocity(pg, F_FRONT);
        bc_velocity(pg, F_BACK);
        interface_velocity(g, pg);
    }
    air_update_qvw(a);
}

static void airpore_update_initial(orc *o)
{
    grid_update_initial(&o->air.g);
    if (o->has_pore) grid_update_initial(&o->pore);
}

static void airpore_set_moving_frame(orc *o, int MF)
{
    /* airpore::SetMovingFrame, airpore.cpp:881-897 */
    grid_set_moving_frame(&o->air.g, MF);
    if (o->gtdbc && MF != 0) { /* the ground state moves with the frame, like the fields */
        grid *g = &o->air.g;
        const int temp_J = g->mf.JMAX - g->mf.lead_DJ, sh = g->mf.trail_DJ - 1;
        if (temp_J != 0)
            for (int i = 0; i < g->I; i++)
                for (int j = 0; j < g->J; j++) {
                    double *d = &o->gpsi[((size_t)i * g->J + j) * 6];
                    if (j < temp_J + 1 && j + g->mf.lead_DJ - 1 < g->J - 1) {
                        const double *s = &o->gpsi[((size_t)i * g->J + j + sh) * 6];
                        for (int q = 0; q < 6; q++) d[q] = s[q];
                    } else if (j >= temp_J + 1) {
                        for (int q = 0; q < 6; q++) d[q] = 0.0;
                    }
                }
    }
    air_set_wind(&o->air, MF);
    air_set_q_move(&o->air, MF);
    if (o->has_pore) grid_set_moving_frame(&o->pore, MF);
}

/* ---------------------------------------------------------- receivers */
/* calculation_2D::get_position, calculation_2D.cpp:317-352 */
static void get_position(const grid *g, int *ii, int *jj, int *kk, const double *rc)
{
    double Y_frame = g->axY[g->JMAX - 1] - g->axY[0];
    int N = (int)(rc[1] / Y_frame + 1.0e-6);
    for (int i = 0; i < g->IMAX; i++)
        if (rc[0] - g->axX[i] <= g->dx1 / 8.0) { *ii = i; break; }
    int NN = N * (g->JMAX - 1);
    if (NN >= g->IJKMAX) { *ii = 0; *jj = 0; *kk = 0; return; }
    for (int j = NN; j < g->IJKMAX && j - NN < g->JMAX; j++)
        if (rc[1] - N * Y_frame - g->axY[j - NN] <= g->dy1 / 8.0) { *jj = j; break; }
    /* terrain: the heights of the column found */
    for (int k = 0; k < g->KMAX; k++) {
        double zk = g->Zt ? g->Zt[(size_t)*jj * g->K + k] : g->axZ[k];
        if (rc[2] - zk <= g->dz1 / 8.0) { *kk = k; return; }
    }
    *ii = 0; *jj = 0; *kk = 0;
}

/* calculation_2D::get_pressure, calculation_2D.cpp:387-403 */
static double get_pressure(const grid *g, int ii, int jj, int kk, int N)
{
    int sh = N * (g->mf.trail_DJ - 1);
    if (jj >= sh && jj < g->JMAX + sh) {
        int jl = jj - sh;
        if (jl > 0 && jl < g->J - 1 && ii > 0 && ii < g->I - 1 && kk > 0 && kk < g->K - 1)
            return g->pn[IX(g, ii, jl, kk)];
    }
    return 0.0;
}

/* ------------------------------------------------------------ terrain */
/* Terrain-following grid (extension of the reference, which pins the cross
 * metrics to zero, calculation_2D.cpp:102-104): an optional
 * case_dir/terrain.dat holds the count of Y nodes and the ground elevation
 * z_g at each. Air nodes are stretched vertically between the ground and
 * the flat top H = Z[K-1]: Z(j,k) = Z[k] + z_g(j) (1 - Z[k] / H), which is
 * exactly Z[k] where z_g = 0; porous nodes follow the ground: Z(j,k) =
 * Z[k] + z_g(j). The PML profiles stay on the file axes. */
static int terrain_grid(grid *g, const double *zg, int porous, char *err, int errlen)
{
    const int K = g->K;
    if (porous ? (K < 3 || g->axZ[K - 2] != 0.0) : (g->axZ[0] != 0.0)) {
        seterr(err, errlen, "terrain needs the air axis to start at Z = 0 and the porous axis to end one node above 0");
        return -1;
    }
    const double H = g->axZ[K - 1];
    g->zg = zalloc(g->J);
    g->Zt = zalloc((size_t)g->J * K);
    g->Zz2 = zalloc((size_t)g->J * K);
    g->Zy2 = zalloc((size_t)g->J * K);
    for (int j = 0; j < g->J; j++) {
        g->zg[j] = zg[j];
        if (!porous && !(zg[j] < H)) { seterr(err, errlen, "terrain reaches the top of the air grid"); return -1; }
        for (int k = 0; k < K; k++)
            g->Zt[(size_t)j * K + k] = porous ? g->axZ[k] + zg[j] : g->axZ[k] + zg[j] * (1.0 - g->axZ[k] / H);
    }
    return 0;
}

static int terrain_setup(orc *o, const char *dir, char *err, int errlen)
{
    char path[4096];
    snprintf(path, sizeof path, "%s/terrain.dat", dir);
    size_t n = 0;
    char *t = slurp(path, &n);
    if (!t) return 0; /* flat ground */
    rdr R = {t, n, 0, 0};
    grid *g = &o->air.g;
    int cnt = rd_i(&R);
    if (R.fail || cnt != g->JMAX || o->mf.Judge == 1 || o->cjudge != 0) {
        free(t);
        seterr(err, errlen, "terrain.dat must hold one elevation per Y node, without moving frame or inclusions");
        return -1;
    }
    double *zg = zalloc(cnt);
    for (int j = 0; j < cnt; j++) zg[j] = rd_d(&R);
    int fail = R.fail;
    free(t);
    if (fail) { free(zg); seterr(err, errlen, "malformed terrain.dat"); return -1; }
    int rc = terrain_grid(g, zg, 0, err, errlen);
    free(zg);
    return rc;
}

/* ------------------------------------------------------------- public */
orc *orc_create(const char *case_dir, char *err, int errlen)
{
    orc *o = (orc *)calloc(1, sizeof(orc));
    if (parse_input(o, case_dir, err, errlen) != 0) { free(o); return NULL; }
    if (o->mf.lead_DJ < 2) { seterr(err, errlen, "moving-frame lead_DJ must be >= 2"); free(o); return NULL; }
    airm *a = &o->air;
    if (grid_init(&a->g, case_dir, "coordi_air", o->dt, o->dx, o->dy, o->dz, o->mf, o->gauss_width, 0, err,
                  errlen) != 0) {
        free(o);
        return NULL;
    }
    if (terrain_setup(o, case_dir, err, errlen) != 0) {
        orc_destroy(o);
        return NULL;
    }
    a->gamma = o->gamma; a->P0 = o->P0; a->Aav = o->Aav; a->c0 = o->c0;
    a->vmethod = o->vmethod; a->vb = o->vcoef; a->vc = o->c0; a->valpha = 1.256431;
    a->vkappa = 0.41; a->vz0 = 0.01;
    { /* optional case_dir/advection.dat: "upwind" or "reference" */
        char path[4096];
        snprintf(path, sizeof path, "%s/advection.dat", case_dir);
        size_t n = 0;
        char *t = slurp(path, &n);
        if (t) {
            a->upwind = strncmp(t, "upwind", 6) == 0;
            int ok = a->upwind || strncmp(t, "reference", 9) == 0;
            free(t);
            if (!ok) { seterr(err, errlen, "advection.dat must hold 'upwind' or 'reference'"); orc_destroy(o); return NULL; }
        }
    }
    if (o->vmethod == 7) { /* optional case_dir/logwind.dat: kappa z0 */
        char path[4096];
        snprintf(path, sizeof path, "%s/logwind.dat", case_dir);
        size_t n = 0;
        char *t = slurp(path, &n);
        if (t) {
            rdr R = {t, n, 0, 0};
            a->vkappa = rd_d(&R); a->vz0 = rd_d(&R);
            int bad = R.fail || !(a->vkappa > 0) || !(a->vz0 > 0);
            free(t);
            if (bad) { seterr(err, errlen, "logwind.dat must hold kappa > 0 and z0 > 0"); orc_destroy(o); return NULL; }
        }
    }
    { /* optional case_dir/tdbc_ground.dat: Zinf tau a0..a5 r0..r5 */
        char path[4096];
        snprintf(path, sizeof path, "%s/tdbc_ground.dat", case_dir);
        size_t n = 0;
        char *t = slurp(path, &n);
        if (t) {
            rdr R = {t, n, 0, 0};
            o->gZ = rd_d(&R); o->gtau = rd_d(&R);
            int bad = 0;
            for (int q = 0; q < 6; q++) { o->ga[q] = rd_d(&R); bad |= !(o->ga[q] >= 0); }
            for (int q = 0; q < 6; q++) { o->gr[q] = rd_d(&R); bad |= !(o->gr[q] >= 0); }
            bad |= R.fail || !(o->gZ > 0) || !(o->gtau > 0);
            free(t);
            if (bad) {
                seterr(err, errlen, "tdbc_ground.dat must hold Zinf > 0, tau > 0, six a >= 0 and six r >= 0");
                orc_destroy(o);
                return NULL;
            }
            if (o->case_no != 1 || o->bc_s != BT_RIGID || o->scheme != S_FB_P_V || a->g.zg || a->g.K < 3) {
                seterr(err, errlen, "the impedance ground needs a rigid south face, scheme FB_p_v and no terrain");
                orc_destroy(o);
                return NULL;
            }
            o->gtdbc = 1;
            o->gpsi = zalloc((size_t)a->g.I * a->g.J * 6);
        }
    }
    size_t N = (size_t)a->g.I * a->g.J * a->g.K;
    a->Uav = zalloc(N); a->Vav = zalloc(N); a->Wav = zalloc(N);
    air_pml_setup(o);
    air_hill_setup(o);
    grid_set_initial(&a->g, o->src, 1);
    o->has_pore = (o->case_no == 1 && o->bc_s == BT_POROUS);
    if (o->has_pore) {
        grid *pg = &o->pore;
        if (grid_init(pg, case_dir, "coordi_pore", o->dt, o->pdx, o->pdy, o->pdz, o->mf, o->gauss_width, 1, err,
                      errlen) != 0) {
            orc_destroy(o);
            return NULL;
        }
        if (pg->I != a->g.I || pg->J != a->g.J) {
            seterr(err, errlen, "porous grid must share the air grid's I and J node counts");
            orc_destroy(o);
            return NULL;
        }
        if (o->air.g.zg && terrain_grid(pg, o->air.g.zg, 1, err, errlen) != 0) {
            orc_destroy(o);
            return NULL;
        }
        pg->eff = 1.0 / o->peff;
        pg->Beta = o->psig * pg->dt * pg->eff;
        pg->Gama = pg->dt / o->pKp / o->pporo;
        pg->invBeta = 1.0 / (pg->Beta + 1.0);
        grid_set_initial(pg, o->src, 1);
    }
    return o;
}

void orc_destroy(orc *o)
{
    if (!o) return;
    grid_free(&o->air.g);
    free(o->air.Uav); free(o->air.Vav); free(o->air.Wav);
    for (int s = 0; s < 6; ++s)
        for (int c = 0; c < 4; ++c) free(o->air.s[s].q[c]);
    free(o->air.cr_uc);
    if (o->has_pore) grid_free(&o->pore);
    free(o->ri); free(o->rj); free(o->rk);
    free(o->gpsi);
    free(o);
}

int orc_dims(const orc *o, int *d)
{
    int ns = 0;
    for (int s = 0; s < 6; ++s) ns += o->air.s[s].n0 ? 1 : 0;
    d[0] = o->air.g.I; d[1] = o->air.g.J; d[2] = o->air.g.K;
    d[3] = o->has_pore;
    d[4] = o->has_pore ? o->pore.I : 0; d[5] = o->has_pore ? o->pore.J : 0; d[6] = o->has_pore ? o->pore.K : 0;
    d[7] = o->time_domain; d[8] = o->scheme; d[9] = ns;
    return 0;
}

int orc_set_receivers(orc *o, int n, const double *xyz, int *idx_out)
{
    free(o->ri); free(o->rj); free(o->rk);
    o->nrec = n;
    o->ri = (int *)calloc((size_t)(n ? n : 1), sizeof(int));
    o->rj = (int *)calloc((size_t)(n ? n : 1), sizeof(int));
    o->rk = (int *)calloc((size_t)(n ? n : 1), sizeof(int));
    const grid *g = &o->air.g;
    for (int r = 0; r < n; ++r) { /* airpore.cpp:454-457 */
        int ii = 0, jj = 0, kk = 0;
        get_position(g, &ii, &jj, &kk, xyz + 3 * r);
        if (ii == 0 && jj == 0 && kk == 0) { ii = 1; jj = 1; kk = 1; }
        if (ii > g->IMAX || jj > g->IJKMAX || kk > g->KMAX) { ii = 1; jj = 1; kk = 1; }
        o->ri[r] = ii; o->rj[r] = jj; o->rk[r] = kk;
        if (idx_out) { idx_out[3 * r] = ii; idx_out[3 * r + 1] = jj; idx_out[3 * r + 2] = kk; }
    }
    return 0;
}

/* airpore::get_output loop, airpore.cpp:539-624 */
int orc_run(orc *o, int nsteps, double *rec_out)
{
    if (o->case_no != 1) return -2;
    if (o->scheme != S_FB_P_V && o->scheme != S_FB_V_P) return -3;
    const grid *g = &o->air.g;
    const mframe mf = o->mf;
    const int JMAX = g->IJKMAX, time_domain = nsteps;
    const double dy = o->dy, dt = o->dt, c0 = o->c0;
    int MF_count = 0, temp_time = 0, index = 0, MF_limit = 0;
    do {
        if (MF_count == (int)((JMAX - mf.JMAX) / (mf.lead_DJ - 1) + 1.e-6) || (JMAX == mf.JMAX)) {
            MF_limit = time_domain - temp_time;
        } else if (MF_count == 0) {
            MF_limit = (int)((mf.JMAX - 1) * dy / c0 / dt * mf.ratio);
        } else {
            MF_limit = (int)((mf.trail_DJ - 1) * dy / c0 / dt);
            double lt1 = 0.0, lt2 = 0.0;
            if (MF_count % 10 == 0) {
                lt1 = (mf.trail_DJ - 1) * dy / c0 / dt - MF_limit;
                lt1 = lt1 * 10.0;
            }
            if (MF_count % 100 == 0) {
                lt2 = (mf.trail_DJ - 1) * dy / c0 / dt - MF_limit;
                lt2 = lt2 * 100 - (int)(lt2 * 10) * 10;
            }
            MF_limit = MF_limit + (int)lt1 + (int)lt2;
            if ((temp_time + MF_limit) > time_domain) MF_limit = time_domain - temp_time;
        }
        airpore_set_moving_frame(o, MF_count);
        /* The reference runs frame 0 for its full MF_limit even when
         * time_domain is shorter, writing receiver samples past its buffer
         * (airpore.cpp:545,566-578); the restatement stops at time_domain. */
        for (int n = 0; n < MF_limit && index < time_domain; n++) {
            index = index + 1;
            for (int r = 0; r < o->nrec; ++r) {
                double t = get_pressure(&o->air.g, o->ri[r], o->rj[r], o->rk[r], MF_count);
                if (fabs(t) < 1.0e-100) t = 0.0;
                if (rec_out) rec_out[(size_t)(index - 1) * o->nrec + r] = t;
            }
            if (o->scheme == S_FB_P_V) {
                airpore_cal_pressure(o);
                airpore_cal_velocity(o);
            } else {
                airpore_cal_velocity(o);
                airpore_cal_pressure(o);
            }
            airpore_update_initial(o);
        }
        MF_count = MF_count + 1;
        temp_time = MF_limit + temp_time;
    } while ((MF_count <= (int)((JMAX - mf.JMAX) / (mf.lead_DJ - 1) + 1.e-6)) && (temp_time < time_domain) &&
             mf.Judge == 1);
    return index;
}

static const grid *medium(const orc *o, int m) { return m == 0 ? &o->air.g : (o->has_pore ? &o->pore : NULL); }

int orc_get_field(const orc *o, int m, int comp, double *out)
{
    const grid *g = medium(o, m);
    if (!g) return -1;
    const double *src = comp == 0 ? g->pn : comp == 1 ? g->un : comp == 2 ? g->vn : g->wn;
    memcpy(out, src, sizeof(double) * g->I * g->J * g->K);
    return 0;
}

int orc_set_field(orc *o, int m, int comp, const double *in)
{
    grid *g = (grid *)medium(o, m);
    if (!g) return -1;
    double *dst = comp == 0 ? g->pn : comp == 1 ? g->un : comp == 2 ? g->vn : g->wn;
    memcpy(dst, in, sizeof(double) * g->I * g->J * g->K);
    return 0;
}

int orc_get_psi(const orc *o, double *out)
{
    memcpy(out, o->air.g.psi, sizeof(double) * o->air.g.I * o->air.g.K * 6);
    return 0;
}

int orc_get_ground_psi(const orc *o, double *out)
{
    if (!o->gtdbc) return -1;
    memcpy(out, o->gpsi, sizeof(double) * o->air.g.I * o->air.g.J * 6);
    return 0;
}

int orc_get_slab(const orc *o, int sid, int comp, double *out, int *dims)
{
    const slab *s = &o->air.s[sid];
    if (!s->n0) { dims[0] = dims[1] = dims[2] = 0; return 0; }
    dims[0] = s->n0; dims[1] = s->n1; dims[2] = s->n2;
    if (out) memcpy(out, s->q[comp], sizeof(double) * s->n0 * s->n1 * s->n2);
    return 1;
}

int orc_get_wind(const orc *o, int comp, double *out)
{
    const double *src = comp == 0 ? o->air.Uav : comp == 1 ? o->air.Vav : o->air.Wav;
    memcpy(out, src, sizeof(double) * o->air.g.I * o->air.g.J * o->air.g.K);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Post-processing: the reference's in-place radix-2 FFT (FFT.cpp:15-83),
 * used by airpore::get_FFT_y1 (airpore.cpp:966-1011) on zero-padded
 * receiver traces.  Restated step for step so that, without FMA
 * contraction, the result matches the compiled reference bit for bit:
 *   1. bit-reversal permutation of the 2^m points;
 *   2. m butterfly stages; within a stage the twiddle factor starts at 1
 *      and is advanced by complex multiplication with the stage root, and
 *      the next stage's root follows from the half-angle formulas
 *      (cos -> sqrt((1+cos)/2), sin -> -+sqrt((1-cos)/2));
 *   3. the forward transform (dir = 1) divides by the point count. */
void orc_fft(int dir, int m, double *re, double *im) {
    long n = 1;
    for (int s = 0; s < m; ++s) n *= 2;
    /* 1. bit reversal: walk j through the reversed counter */
    long j = 0;
    for (long i = 0; i < n - 1; ++i) {
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
        long bit = n >> 1;
        while (bit <= j) { j -= bit; bit >>= 1; }
        j += bit;
    }
    /* 2. butterflies */
    double root_c = -1.0, root_s = 0.0;
    long half = 1;
    for (int s = 0; s < m; ++s) {
        const long span = half * 2;
        double wc = 1.0, ws = 0.0;
        for (long a = 0; a < half; ++a) {
            for (long i = a; i < n; i += span) {
                const long b = i + half;
                const double tr = wc * re[b] - ws * im[b];
                const double ti = wc * im[b] + ws * re[b];
                re[b] = re[i] - tr;
                im[b] = im[i] - ti;
                re[i] += tr;
                im[i] += ti;
            }
            const double next_c = wc * root_c - ws * root_s;
            ws = wc * root_s + ws * root_c;
            wc = next_c;
        }
        root_s = sqrt((1.0 - root_c) / 2.0);
        if (dir == 1) root_s = -root_s;
        root_c = sqrt((1.0 + root_c) / 2.0);
        half = span;
    }
    /* 3. forward scaling */
    if (dir == 1)
        for (long i = 0; i < n; ++i) { re[i] /= n; im[i] /= n; }
}
