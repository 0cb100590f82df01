/* ORACLE / TEST INFRASTRUCTURE ONLY -- see cfd_oracle.h.
 *
 * Restatement of the reference path, line by line in the reference's operation
 * order (compile with -ffp-contract=off, no FMA):
 *   line sweep          zone_FD/src/src/sp_distributor.cpp:3-79
 *   face list           zone_FD/src/include/reconstructor5order.hpp:56-125
 *   char. reconstruction reconstructor5order.hpp:233-323 (1D), 326-429 (2D)
 *   eigensystems        zone_FD/src/src/eigenSystem.cpp:13-213 (2D), 217-323 (1D)
 *   interpolators       zone_FD/src/include/interScheme.hpp:17-45, 85-114, 384-452, 494-584, 1386-1406
 *   Riemann fluxes      zone_FD/src/include/fluxSchemes.hpp:13-71, 74-125, 202-327, 420-553
 *   node fluxes         fluxSchemes.hpp:572-599, solvePointFlux.hpp:33-100
 *   MND6                zone_FD/src/src/differ.cpp:54-103
 *   TRAD6               zone_FD/src/src/differ.cpp:23-52 (ghosts: info.cpp:7-22)
 *   cons -> prim        zone_FD/src/src/equation.cpp:37-93
 *   boundaries          zone_FD/src/src/oneDBnd.cpp:31-114
 *   RK3 and CFL step    zone_FD/src/src/blockSolver.cpp:43-87, 318-349
 * 3D extends the 2D formulas by w and a second shear wave (no reference path).
 */
#include "cfd_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#define G 1.4
#define MAXV 5

static int nvar_of(int dim) { return dim + 2; }

/* ------------------------------------------------------------ interpolators */
static void betas(const double *q, double *b)
{
    b[0] = 1.0 / 1.0 * ((1.0 * q[0] - 2.0 * q[1] + 1.0 * q[2]) * (1.0 * q[0] - 2.0 * q[1] + 1.0 * q[2])) +
           1.0 / 4.0 * ((1.0 * q[0] - 4.0 * q[1] + 3.0 * q[2]) * (1.0 * q[0] - 4.0 * q[1] + 3.0 * q[2]));
    b[1] = 1.0 / 1.0 * ((1.0 * q[1] - 2.0 * q[2] + 1.0 * q[3]) * (1.0 * q[1] - 2.0 * q[2] + 1.0 * q[3])) +
           1.0 / 4.0 * ((1.0 * q[1] + 0.0 * q[2] - 1.0 * q[3]) * (1.0 * q[1] + 0.0 * q[2] - 1.0 * q[3]));
    b[2] = 1.0 / 1.0 * ((1.0 * q[2] - 2.0 * q[3] + 1.0 * q[4]) * (1.0 * q[2] - 2.0 * q[3] + 1.0 * q[4])) +
           1.0 / 4.0 * ((3.0 * q[2] - 4.0 * q[3] + 1.0 * q[4]) * (3.0 * q[2] - 4.0 * q[3] + 1.0 * q[4]));
}

static double teno_stencil(unsigned flag, const double *q)
{
    switch (flag) {
    case 0: return 3.0 / 128.0 * q[0] - 5.0 / 32.0 * q[1] + 45.0 / 64.0 * q[2] + 15.0 / 32.0 * q[3] - 5.0 / 128.0 * q[4];
    case 1: return -1.0 / 16.0 * q[1] + 9.0 / 16.0 * q[2] + 9.0 / 16.0 * q[3] - 1.0 / 16.0 * q[4];
    case 2: case 3: return 3.0 / 8.0 * q[2] + 3.0 / 4.0 * q[3] - 1.0 / 8.0 * q[4];
    case 4: return 1.0 / 16.0 * q[0] - 5.0 / 16.0 * q[1] + 15.0 / 16.0 * q[2] + 5.0 / 16.0 * q[3];
    case 5: return -1.0 / 8.0 * q[1] + 3.0 / 4.0 * q[2] + 3.0 / 8.0 * q[3];
    case 6: return 3.0 / 8.0 * q[0] - 5.0 / 4.0 * q[1] + 15.0 / 8.0 * q[2];
    default: return q[2];
    }
}

double orc_inter5(int fam, double icst, const double *q)
{
    double b[3], u[3];
    if (fam == ORC_MUSCL) {
        double dm = q[2] - q[1], dp = q[3] - q[2], d, beta = 1.0, a1, a2, m;
        if (dp > 0) {
            a1 = (dp < beta * dm) ? dp : beta * dm;           /* std::min(beta*dm, dp) */
            a2 = ((beta * dp) < dm) ? beta * dp : dm;         /* std::min(dm, beta*dp) */
            m = (a1 < a2) ? a2 : a1;                          /* std::max */
            d = (0.0 < m) ? m : 0.0;
        } else {
            a1 = (beta * dm < dp) ? dp : beta * dm;           /* std::max(beta*dm, dp) */
            a2 = (dm < beta * dp) ? beta * dp : dm;           /* std::max(dm, beta*dp) */
            m = (a2 < a1) ? a2 : a1;                          /* std::min */
            d = (m < 0.0) ? m : 0.0;
        }
        return q[2] + d * 0.5;
    }
    betas(q, b);
    if (fam == ORC_WCNS5 || fam == ORC_WENOZ) {
        const double gam[3] = {1.0 / 16.0, 5.0 / 8.0, 5.0 / 16.0};
        u[0] = 3.0 / 8.0 * q[0] - 5.0 / 4.0 * q[1] + 15.0 / 8.0 * q[2];
        u[1] = -1.0 / 8.0 * q[1] + 3.0 / 4.0 * q[2] + 3.0 / 8.0 * q[3];
        u[2] = 3.0 / 8.0 * q[2] + 3.0 / 4.0 * q[3] - 1.0 / 8.0 * q[4];
        double sb = 0, res = 0, tau = fabs(b[2] - b[0]);
        for (int i = 0; i < 3; i++) {
            if (fam == ORC_WCNS5) {
                double s = 1e-6 + b[i];
                b[i] = gam[i] / (s * s);
            } else {
                double x = tau / (b[i] + 1e-40);
                b[i] = gam[i] * (1.0 + x * x);
            }
            sb += b[i];
        }
        for (int i = 0; i < 3; i++) res += b[i] * u[i];
        return res / sb;
    }
    if (fam == ORC_TENOZ) {
        double sb = 0, tau = fabs(b[2] - b[0]);
        for (int i = 0; i < 3; i++) {
            double t = 1.0 + tau / (b[i] + 1e-40);
            t *= t;
            b[i] = t * t * t;
            sb += b[i];
        }
        double ct = icst * sb;
        unsigned f = 0;
        if (b[0] < ct) f += 1;
        if (b[1] < ct) f += 2;
        if (b[2] < ct) f += 4;
        return teno_stencil(f, q);
    }
    /* ORC_TENOCONG */
    int mi = 0;
    for (int i = 1; i < 3; i++)
        if (b[i] < b[mi]) mi = i;
    double CT = icst, CT_1 = 1.0 - icst, tau = fabs(b[2] - b[0]);
    double rr = CT * tau - CT_1 * b[mi], ll = tau * b[mi];
    unsigned f = 0;
    if (ll < rr * b[0]) f += 1;
    if (ll < rr * b[1]) f += 2;
    if (ll < rr * b[2]) f += 4;
    return teno_stencil(f, q);
}

/* ------------------------------------------------------------ state algebra */
static void c2p(int nv, const double *c, double *p)
{
    if (nv == 3) {
        double r = c[0], u = c[1] / r, E = c[2] / r;
        double e = -u * u / 2 + E;
        p[0] = r; p[1] = u; p[2] = r * ((G - 1) * e);
    } else if (nv == 4) {
        double r = c[0], u = c[1] / r, v = c[2] / r, E = c[3] / r;
        double q2 = (u * u + v * v) / 2, e = -q2 + E;
        p[0] = r; p[1] = u; p[2] = v; p[3] = r * ((G - 1) * e);
    } else {
        double r = c[0], u = c[1] / r, v = c[2] / r, w = c[3] / r, E = c[4] / r;
        double q2 = (u * u + v * v + w * w) / 2, e = -q2 + E;
        p[0] = r; p[1] = u; p[2] = v; p[3] = w; p[4] = r * ((G - 1) * e);
    }
}

static void p2c(int nv, const double *p, double *c)
{
    double ek;
    if (nv == 3) ek = (p[1] * p[1]) / 2;
    else if (nv == 4) ek = (p[1] * p[1] + p[2] * p[2]) / 2;
    else ek = (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]) / 2;
    c[0] = p[0];
    for (int i = 1; i < nv - 1; i++) c[i] = p[0] * p[i];
    c[nv - 1] = p[nv - 1] / (G - 1) + p[0] * ek;
}

/* ------------------------------------------------------------ eigensystem */
typedef struct { double L[MAXV][MAXV], R[MAXV][MAXV]; } eig_t;

static void eig_build(int nv, int ax, const double *pl, const double *pr, eig_t *e)
{
    memset(e, 0, sizeof(*e));
    if (nv == 3) {
        double rl = pl[0], ul = pl[1], Pl = pl[2], rr = pr[0], ur = pr[1], Pr = pr[2];
        double HL = (ul * ul) / 2 + Pl / rl * G / (G - 1), HR = (ur * ur) / 2 + Pr / rr * G / (G - 1);
        double c1 = sqrt(rl), c2 = sqrt(rr), dv = 1.0 / (sqrt(rl) + sqrt(rr));
        double u = (c1 * ul + c2 * ur) * dv, ht = (c1 * HL + c2 * HR) * dv;
        double ek = (u * u) / 2, h = ht - ek, c = sqrt((G - 1) * h), g1 = G - 1;
        double le[9] = {ht + c * (u - c) / g1, -u - c / g1, 1.0, -2.0 * ht + 4.0 * c * c / g1, 2.0 * u, -2.0,
                        ht - c * (u + c) / g1, -u + c / g1, 1.0};
        double f = 0.5 * g1 / (c * c);
        double re[9] = {1.0, 1.0, 1.0, u - c, u, u + c, ht - u * c, 0.5 * u * u, ht + u * c};
        for (int i = 0; i < 9; i++) {
            e->L[i / 3][i % 3] = le[i] * f;
            e->R[i / 3][i % 3] = re[i];
        }
        return;
    }
    int D = nv - 2, E = nv - 1;
    double n[3] = {ax == 0, ax == 1, ax == 2};
    double rl = pl[0], rr = pr[0], Pl = pl[E], Pr = pr[E];
    double kl = 0, kr = 0;
    if (D == 2) { kl = pl[1] * pl[1] + pl[2] * pl[2]; kr = pr[1] * pr[1] + pr[2] * pr[2]; }
    else { kl = pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]; kr = pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]; }
    double HL = kl / 2 + Pl / rl * G / (G - 1), HR = kr / 2 + Pr / rr * G / (G - 1);
    double c1 = sqrt(rl), c2 = sqrt(rr), dv = 1.0 / (c1 + c2);
    double vel[3] = {0, 0, 0};
    for (int i = 0; i < D; i++) vel[i] = (c1 * pl[1 + i] + c2 * pr[1 + i]) * dv;
    double ht = (c1 * HL + c2 * HR) * dv;
    double u = vel[0], v = vel[1], w = vel[2], Vn, ek;
    if (D == 2) { Vn = n[0] * u + n[1] * v; ek = (u * u + v * v) / 2; }
    else { Vn = n[0] * u + n[1] * v + n[2] * w; ek = (u * u + v * v + w * w) / 2; }
    double h = ht - ek, c = sqrt((G - 1) * h);
    /* left rows: shear t1, entropy, acoustic -, acoustic +, [shear t2] */
    if (ax != 2) { e->L[0][0] = (-n[1] * u + n[0] * v); e->L[0][1] = n[1]; e->L[0][2] = (-n[0]); }
    else { e->L[0][0] = -u; e->L[0][1] = 1.0; e->L[0][2] = 0.0; }
    e->L[1][0] = h - ek;
    for (int i = 0; i < D; i++) e->L[1][1 + i] = vel[i];
    e->L[1][E] = -1.0;
    e->L[2][0] = (Vn / c + ek / h) / 2;
    e->L[3][0] = (-Vn / c + ek / h) / 2;
    for (int i = 0; i < D; i++) {
        e->L[2][1 + i] = (-n[i] / c - vel[i] / h) / 2;
        e->L[3][1 + i] = (n[i] / c - vel[i] / h) / 2;
    }
    e->L[2][E] = 1.0 / (2.0 * h);
    e->L[3][E] = 1.0 / (2.0 * h);
    if (D == 3) {
        if (ax != 2) { e->L[4][0] = -w; e->L[4][3] = 1.0; }
        else { e->L[4][0] = -v; e->L[4][2] = 1.0; }
    }
    if (ax != 2) { e->R[1][0] = n[1]; e->R[2][0] = -n[0]; e->R[E][0] = n[1] * u - n[0] * v; }
    else { e->R[1][0] = 1.0; e->R[E][0] = u; }
    e->R[0][1] = 1.0 / h;
    for (int i = 0; i < D; i++) e->R[1 + i][1] = vel[i] / h;
    e->R[E][1] = ek / h;
    e->R[0][2] = 1; e->R[0][3] = 1;
    for (int i = 0; i < D; i++) {
        e->R[1 + i][2] = vel[i] - n[i] * c;
        e->R[1 + i][3] = vel[i] + n[i] * c;
    }
    e->R[E][2] = h + ek - Vn * c;
    e->R[E][3] = h + ek + Vn * c;
    if (D == 3) {
        if (ax != 2) { e->R[3][4] = 1.0; e->R[4][4] = w; }
        else { e->R[2][4] = 1.0; e->R[4][4] = v; }
    }
}

static double eig_project(int nv, const eig_t *e, int k, const double *cs)
{
    if (nv == 3) return cs[0] * e->L[k][0] + cs[1] * e->L[k][1] + cs[2] * e->L[k][2];
    if (nv == 4) return cs[1] * e->L[k][1] + cs[2] * e->L[k][2] + cs[3] * e->L[k][3] + cs[0] * e->L[k][0];
    return cs[1] * e->L[k][1] + cs[2] * e->L[k][2] + cs[3] * e->L[k][3] + cs[4] * e->L[k][4] + cs[0] * e->L[k][0];
}

static void eig_back(int nv, const eig_t *e, const double *ch, double *cs)
{
    for (int i = 0; i < nv; i++) {
        if (nv == 3) cs[i] = ch[0] * e->R[i][0] + ch[1] * e->R[i][1] + ch[2] * e->R[i][2];
        else if (nv == 4) cs[i] = ch[2] * e->R[i][2] + ch[3] * e->R[i][3] + ch[1] * e->R[i][1] + ch[0] * e->R[i][0];
        else cs[i] = ch[2] * e->R[i][2] + ch[3] * e->R[i][3] + ch[1] * e->R[i][1] + ch[0] * e->R[i][0] + ch[4] * e->R[i][4];
    }
}

static void back_to_prim(int nv, const double *cs, double *p)
{
    if (nv == 3) {
        double ut = cs[1] / cs[0], ekt = (ut * ut) / 2;
        p[0] = cs[0]; p[1] = ut; p[2] = (G - 1) * (cs[2] - cs[0] * ekt);
        return;
    }
    double rt = cs[0], s = 0;
    for (int i = 1; i < nv - 1; i++) {
        p[i] = cs[i] / rt;
        s = (i == 1) ? cs[i] * cs[i] : s + cs[i] * cs[i];
    }
    p[0] = rt;
    p[nv - 1] = (G - 1) * (cs[nv - 1] - s / rt / 2);
}

static double pos_q(int which, const double *W)
{
    if (which == 0) return W[0];
    double u = W[1] / W[0], ekin = 0.5 * u * u;
    return G * ((G - 1) * (W[2] - W[0] * ekin));
}

static void pos_limit(int which, const double *W, double *Wi)
{
    double qi = pos_q(which, Wi);
    if (qi >= 1e-10) return;
    double q = pos_q(which, W);
    if (q < 1e-10) { for (int i = 0; i < 3; i++) Wi[i] = W[i]; return; }
    double th = (1e-10 - q) / (qi - q);
    for (int i = 0; i < 3; i++) Wi[i] = (1 - th) * W[i] + th * Wi[i];
}

/* The positivity option on a 2D/3D cons state (the library's
   positive_quantity_md / positive_limit_md): gamma p with
   p = (gamma - 1) (rho E - rho |u|^2 / 2), |u|^2 summed by component. */
static double pos_q_md(int nv, int which, const double *W)
{
    if (which == 0) return W[0];
    double rho = W[0], q2 = 0.0;
    for (int i = 1; i < nv - 1; i++) {
        double u = W[i] / rho;
        q2 = q2 + u * u;
    }
    double ekin = 0.5 * q2;
    double p = (G - 1) * (W[nv - 1] - rho * ekin);
    return G * p;
}

static void pos_limit_md(int nv, int which, const double *W, double *Wi)
{
    double qi = pos_q_md(nv, which, Wi);
    if (qi >= 1e-10) return;
    double q = pos_q_md(nv, which, W);
    if (q < 1e-10) { for (int i = 0; i < nv; i++) Wi[i] = W[i]; return; }
    double th = (1e-10 - q) / (qi - q);
    for (int i = 0; i < nv; i++) Wi[i] = (1 - th) * W[i] + th * Wi[i];
}

/* reconI for the face between stencil cells 2 and 3 */
static void recon_face(const orc_cfg *c, int ax, double (*P)[MAXV], double *fl, double *fr)
{
    int nv = nvar_of(c->dim);
    eig_t e;
    eig_build(nv, ax, P[2], P[3], &e);
    double cs[6][MAXV], QL[MAXV], QR[MAXV];
    for (int j = 0; j < 6; j++) p2c(nv, P[j], cs[j]);
    for (int k = 0; k < nv; k++) {
        double q[6], qr[5];
        for (int j = 0; j < 6; j++) q[j] = eig_project(nv, &e, k, cs[j]);
        QL[k] = orc_inter5(c->fam, c->icst, q);
        for (int j = 0; j < 5; j++) qr[j] = q[5 - j];
        QR[k] = orc_inter5(c->fam, c->icst, qr);
    }
    double cl[MAXV], cr[MAXV];
    eig_back(nv, &e, QL, cl);
    eig_back(nv, &e, QR, cr);
    if (nv == 3) {
        double WL[3], WR[3];
        p2c(3, P[2], WL);
        p2c(3, P[3], WR);
        pos_limit(0, WL, cl); pos_limit(0, WR, cr);
        pos_limit(1, WL, cl); pos_limit(1, WR, cr);
        back_to_prim(3, cl, fl);
        back_to_prim(3, cr, fr);
        return;
    }
    if (c->posl) {
        /* the 1D limiter (positive_preserving.hpp:13-46, reconstructor5order.hpp:225-236)
           on the 2D/3D cons: rho of both states, then gamma p of both */
        double WL[MAXV], WR[MAXV];
        p2c(nv, P[2], WL);
        p2c(nv, P[3], WR);
        pos_limit_md(nv, 0, WL, cl); pos_limit_md(nv, 0, WR, cr);
        pos_limit_md(nv, 1, WL, cl); pos_limit_md(nv, 1, WR, cr);
        back_to_prim(nv, cl, fl);
        back_to_prim(nv, cr, fr);
        return;
    }
    back_to_prim(nv, cl, fl);
    back_to_prim(nv, cr, fr);
    if (fl[0] < 0 || fl[nv - 1] < 0) memcpy(fl, P[2], sizeof(double) * nv);
    if (fr[0] < 0 || fr[nv - 1] < 0) {
        fr[0] = P[3][0];
        for (int i = 1; i < nv - 1; i++) fr[i] = P[2][i];
        fr[nv - 1] = P[3][nv - 1];
    }
}

/* ------------------------------------------------------------ fluxes */
static void phys_flux(int nv, int ax, const double *p, double *f)
{
    if (nv == 3) {
        f[0] = p[0] * p[1];
        f[1] = p[0] * p[1] * p[1] + p[2];
        f[2] = (G / (G - 1) * p[2] + p[0] * (p[1] * p[1]) / 2) * p[1];
        return;
    }
    int D = nv - 2, E = nv - 1;
    double n[3] = {ax == 0, ax == 1, ax == 2};
    double Vn = (D == 2) ? (p[1] * n[0] + p[2] * n[1]) : (p[1] * n[0] + p[2] * n[1] + p[3] * n[2]);
    double q2 = (D == 2) ? (p[1] * p[1] + p[2] * p[2]) : (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
    f[0] = p[0] * Vn;
    for (int i = 0; i < D; i++) f[1 + i] = p[0] * p[1 + i] * Vn + n[i] * p[E];
    f[E] = (q2 / 2 * p[0] + G / (G - 1) * p[E]) * Vn;
}

static void hllc1(const double *L, const double *R, double *res)
{
    double rl = L[0], ul = L[1], pl = L[2], rr = R[0], ur = R[1], pr = R[2];
    double HL = pl / rl * G / (G - 1) + (ul * ul) / 2, HR = pr / rr * G / (G - 1) + (ur * ur) / 2;
    double cl = sqrt(G * (pl / rl)), cr = sqrt(G * (pr / rr));
    double SL = ((ul - cl) < (ur - cr)) ? (ul - cl) : (ur - cr);
    double SR = ((ul + cl) < (ur + cr)) ? (ur + cr) : (ul + cl);
    double Ss = ((pr - pl) + (rl * ul * (SL - ul) - rr * ur * (SR - ur))) / (rl * (SL - ul) - rr * (SR - ur));
    if (SL >= 0) { res[0] = rl * ul; res[1] = rl * ul * ul + pl; res[2] = rl * HL * ul; }
    else if (Ss >= 0) {
        double ps = pl + rl * (SL - ul) * (Ss - ul);
        double U[3] = {rl, rl * ul, pl / (G - 1) + rl * ul * ul / 2}, F[3] = {rl * ul, rl * ul * ul + pl, rl * HL * ul};
        double Dd[3] = {0, 1, Ss};
        for (int i = 0; i < 3; i++) res[i] = (Ss * (SL * U[i] - F[i]) + SL * ps * Dd[i]) / (SL - Ss);
    } else if (SR >= 0) {
        double ps = pr + rr * (SR - ur) * (Ss - ur);
        double U[3] = {rr, rr * ur, pr / (G - 1) + rr * ur * ur / 2}, F[3] = {rr * ur, rr * ur * ur + pr, rr * HR * ur};
        double Dd[3] = {0, 1, Ss};
        for (int i = 0; i < 3; i++) res[i] = (Ss * (SR * U[i] - F[i]) + SR * ps * Dd[i]) / (SR - Ss);
    } else { res[0] = rr * ur; res[1] = rr * ur * ur + pr; res[2] = rr * HR * ur; }
}

static void roe1(const double *L, const double *R, double *res)
{
    double rl = L[0], ul = L[1], pl = L[2], rr = R[0], ur = R[1], pr = R[2];
    double HL = pl / rl * G / (G - 1) + (ul * ul) / 2, HR = pr / rr * G / (G - 1) + (ur * ur) / 2;
    double rB = sqrt(rl * rr);
    double uB = (ul * sqrt(rl) + ur * sqrt(rr)) / (sqrt(rl) + sqrt(rr));
    double HB = (HL * sqrt(rl) + HR * sqrt(rr)) / (sqrt(rl) + sqrt(rr));
    double cB = sqrt((G - 1) * (HB - uB * uB / 2)), cB2 = (G - 1) * (HB - uB * uB / 2);
    double dr = rr - rl, du = ur - ul, dp = pr - pl;
    double lam[3] = {fabs(uB), fabs(uB + cB), fabs(uB - cB)}, eps = 0.1 * (fabs(uB) + cB);
    for (int i = 0; i < 3; i++)
        if (lam[i] < eps) lam[i] = (lam[i] * lam[i] + eps * eps) / (2.0 * eps);
    double a0 = lam[0] * (dr - dp / cB2), a1 = lam[1] / (2.0 * cB2) * (dp + rB * cB * du),
           a2 = lam[2] / (2.0 * cB2) * (dp - rB * cB * du);
    double a3 = a0 + a1 + a2, a4 = cB * (a1 - a2);
    double FL[3] = {rl * ul, rl * ul * ul + pl, rl * HL * ul}, FR[3] = {rr * ur, rr * ur * ur + pr, rr * HR * ur};
    for (int i = 0; i < 3; i++) res[i] = (FL[i] + FR[i]) / 2.0;
    res[0] -= 0.5 * a3;
    res[1] -= 0.5 * (a3 * uB + a4);
    res[2] -= 0.5 * (HB * a3 + uB * a4 - cB2 * a0 / (G - 1));
}

static void hllc_star(int nv, int ax, double r, const double *vel, double p, double H, double Vn, double S, double Ss,
                      double *out, int half, int acc)
{
    int D = nv - 2, E = nv - 1;
    double n[3] = {ax == 0, ax == 1, ax == 2};
    double U[MAXV], F[MAXV], Us[MAXV];
    U[0] = r;
    for (int i = 0; i < D; i++) U[1 + i] = r * vel[i];
    U[E] = r * H - p;
    F[0] = r * Vn;
    for (int i = 0; i < D; i++) F[1 + i] = r * vel[i] * Vn + p * n[i];
    F[E] = r * H * Vn;
    double Usf = (S - Vn) / (S - Ss);
    Us[0] = Usf * r;
    for (int i = 0; i < D; i++) Us[1 + i] = Usf * (Ss * n[i] + vel[i] * (1.0 - n[i])) * r;
    Us[E] = Usf * (U[E] + (Ss - Vn) * (r * Ss + p / (S - Vn)));
    for (int i = 0; i < nv; i++) {
        double f = F[i] + S * (Us[i] - U[i]);
        if (half) f = f / 2;
        out[i] = acc ? out[i] + f : f;
    }
}

static void hllc_md(int nv, int ax, const double *L, const double *R, double *res)
{
    int D = nv - 2, E = nv - 1;
    double n[3] = {ax == 0, ax == 1, ax == 2};
    double rl = L[0], rr = R[0], pl = L[E], pr = R[E];
    double kl = (D == 2) ? (L[1] * L[1] + L[2] * L[2]) : (L[1] * L[1] + L[2] * L[2] + L[3] * L[3]);
    double kr = (D == 2) ? (R[1] * R[1] + R[2] * R[2]) : (R[1] * R[1] + R[2] * R[2] + R[3] * R[3]);
    double HL = kl / 2 + pl / rl * G / (G - 1), HR = kr / 2 + pr / rr * G / (G - 1);
    double VL = L[1 + ax], VR = R[1 + ax];
    double cl = sqrt(pl / rl * G), cr = sqrt(pr / rr * G);
    double rB = (rl + rr) / 2, cB = (cl + cr) / 2;
    double ps0 = (pl + pr) / 2 - rB * cB * (VR - VL) / 2, ps = (0.0 < ps0) ? ps0 : 0.0;
    double ql = (ps <= pl) ? 1.0 : sqrt(1.0 + (G + 1.0) / (2.0 * G) * (ps / pl - 1.0));
    double qr = (ps <= pr) ? 1.0 : sqrt(1.0 + (G + 1.0) / (2.0 * G) * (ps / pr - 1.0));
    double SL = VL - cl * ql, SR = VR + cr * qr;
    double Ss = ((pr - pl) + (rl * VL * (SL - VL) - rr * VR * (SR - VR))) / (rl * (SL - VL) - rr * (SR - VR));
    if (SL > 0) {
        res[0] = rl * VL;
        for (int i = 0; i < D; i++) res[1 + i] = rl * L[1 + i] * VL + pl * n[i];
        res[E] = rl * HL * VL;
    } else if (Ss > 0) hllc_star(nv, ax, rl, L + 1, pl, HL, VL, SL, Ss, res, 0, 0);
    else if (Ss == 0) {
        hllc_star(nv, ax, rl, L + 1, pl, HL, VL, SL, Ss, res, 1, 0);
        hllc_star(nv, ax, rr, R + 1, pr, HR, VR, SR, Ss, res, 1, 1);
    } else if (SR > 0) hllc_star(nv, ax, rr, R + 1, pr, HR, VR, SR, Ss, res, 0, 0);
    else {
        res[0] = rr * VR;
        for (int i = 0; i < D; i++) res[1 + i] = rr * R[1 + i] * VR + pr * n[i];
        res[E] = rr * HR * VR;
    }
}

static void roe_md(int nv, int ax, const double *L, const double *R, double *res)
{
    int D = nv - 2, E = nv - 1;
    double n[3] = {ax == 0, ax == 1, ax == 2};
    double rl = L[0], rr = R[0], pl = L[E], pr = R[E];
    double kl = (D == 2) ? (L[1] * L[1] + L[2] * L[2]) : (L[1] * L[1] + L[2] * L[2] + L[3] * L[3]);
    double kr = (D == 2) ? (R[1] * R[1] + R[2] * R[2]) : (R[1] * R[1] + R[2] * R[2] + R[3] * R[3]);
    double HL = kl / 2 + pl / rl * G / (G - 1), HR = kr / 2 + pr / rr * G / (G - 1);
    double VL = L[1 + ax], VR = R[1 + ax];
    double FL[MAXV], FR[MAXV], Fd[MAXV];
    FL[0] = rl * VL; FR[0] = rr * VR;
    for (int i = 0; i < D; i++) {
        FL[1 + i] = rl * L[1 + i] * VL + pl * n[i];
        FR[1 + i] = rr * R[1 + i] * VR + pr * n[i];
    }
    FL[E] = rl * HL * VL; FR[E] = rr * HR * VR;
    double c1 = sqrt(rl), c2 = sqrt(rr), dv = 1.0 / (sqrt(rl) + sqrt(rr));
    double rA = sqrt(rl * rr), vA[3] = {0, 0, 0};
    for (int i = 0; i < D; i++) vA[i] = (c1 * L[1 + i] + c2 * R[1 + i]) * dv;
    double HA = (c1 * HL + c2 * HR) * dv;
    double q2 = (D == 2) ? (vA[0] * vA[0] + vA[1] * vA[1]) / 2 : (vA[0] * vA[0] + vA[1] * vA[1] + vA[2] * vA[2]) / 2;
    double cA = sqrt((G - 1) * (HA - q2)), VA = vA[ax];
    double lam[3] = {fabs(VA - cA), fabs(VA), fabs(VA + cA)}, eps = 0.05 * (fabs(VA) + cA);
    for (int i = 0; i < 3; i++)
        if (lam[i] < eps) lam[i] = (lam[i] * lam[i] + eps * eps) / (2.0 * eps);
    double dP = pr - pl, dVn = VR - VL, dR = rr - rl, dvv[3];
    for (int i = 0; i < D; i++) dvv[i] = R[1 + i] - L[1 + i];
    double k1 = (dP - rA * cA * dVn) / (2.0 * cA * cA);
    Fd[0] = lam[0] * (k1 * 1);
    for (int i = 0; i < D; i++) Fd[1 + i] = lam[0] * (k1 * (vA[i] - cA * n[i]));
    Fd[E] = lam[0] * (k1 * (HA - cA * VA));
    double k3 = (dP + rA * cA * dVn) / (2.0 * cA * cA);
    Fd[0] += lam[2] * (k3 * 1);
    for (int i = 0; i < D; i++) Fd[1 + i] += lam[2] * (k3 * (vA[i] + cA * n[i]));
    Fd[E] += lam[2] * (k3 * (HA + cA * VA));
    double k2 = dR - dP / (cA * cA);
    Fd[0] += lam[1] * (k2 * 1.0 + rA * 0.0);
    double tE = 0;
    int first = 1;
    for (int i = 0; i < D; i++) {
        Fd[1 + i] += lam[1] * (k2 * vA[i] + rA * ((i == ax) ? 0 : dvv[i]));
        if (i != ax) {
            tE = first ? vA[i] * dvv[i] : tE + vA[i] * dvv[i];
            first = 0;
        }
    }
    Fd[E] += lam[1] * (k2 * q2 + rA * tE);
    for (int i = 0; i < nv; i++) res[i] = (FL[i] + FR[i] - Fd[i]) / 2;
}

static void riemann(const orc_cfg *c, int ax, const double *L, const double *R, double *res)
{
    int nv = nvar_of(c->dim);
    if (nv == 3) { if (c->flux == 0) hllc1(L, R, res); else roe1(L, R, res); }
    else { if (c->flux == 0) hllc_md(nv, ax, L, R, res); else roe_md(nv, ax, L, R, res); }
}

/* ------------------------------------------------------------ line sweep */
static long long strides(const orc_cfg *c, int d)
{
    return d == 0 ? 1 : d == 1 ? c->n[0] : (long long)c->n[0] * c->n[1];
}

/* ghost k of one line end (oneDBnd.cpp:31-114, wiring initializer.cpp:743-870) */
static void ghost(const orc_cfg *c, const double *prim, int d, int side, long long first, int k, double *g)
{
    int nv = nvar_of(c->dim), n = c->n[d];
    long long s = strides(c, d), last = first + (long long)(n - 1) * s, src;
    int type = c->bc[d][side];
    if (type == ORC_OUTLET) src = side == 0 ? first : last;
    else if (type == ORC_WRAP) src = side == 0 ? last - k * s : first + k * s;
    else src = side == 0 ? first + k * s : last - k * s; /* mirror copy (symmetry, default PERIODIC1D wiring) */
    memcpy(g, prim + src * nv, sizeof(double) * nv);
    if (type == ORC_SYMMETRY) g[1 + d] = -g[1 + d];
}

static void sweep_line(const orc_cfg *c, const double *prim, double *rhs, int d, long long first, double (*P)[MAXV],
                       double (*Fh)[MAXV], double (*Fn)[MAXV])
{
    int nv = nvar_of(c->dim), n = c->n[d];
    int ng = c->diff ? 5 : 4, nf = n + 2 * ng - 5;
    long long s = strides(c, d);
    /* P[0..n+2ng-1] = ghosts ng-1..0 (reversed, reconstructor5order.hpp:64-84), cells, ghosts 0..ng-1 */
    for (int k = 0; k < ng; k++) ghost(c, prim, d, 0, first, k, P[ng - 1 - k]);
    for (int i = 0; i < n; i++) memcpy(P[ng + i], prim + (first + i * s) * nv, sizeof(double) * nv);
    for (int k = 0; k < ng; k++) ghost(c, prim, d, 1, first, k, P[ng + n + k]);
    /* nf faces x_{-(2ng-5)/2} .. x_{n-1+(2ng-5)/2}: face f uses P[f .. f+5] */
    for (int f = 0; f < nf; f++) {
        double fl[MAXV], fr[MAXV];
        recon_face(c, d, P + f, fl, fr);
        riemann(c, d, fl, fr, Fh[f]);
    }
    if (c->diff) {
        /* ExplicitDif6: faces Fh[i] .. Fh[i+5] are x_{i-5/2} .. x_{i+5/2} */
        const double w0 = 75.0 / 64.0, w1 = 25.0 / (128.0 * 3.0), w2 = 3.0 / (128.0 * 5.0);
        for (int i = 0; i < n; i++) {
            double *r = rhs + (first + i * s) * nv;
            for (int v = 0; v < nv; v++)
                r[v] += (w0 * (Fh[i + 3][v] - Fh[i + 2][v]) - w1 * (Fh[i + 4][v] - Fh[i + 1][v]) +
                         w2 * (Fh[i + 5][v] - Fh[i][v])) / c->h;
        }
        return;
    }
    /* n+2 nodes x_{-1} .. x_n (ghost 0 on each side, nl = nr = 1) */
    for (int m = 0; m < n + 2; m++) phys_flux(nv, d, P[3 + m], Fn[m]);
    const double w0 = 3.0 / 2.0, w1 = -3.0 / 10.0, w2 = 1.0 / 30.0;
    for (int i = 0; i < n; i++) {
        double *r = rhs + (first + i * s) * nv;
        for (int v = 0; v < nv; v++)
            r[v] += (w1 * (Fn[i + 2][v] - Fn[i][v]) + w0 * (Fh[i + 2][v] - Fh[i + 1][v]) + w2 * (Fh[i + 3][v] - Fh[i][v])) / c->h;
    }
}

void orc_rhs(const orc_cfg *c, const double *cons, double *rhs)
{
    int nv = nvar_of(c->dim);
    long long nc = (long long)c->n[0] * c->n[1] * c->n[2];
    double *prim = (double *)malloc(sizeof(double) * nc * nv);
    for (long long i = 0; i < nc; i++) c2p(nv, cons + i * nv, prim + i * nv);
    memset(rhs, 0, sizeof(double) * nc * nv);
    for (int d = 0; d < c->dim; d++) {
        int n = c->n[d], t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
        long long nl = nc / n;
#pragma omp parallel num_threads(c->threads > 0 ? c->threads : omp_get_max_threads())
        {
            double (*P)[MAXV] = malloc(sizeof(double) * MAXV * (n + 10));
            double (*Fh)[MAXV] = malloc(sizeof(double) * MAXV * (n + 5));
            double (*Fn)[MAXV] = malloc(sizeof(double) * MAXV * (n + 2));
#pragma omp for schedule(static)
            for (long long l = 0; l < nl; l++) {
                long long a = l % c->n[t0], b = l / c->n[t0];
                long long first = a * strides(c, t0) + b * strides(c, t1);
                sweep_line(c, prim, rhs, d, first, P, Fh, Fn);
            }
            free(P); free(Fh); free(Fn);
        }
    }
    free(prim);
}

double orc_max_dt(const orc_cfg *c, const double *cons, double cfl)
{
    int nv = nvar_of(c->dim);
    long long nc = (long long)c->n[0] * c->n[1] * c->n[2];
    double lam = 0;
    for (int d = 0; d < c->dim; d++) {
        double mx = 0;
        for (long long i = 0; i < nc; i++) {
            double p[MAXV];
            c2p(nv, cons + i * nv, p);
            double l = (sqrt(G * p[nv - 1] / p[0]) + fabs(p[1 + d])) / c->h;
            mx = (mx < l) ? l : mx;
        }
        lam += mx;
    }
    return cfl / lam;
}

double orc_rk3(const orc_cfg *c, double *cons, double dt)
{
    int nv = nvar_of(c->dim);
    long long n = (long long)c->n[0] * c->n[1] * c->n[2] * nv;
    double *u0 = (double *)malloc(sizeof(double) * n), *r = (double *)malloc(sizeof(double) * n);
    memcpy(u0, cons, sizeof(double) * n);
    orc_rhs(c, cons, r);
    for (long long i = 0; i < n; i++) cons[i] = u0[i] - dt * r[i];
    orc_rhs(c, cons, r);
    for (long long i = 0; i < n; i++) cons[i] = 0.75 * u0[i] - 0.25 * dt * r[i] + 0.25 * cons[i];
    orc_rhs(c, cons, r);
    for (long long i = 0; i < n; i++) cons[i] = 1.0 / 3.0 * u0[i] - 2.0 / 3.0 * dt * r[i] + 2.0 / 3.0 * cons[i];
    double linf = fabs(r[0]);
    for (long long i = 1; i < n / nv; i++)
        if (linf < fabs(r[i * nv])) linf = fabs(r[i * nv]);
    free(u0);
    free(r);
    return linf;
}
