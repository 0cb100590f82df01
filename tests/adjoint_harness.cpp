// Host build of the adjoint arithmetic (cfd_inwsl_b200/csrc/adjoint_math.h) for
// tests/test_adjoint_math.py: forward formulas in long double (finite
// differences) and the hand-written vector-Jacobian products in double.
#include "adjoint_math.h"

using namespace cfd::adj;

extern "C" {
void h_face_fwd(int ax, const long double *u, long double *F)
{
    long double U[6][4];
    for (int j = 0; j < 6; j++)
        for (int v = 0; v < 4; v++) U[j][v] = u[4 * j + v];
    if (ax == 0) face_flux_t<long double, 0>(U, F);
    else face_flux_t<long double, 1>(U, F);
}
void h_face_vjp(int ax, const double *u, const double *Fb, double *ub)
{
    double U[6][4], Ub[6][4] = {};
    for (int j = 0; j < 6; j++)
        for (int v = 0; v < 4; v++) U[j][v] = u[4 * j + v];
    if (ax == 0) face_vjp<0>(U, Fb, Ub);
    else face_vjp<1>(U, Fb, Ub);
    for (int j = 0; j < 6; j++)
        for (int v = 0; v < 4; v++) ub[4 * j + v] = Ub[j][v];
}
void h_roe_fwd(int ax, const long double *L, const long double *R, long double *F)
{
    if (ax == 0) roe_t<long double, 0>(L, R, F);
    else roe_t<long double, 1>(L, R, F);
}
void h_roe_vjp(int ax, const double *L, const double *R, const double *Fb, double *Lb, double *Rb)
{
    for (int i = 0; i < 4; i++) Lb[i] = Rb[i] = 0.0;
    if (ax == 0) roe_vjp<0>(L, R, Fb, Lb, Rb);
    else roe_vjp<1>(L, R, Fb, Lb, Rb);
}
void h_face_fwd_f(int ax, int fam, double ct, const long double *u, long double *F)
{
    long double U[6][4];
    for (int j = 0; j < 6; j++)
        for (int v = 0; v < 4; v++) U[j][v] = u[4 * j + v];
    if (ax == 0) face_flux_t<long double, 0>(U, F, fam, ct);
    else face_flux_t<long double, 1>(U, F, fam, ct);
}
void h_face_vjp_f(int ax, int fam, double ct, const double *u, const double *Fb, double *ub)
{
    double U[6][4], Ub[6][4] = {};
    for (int j = 0; j < 6; j++)
        for (int v = 0; v < 4; v++) U[j][v] = u[4 * j + v];
    if (ax == 0) face_vjp<0>(U, Fb, Ub, fam, ct);
    else face_vjp<1>(U, Fb, Ub, fam, ct);
    for (int j = 0; j < 6; j++)
        for (int v = 0; v < 4; v++) ub[4 * j + v] = Ub[j][v];
}
unsigned h_teno_flag(int fam, const double *q, double ct) { return teno_flag(fam, q, ct); }
long double h_interp_fwd(int fam, const long double *q, double ct) { return interp5_t(fam, q, ct); }
void h_interp_vjp(int fam, const double *q, double ct, double Qb, double *qb)
{
    unsigned flag;
    for (int i = 0; i < 5; i++) qb[i] = 0.0;
    interp5(fam, q, ct, flag);
    interp5_adj(fam, q, flag, Qb, qb);
}
long double h_wcns5_fwd(const long double *q) { return wcns5_t(q); }
void h_wcns5_vjp(const double *q, double Qb, double *qb)
{
    for (int i = 0; i < 5; i++) qb[i] = 0.0;
    wcns5_adj(q, Qb, qb);
}
void h_node_fwd(int ax, const long double *U, long double *G)
{
    if (ax == 0) node_flux_t<long double, 0>(U, G);
    else node_flux_t<long double, 1>(U, G);
}
void h_node_vjp(int ax, const double *U, const double *Gb, double *ub)
{
    for (int i = 0; i < 4; i++) ub[i] = 0.0;
    if (ax == 0) node_vjp<0>(U, Gb, ub);
    else node_vjp<1>(U, Gb, ub);
}
}
