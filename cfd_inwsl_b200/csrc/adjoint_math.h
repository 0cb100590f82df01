// Discrete-adjoint arithmetic of one face and one node of the 2D Euler path
// (WCNS5 or TENO characteristic reconstruction, Roe flux, node fluxes), host
// and device: adjoint.cu runs it on the GPU, and the CPU tests compile it with
// the host compiler to check every vector-Jacobian product against extended-
// precision finite differences of the same forward formulas.
//
// TENO's cut-off decision is a step function of the stencil values. The
// adjoint freezes it: the flag of the forward state selects one of the eight
// fixed linear stencils (interScheme.hpp:445-480), and the derivative of the
// interpolation is that stencil's coefficients.
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define ADJ_HD __host__ __device__ inline
#else
#define ADJ_HD inline
#endif

// unroll factor of the characteristic-field loop of the face adjoint's
// second half
#ifndef ADJ_CHARS_UNROLL
#define ADJ_CHARS_UNROLL 4
#endif

namespace cfd {
namespace adj {

using std::fabs;
using std::sqrt;

constexpr double kGam = 1.4;  // GAMMA (macro.hpp)
constexpr double kGm1 = kGam - 1.0;
constexpr double kGG1 = kGam / (kGam - 1.0);
constexpr double kW0 = 3.0 / 2.0, kW1 = -3.0 / 10.0, kW2 = 1.0 / 30.0;
constexpr int kCharsUnroll = ADJ_CHARS_UNROLL;

// cons (rho, rho u, rho v, rho E) -> prim (rho, u, v, p); returns 1/rho
ADJ_HD double c2p(const double *c, double *p)
{
    const double ir = 1.0 / c[0];
    p[0] = c[0];
    p[1] = c[1] * ir;
    p[2] = c[2] * ir;
    p[3] = kGm1 * (c[3] - (c[1] * c[1] + c[2] * c[2]) * (0.5 * ir));
    return ir;
}

// cb += (d prim / d cons)^T pb, p = c2p(c), ir = 1/rho as c2p returned it
ADJ_HD void c2p_adj(const double *p, double ir, const double *pb, double *cb)
{
    const double u = p[1], v = p[2];
    cb[0] += pb[0] - (u * pb[1] + v * pb[2]) * ir + pb[3] * (0.5 * kGm1) * (u * u + v * v);
    cb[1] += pb[1] * ir - pb[3] * kGm1 * u;
    cb[2] += pb[2] * ir - pb[3] * kGm1 * v;
    cb[3] += pb[3] * kGm1;
}

// 1/s0, 1/s1, 1/s2 from one division of their product (three divisions
// cost about three times as much on the FP64 pipe); the product is guarded
// against overflow (s_k >= 1e-6 here, so it cannot underflow)
ADJ_HD void recip3(double s0, double s1, double s2, double &r0, double &r1, double &r2)
{
    const double s01 = s0 * s1, p = s01 * s2;
    if (p < 1e300) {
        const double ip = 1.0 / p;
        r0 = (s1 * s2) * ip;
        r1 = (s0 * s2) * ip;
        r2 = s01 * ip;
    } else {
        r0 = 1.0 / s0;
        r1 = 1.0 / s1;
        r2 = 1.0 / s2;
    }
}

// weno5_JSchen: gamma_k / (1e-6 + beta_k)^2 weights of the three candidates
ADJ_HD double wcns5(const double *q)
{
    const double a0 = q[0] - 2.0 * q[1] + q[2], b0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
    const double a1 = q[1] - 2.0 * q[2] + q[3], b1 = q[1] - q[3];
    const double a2 = q[2] - 2.0 * q[3] + q[4], b2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
    const double s0 = 1e-6 + a0 * a0 + 0.25 * b0 * b0, s1 = 1e-6 + a1 * a1 + 0.25 * b1 * b1,
                 s2 = 1e-6 + a2 * a2 + 0.25 * b2 * b2;
    double r0, r1, r2;
    recip3(s0, s1, s2, r0, r1, r2);
    const double al0 = (1.0 / 16.0) * (r0 * r0), al1 = (5.0 / 8.0) * (r1 * r1), al2 = (5.0 / 16.0) * (r2 * r2);
    const double u0 = 0.375 * q[0] - 1.25 * q[1] + 1.875 * q[2];
    const double u1 = -0.125 * q[1] + 0.75 * q[2] + 0.375 * q[3];
    const double u2 = 0.375 * q[2] + 0.75 * q[3] - 0.125 * q[4];
    return (al0 * u0 + al1 * u1 + al2 * u2) / (al0 + al1 + al2);
}

// qb += (dW/dq)^T Qb
ADJ_HD void wcns5_adj(const double *q, double Qb, double *qb)
{
    const double a0 = q[0] - 2.0 * q[1] + q[2], b0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
    const double a1 = q[1] - 2.0 * q[2] + q[3], b1 = q[1] - q[3];
    const double a2 = q[2] - 2.0 * q[3] + q[4], b2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
    const double s0 = 1e-6 + a0 * a0 + 0.25 * b0 * b0, s1 = 1e-6 + a1 * a1 + 0.25 * b1 * b1,
                 s2 = 1e-6 + a2 * a2 + 0.25 * b2 * b2;
    double r0, r1, r2;
    recip3(s0, s1, s2, r0, r1, r2);
    const double al0 = (1.0 / 16.0) * (r0 * r0), al1 = (5.0 / 8.0) * (r1 * r1), al2 = (5.0 / 16.0) * (r2 * r2);
    const double u0 = 0.375 * q[0] - 1.25 * q[1] + 1.875 * q[2];
    const double u1 = -0.125 * q[1] + 0.75 * q[2] + 0.375 * q[3];
    const double u2 = 0.375 * q[2] + 0.75 * q[3] - 0.125 * q[4];
    const double iS = 1.0 / (al0 + al1 + al2);
    const double Q = (al0 * u0 + al1 * u1 + al2 * u2) * iS;
    const double g = Qb * iS;
    const double ub0 = g * al0, ub1 = g * al1, ub2 = g * al2;
    // d alpha_k / d beta_k = -2 alpha_k / s_k
    const double bb0 = g * (u0 - Q) * (-2.0 * al0 * r0), bb1 = g * (u1 - Q) * (-2.0 * al1 * r1),
                 bb2 = g * (u2 - Q) * (-2.0 * al2 * r2);
    const double ab0 = 2.0 * a0 * bb0, bq0 = 0.5 * b0 * bb0;
    const double ab1 = 2.0 * a1 * bb1, bq1 = 0.5 * b1 * bb1;
    const double ab2 = 2.0 * a2 * bb2, bq2 = 0.5 * b2 * bb2;
    qb[0] += ab0 + bq0 + 0.375 * ub0;
    qb[1] += -2.0 * ab0 - 4.0 * bq0 + ab1 + bq1 - 1.25 * ub0 - 0.125 * ub1;
    qb[2] += ab0 + 3.0 * bq0 - 2.0 * ab1 + ab2 + 3.0 * bq2 + 1.875 * ub0 + 0.75 * ub1 + 0.375 * ub2;
    qb[3] += ab1 - bq1 - 2.0 * ab2 - 4.0 * bq2 + 0.375 * ub1 + 0.75 * ub2;
    qb[4] += ab2 + bq2 - 0.125 * ub2;
}

// Interpolations the adjoint differentiates (the library's family numbers).
enum AdjInterp : int { ADJ_WCNS5 = 0, ADJ_TENOZ = 2, ADJ_TENOCONG = 3 };

// Coefficients of the fixed stencil a TENO flag selects (bit k: stencil k cut).
template <class T>
ADJ_HD void teno_coeffs(unsigned flag, T *a)
{
    for (int m = 0; m < 5; m++) a[m] = T(0);
    switch (flag & 7u) {
    case 0: a[0] = T(3) / 128; a[1] = T(-5) / 32; a[2] = T(45) / 64; a[3] = T(15) / 32; a[4] = T(-5) / 128; break;
    case 1: a[1] = T(-1) / 16; a[2] = T(9) / 16; a[3] = T(9) / 16; a[4] = T(-1) / 16; break;
    case 2:
    case 3: a[2] = T(3) / 8; a[3] = T(3) / 4; a[4] = T(-1) / 8; break;
    case 4: a[0] = T(1) / 16; a[1] = T(-5) / 16; a[2] = T(15) / 16; a[3] = T(5) / 16; break;
    case 5: a[1] = T(-1) / 8; a[2] = T(3) / 4; a[3] = T(3) / 8; break;
    case 6: a[0] = T(3) / 8; a[1] = T(-5) / 4; a[2] = T(15) / 8; break;
    default: a[2] = T(1); break;
    }
}

// The cut-off flag of the stencil q[0..4]: Teno5_Z (interScheme.hpp:384-452),
// measure_k = (1 + tau / (beta_k + 1e-40))^6 cut below ct * sum_j measure_j;
// Teno5_CongZ (interScheme.hpp:494-584), cut where
// tau beta_min < (ct tau - (1 - ct) beta_min) beta_k.
template <class T>
ADJ_HD unsigned teno_flag(int fam, const T *q, double ct)
{
    const T a0 = q[0] - 2 * q[1] + q[2], b0 = q[0] - 4 * q[1] + 3 * q[2];
    const T a1 = q[1] - 2 * q[2] + q[3], b1 = q[1] - q[3];
    const T a2 = q[2] - 2 * q[3] + q[4], b2 = 3 * q[2] - 4 * q[3] + q[4];
    const T be[3] = {a0 * a0 + T(0.25) * b0 * b0, a1 * a1 + T(0.25) * b1 * b1, a2 * a2 + T(0.25) * b2 * b2};
    const T tau = be[2] > be[0] ? be[2] - be[0] : be[0] - be[2];
    unsigned flag = 0;
    if (fam == ADJ_TENOZ) {
        T m[3], sum = T(0);
        for (int k = 0; k < 3; k++) {
            T t = T(1) + tau / (be[k] + T(1e-40));
            t *= t;
            m[k] = t * t * t;
            sum += m[k];
        }
        for (int k = 0; k < 3; k++)
            if (m[k] < T(ct) * sum) flag += 1u << k;
    } else {
        T bmin = be[0];
        if (be[1] < bmin) bmin = be[1];
        if (be[2] < bmin) bmin = be[2];
        const T rr = T(ct) * tau - (T(1) - T(ct)) * bmin, ll = tau * bmin;
        for (int k = 0; k < 3; k++)
            if (ll < rr * be[k]) flag += 1u << k;
    }
    return flag;
}

// One interpolation of family fam (constant ct) and its frozen flag.
ADJ_HD double interp5(int fam, const double *q, double ct, unsigned &flag)
{
    if (fam == ADJ_WCNS5) {
        flag = 0;
        return wcns5(q);
    }
    flag = teno_flag(fam, q, ct);
    double a[5];
    teno_coeffs(flag, a);
    return a[0] * q[0] + a[1] * q[1] + a[2] * q[2] + a[3] * q[3] + a[4] * q[4];
}

// qb += (dQ/dq)^T Qb with the forward's flag
ADJ_HD void interp5_adj(int fam, const double *q, unsigned flag, double Qb, double *qb)
{
    if (fam == ADJ_WCNS5) {
        wcns5_adj(q, Qb, qb);
        return;
    }
    double a[5];
    teno_coeffs(flag, a);
    for (int m = 0; m < 5; m++) qb[m] += a[m] * Qb;
}

// Lb += (dRoe/dL)^T resb, Rb likewise (L, R: face prims)
template <int AX>
ADJ_HD void roe_vjp(const double *L, const double *R, const double *resb, double *Lb, double *Rb)
{
    const double n[2] = {AX == 0 ? 1.0 : 0.0, AX == 1 ? 1.0 : 0.0};
    const double rl = L[0], pl = L[3], rr = R[0], pr = R[3];
    const double vl[2] = {L[1], L[2]}, vr[2] = {R[1], R[2]};
    const double kl = vl[0] * vl[0] + vl[1] * vl[1], kr = vr[0] * vr[0] + vr[1] * vr[1];
    const double VnL = vl[AX], VnR = vr[AX];
    const double s1 = sqrt(rl), s2 = sqrt(rr), iA = 1.0 / (s1 + s2), rhoA = s1 * s2;
    const double vA[2] = {(s1 * vl[0] + s2 * vr[0]) * iA, (s1 * vl[1] + s2 * vr[1]) * iA};
    // 1/rho of both states, for H here and for the reverse below
    const double irl = 1.0 / rl, irr = 1.0 / rr;
    const double HL = 0.5 * kl + kGG1 * pl * irl, HR = 0.5 * kr + kGG1 * pr * irr;
    const double HA = (s1 * HL + s2 * HR) * iA;
    const double q2 = 0.5 * (vA[0] * vA[0] + vA[1] * vA[1]);
    const double c2 = kGm1 * (HA - q2), c = sqrt(c2), ic2 = 1.0 / c2;
    const double VnA = vA[AX];
    const double x[3] = {VnA - c, VnA, VnA + c};
    const double eps = 0.05 * (fabs(VnA) + c);
    double l0[3], lam[3];
    bool fix[3];
    for (int i = 0; i < 3; i++) {
        l0[i] = fabs(x[i]);
        fix[i] = l0[i] < eps;
        lam[i] = fix[i] ? (l0[i] * l0[i] + eps * eps) / (2.0 * eps) : l0[i];
    }
    const double dP = pr - pl, dVn = VnR - VnL, dRho = rr - rl, rc = rhoA * c * dVn;
    const double a1 = lam[0] * (dP - rc) * (0.5 * ic2), a3 = lam[2] * (dP + rc) * (0.5 * ic2);
    const double a2 = lam[1] * (dRho - dP * ic2), l1r = lam[1] * rhoA;
    double t[2], tE = 0.0;
    for (int i = 0; i < 2; i++) {
        t[i] = (i == AX) ? 0.0 : vr[i] - vl[i];
        if (i != AX) tE += vA[i] * t[i];
    }

    // ---- reverse: res = (Fc - Fd) / 2
    double rlb = 0, rrb = 0, plb = 0, prb = 0, vlb[2] = {0, 0}, vrb[2] = {0, 0}, klb = 0, krb = 0, VnLb = 0, VnRb = 0;
    {
        const double F0 = 0.5 * resb[0];
        rlb += VnL * F0; VnLb += rl * F0; rrb += VnR * F0; VnRb += rr * F0;
        for (int i = 0; i < 2; i++) {
            const double F = 0.5 * resb[1 + i];
            rlb += vl[i] * VnL * F; vlb[i] += rl * VnL * F; VnLb += rl * vl[i] * F;
            rrb += vr[i] * VnR * F; vrb[i] += rr * VnR * F; VnRb += rr * vr[i] * F;
            plb += n[i] * F; prb += n[i] * F;
        }
        const double F3 = 0.5 * resb[3];
        const double XL = 0.5 * rl * kl + kGG1 * pl, XR = 0.5 * rr * kr + kGG1 * pr;
        VnLb += XL * F3; VnRb += XR * F3;
        rlb += 0.5 * kl * VnL * F3; klb += 0.5 * rl * VnL * F3; plb += kGG1 * VnL * F3;
        rrb += 0.5 * kr * VnR * F3; krb += 0.5 * rr * VnR * F3; prb += kGG1 * VnR * F3;
    }
    double a1b = 0, a2b = 0, a3b = 0, l1rb = 0, vAb[2] = {0, 0}, cb = 0, VnAb = 0, HAb = 0, q2b = 0, tb[2] = {0, 0},
           tEb = 0;
    {
        const double F0 = -0.5 * resb[0];
        a1b += F0; a3b += F0; a2b += F0;
        for (int i = 0; i < 2; i++) {
            const double F = -0.5 * resb[1 + i];
            a1b += (vA[i] - c * n[i]) * F; a3b += (vA[i] + c * n[i]) * F; a2b += vA[i] * F; l1rb += t[i] * F;
            vAb[i] += (a1 + a3 + a2) * F; cb += (a3 - a1) * n[i] * F; tb[i] += l1r * F;
        }
        const double F3 = -0.5 * resb[3];
        a1b += (HA - c * VnA) * F3; a3b += (HA + c * VnA) * F3; a2b += q2 * F3; l1rb += tE * F3;
        HAb += (a1 + a3) * F3; cb += (a3 - a1) * VnA * F3; VnAb += (a3 - a1) * c * F3; q2b += a2 * F3; tEb += l1r * F3;
    }
    for (int i = 0; i < 2; i++)
        if (i != AX) {
            vAb[i] += t[i] * tEb;
            tb[i] += vA[i] * tEb;
            vrb[i] += tb[i];
            vlb[i] -= tb[i];
        }
    double lamb[3] = {0, 0, 0}, rhoAb = 0, dPb = 0, dVnb = 0, dRhob = 0, rcb = 0, ic2b = 0;
    lamb[1] += rhoA * l1rb; rhoAb += lam[1] * l1rb;
    lamb[1] += (dRho - dP * ic2) * a2b; dRhob += lam[1] * a2b; dPb -= lam[1] * ic2 * a2b; ic2b -= lam[1] * dP * a2b;
    lamb[0] += (dP - rc) * 0.5 * ic2 * a1b; dPb += lam[0] * 0.5 * ic2 * a1b; rcb -= lam[0] * 0.5 * ic2 * a1b;
    ic2b += lam[0] * (dP - rc) * 0.5 * a1b;
    lamb[2] += (dP + rc) * 0.5 * ic2 * a3b; dPb += lam[2] * 0.5 * ic2 * a3b; rcb += lam[2] * 0.5 * ic2 * a3b;
    ic2b += lam[2] * (dP + rc) * 0.5 * a3b;
    rhoAb += c * dVn * rcb; cb += rhoA * dVn * rcb; dVnb += rhoA * c * rcb;
    prb += dPb; plb -= dPb; VnRb += dVnb; VnLb -= dVnb; rrb += dRhob; rlb -= dRhob;
    double epsb = 0;
    for (int i = 0; i < 3; i++) {
        double l0b = lamb[i];
        if (fix[i]) {
            l0b = lamb[i] * l0[i] / eps;
            epsb += lamb[i] * (0.5 - l0[i] * l0[i] / (2.0 * eps * eps));
        }
        const double xb = x[i] >= 0.0 ? l0b : -l0b;
        VnAb += xb;
        if (i == 0) cb -= xb;
        if (i == 2) cb += xb;
    }
    VnAb += 0.05 * (VnA >= 0.0 ? epsb : -epsb);
    cb += 0.05 * epsb;
    const double c2b = cb * 0.5 * (c * ic2) - ic2 * ic2 * ic2b;  // 1/c = c / c^2
    HAb += kGm1 * c2b;
    q2b -= kGm1 * c2b;
    vAb[AX] += VnAb;
    for (int i = 0; i < 2; i++) vAb[i] += vA[i] * q2b;
    const double HLb = s1 * iA * HAb, HRb = s2 * iA * HAb;
    double s1b = (HL - HA) * iA * HAb, s2b = (HR - HA) * iA * HAb;
    for (int i = 0; i < 2; i++) {
        vlb[i] += s1 * iA * vAb[i];
        vrb[i] += s2 * iA * vAb[i];
        s1b += (vl[i] - vA[i]) * iA * vAb[i];
        s2b += (vr[i] - vA[i]) * iA * vAb[i];
    }
    s1b += s2 * rhoAb;
    s2b += s1 * rhoAb;
    // 1/sqrt(rho) = sqrt(rho) / rho
    klb += 0.5 * HLb; plb += kGG1 * irl * HLb; rlb -= kGG1 * pl * (irl * irl) * HLb;
    krb += 0.5 * HRb; prb += kGG1 * irr * HRb; rrb -= kGG1 * pr * (irr * irr) * HRb;
    rlb += s1b * 0.5 * (s1 * irl);
    rrb += s2b * 0.5 * (s2 * irr);
    for (int i = 0; i < 2; i++) {
        vlb[i] += 2.0 * vl[i] * klb;
        vrb[i] += 2.0 * vr[i] * krb;
    }
    vlb[AX] += VnLb;
    vrb[AX] += VnRb;
    Lb[0] += rlb; Lb[1] += vlb[0]; Lb[2] += vlb[1]; Lb[3] += plb;
    Rb[0] += rrb; Rb[1] += vrb[0]; Rb[2] += vrb[1]; Rb[3] += prb;
}

// Roe average of a face stencil's cells 2 and 3, the eigenvectors (rows of
// L, columns of R) and what they are built from (eigenSystem.cpp:13-86)
template <int AX>
struct FaceEig {
    // i2, i3: 1/rho of cells 2 and 3
    double P2[4], P3[4], i2, i3, s1, s2, iA, HL, HR, u, v, ht, ek, h, c, ic, ih, Vn, L[4][4], R[4][4];
    ADJ_HD explicit FaceEig(const double (&U)[6][4])
    {
        constexpr double nx = (AX == 0) ? 1.0 : 0.0, ny = (AX == 1) ? 1.0 : 0.0;
        i2 = c2p(U[2], P2);
        i3 = c2p(U[3], P3);
        s1 = sqrt(P2[0]); s2 = sqrt(P3[0]); iA = 1.0 / (s1 + s2);
        HL = 0.5 * (P2[1] * P2[1] + P2[2] * P2[2]) + kGG1 * P2[3] * i2;
        HR = 0.5 * (P3[1] * P3[1] + P3[2] * P3[2]) + kGG1 * P3[3] * i3;
        u = (s1 * P2[1] + s2 * P3[1]) * iA; v = (s1 * P2[2] + s2 * P3[2]) * iA;
        ht = (s1 * HL + s2 * HR) * iA;
        ek = 0.5 * (u * u + v * v); h = ht - ek;
        // c^2 = (gamma - 1) h, so 1/h = (gamma - 1) / c^2
        c = sqrt(kGm1 * h); ic = 1.0 / c; ih = kGm1 * (ic * ic); Vn = nx * u + ny * v;
        L[0][0] = -ny * u + nx * v; L[0][1] = ny; L[0][2] = -nx; L[0][3] = 0.0;
        L[1][0] = h - ek; L[1][1] = u; L[1][2] = v; L[1][3] = -1.0;
        L[2][0] = 0.5 * (Vn * ic + ek * ih); L[2][1] = 0.5 * (-nx * ic - u * ih); L[2][2] = 0.5 * (-ny * ic - v * ih);
        L[2][3] = 0.5 * ih;
        L[3][0] = 0.5 * (-Vn * ic + ek * ih); L[3][1] = 0.5 * (nx * ic - u * ih); L[3][2] = 0.5 * (ny * ic - v * ih);
        L[3][3] = 0.5 * ih;
        R[0][0] = 0.0; R[1][0] = ny; R[2][0] = -nx; R[3][0] = ny * u - nx * v;
        R[0][1] = ih; R[1][1] = u * ih; R[2][1] = v * ih; R[3][1] = ek * ih;
        R[0][2] = 1.0; R[1][2] = u - nx * c; R[2][2] = v - ny * c; R[3][2] = h + ek - Vn * c;
        R[0][3] = 1.0; R[1][3] = u + nx * c; R[2][3] = v + ny * c; R[3][3] = h + ek + Vn * c;
    }
};

// What the first half of a face adjoint hands the second: the interpolated
// characteristic states with their TENO flags and the adjoints of the face's
// reconstructed cons (clb, crb) and of the prims of cells 2 and 3 that the
// positivity fallback used (P2b, P3b).
struct FaceStates {
    double QL[4], QR[4], clb[4], crb[4], P2b[4], P3b[4];
    unsigned flL[4], flR[4];
};

// First half of the face adjoint: the forward to the face states and the
// Roe flux's adjoint back to the reconstructed cons.
template <int AX>
ADJ_HD void face_vjp_states(const double (&U)[6][4], const double *Fb, FaceStates &f, int fam, double ct)
{
    const FaceEig<AX> e(U);
    const double(&P2)[4] = e.P2;
    const double(&P3)[4] = e.P3;
    const double(&L)[4][4] = e.L;
    const double(&R)[4][4] = e.R;
    // characteristic values of field k on the six cells (recomputed in the
    // reverse pass rather than kept: the stencil state is register-bound)
    auto char_field = [&](int k, double *q) {
#pragma unroll
        for (int j = 0; j < 6; j++)
            q[j] = L[k][0] * U[j][0] + L[k][1] * U[j][1] + L[k][2] * U[j][2] + L[k][3] * U[j][3];
    };
    double(&QL)[4] = f.QL;
    double(&QR)[4] = f.QR;
    unsigned(&flL)[4] = f.flL;
    unsigned(&flR)[4] = f.flR;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        double q[6];
        char_field(k, q);
        const double qm[5] = {q[5], q[4], q[3], q[2], q[1]};
        QL[k] = interp5(fam, q, ct, flL[k]);
        QR[k] = interp5(fam, qm, ct, flR[k]);
    }
    double cl[4], cr[4], fl[4], fr[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        cl[i] = R[i][0] * QL[0] + R[i][1] * QL[1] + R[i][2] * QL[2] + R[i][3] * QL[3];
        cr[i] = R[i][0] * QR[0] + R[i][1] * QR[1] + R[i][2] * QR[2] + R[i][3] * QR[3];
    }
    const double icl = c2p(cl, fl), icr = c2p(cr, fr);
    // positivity fallback (reconstructor5order.hpp:380-381), right state quirk included
    const bool fbl = fl[0] < 0 || fl[3] < 0, fbr = fr[0] < 0 || fr[3] < 0;
    if (fbl)
        for (int i = 0; i < 4; i++) fl[i] = P2[i];
    if (fbr) {
        fr[0] = P3[0]; fr[1] = P2[1]; fr[2] = P2[2]; fr[3] = P3[3];
    }

    // ---- reverse
    double flb[4] = {0, 0, 0, 0}, frb[4] = {0, 0, 0, 0};
    roe_vjp<AX>(fl, fr, Fb, flb, frb);
    double(&P2b)[4] = f.P2b;
    double(&P3b)[4] = f.P3b;
    double(&clb)[4] = f.clb;
    double(&crb)[4] = f.crb;
#pragma unroll
    for (int i = 0; i < 4; i++) P2b[i] = P3b[i] = clb[i] = crb[i] = 0.0;
    if (fbl) {
        for (int i = 0; i < 4; i++) P2b[i] += flb[i];
    } else {
        c2p_adj(fl, icl, flb, clb);
    }
    if (fbr) {
        P3b[0] += frb[0]; P2b[1] += frb[1]; P2b[2] += frb[2]; P3b[3] += frb[3];
    } else {
        c2p_adj(fr, icr, frb, crb);
    }
}

// Second half: the characteristic projections, the interpolations and the
// eigensystem run backwards (the eigensystem is recomputed from U). Ub += .
template <int AX>
ADJ_HD void face_vjp_chars(const double (&U)[6][4], const FaceStates &f, double (&Ub)[6][4], int fam)
{
    constexpr double nx = (AX == 0) ? 1.0 : 0.0, ny = (AX == 1) ? 1.0 : 0.0;
    const FaceEig<AX> e(U);
    const double(&P2)[4] = e.P2;
    const double(&P3)[4] = e.P3;
    const double(&L)[4][4] = e.L;
    const double(&R)[4][4] = e.R;
    const double s1 = e.s1, s2 = e.s2, iA = e.iA, HL = e.HL, HR = e.HR, u = e.u, v = e.v, ht = e.ht, ek = e.ek,
                 h = e.h, c = e.c, ic = e.ic, ih = e.ih, Vn = e.Vn;
    (void)h;
    // characteristic values of field k on the six cells (recomputed in the
    // reverse pass rather than kept: the stencil state is register-bound)
    auto char_field = [&](int k, double *q) {
#pragma unroll
        for (int j = 0; j < 6; j++)
            q[j] = L[k][0] * U[j][0] + L[k][1] * U[j][1] + L[k][2] * U[j][2] + L[k][3] * U[j][3];
    };
    const double(&QL)[4] = f.QL;
    const double(&QR)[4] = f.QR;
    const double(&clb)[4] = f.clb;
    const double(&crb)[4] = f.crb;
    const unsigned(&flL)[4] = f.flL;
    const unsigned(&flR)[4] = f.flR;
    double P2b[4], P3b[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        P2b[i] = f.P2b[i];
        P3b[i] = f.P3b[i];
    }
    // eigenvector entries -> (u, v, h, c, ek, Vn, 1/c, 1/h); each row of L's
    // adjoint goes into these as soon as it is formed
    double ub = 0, vb = 0, hb = 0, cb = 0, ekb = 0, Vnb = 0, icb = 0, ihb = 0;
#pragma unroll kCharsUnroll
    for (int k = 0; k < 4; k++) {
        const double QLb = R[0][k] * clb[0] + R[1][k] * clb[1] + R[2][k] * clb[2] + R[3][k] * clb[3];
        const double QRb = R[0][k] * crb[0] + R[1][k] * crb[1] + R[2][k] * crb[2] + R[3][k] * crb[3];
        double q[6];
        char_field(k, q);
        double qb[6] = {0, 0, 0, 0, 0, 0};
        interp5_adj(fam, q, flL[k], QLb, qb);
        const double qm[5] = {q[5], q[4], q[3], q[2], q[1]};
        double qmb[5] = {0, 0, 0, 0, 0};
        interp5_adj(fam, qm, flR[k], QRb, qmb);
        qb[5] += qmb[0]; qb[4] += qmb[1]; qb[3] += qmb[2]; qb[2] += qmb[3]; qb[1] += qmb[4];
        double Lb[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            double lb = 0.0;
#pragma unroll
            for (int j = 0; j < 6; j++) {
                Ub[j][m] += L[k][m] * qb[j];
                lb += qb[j] * U[j][m];
            }
            Lb[m] = lb;
        }
        if (k == 0) {
            ub += -ny * Lb[0]; vb += nx * Lb[0];
        } else if (k == 1) {
            hb += Lb[0]; ekb -= Lb[0]; ub += Lb[1]; vb += Lb[2];
        } else {  // rows 2 and 3 differ in the sign of their 1/c terms
            const double sg = (k == 2) ? 1.0 : -1.0;
            const double g0 = 0.5 * Lb[0], g1 = 0.5 * Lb[1], g2 = 0.5 * Lb[2], g3 = 0.5 * Lb[3];
            Vnb += sg * ic * g0; icb += sg * Vn * g0; ekb += ih * g0; ihb += ek * g0;
            icb -= sg * nx * g1; ub -= ih * g1; ihb -= u * g1;
            icb -= sg * ny * g2; vb -= ih * g2; ihb -= v * g2;
            ihb += g3;
        }
    }
    // adjoint of R entry (i, k)
    auto Rb = [&](int i, int k) { return QL[k] * clb[i] + QR[k] * crb[i]; };
    ub += ny * Rb(3, 0); vb -= nx * Rb(3, 0);
    ihb += Rb(0, 1) + u * Rb(1, 1) + v * Rb(2, 1) + ek * Rb(3, 1);
    ub += ih * Rb(1, 1); vb += ih * Rb(2, 1); ekb += ih * Rb(3, 1);
    ub += Rb(1, 2); cb -= nx * Rb(1, 2); vb += Rb(2, 2); cb -= ny * Rb(2, 2);
    hb += Rb(3, 2); ekb += Rb(3, 2); Vnb -= c * Rb(3, 2); cb -= Vn * Rb(3, 2);
    ub += Rb(1, 3); cb += nx * Rb(1, 3); vb += Rb(2, 3); cb += ny * Rb(2, 3);
    hb += Rb(3, 3); ekb += Rb(3, 3); Vnb += c * Rb(3, 3); cb += Vn * Rb(3, 3);
    cb -= ic * ic * icb;
    hb -= ih * ih * ihb;
    hb += cb * kGm1 * 0.5 * ic;
    ub += nx * Vnb; vb += ny * Vnb;
    const double htb = hb;
    ekb -= hb;
    ub += u * ekb; vb += v * ekb;
    // Roe average -> prims of cells 2 and 3
    const double uLb = s1 * iA * ub, uRb = s2 * iA * ub, vLb = s1 * iA * vb, vRb = s2 * iA * vb;
    const double HLb = s1 * iA * htb, HRb = s2 * iA * htb;
    const double s1b = iA * ((P2[1] - u) * ub + (P2[2] - v) * vb + (HL - ht) * htb);
    const double s2b = iA * ((P3[1] - u) * ub + (P3[2] - v) * vb + (HR - ht) * htb);
    // 1/rho and 1/sqrt(rho) = sqrt(rho)/rho of both cells from one reciprocal each
    const double i2 = e.i2, i3 = e.i3;
    P2b[1] += uLb + P2[1] * HLb; P2b[2] += vLb + P2[2] * HLb; P2b[3] += kGG1 * i2 * HLb;
    P2b[0] += -kGG1 * P2[3] * (i2 * i2) * HLb + s1b * 0.5 * (s1 * i2);
    P3b[1] += uRb + P3[1] * HRb; P3b[2] += vRb + P3[2] * HRb; P3b[3] += kGG1 * i3 * HRb;
    P3b[0] += -kGG1 * P3[3] * (i3 * i3) * HRb + s2b * 0.5 * (s2 * i3);
    c2p_adj(P2, i2, P2b, Ub[2]);
    c2p_adj(P3, i3, P3b, Ub[3]);
}

// Forward face flux of stencil U[6][4] and Ub += (dF/dU)^T Fb; interpolation
// family fam (AdjInterp) with constant ct.
template <int AX>
ADJ_HD void face_vjp(const double (&U)[6][4], const double *Fb, double (&Ub)[6][4], int fam = ADJ_WCNS5,
                     double ct = 0.0)
{
    FaceStates f;
    face_vjp_states<AX>(U, Fb, f, fam, ct);
    face_vjp_chars<AX>(U, f, Ub, fam);
}

// node flux (fluxSolveEuler2D) adjoint w.r.t. the cell's cons: cb += (dG/dU)^T Gb
template <int AX>
ADJ_HD void node_vjp(const double *U, const double *Gb, double *cb)
{
    constexpr double nx = (AX == 0) ? 1.0 : 0.0, ny = (AX == 1) ? 1.0 : 0.0;
    double p[4];
    const double ir = c2p(U, p);
    const double r = p[0], u = p[1], v = p[2], pp = p[3];
    const double Vn = nx * u + ny * v, q2 = u * u + v * v;
    double pb[4];
    pb[0] = Vn * Gb[0] + u * Vn * Gb[1] + v * Vn * Gb[2] + 0.5 * q2 * Vn * Gb[3];
    const double Vnb = r * Gb[0] + r * u * Gb[1] + r * v * Gb[2] + (0.5 * q2 * r + kGG1 * pp) * Gb[3];
    pb[1] = r * Vn * Gb[1] + u * r * Vn * Gb[3] + nx * Vnb;
    pb[2] = r * Vn * Gb[2] + v * r * Vn * Gb[3] + ny * Vnb;
    pb[3] = nx * Gb[1] + ny * Gb[2] + kGG1 * Vn * Gb[3];
    c2p_adj(p, ir, pb, cb);
}


// ---- forward formulas in a generic real type (the CPU tests evaluate them in
// long double for finite differences; the kernels use the adjoints above)
template <class T>
ADJ_HD void c2p_t(const T *c, T *p)
{
    const T ir = T(1) / c[0];
    p[0] = c[0];
    p[1] = c[1] * ir;
    p[2] = c[2] * ir;
    p[3] = T(kGm1) * (c[3] - (c[1] * c[1] + c[2] * c[2]) * (T(0.5) * ir));
}

template <class T>
ADJ_HD T wcns5_t(const T *q)
{
    const T a0 = q[0] - 2 * q[1] + q[2], b0 = q[0] - 4 * q[1] + 3 * q[2];
    const T a1 = q[1] - 2 * q[2] + q[3], b1 = q[1] - q[3];
    const T a2 = q[2] - 2 * q[3] + q[4], b2 = 3 * q[2] - 4 * q[3] + q[4];
    const T s0 = T(1e-6) + a0 * a0 + T(0.25) * b0 * b0, s1 = T(1e-6) + a1 * a1 + T(0.25) * b1 * b1,
            s2 = T(1e-6) + a2 * a2 + T(0.25) * b2 * b2;
    const T al0 = (T(1) / 16) / (s0 * s0), al1 = (T(5) / 8) / (s1 * s1), al2 = (T(5) / 16) / (s2 * s2);
    const T u0 = T(0.375) * q[0] - T(1.25) * q[1] + T(1.875) * q[2];
    const T u1 = T(-0.125) * q[1] + T(0.75) * q[2] + T(0.375) * q[3];
    const T u2 = T(0.375) * q[2] + T(0.75) * q[3] - T(0.125) * q[4];
    return (al0 * u0 + al1 * u1 + al2 * u2) / (al0 + al1 + al2);
}

template <class T, int AX>
ADJ_HD void roe_t(const T *L, const T *R, T *res)
{
    using std::fabs;
    using std::sqrt;
    const T n[2] = {T(AX == 0 ? 1 : 0), T(AX == 1 ? 1 : 0)};
    const T rl = L[0], pl = L[3], rr = R[0], pr = R[3];
    const T vl[2] = {L[1], L[2]}, vr[2] = {R[1], R[2]};
    const T kl = vl[0] * vl[0] + vl[1] * vl[1], kr = vr[0] * vr[0] + vr[1] * vr[1];
    const T VnL = vl[AX], VnR = vr[AX];
    T Fc[4];
    Fc[0] = rl * VnL + rr * VnR;
    for (int i = 0; i < 2; i++) Fc[1 + i] = rl * vl[i] * VnL + rr * vr[i] * VnR + (pl + pr) * n[i];
    Fc[3] = (T(0.5) * rl * kl + T(kGG1) * pl) * VnL + (T(0.5) * rr * kr + T(kGG1) * pr) * VnR;
    const T s1 = sqrt(rl), s2 = sqrt(rr), iA = T(1) / (s1 + s2), rhoA = s1 * s2;
    const T vA[2] = {(s1 * vl[0] + s2 * vr[0]) * iA, (s1 * vl[1] + s2 * vr[1]) * iA};
    const T HL = T(0.5) * kl + T(kGG1) * pl / rl, HR = T(0.5) * kr + T(kGG1) * pr / rr;
    const T HA = (s1 * HL + s2 * HR) * iA;
    const T q2 = T(0.5) * (vA[0] * vA[0] + vA[1] * vA[1]);
    const T c2 = T(kGm1) * (HA - q2), c = sqrt(c2), ic2 = T(1) / c2;
    const T VnA = vA[AX];
    const T x[3] = {VnA - c, VnA, VnA + c};
    const T eps = T(0.05) * (fabs(VnA) + c);
    T lam[3];
    for (int i = 0; i < 3; i++) {
        lam[i] = fabs(x[i]);
        if (lam[i] < eps) lam[i] = (lam[i] * lam[i] + eps * eps) / (2 * eps);
    }
    const T dP = pr - pl, dVn = VnR - VnL, dRho = rr - rl, rc = rhoA * c * dVn;
    const T a1 = lam[0] * (dP - rc) * (T(0.5) * ic2), a3 = lam[2] * (dP + rc) * (T(0.5) * ic2);
    const T a2 = lam[1] * (dRho - dP * ic2), l1r = lam[1] * rhoA;
    T Fd[4], tE = 0;
    Fd[0] = a1 + a3 + a2;
    for (int i = 0; i < 2; i++) {
        const T ti = (i == AX) ? T(0) : vr[i] - vl[i];
        Fd[1 + i] = a1 * (vA[i] - c * n[i]) + a3 * (vA[i] + c * n[i]) + a2 * vA[i] + l1r * ti;
        if (i != AX) tE += vA[i] * ti;
    }
    Fd[3] = a1 * (HA - c * VnA) + a3 * (HA + c * VnA) + a2 * q2 + l1r * tE;
    for (int i = 0; i < 4; i++) res[i] = T(0.5) * (Fc[i] - Fd[i]);
}

// interp5 in the generic type (flag from the same decision in T)
template <class T>
ADJ_HD T interp5_t(int fam, const T *q, double ct)
{
    if (fam == ADJ_WCNS5) return wcns5_t(q);
    T a[5];
    teno_coeffs(teno_flag(fam, q, ct), a);
    return a[0] * q[0] + a[1] * q[1] + a[2] * q[2] + a[3] * q[3] + a[4] * q[4];
}

template <class T, int AX>
ADJ_HD void face_flux_t(const T (&U)[6][4], T *F, int fam = ADJ_WCNS5, double ct = 0.0)
{
    using std::sqrt;
    const T nx = T(AX == 0 ? 1 : 0), ny = T(AX == 1 ? 1 : 0);
    T P2[4], P3[4];
    c2p_t(U[2], P2);
    c2p_t(U[3], P3);
    const T s1 = sqrt(P2[0]), s2 = sqrt(P3[0]), iA = T(1) / (s1 + s2);
    const T HL = T(0.5) * (P2[1] * P2[1] + P2[2] * P2[2]) + T(kGG1) * P2[3] / P2[0];
    const T HR = T(0.5) * (P3[1] * P3[1] + P3[2] * P3[2]) + T(kGG1) * P3[3] / P3[0];
    const T u = (s1 * P2[1] + s2 * P3[1]) * iA, v = (s1 * P2[2] + s2 * P3[2]) * iA;
    const T ht = (s1 * HL + s2 * HR) * iA;
    const T ek = T(0.5) * (u * u + v * v), h = ht - ek;
    const T c = sqrt(T(kGm1) * h), ic = T(1) / c, ih = T(1) / h, Vn = nx * u + ny * v;
    T L[4][4], R[4][4];
    L[0][0] = -ny * u + nx * v; L[0][1] = ny; L[0][2] = -nx; L[0][3] = 0;
    L[1][0] = h - ek; L[1][1] = u; L[1][2] = v; L[1][3] = -1;
    L[2][0] = T(0.5) * (Vn * ic + ek * ih); L[2][1] = T(0.5) * (-nx * ic - u * ih); L[2][2] = T(0.5) * (-ny * ic - v * ih);
    L[2][3] = T(0.5) * ih;
    L[3][0] = T(0.5) * (-Vn * ic + ek * ih); L[3][1] = T(0.5) * (nx * ic - u * ih); L[3][2] = T(0.5) * (ny * ic - v * ih);
    L[3][3] = T(0.5) * ih;
    R[0][0] = 0; R[1][0] = ny; R[2][0] = -nx; R[3][0] = ny * u - nx * v;
    R[0][1] = ih; R[1][1] = u * ih; R[2][1] = v * ih; R[3][1] = ek * ih;
    R[0][2] = 1; R[1][2] = u - nx * c; R[2][2] = v - ny * c; R[3][2] = h + ek - Vn * c;
    R[0][3] = 1; R[1][3] = u + nx * c; R[2][3] = v + ny * c; R[3][3] = h + ek + Vn * c;
    T QL[4], QR[4];
    for (int k = 0; k < 4; k++) {
        T q[6];
        for (int j = 0; j < 6; j++) q[j] = L[k][0] * U[j][0] + L[k][1] * U[j][1] + L[k][2] * U[j][2] + L[k][3] * U[j][3];
        const T qm[5] = {q[5], q[4], q[3], q[2], q[1]};
        QL[k] = interp5_t(fam, q, ct);
        QR[k] = interp5_t(fam, qm, ct);
    }
    T cl[4], cr[4], fl[4], fr[4];
    for (int i = 0; i < 4; i++) {
        cl[i] = R[i][0] * QL[0] + R[i][1] * QL[1] + R[i][2] * QL[2] + R[i][3] * QL[3];
        cr[i] = R[i][0] * QR[0] + R[i][1] * QR[1] + R[i][2] * QR[2] + R[i][3] * QR[3];
    }
    c2p_t(cl, fl);
    c2p_t(cr, fr);
    if (fl[0] < 0 || fl[3] < 0)
        for (int i = 0; i < 4; i++) fl[i] = P2[i];
    if (fr[0] < 0 || fr[3] < 0) {
        fr[0] = P3[0]; fr[1] = P2[1]; fr[2] = P2[2]; fr[3] = P3[3];
    }
    roe_t<T, AX>(fl, fr, F);
}

template <class T, int AX>
ADJ_HD void node_flux_t(const T *U, T *G)
{
    const T nx = T(AX == 0 ? 1 : 0), ny = T(AX == 1 ? 1 : 0);
    T p[4];
    c2p_t(U, p);
    const T Vn = nx * p[1] + ny * p[2], q2 = p[1] * p[1] + p[2] * p[2];
    G[0] = p[0] * Vn;
    G[1] = p[0] * p[1] * Vn + nx * p[3];
    G[2] = p[0] * p[2] * Vn + ny * p[3];
    G[3] = (q2 / 2 * p[0] + T(kGG1) * p[3]) * Vn;
}

} // namespace adj
} // namespace cfd
