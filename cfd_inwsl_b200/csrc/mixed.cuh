// Mixed FP32/FP64 face reconstruction (cfd_config.precision = CFD_PREC_MIXED).
//
// The characteristic projection, the five-point interpolations and the back
// projection run in FP32, the Riemann flux, the MND6 difference, the state and
// the RK combination stay FP64. FP32 works on increments, not on the values:
// every stencil value enters as its FP64 difference to the stencil's centre
// cell (j = 2), which is O(h) in smooth regions, so FP32 rounding is relative
// to the increment and the rebuilt FP64 face state keeps about seven digits of
// the increment instead of seven digits of the state. All interpolators are
// invariant under adding a constant to the stencil (their smoothness measures
// use differences and their candidate stencils sum to one), so interpolating
// the increments and adding the centre value back is the same reconstruction.
//
// FP32 cannot hold the FP64 constants of the TENO family as they are:
//   * eps = 1e-40 is below FP32's normal range: 1e-30 is used;
//   * (1 + tau/beta)^6 overflows FP32 once tau/beta exceeds ~2.6e6: the cut-off
//     test measure_k < c * sum_j measure_j is evaluated on measures divided by
//     the largest one, which leaves the decision unchanged;
//   * WENO-Z's (tau/beta)^2 is capped at 1e36 for the same reason.
#pragma once
#include "euler_math.cuh"

namespace cfd {

template <int FAM>
__device__ __forceinline__ float inter5f(float q0, float q1, float q2, float q3, float q4, float c)
{
    float b0, b1, b2;
    {
        float a = q0 - 2.0f * q1 + q2, b = q0 - 4.0f * q1 + 3.0f * q2;
        b0 = a * a + 0.25f * (b * b);
        a = q1 - 2.0f * q2 + q3;
        b = q1 - q3;
        b1 = a * a + 0.25f * (b * b);
        a = q2 - 2.0f * q3 + q4;
        b = 3.0f * q2 - 4.0f * q3 + q4;
        b2 = a * a + 0.25f * (b * b);
    }
    if constexpr (FAM == FAM_WCNS5 || FAM == FAM_WENOZ) {
        const float u0 = 0.375f * q0 - 1.25f * q1 + 1.875f * q2;
        const float u1 = -0.125f * q1 + 0.75f * q2 + 0.375f * q3;
        const float u2 = 0.375f * q2 + 0.75f * q3 - 0.125f * q4;
        float w0, w1, w2;
        if constexpr (FAM == FAM_WCNS5) {
            float s0 = 1e-6f + b0, s1 = 1e-6f + b1, s2 = 1e-6f + b2;
            s0 *= s0; s1 *= s1; s2 *= s2;
            // weights gamma_k / s_k (s_k >= 1e-12: no overflow)
            w0 = 0.0625f * __fdividef(1.0f, s0);
            w1 = 0.625f * __fdividef(1.0f, s1);
            w2 = 0.3125f * __fdividef(1.0f, s2);
        } else {
            const float tau = fabsf(b2 - b0);
            float x;
            x = fminf(tau / (b0 + 1e-30f), 1e18f); w0 = 0.0625f * (1.0f + x * x);
            x = fminf(tau / (b1 + 1e-30f), 1e18f); w1 = 0.625f * (1.0f + x * x);
            x = fminf(tau / (b2 + 1e-30f), 1e18f); w2 = 0.3125f * (1.0f + x * x);
        }
        return (w0 * u0 + w1 * u1 + w2 * u2) / (w0 + w1 + w2);
    } else if constexpr (FAM == FAM_TENOZ) {
        const float tau = fabsf(b2 - b0);
        float t0 = 1.0f + tau / (b0 + 1e-30f), t1 = 1.0f + tau / (b1 + 1e-30f), t2 = 1.0f + tau / (b2 + 1e-30f);
        const float tm = fmaxf(t0, fmaxf(t1, t2));
        const float itm = 1.0f / tm;
        t0 *= itm; t1 *= itm; t2 *= itm;
        float m0 = t0 * t0, m1 = t1 * t1, m2 = t2 * t2;
        m0 = m0 * m0 * m0; m1 = m1 * m1 * m1; m2 = m2 * m2 * m2;
        const float CT = c * (m0 + m1 + m2);
        unsigned flag = (m0 < CT ? 1u : 0u) + (m1 < CT ? 2u : 0u) + (m2 < CT ? 4u : 0u);
        switch (flag) {
        case 0: return 0.0234375f * q0 - 0.15625f * q1 + 0.703125f * q2 + 0.46875f * q3 - 0.0390625f * q4;
        case 1: return -0.0625f * q1 + 0.5625f * q2 + 0.5625f * q3 - 0.0625f * q4;
        case 2:
        case 3: return 0.375f * q2 + 0.75f * q3 - 0.125f * q4;
        case 4: return 0.0625f * q0 - 0.3125f * q1 + 0.9375f * q2 + 0.3125f * q3;
        case 5: return -0.125f * q1 + 0.75f * q2 + 0.375f * q3;
        case 6: return 0.375f * q0 - 1.25f * q1 + 1.875f * q2;
        default: return q2;
        }
    } else if constexpr (FAM == FAM_TENOCONG) {
        float bmin = b0;
        if (b1 < bmin) bmin = b1;
        if (b2 < bmin) bmin = b2;
        const float tau = fabsf(b2 - b0);
        const float rr = c * tau - (1.0f - c) * bmin, ll = tau * bmin;
        unsigned flag = (ll < rr * b0 ? 1u : 0u) + (ll < rr * b1 ? 2u : 0u) + (ll < rr * b2 ? 4u : 0u);
        switch (flag) {
        case 0: return 0.0234375f * q0 - 0.15625f * q1 + 0.703125f * q2 + 0.46875f * q3 - 0.0390625f * q4;
        case 1: return -0.0625f * q1 + 0.5625f * q2 + 0.5625f * q3 - 0.0625f * q4;
        case 2:
        case 3: return 0.375f * q2 + 0.75f * q3 - 0.125f * q4;
        case 4: return 0.0625f * q0 - 0.3125f * q1 + 0.9375f * q2 + 0.3125f * q3;
        case 5: return -0.125f * q1 + 0.75f * q2 + 0.375f * q3;
        case 6: return 0.375f * q0 - 1.25f * q1 + 1.875f * q2;
        default: return q2;
        }
    } else {
        const float dm = q2 - q1, dp = q3 - q2;
        float d;
        if (dp > 0.0f) d = fmaxf(0.0f, fmaxf(fminf(dm, dp), fminf(dm, dp)));
        else d = fminf(0.0f, fminf(fmaxf(dm, dp), fmaxf(dm, dp)));
        return q2 + 0.5f * d;
    }
}

// Roe-averaged eigenvectors in FP32 from the FP64 base quantities.
template <int NV, int AX>
struct EigenF {
    float u, v, w, h, c, ek, Vn, ic, ih;
    static constexpr float nx = (AX == 0) ? 1.0f : 0.0f, ny = (AX == 1) ? 1.0f : 0.0f, nz = (AX == 2) ? 1.0f : 0.0f;
    template <class PR>
    __device__ __forceinline__ EigenF(const PR &pr)
    {
        constexpr int D = NV - 2;
        double vl[3] = {pr(2, 1), pr(2, 2), D == 3 ? pr(2, 3) : 0.0};
        double vr[3] = {pr(3, 1), pr(3, 2), D == 3 ? pr(3, 3) : 0.0};
        double rl = pr(2, 0), rr = pr(3, 0), pL = pr(2, NV - 1), pR = pr(3, NV - 1);
        float kl = (float)(vl[0] * vl[0] + vl[1] * vl[1] + vl[2] * vl[2]);
        float kr = (float)(vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]);
        const float g1 = (float)(kGamma / (kGamma - 1));
        float HL = 0.5f * kl + (float)pL * (g1 / (float)rl);
        float HR = 0.5f * kr + (float)pR * (g1 / (float)rr);
        float c1 = sqrtf((float)rl), c2 = sqrtf((float)rr);
        float dv = 1.0f / (c1 + c2);
        u = (c1 * (float)vl[0] + c2 * (float)vr[0]) * dv;
        v = (c1 * (float)vl[1] + c2 * (float)vr[1]) * dv;
        w = (c1 * (float)vl[2] + c2 * (float)vr[2]) * dv;
        float ht = (c1 * HL + c2 * HR) * dv;
        Vn = nx * u + ny * v + nz * w;
        ek = 0.5f * (u * u + v * v + w * w);
        h = ht - ek;
        c = sqrtf((float)(kGamma - 1) * h);
        ic = 1.0f / c;
        ih = 1.0f / h;
    }
    __device__ __forceinline__ float L(int k, int m) const
    {
        constexpr int E = NV - 1;
        if (k == 0) {
            if (AX != 2) return m == 0 ? (-ny * u + nx * v) : m == 1 ? ny : m == 2 ? (-nx) : 0.0f;
            return m == 0 ? -u : m == 1 ? 1.0f : 0.0f;
        }
        if (k == 1) return m == 0 ? (h - ek) : m == 1 ? u : m == 2 ? v : m == E ? -1.0f : w;
        if (k == 2 || k == 3) {
            const float s = (k == 2) ? -1.0f : 1.0f;
            if (m == E) return 0.5f * ih;
            if (m == 0) return 0.5f * (-s * Vn * ic + ek * ih);
            if (m == 1) return 0.5f * (s * nx * ic - u * ih);
            if (m == 2) return 0.5f * (s * ny * ic - v * ih);
            return 0.5f * (s * nz * ic - w * ih);
        }
        if (AX != 2) return m == 0 ? -w : m == 3 ? 1.0f : 0.0f;
        return m == 0 ? -v : m == 2 ? 1.0f : 0.0f;
    }
    __device__ __forceinline__ float R(int i, int k) const
    {
        constexpr int E = NV - 1;
        if (k == 0) {
            if (AX != 2) return i == 1 ? ny : i == 2 ? -nx : i == E ? ny * u - nx * v : 0.0f;
            return i == 1 ? 1.0f : i == E ? u : 0.0f;
        }
        if (k == 1) return (i == 0 ? 1.0f : i == 1 ? u : i == 2 ? v : i == E ? ek : w) * ih;
        if (k == 2 || k == 3) {
            const float s = (k == 2) ? -1.0f : 1.0f;
            if (i == 0) return 1.0f;
            if (i == E) return h + ek + s * Vn * c;
            if (i == 1) return u + s * nx * c;
            if (i == 2) return v + s * ny * c;
            return w + s * nz * c;
        }
        if (AX != 2) return i == 3 ? 1.0f : i == 4 ? w : 0.0f;
        return i == 2 ? 1.0f : i == 4 ? v : 0.0f;
    }
};

// The linear five-point interpolation (all three candidate stencils with
// their ideal weights, interScheme.hpp:148-149).
__device__ __forceinline__ float lin5f(float q0, float q1, float q2, float q3, float q4)
{
    return 0.0234375f * q0 - 0.15625f * q1 + 0.703125f * q2 + 0.46875f * q3 - 0.0390625f * q4;
}

// cs(j, v) / pr(j, v): FP64 cons and prim of stencil cell j; writes FP64 face prims.
//
// The face increment is split as U_face - U_2 = Lin(dU) + R (NL(q) - Lin(q)),
// q = L dU, which equals R NL(L dU) in exact arithmetic because the linear
// interpolation commutes with the projection. The linear part is interpolated
// component by component, so its FP32 error is relative to dU itself; only the
// nonlinear correction passes through the FP32 eigenvectors, whose R L differs
// from the identity by about 1e-7 times their condition number (large at low
// Mach number, where h = c^2/(gamma-1) dominates). The correction vanishes
// where the scheme is linear (TENO with every stencil kept) and is small
// wherever the data are smooth.
template <int NV, int AX, int FAM, class CS, class PR>
__device__ __forceinline__ void reconstruct_face_mixed(const CS &cs, const PR &pr, double icst, double *fl,
                                                       double *fr)
{
    const EigenF<NV, AX> eb(pr);
    // increments of the stencil cons relative to cell 2, in FP32
    float d[6][NV];
#pragma unroll
    for (int j = 0; j < 6; j++)
#pragma unroll
        for (int m = 0; m < NV; m++) d[j][m] = (j == 2) ? 0.0f : (float)(cs(j, m) - cs(2, m));
    float dl[NV], dr[NV];
#pragma unroll
    for (int i = 0; i < NV; i++) {
        dl[i] = lin5f(d[0][i], d[1][i], d[2][i], d[3][i], d[4][i]);
        dr[i] = lin5f(d[5][i], d[4][i], d[3][i], d[2][i], d[1][i]);
    }
    const float fc = (float)icst;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        float l[NV];
#pragma unroll
        for (int m = 0; m < NV; m++) l[m] = eb.L(k, m);
        float q[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {
            float a = 0.0f;
#pragma unroll
            for (int m = 0; m < NV; m++) a += d[j][m] * l[m];
            q[j] = a;
        }
        const float CL = inter5f<FAM>(q[0], q[1], q[2], q[3], q[4], fc) - lin5f(q[0], q[1], q[2], q[3], q[4]);
        const float CR = inter5f<FAM>(q[5], q[4], q[3], q[2], q[1], fc) - lin5f(q[5], q[4], q[3], q[2], q[1]);
#pragma unroll
        for (int i = 0; i < NV; i++) {
            const float r = eb.R(i, k);
            dl[i] += CL * r;
            dr[i] += CR * r;
        }
    }
    double cl[NV], cr[NV];
#pragma unroll
    for (int i = 0; i < NV; i++) {
        const double base = cs(2, i);
        cl[i] = base + (double)dl[i];
        cr[i] = base + (double)dr[i];
    }
    char_cons_to_prim<NV>(cl, fl);
    char_cons_to_prim<NV>(cr, fr);
    if (fl[0] < 0 || fl[NV - 1] < 0) {
        for (int i = 0; i < NV; i++) fl[i] = pr(2, i);
    }
    if (fr[0] < 0 || fr[NV - 1] < 0) {
        fr[0] = pr(3, 0);
        for (int i = 1; i < NV - 1; i++) fr[i] = pr(2, i);
        fr[NV - 1] = pr(3, NV - 1);
    }
}

} // namespace cfd
