// Mixed FP32/FP64 face reconstruction and Roe flux (cfd_config.precision =
// CFD_PREC_MIXED).
//
// The state, the face values fed to the Riemann solver, the central part of
// the flux, the MND6 difference and the RK combination stay FP64. FP32 does the
// work whose rounding the scheme does not see:
//
//   * TENO families (flag-selected stencils): the smoothness measures and the
//     cut-off decision of every characteristic field run in FP32. When one side
//     of a face selects the same stencil in every field, the characteristic
//     projection and its inverse cancel (R L = I), so the face value is that
//     stencil applied to the FP64 cons component by component; otherwise the
//     FP64 projection is applied with the FP32-selected stencils. Either way the
//     face value is an FP64 linear combination of FP64 cells: FP32 only decides
//     which combination, and a decision can differ from the FP64 one only where
//     a stencil's measure sits within FP32 rounding of the cut-off.
//   * Continuous-weight families (WCNS5, WENO-Z, MUSCL): the face increment is
//     split into the component-wise linear interpolation (FP32 on increments,
//     error relative to the increment) plus the characteristic nonlinear
//     correction R (NL(L dU) - Lin(L dU)) in FP32.
//   * Roe flux: the central part (F_L + F_R) / 2 in FP64, the upwind
//     dissipation R |Lambda| L (U_R - U_L) / 2 in FP32 from FP64 jumps; the
//     dissipation is O(jump), small wherever the data are smooth.
//   * HLLC flux: the upwind side's physical flux in FP64, the wave speeds and
//     the star-state correction S_K (U*_K - U_K), which is O(jump), in FP32.
//
// FP32 works on increments, never on the values: every stencil value enters as
// cons(j) - cons(2), formed from an FP32 hi/lo split of each cell's cons
// (hi = (float)U, lo = (float)(U - hi)), so neighbouring hi parts subtract
// exactly and the increment keeps about seven digits of itself. All
// interpolators are invariant under adding a constant to the stencil (their
// smoothness measures use differences and their candidate stencils sum to one).
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

// The 3-bit cut-off flag of the TENO families in FP32 (bit k set = stencil k
// cut), the decision of inter5<FAM_TENOZ / FAM_TENOCONG> in euler_math.cuh.
template <int FAM>
__device__ __forceinline__ unsigned teno_flag_f(float q0, float q1, float q2, float q3, float q4, float c, float kap)
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
    const float tau = fabsf(b2 - b0);
    if constexpr (FAM == FAM_TENOZ) {
        {
            // the keep-all bound of teno_z_all_kept (euler_math.cuh)
            const float s0 = b0 + 1e-30f, s1 = b1 + 1e-30f, s2 = b2 + 1e-30f;
            const float smin = fminf(s0, fminf(s1, s2)), smax = fmaxf(s0, fmaxf(s1, s2));
            const float rhs = (smin + tau) * smax;
            if (rhs < 1e36f && (smax + tau) * smin >= kap * rhs) return 0u;
        }
        float t0 = 1.0f + __fdividef(tau, b0 + 1e-30f), t1 = 1.0f + __fdividef(tau, b1 + 1e-30f),
              t2 = 1.0f + __fdividef(tau, b2 + 1e-30f);
        const float itm = __fdividef(1.0f, fmaxf(t0, fmaxf(t1, t2)));
        t0 *= itm; t1 *= itm; t2 *= itm;
        float m0 = t0 * t0, m1 = t1 * t1, m2 = t2 * t2;
        m0 = m0 * m0 * m0; m1 = m1 * m1 * m1; m2 = m2 * m2 * m2;
        const float CT = c * (m0 + m1 + m2);
        return (m0 < CT ? 1u : 0u) + (m1 < CT ? 2u : 0u) + (m2 < CT ? 4u : 0u);
    } else {
        float bmin = b0;
        if (b1 < bmin) bmin = b1;
        if (b2 < bmin) bmin = b2;
        const float rr = c * tau - (1.0f - c) * bmin, ll = tau * bmin;
        return (ll < rr * b0 ? 1u : 0u) + (ll < rr * b1 ? 2u : 0u) + (ll < rr * b2 ? 4u : 0u);
    }
}

// The cut-off decision of a TENO family from its three smoothness measures
// (the part of teno_flag_f after the measures), for one stencil.
template <int FAM>
__device__ __noinline__ unsigned teno_flag_beta(float b0, float b1, float b2, float tau, float c)
{
    if constexpr (FAM == FAM_TENOZ) {
        float t0 = 1.0f + __fdividef(tau, b0 + 1e-30f), t1 = 1.0f + __fdividef(tau, b1 + 1e-30f),
              t2 = 1.0f + __fdividef(tau, b2 + 1e-30f);
        const float itm = __fdividef(1.0f, fmaxf(t0, fmaxf(t1, t2)));
        t0 *= itm; t1 *= itm; t2 *= itm;
        float m0 = t0 * t0, m1 = t1 * t1, m2 = t2 * t2;
        m0 = m0 * m0 * m0; m1 = m1 * m1 * m1; m2 = m2 * m2 * m2;
        const float CT = c * (m0 + m1 + m2);
        return (m0 < CT ? 1u : 0u) + (m1 < CT ? 2u : 0u) + (m2 < CT ? 4u : 0u);
    } else {
        float bmin = b0;
        if (b1 < bmin) bmin = b1;
        if (b2 < bmin) bmin = b2;
        const float rr = c * tau - (1.0f - c) * bmin, ll = tau * bmin;
        return (ll < rr * b0 ? 1u : 0u) + (ll < rr * b1 ? 2u : 0u) + (ll < rr * b2 ? 4u : 0u);
    }
}

// Both faces' stencils of one characteristic field at once, in packed FP32
// pairs (one FFMA2 / FADD2 / FMUL2 instruction per pair): Q_i = (q_i, q_{5-i}),
// so the left stencil q0..q4 is the .x lane of Q0..Q4 and the mirrored right
// stencil q5..q1 the .y lane. Q3 and Q4 are Q2 and Q1 with the lanes swapped.
template <int FAM>
__device__ __forceinline__ void teno_flags2(float2 Q0, float2 Q1, float2 Q2, float c, float kap, unsigned &fl,
                                            unsigned &fr)
{
    const float2 Q3 = make_float2(Q2.y, Q2.x), Q4 = make_float2(Q1.y, Q1.x);
    const float2 m1 = make_float2(-1.0f, -1.0f), m2 = make_float2(-2.0f, -2.0f), m4 = make_float2(-4.0f, -4.0f),
                 p3 = make_float2(3.0f, 3.0f), h = make_float2(0.5f, 0.5f);
    float2 a = __ffma2_rn(m2, Q1, __fadd2_rn(Q0, Q2));
    float2 b = __fmul2_rn(h, __ffma2_rn(p3, Q2, __ffma2_rn(m4, Q1, Q0)));
    const float2 B0 = __ffma2_rn(a, a, __fmul2_rn(b, b));
    a = __ffma2_rn(m2, Q2, __fadd2_rn(Q1, Q3));
    b = __fmul2_rn(h, __ffma2_rn(m1, Q3, Q1));
    const float2 B1 = __ffma2_rn(a, a, __fmul2_rn(b, b));
    a = __ffma2_rn(m2, Q3, __fadd2_rn(Q2, Q4));
    b = __fmul2_rn(h, __ffma2_rn(p3, Q2, __ffma2_rn(m4, Q3, Q4)));
    const float2 B2 = __ffma2_rn(a, a, __fmul2_rn(b, b));
    float2 T = __ffma2_rn(m1, B0, B2);
    T.x = fabsf(T.x);
    T.y = fabsf(T.y);
    bool keep_x = false, keep_y = false;
    if constexpr (FAM == FAM_TENOZ) {
        // the keep-all bound of teno_z_all_kept (euler_math.cuh), per lane
        const float2 e = make_float2(1e-30f, 1e-30f);
        const float2 S0 = __fadd2_rn(B0, e), S1 = __fadd2_rn(B1, e), S2 = __fadd2_rn(B2, e);
        const float2 smin = make_float2(fminf(S0.x, fminf(S1.x, S2.x)), fminf(S0.y, fminf(S1.y, S2.y)));
        const float2 smax = make_float2(fmaxf(S0.x, fmaxf(S1.x, S2.x)), fmaxf(S0.y, fmaxf(S1.y, S2.y)));
        const float2 rhs = __fmul2_rn(__fadd2_rn(smin, T), smax), lhs = __fmul2_rn(__fadd2_rn(smax, T), smin);
        keep_x = rhs.x < 1e36f && lhs.x >= kap * rhs.x;
        keep_y = rhs.y < 1e36f && lhs.y >= kap * rhs.y;
    }
    fl = keep_x ? 0u : teno_flag_beta<FAM>(B0.x, B1.x, B2.x, T.x, c);
    fr = keep_y ? 0u : teno_flag_beta<FAM>(B0.y, B1.y, B2.y, T.y, c);
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
        float HL = 0.5f * kl + (float)pL * __fdividef(g1, (float)rl);
        float HR = 0.5f * kr + (float)pR * __fdividef(g1, (float)rr);
        float c1 = sqrtf((float)rl), c2 = sqrtf((float)rr);
        float dv = __fdividef(1.0f, c1 + c2);
        u = (c1 * (float)vl[0] + c2 * (float)vr[0]) * dv;
        v = (c1 * (float)vl[1] + c2 * (float)vr[1]) * dv;
        w = (c1 * (float)vl[2] + c2 * (float)vr[2]) * dv;
        float ht = (c1 * HL + c2 * HR) * dv;
        Vn = nx * u + ny * v + nz * w;
        ek = 0.5f * (u * u + v * v + w * w);
        h = ht - ek;
        c = sqrtf((float)(kGamma - 1) * h);
        ic = __fdividef(1.0f, c);
        ih = __fdividef(1.0f, h);
    }
    // entries of L that are the constant 0 (skipped in the projections)
    static __device__ __forceinline__ constexpr bool Lzero(int k, int m)
    {
        constexpr int E = NV - 1;
        if (k == 0) {
            if (AX != 2) return m == E || (m == 1 && AX == 0) || (m == 2 && AX == 1) || (NV == 5 && m == 3);
            return m != 0 && m != 1;
        }
        if (k == 4) return (AX != 2) ? (m != 0 && m != 3) : (m != 0 && m != 2);
        return false;
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

// FP64 face states from per-field stencil flags: the characteristic projection
// of reconstruct_face_stream (euler_math.cuh) with the interpolation replaced
// by the selected fixed stencil. fL/fR hold 3 bits per field.
template <int NV, int AX, class CS, class PR>
__device__ __noinline__ void recon_flags64(const CS &cs, const PR &pr, unsigned fL, unsigned fR, double *cl,
                                           double *cr)
{
    const EigenBase<NV, AX> eb(pr);
#pragma unroll
    for (int i = 0; i < NV; i++) cl[i] = cr[i] = 0.0;
#pragma unroll 1
    for (int k = 0; k < NV; k++) {
        double l[NV];
#pragma unroll
        for (int m = 0; m < NV; m++) l[m] = eb.L(k, m);
        double q[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {
            double a = cs(j, 1) * l[1] + cs(j, 2) * l[2];
#pragma unroll
            for (int m = 3; m < NV; m++) a = a + cs(j, m) * l[m];
            q[j] = a + cs(j, 0) * l[0];
        }
        const double QL = teno_select((fL >> (3 * k)) & 7u, q[0], q[1], q[2], q[3], q[4]);
        const double QR = teno_select((fR >> (3 * k)) & 7u, q[5], q[4], q[3], q[2], q[1]);
#pragma unroll
        for (int i = 0; i < NV; i++) {
            const double r = eb.R(i, k);
            cl[i] = cl[i] + QL * r;
            cr[i] = cr[i] + QR * r;
        }
    }
}

// cs(j, v) / pr(j, v): FP64 cons and prim of stencil cell j; hl(j, v): the FP32
// hi/lo split (hi, lo) of cons(j, v), whose differences to cell 2 give the FP32
// increments. Writes FP64 face prims.
//
// Continuous-weight families: the face increment is split as
// U_face - U_2 = Lin(dU) + R (NL(q) - Lin(q)), q = L dU, which equals
// R NL(L dU) in exact arithmetic because the linear interpolation commutes with
// the projection. The linear part is interpolated component by component, so
// its FP32 error is relative to dU itself; only the nonlinear correction passes
// through the FP32 eigenvectors, whose R L differs from the identity by about
// 1e-7 times their condition number (large at low Mach number, where
// h = c^2/(gamma-1) dominates).
template <int NV, int AX, int FAM, class CS, class PR, class HL>
__device__ __forceinline__ void reconstruct_face_mixed(const CS &cs, const PR &pr, const HL &hl, double icst,
                                                       double kap, double *fl, double *fr)
{
    const EigenF<NV, AX> eb(pr);
    const float fc = (float)icst, fk = (float)kap;
    double cl[NV], cr[NV];
    if constexpr (FAM == FAM_TENOZ || FAM == FAM_TENOCONG) {
        // increments of the stencil pairs (0, 5), (1, 4), (2, 3), packed; cell 2's is 0
        float2 D[3][NV];
        const float2 m1 = make_float2(-1.0f, -1.0f);
#pragma unroll
        for (int m = 0; m < NV; m++) {
            const float2 c2 = hl(2, m), c0 = hl(0, m), c5 = hl(5, m), c1 = hl(1, m), c4 = hl(4, m), c3 = hl(3, m);
            const float2 H2 = make_float2(c2.x, c2.x), L2 = make_float2(c2.y, c2.y);
            D[0][m] = __fadd2_rn(__ffma2_rn(m1, H2, make_float2(c0.x, c5.x)), __ffma2_rn(m1, L2, make_float2(c0.y, c5.y)));
            D[1][m] = __fadd2_rn(__ffma2_rn(m1, H2, make_float2(c1.x, c4.x)), __ffma2_rn(m1, L2, make_float2(c1.y, c4.y)));
            D[2][m] = make_float2(0.0f, (c3.x - c2.x) + (c3.y - c2.y));
        }
        unsigned fL = 0, fR = 0;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            float2 Q[3];
#pragma unroll
            for (int i = 0; i < 3; i++) {
                float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
                for (int m = 0; m < NV; m++) {
                    if (EigenF<NV, AX>::Lzero(k, m)) continue;
                    const float l = eb.L(k, m);
                    acc = __ffma2_rn(make_float2(l, l), D[i][m], acc);
                }
                Q[i] = acc;
            }
            unsigned fl, fr;
            teno_flags2<FAM>(Q[0], Q[1], Q[2], fc, fk, fl, fr);
            fL |= fl << (3 * k);
            fR |= fr << (3 * k);
        }
        // one stencil in every field: R L = I, apply it to the cons directly
        constexpr unsigned kRep = (NV == 4) ? 01111u : 011111u;
        const unsigned sL = fL & 7u, sR = fR & 7u;
        if (fL == sL * kRep && fR == sR * kRep) {
#pragma unroll
            for (int m = 0; m < NV; m++) {
                cl[m] = teno_select(sL, cs(0, m), cs(1, m), cs(2, m), cs(3, m), cs(4, m));
                cr[m] = teno_select(sR, cs(5, m), cs(4, m), cs(3, m), cs(2, m), cs(1, m));
            }
        } else {
            recon_flags64<NV, AX>(cs, pr, fL, fR, cl, cr);
        }
    } else {
        float d[6][NV];
#pragma unroll
        for (int j = 0; j < 6; j++)
#pragma unroll
            for (int m = 0; m < NV; m++) {
                const float2 cj = hl(j, m), c2 = hl(2, m);
                d[j][m] = (j == 2) ? 0.0f : (cj.x - c2.x) + (cj.y - c2.y);
            }
        float dl[NV], dr[NV];
#pragma unroll
        for (int i = 0; i < NV; i++) {
            dl[i] = lin5f(d[0][i], d[1][i], d[2][i], d[3][i], d[4][i]);
            dr[i] = lin5f(d[5][i], d[4][i], d[3][i], d[2][i], d[1][i]);
        }
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
#pragma unroll
        for (int i = 0; i < NV; i++) {
            const double base = cs(2, i);
            cl[i] = base + (double)dl[i];
            cr[i] = base + (double)dr[i];
        }
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

// roeFlux2DSym (fluxSchemes.hpp:420-553) and its 3D extension with the central
// part in FP64 and the dissipation in FP32. rho H = rho |v|^2 / 2 + gamma p /
// (gamma - 1) needs no division in the central part.
template <int NV, int AX>
__device__ __forceinline__ void roe_md_mixed(const double *L, const double *R, double *res)
{
    constexpr int D = NV - 2, E = NV - 1;
    const double n[3] = {AX == 0 ? 1.0 : 0.0, AX == 1 ? 1.0 : 0.0, AX == 2 ? 1.0 : 0.0};
    const double rl = L[0], rr = R[0], pl = L[E], pr = R[E];
    const double *vl = L + 1, *vr = R + 1;
    double kl = vl[0] * vl[0] + vl[1] * vl[1], kr = vr[0] * vr[0] + vr[1] * vr[1];
    if constexpr (D == 3) { kl += vl[2] * vl[2]; kr += vr[2] * vr[2]; }
    const double VnL = vl[AX], VnR = vr[AX];
    constexpr double kg1 = kGamma / (kGamma - 1);
    double Fc[NV];
    Fc[0] = rl * VnL + rr * VnR;
#pragma unroll
    for (int i = 0; i < D; i++) Fc[1 + i] = rl * vl[i] * VnL + rr * vr[i] * VnR + (pl + pr) * n[i];
    Fc[E] = (0.5 * rl * kl + kg1 * pl) * VnL + (0.5 * rr * kr + kg1 * pr) * VnR;

    // jumps in FP64, then FP32
    const float dP = (float)(pr - pl), dVn = (float)(VnR - VnL), dRho = (float)(rr - rl);
    float dv[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int i = 0; i < D; i++) dv[i] = (float)(vr[i] - vl[i]);
    const float rlf = (float)rl, rrf = (float)rr;
    float vlf[3], vrf[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        vlf[i] = i < D ? (float)vl[i] : 0.0f;
        vrf[i] = i < D ? (float)vr[i] : 0.0f;
    }
    const float g1 = (float)kg1;
    const float HL = 0.5f * (float)kl + (float)pl * __fdividef(g1, rlf);
    const float HR = 0.5f * (float)kr + (float)pr * __fdividef(g1, rrf);
    const float c1 = sqrtf(rlf), c2 = sqrtf(rrf);
    const float dvs = __fdividef(1.0f, c1 + c2);
    const float rhoAvg = c1 * c2;
    float vAvg[3];
#pragma unroll
    for (int i = 0; i < 3; i++) vAvg[i] = (c1 * vlf[i] + c2 * vrf[i]) * dvs;
    const float HAvg = (c1 * HL + c2 * HR) * dvs;
    const float q2 = 0.5f * (vAvg[0] * vAvg[0] + vAvg[1] * vAvg[1] + vAvg[2] * vAvg[2]);
    const float cAvg = sqrtf((float)(kGamma - 1) * (HAvg - q2));
    const float VnAvg = vAvg[AX];
    float lam[3] = {fabsf(VnAvg - cAvg), fabsf(VnAvg), fabsf(VnAvg + cAvg)};
    const float eps = 0.05f * (fabsf(VnAvg) + cAvg);
    const float ie2 = __fdividef(0.5f, eps);
#pragma unroll
    for (int i = 0; i < 3; i++)
        if (lam[i] < eps) lam[i] = (lam[i] * lam[i] + eps * eps) * ie2;
    const float ic2 = __fdividef(1.0f, cAvg * cAvg);
    const float a1 = lam[0] * ((dP - rhoAvg * cAvg * dVn) * (0.5f * ic2));
    const float a3 = lam[2] * ((dP + rhoAvg * cAvg * dVn) * (0.5f * ic2));
    const float a2 = lam[1] * (dRho - dP * ic2);
    const float l1r = lam[1] * rhoAvg;
    float Fd[NV];
    Fd[0] = a1 + a3 + a2;
    float tE = 0.0f;
#pragma unroll
    for (int i = 0; i < D; i++) {
        const float ni = (i == AX) ? 1.0f : 0.0f;
        const float ti = (i == AX) ? 0.0f : dv[i];
        Fd[1 + i] = a1 * (vAvg[i] - cAvg * ni) + a3 * (vAvg[i] + cAvg * ni) + a2 * vAvg[i] + l1r * ti;
        if (i != AX) tE += vAvg[i] * dv[i];
    }
    Fd[E] = a1 * (HAvg - cAvg * VnAvg) + a3 * (HAvg + cAvg * VnAvg) + a2 * q2 + l1r * tE;
#pragma unroll
    for (int i = 0; i < NV; i++) res[i] = 0.5 * (Fc[i] - (double)Fd[i]);
}

// HLLC (HLLCFlux2D2, fluxSchemes.hpp, as hllc_md in euler_math.cuh) with the
// physical flux of the upwind side in FP64 and everything of size O(jump) in
// FP32: the wave-speed estimates and the star-state correction
// S_K (U*_K - U_K). Every term of U*_K - U_K carries the factor
// d_K = (S* - Vn_K) / (S_K - S*), and S* - Vn_K is formed from the FP64 jumps
// without cancellation:
//   S* - VnL = (dp - rR (SR - VnR) dVn) / den,  S* - VnR = (dp - rL (SL - VnL) dVn) / den,
//   den = rL (SL - VnL) - rR (SR - VnR)  (two terms of one sign).
// The flux is continuous where the branch (SL > 0, S* > 0, SR > 0) changes,
// so branch decisions taken in FP32 shift it only by rounding of the jump.
template <int NV, int AX>
__device__ __forceinline__ void hllc_md_mixed(const double *L, const double *R, double *res)
{
    constexpr int D = NV - 2, E = NV - 1;
    const double n[3] = {AX == 0 ? 1.0 : 0.0, AX == 1 ? 1.0 : 0.0, AX == 2 ? 1.0 : 0.0};
    const double rl = L[0], rr = R[0], pl = L[E], pr = R[E];
    const double *vl = L + 1, *vr = R + 1;
    double kl = vl[0] * vl[0] + vl[1] * vl[1], kr = vr[0] * vr[0] + vr[1] * vr[1];
    if constexpr (D == 3) { kl += vl[2] * vl[2]; kr += vr[2] * vr[2]; }
    const double VnL = vl[AX], VnR = vr[AX];
    constexpr double kg1 = kGamma / (kGamma - 1);
    // wave speeds in FP32
    const float g = (float)kGamma;
    const float rlf = (float)rl, rrf = (float)rr, plf = (float)pl, prf = (float)pr;
    const float cl = sqrtf(g * __fdividef(plf, rlf)), cr = sqrtf(g * __fdividef(prf, rrf));
    const float dVn = (float)(VnR - VnL), dp = (float)(pr - pl);
    const float ps0 = 0.5f * (plf + prf) - 0.25f * (rlf + rrf) * (0.5f * (cl + cr)) * dVn;
    const float ps = fmaxf(ps0, 0.0f);
    const float gk = (float)((kGamma + 1.0) / (2.0 * kGamma));
    const float ql = (ps <= plf) ? 1.0f : sqrtf(1.0f + gk * (__fdividef(ps, plf) - 1.0f));
    const float qr = (ps <= prf) ? 1.0f : sqrtf(1.0f + gk * (__fdividef(ps, prf) - 1.0f));
    const float aL = -cl * ql, aR = cr * qr;  // SL - VnL, SR - VnR
    const float iden = __fdividef(1.0f, rlf * aL - rrf * aR);
    const float sL = (dp - rrf * aR * dVn) * iden;  // S* - VnL
    const float sR = (dp - rlf * aL * dVn) * iden;  // S* - VnR
    const float VnLf = (float)VnL, VnRf = (float)VnR;
    const float SL = VnLf + aL, SR = VnRf + aR, Sstar = VnLf + sL;

    // FP64 physical flux of one side plus `scale` times its FP32 star correction
    auto side = [&](double r, const double *v, double p, double k, double Vn, float a, float sK, double *out,
                    bool star, double scale, bool accumulate) {
        const double rH = 0.5 * r * k + kg1 * p;  // rho H
        double F[NV];
        F[0] = r * Vn;
#pragma unroll
        for (int i = 0; i < D; i++) F[1 + i] = r * v[i] * Vn + p * n[i];
        F[E] = rH * Vn;
        float C[NV];
#pragma unroll
        for (int i = 0; i < NV; i++) C[i] = 0.0f;
        if (star) {
            const float S = (float)Vn + a;                        // S_K
            const float delta = __fdividef(sK, a - sK);          // (S* - Vn) / (S_K - S*)
            const float rf = (float)r;
            C[0] = S * rf * delta;
#pragma unroll
            for (int i = 0; i < D; i++) C[1 + i] = S * rf * delta * ((i == AX) ? S : (float)v[i]);
            const float UE = (float)(rH - p);
            const float Ss = (float)Vn + sK;                      // S*
            C[E] = S * (delta * UE + (1.0f + delta) * sK * (rf * Ss + __fdividef((float)p, a)));
        }
#pragma unroll
        for (int i = 0; i < NV; i++) {
            const double f = (F[i] + (double)C[i]) * scale;
            out[i] = accumulate ? out[i] + f : f;
        }
    };
    if (SL > 0.0f) side(rl, vl, pl, kl, VnL, aL, sL, res, false, 1.0, false);
    else if (Sstar > 0.0f) side(rl, vl, pl, kl, VnL, aL, sL, res, true, 1.0, false);
    else if (Sstar == 0.0f) {
        side(rl, vl, pl, kl, VnL, aL, sL, res, true, 0.5, false);
        side(rr, vr, pr, kr, VnR, aR, sR, res, true, 0.5, true);
    } else if (SR > 0.0f) side(rr, vr, pr, kr, VnR, aR, sR, res, true, 1.0, false);
    else side(rr, vr, pr, kr, VnR, aR, sR, res, false, 1.0, false);
}

} // namespace cfd
