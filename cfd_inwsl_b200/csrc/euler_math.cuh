// Pointwise arithmetic of the zone_FD right-hand side, written for sm_100a.
//
// Every function keeps the reference's operation order term by term, so that a
// translation unit compiled with --fmad=false reproduces the reference's FP64
// results bit for bit (the reference is built for generic x86-64 without FMA
// contraction). Translation units compiled with --fmad=true get contracted
// FMAs and, where CFD_FAST is defined, a few algebraic rewrites that trade the
// last ulp for fewer divisions; those are marked "fast path".
//
// Layout conventions: prim = (rho, u, v[, w], p), cons = (rho, rho u, rho v
// [, rho w], rho E); NV = 3 (1D), 4 (2D), 5 (3D). AX is the sweep axis
// (0 = x, 1 = y, 2 = z); the face normal is the unit vector along AX.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#ifndef CFD_HD
#define CFD_HD __host__ __device__ __forceinline__
#endif

namespace cfd {

// zone_FD/src/include/macro.hpp:28 (#define GAMMA 1.4)
constexpr double kGamma = 1.4;

#if defined(CFD_FAST)
// fast path: reciprocals shared across a state or a face, multiplications
// instead of repeated IEEE divisions (about 1 ulp from the reference's order).
constexpr double kG1 = kGamma / (kGamma - 1);   // gamma / (gamma - 1)
constexpr double kInvGm1 = 1.0 / (kGamma - 1);  // 1 / (gamma - 1)
#endif
constexpr double kGm1 = kGamma - 1;             // gamma - 1 as the reference rounds it
constexpr double kRcpGm1 = 1.0 / kGm1;          // RN(1 / (gamma - 1))

// ---------------------------------------------------------------------------
// Correctly rounded division by a shared reciprocal (strict flavour).
//
// The strict flavour must round every quotient exactly as an IEEE division
// does. Where several numerators share one denominator b, y = RN(1/b) is formed
// once and each quotient is derived from it with Markstein's correction
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34(1), 1990, and the FMA-based
// division proofs of Cornea-Hasegan, Golliver and Markstein, 1999): if q is
// within one ulp of a/b and y = RN(1/b), the residual r = a - b q is exact in
// an FMA and RN(q + r y) = RN(a/b). q0 = RN(a y) can lie slightly more than
// one ulp away, so a first correction brings it within a small fraction of an
// ulp and a second applies the theorem: five FP64 operations against about
// thirteen FP64 issue slots for a division on B200 (measured). Dividends that
// are tiny (below 2^-960, where the residual could be subnormal), huge or not
// finite take the IEEE division itself; zeros keep their sign through the
// sign of RN(a y). Quotients formed together share one test and one branch
// (divs_rn). The denominators here are densities, sound speeds, enthalpies
// and spacings, normal numbers far from the ends of the exponent range.
// ---------------------------------------------------------------------------
CFD_HD double rcp_rn(double b)
{
#if defined(__CUDA_ARCH__)
    return __drcp_rn(b);
#else
    return 1.0 / b;
#endif
}

#if defined(__CUDACC__)
// The IEEE division itself, out of line: the rare operands of div_rn take it,
// and keeping its inline expansion out of every call site keeps the sweep's
// instruction footprint small.
static __device__ __noinline__ double div_ieee(double a, double b) { return a / b; }
#endif

#if defined(__CUDA_ARCH__)
// Whether a's quotient may take the Markstein correction: 2^-960 <= |a| <
// 2^960 (biased exponent 63..1982) or a = +-0, tested on the bits with integer
// operations (no FP64 compares on the FP64 pipe).
__device__ __forceinline__ bool mk_ok(double a)
{
    // t = |a|'s high word: biased exponent in bits 20..30
    const unsigned t = (unsigned)__double2hiint(a) & 0x7fffffffu, lo = (unsigned)__double2loint(a);
    return (t - (63u << 20) < (1920u << 20)) | ((t | lo) == 0u);
}

// Markstein's quotient of a by b from y = RN(1/b). The sign is taken from
// q0 = RN(a y), which carries sign(a) sign(b) also for a = +-0, where the
// corrections can turn -0 into +0.
__device__ __forceinline__ double mk_div(double a, double b, double y)
{
    const double q0 = a * y;
    double r = fma(-b, q0, a);
    const double q = fma(r, y, q0);
    r = fma(-b, q, a);
    return copysign(fma(r, y, q), q0);
}
#endif

CFD_HD double div_rn(double a, double b, double y)
{
#if defined(__CUDA_ARCH__)
    const double q = mk_div(a, b, y);
    return mk_ok(a) ? q : div_ieee(a, b);
#else
    (void)y;
    return a / b;
#endif
}

#if defined(__CUDACC__)
template <int N>
struct DivN {
    double v[N];
};
// A group's IEEE divisions, out of line (one call site per group)
template <int N>
static __device__ __noinline__ DivN<N> divs_ieee(DivN<N> a, DivN<N> b)
{
    DivN<N> q;
#pragma unroll
    for (int i = 0; i < N; i++) q.v[i] = a.v[i] / b.v[i];
    return q;
}
#endif

// q[i] = RN(a[i] / b[i]), y[i] = RN(1/b[i]), for N quotients formed together:
// one branch to the IEEE division for the group instead of one per quotient.
template <int N>
CFD_HD void divs_rn(const double *a, const double *b, const double *y, double *q)
{
#if defined(__CUDA_ARCH__)
    bool ok = true;
#pragma unroll
    for (int i = 0; i < N; i++) {
        q[i] = mk_div(a[i], b[i], y[i]);
        ok = ok & mk_ok(a[i]);
    }
    if (!ok) {
        DivN<N> A, B;
#pragma unroll
        for (int i = 0; i < N; i++) {
            A.v[i] = a[i];
            B.v[i] = b[i];
        }
        const DivN<N> Q = divs_ieee<N>(A, B);
#pragma unroll
        for (int i = 0; i < N; i++) q[i] = Q.v[i];
    }
#else
    (void)y;
    for (int i = 0; i < N; i++) q[i] = a[i] / b[i];
#endif
}

// ---------------------------------------------------------------------------
// Five-point interpolators (zone_FD/src/include/interScheme.hpp).
// q0..q4 are the five upwind-ordered point values; the result is the value at
// the face between q2 and q3.
// ---------------------------------------------------------------------------

// Smoothness indicators shared by every WCNS/TENO variant
// (interScheme.hpp:21-28, repeated in each variant).
CFD_HD void smoothness3(double q0, double q1, double q2, double q3, double q4,
                        double &b0, double &b1, double &b2)
{
#if defined(__CUDA_ARCH__) && !defined(CFD_FAST)
    // The same roundings with fewer instructions: a product by a power of two
    // is exact, so x - 2 y, x - 4 y and x + 0.25 y each round once whether
    // they are fused or not; 0.0 * q2 adds a signed zero, which changes no
    // finite sum (and b1 only enters squared).
    double a, b;
    a = fma(-2.0, q1, q0) + q2;
    b = fma(-4.0, q1, q0) + 3.0 * q2;
    b0 = fma(0.25, b * b, a * a);
    a = fma(-2.0, q2, q1) + q3;
    b = q1 - q3;
    b1 = fma(0.25, b * b, a * a);
    a = fma(-2.0, q3, q2) + q4;
    b = fma(-4.0, q3, 3.0 * q2) + q4;
    b2 = fma(0.25, b * b, a * a);
#else
    double a, b;
    a = 1.0 * q0 - 2.0 * q1 + 1.0 * q2;
    b = 1.0 * q0 - 4.0 * q1 + 3.0 * q2;
    b0 = 1.0 / 1.0 * (a * a) + 1.0 / 4.0 * (b * b);
    a = 1.0 * q1 - 2.0 * q2 + 1.0 * q3;
    b = 1.0 * q1 + 0.0 * q2 - 1.0 * q3;
    b1 = 1.0 / 1.0 * (a * a) + 1.0 / 4.0 * (b * b);
    a = 1.0 * q2 - 2.0 * q3 + 1.0 * q4;
    b = 3.0 * q2 - 4.0 * q3 + 1.0 * q4;
    b2 = 1.0 / 1.0 * (a * a) + 1.0 / 4.0 * (b * b);
#endif
}

// The three third-order candidate values (interScheme.hpp:31-33).
CFD_HD void candidates3(double q0, double q1, double q2, double q3, double q4,
                        double &u0, double &u1, double &u2)
{
    u0 = 3.0 / 8.0 * q0 - 5.0 / 4.0 * q1 + 15.0 / 8.0 * q2;
    u1 = -1.0 / 8.0 * q1 + 3.0 / 4.0 * q2 + 3.0 / 8.0 * q3;
    u2 = 3.0 / 8.0 * q2 + 3.0 / 4.0 * q3 - 1.0 / 8.0 * q4;
}

// The eight fixed stencils selected by a TENO flag word (bit k set = stencil k
// cut off), interScheme.hpp:445-480 (identical in every TENO variant). On the
// device the stencil is a row of a coefficient table applied as one 5-term sum,
// in the reference's term order: every coefficient is exact in binary, a zero
// coefficient adds an exact zero and a negative one subtracts, so each row
// rounds exactly like the reference's expression for finite stencil values.
#if defined(__CUDACC__)
static __constant__ double kTenoStencil[8][5] = {
    {3.0 / 128.0, -5.0 / 32.0, 45.0 / 64.0, 15.0 / 32.0, -5.0 / 128.0},
    {0.0, -1.0 / 16.0, 9.0 / 16.0, 9.0 / 16.0, -1.0 / 16.0},
    {0.0, 0.0, 3.0 / 8.0, 3.0 / 4.0, -1.0 / 8.0},
    {0.0, 0.0, 3.0 / 8.0, 3.0 / 4.0, -1.0 / 8.0},
    {1.0 / 16.0, -5.0 / 16.0, 15.0 / 16.0, 5.0 / 16.0, 0.0},
    {0.0, -1.0 / 8.0, 3.0 / 4.0, 3.0 / 8.0, 0.0},
    {3.0 / 8.0, -5.0 / 4.0, 15.0 / 8.0, 0.0, 0.0},
    {0.0, 0.0, 1.0, 0.0, 0.0},
};
#endif
CFD_HD double teno_select(unsigned flag, double q0, double q1, double q2, double q3, double q4)
{
#if defined(__CUDA_ARCH__)
    const double *c = kTenoStencil[flag & 7u];
    double t = c[0] * q0;
    t = t + c[1] * q1;
    t = t + c[2] * q2;
    t = t + c[3] * q3;
    return t + c[4] * q4;
#else
    switch (flag) {
    case 0: return 3.0 / 128.0 * q0 - 5.0 / 32.0 * q1 + 45.0 / 64.0 * q2 + 15.0 / 32.0 * q3 - 5.0 / 128.0 * q4;
    case 1: return -1.0 / 16.0 * q1 + 9.0 / 16.0 * q2 + 9.0 / 16.0 * q3 - 1.0 / 16.0 * q4;
    case 2:
    case 3: return 3.0 / 8.0 * q2 + 3.0 / 4.0 * q3 - 1.0 / 8.0 * q4;
    case 4: return 1.0 / 16.0 * q0 - 5.0 / 16.0 * q1 + 15.0 / 16.0 * q2 + 5.0 / 16.0 * q3;
    case 5: return -1.0 / 8.0 * q1 + 3.0 / 4.0 * q2 + 3.0 / 8.0 * q3;
    case 6: return 3.0 / 8.0 * q0 - 5.0 / 4.0 * q1 + 15.0 / 8.0 * q2;
    default: return q2;
    }
#endif
}

// TENO-Z keeps all three stencils (flag 0) when
// min_k m_k >= CT = c sum_k m_k, m_k = (1 + tau/s_k)^6, s_k = beta_k + eps. A
// sufficient condition without divisions: m_min >= 3.3 c m_max, i.e.
// t_min / t_max = (s_max + tau) s_min / ((s_min + tau) s_max) >= kappa with
// kappa = (3.3 c)^(1/6) (teno_kappa). Its 10% margin over the 3c that
// sum_k m_k <= 3 m_max needs is far above the rounding of either evaluation, so
// the early answer is the reference's own flag 0, bit for bit.
inline double teno_kappa(double c) { return c > 0.0 ? ::pow(3.3 * c, 1.0 / 6.0) : 0.0; }

CFD_HD bool teno_z_all_kept(double s0, double s1, double s2, double tau, double kap)
{
    const double smin = fmin(s0, fmin(s1, s2)), smax = fmax(s0, fmax(s1, s2));
    const double lhs = (smax + tau) * smin, rhs = (smin + tau) * smax;
    return rhs < 1e300 && lhs >= kap * rhs;
}

// Interpolator families. Each selector entry of the reference maps onto one
// family plus a runtime constant (InterSpec::c).
enum InterFamily : int {
    FAM_WCNS5 = 0,   // weno5_JSchen                       interScheme.hpp:17-45
    FAM_WENOZ = 1,   // weno5_Z                            interScheme.hpp:85-114
    FAM_TENOZ = 2,   // Teno5_Z / ZCT4 / ZCT7 / congTcns5_ZCT5 / ZCT10 / new_Teno5_Z
                     //   (c = cutoff factor 1e-5, 1e-4, 1e-7, 1e-5, 1e-10, 1e-5)
    FAM_TENOCONG = 3,// Teno5_CongZ / CongZCT4 / CongZCT7 / new_Teno5_CongZ (c = CT)
    FAM_MUSCL = 4,   // musclIn5 (minmod on q1..q3)        interScheme.hpp:1386-1406
    FAM_RESEARCH = 5,// the adaptive-cut-off TENO research variants (whf_*, TCNS_AS_*, Teno5_CongAA),
                     //   interScheme.hpp:304-382, 1458-1762, 1901-4209 (c = the variant, ResearchVariant)
};

// The research variants of the selector (InterMethod entries 17-21, 24-34, 36,
// 38, 39, and entry 10 in 1D). All of them interpolate with the eight fixed
// TENO stencils of teno_select and differ only in the cut-off decision.
enum ResearchVariant : int {
    RV_TCNSN = 0,     // whf_TcnsN              interScheme.hpp:1458-1517
    RV_TCNSN_A,       // whf_TcnsN_A            interScheme.hpp:3253-3361
    RV_TCNSN_AS,      // whf_TcnsN_AS           interScheme.hpp:1581-1679
    RV_TCNSN_S,       // whf_TcnsN_S            interScheme.hpp:1519-1579
    RV_TCNSN_LAD,     // whf_TcnsN_LAD          interScheme.hpp:1681-1761
    RV_AI_S,          // whf_ai_TcnsN_S_1       interScheme.hpp:1901-1994
    RV_AI_A,          // whf_ai_TcnsN_A_2       interScheme.hpp:2216-2327
    RV_AI_AS1,        // whf_ai_TcnsN_AS_1      interScheme.hpp:2329-2422
    RV_AI_AS2,        // whf_ai_TcnsN_AS_2      interScheme.hpp:2424-2510
    RV_AI_LADS,       // whf_ai_TcnsN_LADS_yuanbao interScheme.hpp:2512-2645
    RV_AI_AZS,        // whf_ai_TcnsN_AZS_yuanbao  interScheme.hpp:2862-2934
    RV_AI_ASF1,       // whf_ai_TcnsN_myASF002_1   interScheme.hpp:2936-3027
    RV_AI_ASF2,       // whf_ai_TcnsN_myASF002_2   interScheme.hpp:3029-3112
    RV_AI_ASFAI1,     // whf_ai_TcnsN_myASF002_ai1 interScheme.hpp:3114-3241
    RV_ZYC,           // whf_zyc_TcnsN_myASF002_1  interScheme.hpp:3363-3470
    RV_COMPARE,       // whf_TcnsN_COMPARE      interScheme.hpp:3472-3726
    RV_NEW_A,         // new_whf_TCNS_A         interScheme.hpp:3863-3982
    RV_F203,          // whf_TCNS_AS_myF203_NoS interScheme.hpp:3984-4091
    RV_F202,          // whf_TCNS_AS_myF202_NoS interScheme.hpp:4093-4209
    RV_CONGAA,        // Teno5_CongAA (1D WCNS5CONGZCT7) interScheme.hpp:304-382
};

// The TENO-Z cut-off flag (Teno5_Z, interScheme.hpp:384-452) from the three
// smoothness measures: measure_k = (1 + tau / (beta_k + eps))^6, stencil k cut
// when measure_k < c * sum_j measure_j. Out of line on the device: behind the
// keep-all test it is the rare path, and keeping it out of the unrolled face
// code shortens the hot loop's instruction footprint (5.6% faster TENO5 + Roe
// steps on B200).
#if defined(__CUDACC__)
static __host__ __device__ __noinline__
#else
CFD_HD
#endif
unsigned teno_z_flag(double b0, double b1, double b2, double tau, double c)
{
    const double eps = 1e-40;
    double t;
#if defined(CFD_FAST)
    // tau/s_k from one reciprocal of s0 s1 s2 (guarded against overflow and
    // underflow of the product)
    const double s0 = b0 + eps, s1 = b1 + eps, s2 = b2 + eps;
    const double s01 = s0 * s1, prod = s01 * s2;
    double r0, r1, r2;
    if (prod > 1e-280 && prod < 1e280) {
        const double ti = tau / prod;
        r0 = ti * (s1 * s2); r1 = ti * (s0 * s2); r2 = ti * s01;
    } else {
        r0 = tau / s0; r1 = tau / s1; r2 = tau / s2;
    }
    t = 1.0 + r0; t *= t; b0 = t * t * t;
    t = 1.0 + r1; t *= t; b1 = t * t * t;
    t = 1.0 + r2; t *= t; b2 = t * t * t;
#else
    t = 1.0 + tau / (b0 + eps); t *= t; b0 = t * t * t;
    t = 1.0 + tau / (b1 + eps); t *= t; b1 = t * t * t;
    t = 1.0 + tau / (b2 + eps); t *= t; b2 = t * t * t;
#endif
    double sumbeta = 0.0;
    sumbeta += b0; sumbeta += b1; sumbeta += b2;
    const double CT = c * sumbeta;
    unsigned flag = 0;
    if (b0 < CT) flag += 1;
    if (b1 < CT) flag += 2;
    if (b2 < CT) flag += 4;
    return flag;
}

// The cut-off flag of a research variant (bit k set = stencil k cut), in the
// reference's operation order wherever the variant uses only + - * / floor
// min max (bitwise parity); variants that call pow() agree to pow's rounding
// (libm's and CUDA's pow differ by up to a few ulps, which can flip a decision
// only at its threshold). Out of line on the device: one copy serves the eight
// interpolations of a face.
#if defined(__CUDACC__)
static __host__ __device__ __noinline__
#else
static inline
#endif
unsigned research_flag(int variant, double q0, double q1, double q2, double q3, double q4)
{
    double b0, b1, b2;
    smoothness3(q0, q1, q2, q3, q4, b0, b1, b2);
    const double tau = fabs(b2 - b0);
    // the smallest measure (std::min over {beta0, beta1, beta2}, or its
    // std::min_element: the same value)
    double bmin = b0;
    if (b1 < bmin) bmin = b1;
    if (b2 < bmin) bmin = b2;
    // gamma-type measures (1 + tau / (beta_k + 1e-40))^6 by pow, and by squares and cubes
    auto gpow = [&](double b) { return pow(1.0 + tau / (b + 1e-40), 6.0); };
    auto gsq = [&](double b) {
        double g = 1.0 + tau / (b + 1e-40);
        g = g * g;
        return g * g * g;
    };
    // cut when gamma_k / sum < CT
    auto cut_ratio = [](double g0, double g1, double g2, double CT) {
        const double s = g0 + g1 + g2;
        return (g0 / s < CT ? 1u : 0u) + (g1 / s < CT ? 2u : 0u) + (g2 / s < CT ? 4u : 0u);
    };
    // cut when gamma_k < CT * sum
    auto cut_prod = [](double g0, double g1, double g2, double CT) {
        const double rr = CT * (g0 + g1 + g2);
        return (g0 < rr ? 1u : 0u) + (g1 < rr ? 2u : 0u) + (g2 < rr ? 4u : 0u);
    };
    // cut when beta_k tau < (CTp tau - (1 - CTp) beta_k) beta_min (whf_TcnsN_S form)
    auto cut_cross_a = [&](double CTp) {
        unsigned f = 0;
        if (b0 * tau < (CTp * tau - 1.0 * (1.0 - CTp) * b0) * bmin) f += 1;
        if (b1 * tau < (CTp * tau - 1.0 * (1.0 - CTp) * b1) * bmin) f += 2;
        if (b2 * tau < (CTp * tau - 1.0 * (1.0 - CTp) * b2) * bmin) f += 4;
        return f;
    };
    // cut when beta_min tau < (CTp tau - (1 - CTp) beta_min) beta_k (the ai_* form)
    auto cut_cross_b = [&](double CTp) {
        const double th = CTp * tau - 1.0 * (1.0 - CTp) * bmin;
        const double l = bmin * tau;
        return (l < th * b0 ? 1u : 0u) + (l < th * b1 ? 2u : 0u) + (l < th * b2 ? 4u : 0u);
    };
    // cut when tau beta_min < (CT tau - (1 - CT) beta_min) beta_k (Teno5_CongZ form)
    auto cut_cong = [&](double CT) {
        const double rr = CT * tau - (1 - CT) * bmin, ll = tau * bmin;
        return (ll < rr * b0 ? 1u : 0u) + (ll < rr * b1 ? 2u : 0u) + (ll < rr * b2 ? 4u : 0u);
    };
    auto ctp_of = [](double CT) { return pow(1.5 * CT / (1.0 - CT), 1.0 / 6.0); };
    // eta on neighbouring differences dq(k+1/2) = q_{k+1} - q_k of the stencil (ai_* variants)
    constexpr double kEpsA = (0.9 * 0.24) / (1 - 0.9 * 0.24) * 1e-3 * 1e-3;
    auto eta_ai = [&](double epsA) {
        const double dm3 = q1 - q0, dm1 = q2 - q1, dp1 = q3 - q2, dp3 = q4 - q3;
        const double e0 = (fabs(2 * dm1 * dm3) + epsA) / (dm1 * dm1 + dm3 * dm3 + epsA);
        const double e1 = (fabs(2 * dp1 * dm1) + epsA) / (dp1 * dp1 + dm1 * dm1 + epsA);
        const double e2 = (fabs(2 * dp3 * dp1) + epsA) / (dp3 * dp3 + dp1 * dp1 + epsA);
        double m = e0;
        if (e1 < m) m = e1;
        if (e2 < m) m = e2;
        return m;
    };
    // eta on the stencil values themselves (whf_TcnsN_AS, Teno5_CongAA)
    auto eta_raw = [&]() {
        auto e = [&](double a, double b, double c) {
            const double x1 = (fabs(2 * b * a) + kEpsA) / (b * b + a * a + kEpsA);
            const double x2 = (fabs(2 * c * b) + kEpsA) / (c * c + b * b + kEpsA);
            return (x2 < x1) ? x2 : x1;
        };
        const double e0 = e(q0, q1, q2), e1 = e(q1, q2, q3), e2 = e(q2, q3, q4);
        double m = e0;
        if (e1 < m) m = e1;
        if (e2 < m) m = e2;
        return m;
    };
    // CT of the A-type variants from the switch on floor(10 - 5 (1 - g))
    auto ct_switch = [](int beta_A) {
        switch (beta_A) {
        case 5: return 1e-5;
        case 6: return 1e-6;
        case 7: return 1e-7;
        case 8: return 1e-8;
        case 9: return 1e-9;
        default: return 1e-10;
        }
    };
    switch (variant) {
    case RV_TCNSN:
        return cut_ratio(gpow(b0), gpow(b1), gpow(b2), 1e-10);
    case RV_TCNSN_S:
        return cut_cross_a(ctp_of(1e-5));
    case RV_TCNSN_AS: {
        const double m = 1.0 - fmin(1.0, eta_raw() / 0.24);
        const double g = pow(1 - m, 4.0) * (1 + 4 * m);
        const int bA = (int)floor(10.0 - 5.0 * (1 - g));
        return cut_cross_a(ctp_of(pow(10.0, (double)-bA)));
    }
    case RV_TCNSN_LAD: {
        const double c0 = tau / (b0 + 1e-40), c1 = tau / (b1 + 1e-40), c2 = tau / (b2 + 1e-40);
        const double cmax = fmax(c0, fmax(c1, c2));
        const double theta = 1.0 / (1.0 + cmax / 10.0);
        int m = 4 + (int)floor(theta * 6);
        m = m < 4 ? 4 : (m > 10 ? 10 : m);
        const double tab[7] = {1e-4, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9, 1e-10};
        return cut_ratio(gpow(b0), gpow(b1), gpow(b2), tab[m - 4]);
    }
    case RV_TCNSN_A: case RV_COMPARE: case RV_NEW_A: {
        const double epsA = (variant == RV_COMPARE) ? kEpsA : 2.7551 * 1e-7;
        const double d0 = q0 - q1, d1 = q1 - q2, d2 = q2 - q3, d3 = q3 - q4;
        double e0, e1, e2;
        if (variant == RV_NEW_A) {
            e0 = (fabs(2.0 * d0 * d1) + epsA) / (d0 * d0 + d1 * d1 + epsA);
            e1 = (fabs(2.0 * d1 * d2) + epsA) / (d1 * d1 + d2 * d2 + epsA);
            e2 = (fabs(2.0 * d2 * d3) + epsA) / (d2 * d2 + d3 * d3 + epsA);
        } else {
            e0 = (fabs(2.0 * d0 * d2) + epsA) / (d0 * d0 + d2 * d2 + epsA);
            e1 = (fabs(2.0 * d1 * d3) + epsA) / (d1 * d1 + d3 * d3 + epsA);
            e2 = (fabs(2.0 * d2 * d1) + epsA) / (d2 * d2 + d1 * d1 + epsA);
        }
        double emin = e0;
        if (e1 < emin) emin = e1;
        if (e2 < emin) emin = e2;
        double g;
        if (variant == RV_NEW_A) {
            const double mn = fmin(1.0, 4.1666667 * emin);
            g = mn * mn * mn * mn * (5.0 - 4 * mn);
        } else {
            const double m = 1.0 - fmin(1.0, variant == RV_COMPARE ? emin / 0.24 : 4.1666667 * emin);
            g = (1 - m) * (1 - m) * (1 - m) * (1 - m) * (1 + 4 * m);
        }
        const int bA = (int)floor(10.0 - 5.0 * (1 - g));
        return cut_prod(gsq(b0), gsq(b1), gsq(b2), ct_switch(bA));
    }
    case RV_AI_S:
        return cut_cross_b(ctp_of(1e-5));
    case RV_AI_A: {
        const double m = 1.0 - fmin(1.0, eta_ai(kEpsA) / 0.24);
        const double g = pow(1 - m, 4.0) * (1 + 4 * m);
        const double CT = pow(10.0, -floor(10.0 - 5.0 * (1 - g)));
        return cut_ratio(gpow(b0), gpow(b1), gpow(b2), CT);
    }
    case RV_AI_AS1: case RV_AI_AS2: {
        const double m = 1.0 - fmin(1.0, eta_ai(kEpsA) / 0.24);
        const double g = pow(1.0 - m, 4.0) * (1.0 + 4.0 * m);
        const double CT = pow(10.0, -floor(10.0 - 5.0 * (1.0 - g)));
        return cut_cross_b(ctp_of(CT));
    }
    case RV_AI_LADS: {
        const double c0 = tau / (b0 + 1e-40), c1 = tau / (b1 + 1e-40), c2 = tau / (b2 + 1e-40);
        const double cmax = fmax(c0, fmax(c1, c2));
        const double theta = 1.0 / (1.0 + cmax / 10.0);
        const int m = 5 + (int)floor(theta * 5);
        return cut_cross_b(ctp_of(pow(10.0, (double)-m)));
    }
    case RV_AI_AZS: {
        const double tauA = fabs(b0 + b2 - 2 * b1);
        return cut_cross_b(ctp_of(fmin(1e-5, tauA)));
    }
    case RV_AI_ASF1: case RV_AI_ASF2: case RV_AI_ASFAI1: {
        const double x = fmin(1.0, eta_ai(kEpsA) / 0.24);
        return cut_cross_b(0.157 / (11.351092 * x * x - 5.740650 * x + 1.506631));
    }
    case RV_ZYC: {
        const double mn = fmin(1.0, 4.1666667 * eta_ai(2.7551 * 1e-7));
        return cut_cong(0.157 / (11.351092 * mn * mn - 5.740650 * mn + 1.506631));
    }
    case RV_F203: case RV_F202: {
        const double epsA = 2.7551 * 1e-7;
        const double d0 = q0 - q1, d1 = q1 - q2, d2 = q2 - q3, d3 = q3 - q4;
        const double e0 = (fabs(2.0 * d1 * d0) + epsA) / (d1 * d1 + d0 * d0 + epsA);
        const double e1 = (fabs(2.0 * d2 * d1) + epsA) / (d2 * d2 + d1 * d1 + epsA);
        const double e2 = (fabs(2.0 * d3 * d2) + epsA) / (d3 * d3 + d2 * d2 + epsA);
        double emin = e0;
        if (e1 < emin) emin = e1;
        if (e2 < emin) emin = e2;
        const double m = 1 - fmin(0.24, emin) / 0.24;
        double CT;
        if (variant == RV_F203) {
            const double mm = m * m, mmm = m * mm;
            CT = -0.452662 * mmm + 0.590811 * mm - 0.012189 * m + 0.022010;
        } else {
            CT = -0.088182 * m * m + 0.259395 * m - 0.000616;
        }
        return cut_cong(CT);
    }
    case RV_CONGAA: {
        const double m = 1.0 - fmin(1.0, eta_raw() / 0.24);
        const double g = pow(1 - m, 4.0) * (1 + 4 * m);
        return cut_cong(pow(10.0, -round(10.0 - 5.0 * (1 - g))));
    }
    default:
        return 7u;
    }
}

template <int FAM>
CFD_HD double inter5(double q0, double q1, double q2, double q3, double q4, double c, double kap = 0.0)
{
    if constexpr (FAM == FAM_WCNS5) {
        // weno5_JSchen: omega_k = gamma_k / (eps + beta_k)^2, eps = 1e-6.
        const double eps = 1e-6;
        double b0, b1, b2, u0, u1, u2;
        smoothness3(q0, q1, q2, q3, q4, b0, b1, b2);
        candidates3(q0, q1, q2, q3, q4, u0, u1, u2);
#if defined(CFD_FAST)
        // fast path: one division instead of four. With s_k = eps + beta_k,
        // sum_k g_k u_k / s_k^2 / sum_k g_k / s_k^2 equals the same sums with
        // every term multiplied by prod_k s_k^2, i.e. weights g_k * prod_{j!=k} s_j^2.
        double s0 = eps + b0, s1 = eps + b1, s2 = eps + b2;
        s0 *= s0; s1 *= s1; s2 *= s2;
        double w0 = (1.0 / 16.0) * (s1 * s2), w1 = (5.0 / 8.0) * (s0 * s2), w2 = (5.0 / 16.0) * (s0 * s1);
        return (w0 * u0 + w1 * u1 + w2 * u2) / (w0 + w1 + w2);
#else
        double s;
        // (1/16) / s^2 = RN(1 / s^2) / 16 exactly (a power-of-two scaling)
        s = eps + b0; b0 = rcp_rn(s * s) * (1.0 / 16.0);
        s = eps + b1; b1 = (5.0 / 8.0) / (s * s);
        s = eps + b2; b2 = (5.0 / 16.0) / (s * s);
        double sumbeta = 0.0, result = 0.0;
        sumbeta += b0; sumbeta += b1; sumbeta += b2;
        result += b0 * u0; result += b1 * u1; result += b2 * u2;
        return result / sumbeta;
#endif
    } else if constexpr (FAM == FAM_WENOZ) {
        // weno5_Z: omega_k = gamma_k (1 + (tau / (beta_k + eps))^2), eps = 1e-40.
        const double eps = 1e-40;
        double b0, b1, b2, u0, u1, u2;
        smoothness3(q0, q1, q2, q3, q4, b0, b1, b2);
        candidates3(q0, q1, q2, q3, q4, u0, u1, u2);
        double tau = fabs(b2 - b0), x;
        x = tau / (b0 + eps); b0 = (1.0 / 16.0) * (1.0 + x * x);
        x = tau / (b1 + eps); b1 = (5.0 / 8.0) * (1.0 + x * x);
        x = tau / (b2 + eps); b2 = (5.0 / 16.0) * (1.0 + x * x);
        double sumbeta = 0.0, result = 0.0;
        sumbeta += b0; sumbeta += b1; sumbeta += b2;
        result += b0 * u0; result += b1 * u1; result += b2 * u2;
        return result / sumbeta;
    } else if constexpr (FAM == FAM_TENOZ) {
        // TENO5 with the Z-type measure (1 + tau/(beta_k + eps))^6 and the
        // cutoff measure_k < c * sum_j measure_j (Teno5_Z: interScheme.hpp:384-452).
        const double eps = 1e-40;
        double b0, b1, b2;
        smoothness3(q0, q1, q2, q3, q4, b0, b1, b2);
        double tau = fabs(b2 - b0), t;
        (void)t;
        if (kap > 0.0 && teno_z_all_kept(b0 + eps, b1 + eps, b2 + eps, tau, kap))
            return teno_select(0u, q0, q1, q2, q3, q4);
        return teno_select(teno_z_flag(b0, b1, b2, tau, c), q0, q1, q2, q3, q4);
    } else if constexpr (FAM == FAM_TENOCONG) {
        // Cross-multiplied TENO cutoff of Teno5_CongZ (interScheme.hpp:494-584):
        // stencil k is cut when tau*beta_min < (CT*tau - (1-CT)*beta_min) * beta_k.
        double b0, b1, b2;
        smoothness3(q0, q1, q2, q3, q4, b0, b1, b2);
        // std::min_element: first index of the smallest value.
        double bmin = b0;
        if (b1 < bmin) bmin = b1;
        if (b2 < bmin) bmin = b2;
        const double CT = c, CT_1 = 1.0 - c;
        double tau = fabs(b2 - b0);
        double rr = CT * tau - CT_1 * bmin;
        double ll = tau * bmin;
        unsigned flag = 0;
        if (ll < rr * b0) flag += 1;
        if (ll < rr * b1) flag += 2;
        if (ll < rr * b2) flag += 4;
        return teno_select(flag, q0, q1, q2, q3, q4);
    } else if constexpr (FAM == FAM_RESEARCH) {
        (void)kap;
        return teno_select(research_flag((int)c, q0, q1, q2, q3, q4), q0, q1, q2, q3, q4);
    } else {
        // musclIn5: minmod limited slope on (q1, q2, q3).
        double deltam = q2 - q1, deltap = q3 - q2, delta;
        const double beta = 1.0;
        // std::max(a,b) = (a < b) ? b : a ; std::min(a,b) = (b < a) ? b : a
        auto smax = [](double a, double b) { return (a < b) ? b : a; };
        auto smin = [](double a, double b) { return (b < a) ? b : a; };
        if (deltap > 0) {
            delta = smax(0.0, smax(smin(beta * deltam, deltap), smin(deltam, beta * deltap)));
        } else {
            delta = smin(0.0, smin(smax(beta * deltam, deltap), smax(deltam, beta * deltap)));
        }
        return q2 + delta * 0.5;
    }
}

// ---------------------------------------------------------------------------
// cons -> prim as Equation::consToPrimEuler{1D,2D} (equation.cpp:37-93); the
// 3D form adds w the same way.
// ---------------------------------------------------------------------------
template <int NV>
CFD_HD void cons_to_prim(const double *c, double *p)
{
    const double gamma = kGamma;
    if constexpr (NV == 3) {
        double r = c[0], ru = c[1], rE = c[2];
#if defined(CFD_FAST)
        const double ir = 1.0 / r;
        double u = ru * ir;
        double E = rE * ir;
#else
        const double ir = rcp_rn(r);
        const double a[2] = {ru, rE}, bb[2] = {r, r}, yy[2] = {ir, ir};
        double qq[2];
        divs_rn<2>(a, bb, yy, qq);
        double u = qq[0], E = qq[1];
#endif
        double e = -u * u / 2 + E;
        double RT = (gamma - 1) * e;
        p[0] = r; p[1] = u; p[2] = r * RT;
    } else if constexpr (NV == 4) {
        double r = c[0], ru = c[1], rv = c[2], rE = c[3];
#if defined(CFD_FAST)
        const double ir = 1.0 / r;
        double u = ru * ir, v = rv * ir, E = rE * ir;
#else
        const double ir = rcp_rn(r);
        const double a[3] = {ru, rv, rE}, bb[3] = {r, r, r}, yy[3] = {ir, ir, ir};
        double qq[3];
        divs_rn<3>(a, bb, yy, qq);
        double u = qq[0], v = qq[1], E = qq[2];
#endif
        double q2 = (u * u + v * v) / 2;
        double e = -q2 + E;
        double RT = (gamma - 1) * e;
        p[0] = r; p[1] = u; p[2] = v; p[3] = r * RT;
    } else {
        double r = c[0], ru = c[1], rv = c[2], rw = c[3], rE = c[4];
#if defined(CFD_FAST)
        const double ir = 1.0 / r;
        double u = ru * ir, v = rv * ir, w = rw * ir, E = rE * ir;
#else
        const double ir = rcp_rn(r);
        const double a[4] = {ru, rv, rw, rE}, bb[4] = {r, r, r, r}, yy[4] = {ir, ir, ir, ir};
        double qq[4];
        divs_rn<4>(a, bb, yy, qq);
        double u = qq[0], v = qq[1], w = qq[2], E = qq[3];
#endif
        double q2 = (u * u + v * v + w * w) / 2;
        double e = -q2 + E;
        double RT = (gamma - 1) * e;
        p[0] = r; p[1] = u; p[2] = v; p[3] = w; p[4] = r * RT;
    }
}

// prim -> cons as the eigensystem's primToCons/primToChar prologue
// (eigenSystem.cpp:91-93 for 2D, :254-256 for 1D).
template <int NV>
CFD_HD void prim_to_cons(const double *p, double *c)
{
    const double gamma = kGamma;
    if constexpr (NV == 3) {
        double rt = p[0], ut = p[1], pt = p[2];
        double ekt = (ut * ut) / 2;
#if defined(CFD_FAST)
        c[0] = rt; c[1] = rt * ut; c[2] = pt * kInvGm1 + rt * ekt;
#else
        c[0] = rt; c[1] = rt * ut; c[2] = div_rn(pt, kGm1, kRcpGm1) + rt * ekt;
#endif
    } else if constexpr (NV == 4) {
        double rt = p[0], ut = p[1], vt = p[2], pt = p[3];
        double ekt = (ut * ut + vt * vt) / 2;
#if defined(CFD_FAST)
        c[0] = rt; c[1] = rt * ut; c[2] = rt * vt; c[3] = pt * kInvGm1 + rt * ekt;
#else
        c[0] = rt; c[1] = rt * ut; c[2] = rt * vt; c[3] = div_rn(pt, kGm1, kRcpGm1) + rt * ekt;
#endif
    } else {
        double rt = p[0], ut = p[1], vt = p[2], wt = p[3], pt = p[4];
        double ekt = (ut * ut + vt * vt + wt * wt) / 2;
#if defined(CFD_FAST)
        c[0] = rt; c[1] = rt * ut; c[2] = rt * vt; c[3] = rt * wt; c[4] = pt * kInvGm1 + rt * ekt;
#else
        c[0] = rt; c[1] = rt * ut; c[2] = rt * vt; c[3] = rt * wt; c[4] = div_rn(pt, kGm1, kRcpGm1) + rt * ekt;
#endif
    }
}

// ---------------------------------------------------------------------------
// Roe-averaged characteristic system.
// 1D: eigensystemEuler1D (eigenSystem.cpp:217-323).
// 2D: eigensystemEuler2D (eigenSystem.cpp:13-213), normal = unit vector AX.
// 3D: the 2D system extended by a second shear wave (this library's own
//     extension; the reference has no 3D Euler path). For a field with w = 0
//     that does not vary along z, it reduces to the 2D system value for value.
// ---------------------------------------------------------------------------
template <int NV, int AX>
struct Eigen {
    double L[NV][NV];  // rows = left eigenvectors (char = L * cons)
    double R[NV][NV];  // R[row][col]: cons = R * char

    CFD_HD Eigen(const double *pl, const double *pr)
    {
        const double gamma = kGamma;
        if constexpr (NV == 3) {
            double rl = pl[0], ul = pl[1], pL = pl[2];
            double rr = pr[0], ur = pr[1], pR = pr[2];
#if defined(CFD_FAST)
            double HL = 0.5 * (ul * ul) + pL * (kG1 / rl);
            double HR = 0.5 * (ur * ur) + pR * (kG1 / rr);
#else
            double HL = (ul * ul) / 2 + pL / rl * gamma / (gamma - 1);
            double HR = (ur * ur) / 2 + pR / rr * gamma / (gamma - 1);
#endif
            double coef1 = sqrt(rl), coef2 = sqrt(rr);
            double divisor = 1.0 / (coef1 + coef2);
            double u = (coef1 * ul + coef2 * ur) * divisor;
            double ht = (coef1 * HL + coef2 * HR) * divisor;
            double ek = (u * u) / 2;
            double h = ht - ek;
            double c = sqrt((gamma - 1) * h);
            double g1 = gamma - 1;
            double le[9] = {ht + c * (u - c) / g1, -u - c / g1, 1.0,
                            -2.0 * ht + 4.0 * c * c / g1, 2.0 * u, -2.0,
                            ht - c * (u + c) / g1, -u + c / g1, 1.0};
            double f = 0.5 * g1 / (c * c);
            for (int i = 0; i < 9; i++) L[i / 3][i % 3] = le[i] * f;
            double re[9] = {1.0, 1.0, 1.0, u - c, u, u + c, ht - u * c, 0.5 * u * u, ht + u * c};
            for (int i = 0; i < 9; i++) R[i / 3][i % 3] = re[i];
        } else {
            constexpr int D = (NV == 4) ? 2 : 3;
            double vl[3] = {pl[1], pl[2], D == 3 ? pl[3] : 0.0};
            double vr[3] = {pr[1], pr[2], D == 3 ? pr[3] : 0.0};
            double rl = pl[0], rr = pr[0], pL = pl[NV - 1], pR = pr[NV - 1];
            double HL, HR;
#if defined(CFD_FAST)
            {
                double kl = vl[0] * vl[0] + vl[1] * vl[1], kr = vr[0] * vr[0] + vr[1] * vr[1];
                if constexpr (D == 3) { kl += vl[2] * vl[2]; kr += vr[2] * vr[2]; }
                HL = 0.5 * kl + pL * (kG1 / rl);
                HR = 0.5 * kr + pR * (kG1 / rr);
            }
#else
            if constexpr (D == 2) {
                HL = (vl[0] * vl[0] + vl[1] * vl[1]) / 2 + pL / rl * gamma / (gamma - 1);
                HR = (vr[0] * vr[0] + vr[1] * vr[1]) / 2 + pR / rr * gamma / (gamma - 1);
            } else {
                HL = (vl[0] * vl[0] + vl[1] * vl[1] + vl[2] * vl[2]) / 2 + pL / rl * gamma / (gamma - 1);
                HR = (vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]) / 2 + pR / rr * gamma / (gamma - 1);
            }
#endif
            double coef1 = sqrt(rl), coef2 = sqrt(rr);
            double divisor = 1.0 / (coef1 + coef2);
            double u = (coef1 * vl[0] + coef2 * vr[0]) * divisor;
            double v = (coef1 * vl[1] + coef2 * vr[1]) * divisor;
            double w = (D == 3) ? (coef1 * vl[2] + coef2 * vr[2]) * divisor : 0.0;
            double ht = (coef1 * HL + coef2 * HR) * divisor;
            const double nx = (AX == 0) ? 1.0 : 0.0, ny = (AX == 1) ? 1.0 : 0.0, nz = (AX == 2) ? 1.0 : 0.0;
            double Vn, ek;
            if constexpr (D == 2) {
                Vn = nx * u + ny * v;
                ek = (u * u + v * v) / 2;
            } else {
                Vn = nx * u + ny * v + nz * w;
                ek = (u * u + v * v + w * w) / 2;
            }
            double h = ht - ek;
            double c = sqrt((gamma - 1) * h);
            // rows: 0 shear (tangent t1), 1 entropy, 2 acoustic (Vn - c), 3 acoustic (Vn + c)
            // [, 4 shear (tangent t2) in 3D]
            // column order in L rows and R rows: rho, rho u, rho v, [rho w,] rho E
            constexpr int E = NV - 1;
#if defined(CFD_FAST)
            // fast path: share the reciprocals of c and h.
            const double ic = 1.0 / c, ih = 1.0 / h;
#define CFD_DIV_C(a) ((a) * ic)
#define CFD_DIV_H(a) ((a) * ih)
#else
#define CFD_DIV_C(a) ((a) / c)
#define CFD_DIV_H(a) ((a) / h)
#endif
            if constexpr (AX != 2) {
                L[0][0] = (-ny * u + nx * v); L[0][1] = ny; L[0][2] = (-nx);
            } else {
                L[0][0] = -u; L[0][1] = 1.0; L[0][2] = 0.0;
            }
            if constexpr (D == 3) L[0][3] = 0.0;
            L[0][E] = 0;
            L[1][0] = (h - ek); L[1][1] = u; L[1][2] = v;
            if constexpr (D == 3) L[1][3] = w;
            L[1][E] = -1.0;
            L[2][0] = (CFD_DIV_C(Vn) + CFD_DIV_H(ek)) / 2;
            L[2][1] = (CFD_DIV_C(-nx) - CFD_DIV_H(u)) / 2;
            L[2][2] = (CFD_DIV_C(-ny) - CFD_DIV_H(v)) / 2;
            if constexpr (D == 3) L[2][3] = (CFD_DIV_C(-nz) - CFD_DIV_H(w)) / 2;
#if defined(CFD_FAST)
            L[2][E] = 0.5 * ih;
#else
            L[2][E] = 1.0 / (2.0 * h);
#endif
            L[3][0] = (CFD_DIV_C(-Vn) + CFD_DIV_H(ek)) / 2;
            L[3][1] = (CFD_DIV_C(nx) - CFD_DIV_H(u)) / 2;
            L[3][2] = (CFD_DIV_C(ny) - CFD_DIV_H(v)) / 2;
            if constexpr (D == 3) L[3][3] = (CFD_DIV_C(nz) - CFD_DIV_H(w)) / 2;
            L[3][E] = L[2][E];
            if constexpr (D == 3) {
                if constexpr (AX != 2) {
                    L[4][0] = -w; L[4][1] = 0.0; L[4][2] = 0.0; L[4][3] = 1.0; L[4][4] = 0.0;
                } else {
                    L[4][0] = -v; L[4][1] = 0.0; L[4][2] = 1.0; L[4][3] = 0.0; L[4][4] = 0.0;
                }
            }
            // right eigenvectors, stored by row of cons
            if constexpr (AX != 2) {
                R[0][0] = 0; R[1][0] = ny; R[2][0] = -nx; R[E][0] = ny * u - nx * v;
                if constexpr (D == 3) R[3][0] = 0.0;
            } else {
                R[0][0] = 0; R[1][0] = 1.0; R[2][0] = 0.0; R[3][0] = 0.0; R[E][0] = u;
            }
            R[0][1] = CFD_DIV_H(1.0); R[1][1] = CFD_DIV_H(u); R[2][1] = CFD_DIV_H(v); R[E][1] = CFD_DIV_H(ek);
            if constexpr (D == 3) R[3][1] = CFD_DIV_H(w);
            R[0][2] = 1; R[1][2] = u - nx * c; R[2][2] = v - ny * c; R[E][2] = h + ek - Vn * c;
            if constexpr (D == 3) R[3][2] = w - nz * c;
            R[0][3] = 1; R[1][3] = u + nx * c; R[2][3] = v + ny * c; R[E][3] = h + ek + Vn * c;
            if constexpr (D == 3) R[3][3] = w + nz * c;
            if constexpr (D == 3) {
                if constexpr (AX != 2) {
                    R[0][4] = 0.0; R[1][4] = 0.0; R[2][4] = 0.0; R[3][4] = 1.0; R[4][4] = w;
                } else {
                    R[0][4] = 0.0; R[1][4] = 0.0; R[2][4] = 1.0; R[3][4] = 0.0; R[4][4] = v;
                }
            }
#undef CFD_DIV_C
#undef CFD_DIV_H
        }
    }

    // char = L * cons with the reference's summation order
    // (1D: rt L0 + rut L1 + ret L2, eigenSystem.cpp:260-264;
    //  2D: rut L1 + rvt L2 + ret L3 + rt L0, eigenSystem.cpp:97-106;
    //  3D: rut L1 + rvt L2 + rwt L3 + ret L4 + rt L0).
    CFD_HD double project(int k, const double *cs) const
    {
        if constexpr (NV == 3) {
            return cs[0] * L[k][0] + cs[1] * L[k][1] + cs[2] * L[k][2];
        } else if constexpr (NV == 4) {
            return cs[1] * L[k][1] + cs[2] * L[k][2] + cs[3] * L[k][3] + cs[0] * L[k][0];
        } else {
            return cs[1] * L[k][1] + cs[2] * L[k][2] + cs[3] * L[k][3] + cs[4] * L[k][4] + cs[0] * L[k][0];
        }
    }

    // cons = R * char with the reference's summation order
    // (1D: ch1 R0 + ch2 R1 + ch3 R2, eigenSystem.cpp:300-302;
    //  2D: ch3 R2 + ch4 R3 + ch2 R1 + ch1 R0, eigenSystem.cpp:139-149;
    //  3D: the 2D order followed by + ch5 R4).
    CFD_HD void back(const double *ch, double *cs) const
    {
        for (int i = 0; i < NV; i++) {
            if constexpr (NV == 3) {
                cs[i] = ch[0] * R[i][0] + ch[1] * R[i][1] + ch[2] * R[i][2];
            } else if constexpr (NV == 4) {
                cs[i] = ch[2] * R[i][2] + ch[3] * R[i][3] + ch[1] * R[i][1] + ch[0] * R[i][0];
            } else {
                cs[i] = ch[2] * R[i][2] + ch[3] * R[i][3] + ch[1] * R[i][1] + ch[0] * R[i][0] + ch[4] * R[i][4];
            }
        }
    }
};

// charToPrim's cons -> prim tail (2D: eigenSystem.cpp:163-167; 3D adds w).
template <int NV>
CFD_HD void char_cons_to_prim(const double *cs, double *p)
{
    const double gamma = kGamma;
    if constexpr (NV == 3) {
        // eigensystemEuler1D::consToPrim (eigenSystem.cpp:309-322)
        double rt = cs[0], rut = cs[1], ret = cs[2];
        double ut = rut / rt;
        double ekt = (ut * ut) / 2;  // one division only
        p[0] = rt; p[1] = ut; p[2] = (gamma - 1) * (ret - rt * ekt);
    } else if constexpr (NV == 4) {
        double rt = cs[0], rut = cs[1], rvt = cs[2], ret = cs[3];
#if defined(CFD_FAST)
        const double irt = 1.0 / rt;
        double ut = rut * irt, vt = rvt * irt;
        double rekt = (rut * rut + rvt * rvt) * (0.5 * irt);
#else
        const double irt = rcp_rn(rt);
        const double a[3] = {rut, rvt, rut * rut + rvt * rvt}, bb[3] = {rt, rt, rt}, yy[3] = {irt, irt, irt};
        double qq[3];
        divs_rn<3>(a, bb, yy, qq);
        double ut = qq[0], vt = qq[1];
        double rekt = qq[2] / 2;
#endif
        p[0] = rt; p[1] = ut; p[2] = vt; p[3] = (gamma - 1) * (ret - rekt);
    } else {
        double rt = cs[0], rut = cs[1], rvt = cs[2], rwt = cs[3], ret = cs[4];
#if defined(CFD_FAST)
        const double irt = 1.0 / rt;
        double ut = rut * irt, vt = rvt * irt, wt = rwt * irt;
        double rekt = (rut * rut + rvt * rvt + rwt * rwt) * (0.5 * irt);
#else
        const double irt = rcp_rn(rt);
        const double a[4] = {rut, rvt, rwt, rut * rut + rvt * rvt + rwt * rwt}, bb[4] = {rt, rt, rt, rt},
                     yy[4] = {irt, irt, irt, irt};
        double qq[4];
        divs_rn<4>(a, bb, yy, qq);
        double ut = qq[0], vt = qq[1], wt = qq[2];
        double rekt = qq[3] / 2;
#endif
        p[0] = rt; p[1] = ut; p[2] = vt; p[3] = wt; p[4] = (gamma - 1) * (ret - rekt);
    }
}

// variable_positive_limiter (positive_preserving.hpp:13-46) applied to the
// density (which = 0) or to gamma * p (which = 1) of a 1D cons triple.
CFD_HD double positive_quantity_1d(int which, const double *W)
{
    if (which == 0) return W[0];
    double rho = W[0], rhou = W[1], rhoE = W[2];
    double u = rhou / rho;
    double ekin = 0.5 * u * u;
    double p = (kGamma - 1) * (rhoE - rho * ekin);
    return kGamma * p;
}
CFD_HD void positive_limit_1d(int which, const double *W, double *Wi)
{
    const double EPS = 1e-10;
    double qi = positive_quantity_1d(which, Wi);
    if (qi >= EPS) return;
    double q = positive_quantity_1d(which, W);
    if (q < EPS) {
        for (int i = 0; i < 3; i++) Wi[i] = W[i];
        return;
    }
    double theta = (EPS - q) / (qi - q);
    for (int i = 0; i < 3; i++) Wi[i] = (1 - theta) * W[i] + theta * Wi[i];
}

// variable_positive_limiter (positive_preserving.hpp:13-46) on a 2D/3D cons
// state, the option cfd_config.positivity: which = 0 limits the density,
// which = 1 gamma p with p = (gamma - 1) (rho E - rho |u|^2 / 2), u = (rho u) / rho
// by component. This extends the 1D quantity of reconstructor5order.hpp:210-223
// to the multi-dimensional kinetic energy; the reference itself limits only
// in 1D.
template <int NV>
CFD_HD double positive_quantity_md(int which, const double *W)
{
    if (which == 0) return W[0];
    const double rho = W[0];
    double q2 = 0.0;
    for (int i = 1; i < NV - 1; i++) {
        const double u = W[i] / rho;
        q2 = q2 + u * u;
    }
    const double ekin = 0.5 * q2;
    const double p = (kGamma - 1) * (W[NV - 1] - rho * ekin);
    return kGamma * p;
}
template <int NV>
CFD_HD void positive_limit_md(int which, const double *W, double *Wi)
{
    const double EPS = 1e-10;
    const double qi = positive_quantity_md<NV>(which, Wi);
    if (qi >= EPS) return;
    const double q = positive_quantity_md<NV>(which, W);
    if (q < EPS) {
        for (int i = 0; i < NV; i++) Wi[i] = W[i];
        return;
    }
    const double theta = (EPS - q) / (qi - q);
    for (int i = 0; i < NV; i++) Wi[i] = (1 - theta) * W[i] + theta * Wi[i];
}

// ---------------------------------------------------------------------------
// Face reconstruction (Recon5Order{1D,2D}EulerEig::reconI,
// reconstructor5order.hpp:233-323 and 326-429). cs6/pr6 are the re-derived
// cons and the prim of the six stencil cells (face between cell 2 and 3).
// Writes the left and right face prim states.
// ---------------------------------------------------------------------------
template <int NV, int AX, int FAM>
CFD_HD void reconstruct_face(const double (*pr6)[NV], const double (*cs6)[NV], double icst, double kap,
                             double *fl, double *fr)
{
    Eigen<NV, AX> eig(pr6[2], pr6[3]);
    double QL[NV], QR[NV];
    for (int k = 0; k < NV; k++) {
        double q[6];
        for (int j = 0; j < 6; j++) q[j] = eig.project(k, cs6[j]);
        QL[k] = inter5<FAM>(q[0], q[1], q[2], q[3], q[4], icst, kap);
        QR[k] = inter5<FAM>(q[5], q[4], q[3], q[2], q[1], icst, kap);
    }
    double cl[NV], cr[NV];
    eig.back(QL, cl);
    eig.back(QR, cr);
    if constexpr (NV == 3) {
        double consL[3], consR[3];
        prim_to_cons<3>(pr6[2], consL);
        prim_to_cons<3>(pr6[3], consR);
        positive_limit_1d(0, consL, cl);
        positive_limit_1d(0, consR, cr);
        positive_limit_1d(1, consL, cl);
        positive_limit_1d(1, consR, cr);
        char_cons_to_prim<3>(cl, fl);
        char_cons_to_prim<3>(cr, fr);
    } else {
        char_cons_to_prim<NV>(cl, fl);
        char_cons_to_prim<NV>(cr, fr);
        // crude positivity fallback (reconstructor5order.hpp:380-381), including
        // the reference's mix of right density/pressure with left velocity.
        if (fl[0] < 0 || fl[NV - 1] < 0) {
            for (int i = 0; i < NV; i++) fl[i] = pr6[2][i];
        }
        if (fr[0] < 0 || fr[NV - 1] < 0) {
            fr[0] = pr6[3][0];
            for (int i = 1; i < NV - 1; i++) fr[i] = pr6[2][i];
            fr[NV - 1] = pr6[3][NV - 1];
        }
    }
}

// ---------------------------------------------------------------------------
// Streaming form of the multi-dimensional reconstruction (NV = 4, 5): the Roe
// average is kept as a handful of scalars, eigenvector entries are formed when
// a characteristic field needs them, stencil values are read through an
// accessor (shared memory in the sweep), and the fields are processed in the
// reference's back-projection order 2, 3, 1, 0 (then 4), so each face state
// component accumulates with exactly the rounding of eigenSystem.cpp:139-149.
// Far fewer values are live at once than with the full 4x4 / 5x5 matrices.
// ---------------------------------------------------------------------------
template <int NV, int AX>
struct EigenBase {
    double u, v, w, h, c, ek, Vn;
    double ic, ih;  // 1/c and 1/h (strict: RN(1/c), RN(1/h))
#if !defined(CFD_FAST)
    // strict: the correctly rounded quotients the eigenvectors use, each formed
    // once per face (Vn/c, ek/h, u/h, v/h, w/h)
    double Vc, ekh, uh, vh, wh;
#endif
    static constexpr double nx = (AX == 0) ? 1.0 : 0.0, ny = (AX == 1) ? 1.0 : 0.0, nz = (AX == 2) ? 1.0 : 0.0;

    // the same base quantities as Eigen<NV,AX>'s constructor (eigenSystem.cpp:13-52)
    template <class PR>
    CFD_HD EigenBase(const PR &pr)
    {
        double pl[NV], prr[NV], kl[NV], kr[NV];
#pragma unroll
        for (int m = 0; m < NV; m++) {
            pl[m] = pr(2, m);
            prr[m] = pr(3, m);
        }
        roe_weights(pl, kl);
        roe_weights(prr, kr);
        init(kl, kr);
    }
    // from the two cells' Roe weights (roe_weights), e.g. kept per cell by the sweep
    CFD_HD EigenBase(const double *kl, const double *kr) { init(kl, kr); }

    // A cell's share of the Roe average: (sqrt(rho), sqrt(rho) u, sqrt(rho) v,
    // [sqrt(rho) w,] sqrt(rho) H), each product rounded as the reference's
    // coef * v and coef * H are (eigenSystem.cpp:17-30); H = |v|^2 / 2 +
    // p / rho * gamma / (gamma - 1).
    static CFD_HD void roe_weights(const double *p, double *k)
    {
        constexpr int D = NV - 2, E = NV - 1;
        const double r = p[0], pp = p[E];
        double q2 = p[1] * p[1] + p[2] * p[2];
        if constexpr (D == 3) q2 = q2 + p[3] * p[3];
#if defined(CFD_FAST)
        // sqrt(rho) = rho rsqrt(rho), sqrt(rho) H = sqrt(rho) |v|^2 / 2 +
        // gamma/(gamma-1) p rsqrt(rho)
        const double ir = rsqrt(r);
        const double coef = r * ir;
        k[E] = 0.5 * (coef * q2) + kG1 * (pp * ir);
#else
        const double coef = sqrt(r);
        const double H = q2 / 2 + div_rn(pp / r * kGamma, kGm1, kRcpGm1);
        k[E] = coef * H;
#endif
        k[0] = coef;
#pragma unroll
        for (int i = 0; i < D; i++) k[1 + i] = coef * p[1 + i];
    }

  private:
    CFD_HD void init(const double *kl, const double *kr)
    {
        constexpr int D = NV - 2;
        const double gamma = kGamma;
        const double divisor = 1.0 / (kl[0] + kr[0]);
        u = (kl[1] + kr[1]) * divisor;
        v = (kl[2] + kr[2]) * divisor;
        w = (D == 3) ? (kl[3] + kr[3]) * divisor : 0.0;
        const double ht = (kl[NV - 1] + kr[NV - 1]) * divisor;
        if constexpr (D == 2) {
            Vn = nx * u + ny * v;
            ek = (u * u + v * v) / 2;
        } else {
            Vn = nx * u + ny * v + nz * w;
            ek = (u * u + v * v + w * w) / 2;
        }
        h = ht - ek;
#if defined(CFD_FAST)
        // 1/c = rsqrt(c^2), 1/h = (gamma - 1) / c^2
        const double c2 = (gamma - 1) * h;
        ic = rsqrt(c2);
        c = c2 * ic;
        ih = (gamma - 1) * (ic * ic);
#else
        c = sqrt((gamma - 1) * h);
        ic = rcp_rn(c);
        ih = rcp_rn(h);
        if constexpr (D == 2) {
            const double a[4] = {Vn, ek, u, v}, bb[4] = {c, h, h, h}, yy[4] = {ic, ih, ih, ih};
            double qq[4];
            divs_rn<4>(a, bb, yy, qq);
            Vc = qq[0]; ekh = qq[1]; uh = qq[2]; vh = qq[3];
            wh = 0.0;
        } else {
            const double a[5] = {Vn, ek, u, v, w}, bb[5] = {c, h, h, h, h}, yy[5] = {ic, ih, ih, ih, ih};
            double qq[5];
            divs_rn<5>(a, bb, yy, qq);
            Vc = qq[0]; ekh = qq[1]; uh = qq[2]; vh = qq[3]; wh = qq[4];
        }
#endif
    }

  public:
#if defined(CFD_FAST)
    CFD_HD double dc(double a) const { return a * ic; }
    CFD_HD double dh(double a) const { return a * ih; }
#endif
    // (s n_i) / c for a unit normal component n_i (0 or 1) and s = -1 or 1:
    // the correctly rounded 1/c with the sign, or a signed zero, exactly as
    // the division rounds it
    CFD_HD double sn_c(double s, double n) const { return (s * n) * ic; }
    // left eigenvector k, column m (eigenSystem.cpp:53-68 and the 3D extension)
    CFD_HD double L(int k, int m) const
    {
        constexpr int E = NV - 1;
        if (k == 0) {
            if (AX != 2) return m == 0 ? (-ny * u + nx * v) : m == 1 ? ny : m == 2 ? (-nx) : (m == E ? 0 : 0.0);
            return m == 0 ? -u : m == 1 ? 1.0 : 0.0;
        }
        if (k == 1) return m == 0 ? (h - ek) : m == 1 ? u : m == 2 ? v : m == E ? -1.0 : w;
        if (k == 2 || k == 3) {
            const double s = (k == 2) ? -1.0 : 1.0;
            // 1 / (2 h) = RN(1/h) / 2 exactly
            if (m == E) return 0.5 * ih;
#if defined(CFD_FAST)
            if (m == 0) return (k == 2) ? (dc(Vn) + dh(ek)) / 2 : (dc(-Vn) + dh(ek)) / 2;
            if (m == 1) return (dc(s * nx) - dh(u)) / 2;
            if (m == 2) return (dc(s * ny) - dh(v)) / 2;
            return (dc(s * nz) - dh(w)) / 2;
#else
            // (-Vn) / c = -(Vn / c) exactly
            if (m == 0) return (k == 2) ? (Vc + ekh) / 2 : (-Vc + ekh) / 2;
            if (m == 1) return (sn_c(s, nx) - uh) / 2;
            if (m == 2) return (sn_c(s, ny) - vh) / 2;
            return (sn_c(s, nz) - wh) / 2;
#endif
        }
        // k == 4: second shear wave (3D only)
        if (AX != 2) return m == 0 ? -w : m == 3 ? 1.0 : 0.0;
        return m == 0 ? -v : m == 2 ? 1.0 : 0.0;
    }
    // right eigenvector k, row i (eigenSystem.cpp:70-85 and the 3D extension)
    CFD_HD double R(int i, int k) const
    {
        constexpr int E = NV - 1;
        if (k == 0) {
            if (AX != 2) return i == 0 ? 0.0 : i == 1 ? ny : i == 2 ? -nx : i == E ? ny * u - nx * v : 0.0;
            return i == 1 ? 1.0 : i == E ? u : 0.0;
        }
#if defined(CFD_FAST)
        if (k == 1) return i == 0 ? dh(1.0) : i == 1 ? dh(u) : i == 2 ? dh(v) : i == E ? dh(ek) : dh(w);
#else
        if (k == 1) return i == 0 ? ih : i == 1 ? uh : i == 2 ? vh : i == E ? ekh : wh;
#endif
        if (k == 2 || k == 3) {
            const double s = (k == 2) ? -1.0 : 1.0;
            if (i == 0) return 1.0;
            if (i == E) return (k == 2) ? h + ek - Vn * c : h + ek + Vn * c;
            if (i == 1) return (k == 2) ? u - nx * c : u + nx * c;
            if (i == 2) return (k == 2) ? v - ny * c : v + ny * c;
            (void)s;
            return (k == 2) ? w - nz * c : w + nz * c;
        }
        if (AX != 2) return i == 3 ? 1.0 : i == 4 ? w : 0.0;
        return i == 2 ? 1.0 : i == 4 ? v : 0.0;
    }
};

// cs(j, v): re-derived cons of stencil cell j (0..5), pr(j, v): its prim;
// eb: the face's Roe-averaged eigensystem; posl: the positivity option
// (cfd_config.positivity) instead of the reference's fallback.
template <int NV, int AX, int FAM, class CS, class PR>
CFD_HD void reconstruct_face_stream(const EigenBase<NV, AX> &eb, const CS &cs, const PR &pr, double icst, double kap,
                                    double *fl, double *fr, int posl = 0)
{
    static_assert(NV == 4 || NV == 5, "multi-dimensional form");
    double cl[NV], cr[NV];
    // Fully unrolled: the instruction-level parallelism across fields beats the
    // smaller code of a rolled loop (measured on B200: 22.0 vs 31.9 ms per 3D
    // 256^3 step). CFD_ROLL_FIELDS builds the rolled form (uniform branches).
#if defined(CFD_ROLL_FIELDS)
#pragma unroll 1
#else
#pragma unroll
#endif
    for (int kk = 0; kk < NV; kk++) {
        const int k = (kk == 0) ? 2 : (kk == 1) ? 3 : (kk == 2) ? 1 : (kk == 3) ? 0 : 4;
        double l[NV];
#pragma unroll
        for (int m = 0; m < NV; m++) l[m] = eb.L(k, m);
        double q[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {
            // primToChar's order: rut L1 + rvt L2 [+ rwt L3] + ret LE + rt L0
            double a = cs(j, 1) * l[1] + cs(j, 2) * l[2];
#pragma unroll
            for (int m = 3; m < NV; m++) a = a + cs(j, m) * l[m];
            q[j] = a + cs(j, 0) * l[0];
        }
        double QL, QR;
#if !defined(CFD_ROLL_FIELDS)
        QL = inter5<FAM>(q[0], q[1], q[2], q[3], q[4], icst, kap);
        QR = inter5<FAM>(q[5], q[4], q[3], q[2], q[1], icst, kap);
#else
        // one interpolator body for both states (mirrored stencil on side 1)
#pragma unroll 1
        for (int side = 0; side < 2; side++) {
            const bool m = side != 0;
            const double r = inter5<FAM>(m ? q[5] : q[0], m ? q[4] : q[1], q[m ? 3 : 2], q[m ? 2 : 3],
                                         m ? q[1] : q[4], icst, kap);
            if (m) QR = r; else QL = r;
        }
#endif
#pragma unroll
        for (int i = 0; i < NV; i++) {
            const double r = eb.R(i, k);
            if (kk == 0) {
                cl[i] = QL * r;
                cr[i] = QR * r;
            } else {
                cl[i] = cl[i] + QL * r;
                cr[i] = cr[i] + QR * r;
            }
        }
    }
    if (posl) {
        // the 1D char-recon limiter (reconstructor5order.hpp:225-236): density
        // of both states, then gamma p of both, against the cells' cons
        double WL[NV], WR[NV];
#pragma unroll
        for (int i = 0; i < NV; i++) {
            WL[i] = cs(2, i);
            WR[i] = cs(3, i);
        }
        positive_limit_md<NV>(0, WL, cl);
        positive_limit_md<NV>(0, WR, cr);
        positive_limit_md<NV>(1, WL, cl);
        positive_limit_md<NV>(1, WR, cr);
        char_cons_to_prim<NV>(cl, fl);
        char_cons_to_prim<NV>(cr, fr);
        return;
    }
    char_cons_to_prim<NV>(cl, fl);
    char_cons_to_prim<NV>(cr, fr);
    // crude positivity fallback (reconstructor5order.hpp:380-381), including
    // the reference's mix of right density/pressure with left velocity.
    if (fl[0] < 0 || fl[NV - 1] < 0) {
        for (int i = 0; i < NV; i++) fl[i] = pr(2, i);
    }
    if (fr[0] < 0 || fr[NV - 1] < 0) {
        fr[0] = pr(3, 0);
        for (int i = 1; i < NV - 1; i++) fr[i] = pr(2, i);
        fr[NV - 1] = pr(3, NV - 1);
    }
}

// The same with the eigensystem formed from the prim of stencil cells 2 and 3.
template <int NV, int AX, int FAM, class CS, class PR>
CFD_HD void reconstruct_face_stream(const CS &cs, const PR &pr, double icst, double kap, double *fl, double *fr,
                                    int posl = 0)
{
    const EigenBase<NV, AX> eb(pr);
    reconstruct_face_stream<NV, AX, FAM>(eb, cs, pr, icst, kap, fl, fr, posl);
}

// ---------------------------------------------------------------------------
// Riemann fluxes.
// ---------------------------------------------------------------------------
enum FluxKind : int { FLUX_HLLC = 0, FLUX_ROE = 1 };

// HLLCFlux1D (fluxSchemes.hpp:74-125)
CFD_HD void hllc_1d(const double *L, const double *R, double *res)
{
    const double gamma = kGamma;
    double rl = L[0], ul = L[1], pl = L[2], rr = R[0], ur = R[1], pr = R[2];
    double HL = pl / rl * kGamma / (kGamma - 1) + (ul * ul) / 2;
    double HR = pr / rr * kGamma / (kGamma - 1) + (ur * ur) / 2;
    double cl = sqrt(gamma * (pl / rl));
    double cr = sqrt(gamma * (pr / rr));
    // std::min(ur - cr, ul - cl) and std::max(ul + cl, ur + cr)
    double SL = ((ul - cl) < (ur - cr)) ? (ul - cl) : (ur - cr);
    double SR = ((ul + cl) < (ur + cr)) ? (ur + cr) : (ul + cl);
    double Sstar = ((pr - pl) + (rl * ul * (SL - ul) - rr * ur * (SR - ur))) / (rl * (SL - ul) - rr * (SR - ur));
    if (SL >= 0) {
        res[0] = rl * ul; res[1] = rl * ul * ul + pl; res[2] = rl * HL * ul;
    } else if (Sstar >= 0) {
        double pStar = pl + rl * (SL - ul) * (Sstar - ul);
        double U[3] = {rl, rl * ul, pl / (gamma - 1) + rl * ul * ul / 2};
        double F[3] = {rl * ul, rl * ul * ul + pl, rl * HL * ul};
        double D[3] = {0, 1, Sstar};
        for (int i = 0; i < 3; i++) res[i] = (Sstar * (SL * U[i] - F[i]) + SL * pStar * D[i]) / (SL - Sstar);
    } else if (SR >= 0) {
        double pStar = pr + rr * (SR - ur) * (Sstar - ur);
        double U[3] = {rr, rr * ur, pr / (gamma - 1) + rr * ur * ur / 2};
        double F[3] = {rr * ur, rr * ur * ur + pr, rr * HR * ur};
        double D[3] = {0, 1, Sstar};
        for (int i = 0; i < 3; i++) res[i] = (Sstar * (SR * U[i] - F[i]) + SR * pStar * D[i]) / (SR - Sstar);
    } else {
        res[0] = rr * ur; res[1] = rr * ur * ur + pr; res[2] = rr * HR * ur;
    }
}

// roeFlux1D2 (fluxSchemes.hpp:13-71)
CFD_HD void roe_1d(const double *L, const double *R, double *res)
{
    const double gamma = kGamma;
    double rl = L[0], ul = L[1], pl = L[2], rr = R[0], ur = R[1], pr = R[2];
    double HL = pl / rl * kGamma / (kGamma - 1) + (ul * ul) / 2;
    double HR = pr / rr * kGamma / (kGamma - 1) + (ur * ur) / 2;
    double srl = sqrt(rl), srr = sqrt(rr);
    double rBar = sqrt(rl * rr);
    double uBar = (ul * srl + ur * srr) / (srl + srr);
    double HBar = (HL * srl + HR * srr) / (srl + srr);
    double cBar = sqrt((gamma - 1) * (HBar - uBar * uBar / 2));
    double cBar2 = (gamma - 1) * (HBar - uBar * uBar / 2);
    double dr = rr - rl, du = ur - ul, dp = pr - pl;
    double lambda[3] = {fabs(uBar), fabs(uBar + cBar), fabs(uBar - cBar)};
    double eps = 0.1 * (fabs(uBar) + cBar);
    for (int i = 0; i < 3; i++)
        if (lambda[i] < eps) lambda[i] = (lambda[i] * lambda[i] + eps * eps) / (2.0 * eps);
    double a0 = lambda[0] * (dr - dp / cBar2);
    double a1 = lambda[1] / (2.0 * cBar2) * (dp + rBar * cBar * du);
    double a2 = lambda[2] / (2.0 * cBar2) * (dp - rBar * cBar * du);
    double a3 = a0 + a1 + a2;
    double a4 = cBar * (a1 - a2);
    double FL[3] = {rl * ul, rl * ul * ul + pl, rl * HL * ul};
    double FR[3] = {rr * ur, rr * ur * ur + pr, rr * HR * ur};
    for (int i = 0; i < 3; i++) res[i] = (FL[i] + FR[i]) / 2.0;
    res[0] -= 0.5 * a3;
    res[1] -= 0.5 * (a3 * uBar + a4);
    res[2] -= 0.5 * (HBar * a3 + uBar * a4 - cBar2 * a0 / (gamma - 1));
}

// HLLCFlux2D2 (fluxSchemes.hpp:202-327); the 3D form treats the two
// tangential momentum components alike.
template <int NV, int AX>
CFD_HD void hllc_md(const double *L, const double *R, double *res)
{
    constexpr int D = NV - 2, E = NV - 1;
    const double gamma = kGamma;
    const double n[3] = {AX == 0 ? 1.0 : 0.0, AX == 1 ? 1.0 : 0.0, AX == 2 ? 1.0 : 0.0};
    double rl = L[0], rr = R[0], pl = L[E], pr = R[E];
    const double *vl = L + 1, *vr = R + 1;
    double HL, HR;
#if defined(CFD_FAST)
    const double prl = pl * (1.0 / rl), prr = pr * (1.0 / rr);  // p / rho
    {
        double kl = vl[0] * vl[0] + vl[1] * vl[1], kr = vr[0] * vr[0] + vr[1] * vr[1];
        if constexpr (D == 3) { kl += vl[2] * vl[2]; kr += vr[2] * vr[2]; }
        HL = 0.5 * kl + prl * kG1;
        HR = 0.5 * kr + prr * kG1;
    }
    double VnL = vl[AX], VnR = vr[AX];
    double cl = sqrt(prl * gamma), cr = sqrt(prr * gamma);
#else
    const double prl = pl / rl, prr = pr / rr;
    // x / (gamma - 1) by its correctly rounded reciprocal (divs_rn)
    {
        const double a[2] = {prl * kGamma, prr * kGamma}, bb[2] = {kGm1, kGm1}, yy[2] = {kRcpGm1, kRcpGm1};
        double qq[2];
        divs_rn<2>(a, bb, yy, qq);
        if constexpr (D == 2) {
            HL = (vl[0] * vl[0] + vl[1] * vl[1]) / 2 + qq[0];
            HR = (vr[0] * vr[0] + vr[1] * vr[1]) / 2 + qq[1];
        } else {
            HL = (vl[0] * vl[0] + vl[1] * vl[1] + vl[2] * vl[2]) / 2 + qq[0];
            HR = (vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]) / 2 + qq[1];
        }
    }
    double VnL = vl[AX], VnR = vr[AX];
    double cl = sqrt(prl * gamma), cr = sqrt(prr * gamma);
#endif
    double rBar = (rl + rr) / 2, cBar = (cl + cr) / 2;
    double ps0 = (pl + pr) / 2 - rBar * cBar * (VnR - VnL) / 2;
    double ps = (0.0 < ps0) ? ps0 : 0.0;  // std::max(0.0, .)
    double ql = (ps <= pl) ? 1.0 : sqrt(1.0 + (gamma + 1.0) / (2.0 * gamma) * (ps / pl - 1.0));
    double qr = (ps <= pr) ? 1.0 : sqrt(1.0 + (gamma + 1.0) / (2.0 * gamma) * (ps / pr - 1.0));
    double SL = VnL - cl * ql, SR = VnR + cr * qr;
    double Sstar = ((pr - pl) + (rl * VnL * (SL - VnL) - rr * VnR * (SR - VnR))) / (rl * (SL - VnL) - rr * (SR - VnR));

    // Physical flux F and star-state difference for one side
    // (the reference spells the tangential selector as u*norm[1] / v*norm[0];
    // for unit axis normals that is u_i * (1 - n_i)).
    auto side_flux = [&](double r, const double *v, double p, double H, double Vn, double S, double *out, double scale,
                         bool accumulate) {
        double U[NV], F[NV], Ustar[NV];
        U[0] = r;
        for (int i = 0; i < D; i++) U[1 + i] = r * v[i];
        U[E] = r * H - p;
        F[0] = r * Vn;
        for (int i = 0; i < D; i++) F[1 + i] = r * v[i] * Vn + p * n[i];
        F[E] = r * H * Vn;
        double Usf = (S - Vn) / (S - Sstar);
        Ustar[0] = Usf * r;
        for (int i = 0; i < D; i++) Ustar[1 + i] = Usf * (Sstar * n[i] + v[i] * (1.0 - n[i])) * r;
        Ustar[E] = Usf * (U[E] + (Sstar - Vn) * (r * Sstar + p / (S - Vn)));
        for (int i = 0; i < NV; i++) {
            double f = F[i] + S * (Ustar[i] - U[i]);
            f = (scale != 1.0) ? f / 2 : f;
            out[i] = accumulate ? out[i] + f : f;
        }
    };
    if (SL > 0) {
        res[0] = rl * VnL;
        for (int i = 0; i < D; i++) res[1 + i] = rl * vl[i] * VnL + pl * n[i];
        res[E] = rl * HL * VnL;
    } else if (Sstar > 0 || Sstar == 0 || SR > 0) {
        // The star-region branches of the reference in one body: S* > 0 takes
        // the left side, S* < 0 < SR the right one, and S* = 0 the average of
        // both halves (left first, then the right half added), so the side
        // flux is emitted once.
        const bool avg = (Sstar == 0);
        const bool left = (Sstar > 0) || avg;
#pragma unroll 1
        for (int it = 0; it < (avg ? 2 : 1); it++) {
            const bool useL = left && it == 0;
            double vs[D];
#pragma unroll
            for (int i = 0; i < D; i++) vs[i] = useL ? vl[i] : vr[i];
            side_flux(useL ? rl : rr, vs, useL ? pl : pr, useL ? HL : HR, useL ? VnL : VnR, useL ? SL : SR, res,
                      avg ? 0.5 : 1.0, it > 0);
        }
    } else {
        res[0] = rr * VnR;
        for (int i = 0; i < D; i++) res[1 + i] = rr * vr[i] * VnR + pr * n[i];
        res[E] = rr * HR * VnR;
    }
}

#if defined(CFD_FAST)
// roeFlux2DSym with reciprocal square roots instead of its divisions and square
// roots: sqrt(rho) = rho rsqrt(rho), sqrt(rho) H = sqrt(rho) |v|^2 / 2 +
// gamma/(gamma-1) p rsqrt(rho), rho H = rho |v|^2 / 2 + gamma/(gamma-1) p,
// 1/c = rsqrt(c^2); the entropy fix's 1/(2 eps) only where a wave needs it.
template <int NV, int AX>
CFD_HD void roe_md_fast(const double *L, const double *R, double *res)
{
    constexpr int D = NV - 2, E = NV - 1;
    const double n[3] = {AX == 0 ? 1.0 : 0.0, AX == 1 ? 1.0 : 0.0, AX == 2 ? 1.0 : 0.0};
    const double rl = L[0], rr = R[0], pl = L[E], pr = R[E];
    const double *vl = L + 1, *vr = R + 1;
    double kl = vl[0] * vl[0] + vl[1] * vl[1], kr = vr[0] * vr[0] + vr[1] * vr[1];
    if constexpr (D == 3) { kl += vl[2] * vl[2]; kr += vr[2] * vr[2]; }
    const double VnL = vl[AX], VnR = vr[AX];
    double Fc[NV];
    Fc[0] = rl * VnL + rr * VnR;
    for (int i = 0; i < D; i++) Fc[1 + i] = rl * vl[i] * VnL + rr * vr[i] * VnR + (pl + pr) * n[i];
    Fc[E] = (0.5 * rl * kl + kG1 * pl) * VnL + (0.5 * rr * kr + kG1 * pr) * VnR;

    const double ir1 = rsqrt(rl), ir2 = rsqrt(rr);
    const double coef1 = rl * ir1, coef2 = rr * ir2;
    const double divisor = 1.0 / (coef1 + coef2);
    const double rhoAvg = coef1 * coef2;
    double vAvg[3];
    for (int i = 0; i < D; i++) vAvg[i] = (coef1 * vl[i] + coef2 * vr[i]) * divisor;
    const double HAvg = (0.5 * (coef1 * kl + coef2 * kr) + kG1 * (pl * ir1 + pr * ir2)) * divisor;
    double q_2Avg;
    if constexpr (D == 2) q_2Avg = (vAvg[0] * vAvg[0] + vAvg[1] * vAvg[1]) / 2;
    else q_2Avg = (vAvg[0] * vAvg[0] + vAvg[1] * vAvg[1] + vAvg[2] * vAvg[2]) / 2;
    const double c2 = (kGamma - 1) * (HAvg - q_2Avg);
    const double ic = rsqrt(c2);
    const double cAvg = c2 * ic, ic2 = ic * ic;
    const double VnAvg = vAvg[AX];
    double lambda[3] = {fabs(VnAvg - cAvg), fabs(VnAvg), fabs(VnAvg + cAvg)};
    const double eps = 0.05 * (fabs(VnAvg) + cAvg);
    if (lambda[0] < eps || lambda[1] < eps || lambda[2] < eps) {
        const double ie2 = 0.5 / eps;
        for (int i = 0; i < 3; i++)
            if (lambda[i] < eps) lambda[i] = (lambda[i] * lambda[i] + eps * eps) * ie2;
    }
    const double deltaP = pr - pl, deltaVn = VnR - VnL, deltaRho = rr - rl;
    const double rc = rhoAvg * cAvg * deltaVn;
    const double a1 = lambda[0] * ((deltaP - rc) * (0.5 * ic2));
    const double a3 = lambda[2] * ((deltaP + rc) * (0.5 * ic2));
    const double a2 = lambda[1] * (deltaRho - deltaP * ic2);
    const double l1r = lambda[1] * rhoAvg;
    double Fd[NV];
    Fd[0] = a1 + a3 + a2;
    double tE = 0.0;
    for (int i = 0; i < D; i++) {
        const double ti = (i == AX) ? 0.0 : vr[i] - vl[i];
        Fd[1 + i] = a1 * (vAvg[i] - cAvg * n[i]) + a3 * (vAvg[i] + cAvg * n[i]) + a2 * vAvg[i] + l1r * ti;
        if (i != AX) tE += vAvg[i] * ti;
    }
    Fd[E] = a1 * (HAvg - cAvg * VnAvg) + a3 * (HAvg + cAvg * VnAvg) + a2 * q_2Avg + l1r * tE;
    for (int i = 0; i < NV; i++) res[i] = 0.5 * (Fc[i] - Fd[i]);
}
#endif

// Harten's entropy fix of roeFlux2DSym (fluxSchemes.hpp:499-505): a wave speed
// below eps becomes (lambda^2 + eps^2) / (2 eps). Out of line: few faces take
// it, and its three divisions stay out of the sweep's instruction stream.
struct Lam3 {
    double a, b, c;
};
#if defined(__CUDACC__)
static __host__ __device__ __noinline__
#else
static inline
#endif
Lam3 entropy_fix3(double l0, double l1, double l2, double eps)
{
    double l[3] = {l0, l1, l2};
    for (int i = 0; i < 3; i++)
        if (l[i] < eps) l[i] = (l[i] * l[i] + eps * eps) / (2.0 * eps);
    return Lam3{l[0], l[1], l[2]};
}

// roeFlux2DSym (fluxSchemes.hpp:420-553), 3D form with both tangential
// components in the linear wave.
template <int NV, int AX>
CFD_HD void roe_md(const double *L, const double *R, double *res)
{
#if defined(CFD_FAST)
    roe_md_fast<NV, AX>(L, R, res);
#else
    constexpr int D = NV - 2, E = NV - 1;
    const double n[3] = {AX == 0 ? 1.0 : 0.0, AX == 1 ? 1.0 : 0.0, AX == 2 ? 1.0 : 0.0};
    double rl = L[0], rr = R[0], pl = L[E], pr = R[E];
    const double *vl = L + 1, *vr = R + 1;
    double HL, HR;
    // x / (gamma - 1) by its correctly rounded reciprocal (divs_rn)
    {
        const double a[2] = {pl / rl * kGamma, pr / rr * kGamma}, bb[2] = {kGm1, kGm1}, yy[2] = {kRcpGm1, kRcpGm1};
        double qq[2];
        divs_rn<2>(a, bb, yy, qq);
        if constexpr (D == 2) {
            HL = (vl[0] * vl[0] + vl[1] * vl[1]) / 2 + qq[0];
            HR = (vr[0] * vr[0] + vr[1] * vr[1]) / 2 + qq[1];
        } else {
            HL = (vl[0] * vl[0] + vl[1] * vl[1] + vl[2] * vl[2]) / 2 + qq[0];
            HR = (vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]) / 2 + qq[1];
        }
    }
    double VnL = vl[AX], VnR = vr[AX];
    double FcL[NV], FcR[NV];
    FcL[0] = rl * VnL;
    for (int i = 0; i < D; i++) FcL[1 + i] = rl * vl[i] * VnL + pl * n[i];
    FcL[E] = rl * HL * VnL;
    FcR[0] = rr * VnR;
    for (int i = 0; i < D; i++) FcR[1 + i] = rr * vr[i] * VnR + pr * n[i];
    FcR[E] = rr * HR * VnR;

    double coef1 = sqrt(rl), coef2 = sqrt(rr);
    double divisor = 1.0 / (coef1 + coef2);
    double rhoAvg = sqrt(rl * rr);
    double vAvg[3];
    for (int i = 0; i < D; i++) vAvg[i] = (coef1 * vl[i] + coef2 * vr[i]) * divisor;
    double HAvg = (coef1 * HL + coef2 * HR) * divisor;
    double q_2Avg;
    if constexpr (D == 2) q_2Avg = (vAvg[0] * vAvg[0] + vAvg[1] * vAvg[1]) / 2;
    else q_2Avg = (vAvg[0] * vAvg[0] + vAvg[1] * vAvg[1] + vAvg[2] * vAvg[2]) / 2;
    double cAvg = sqrt((kGamma - 1) * (HAvg - q_2Avg));
    double VnAvg = vAvg[AX];
    double lambda[3] = {fabs(VnAvg - cAvg), fabs(VnAvg), fabs(VnAvg + cAvg)};
    double eps = 0.05 * (fabs(VnAvg) + cAvg);
    if (lambda[0] < eps || lambda[1] < eps || lambda[2] < eps) {
        const Lam3 fx = entropy_fix3(lambda[0], lambda[1], lambda[2], eps);
        lambda[0] = fx.a;
        lambda[1] = fx.b;
        lambda[2] = fx.c;
    }

    double deltaP = pr - pl, deltaVn = VnR - VnL, deltaRho = rr - rl;
    double dv[3];
    for (int i = 0; i < D; i++) dv[i] = vr[i] - vl[i];
    double Fd[NV];
    // the three quotients by c^2 and 2 c^2 from one correctly rounded
    // reciprocal: (2 c) c = 2 RN(c c) exactly, so x / (2 c c) = RN(x / (c c)) / 2
    const double cc2 = cAvg * cAvg, icc2 = rcp_rn(cc2);
    double qc[3];
    {
        const double a[3] = {deltaP - rhoAvg * cAvg * deltaVn, deltaP + rhoAvg * cAvg * deltaVn, deltaP},
                     bb[3] = {cc2, cc2, cc2}, yy[3] = {icc2, icc2, icc2};
        divs_rn<3>(a, bb, yy, qc);
    }
    double c1 = qc[0] / 2;
    Fd[0] = lambda[0] * (c1 * 1);
    for (int i = 0; i < D; i++) Fd[1 + i] = lambda[0] * (c1 * (vAvg[i] - cAvg * n[i]));
    Fd[E] = lambda[0] * (c1 * (HAvg - cAvg * VnAvg));

    double cc = qc[1] / 2;
    Fd[0] += lambda[2] * (cc * 1);
    for (int i = 0; i < D; i++) Fd[1 + i] += lambda[2] * (cc * (vAvg[i] + cAvg * n[i]));
    Fd[E] += lambda[2] * (cc * (HAvg + cAvg * VnAvg));

    double c2 = deltaRho - qc[2];
    Fd[0] += lambda[1] * (c2 * 1.0 + rhoAvg * 0.0);
    // tangential components carry rhoAvg * dv_i, the normal one 0
    // (fluxSchemes.hpp:526-528 for axis normals).
    double tE = 0.0;
    bool first = true;
    for (int i = 0; i < D; i++) {
        double ti = (i == AX) ? 0 : dv[i];
        Fd[1 + i] += lambda[1] * (c2 * vAvg[i] + rhoAvg * ti);
        if (i != AX) {
            double term = vAvg[i] * dv[i];
            if (first) { tE = term; first = false; } else tE = tE + term;
        }
    }
    Fd[E] += lambda[1] * (c2 * q_2Avg + rhoAvg * tE);
    for (int i = 0; i < NV; i++) res[i] = (FcL[i] + FcR[i] - Fd[i]) / 2;
#endif
}

template <int NV, int AX, int FLUX>
CFD_HD void riemann(const double *L, const double *R, double *res)
{
    if constexpr (NV == 3) {
        if constexpr (FLUX == FLUX_HLLC) hllc_1d(L, R, res); else roe_1d(L, R, res);
    } else {
        if constexpr (FLUX == FLUX_HLLC) hllc_md<NV, AX>(L, R, res); else roe_md<NV, AX>(L, R, res);
    }
}

// Physical (node) flux: fluxSolveEuler1D / fluxSolveEuler2D
// (fluxSchemes.hpp:572-599); the 3D form adds w.
template <int NV, int AX>
CFD_HD void node_flux(const double *p, double *f)
{
    if constexpr (NV == 3) {
        double r = p[0], u = p[1], pp = p[2];
        f[0] = r * u;
        f[1] = r * u * u + pp;
        f[2] = (kGamma / (kGamma - 1) * pp + r * (u * u) / 2) * u;
    } else {
        constexpr int D = NV - 2, E = NV - 1;
        const double n[3] = {AX == 0 ? 1.0 : 0.0, AX == 1 ? 1.0 : 0.0, AX == 2 ? 1.0 : 0.0};
        double r = p[0], pp = p[E];
        double Vn;
        if constexpr (D == 2) Vn = (p[1] * n[0] + p[2] * n[1]);
        else Vn = (p[1] * n[0] + p[2] * n[1] + p[3] * n[2]);
        f[0] = r * Vn;
        for (int i = 0; i < D; i++) f[1 + i] = r * p[1 + i] * Vn + n[i] * pp;
        double q2;
        if constexpr (D == 2) q2 = (p[1] * p[1] + p[2] * p[2]);
        else q2 = (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
        f[E] = (q2 / 2 * r + kGamma / (kGamma - 1) * pp) * Vn;
    }
}

// MidNodeAndNodeDif6 (differ.cpp:54-103): one cell's contribution,
// (w1 (Fn[i+1]-Fn[i-1]) + w0 (Fh[i+1/2]-Fh[i-1/2]) + w2 (Fh[i+3/2]-Fh[i-3/2])) / h.
// The numerator of mnd6 (the difference before the division by h).
CFD_HD double mnd6_num(double fnm1, double fnp1, double fhm3, double fhm1, double fhp1, double fhp3)
{
    const double w0 = 3.0 / 2.0, w1 = -3.0 / 10.0, w2 = 1.0 / 30.0;
    return w1 * (fnp1 - fnm1) + w0 * (fhp1 - fhm1) + w2 * (fhp3 - fhm3);
}

CFD_HD double mnd6(double fnm1, double fnp1, double fhm3, double fhm1, double fhp1, double fhp3, double h,
                   double inv_h)
{
    const double w0 = 3.0 / 2.0, w1 = -3.0 / 10.0, w2 = 1.0 / 30.0;
#if defined(CFD_FAST)
    (void)h;
    return (w1 * (fnp1 - fnm1) + w0 * (fhp1 - fhm1) + w2 * (fhp3 - fhm3)) * inv_h;
#else
    return div_rn(w1 * (fnp1 - fnm1) + w0 * (fhp1 - fhm1) + w2 * (fhp3 - fhm3), h, inv_h);
#endif
}

// ExplicitDif6::solve (differ.cpp:23-52): the sixth-order explicit difference
// of the face fluxes x_{i-5/2} .. x_{i+5/2} (no node fluxes), in the
// reference's order of operations.
CFD_HD double trad6(double fhm5, double fhm3, double fhm1, double fhp1, double fhp3, double fhp5, double h,
                    double inv_h)
{
    const double w0 = 75.0 / 64.0, w1 = 25.0 / (128.0 * 3.0), w2 = 3.0 / (128.0 * 5.0);
#if defined(CFD_FAST)
    (void)h;
    return (w0 * (fhp1 - fhm1) - w1 * (fhp3 - fhm3) + w2 * (fhp5 - fhm5)) * inv_h;
#else
    return div_rn(w0 * (fhp1 - fhm1) - w1 * (fhp3 - fhm3) + w2 * (fhp5 - fhm5), h, inv_h);
#endif
}

} // namespace cfd
