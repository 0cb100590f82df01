// Discrete adjoint of one RHS evaluation (cfd_rhs_vjp, cfd_adjoint_*), fast
// flavour (FMA), 2D Euler, WCNS5 or TENO (frozen cut-off) + Roe + MND6,
// periodic in both directions.
//
// The forward path per line (SpDistributor::rhsSolve, sp_distributor.cpp:3-79):
//   face j (x_{j-1/2}), stencil cells j-3..j+2:
//     Roe average of cells j-1, j           (eigensystemEuler2D, eigenSystem.cpp:13-86)
//     q_k = L_k . U for the six cells        (primToChar, eigenSystem.cpp:88-123)
//     QL_k = W(q_k[0..4]), QR_k = W(q_k[5..1]) (weno5_JSchen, interScheme.hpp:17-45, or a
//                                            TENO stencil with its flag frozen, adjoint_math.h)
//     face cons R QL / R QR, then prims, positivity fallback
//                                            (Recon5Order2DEulerEig::reconI, reconstructor5order.hpp:246-356)
//     F_j = Roe(face prims)                  (roeFlux2DSym, fluxSchemes.hpp:420-553)
//   node fluxes G_i                          (fluxSolveEuler2D, fluxSchemes.hpp:572-599)
//   R_i = (w1 (G_{i+1} - G_{i-1}) + w0 (F_{i+1} - F_i) + w2 (F_{i+2} - F_{i-1})) / h
//                                            (MidNodeAndNodeDif6, differ.cpp:54-103)
// Reverse: the face adjoint is Fbar_j = (w0 (mu_{j-1} - mu_j) + w2 (mu_{j-2} - mu_{j+1})) / h and the
// node adjoint Gbar_i = w1 (mu_{i-1} - mu_{i+1}) / h. One thread per face (both
// directions in one launch) recomputes the face forward in registers and runs
// it backwards, writing its 6 x 4 contributions to a per-face buffer; a gather
// kernel sums each cell's twelve face contributions and its two node
// contributions (no atomics: the result is deterministic) and applies the
// stage-adjoint combination the caller asks for.
#include "adjoint.h"
#include "adjoint_math.h"

namespace cfd {
namespace adj {
namespace {

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// one stencil position's contribution from the x face and the y face
__device__ __forceinline__ double P_sum(const double *__restrict__ Px, const double *__restrict__ Py, long long off,
                                        long long fx, long long fy)
{
    return Px[off + fx] + Py[off + fy];
}

// 128-thread CTAs per SM of the two face-adjoint halves. The first runs 4
// (128 registers, ~0.3 KB of spills per thread: faster than 3 without
// spills, and than 5); the second needs the full 255 (3 per SM, at 168
// registers, spills 0.7-2.3 KB per thread and is 15% slower on the reverse)
#ifndef ADJ_STATES_MINB
#define ADJ_STATES_MINB 4
#endif
#ifndef ADJ_CHARS_MINB
#define ADJ_CHARS_MINB 2
#endif

// The stencil of face t of direction AX (face t lies before cell t along AX)
// and the face's adjoint weight Fb (the MND6 transpose applied to mu).
template <int AX>
struct FaceAt {
    long long ncell, t, cells[6];
    __device__ FaceAt(long long t_, int nx, int ny) : ncell((long long)nx * ny), t(t_)
    {
        const int nd = (AX == 0) ? nx : ny;
        const int x = (int)(t % nx), y = (int)(t / nx);
        const int f = (AX == 0) ? x : y;
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const int pos = wrap(f - 3 + m, nd);
            cells[m] = (AX == 0) ? (long long)y * nx + pos : (long long)pos * nx + x;
        }
    }
    __device__ void stencil(const double *__restrict__ u, double (&U)[6][4]) const
    {
#pragma unroll
        for (int m = 0; m < 6; m++)
#pragma unroll
            for (int v = 0; v < 4; v++) U[m][v] = u[v * ncell + cells[m]];
    }
    __device__ void weight(const double *__restrict__ mu, double inv_h, double (&Fb)[4]) const
    {
        // cells f-2, f-1, f, f+1 are stencil positions 1..4
#pragma unroll
        for (int v = 0; v < 4; v++)
            Fb[v] = (kW0 * (mu[v * ncell + cells[2]] - mu[v * ncell + cells[3]]) +
                     kW2 * (mu[v * ncell + cells[1]] - mu[v * ncell + cells[4]])) * inv_h;
    }
};

// First half of the face adjoint (forward to the face states, Roe flux
// adjoint): its FaceStates go to slots 0..23 of the face's P entries, the
// eight 3-bit TENO flags to fl[t].
template <int AX, int FAM>
__device__ __forceinline__ void face_states_at(long long t, const double *__restrict__ u,
                                               const double *__restrict__ mu, double *__restrict__ P,
                                               unsigned *__restrict__ fl, int nx, int ny, double inv_h, double ct)
{
    const FaceAt<AX> fa(t, nx, ny);
    double U[6][4], Fb[4];
    fa.stencil(u, U);
    fa.weight(mu, inv_h, Fb);
    FaceStates fs;
    face_vjp_states<AX>(U, Fb, fs, FAM, ct);
    const long long n = fa.ncell;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        P[(0 + k) * n + t] = fs.QL[k];
        P[(4 + k) * n + t] = fs.QR[k];
        P[(8 + k) * n + t] = fs.clb[k];
        P[(12 + k) * n + t] = fs.crb[k];
        P[(16 + k) * n + t] = fs.P2b[k];
        P[(20 + k) * n + t] = fs.P3b[k];
    }
    if (FAM != ADJ_WCNS5) {
        unsigned w = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) w |= (fs.flL[k] << (3 * k)) | (fs.flR[k] << (12 + 3 * k));
        fl[t] = w;
    }
}

// Second half (characteristic projections, interpolations and eigensystem
// backwards): reads the face's FaceStates from its P entries and overwrites
// them with P[(m * 4 + v) * ncell + t] = d(mu . R)/dU of stencil cell m.
template <int AX, int FAM>
__device__ __forceinline__ void face_chars_at(long long t, const double *__restrict__ u, double *P,
                                              const unsigned *__restrict__ fl, int nx, int ny)
{
    const FaceAt<AX> fa(t, nx, ny);
    const long long n = fa.ncell;
    FaceStates fs;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        fs.QL[k] = P[(0 + k) * n + t];
        fs.QR[k] = P[(4 + k) * n + t];
        fs.clb[k] = P[(8 + k) * n + t];
        fs.crb[k] = P[(12 + k) * n + t];
        fs.P2b[k] = P[(16 + k) * n + t];
        fs.P3b[k] = P[(20 + k) * n + t];
    }
    const unsigned w = (FAM != ADJ_WCNS5) ? fl[t] : 0u;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        fs.flL[k] = (w >> (3 * k)) & 7u;
        fs.flR[k] = (w >> (12 + 3 * k)) & 7u;
    }
    double U[6][4], Ub[6][4];
    fa.stencil(u, U);
#pragma unroll
    for (int m = 0; m < 6; m++)
#pragma unroll
        for (int v = 0; v < 4; v++) Ub[m][v] = 0.0;
    face_vjp_chars<AX>(U, fs, Ub, FAM);
#pragma unroll
    for (int m = 0; m < 6; m++)
#pragma unroll
        for (int v = 0; v < 4; v++) P[(m * 4 + v) * n + t] = Ub[m][v];
}

// one thread per face, the faces of both directions in one launch (items
// 0 .. ncell-1 along x into Px, ncell .. 2 ncell-1 along y into Py); the two
// halves of the face adjoint are two launches so that each fits in fewer
// registers and runs more warps per SM
template <int FAM>
__global__ void __launch_bounds__(128, ADJ_STATES_MINB)
    face_states_kernel(const double *__restrict__ u, const double *__restrict__ mu, double *__restrict__ Px,
                       double *__restrict__ Py, unsigned *__restrict__ fl, int nx, int ny, double inv_hx,
                       double inv_hy, double ct)
{
    const long long ncell = (long long)nx * ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 2 * ncell;
         t += (long long)gridDim.x * blockDim.x) {
        if (t < ncell) face_states_at<0, FAM>(t, u, mu, Px, fl, nx, ny, inv_hx, ct);
        else face_states_at<1, FAM>(t - ncell, u, mu, Py, fl + ncell, nx, ny, inv_hy, ct);
    }
}

template <int FAM>
__global__ void __launch_bounds__(128, ADJ_CHARS_MINB)
    face_chars_kernel(const double *__restrict__ u, double *Px, double *Py, const unsigned *__restrict__ fl, int nx,
                      int ny)
{
    const long long ncell = (long long)nx * ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 2 * ncell;
         t += (long long)gridDim.x * blockDim.x) {
        if (t < ncell) face_chars_at<0, FAM>(t, u, Px, fl, nx, ny);
        else face_chars_at<1, FAM>(t - ncell, u, Py, fl + ncell, nx, ny);
    }
}

// one thread per cell: the six faces whose stencil holds it and its node flux,
// in both directions; their sum g goes to o (VjpOut)
__global__ void gather_kernel(const double *__restrict__ u, const double *__restrict__ mu,
                              const double *__restrict__ Px, const double *__restrict__ Py, const VjpOut o,
                              int nx, int ny, double inv_hx, double inv_hy)
{
    const long long ncell = (long long)nx * ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncell;
         t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % nx), y = (int)(t / nx);
        auto cx = [&](int pos) -> long long { return (long long)y * nx + wrap(pos, nx); };
        auto cy = [&](int pos) -> long long { return (long long)wrap(pos, ny) * nx + x; };
        double acc[4] = {0, 0, 0, 0};
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const long long fx = cx(x + 3 - m), fy = cy(y + 3 - m);  // faces whose stencil position m is this cell
#pragma unroll
            for (int v = 0; v < 4; v++) acc[v] += P_sum(Px, Py, (m * 4 + v) * ncell, fx, fy);
        }
        double U[4], Gx[4], Gy[4];
        const long long xm = cx(x - 1), xp = cx(x + 1), ym = cy(y - 1), yp = cy(y + 1);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            U[v] = u[v * ncell + t];
            Gx[v] = kW1 * (mu[v * ncell + xm] - mu[v * ncell + xp]) * inv_hx;
            Gy[v] = kW1 * (mu[v * ncell + ym] - mu[v * ncell + yp]) * inv_hy;
        }
        node_vjp<0>(U, Gx, acc);
        node_vjp<1>(U, Gy, acc);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const long long i = v * ncell + t;
            double r = o.b * acc[v];
            if (o.x) r = o.a * o.x[i] + r;
            if (o.z) r += o.e * o.z[i];
            o.out[i] = r;
            if (o.out2) o.out2[i] = o.c * o.out2[i] + o.d * o.y[i];
        }
    }
}

unsigned grid_for(long long n, int threads)
{
    long long g = (n + threads - 1) / threads;
    if (g > 148LL * 32) g = 148LL * 32;
    return (unsigned)(g < 1 ? 1 : g);
}

} // namespace

cudaError_t launch_rhs_vjp(int fam, double ct, const double *u, const double *mu, const VjpOut &o, double *P,
                           int nx, int ny, double hx, double hy, cudaStream_t st)
{
    const long long ncell = (long long)nx * ny;
    double *Px = P, *Py = P + 24 * ncell;
    unsigned *fl = reinterpret_cast<unsigned *>(P + 48 * ncell);
    const double ihx = 1.0 / hx, ihy = 1.0 / hy;
    const unsigned gf = grid_for(2 * ncell, 128);
    switch (fam) {
    case ADJ_WCNS5:
        face_states_kernel<ADJ_WCNS5><<<gf, 128, 0, st>>>(u, mu, Px, Py, fl, nx, ny, ihx, ihy, ct);
        face_chars_kernel<ADJ_WCNS5><<<gf, 128, 0, st>>>(u, Px, Py, fl, nx, ny);
        break;
    case ADJ_TENOZ:
        face_states_kernel<ADJ_TENOZ><<<gf, 128, 0, st>>>(u, mu, Px, Py, fl, nx, ny, ihx, ihy, ct);
        face_chars_kernel<ADJ_TENOZ><<<gf, 128, 0, st>>>(u, Px, Py, fl, nx, ny);
        break;
    case ADJ_TENOCONG:
        face_states_kernel<ADJ_TENOCONG><<<gf, 128, 0, st>>>(u, mu, Px, Py, fl, nx, ny, ihx, ihy, ct);
        face_chars_kernel<ADJ_TENOCONG><<<gf, 128, 0, st>>>(u, Px, Py, fl, nx, ny);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    gather_kernel<<<grid_for(ncell, 256), 256, 0, st>>>(u, mu, Px, Py, o, nx, ny, ihx, ihy);
    return cudaGetLastError();
}

} // namespace adj
} // namespace cfd
