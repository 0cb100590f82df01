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
// contributions (no atomics: the result is deterministic).
#include "adjoint.h"
#include "adjoint_math.h"

namespace cfd {
namespace adj {
namespace {

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// a read-only global load the compiler neither merges with an earlier load of
// the same address nor moves
__device__ __forceinline__ double ld_stream(const double *p)
{
    double x;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(x) : "l"(p));
    return x;
}

// one stencil position's contribution from the x face and the y face
__device__ __forceinline__ double P_sum(const double *__restrict__ Px, const double *__restrict__ Py, long long off,
                                        long long fx, long long fy)
{
    return Px[off + fx] + Py[off + fy];
}

// Face t of direction AX: P[(m * 4 + v) * ncell + t] = d(mu . R)/dU of stencil
// cell m (face t lies before cell t along AX).
template <int AX, int FAM>
__device__ __forceinline__ void face_vjp_at(long long t, const double *__restrict__ u, const double *__restrict__ mu,
                                            double *__restrict__ P, int nx, int ny, double inv_h, double ct)
{
    const long long ncell = (long long)nx * ny;
    const int nd = (AX == 0) ? nx : ny;
    const int x = (int)(t % nx), y = (int)(t / nx);
    const int f = (AX == 0) ? x : y;
    auto cell = [&](int pos) -> long long {
        pos = wrap(pos, nd);
        return (AX == 0) ? (long long)y * nx + pos : (long long)pos * nx + x;
    };
    // the stencil is read twice, once per half of the face adjoint: the
    // volatile loads keep the compiler from holding the first copy in
    // registers across the Roe flux's adjoint (where it would spill)
    auto load_stencil = [&](double (&U)[6][4]) {
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const long long cm = cell(f - 3 + m);
#pragma unroll
            for (int v = 0; v < 4; v++) U[m][v] = ld_stream(u + v * ncell + cm);
        }
    };
    FaceStates fs;
    {
        double U[6][4], Fb[4];
        load_stencil(U);
        const long long cm2 = cell(f - 2), cm1 = cell(f - 1), c0 = cell(f), cp1 = cell(f + 1);
#pragma unroll
        for (int v = 0; v < 4; v++)
            Fb[v] = (kW0 * (mu[v * ncell + cm1] - mu[v * ncell + c0]) +
                     kW2 * (mu[v * ncell + cm2] - mu[v * ncell + cp1])) * inv_h;
        face_vjp_states<AX>(U, Fb, fs, FAM, ct);
    }
    double U[6][4], Ub[6][4];
    load_stencil(U);
#pragma unroll
    for (int m = 0; m < 6; m++)
#pragma unroll
        for (int v = 0; v < 4; v++) Ub[m][v] = 0.0;
    face_vjp_chars<AX>(U, fs, Ub, FAM);
#pragma unroll
    for (int m = 0; m < 6; m++)
#pragma unroll
        for (int v = 0; v < 4; v++) P[(m * 4 + v) * ncell + t] = Ub[m][v];
}

// one thread per face, the faces of both directions in one launch (items
// 0 .. ncell-1 along x into Px, ncell .. 2 ncell-1 along y into Py): twice the
// work per launch keeps the register-heavy kernel's last wave short
template <int FAM>
__global__ void face_vjp_kernel(const double *__restrict__ u, const double *__restrict__ mu, double *__restrict__ Px,
                                double *__restrict__ Py, int nx, int ny, double inv_hx, double inv_hy, double ct)
{
    const long long ncell = (long long)nx * ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 2 * ncell;
         t += (long long)gridDim.x * blockDim.x) {
        if (t < ncell) face_vjp_at<0, FAM>(t, u, mu, Px, nx, ny, inv_hx, ct);
        else face_vjp_at<1, FAM>(t - ncell, u, mu, Py, nx, ny, inv_hy, ct);
    }
}

// one thread per cell: the six faces whose stencil holds it and its node flux,
// in both directions; lam = the sum
__global__ void gather_kernel(const double *__restrict__ u, const double *__restrict__ mu,
                              const double *__restrict__ Px, const double *__restrict__ Py, double *__restrict__ lam,
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
        for (int v = 0; v < 4; v++) lam[v * ncell + t] = acc[v];
    }
}

__global__ void axpby_kernel(double a, const double *__restrict__ x, double b, double *__restrict__ y, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = a * x[i] + b * y[i];
}

unsigned grid_for(long long n, int threads)
{
    long long g = (n + threads - 1) / threads;
    if (g > 148LL * 32) g = 148LL * 32;
    return (unsigned)(g < 1 ? 1 : g);
}

} // namespace

cudaError_t launch_rhs_vjp(int fam, double ct, const double *u, const double *mu, double *lam, double *P, int nx,
                           int ny, double hx, double hy, cudaStream_t st)
{
    const long long ncell = (long long)nx * ny;
    double *Px = P, *Py = P + 24 * ncell;
    const double ihx = 1.0 / hx, ihy = 1.0 / hy;
    const unsigned gf = grid_for(2 * ncell, 128);
    if (fam == ADJ_WCNS5)
        face_vjp_kernel<ADJ_WCNS5><<<gf, 128, 0, st>>>(u, mu, Px, Py, nx, ny, ihx, ihy, ct);
    else if (fam == ADJ_TENOZ)
        face_vjp_kernel<ADJ_TENOZ><<<gf, 128, 0, st>>>(u, mu, Px, Py, nx, ny, ihx, ihy, ct);
    else if (fam == ADJ_TENOCONG)
        face_vjp_kernel<ADJ_TENOCONG><<<gf, 128, 0, st>>>(u, mu, Px, Py, nx, ny, ihx, ihy, ct);
    else
        return cudaErrorInvalidValue;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    gather_kernel<<<grid_for(ncell, 256), 256, 0, st>>>(u, mu, Px, Py, lam, nx, ny, ihx, ihy);
    return cudaGetLastError();
}

cudaError_t launch_axpby(double a, const double *x, double b, double *y, long long n, cudaStream_t st)
{
    axpby_kernel<<<grid_for(n, 256), 256, 0, st>>>(a, x, b, y, n);
    return cudaGetLastError();
}

} // namespace adj
} // namespace cfd
