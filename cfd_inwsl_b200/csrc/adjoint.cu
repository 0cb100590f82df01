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
// node adjoint Gbar_i = w1 (mu_{i-1} - mu_{i+1}) / h. One thread per face
// recomputes the face forward in registers and runs it backwards, writing its
// 6 x 4 contributions to a per-face buffer; a gather kernel sums each cell's
// six face contributions and its node contribution (no atomics: the result is
// deterministic).
#include "adjoint.h"
#include "adjoint_math.h"

namespace cfd {
namespace adj {
namespace {

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// one thread per face: P[(m * 4 + v) * ncell + cell(face)] = d(mu . R)/dU of stencil cell m
template <int AX, int FAM>
__global__ void face_vjp_kernel(const double *__restrict__ u, const double *__restrict__ mu, double *__restrict__ P,
                                int nx, int ny, double inv_h, double ct)
{
    const long long ncell = (long long)nx * ny;
    const int nd = (AX == 0) ? nx : ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncell;
         t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % nx), y = (int)(t / nx);
        const int f = (AX == 0) ? x : y;
        auto cell = [&](int pos) -> long long {
            pos = wrap(pos, nd);
            return (AX == 0) ? (long long)y * nx + pos : (long long)pos * nx + x;
        };
        double U[6][4], Ub[6][4];
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const long long cm = cell(f - 3 + m);
#pragma unroll
            for (int v = 0; v < 4; v++) {
                U[m][v] = u[v * ncell + cm];
                Ub[m][v] = 0.0;
            }
        }
        double Fb[4];
        const long long cm2 = cell(f - 2), cm1 = cell(f - 1), c0 = cell(f), cp1 = cell(f + 1);
#pragma unroll
        for (int v = 0; v < 4; v++)
            Fb[v] = (kW0 * (mu[v * ncell + cm1] - mu[v * ncell + c0]) +
                     kW2 * (mu[v * ncell + cm2] - mu[v * ncell + cp1])) * inv_h;
        face_vjp<AX>(U, Fb, Ub, FAM, ct);
#pragma unroll
        for (int m = 0; m < 6; m++)
#pragma unroll
            for (int v = 0; v < 4; v++) P[(m * 4 + v) * ncell + t] = Ub[m][v];
    }
}

// one thread per cell: the six faces whose stencil holds it, and its node flux
template <int AX>
__global__ void gather_kernel(const double *__restrict__ u, const double *__restrict__ mu,
                              const double *__restrict__ P, double *__restrict__ lam, int nx, int ny, double inv_h,
                              int accumulate)
{
    const long long ncell = (long long)nx * ny;
    const int nd = (AX == 0) ? nx : ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncell;
         t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % nx), y = (int)(t / nx);
        const int i = (AX == 0) ? x : y;
        auto cell = [&](int pos) -> long long {
            pos = wrap(pos, nd);
            return (AX == 0) ? (long long)y * nx + pos : (long long)pos * nx + x;
        };
        double acc[4] = {0, 0, 0, 0};
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const long long cf = cell(i + 3 - m);  // face whose stencil position m is cell i
#pragma unroll
            for (int v = 0; v < 4; v++) acc[v] += P[(m * 4 + v) * ncell + cf];
        }
        const long long cm1 = cell(i - 1), cp1 = cell(i + 1);
        double U[4], Gb[4];
#pragma unroll
        for (int v = 0; v < 4; v++) {
            U[v] = u[v * ncell + t];
            Gb[v] = kW1 * (mu[v * ncell + cm1] - mu[v * ncell + cp1]) * inv_h;
        }
        node_vjp<AX>(U, Gb, acc);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            if (accumulate) lam[v * ncell + t] += acc[v];
            else lam[v * ncell + t] = acc[v];
        }
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

template <int AX>
cudaError_t launch_faces(int fam, double ct, const double *u, const double *mu, double *P, int nx, int ny,
                         double inv_h, cudaStream_t st)
{
    const long long ncell = (long long)nx * ny;
    if (fam == ADJ_WCNS5)
        face_vjp_kernel<AX, ADJ_WCNS5><<<grid_for(ncell, 128), 128, 0, st>>>(u, mu, P, nx, ny, inv_h, ct);
    else if (fam == ADJ_TENOZ)
        face_vjp_kernel<AX, ADJ_TENOZ><<<grid_for(ncell, 128), 128, 0, st>>>(u, mu, P, nx, ny, inv_h, ct);
    else if (fam == ADJ_TENOCONG)
        face_vjp_kernel<AX, ADJ_TENOCONG><<<grid_for(ncell, 128), 128, 0, st>>>(u, mu, P, nx, ny, inv_h, ct);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_sweep_vjp(int axis, int fam, double ct, const double *u, const double *mu, double *lam, double *P,
                             int nx, int ny, double h, bool accumulate, cudaStream_t st)
{
    const long long ncell = (long long)nx * ny;
    const double inv_h = 1.0 / h;
    cudaError_t e = axis == 0 ? launch_faces<0>(fam, ct, u, mu, P, nx, ny, inv_h, st)
                              : launch_faces<1>(fam, ct, u, mu, P, nx, ny, inv_h, st);
    if (e != cudaSuccess) return e;
    if (axis == 0)
        gather_kernel<0><<<grid_for(ncell, 256), 256, 0, st>>>(u, mu, P, lam, nx, ny, inv_h, accumulate ? 1 : 0);
    else
        gather_kernel<1><<<grid_for(ncell, 256), 256, 0, st>>>(u, mu, P, lam, nx, ny, inv_h, accumulate ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_axpby(double a, const double *x, double b, double *y, long long n, cudaStream_t st)
{
    axpby_kernel<<<grid_for(n, 256), 256, 0, st>>>(a, x, b, y, n);
    return cudaGetLastError();
}

} // namespace adj
} // namespace cfd
