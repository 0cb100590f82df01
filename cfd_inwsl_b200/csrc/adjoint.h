// Launchers of the discrete-adjoint kernels (adjoint.cu, fast flavour).
//
// The adjoint differentiates one RHS evaluation of the 2D Euler path with
// WCNS5 (weno5_JSchen) or TENO (cut-off frozen) characteristic reconstruction, the Roe flux
// (roeFlux2DSym) and the MND6 difference on a grid periodic in both
// directions: lam = (dR/dU)^T mu, R the RHS of SpDistributor::rhsSolve.
#pragma once
#include <cuda_runtime.h>

namespace cfd {
namespace adj {

// lam = (dR/dU)^T mu, all arrays planar SoA [4][nx*ny]. fam: interpolation
// family (0 WCNS5, 2 TENO-Z, 3 TENO-Cong) with constant ct; hx, hy the
// spacings of the x and y differences. P is scratch of 49 * nx * ny doubles
// (per-face contributions of both directions, then one 32-bit word of TENO
// flags per face).
cudaError_t launch_rhs_vjp(int fam, double ct, const double *u, const double *mu, double *lam, double *P, int nx,
                           int ny, double hx, double hy, cudaStream_t st);

// y = a * x + b * y over n doubles
cudaError_t launch_axpby(double a, const double *x, double b, double *y, long long n, cudaStream_t st);

} // namespace adj
} // namespace cfd
