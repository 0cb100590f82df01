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

// Where a product g = (dR/dU)^T mu goes, per entry i (the combinations of the
// SSP-RK3 stage adjoints, applied as the product is formed):
//   out[i] = a * x[i] + b * g[i] + e * z[i]     (x, z may be null: term absent)
//   out2[i] = c * out2[i] + d * y[i]            (when out2 is not null)
// out may be x or z. None of out, out2 may be mu: mu is read at neighbours.
struct VjpOut {
    double *out;
    const double *x;
    double a, b;
    const double *z;
    double e;
    double *out2;
    const double *y;
    double c, d;
};

// (dR/dU)^T mu into o, all arrays planar SoA [4][nx*ny]. fam: interpolation
// family (0 WCNS5, 2 TENO-Z, 3 TENO-Cong) with constant ct; hx, hy the
// spacings of the x and y differences. P is scratch of 49 * nx * ny doubles
// (per-face contributions of both directions, then one 32-bit word of TENO
// flags per face).
cudaError_t launch_rhs_vjp(int fam, double ct, const double *u, const double *mu, const VjpOut &o, double *P,
                           int nx, int ny, double hx, double hy, cudaStream_t st);

} // namespace adj
} // namespace cfd
