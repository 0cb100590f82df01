// Parameter blocks shared by the sweep kernels and the host launcher.
#pragma once
#include <cuda_runtime.h>

namespace cfd {

// Tile shapes of the sweeps: cells per chunk (S) x lines per CTA (W). CTAs of
// 128 threads run three or four per SM (barriers across 4 warps instead of 8):
// every 2D/3D sweep takes them; the 32-line shapes (256 threads) remain for
// the batched kernel and the TRAD6 difference.
#ifndef CFD_XS
#define CFD_XS 32
#endif
#ifndef CFD_XW
#define CFD_XW 4
#endif
#ifndef CFD_YS
#define CFD_YS 8
#endif
#ifndef CFD_YW
#define CFD_YW 32
#endif
constexpr int kXS = CFD_XS, kXW = CFD_XW;  // along x (2D mixed, TRAD6, batched default)
constexpr int kXSn = 16, kXWn = 8;          // along x: 3D, and 2D FP64 (single grid)
constexpr int kYS = CFD_YS, kYW = CFD_YW;  // along y and z
#ifndef CFD_YSM
#define CFD_YSM 8
#endif
#ifndef CFD_YWM
#define CFD_YWM 16
#endif
constexpr int kYSm = CFD_YSM, kYWm = CFD_YWM;  // along y, mixed form (single grid)
#ifndef CFD_FP64_3D_YZ16
#define CFD_FP64_3D_YZ16 1  // the FP64 3D y/z sweeps take the kYSm x kYWm shape too (0: kYS x kYW)
#endif
#ifndef CFD_FP64_2D_Y16
#define CFD_FP64_2D_Y16 1  // the FP64 2D y sweep takes the kYSm x kYWm shape too (0: kYS x kYW)
#endif
#ifndef CFD_MIXED_Z16
#define CFD_MIXED_Z16 1  // the mixed form's z sweep takes the kYSm x kYWm shape too (0: kYS x kYW)
#endif
constexpr int k1S = 128, k1W = 1;          // 1D
// Alternative shapes of the batched 2D/3D FP64 sweeps, picked per direction by
// the batch autotuner: 32 threads per x line (8 lines per CTA), 8 threads per
// y/z line (16 lines per CTA, the single-grid FP64 shape).
constexpr int kXS2 = 32, kXW2 = 8;
constexpr int kYS2 = 8, kYW2 = 16;


// BndType values (zone_FD/src/include/macro.hpp:33-34) plus the 3D mirror.
enum : int {
    BND_TYPENULL = 0,
    BND_PERIODIC1D = 1,
    BND_SYMMETRY1D = 2,
    BND_DIRICLET = 3,
    BND_SUPERSONICOUTLET = 7,
    BND_DOUBLEMACHUP = 8,
    BND_SYMMETRYX = 10,
    BND_SYMMETRYY = 11,
    BND_SYMMETRYZ = 12,
    BND_HALO = 101,      // ghost cells from a neighbour's rows (slab decomposition): i0 = line, offset = side
};

// One line end's ghost wiring, the device image of a OneDBnd
// (zone_FD/src/include/oneDBnd.hpp:10-33): source cell i0 and stride offset
// for the copying types, a slot in the static ghost-value table for the
// others, and the coordinates DoubleMachUp evaluates its exact state at.
struct BcLine {
    long long i0;
    int offset;
    int type;
    int slot;      // -1: no static data (zeros)
    int pad;
    double coor_x; // DoubleMachUp: x of the line's edge cell centre
    double dh_y;   // DoubleMachUp: edge cell centre minus its inner neighbour, y
};

// DiffMethod values (zone_FD/src/include/macro.hpp:82) the sweeps implement;
// any other value of SweepParams::diff runs MND6.
enum : int { DIFF_TRAD6 = 1, DIFF_MND6 = 3 };

enum SweepMode : int { MODE_WRITE = 0, MODE_RK = 2 };
enum ErrBits : unsigned { ERR_NONFINITE = 1u, ERR_NEGATIVE = 2u, ERR_TIMEOUT = 4u };

// Device-resident state of the time loop of BlockSolver::stepsLoopCFL
// (blockSolver.cpp:170-235), advanced by single-thread control kernels so that
// whole steps can be captured in CUDA graphs without host round trips.
struct StepCtl {
    double t, outputT, outputDt, cfl, dt;
    double bdt[4];   // per stage: dt, 0.25*dt, (2/3)*dt (index = stage)
    double tst[4];   // stage times t, t+dt, (t+dt)-dt/2
    int step, endStep, k, maxSteps, done, pad;
};

struct SweepParams {
    const double *u;    // current state U_k, planar SoA u[v * ncell + cell]
    const double *u0;   // RK base state U_0
    double *rhs;        // running right-hand side (SoA)
    double *u_out;      // RK stage output (SoA); never aliases u
    long long ncell;
    int n[3];
    long long stride[3];
    double h;           // spacing used by the difference along this axis (Info::geth)
    double hdir[3];     // spacings for the wave-speed reduction
    int mode;           // MODE_WRITE: rhs = prev + D ; MODE_RK: stage combination
    int first;          // 1: this is the first sweep of the stage (prev = 0)
    int rk_stage;       // 1, 2, 3
    double rkA, rkBdt, rkC;  // U_out = (A U0 - Bdt R) + C U_k   (stage 1: U0 - dt R)
    int want_reduce;    // 1: max |R_rho| and per-direction max wave speed of U_out
    unsigned long long *red;  // [0] max |R_rho| bits, [1..3] wave-speed maxima bits
    unsigned *err;      // ErrBits
    const BcLine *bc_lo;  // per line (index a + n[T0] * b), low end
    const BcLine *bc_hi;  // per line, high end
    const double *bc_vals; // static ghost prim values [slot][ghosts per side][NV]
    double t;           // stage time (ignored when ctl is set)
    const StepCtl *ctl; // device-resident step control (null: use rkBdt/t)
    double dm_u, dm_v;  // DoubleMachUp post-shock velocity, 8.25 cos(pi/6) and -8.25 sin(pi/6) from the host libm
    double icst;        // interpolator constant (TENO cutoff)
    double icst_k;      // TENO-Z early keep-all bound (teno_kappa(icst)); 0 disables it
    int seg_len;        // cells per CTA segment along the sweep
    int prec;           // 0: FP64 reconstruction, 1: mixed FP32/FP64 (fast flavour only)
    int gravity;        // 1: add the gravity source of the stage's input state (last direction only)
    const double *halo_lo, *halo_hi;  // BND_HALO ghosts: [var][4 rows, ascending][line]
    long long halo_nl;                // lines per halo row
    int diff;                         // DIFF_TRAD6: ExplicitDif6 with 5 ghosts; else MND6 with 4
    int posl;                         // 1: the 1D positivity limiter on 2D/3D face states (cfd_config.positivity)
    // Partial sweeps (cfd_step_host): part_lo < part_hi restricts the launch
    // to the lines and segments covering indices [part_lo, part_hi) of the
    // grid's last dimension (for a sweep along it, whole segments, with
    // seg_outer = 1 so that they are a contiguous tile range). tile0: first
    // tile of the launch (set by the launcher).
    int part_lo, part_hi;
    int seg_outer;
    long long tile0;
};

// One batched sweep launch: the parameter blocks of every case (device array)
// and the prefix sums of their tile counts (ncases + 1 entries, device array).
struct BatchSweep {
    const SweepParams *cases;
    const long long *tile_start;
    int ncases;
    long long total_tiles;
    int num_sms;
    int prec;
    int shape;      // 0: default tile shape, 1: the alternative (kXS2 x kXW2 / kYS2 x kYW2; 2D/3D FP64 only)
    int one_cta;    // 1: one persistent CTA per SM, 0: as many as fit
};

// Block-wide max of non-negative doubles followed by one atomicMax per value.
// NaN inputs are ignored (fmax), like the reference's comparisons that never
// let a NaN replace the running maximum.
template <int NT, int NRED>
__device__ __forceinline__ void block_max_reduce(double v0, const double *v123, unsigned long long *out)
{
    __shared__ double red_s[NRED][NT / 32];
    double v[NRED];
    v[0] = v0;
    for (int k = 1; k < NRED; k++) v[k] = v123[k - 1];
    for (int k = 0; k < NRED; k++) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        v[k] = x;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < NRED; k++) red_s[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x < NRED) {
        double x = 0.0;
        for (int w = 0; w < NT / 32; w++) x = fmax(x, red_s[threadIdx.x][w]);
        if (x > 0.0) atomicMax(out + threadIdx.x, (unsigned long long)__double_as_longlong(x));
    }
}

} // namespace cfd
