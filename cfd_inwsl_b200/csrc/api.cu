// C ABI of the zone_FD RHS + SSP-RK3 library (include/cfdgpu.h).
//
// Host orchestration of the sweep kernels: boundary wiring tables, state
// buffers, stage sequencing of BlockSolver::RK3_SSP (blockSolver.cpp:43-87),
// the CFL step of getTimeIntervalExplicit (blockSolver.cpp:318-349) and the
// device-resident loop of stepsLoopCFL (blockSolver.cpp:170-235).
//
// This translation unit is compiled with --fmad=false: its small kernels
// (layout transposes, wave-speed reduction, step control) reproduce the
// reference's arithmetic bit for bit.
#include "cfdgpu.h"
#include "euler_math.cuh"
#include "mixed.cuh"
#include "sweep_dispatch.h"
#include "adjoint.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using cfd::BcLine;
using cfd::SweepParams;

namespace cfd {
int default_seg_len_for(const cfd_config *cfg, int fam, bool strict, int d);
bool config_bc_ok(const cfd_config *cfg, const char **why);
}

namespace {

constexpr int kGhost = 4;

// ------------------------------------------------------------------ kernels

// The transposes and the wave-speed reduction work on the cells [c0, c1).
template <int NV>
__global__ void aos_to_soa_kernel(const double *__restrict__ aos, double *__restrict__ soa, long long ncell,
                                  long long c0, long long c1)
{
    for (long long c = c0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; c < c1; c += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int v = 0; v < NV; v++) soa[v * ncell + c] = aos[c * NV + v];
    }
}

template <int NV>
__global__ void soa_to_aos_kernel(const double *__restrict__ soa, double *__restrict__ aos, long long ncell, int to_prim,
                                  long long c0, long long c1)
{
    for (long long c = c0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; c < c1; c += (long long)gridDim.x * blockDim.x) {
        double x[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) x[v] = soa[v * ncell + c];
        if (to_prim) {
            double p[NV];
            cfd::cons_to_prim<NV>(x, p);
#pragma unroll
            for (int v = 0; v < NV; v++) x[v] = p[v];
        }
#pragma unroll
        for (int v = 0; v < NV; v++) aos[c * NV + v] = x[v];
    }
}

// Per-direction max of (sqrt(gamma p / rho) + |u_d|) / h_d over the state,
// as getTimeIntervalExplicit's OpenMP max loops (blockSolver.cpp:327-338).
template <int NV>
__global__ void __launch_bounds__(256) wave_speed_kernel(const double *__restrict__ u, long long ncell, double h0,
                                                          double h1, double h2, unsigned long long *red, long long c0,
                                                          long long c1)
{
    double lam[3] = {0.0, 0.0, 0.0};
    const double hd[3] = {h0, h1, h2};
    for (long long c = c0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; c < c1; c += (long long)gridDim.x * blockDim.x) {
        double x[NV], p[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) x[v] = u[v * ncell + c];
        cfd::cons_to_prim<NV>(x, p);
        double cs = sqrt(cfd::kGamma * p[NV - 1] / p[0]);
#pragma unroll
        for (int d = 0; d < NV - 2; d++) lam[d] = fmax(lam[d], (cs + fabs(p[1 + d])) / hd[d]);
    }
    cfd::block_max_reduce<256, 4>(0.0, lam, red);
}

// Step control of stepsLoopCFL (blockSolver.cpp:176-201) on the device: the
// loop test, dt = CFL / sum_d lambda_d from the wave-speed maxima of the
// current state, clipping to the output interval, stage coefficients.
__global__ void step_begin_kernel(cfd::StepCtl *c, unsigned long long *red, int dim, double *dts)
{
    if (c->done) return;
    if (!(c->step < c->endStep && c->k < c->maxSteps)) {
        c->done = 1;
        return;
    }
    double lambda = 0;
    for (int d = 0; d < dim; d++) lambda += __longlong_as_double((long long)red[1 + d]);
    double dt = c->cfl / lambda;
    if (c->outputT + dt > c->outputDt) {
        dt = c->outputDt - c->outputT;
        c->outputT = 0.0;
        c->step++;
    } else
        c->outputT += dt;
    c->dt = dt;
    c->bdt[1] = dt;
    c->bdt[2] = 0.25 * dt;
    c->bdt[3] = 2.0 / 3.0 * dt;
    c->tst[1] = c->t;
    c->tst[2] = c->t + dt;
    c->tst[3] = c->tst[2] - dt / 2;
    if (dts) dts[c->k] = dt;
    // the wave speeds are consumed: clear the reduction words for this step's
    // third stage (only when the step runs, so a finished loop keeps them)
    for (int i = 0; i < 4; i++) red[i] = 0ULL;
}

// BlockSolver::solve's time update and the per-step log value (rhoLinf).
__global__ void step_end_kernel(cfd::StepCtl *c, const unsigned long long *red, double *linf)
{
    if (c->done) return;
    if (linf) linf[c->k] = __longlong_as_double((long long)red[0]);
    double dt = c->dt;
    c->t = (((c->t + dt) - dt / 2) - dt / 2) + dt;
    c->k++;
}

// FP64 peak probe: eight independent DFMA chains per thread over every SM,
// the denominator of the FP64 roofline (measured on the device that runs the
// sweeps instead of a datasheet figure).
__device__ double g_dfma_sink;

__global__ void dfma_probe_kernel(long long iters, double seed)
{
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = seed + threadIdx.x * 1e-9 + i * 1e-3;
    const double a = 0.999999999, b = 1e-9;
    for (long long it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = fma(x[i], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += x[i];
    if (s == -1.0) g_dfma_sink = s;  // never true: keeps the chains live
}

// Self-check of the strict flavour's shared-reciprocal division (div_rn)
// against the device's IEEE division, bit for bit, on n seeded operand pairs:
// random significands and exponents, quotients constructed next to a rounding
// midpoint (a = RN(b (q + ulp(q)/2))), physical ranges, zeros of both signs
// and tiny dividends.
__device__ unsigned long long splitmix64(unsigned long long &x)
{
    unsigned long long z = (x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__device__ double rand_double(unsigned long long &st, int emin, int emax)
{
    const unsigned long long r = splitmix64(st);
    const int e = emin + (int)(splitmix64(st) % (unsigned long long)(emax - emin + 1));
    const unsigned long long bits = ((unsigned long long)(1023 + e) << 52) | (r & ((1ULL << 52) - 1));
    return __longlong_as_double((long long)bits) * ((r >> 63) ? -1.0 : 1.0);
}

__global__ void division_check_kernel(long long n, unsigned long long seed, unsigned long long *bad)
{
    unsigned long long cnt = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long st = seed ^ ((unsigned long long)i * 0xD1B54A32D192ED03ULL);
        double a, b;
        switch (i % 4) {
        case 0:
            a = rand_double(st, -60, 60);
            b = fabs(rand_double(st, -60, 60));
            break;
        case 1: {  // the quotient next to a midpoint between two doubles
            b = fabs(rand_double(st, -20, 20));
            const double q = fabs(rand_double(st, -20, 20));
            const double half_ulp = ldexp(1.0, ilogb(q) - 53);
            a = fma(b, q, b * half_ulp);
            break;
        }
        case 2:  // densities, sound speeds, enthalpies over momenta, energies, velocities
            a = rand_double(st, -30, 12);
            b = fabs(rand_double(st, -10, 10));
            break;
        default: {  // zeros, tiny and huge dividends (IEEE fallback)
            const unsigned long long k = splitmix64(st) % 4;
            a = (k == 0) ? 0.0 : (k == 1) ? -0.0 : (k == 2) ? rand_double(st, -1010, -950) : rand_double(st, 950, 1000);
            b = fabs(rand_double(st, -5, 5));
            break;
        }
        }
        const double y = cfd::rcp_rn(b);
        const double got = cfd::div_rn(a, b, y), want = a / b;
        if (__double_as_longlong(got) != __double_as_longlong(want) || __double_as_longlong(y) != __double_as_longlong(1.0 / b))
            cnt++;
        // the grouped form: a with two more dividends over the same b (a
        // random one and, one time in four each, a signed zero or a dividend
        // outside the corrected range), either sign of b
        {
            const unsigned long long k = splitmix64(st) % 8;
            const double a2 = rand_double(st, -40, 40);
            const double a3 = (k == 0) ? 0.0 : (k == 1) ? -0.0 : (k == 2) ? rand_double(st, 962, 1000)
                                                                           : rand_double(st, -40, 40);
            const double bs = (splitmix64(st) & 1) ? -b : b, ys = cfd::rcp_rn(bs);
            const double A[3] = {a, a2, a3}, B[3] = {bs, bs, bs}, Y[3] = {ys, ys, ys};
            double Q[3];
            cfd::divs_rn<3>(A, B, Y, Q);
            for (int j = 0; j < 3; j++)
                if (__double_as_longlong(Q[j]) != __double_as_longlong(A[j] / bs)) cnt++;
        }
    }
    if (cnt) atomicAdd(bad, cnt);
}

// Pointwise test kernels.
template <int FAM>
__global__ void eval_inter5_kernel(const double *q, int n, double c, double kap, double *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = cfd::inter5<FAM>(q[5 * i], q[5 * i + 1], q[5 * i + 2], q[5 * i + 3], q[5 * i + 4], c, kap);
}

template <int NV, int AX, int FLUX>
__global__ void eval_flux_kernel(const double *lr, int n, double *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double L[NV], R[NV], f[NV];
        for (int v = 0; v < NV; v++) {
            L[v] = lr[2 * NV * i + v];
            R[v] = lr[2 * NV * i + NV + v];
        }
        cfd::riemann<NV, AX, FLUX>(L, R, f);
        for (int v = 0; v < NV; v++) out[NV * i + v] = f[v];
    }
}

// Scalar accuracy test: face values by the left-biased five-point interpolation
// of q (the upwind face flux of a unit-speed scalar), node fluxes = q, MND6
// difference: d q / d x at the n cells. q holds 4 ghost values on each side.
template <int FAM>
__global__ void accuracy_kernel(const double *q, int n, double h, double c, double *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *g = q + 4;  // g[k] = value at cell k, k in [-4, n+3]
    // face x_{k+1/2} from cells k-2 .. k+2
    auto face = [&](int k) { return cfd::inter5<FAM>(g[k - 2], g[k - 1], g[k], g[k + 1], g[k + 2], c); };
    out[i] = cfd::mnd6(g[i - 1], g[i + 1], face(i - 2), face(i - 1), face(i), face(i + 1), h, 1.0 / h);
}

// One face reconstruction per thread from six stencil prims (known-answer hook).
template <int NV, int AX, int FAM, int PREC>
__global__ void eval_face_kernel(const double *prims6, int n, double c, double kap, double *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double pr6[6][NV], cs6[6][NV];
    for (int j = 0; j < 6; j++) {
        for (int v = 0; v < NV; v++) pr6[j][v] = prims6[(i * 6 + j) * NV + v];
        cfd::prim_to_cons<NV>(pr6[j], cs6[j]);
    }
    double fl[NV], fr[NV];
    if constexpr (NV == 3) {
        cfd::reconstruct_face<NV, AX, FAM>(pr6, cs6, c, kap, fl, fr);
    } else {
        auto cs = [&](int j, int v) { return cs6[j][v]; };
        auto pr = [&](int j, int v) { return pr6[j][v]; };
        if constexpr (PREC == 1) {
            // the sweep's FP32 hi/lo split of each stencil cell's cons
            float hi[6][NV], lo[6][NV];
            for (int j = 0; j < 6; j++)
                for (int v = 0; v < NV; v++) {
                    hi[j][v] = (float)cs6[j][v];
                    lo[j][v] = (float)(cs6[j][v] - (double)hi[j][v]);
                }
            auto hl = [&](int j, int v) { return make_float2(hi[j][v], lo[j][v]); };
            cfd::reconstruct_face_mixed<NV, AX, FAM>(cs, pr, hl, c, kap, fl, fr);
        } else {
            cfd::reconstruct_face_stream<NV, AX, FAM>(cs, pr, c, kap, fl, fr);
        }
    }
    for (int v = 0; v < NV; v++) {
        out[i * 2 * NV + v] = fl[v];
        out[i * 2 * NV + NV + v] = fr[v];
    }
}

// ------------------------------------------------------------------ helpers

struct InterMap {
    int fam;
    double c;
    bool ok;
};

// InterMethod (macro.hpp:37-78) -> interpolator family, following the
// Euler branches of SolverType::initReconer (solverType.cpp:217-598).
InterMap map_inter_method(int m, int dim)
{
    switch (m) {
    case 2: return {cfd::FAM_WCNS5, 0.0, true};                 // WCNS5 -> weno5_JSchen
    case 3: return {cfd::FAM_WENOZ, 0.0, true};                 // WCNSZ5 -> weno5_Z
    case 11: return {cfd::FAM_TENOZ, 1e-5, true};               // TCNS5 -> Teno5_Z
    case 12: return {cfd::FAM_TENOZ, 1e-4, true};               // TCNS5CT4 -> Teno5_ZCT4
    case 13: return {cfd::FAM_TENOZ, 1e-7, true};               // TCNS5CT7 -> Teno5_ZCT7
    case 22: return {cfd::FAM_TENOZ, 1e-5, true};               // congTCNS5CT5 -> congTcns5_ZCT5
    case 23: return {cfd::FAM_TENOZ, 1e-10, true};              // congTCNS5CT10 -> congTcns5_ZCT10
    case 35: return {cfd::FAM_TENOZ, 1e-5, true};               // new_TCNS5 -> new_Teno5_Z
    case 8: return {cfd::FAM_TENOCONG, 0.15704178024750198, true};   // WCNS5CONGZ -> Teno5_CongZ
    case 37: return {cfd::FAM_TENOCONG, 0.15704178024750198, true};  // new_WCNS5CONGZ -> new_Teno5_CongZ
    case 9: return {cfd::FAM_TENOCONG, 0.23050581003334941, true};   // WCNS5CONGZCT4 -> Teno5_CongZCT4
    case 10:
        // WCNS5CONGZCT7: Teno5_CongZCT7 in 2D, but Teno5_CongAA in 1D (solverType.cpp:248-250).
        if (dim == 1) return {cfd::FAM_RESEARCH, (double)cfd::RV_CONGAA, true};
        return {cfd::FAM_TENOCONG, 0.072892337360747711, true};
    // the research variants (solverType.cpp:262-388, 1D; 445-576, 2D)
    case 17: return {cfd::FAM_RESEARCH, (double)cfd::RV_TCNSN, true};      // whfTCNSN
    case 18: return {cfd::FAM_RESEARCH, (double)cfd::RV_TCNSN_A, true};    // whfTCNSNA
    case 19: return {cfd::FAM_RESEARCH, (double)cfd::RV_TCNSN_AS, true};   // whfTCNSNAS
    case 20: return {cfd::FAM_RESEARCH, (double)cfd::RV_TCNSN_S, true};    // whfTCNSNS
    case 21: return {cfd::FAM_RESEARCH, (double)cfd::RV_TCNSN_LAD, true};  // whfTCNSNLAD
    case 24: return {cfd::FAM_RESEARCH, (double)cfd::RV_AI_S, true};       // whfAITCNSNS
    case 25: return {cfd::FAM_RESEARCH, (double)cfd::RV_AI_A, true};       // whfAITCNSNA
    case 26: return {cfd::FAM_RESEARCH, (double)cfd::RV_AI_AS1, true};     // whfAITCNSNAS_1
    case 27: return {cfd::FAM_RESEARCH, (double)cfd::RV_AI_AS2, true};     // whfAITCNSNAS_2
    case 28: return {cfd::FAM_RESEARCH, (double)cfd::RV_AI_LADS, true};    // whfAITCNSNLADS
    case 29: return {cfd::FAM_RESEARCH, (double)cfd::RV_AI_AZS, true};     // whfAITCNSNAZS
    case 30: return {cfd::FAM_RESEARCH, (double)cfd::RV_AI_ASF1, true};    // whfAITCNSNmyASF002_1
    case 31: return {cfd::FAM_RESEARCH, (double)cfd::RV_AI_ASF2, true};    // whfAITCNSNmyASF002_2
    case 32: return {cfd::FAM_RESEARCH, (double)cfd::RV_AI_ASFAI1, true};  // whfAITCNSNmyASF002_ai1
    case 33: return {cfd::FAM_RESEARCH, (double)cfd::RV_ZYC, true};        // whfzycTCNSNmyASF002_1
    case 34: return {cfd::FAM_RESEARCH, (double)cfd::RV_COMPARE, true};    // whfCOMPARE
    case 36: return {cfd::FAM_RESEARCH, (double)cfd::RV_NEW_A, true};      // new_WHFTCNSA
    case 38: return {cfd::FAM_RESEARCH, (double)cfd::RV_F203, true};       // new_WHFTCNSASF203_NoS
    case 39: return {cfd::FAM_RESEARCH, (double)cfd::RV_F202, true};       // new_WHFTCNSASF202_NoS
    case 15: return {cfd::FAM_MUSCL, 0.0, true};                // MUCSLIN5 -> musclIn5
    case 0: case 1: case 4: case 5: case 6: case 7: case 14: case 16:
        return {cfd::FAM_WCNS5, 0.0, true};                     // selector default: weno5_JSchen
    default:
        return {0, 0.0, false};                                 // not an InterMethod
    }
}

} // namespace

// chunks of the overlapped host step (cfd_step_host), each direction
constexpr int kHostChunks = 8;

struct cfd_handle {
    cfd_config cfg;
    int dim = 0, nv = 0;
    long long ncell = 0;
    long long stride[3] = {1, 1, 1};
    int fam = 0;
    int ng = 4;                  // ghost cells per line end (Info::nGhostCell)
    double icst = 0.0;
    double icst_k = 0.0;
    bool strict = false;
    cudaStream_t stream = nullptr;
    double *u[3] = {nullptr, nullptr, nullptr};
    int cur = 0;
    double *rhs = nullptr;
    double *stage = nullptr;  // AoS staging buffer
    unsigned long long *red = nullptr;
    unsigned *err = nullptr;
    std::vector<BcLine> bc_lo[3], bc_hi[3];
    std::vector<double> bc_vals;
    BcLine *d_bclo[3] = {nullptr, nullptr, nullptr};
    BcLine *d_bchi[3] = {nullptr, nullptr, nullptr};
    double *d_bcvals = nullptr;
    size_t d_bcvals_cap = 0;
    bool bc_dirty = true;
    int seg_len[3] = {1, 1, 1};
    bool ws_valid = false;       // red[1..3] hold the wave speeds of the current state
    double dm_u = 0.0, dm_v = 0.0;
    std::string msg;
    cudaStream_t own_stream = nullptr;   // created by cfd_create
    cfd::StepCtl *ctl = nullptr;         // device step control
    cfd::StepCtl *ctl_host = nullptr;    // pinned mirror
    double *d_dts = nullptr, *d_linf = nullptr;
    int log_cap = 0;
    // captured step graphs, by (steps per graph index: 1, 3, 12) x (start slot)
    cudaGraphExec_t graph[3][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    unsigned long long launches = 0;     // kernels this library launched
    // discrete adjoint: forward checkpoints and reverse work buffers
    std::vector<double *> adj_ckpt;      // state at steps 0, K, 2K, ... of the recorded run
    std::vector<double *> adj_stage;     // U^0, U^(1), U^(2) of each step of one segment
    double *adj_buf[4] = {nullptr, nullptr, nullptr, nullptr};  // lambda, w, w2, face scratch (24 states)
    double adj_dt = 0.0;
    int adj_nsteps = 0, adj_every = 0;
    // captured adjoint segments: K forward steps from each state slot (record)
    // and one full segment's recomputation and reverse sweep; valid for
    // (adj_graph_K, adj_graph_dt)
    cudaGraphExec_t adj_rec_graph[3] = {nullptr, nullptr, nullptr};
    // the reverse pass, per stage-buffer set: the segment's recomputation (on
    // adj_aux) and its reverse sweep (on the handle's stream)
    cudaGraphExec_t adj_recomp_graph[2] = {nullptr, nullptr};
    cudaGraphExec_t adj_back_graph[2] = {nullptr, nullptr};
    // the record pass's last segment, run keeping its stage states in
    // adj_stage (the first set of the reverse pass), so that the reverse pass
    // starts without recomputing it; adj_last_valid until a reverse pass
    // consumes them
    cudaGraphExec_t adj_last_graph = nullptr;
    bool adj_last_valid = false;
    std::vector<double *> adj_stage_b;   // the second set of stage states (overlap)
    cudaStream_t adj_aux = nullptr;      // recomputation stream of the reverse pass
    cudaEvent_t adj_ev[4] = {nullptr, nullptr, nullptr, nullptr};  // recomputed[set], reversed[set]
    // cfd_step_host: the copy stream and one event per chunk and direction
    cudaStream_t copy_st = nullptr;
    // a line end of direction d was wired by cfd_set_line_bc (its ghost cells
    // may come from any cell of the grid)
    bool line_bc_set[3] = {false, false, false};
    cudaEvent_t host_ev[2][kHostChunks] = {};
    int adj_graph_K = 0;
    double adj_graph_dt = 0.0;
    // slab decomposition: halo rows of the last direction's low / high side
    double *halo[2] = {nullptr, nullptr};
};

namespace {

void drop_graphs(cfd_handle *h);

int fail(cfd_handle *h, int code, const std::string &m)
{
    if (h) h->msg = m;
    return code;
}

int cuda_fail(cfd_handle *h, cudaError_t e, const char *what)
{
    return fail(h, CFD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CFD_CUDA(h, call)                                  \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

long long nlines(const cfd_handle *h, int d) { return h->ncell / h->cfg.n[d]; }

void transverse_axes(int d, int &t0, int &t1)
{
    t0 = (d == 0) ? 1 : 0;
    t1 = (d == 2) ? 1 : 2;
}

// Cell-centre coordinate as Initializer::initUniformBlock computes it
// (initializer.cpp:676-677): every direction starts from calZone[0].
double cell_coor(const cfd_handle *h, long long cell, int idim)
{
    long long idx[3];
    idx[0] = cell % h->cfg.n[0];
    idx[1] = (cell / h->cfg.n[0]) % h->cfg.n[1];
    idx[2] = cell / ((long long)h->cfg.n[0] * h->cfg.n[1]);
    return h->cfg.x0[0] + (idx[idim] + 0.5) * h->cfg.h[0];
}

void set_line(cfd_handle *h, int d, long long lid, int side, int type, long long i0, int offset, int slot)
{
    BcLine b;
    std::memset(&b, 0, sizeof(b));
    b.slot = slot;
    if (type == CFD_BND_PERIODIC_WRAP) {
        // true wrap: the low end copies the far end of the line and vice versa
        int t0, t1;
        transverse_axes(d, t0, t1);
        long long a = lid % h->cfg.n[t0], bb = lid / h->cfg.n[t0];
        long long base = a * h->stride[t0] + bb * h->stride[t1];
        long long last = base + (long long)(h->cfg.n[d] - 1) * h->stride[d];
        b.type = cfd::BND_PERIODIC1D;
        b.i0 = side == 0 ? last : base;
        b.offset = side == 0 ? -(int)h->stride[d] : (int)h->stride[d];
    } else {
        b.type = type;
        b.i0 = i0;
        b.offset = offset;
    }
    if (b.type == cfd::BND_DOUBLEMACHUP) {
        // OneDBnd::setCoor as wired by initDoubleMachBnds (initializer.cpp:933-941)
        b.coor_x = cell_coor(h, b.i0, 0);
        b.dh_y = cell_coor(h, b.i0, 1) - cell_coor(h, b.i0 + b.offset, 1);
    }
    (side == 0 ? h->bc_lo[d] : h->bc_hi[d])[lid] = b;
    h->bc_dirty = true;
}

// Default per-line wiring of Initializer::initBnds (initializer.cpp:743-870):
// the low end reads from the first cell with +stride (calOffset), the high end
// from the last cell with -stride (calOffsetInverse).
void wire_defaults(cfd_handle *h)
{
    for (int d = 0; d < h->dim; d++) {
        long long nl = nlines(h, d);
        h->bc_lo[d].assign(nl, BcLine{});
        h->bc_hi[d].assign(nl, BcLine{});
        int t0, t1;
        transverse_axes(d, t0, t1);
        for (long long lid = 0; lid < nl; lid++) {
            long long a = lid % h->cfg.n[t0], bb = lid / h->cfg.n[t0];
            long long base = a * h->stride[t0] + bb * h->stride[t1];
            long long last = base + (long long)(h->cfg.n[d] - 1) * h->stride[d];
            set_line(h, d, lid, 0, h->cfg.bc[d][0], base, (int)h->stride[d], -1);
            set_line(h, d, lid, 1, h->cfg.bc[d][1], last, -(int)h->stride[d], -1);
        }
    }
}

int sync_bc(cfd_handle *h)
{
    if (!h->bc_dirty) return CFD_OK;
    for (int d = 0; d < h->dim; d++) {
        size_t bytes = h->bc_lo[d].size() * sizeof(BcLine);
        CFD_CUDA(h, cudaMemcpyAsync(h->d_bclo[d], h->bc_lo[d].data(), bytes, cudaMemcpyHostToDevice, h->stream));
        CFD_CUDA(h, cudaMemcpyAsync(h->d_bchi[d], h->bc_hi[d].data(), bytes, cudaMemcpyHostToDevice, h->stream));
    }
    if (!h->bc_vals.empty()) {
        size_t bytes = h->bc_vals.size() * sizeof(double);
        if (bytes > h->d_bcvals_cap) {
            drop_graphs(h);
            if (h->d_bcvals) cudaFree(h->d_bcvals);
            h->d_bcvals = nullptr;
            CFD_CUDA(h, cudaMalloc(&h->d_bcvals, bytes));
            h->d_bcvals_cap = bytes;
        }
        CFD_CUDA(h, cudaMemcpyAsync(h->d_bcvals, h->bc_vals.data(), bytes, cudaMemcpyHostToDevice, h->stream));
    }
    // the host tables may change after this call returns
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    h->bc_dirty = false;
    return CFD_OK;
}

int grid_for(long long n)
{
    long long g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    if (g < 1) g = 1;
    return (int)g;
}

int launch_aos_to_soa(cfd_handle *h, const double *aos, double *soa, long long c0 = 0, long long c1 = -1)
{
    if (c1 < 0) c1 = h->ncell;
    if (c1 <= c0) return CFD_OK;
    int g = grid_for(c1 - c0);
    if (h->nv == 3) aos_to_soa_kernel<3><<<g, 256, 0, h->stream>>>(aos, soa, h->ncell, c0, c1);
    else if (h->nv == 4) aos_to_soa_kernel<4><<<g, 256, 0, h->stream>>>(aos, soa, h->ncell, c0, c1);
    else aos_to_soa_kernel<5><<<g, 256, 0, h->stream>>>(aos, soa, h->ncell, c0, c1);
    CFD_CUDA(h, cudaGetLastError());
    h->launches++;
    return CFD_OK;
}

int launch_soa_to_aos(cfd_handle *h, const double *soa, double *aos, int to_prim, long long c0 = 0, long long c1 = -1)
{
    if (c1 < 0) c1 = h->ncell;
    if (c1 <= c0) return CFD_OK;
    int g = grid_for(c1 - c0);
    if (h->nv == 3) soa_to_aos_kernel<3><<<g, 256, 0, h->stream>>>(soa, aos, h->ncell, to_prim, c0, c1);
    else if (h->nv == 4) soa_to_aos_kernel<4><<<g, 256, 0, h->stream>>>(soa, aos, h->ncell, to_prim, c0, c1);
    else soa_to_aos_kernel<5><<<g, 256, 0, h->stream>>>(soa, aos, h->ncell, to_prim, c0, c1);
    CFD_CUDA(h, cudaGetLastError());
    h->launches++;
    return CFD_OK;
}

SweepParams base_params(cfd_handle *h, int d)
{
    SweepParams p;
    std::memset(&p, 0, sizeof(p));
    p.ncell = h->ncell;
    for (int k = 0; k < 3; k++) {
        p.n[k] = h->cfg.n[k];
        p.stride[k] = h->stride[k];
        p.hdir[k] = h->cfg.h[k];
    }
    p.h = h->cfg.h[d];
    p.red = h->red;
    p.err = h->err;
    p.bc_lo = h->d_bclo[d];
    p.bc_hi = h->d_bchi[d];
    p.bc_vals = h->d_bcvals;
    p.icst = h->icst;
    p.icst_k = h->icst_k;
    p.seg_len = h->seg_len[d];
    p.prec = h->cfg.precision == CFD_PREC_MIXED ? 1 : 0;
    p.dm_u = h->dm_u;
    p.dm_v = h->dm_v;
    p.halo_lo = h->halo[0];
    p.halo_hi = h->halo[1];
    p.halo_nl = h->ncell / h->cfg.n[h->dim - 1];
    p.diff = h->cfg.diff_method;
    p.posl = h->cfg.positivity;
    return p;
}

int sweep(cfd_handle *h, int d, const SweepParams &p)
{
    cudaError_t e = cfd::launch_sweep_any(h->strict, h->nv, h->fam, d, h->cfg.flux_method, p, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "sweep kernel launch");
    h->launches++;
    return CFD_OK;
}

// One RHS evaluation into h->rhs (all directions, x first as rhsSolve does).
int rhs_all(cfd_handle *h, const double *u, double t)
{
    for (int d = 0; d < h->dim; d++) {
        SweepParams p = base_params(h, d);
        p.u = u;
        p.rhs = h->rhs;
        p.mode = cfd::MODE_WRITE;
        p.first = (d == 0);
        p.t = t;
        p.gravity = (h->cfg.source_type == 1 && d == h->dim - 1) ? 1 : 0;
        int rc = sweep(h, d, p);
        if (rc) return rc;
    }
    return CFD_OK;
}

// One RK stage: RHS of uin, then uout = combination (blockSolver.cpp:51-86).
// The sweep along d of one RK stage: a partial RHS for the leading
// directions, the stage combination in the last one.
SweepParams stage_params(cfd_handle *h, int d, int stage, const double *uin, const double *u0, double *uout, double A,
                         double Bdt, double C, double t, bool reduce, const cfd::StepCtl *ctl)
{
    SweepParams p = base_params(h, d);
    p.u = uin;
    p.u0 = u0;
    p.rhs = h->rhs;
    p.u_out = uout;
    bool last = (d == h->dim - 1);
    p.mode = last ? cfd::MODE_RK : cfd::MODE_WRITE;
    p.first = (d == 0);
    p.rk_stage = stage;
    p.rkA = A;
    p.rkBdt = Bdt;
    p.rkC = C;
    p.want_reduce = (reduce && last) ? 1 : 0;
    p.t = t;
    p.ctl = ctl;
    p.gravity = (h->cfg.source_type == 1 && last) ? 1 : 0;
    return p;
}

// the sweeps of one RK stage along directions [d0, d1) (d1 < 0: all)
int rk_stage(cfd_handle *h, int stage, const double *uin, const double *u0, double *uout, double A, double Bdt,
             double C, double t, bool reduce, const cfd::StepCtl *ctl = nullptr, int d0 = 0, int d1 = -1)
{
    if (d1 < 0) d1 = h->dim;
    for (int d = d0; d < d1; d++) {
        int rc = sweep(h, d, stage_params(h, d, stage, uin, u0, uout, A, Bdt, C, t, reduce, ctl));
        if (rc) return rc;
    }
    return CFD_OK;
}

int default_seg_len(const cfd_handle *h, int d)
{
    return cfd::default_seg_len_for(&h->cfg, h->fam, h->strict, d);
}


void drop_graphs(cfd_handle *h)
{
    for (int g = 0; g < 3; g++)
        for (int k = 0; k < 3; k++) {
            if (h->graph[g][k]) cudaGraphExecDestroy(h->graph[g][k]);
            h->graph[g][k] = nullptr;
        }
    for (int k = 0; k < 3; k++) {
        if (h->adj_rec_graph[k]) cudaGraphExecDestroy(h->adj_rec_graph[k]);
        h->adj_rec_graph[k] = nullptr;
    }
    for (int k = 0; k < 2; k++) {
        if (h->adj_recomp_graph[k]) cudaGraphExecDestroy(h->adj_recomp_graph[k]);
        if (h->adj_back_graph[k]) cudaGraphExecDestroy(h->adj_back_graph[k]);
        h->adj_recomp_graph[k] = h->adj_back_graph[k] = nullptr;
    }
    if (h->adj_last_graph) cudaGraphExecDestroy(h->adj_last_graph);
    h->adj_last_graph = nullptr;
    h->adj_graph_K = 0;
}

// Capture the work `enqueue` puts on the handle's stream into an executable
// graph (the launch count is the graph's, not the capture's).
template <class F>
int capture_graph(cfd_handle *h, F &&enqueue, cudaGraphExec_t *exec)
{
    unsigned long long saved = h->launches;
    cudaGraph_t g;
    CFD_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue();
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->launches = saved;
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
    return CFD_OK;
}

constexpr int kGraphSteps[3] = {1, 3, 12};

int check_err(cfd_handle *h, unsigned err)
{
    if (err & cfd::ERR_NONFINITE) return fail(h, CFD_ERR_NONFINITE, "non-finite value in the state after an RK3 step");
    if (err & cfd::ERR_NEGATIVE) return fail(h, CFD_ERR_NEGATIVE_STATE, "density or pressure <= 0 after an RK3 step");
    return CFD_OK;
}

// wave-speed maxima of the current state's cells [c0, c1) folded into red
// (the caller clears red before the first range)
int launch_wave_speed_range(cfd_handle *h, long long c0, long long c1)
{
    if (c1 <= c0) return CFD_OK;
    int g = grid_for(c1 - c0);
    const double *u = h->u[h->cur];
    const double *hh = h->cfg.h;
    if (h->nv == 3) wave_speed_kernel<3><<<g, 256, 0, h->stream>>>(u, h->ncell, hh[0], hh[1], hh[2], h->red, c0, c1);
    else if (h->nv == 4) wave_speed_kernel<4><<<g, 256, 0, h->stream>>>(u, h->ncell, hh[0], hh[1], hh[2], h->red, c0, c1);
    else wave_speed_kernel<5><<<g, 256, 0, h->stream>>>(u, h->ncell, hh[0], hh[1], hh[2], h->red, c0, c1);
    CFD_CUDA(h, cudaGetLastError());
    h->launches++;
    return CFD_OK;
}

int launch_wave_speed(cfd_handle *h)
{
    CFD_CUDA(h, cudaMemsetAsync(h->red, 0, 4 * sizeof(unsigned long long), h->stream));
    int rc = launch_wave_speed_range(h, 0, h->ncell);
    if (rc) return rc;
    h->ws_valid = true;
    return CFD_OK;
}

int ensure_run_buffers(cfd_handle *h, int max_steps)
{
    if (!h->ctl) {
        CFD_CUDA(h, cudaMalloc(&h->ctl, sizeof(cfd::StepCtl)));
        CFD_CUDA(h, cudaMallocHost(&h->ctl_host, sizeof(cfd::StepCtl)));
    }
    if (max_steps > h->log_cap) {
        cudaFree(h->d_dts);
        cudaFree(h->d_linf);
        h->d_dts = h->d_linf = nullptr;
        int cap = max_steps + 16;  // steps past the end stay inside the buffers
        CFD_CUDA(h, cudaMalloc(&h->d_dts, sizeof(double) * cap));
        CFD_CUDA(h, cudaMalloc(&h->d_linf, sizeof(double) * cap));
        h->log_cap = max_steps;
        drop_graphs(h);
    }
    return CFD_OK;
}

// Enqueue one device-controlled SSP-RK3 step (buffers by role).
int enqueue_step(cfd_handle *h, int cur)
{
    double *U0 = h->u[cur], *U1 = h->u[(cur + 1) % 3], *U2 = h->u[(cur + 2) % 3];
    step_begin_kernel<<<1, 1, 0, h->stream>>>(h->ctl, h->red, h->dim, h->d_dts);
    CFD_CUDA(h, cudaGetLastError());
    int rc;
    if ((rc = rk_stage(h, 1, U0, U0, U1, 1.0, 0.0, 0.0, 0.0, false, h->ctl))) return rc;
    if ((rc = rk_stage(h, 2, U1, U0, U2, 0.75, 0.0, 0.25, 0.0, false, h->ctl))) return rc;
    if ((rc = rk_stage(h, 3, U2, U0, U1, 1.0 / 3.0, 0.0, 2.0 / 3.0, 0.0, true, h->ctl))) return rc;
    step_end_kernel<<<1, 1, 0, h->stream>>>(h->ctl, h->red, h->d_linf);
    CFD_CUDA(h, cudaGetLastError());
    return CFD_OK;
}

// Capture kGraphSteps[gi] device-controlled steps starting at state slot
// `slot` into one CUDA graph (kept until the buffers change).
int ensure_graph(cfd_handle *h, int gi, int slot)
{
    if (h->graph[gi][slot]) return CFD_OK;
    const int G = kGraphSteps[gi];
    unsigned long long saved = h->launches;
    cudaGraph_t g;
    CFD_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = CFD_OK;
    for (int s = 0; s < G && rc == CFD_OK; s++) rc = enqueue_step(h, (slot + s) % 3);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->launches = saved;
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&h->graph[gi][slot], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
    return CFD_OK;
}

} // namespace

extern "C" {

const char *cfd_version(void) { return "cfdgpu 0.1 (sm_100a)"; }

void cfd_config_default(cfd_config *c)
{
    std::memset(c, 0, sizeof(*c));
    c->dim = 2;
    c->n[0] = c->n[1] = 200;
    c->n[2] = 1;
    c->h[0] = c->h[1] = c->h[2] = 0.3 / 200;
    c->n_ghost = kGhost;
    c->gamma = 1.4;
    c->inter_method = 2;   // WCNS5
    c->flux_method = CFD_FLUX_HLLC;
    c->diff_method = CFD_DIFF_MND6;
    c->precision = CFD_PREC_FP64;
    c->strict = 0;
    for (int d = 0; d < 3; d++) c->bc[d][0] = c->bc[d][1] = CFD_BND_SUPERSONICOUTLET;
    c->device = 0;
}

int cfd_create(const cfd_config *cfg, cfd_handle **out)
{
    if (!cfg || !out) return CFD_ERR_CONFIG;
    *out = nullptr;
    if (cfg->dim < 1 || cfg->dim > 3) return CFD_ERR_CONFIG;
    if (cfg->diff_method != CFD_DIFF_MND6 && cfg->diff_method != CFD_DIFF_TRAD6) return CFD_ERR_UNSUPPORTED;
    // Info::nGhostCell (info.cpp:7-22): WCNS5 + MND6 -> 4, WCNS5 + TRAD6 -> 5
    if (cfg->n_ghost != (cfg->diff_method == CFD_DIFF_TRAD6 ? kGhost + 1 : kGhost)) return CFD_ERR_UNSUPPORTED;
    if (cfg->gamma != 1.4) return CFD_ERR_UNSUPPORTED;
    if (cfg->diff_method == CFD_DIFF_TRAD6 && cfg->precision != CFD_PREC_FP64) return CFD_ERR_UNSUPPORTED;
    if (cfg->flux_method != CFD_FLUX_HLLC && cfg->flux_method != CFD_FLUX_ROE) return CFD_ERR_CONFIG;
    if (cfg->precision != CFD_PREC_FP64 && cfg->precision != CFD_PREC_MIXED) return CFD_ERR_CONFIG;
    // the mixed form reconstructs in FP32 (multi-dimensional fast flavour only);
    // the strict flavour is the bit-for-bit FP64 build
    if (cfg->precision == CFD_PREC_MIXED && (cfg->dim < 2 || cfg->strict)) return CFD_ERR_UNSUPPORTED;
    if (cfg->precision == CFD_PREC_MIXED && map_inter_method(cfg->inter_method, cfg->dim).fam == cfd::FAM_RESEARCH)
        return CFD_ERR_UNSUPPORTED;  // the research variants have no FP32 decision form
    if (cfg->source_type != 0 && !(cfg->source_type == 1 && cfg->dim == 2)) return CFD_ERR_UNSUPPORTED;
    if (cfg->positivity != 0 && cfg->positivity != 1) return CFD_ERR_CONFIG;
    if (cfg->positivity && cfg->precision == CFD_PREC_MIXED) return CFD_ERR_UNSUPPORTED;  // FP64 faces only
    for (int d = 0; d < 3; d++) {
        if (d < cfg->dim && (cfg->n[d] < 5 || !(cfg->h[d] > 0.0))) return CFD_ERR_CONFIG;
        if (d >= cfg->dim && cfg->n[d] != 1) return CFD_ERR_CONFIG;
    }
    InterMap im = map_inter_method(cfg->inter_method, cfg->dim);
    if (!im.ok) return CFD_ERR_UNSUPPORTED;
    const char *why = nullptr;
    if (!cfd::config_bc_ok(cfg, &why)) {
        fprintf(stderr, "cfd_create: %s\n", why);
        return CFD_ERR_CONFIG;
    }

    cfd_handle *h = new cfd_handle();
    h->cfg = *cfg;
    h->dim = cfg->dim;
    h->nv = cfg->dim + 2;
    h->ncell = (long long)cfg->n[0] * cfg->n[1] * cfg->n[2];
    h->stride[0] = 1;
    h->stride[1] = cfg->n[0];
    h->stride[2] = (long long)cfg->n[0] * cfg->n[1];
    h->fam = im.fam;
    h->ng = cfg->n_ghost;
    h->icst = im.c;
    h->icst_k = (im.fam == cfd::FAM_TENOZ) ? cfd::teno_kappa(im.c) : 0.0;
    h->strict = cfg->strict != 0;
    h->dm_u = 8.25 * std::cos(M_PI / 6);
    h->dm_v = -8.25 * std::sin(M_PI / 6);
    for (int d = 0; d < 3; d++) {
        h->seg_len[d] = 1;
        if (d < h->dim) h->seg_len[d] = cfg->seg_len[d] > 0 ? cfg->seg_len[d] : default_seg_len(h, d);
    }

    auto bail = [&](cudaError_t e, const char *what) {
        int code = (e == cudaErrorMemoryAllocation) ? CFD_ERR_NOMEM : CFD_ERR_CUDA;
        fprintf(stderr, "cfd_create: %s: %s\n", what, cudaGetErrorString(e));
        cfd_destroy(h);
        return code;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(cfg->device)) != cudaSuccess) return bail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    h->stream = h->own_stream;
    size_t bytes = sizeof(double) * h->ncell * h->nv;
    for (int k = 0; k < 3; k++)
        if ((e = cudaMalloc(&h->u[k], bytes)) != cudaSuccess) return bail(e, "state");
    if ((e = cudaMalloc(&h->rhs, bytes)) != cudaSuccess) return bail(e, "rhs");
    if ((e = cudaMalloc(&h->stage, bytes)) != cudaSuccess) return bail(e, "staging");
    if ((e = cudaMalloc(&h->red, 8 * sizeof(unsigned long long))) != cudaSuccess) return bail(e, "reductions");
    if ((e = cudaMalloc(&h->err, sizeof(unsigned))) != cudaSuccess) return bail(e, "error word");
    if ((e = cudaMemsetAsync(h->err, 0, sizeof(unsigned), h->stream)) != cudaSuccess) return bail(e, "memset");
    for (int k = 0; k < 3; k++)
        if ((e = cudaMemsetAsync(h->u[k], 0, bytes, h->stream)) != cudaSuccess) return bail(e, "memset");
    for (int d = 0; d < h->dim; d++) {
        size_t lb = sizeof(BcLine) * (h->ncell / cfg->n[d]);
        if ((e = cudaMalloc(&h->d_bclo[d], lb)) != cudaSuccess) return bail(e, "bc tables");
        if ((e = cudaMalloc(&h->d_bchi[d], lb)) != cudaSuccess) return bail(e, "bc tables");
    }
    wire_defaults(h);
    if (sync_bc(h) != CFD_OK) {
        fprintf(stderr, "cfd_create: %s\n", h->msg.c_str());
        cfd_destroy(h);
        return CFD_ERR_CUDA;
    }
    *out = h;
    return CFD_OK;
}

void cfd_destroy(cfd_handle *h)
{
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (int k = 0; k < 3; k++) cudaFree(h->u[k]);
    cudaFree(h->rhs);
    cudaFree(h->stage);
    cudaFree(h->red);
    cudaFree(h->err);
    for (int d = 0; d < 3; d++) {
        cudaFree(h->d_bclo[d]);
        cudaFree(h->d_bchi[d]);
    }
    cudaFree(h->d_bcvals);
    cudaFree(h->ctl);
    if (h->ctl_host) cudaFreeHost(h->ctl_host);
    cudaFree(h->d_dts);
    cudaFree(h->d_linf);
    for (double *b : h->adj_ckpt) cudaFree(b);
    for (double *b : h->adj_stage) cudaFree(b);
    for (double *b : h->adj_buf) cudaFree(b);
    cudaFree(h->halo[0]);
    cudaFree(h->halo[1]);
    for (double *b : h->adj_stage_b) cudaFree(b);
    drop_graphs(h);
    if (h->adj_aux) {
        cudaStreamSynchronize(h->adj_aux);
        cudaStreamDestroy(h->adj_aux);
    }
    for (cudaEvent_t ev : h->adj_ev)
        if (ev) cudaEventDestroy(ev);
    if (h->copy_st) {
        cudaStreamSynchronize(h->copy_st);
        cudaStreamDestroy(h->copy_st);
    }
    for (auto &row : h->host_ev)
        for (cudaEvent_t ev : row)
            if (ev) cudaEventDestroy(ev);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
}

const char *cfd_last_error(const cfd_handle *h) { return h ? h->msg.c_str() : "null handle"; }

int cfd_set_line_bc(cfd_handle *h, int idim, int i, int j, int side, int bnd_type, long long i0, int offset,
                    const double *ghost_prim)
{
    if (!h) return CFD_ERR_CONFIG;
    int d = idim - 1;
    if (d < 0 || d >= h->dim || (side != 0 && side != 1)) return fail(h, CFD_ERR_CONFIG, "bad idim/side");
    int t0, t1;
    transverse_axes(d, t0, t1);
    if (i < 0 || i >= h->cfg.n[t0] || j < 0 || j >= h->cfg.n[t1]) return fail(h, CFD_ERR_CONFIG, "line index out of range");
    if (bnd_type == CFD_BND_HALO) return fail(h, CFD_ERR_CONFIG, "halo ends are wired by cfd_enable_halo");
    h->line_bc_set[d] = true;
    // BndType values (macro.hpp:33-34) and the true wrap; anything else would
    // leave the line end's ghosts undefined
    if (!((bnd_type >= CFD_BND_TYPENULL && bnd_type <= CFD_BND_SYMMETRYZ) || bnd_type == CFD_BND_PERIODIC_WRAP))
        return fail(h, CFD_ERR_CONFIG, "unknown boundary type");
    if (bnd_type != CFD_BND_PERIODIC_WRAP && (i0 < 0 || i0 >= h->ncell)) return fail(h, CFD_ERR_CONFIG, "i0 out of range");
    if (bnd_type == CFD_BND_PERIODIC1D || (bnd_type >= CFD_BND_SYMMETRYX && bnd_type <= CFD_BND_SYMMETRYZ) ||
        bnd_type == CFD_BND_SYMMETRY1D) {
        long long last = i0 + (long long)(h->ng - 1) * offset;
        if (last < 0 || last >= h->ncell) return fail(h, CFD_ERR_CONFIG, "ghost source outside the grid");
    }
    int slot = -1;
    if (ghost_prim) {
        slot = (int)(h->bc_vals.size() / (h->ng * h->nv));
        h->bc_vals.insert(h->bc_vals.end(), ghost_prim, ghost_prim + h->ng * h->nv);
    }
    long long lid = i + (long long)h->cfg.n[t0] * j;
    set_line(h, d, lid, side, bnd_type, i0, offset, slot);
    return CFD_OK;
}

int cfd_upload_cons(cfd_handle *h, const double *aos)
{
    if (!h || !aos) return CFD_ERR_CONFIG;
    size_t bytes = sizeof(double) * h->ncell * h->nv;
    CFD_CUDA(h, cudaMemcpyAsync(h->stage, aos, bytes, cudaMemcpyHostToDevice, h->stream));
    int rc = launch_aos_to_soa(h, h->stage, h->u[h->cur]);
    if (rc) return rc;
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    h->ws_valid = false;
    return CFD_OK;
}

int cfd_download_cons(cfd_handle *h, double *aos)
{
    if (!h || !aos) return CFD_ERR_CONFIG;
    int rc = launch_soa_to_aos(h, h->u[h->cur], h->stage, 0);
    if (rc) return rc;
    CFD_CUDA(h, cudaMemcpyAsync(aos, h->stage, sizeof(double) * h->ncell * h->nv, cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    return CFD_OK;
}

int cfd_download_prim(cfd_handle *h, double *aos)
{
    if (!h || !aos) return CFD_ERR_CONFIG;
    int rc = launch_soa_to_aos(h, h->u[h->cur], h->stage, 1);
    if (rc) return rc;
    CFD_CUDA(h, cudaMemcpyAsync(aos, h->stage, sizeof(double) * h->ncell * h->nv, cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    return CFD_OK;
}

int cfd_rhs(cfd_handle *h, double t, double *aos_rhs)
{
    if (!h) return CFD_ERR_CONFIG;
    int rc = sync_bc(h);
    if (rc) return rc;
    rc = rhs_all(h, h->u[h->cur], t);
    if (rc) return rc;
    if (aos_rhs) {
        rc = launch_soa_to_aos(h, h->rhs, h->stage, 0);
        if (rc) return rc;
        CFD_CUDA(h, cudaMemcpyAsync(aos_rhs, h->stage, sizeof(double) * h->ncell * h->nv, cudaMemcpyDeviceToHost,
                                    h->stream));
    }
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    return CFD_OK;
}

int cfd_max_dt(cfd_handle *h, double cfl, double *dt)
{
    if (!h || !dt) return CFD_ERR_CONFIG;
    unsigned long long r[4];
    if (!h->ws_valid) {
        int rc = launch_wave_speed(h);
        if (rc) return rc;
    }
    CFD_CUDA(h, cudaMemcpyAsync(r, h->red, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    double lambda = 0;
    for (int d = 0; d < h->dim; d++) {
        double l;
        std::memcpy(&l, &r[1 + d], sizeof(double));
        lambda += l;
    }
    *dt = cfl / lambda;
    return CFD_OK;
}

int cfd_rk3_step(cfd_handle *h, double dt, double t, double *rho_linf)
{
    if (!h) return CFD_ERR_CONFIG;
    int rc = sync_bc(h);
    if (rc) return rc;
    double *U0 = h->u[h->cur], *U1 = h->u[(h->cur + 1) % 3], *U2 = h->u[(h->cur + 2) % 3];
    CFD_CUDA(h, cudaMemsetAsync(h->err, 0, sizeof(unsigned), h->stream));
    // stage times follow info->t in RK3_SSP: t, t + dt, (t + dt) - dt/2
    double t1 = t, t2 = t + dt, t3 = t2 - dt / 2;
    if ((rc = rk_stage(h, 1, U0, U0, U1, 1.0, dt, 0.0, t1, false))) return rc;
    if ((rc = rk_stage(h, 2, U1, U0, U2, 0.75, 0.25 * dt, 0.25, t2, false))) return rc;
    CFD_CUDA(h, cudaMemsetAsync(h->red, 0, 4 * sizeof(unsigned long long), h->stream));
    if ((rc = rk_stage(h, 3, U2, U0, U1, 1.0 / 3.0, 2.0 / 3.0 * dt, 2.0 / 3.0, t3, true))) return rc;
    h->cur = (h->cur + 1) % 3;
    h->ws_valid = true;
    unsigned long long r0;
    unsigned err;
    CFD_CUDA(h, cudaMemcpyAsync(&r0, h->red, sizeof(r0), cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaMemcpyAsync(&err, h->err, sizeof(err), cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    if (rho_linf) std::memcpy(rho_linf, &r0, sizeof(double));
    return check_err(h, err);
}

int cfd_run(cfd_handle *h, double cfl, int end_step, double output_dt, int max_steps, double *t, int *nsteps,
            double *dts, double *linf)
{
    if (!h || !t || !nsteps || max_steps < 0) return CFD_ERR_CONFIG;
    *nsteps = 0;
    if (max_steps == 0 || end_step <= 0) return CFD_OK;
    int rc = sync_bc(h);
    if (rc) return rc;
    if ((rc = ensure_run_buffers(h, max_steps))) return rc;
    if (!h->ws_valid && (rc = launch_wave_speed(h))) return rc;
    // stepsLoopCFL state: step counts output intervals, outputT the time since the last one
    cfd::StepCtl *c = h->ctl_host;
    std::memset(c, 0, sizeof(*c));
    c->t = *t;
    c->outputT = 0.0;
    c->outputDt = output_dt;
    c->cfl = cfl;
    c->endStep = end_step;
    c->maxSteps = max_steps;
    CFD_CUDA(h, cudaMemcpyAsync(h->ctl, c, sizeof(*c), cudaMemcpyHostToDevice, h->stream));
    CFD_CUDA(h, cudaMemsetAsync(h->err, 0, sizeof(unsigned), h->stream));
    const int cur0 = h->cur;
    // Steps are launched as captured graphs of 12, 3 or 1 steps covering
    // exactly max_steps; if the output-interval test ends the loop earlier the
    // remaining launched steps are no-ops on the device. The host checks the
    // device state between batches whose size doubles.
    int launched = 0, slot = cur0, quota = 12;
    const unsigned long long per_step = 2 + 3ULL * h->dim;
    while (true) {
        int target = launched + quota;
        if (target > max_steps) target = max_steps;
        while (launched < target) {
            int rem = target - launched;
            int gi = rem >= 12 ? 2 : rem >= 3 ? 1 : 0;
            if ((rc = ensure_graph(h, gi, slot))) return rc;
            CFD_CUDA(h, cudaGraphLaunch(h->graph[gi][slot], h->stream));
            h->launches += per_step * kGraphSteps[gi];
            launched += kGraphSteps[gi];
            slot = (slot + kGraphSteps[gi]) % 3;
        }
        CFD_CUDA(h, cudaMemcpyAsync(c, h->ctl, sizeof(*c), cudaMemcpyDeviceToHost, h->stream));
        CFD_CUDA(h, cudaStreamSynchronize(h->stream));
        if (c->done || launched >= max_steps) break;
        if (quota < (1 << 20)) quota *= 2;
    }
    // a step that met the loop test before `done` was set still has to finish
    int k = c->k;
    *nsteps = k;
    *t = c->t;
    h->cur = (cur0 + k) % 3;
    h->ws_valid = true;  // stage 3 of the last step left the wave speeds in red[1..3]
    if (k > 0 && dts) CFD_CUDA(h, cudaMemcpy(dts, h->d_dts, sizeof(double) * k, cudaMemcpyDeviceToHost));
    if (k > 0 && linf) CFD_CUDA(h, cudaMemcpy(linf, h->d_linf, sizeof(double) * k, cudaMemcpyDeviceToHost));
    unsigned err;
    CFD_CUDA(h, cudaMemcpy(&err, h->err, sizeof(err), cudaMemcpyDeviceToHost));
    return check_err(h, err);
}

int cfd_step_host(cfd_handle *h, double cfl, double output_dt, const double *in_aos, double *out_aos, double *t,
                  double *dt)
{
    if (!h || !in_aos || !out_aos || !t || !(output_dt > 0.0)) return CFD_ERR_CONFIG;
    if (h->halo[0] || h->halo[1])
        return fail(h, CFD_ERR_UNSUPPORTED, "cfd_step_host: slab halos need an exchange before every stage");
    const int L = h->dim - 1;
    const long long nL = h->cfg.n[L];
    const long long plane = h->ncell / nL;  // cells per index of the last dimension
    const long long seg = h->seg_len[L];
    const long long nseg = (nL + seg - 1) / seg;
    int rc;
    if (h->dim < 2 || nL < 64 || nseg < 2) {
        // too small to overlap: the three calls in turn
        if ((rc = cfd_upload_cons(h, in_aos))) return rc;
        int ns = 0;
        double dts[1] = {0.0};
        if ((rc = cfd_run(h, cfl, 1, output_dt, 1, t, &ns, dts, nullptr))) return rc;
        if (dt) *dt = ns ? dts[0] : 0.0;
        return cfd_download_cons(h, out_aos);
    }
    if ((rc = sync_bc(h)) || (rc = ensure_run_buffers(h, 1))) return rc;
    if (!h->copy_st) CFD_CUDA(h, cudaStreamCreateWithFlags(&h->copy_st, cudaStreamNonBlocking));
    for (auto &row : h->host_ev)
        for (cudaEvent_t &ev : row)
            if (!ev) CFD_CUDA(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaStream_t st = h->stream, cs = h->copy_st;
    const size_t cell_bytes = sizeof(double) * h->nv;
    // step control as cfd_run(h, cfl, 1, output_dt, 1) sets it; the first
    // sweep of stage 1 runs before step_begin_kernel, so its stage time (the
    // current t) is set here as well
    cfd::StepCtl *c = h->ctl_host;
    std::memset(c, 0, sizeof(*c));
    c->t = *t;
    c->outputDt = output_dt;
    c->cfl = cfl;
    c->endStep = 1;
    c->maxSteps = 1;
    c->tst[1] = *t;
    CFD_CUDA(h, cudaMemcpyAsync(h->ctl, c, sizeof(*c), cudaMemcpyHostToDevice, st));
    CFD_CUDA(h, cudaMemsetAsync(h->err, 0, sizeof(unsigned), st));
    CFD_CUDA(h, cudaMemsetAsync(h->red, 0, 4 * sizeof(unsigned long long), st));
    // the copies start after the work queued so far on the handle's stream
    CFD_CUDA(h, cudaEventRecord(h->host_ev[1][0], st));
    CFD_CUDA(h, cudaStreamWaitEvent(cs, h->host_ev[1][0], 0));
    const int cur = h->cur;
    double *U0 = h->u[cur], *U1 = h->u[(cur + 1) % 3], *U2 = h->u[(cur + 2) % 3];
    // Upload in chunks of lines of the last dimension (multiples of 32, which
    // every first-direction tile height divides): each chunk is transposed,
    // its wave speeds folded into the reduction and its lines of stage 1's
    // leading sweeps computed while the next one copies. Stage 1's last sweep
    // (which needs no dt until its combination) runs as a partial RHS in
    // whole segments as soon as their cells and ghost sources are in: the
    // last chunk is uploaded first, so the periodic wrap of the first
    // segments is there. With line ends wired by cfd_set_line_bc along the
    // last direction (ghosts from anywhere) it waits for the whole upload.
    // dt then gives the stage-1 combination (rk_combine), the flavour's own
    // rounding of the epilogue it replaces.
    const long long lines_up = ((nL + kHostChunks - 1) / kHostChunks + 31) / 32 * 32;
    const int nup = (int)((nL + lines_up - 1) / lines_up);
    const long long tail0 = (long long)(nup - 1) * lines_up;  // first row of the last chunk
    const bool early_last = !h->line_bc_set[L];
    const long long halo = 5;  // ghost cells each side of a segment (4 with MND6, 5 with TRAD6)
    long long avail = 0, next_seg = 0;
    auto last_sweep_write = [&](long long s0, long long s1) -> int {
        if (s1 <= s0) return CFD_OK;
        SweepParams p = stage_params(h, L, 1, U0, U0, U1, 1.0, 0.0, 0.0, 0.0, false, h->ctl);
        p.mode = cfd::MODE_WRITE;  // the RHS only; rk_combine applies the stage
        p.part_lo = (int)(s0 * seg);
        p.part_hi = (int)std::min(nL, s1 * seg);
        p.seg_outer = 1;
        return sweep(h, L, p);
    };
    for (int i = 0; i < nup; i++) {
        const int k = (i == 0) ? nup - 1 : i - 1;  // the last chunk first
        const long long r0 = k * lines_up, r1 = std::min(nL, r0 + lines_up), c0 = r0 * plane, c1 = r1 * plane;
        CFD_CUDA(h, cudaMemcpyAsync(h->stage + c0 * h->nv, in_aos + c0 * h->nv, (c1 - c0) * cell_bytes,
                                    cudaMemcpyHostToDevice, cs));
        CFD_CUDA(h, cudaEventRecord(h->host_ev[0][i], cs));
        CFD_CUDA(h, cudaStreamWaitEvent(st, h->host_ev[0][i], 0));
        if ((rc = launch_aos_to_soa(h, h->stage, U0, c0, c1)) || (rc = launch_wave_speed_range(h, c0, c1))) return rc;
        for (int d = 0; d < L; d++) {
            SweepParams p = stage_params(h, d, 1, U0, U0, U1, 1.0, 0.0, 0.0, 0.0, false, h->ctl);
            p.part_lo = (int)r0;
            p.part_hi = (int)r1;
            if ((rc = sweep(h, d, p))) return rc;
        }
        if (k != nup - 1) avail = r1;  // rows [0, avail) and [tail0, nL) are in
        if (!early_last) continue;
        // segment s needs rows [s seg - halo, (s + 1) seg + halo), wrapped; the
        // wrap of the first ones lies in the last chunk if that holds halo rows
        const long long s_end = (avail >= tail0) ? nseg : (nL - tail0 < halo) ? 0 : std::max(0LL, (avail - halo) / seg);
        if (s_end > next_seg) {
            if ((rc = last_sweep_write(next_seg, s_end))) return rc;
            next_seg = s_end;
        }
    }
    if ((rc = last_sweep_write(next_seg, nseg))) return rc;
    step_begin_kernel<<<1, 1, 0, st>>>(h->ctl, h->red, h->dim, h->d_dts);
    CFD_CUDA(h, cudaGetLastError());
    h->launches++;
    {
        SweepParams p = stage_params(h, L, 1, U0, U0, U1, 1.0, 0.0, 0.0, 0.0, false, h->ctl);
        cudaError_t e = cfd::launch_rk_combine_any(h->strict, h->nv, p, st);
        if (e != cudaSuccess) return cuda_fail(h, e, "stage combination launch");
        h->launches++;
    }
    if ((rc = rk_stage(h, 2, U1, U0, U2, 0.75, 0.0, 0.25, 0.0, false, h->ctl)) ||
        (rc = rk_stage(h, 3, U2, U0, U1, 1.0 / 3.0, 0.0, 2.0 / 3.0, 0.0, true, h->ctl, 0, L)))
        return rc;
    // The last sweep of stage 3 in chunks of whole segments along the last
    // dimension: each chunk is transposed and copied out while the next one
    // is computed.
    const long long segs_dn = (nseg + kHostChunks - 1) / kHostChunks;
    int k = 0;
    for (long long s0 = 0; s0 < nseg; s0 += segs_dn, k++) {
        const long long r0 = s0 * seg, r1 = std::min(nL, (s0 + segs_dn) * seg), c0 = r0 * plane, c1 = r1 * plane;
        SweepParams p = stage_params(h, L, 3, U2, U0, U1, 1.0 / 3.0, 0.0, 2.0 / 3.0, 0.0, true, h->ctl);
        p.part_lo = (int)r0;
        p.part_hi = (int)r1;
        p.seg_outer = 1;
        if ((rc = sweep(h, L, p)) || (rc = launch_soa_to_aos(h, U1, h->stage, 0, c0, c1))) return rc;
        CFD_CUDA(h, cudaEventRecord(h->host_ev[1][k], st));
        CFD_CUDA(h, cudaStreamWaitEvent(cs, h->host_ev[1][k], 0));
        CFD_CUDA(h, cudaMemcpyAsync(out_aos + c0 * h->nv, h->stage + c0 * h->nv, (c1 - c0) * cell_bytes,
                                    cudaMemcpyDeviceToHost, cs));
    }
    step_end_kernel<<<1, 1, 0, st>>>(h->ctl, h->red, h->d_linf);
    CFD_CUDA(h, cudaGetLastError());
    h->launches++;
    CFD_CUDA(h, cudaMemcpyAsync(c, h->ctl, sizeof(*c), cudaMemcpyDeviceToHost, st));
    unsigned err = 0;
    CFD_CUDA(h, cudaMemcpyAsync(&err, h->err, sizeof(err), cudaMemcpyDeviceToHost, st));
    CFD_CUDA(h, cudaStreamSynchronize(st));
    CFD_CUDA(h, cudaStreamSynchronize(cs));
    h->cur = (cur + c->k) % 3;
    *t = c->t;
    if (dt) *dt = c->dt;
    h->ws_valid = true;  // stage 3 left the next step's wave speeds in red[1..3]
    return check_err(h, err);
}

int cfd_set_stream(cfd_handle *h, void *stream)
{
    if (!h) return CFD_ERR_CONFIG;
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return CFD_OK;
}

unsigned long long cfd_launch_count(const cfd_handle *h) { return h ? h->launches : 0; }

int cfd_sweep(cfd_handle *h, int idim, int mode, double t)
{
    if (!h) return CFD_ERR_CONFIG;
    int d = idim - 1;
    if (d < 0 || d >= h->dim || mode < 0 || mode > 2) return fail(h, CFD_ERR_CONFIG, "bad idim/mode");
    int rc = sync_bc(h);
    if (rc) return rc;
    SweepParams p = base_params(h, d);
    p.u = h->u[h->cur];
    p.rhs = h->rhs;
    p.t = t;
    if (mode == 2) {
        // the stage-2 combination into the next slot; the current state is kept
        p.mode = cfd::MODE_RK;
        p.first = 0;
        p.rk_stage = 2;
        p.u0 = h->u[h->cur];
        p.u_out = h->u[(h->cur + 2) % 3];
        p.rkA = 0.75;
        p.rkBdt = 0.0;
        p.rkC = 0.25;
    } else {
        p.mode = cfd::MODE_WRITE;
        p.first = (mode == 0);
    }
    return sweep(h, d, p);
}

int cfd_device_state(cfd_handle *h, double **state, long long *ncell, void **stream)
{
    if (!h) return CFD_ERR_CONFIG;
    if (state) *state = h->u[h->cur];
    if (ncell) *ncell = h->ncell;
    if (stream) *stream = (void *)h->stream;
    return CFD_OK;
}

int cfd_set_state_device(cfd_handle *h, const double *soa_dev)
{
    if (!h || !soa_dev) return CFD_ERR_CONFIG;
    CFD_CUDA(h, cudaMemcpyAsync(h->u[h->cur], soa_dev, sizeof(double) * h->ncell * h->nv, cudaMemcpyDeviceToDevice,
                                h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    h->ws_valid = false;
    return CFD_OK;
}

int cfd_fp64_peak_probe(long long iters, void *stream, double *flops)
{
    if (iters < 1 || !flops) return CFD_ERR_CONFIG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return CFD_ERR_CUDA;
    const int blocks = sms * 8, threads = 256;
    dfma_probe_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, 1.0);
    if (cudaGetLastError() != cudaSuccess) return CFD_ERR_CUDA;
    *flops = 2.0 * 8.0 * (double)iters * blocks * threads;
    return CFD_OK;
}

int cfd_check_division(long long n, unsigned long long seed, unsigned long long *mismatches)
{
    if (n < 0 || !mismatches) return CFD_ERR_CONFIG;
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, sizeof(unsigned long long)) != cudaSuccess) return CFD_ERR_NOMEM;
    cudaMemset(d, 0, sizeof(unsigned long long));
    division_check_kernel<<<148 * 8, 256>>>(n, seed, d);
    cudaError_t e = cudaMemcpy(mismatches, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? CFD_OK : CFD_ERR_CUDA;
}

int cfd_eval_inter5(int inter_method, int strict, const double *q, int n, double *out)
{
    (void)strict;
    InterMap im = map_inter_method(inter_method, 2);
    const double kap = (im.fam == cfd::FAM_TENOZ) ? cfd::teno_kappa(im.c) : 0.0;
    if (!im.ok) return CFD_ERR_UNSUPPORTED;
    if (n <= 0) return CFD_OK;
    double *dq = nullptr, *dout = nullptr;
    if (cudaMalloc(&dq, sizeof(double) * 5 * n) != cudaSuccess) return CFD_ERR_NOMEM;
    if (cudaMalloc(&dout, sizeof(double) * n) != cudaSuccess) { cudaFree(dq); return CFD_ERR_NOMEM; }
    cudaMemcpy(dq, q, sizeof(double) * 5 * n, cudaMemcpyHostToDevice);
    int g = (n + 255) / 256;
    switch (im.fam) {
    case cfd::FAM_WCNS5: eval_inter5_kernel<cfd::FAM_WCNS5><<<g, 256>>>(dq, n, im.c, kap, dout); break;
    case cfd::FAM_WENOZ: eval_inter5_kernel<cfd::FAM_WENOZ><<<g, 256>>>(dq, n, im.c, kap, dout); break;
    case cfd::FAM_TENOZ: eval_inter5_kernel<cfd::FAM_TENOZ><<<g, 256>>>(dq, n, im.c, kap, dout); break;
    case cfd::FAM_TENOCONG: eval_inter5_kernel<cfd::FAM_TENOCONG><<<g, 256>>>(dq, n, im.c, kap, dout); break;
    case cfd::FAM_RESEARCH: eval_inter5_kernel<cfd::FAM_RESEARCH><<<g, 256>>>(dq, n, im.c, kap, dout); break;
    default: eval_inter5_kernel<cfd::FAM_MUSCL><<<g, 256>>>(dq, n, im.c, kap, dout); break;
    }
    cudaError_t e = cudaMemcpy(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(dq);
    cudaFree(dout);
    return e == cudaSuccess ? CFD_OK : CFD_ERR_CUDA;
}

int cfd_eval_flux(int dim, int ax, int flux_method, int strict, const double *lr, int n, double *out)
{
    (void)strict;
    if (dim < 1 || dim > 3 || ax < 0 || ax >= dim) return CFD_ERR_CONFIG;
    if (n <= 0) return CFD_OK;
    int nv = dim + 2;
    double *din = nullptr, *dout = nullptr;
    if (cudaMalloc(&din, sizeof(double) * 2 * nv * n) != cudaSuccess) return CFD_ERR_NOMEM;
    if (cudaMalloc(&dout, sizeof(double) * nv * n) != cudaSuccess) { cudaFree(din); return CFD_ERR_NOMEM; }
    cudaMemcpy(din, lr, sizeof(double) * 2 * nv * n, cudaMemcpyHostToDevice);
    int g = (n + 255) / 256;
    bool hllc = flux_method == CFD_FLUX_HLLC;
#define CFD_EF(NV, AX)                                                                                   \
    if (nv == NV && ax == AX) {                                                                          \
        if (hllc) eval_flux_kernel<NV, AX, cfd::FLUX_HLLC><<<g, 256>>>(din, n, dout);                   \
        else eval_flux_kernel<NV, AX, cfd::FLUX_ROE><<<g, 256>>>(din, n, dout);                         \
    }
    CFD_EF(3, 0) CFD_EF(4, 0) CFD_EF(4, 1) CFD_EF(5, 0) CFD_EF(5, 1) CFD_EF(5, 2)
#undef CFD_EF
    cudaError_t e = cudaMemcpy(out, dout, sizeof(double) * nv * n, cudaMemcpyDeviceToHost);
    cudaFree(din);
    cudaFree(dout);
    return e == cudaSuccess ? CFD_OK : CFD_ERR_CUDA;
}

} // extern "C"

extern "C" int cfd_eval_face(int dim, int ax, int inter_method, int precision, const double *prims6, int n,
                             double *out)
{
    if (dim < 1 || dim > 3 || ax < 0 || ax >= dim || (precision != 0 && precision != 1)) return CFD_ERR_CONFIG;
    if (precision == 1 && dim == 1) return CFD_ERR_UNSUPPORTED;
    InterMap im = map_inter_method(inter_method, dim);
    const double kap = (im.fam == cfd::FAM_TENOZ) ? cfd::teno_kappa(im.c) : 0.0;
    if (!im.ok || (precision == 1 && im.fam == cfd::FAM_RESEARCH)) return CFD_ERR_UNSUPPORTED;
    if (n <= 0) return CFD_OK;
    int nv = dim + 2;
    double *din = nullptr, *dout = nullptr;
    if (cudaMalloc(&din, sizeof(double) * 6 * nv * n) != cudaSuccess) return CFD_ERR_NOMEM;
    if (cudaMalloc(&dout, sizeof(double) * 2 * nv * n) != cudaSuccess) {
        cudaFree(din);
        return CFD_ERR_NOMEM;
    }
    cudaMemcpy(din, prims6, sizeof(double) * 6 * nv * n, cudaMemcpyHostToDevice);
    int g = (n + 127) / 128;
    bool launched = false;
#define CFD_EFACE(NV, AX, F)                                                                                  \
    if (!launched && nv == NV && ax == AX && im.fam == F) {                                                   \
        if (precision == 1) eval_face_kernel<NV, AX, F, (NV >= 4 && F != 5 ? 1 : 0)><<<g, 128>>>(din, n, im.c, kap, dout); \
        else eval_face_kernel<NV, AX, F, 0><<<g, 128>>>(din, n, im.c, kap, dout);                             \
        launched = true;                                                                                      \
    }
#define CFD_EFACE_F(F) CFD_EFACE(3, 0, F) CFD_EFACE(4, 0, F) CFD_EFACE(4, 1, F) CFD_EFACE(5, 0, F) \
                       CFD_EFACE(5, 1, F) CFD_EFACE(5, 2, F)
    CFD_EFACE_F(0) CFD_EFACE_F(1) CFD_EFACE_F(2) CFD_EFACE_F(3) CFD_EFACE_F(4) CFD_EFACE_F(5)
#undef CFD_EFACE_F
#undef CFD_EFACE
    cudaError_t e = cudaMemcpy(out, dout, sizeof(double) * 2 * nv * n, cudaMemcpyDeviceToHost);
    cudaFree(din);
    cudaFree(dout);
    return e == cudaSuccess ? CFD_OK : CFD_ERR_CUDA;
}

extern "C" int cfd_accuracy_test(int inter_method, int n, double h, const double *q, double *dqdx)
{
    InterMap im = map_inter_method(inter_method, 1);
    if (!im.ok) return CFD_ERR_UNSUPPORTED;
    if (n < 1 || !(h > 0)) return CFD_ERR_CONFIG;
    double *dq = nullptr, *dout = nullptr;
    if (cudaMalloc(&dq, sizeof(double) * (n + 8)) != cudaSuccess) return CFD_ERR_NOMEM;
    if (cudaMalloc(&dout, sizeof(double) * n) != cudaSuccess) {
        cudaFree(dq);
        return CFD_ERR_NOMEM;
    }
    cudaMemcpy(dq, q, sizeof(double) * (n + 8), cudaMemcpyHostToDevice);
    int g = (n + 127) / 128;
    switch (im.fam) {
    case cfd::FAM_WCNS5: accuracy_kernel<cfd::FAM_WCNS5><<<g, 128>>>(dq, n, h, im.c, dout); break;
    case cfd::FAM_WENOZ: accuracy_kernel<cfd::FAM_WENOZ><<<g, 128>>>(dq, n, h, im.c, dout); break;
    case cfd::FAM_TENOZ: accuracy_kernel<cfd::FAM_TENOZ><<<g, 128>>>(dq, n, h, im.c, dout); break;
    case cfd::FAM_TENOCONG: accuracy_kernel<cfd::FAM_TENOCONG><<<g, 128>>>(dq, n, h, im.c, dout); break;
    case cfd::FAM_RESEARCH: accuracy_kernel<cfd::FAM_RESEARCH><<<g, 128>>>(dq, n, h, im.c, dout); break;
    default: accuracy_kernel<cfd::FAM_MUSCL><<<g, 128>>>(dq, n, h, im.c, dout); break;
    }
    cudaError_t e = cudaMemcpy(dqdx, dout, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(dq);
    cudaFree(dout);
    return e == cudaSuccess ? CFD_OK : CFD_ERR_CUDA;
}

namespace cfd {
// Default cells per CTA segment along direction d for the tile shapes that
// launch_sweep picks for this configuration: about six waves of CTAs over the
// 148 SMs. Shared with the allocation-free entry point (noalloc.cu).
int default_seg_len_for(const cfd_config *cfg, int fam, bool strict, int d)
{
    int n = cfg->n[d];
    int S = (cfg->dim == 1) ? cfd::k1S : (d == 0 ? cfd::kXS : cfd::kYS);
    int W = (cfg->dim == 1) ? cfd::k1W : (d == 0 ? cfd::kXW : cfd::kYW);
    if (cfg->dim > 1 && d == 0 && cfg->diff_method != CFD_DIFF_TRAD6 &&
        (cfg->dim == 3 || cfg->precision == CFD_PREC_FP64)) {
        S = cfd::kXSn;  // the x sweep shape of launch_sweep
        W = cfd::kXWn;
    }
    const bool mixed_shape = (d == 1 || (d == 2 && CFD_MIXED_Z16)) && cfg->precision == CFD_PREC_MIXED && !strict &&
                             fam != cfd::FAM_RESEARCH;
    const bool fp64_shape = cfg->precision == CFD_PREC_FP64 &&
                            ((CFD_FP64_3D_YZ16 && cfg->dim == 3 && d > 0) || (CFD_FP64_2D_Y16 && cfg->dim == 2 && d == 1));
    if (cfg->dim > 1 && (mixed_shape || fp64_shape) && cfg->diff_method != CFD_DIFF_TRAD6) {
        S = cfd::kYSm;  // the mixed form's y sweep shape (launch_sweep)
        W = cfd::kYWm;
    }
    int t0, t1;
    transverse_axes(d, t0, t1);
    long long blocks_per_seg = (long long)((cfg->n[t0] + W - 1) / W) * cfg->n[t1];
    // about 1,800 CTAs (3 to 6 waves at 2 to 4 resident per SM); the mixed
    // form's x sweep measured fastest with half as many, longer segments
    const bool mixed_x = d == 0 && cfg->dim > 1 && cfg->precision == CFD_PREC_MIXED;
    const long long target = mixed_x ? 148LL * 2 * 3 : 148LL * 2 * 6;
    int seg = n;
    while (blocks_per_seg * ((n + seg - 1) / seg) < target && seg > 4 * S) seg = (seg + 1) / 2;
    return seg;
}

// The boundary types cfg->bc can wire by itself, i.e. every line end of a
// direction with no per-line data: the copying types (PERIODIC1D and
// SUPERSONICOUTLET with the Initializer::initBnds source cells, the true
// wrap), the mirrors of the directions the grid has (SYMMETRY1D in 1D only:
// in 2D and 3D it leaves the pressure ghost to static data), and the moving
// DoubleMachUp top in 2D. DIRICLET and the other static types need ghost
// values (cfd_set_line_bc), HALO ends are wired by cfd_enable_halo, and any
// other value is not a BndType (macro.hpp:33-34). Checked before any device
// work: a line end of one of those types would read ghost data that does not
// exist (all-zero ghosts, or a null halo buffer).
bool config_bc_ok(const cfd_config *cfg, const char **why)
{
    for (int d = 0; d < cfg->dim; d++)
        for (int s = 0; s < 2; s++) {
            const int t = cfg->bc[d][s];
            bool ok = false;
            switch (t) {
            case CFD_BND_PERIODIC1D:
            case CFD_BND_SUPERSONICOUTLET:
            case CFD_BND_PERIODIC_WRAP:
            case CFD_BND_SYMMETRYX: ok = true; break;
            case CFD_BND_SYMMETRY1D: ok = cfg->dim == 1; break;
            case CFD_BND_SYMMETRYY: ok = cfg->dim >= 2; break;
            case CFD_BND_SYMMETRYZ: ok = cfg->dim == 3; break;
            case CFD_BND_DOUBLEMACHUP: ok = cfg->dim == 2; break;
            default: ok = false;
            }
            if (!ok) {
                if (why)
                    *why = (t == CFD_BND_HALO) ? "CFD_BND_HALO in cfg->bc (halo ends are wired by cfd_enable_halo)"
                           : (t == CFD_BND_DIRICLET || t == CFD_BND_TYPENULL || (t >= 4 && t <= 6) || t == 9)
                               ? "a static boundary type in cfg->bc (its ghost values are set per line by cfd_set_line_bc)"
                               : "cfg->bc holds a boundary type this dimension cannot wire";
                return false;
            }
        }
    return true;
}

// Selector lookup shared with the allocation-free entry point (noalloc.cu).
bool map_inter_method_for(int inter_method, int dim, int *fam, double *c)
{
    InterMap im = map_inter_method(inter_method, dim);
    if (!im.ok) return false;
    *fam = im.fam;
    *c = im.c;
    return true;
}
} // namespace cfd

// ===================================================================== batch
// Many independent cases advanced together: one persistent sweep launch per
// direction and stage covers the tiles of every unfinished case, and one
// control kernel advances every case's own stepsLoopCFL state (own dt,
// own output clipping, own step count).

namespace {

__global__ void batch_step_begin_kernel(cfd::StepCtl *ctl, unsigned long long *const *reds, int ncases, int dim,
                                        int *active)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncases) return;
    cfd::StepCtl *cc = ctl + c;
    if (cc->done) return;
    if (!(cc->step < cc->endStep && cc->k < cc->maxSteps)) {
        cc->done = 1;
        return;
    }
    unsigned long long *red = reds[c];
    double lambda = 0;
    for (int d = 0; d < dim; d++) lambda += __longlong_as_double((long long)red[1 + d]);
    double dt = cc->cfl / lambda;
    if (cc->outputT + dt > cc->outputDt) {
        dt = cc->outputDt - cc->outputT;
        cc->outputT = 0.0;
        cc->step++;
    } else
        cc->outputT += dt;
    cc->dt = dt;
    cc->bdt[1] = dt;
    cc->bdt[2] = 0.25 * dt;
    cc->bdt[3] = 2.0 / 3.0 * dt;
    cc->tst[1] = cc->t;
    cc->tst[2] = cc->t + dt;
    cc->tst[3] = cc->tst[2] - dt / 2;
    for (int i = 0; i < 4; i++) red[i] = 0ULL;
    atomicAdd(active, 1);
}

__global__ void batch_step_end_kernel(cfd::StepCtl *ctl, int ncases)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncases) return;
    cfd::StepCtl *cc = ctl + c;
    if (cc->done) return;
    double dt = cc->dt;
    cc->t = (((cc->t + dt) - dt / 2) - dt / 2) + dt;
    cc->k++;
}

} // namespace

struct cfd_batch {
    std::vector<cfd_handle *> h;
    int ncases = 0, dim = 0, nv = 0, fam = 0, flux = 0, prec = 0;
    bool strict = false;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    cfd::StepCtl *ctl = nullptr, *ctl_host = nullptr;
    unsigned long long **d_reds = nullptr;
    int *d_active = nullptr;
    // params[(slot * 3 + (stage - 1)) * dim + d][case]
    std::vector<SweepParams> params_host;
    SweepParams *d_params = nullptr;
    long long *d_tile_start = nullptr;  // [dim][ncases + 1]
    std::vector<long long> tile_total;
    // work-list order: cases by decreasing cell count, so that the persistent
    // CTAs take the longest tiles first and the tail holds the short ones
    std::vector<int> order;
    // tiling per direction, chosen by cfd_batch_autotune: tile shape (0 the
    // single-grid shape, 1 the alternative), segments per line, one persistent
    // CTA per SM instead of as many as fit
    int shape[3] = {0, 0, 0}, split[3] = {1, 1, 1}, one_cta[3] = {0, 0, 0};
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    unsigned long long launches = 0;
    std::string msg;
};

namespace {

int bfail(cfd_batch *b, int code, const std::string &m)
{
    if (b) b->msg = m;
    return code;
}

#define CFD_BCUDA(b, call)                                                         \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) return bfail(b, CFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Parameter block of case c for the sweep along d in stage `stage`, with the
// state buffers taken `slot` steps after the case's current slot.
SweepParams batch_params(cfd_batch *b, int c, int slot, int stage, int d)
{
    cfd_handle *h = b->h[c];
    int cur = (h->cur + slot) % 3;
    double *U0 = h->u[cur], *U1 = h->u[(cur + 1) % 3], *U2 = h->u[(cur + 2) % 3];
    SweepParams p = base_params(h, d);
    const double *uin = stage == 1 ? U0 : stage == 2 ? U1 : U2;
    double *uout = stage == 2 ? U2 : U1;
    bool last = (d == b->dim - 1);
    p.u = uin;
    p.u0 = U0;
    p.rhs = h->rhs;
    p.u_out = uout;
    p.mode = last ? cfd::MODE_RK : cfd::MODE_WRITE;
    p.first = (d == 0);
    p.rk_stage = stage;
    p.rkA = stage == 1 ? 1.0 : stage == 2 ? 0.75 : 1.0 / 3.0;
    p.rkC = stage == 1 ? 0.0 : stage == 2 ? 0.25 : 2.0 / 3.0;
    p.want_reduce = (stage == 3 && last) ? 1 : 0;
    p.ctl = b->ctl + c;
    p.gravity = (h->cfg.source_type == 1 && last) ? 1 : 0;
    return p;
}

// Cells per chunk of the sweep along d with the batch's tile shape.
int batch_chunk(const cfd_batch *b, int d)
{
    if (b->nv == 3) return cfd::k1S;
    if (d == 0) return b->shape[0] ? cfd::kXS2 : cfd::kXS;
    return b->shape[d] ? cfd::kYS2 : cfd::kYS;
}

// Segment lengths of every case (lines cut into split[d] segments of whole
// chunks) and the work list's tile prefix sums for the current tiling.
int batch_layout(cfd_batch *b)
{
    std::vector<long long> ts((size_t)b->dim * (b->ncases + 1));
    b->tile_total.assign(b->dim, 0);
    for (int d = 0; d < b->dim; d++) {
        const int S = batch_chunk(b, d);
        long long acc = 0;
        for (int i = 0; i < b->ncases; i++) {
            cfd_handle *h = b->h[b->order[i]];
            const int n = h->cfg.n[d];
            int seg = (n + b->split[d] - 1) / b->split[d];
            seg = ((seg + S - 1) / S) * S;
            h->seg_len[d] = seg < n ? seg : n;
            ts[(size_t)d * (b->ncases + 1) + i] = acc;
            acc += cfd::sweep_tile_count(b->nv, d, base_params(h, d), b->shape[d]);
        }
        ts[(size_t)d * (b->ncases + 1) + b->ncases] = acc;
        b->tile_total[d] = acc;
    }
    CFD_BCUDA(b, cudaMemcpy(b->d_tile_start, ts.data(), sizeof(long long) * ts.size(), cudaMemcpyHostToDevice));
    if (b->graph) {  // captured with the old tiling
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return CFD_OK;
}

cfd::BatchSweep batch_sweep(cfd_batch *b, int slot, int stage, int d)
{
    cfd::BatchSweep bs;
    bs.cases = b->d_params + (size_t)((slot * 3 + (stage - 1)) * b->dim + d) * b->ncases;
    bs.tile_start = b->d_tile_start + (size_t)d * (b->ncases + 1);
    bs.ncases = b->ncases;
    bs.total_tiles = b->tile_total[d];
    bs.num_sms = b->num_sms;
    bs.prec = b->prec;
    bs.shape = b->shape[d];
    bs.one_cta = b->one_cta[d];
    return bs;
}

int batch_enqueue_step(cfd_batch *b, int slot)
{
    int g = (b->ncases + 127) / 128;
    batch_step_begin_kernel<<<g, 128, 0, b->stream>>>(b->ctl, b->d_reds, b->ncases, b->dim, b->d_active);
    CFD_BCUDA(b, cudaGetLastError());
    for (int stage = 1; stage <= 3; stage++) {
        for (int d = 0; d < b->dim; d++) {
            const cfd::BatchSweep bs = batch_sweep(b, slot, stage, d);
            cudaError_t e = cfd::launch_sweep_batched_any(b->strict, b->nv, b->fam, d, b->flux, bs, b->stream);
            if (e != cudaSuccess) return bfail(b, CFD_ERR_CUDA, std::string("batched sweep: ") + cudaGetErrorString(e));
        }
    }
    batch_step_end_kernel<<<g, 128, 0, b->stream>>>(b->ctl, b->ncases);
    CFD_BCUDA(b, cudaGetLastError());
    return CFD_OK;
}

} // namespace

extern "C" {

int cfd_batch_create(const cfd_config *cfgs, int ncases, cfd_batch **out)
{
    if (!cfgs || !out || ncases < 1) return CFD_ERR_CONFIG;
    *out = nullptr;
    for (int c = 1; c < ncases; c++) {
        const cfd_config &a = cfgs[0], &z = cfgs[c];
        if (a.dim != z.dim || a.inter_method != z.inter_method || a.flux_method != z.flux_method ||
            a.strict != z.strict || a.precision != z.precision || a.device != z.device)
            return CFD_ERR_CONFIG;  // one kernel instantiation serves the batch
    }
    for (int c = 0; c < ncases; c++)
        if (cfgs[c].diff_method != CFD_DIFF_MND6) return CFD_ERR_UNSUPPORTED;  // the batched kernel is MND6 only
    cfd_batch *b = new cfd_batch();
    b->ncases = ncases;
    for (int c = 0; c < ncases; c++) {
        cfd_config cc = cfgs[c];
        for (int d = 0; d < 3; d++)
            if (cc.seg_len[d] <= 0) cc.seg_len[d] = cc.n[d];  // whole lines: the batch has tiles to spare
        cfd_handle *h = nullptr;
        int rc = cfd_create(&cc, &h);
        if (rc) {
            cfd_batch_destroy(b);
            return rc;
        }
        b->h.push_back(h);
    }
    cfd_handle *h0 = b->h[0];
    b->dim = h0->dim;
    b->nv = h0->nv;
    b->fam = h0->fam;
    b->flux = h0->cfg.flux_method;
    b->strict = h0->strict;
    b->prec = h0->cfg.precision == CFD_PREC_MIXED ? 1 : 0;
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, h0->cfg.device);
    auto bail = [&](cudaError_t e) {
        fprintf(stderr, "cfd_batch_create: %s\n", cudaGetErrorString(e));
        cfd_batch_destroy(b);
        return e == cudaErrorMemoryAllocation ? CFD_ERR_NOMEM : CFD_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e);
    b->stream = b->own_stream;
    if ((e = cudaMalloc(&b->ctl, sizeof(cfd::StepCtl) * ncases)) != cudaSuccess) return bail(e);
    if ((e = cudaMallocHost(&b->ctl_host, sizeof(cfd::StepCtl) * ncases)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&b->d_reds, sizeof(unsigned long long *) * ncases)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&b->d_active, sizeof(int))) != cudaSuccess) return bail(e);
    std::vector<unsigned long long *> reds(ncases);
    for (int c = 0; c < ncases; c++) reds[c] = b->h[c]->red;
    if ((e = cudaMemcpy(b->d_reds, reds.data(), sizeof(void *) * ncases, cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(e);
    size_t np = (size_t)9 * b->dim * ncases;
    b->params_host.resize(np);
    if ((e = cudaMalloc(&b->d_params, sizeof(SweepParams) * np)) != cudaSuccess) return bail(e);
    b->order.resize(ncases);
    for (int c = 0; c < ncases; c++) b->order[c] = c;
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return b->h[x]->ncell > b->h[y]->ncell; });
    // whole lines by default (cfd_batch_autotune may cut them); the config's
    // seg_len of each case is replaced by the batch's tiling
    if ((e = cudaMalloc(&b->d_tile_start, sizeof(long long) * b->dim * (ncases + 1))) != cudaSuccess) return bail(e);
    int rc = batch_layout(b);
    if (rc) {
        fprintf(stderr, "cfd_batch_create: %s\n", b->msg.c_str());
        cfd_batch_destroy(b);
        return rc;
    }
    *out = b;
    return CFD_OK;
}

void cfd_batch_destroy(cfd_batch *b)
{
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (cfd_handle *h : b->h) cfd_destroy(h);
    cudaFree(b->ctl);
    if (b->ctl_host) cudaFreeHost(b->ctl_host);
    cudaFree(b->d_reds);
    cudaFree(b->d_active);
    cudaFree(b->d_params);
    cudaFree(b->d_tile_start);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    delete b;
}

const char *cfd_batch_last_error(const cfd_batch *b) { return b ? b->msg.c_str() : "null batch"; }

int cfd_batch_case(cfd_batch *b, int c, cfd_handle **h)
{
    if (!b || !h || c < 0 || c >= b->ncases) return CFD_ERR_CONFIG;
    *h = b->h[c];
    return CFD_OK;
}

int cfd_batch_set_stream(cfd_batch *b, void *stream)
{
    if (!b) return CFD_ERR_CONFIG;
    CFD_BCUDA(b, cudaStreamSynchronize(b->stream));
    b->stream = stream ? (cudaStream_t)stream : b->own_stream;
    return CFD_OK;
}

unsigned long long cfd_batch_launch_count(const cfd_batch *b) { return b ? b->launches : 0; }

int cfd_batch_run(cfd_batch *b, double cfl, int end_step, const double *output_dt, int max_steps, double *t,
                  int *nsteps)
{
    if (!b || !output_dt || !t || !nsteps || max_steps < 0 || end_step < 0) return CFD_ERR_CONFIG;
    for (int c = 0; c < b->ncases; c++) nsteps[c] = 0;
    if (max_steps == 0 || end_step == 0) return CFD_OK;
    // every case's boundary tables and initial wave speeds on the handle streams
    for (int c = 0; c < b->ncases; c++) {
        cfd_handle *h = b->h[c];
        int rc = sync_bc(h);
        if (rc) return bfail(b, rc, h->msg);
        if (!h->ws_valid && (rc = launch_wave_speed(h))) return bfail(b, rc, h->msg);
        CFD_BCUDA(b, cudaMemsetAsync(h->err, 0, sizeof(unsigned), h->stream));
        CFD_BCUDA(b, cudaStreamSynchronize(h->stream));
    }
    // parameter blocks for the three buffer rotations, stages and directions
    for (int slot = 0; slot < 3; slot++)
        for (int stage = 1; stage <= 3; stage++)
            for (int d = 0; d < b->dim; d++)
                for (int i = 0; i < b->ncases; i++)
                    b->params_host[(size_t)((slot * 3 + (stage - 1)) * b->dim + d) * b->ncases + i] =
                        batch_params(b, b->order[i], slot, stage, d);
    CFD_BCUDA(b, cudaMemcpyAsync(b->d_params, b->params_host.data(), sizeof(SweepParams) * b->params_host.size(),
                                 cudaMemcpyHostToDevice, b->stream));
    for (int c = 0; c < b->ncases; c++) {
        cfd::StepCtl &cc = b->ctl_host[c];
        std::memset(&cc, 0, sizeof(cc));
        cc.t = t[c];
        cc.outputDt = output_dt[c];
        cc.cfl = cfl;
        cc.endStep = end_step;
        cc.maxSteps = max_steps;
    }
    CFD_BCUDA(b, cudaMemcpyAsync(b->ctl, b->ctl_host, sizeof(cfd::StepCtl) * b->ncases, cudaMemcpyHostToDevice,
                                 b->stream));
    // graph of 3 steps (the buffers return to their roles after each graph)
    const int G = 3;
    if (!b->graph) {
        cudaGraph_t g;
        CFD_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = CFD_OK;
        for (int s = 0; s < G && rc == CFD_OK; s++) rc = batch_enqueue_step(b, s);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return bfail(b, CFD_ERR_CUDA, cudaGetErrorString(e));
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return bfail(b, CFD_ERR_CUDA, cudaGetErrorString(e));
        b->graph_steps = G;
    }
    int launched = 0, quota = 3;
    int active = 0;
    const unsigned long long per_step = 2 + 3ULL * b->dim;
    while (launched < max_steps) {
        CFD_BCUDA(b, cudaMemsetAsync(b->d_active, 0, sizeof(int), b->stream));
        for (int q = 0; q < quota && launched < max_steps; q += G) {
            CFD_BCUDA(b, cudaGraphLaunch(b->graph, b->stream));
            b->launches += per_step * G;
            launched += G;
        }
        CFD_BCUDA(b, cudaMemcpyAsync(&active, b->d_active, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
        CFD_BCUDA(b, cudaStreamSynchronize(b->stream));
        if (active == 0) break;  // no case took a step in the last batch of graphs
        if (quota < (1 << 16)) quota *= 2;
    }
    CFD_BCUDA(b, cudaMemcpyAsync(b->ctl_host, b->ctl, sizeof(cfd::StepCtl) * b->ncases, cudaMemcpyDeviceToHost,
                                 b->stream));
    CFD_BCUDA(b, cudaStreamSynchronize(b->stream));
    int rc = CFD_OK;
    for (int c = 0; c < b->ncases; c++) {
        cfd_handle *h = b->h[c];
        int k = b->ctl_host[c].k;
        nsteps[c] = k;
        t[c] = b->ctl_host[c].t;
        h->cur = (h->cur + k) % 3;
        h->ws_valid = true;
        unsigned err = 0;
        CFD_BCUDA(b, cudaMemcpy(&err, h->err, sizeof(err), cudaMemcpyDeviceToHost));
        int r = check_err(h, err);
        if (r && !rc) {
            rc = r;
            b->msg = "case " + std::to_string(c) + ": " + h->msg;
        }
    }
    return rc;
}

int cfd_batch_set_tiling(cfd_batch *b, int idim, int shape, int segments, int one_cta)
{
    if (!b) return CFD_ERR_CONFIG;
    const int d = idim - 1;
    if (d < 0 || d >= b->dim || shape < 0 || shape > 1 || segments < 1 || segments > 64 || one_cta < 0 ||
        one_cta > 1)
        return bfail(b, CFD_ERR_CONFIG, "bad tiling");
    if (shape == 1 && !(b->nv >= 4 && b->prec == 0))
        return bfail(b, CFD_ERR_UNSUPPORTED, "the alternative tile shape is 2D/3D FP64 only");
    b->shape[d] = shape;
    b->split[d] = segments;
    b->one_cta[d] = one_cta;
    return batch_layout(b);
}

int cfd_batch_autotune(cfd_batch *b, int *choice, double *ms)
{
    if (!b) return CFD_ERR_CONFIG;
    // first-stage sweeps read U^0 and write only the RHS and U^(1), both
    // scratch between steps; step control: not done, dt = 0
    for (int c = 0; c < b->ncases; c++) {
        int rc = sync_bc(b->h[c]);
        if (rc) return bfail(b, rc, b->h[c]->msg);
    }
    std::memset(b->ctl_host, 0, sizeof(cfd::StepCtl) * b->ncases);
    CFD_BCUDA(b, cudaMemcpyAsync(b->ctl, b->ctl_host, sizeof(cfd::StepCtl) * b->ncases, cudaMemcpyHostToDevice,
                                 b->stream));
    const bool alt = b->nv >= 4 && b->prec == 0;  // the alternative shapes: 2D/3D FP64
    cudaEvent_t e0, e1;
    CFD_BCUDA(b, cudaEventCreate(&e0));
    CFD_BCUDA(b, cudaEventCreate(&e1));
    int rc = CFD_OK;
    for (int d = 0; d < b->dim && rc == CFD_OK; d++) {
        float best = 3.4e38f;
        int best_cfg[3] = {b->shape[d], b->split[d], b->one_cta[d]};
        for (int shape = 0; shape <= (alt ? 1 : 0) && rc == CFD_OK; shape++)
            for (int split = 1; split <= 2 && rc == CFD_OK; split++)
                for (int one = 0; one <= 1 && rc == CFD_OK; one++) {
                    b->shape[d] = shape;
                    b->split[d] = split;
                    b->one_cta[d] = one;
                    if ((rc = batch_layout(b))) break;
                    for (int i = 0; i < b->ncases; i++)
                        b->params_host[(size_t)d * b->ncases + i] = batch_params(b, b->order[i], 0, 1, d);
                    const cfd::BatchSweep bs = batch_sweep(b, 0, 1, d);
                    CFD_BCUDA(b, cudaMemcpyAsync(b->d_params + (size_t)d * b->ncases,
                                                 b->params_host.data() + (size_t)d * b->ncases,
                                                 sizeof(SweepParams) * b->ncases, cudaMemcpyHostToDevice, b->stream));
                    float t = 0.0f;
                    for (int rep = 0; rep < 4 && rc == CFD_OK; rep++) {  // one warm-up, three timed
                        CFD_BCUDA(b, cudaEventRecord(e0, b->stream));
                        cudaError_t e =
                            cfd::launch_sweep_batched_any(b->strict, b->nv, b->fam, d, b->flux, bs, b->stream);
                        if (e != cudaSuccess)
                            rc = bfail(b, CFD_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
                        CFD_BCUDA(b, cudaEventRecord(e1, b->stream));
                        CFD_BCUDA(b, cudaEventSynchronize(e1));
                        float ms1 = 0.0f;
                        CFD_BCUDA(b, cudaEventElapsedTime(&ms1, e0, e1));
                        if (rep > 0) t += ms1;
                    }
                    if (rc == CFD_OK && t < best) {
                        best = t;
                        best_cfg[0] = shape;
                        best_cfg[1] = split;
                        best_cfg[2] = one;
                    }
                }
        b->shape[d] = best_cfg[0];
        b->split[d] = best_cfg[1];
        b->one_cta[d] = best_cfg[2];
        if (choice) {
            choice[3 * d] = best_cfg[0];
            choice[3 * d + 1] = best_cfg[1];
            choice[3 * d + 2] = best_cfg[2];
        }
        if (ms) ms[d] = best / 3.0;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rc2 = batch_layout(b);
    for (int c = 0; c < b->ncases && rc == CFD_OK; c++)
        CFD_BCUDA(b, cudaMemsetAsync(b->h[c]->err, 0, sizeof(unsigned), b->stream));
    CFD_BCUDA(b, cudaStreamSynchronize(b->stream));
    return rc ? rc : rc2;
}

} // extern "C"

// ------------------------------------------------------------------ discrete adjoint

namespace {

int adjoint_supported(cfd_handle *h)
{
    const bool fam_ok = h->fam == cfd::FAM_WCNS5 || h->fam == cfd::FAM_TENOZ || h->fam == cfd::FAM_TENOCONG;
    if (h->dim != 2 || !fam_ok || h->cfg.flux_method != CFD_FLUX_ROE || h->cfg.precision != CFD_PREC_FP64 ||
        h->cfg.source_type != 0 || h->cfg.diff_method != CFD_DIFF_MND6 || h->cfg.positivity != 0)
        return fail(h, CFD_ERR_UNSUPPORTED,
                    "the adjoint covers 2D WCNS5 / TENO-Z / TENO-Cong + Roe + MND6, FP64, without source terms "
                    "or the positivity option");
    for (int d = 0; d < 2; d++)
        for (int sd = 0; sd < 2; sd++)
            if (h->cfg.bc[d][sd] != CFD_BND_PERIODIC_WRAP)
                return fail(h, CFD_ERR_UNSUPPORTED, "the adjoint needs periodic (CFD_BND_PERIODIC_WRAP) boundaries");
    return CFD_OK;
}

int adjoint_buffers(cfd_handle *h)
{
    const size_t state = sizeof(double) * h->ncell * h->nv;
    for (int k = 0; k < 4; k++) {
        if (h->adj_buf[k]) continue;
        cudaError_t e = cudaMalloc(&h->adj_buf[k], k == 3 ? 12 * state + sizeof(double) * h->ncell : state);
        if (e != cudaSuccess) {
            h->adj_buf[k] = nullptr;
            return fail(h, CFD_ERR_NOMEM, "adjoint work buffers");
        }
    }
    return CFD_OK;
}

// g = (dR/dU)^T mu at the state U (both directions) into o
int rhs_vjp(cfd_handle *h, const double *U, const double *mu, const cfd::adj::VjpOut &o)
{
    const int nx = h->cfg.n[0], ny = h->cfg.n[1];
    cudaError_t e = cfd::adj::launch_rhs_vjp(h->fam, h->icst, U, mu, o, h->adj_buf[3], nx, ny, h->cfg.h[0],
                                             h->cfg.h[1], h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "adjoint sweep");
    h->launches += 3;
    return CFD_OK;
}

// out = a x + b g + e z (x, z: nullptr when absent)
cfd::adj::VjpOut vjp_out(double *out, const double *x = nullptr, double a = 0.0, double b = 1.0,
                         const double *z = nullptr, double e = 0.0)
{
    return cfd::adj::VjpOut{out, x, a, b, z, e, nullptr, nullptr, 0.0, 0.0};
}

void adjoint_release(std::vector<double *> &v)
{
    for (double *b : v) cudaFree(b);
    v.clear();
}

int adjoint_states(cfd_handle *h, std::vector<double *> &v, size_t count)
{
    const size_t state = sizeof(double) * h->ncell * h->nv;
    while (v.size() < count) {
        double *b = nullptr;
        if (cudaMalloc(&b, state) != cudaSuccess) return fail(h, CFD_ERR_NOMEM, "adjoint checkpoints");
        v.push_back(b);
    }
    return CFD_OK;
}

// one SSP-RK3 step with frozen dt from S[0], keeping its stage states in S[1], S[2]; out = U^(n+1)
int adjoint_step(cfd_handle *h, double dt, double *const *S, double *out)
{
    int rc;
    if ((rc = rk_stage(h, 1, S[0], S[0], S[1], 1.0, dt, 0.0, 0.0, false))) return rc;
    if ((rc = rk_stage(h, 2, S[1], S[0], S[2], 0.75, 0.25 * dt, 0.25, 0.0, false))) return rc;
    return rk_stage(h, 3, S[2], S[0], out, 1.0 / 3.0, 2.0 / 3.0 * dt, 2.0 / 3.0, 0.0, false);
}

} // namespace

int cfd_rhs_vjp(cfd_handle *h, const double *mu_aos, double *lam_aos)
{
    if (!h || !mu_aos || !lam_aos) return CFD_ERR_CONFIG;
    int rc;
    if ((rc = adjoint_supported(h)) || (rc = adjoint_buffers(h))) return rc;
    CFD_CUDA(h, cudaMemcpyAsync(h->stage, mu_aos, sizeof(double) * h->ncell * h->nv, cudaMemcpyHostToDevice,
                                h->stream));
    if ((rc = launch_aos_to_soa(h, h->stage, h->adj_buf[0]))) return rc;
    if ((rc = rhs_vjp(h, h->u[h->cur], h->adj_buf[0], vjp_out(h->adj_buf[1])))) return rc;
    if ((rc = launch_soa_to_aos(h, h->adj_buf[1], h->stage, 0))) return rc;
    CFD_CUDA(h, cudaMemcpyAsync(lam_aos, h->stage, sizeof(double) * h->ncell * h->nv, cudaMemcpyDeviceToHost,
                                h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    return CFD_OK;
}

int cfd_adjoint_record(cfd_handle *h, double dt, int nsteps, int ckpt_every)
{
    if (!h || nsteps < 1 || ckpt_every < 1 || !(dt > 0.0)) return CFD_ERR_CONFIG;
    int rc;
    if ((rc = adjoint_supported(h)) || (rc = sync_bc(h))) return rc;
    const size_t nck = (size_t)((nsteps + ckpt_every - 1) / ckpt_every);
    // checkpoint buffers persist across records (they only grow): no
    // cudaFree / cudaMalloc pair on the timed path of repeated gradients
    if ((rc = adjoint_states(h, h->adj_ckpt, nck))) return rc;
    const size_t state = sizeof(double) * h->ncell * h->nv;
    const int K = ckpt_every;
    h->adj_last_valid = false;
    if ((rc = adjoint_states(h, h->adj_stage, 3 * (size_t)K + 1))) return rc;
    CFD_CUDA(h, cudaMemsetAsync(h->err, 0, sizeof(unsigned), h->stream));
    if (h->adj_graph_K != ckpt_every || h->adj_graph_dt != dt) {
        drop_graphs(h);
        h->adj_graph_K = ckpt_every;
        h->adj_graph_dt = dt;
    }
    // `cnt` steps from state slot `slot` (buffers by role)
    auto steps_from = [&](int slot, int cnt) -> int {
        for (int j = 0; j < cnt; j++) {
            const int c = (slot + j) % 3;
            double *S[3] = {h->u[c], h->u[(c + 1) % 3], h->u[(c + 2) % 3]};
            int r = adjoint_step(h, dt, S, S[1]);
            if (r) return r;
        }
        return CFD_OK;
    };
    // the last segment's steps with every stage state kept in adj_stage
    // (the same launches as the reverse pass's recomputation of it)
    auto keep_stages = [&](int cnt) -> int {
        std::vector<double *> &st = h->adj_stage;
        for (int j = 0; j < cnt; j++) {
            double *S[3] = {st[3 * j], st[3 * j + 1], st[3 * j + 2]};
            int r = adjoint_step(h, dt, S, st[3 * (j + 1)]);
            if (r) return r;
        }
        return CFD_OK;
    };
    for (int s0 = 0; s0 < nsteps; s0 += K) {
        const int cnt = std::min(K, nsteps - s0);
        CFD_CUDA(h, cudaMemcpyAsync(h->adj_ckpt[s0 / K], h->u[h->cur], state, cudaMemcpyDeviceToDevice, h->stream));
        if (s0 + cnt >= nsteps) {  // the last segment
            CFD_CUDA(h, cudaMemcpyAsync(h->adj_stage[0], h->u[h->cur], state, cudaMemcpyDeviceToDevice, h->stream));
            if (cnt == K) {
                if (!h->adj_last_graph && (rc = capture_graph(h, [&] { return keep_stages(K); }, &h->adj_last_graph)))
                    return rc;
                CFD_CUDA(h, cudaGraphLaunch(h->adj_last_graph, h->stream));
                h->launches += 3ULL * h->dim * K;
            } else if ((rc = keep_stages(cnt))) {
                return rc;
            }
            CFD_CUDA(h, cudaMemcpyAsync(h->u[(h->cur + cnt) % 3], h->adj_stage[3 * cnt], state,
                                        cudaMemcpyDeviceToDevice, h->stream));
        } else if (cnt == K) {  // a full segment: one graph per starting slot
            const int slot = h->cur;
            if (!h->adj_rec_graph[slot] &&
                (rc = capture_graph(h, [&] { return steps_from(slot, K); }, &h->adj_rec_graph[slot])))
                return rc;
            CFD_CUDA(h, cudaGraphLaunch(h->adj_rec_graph[slot], h->stream));
            h->launches += 3ULL * h->dim * K;
        } else if ((rc = steps_from(h->cur, cnt))) {
            return rc;
        }
        h->cur = (h->cur + cnt) % 3;
    }
    h->ws_valid = false;
    h->adj_dt = dt;
    h->adj_nsteps = nsteps;
    h->adj_every = ckpt_every;
    unsigned err = 0;
    CFD_CUDA(h, cudaMemcpyAsync(&err, h->err, sizeof(err), cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    rc = check_err(h, err);
    h->adj_last_valid = (rc == CFD_OK);
    return rc;
}

int cfd_run_fixed(cfd_handle *h, double dt, int nsteps, int steps_per_graph)
{
    if (!h || nsteps < 0 || !(dt > 0.0) || steps_per_graph < 1) return CFD_ERR_CONFIG;
    // the stage times stay at 0: refuse boundaries that depend on time
    for (int d = 0; d < h->dim; d++)
        for (const auto *tab : {&h->bc_lo[d], &h->bc_hi[d]})
            for (const BcLine &b : *tab)
                if (b.type == cfd::BND_DOUBLEMACHUP)
                    return fail(h, CFD_ERR_UNSUPPORTED, "cfd_run_fixed: a DoubleMachUp boundary depends on time");
    int rc;
    if ((rc = sync_bc(h))) return rc;
    CFD_CUDA(h, cudaMemsetAsync(h->err, 0, sizeof(unsigned), h->stream));
    // the K-step graphs are those of cfd_adjoint_record (the same steps)
    const int K = steps_per_graph;
    if (h->adj_graph_K != K || h->adj_graph_dt != dt) {
        drop_graphs(h);
        h->adj_graph_K = K;
        h->adj_graph_dt = dt;
    }
    auto steps_from = [&](int slot, int cnt) -> int {
        for (int j = 0; j < cnt; j++) {
            const int c = (slot + j) % 3;
            double *S[3] = {h->u[c], h->u[(c + 1) % 3], h->u[(c + 2) % 3]};
            int r = adjoint_step(h, dt, S, S[1]);
            if (r) return r;
        }
        return CFD_OK;
    };
    for (int s0 = 0; s0 < nsteps; s0 += K) {
        const int cnt = std::min(K, nsteps - s0);
        if (cnt == K) {
            const int slot = h->cur;
            if (!h->adj_rec_graph[slot] &&
                (rc = capture_graph(h, [&] { return steps_from(slot, K); }, &h->adj_rec_graph[slot])))
                return rc;
            CFD_CUDA(h, cudaGraphLaunch(h->adj_rec_graph[slot], h->stream));
            h->launches += 3ULL * h->dim * K;
        } else if ((rc = steps_from(h->cur, cnt))) {
            return rc;
        }
        h->cur = (h->cur + cnt) % 3;
    }
    h->ws_valid = false;
    unsigned err = 0;
    CFD_CUDA(h, cudaMemcpyAsync(&err, h->err, sizeof(err), cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    return check_err(h, err);
}

int cfd_adjoint_reverse(cfd_handle *h, const double *dJ_dUN_aos, double *dJ_dU0_aos)
{
    if (!h || !dJ_dUN_aos || !dJ_dU0_aos) return CFD_ERR_CONFIG;
    if (h->adj_nsteps < 1) return fail(h, CFD_ERR_CONFIG, "cfd_adjoint_reverse needs a cfd_adjoint_record run first");
    int rc;
    if ((rc = adjoint_supported(h)) || (rc = adjoint_buffers(h))) return rc;
    const int K = h->adj_every, N = h->adj_nsteps;
    const double dt = h->adj_dt;
    // the record pass left the last segment's stage states in the first set
    // (once: this pass overwrites that set)
    const bool have_last = h->adj_last_valid;
    h->adj_last_valid = false;
    if ((rc = adjoint_states(h, h->adj_stage, 3 * (size_t)K + 1))) return rc;
    const size_t state = sizeof(double) * h->ncell * h->nv;
    double *lam = h->adj_buf[0], *w = h->adj_buf[1], *w2 = h->adj_buf[2];
    CFD_CUDA(h, cudaMemcpyAsync(h->stage, dJ_dUN_aos, state, cudaMemcpyHostToDevice, h->stream));
    if ((rc = launch_aos_to_soa(h, h->stage, lam))) return rc;
    const int nseg = (N + K - 1) / K;
    // Two sets of stage states: while the reverse sweep of segment s runs on
    // the handle's stream from one set, segment s - 1 is recomputed from its
    // checkpoint into the other on a second stream; events order each set's
    // reuse. Both passes are latency bound on the adjoint's grids, so they
    // share the SMs instead of running one after the other.
    if ((rc = adjoint_states(h, h->adj_stage_b, 3 * (size_t)K + 1))) return rc;
    if (!h->adj_aux) CFD_CUDA(h, cudaStreamCreateWithFlags(&h->adj_aux, cudaStreamNonBlocking));
    for (int k = 0; k < 4; k++)
        if (!h->adj_ev[k]) CFD_CUDA(h, cudaEventCreateWithFlags(&h->adj_ev[k], cudaEventDisableTiming));
    std::vector<double *> *sets[2] = {&h->adj_stage, &h->adj_stage_b};
    // recompute cnt steps from st[0], keeping every stage state
    auto recompute = [&](std::vector<double *> &st, int cnt) -> int {
        int r;
        for (int j = 0; j < cnt; j++) {
            double *S[3] = {st[3 * j], st[3 * j + 1], st[3 * j + 2]};
            if (j + 1 < cnt && (r = adjoint_step(h, dt, S, st[3 * (j + 1)]))) return r;
            if (j + 1 == cnt) {
                // the last step's stages only (its output is not needed)
                if ((r = rk_stage(h, 1, S[0], S[0], S[1], 1.0, dt, 0.0, 0.0, false))) return r;
                if ((r = rk_stage(h, 2, S[1], S[0], S[2], 0.75, 0.25 * dt, 0.25, 0.0, false))) return r;
            }
        }
        return CFD_OK;
    };
    // reverse through the segment's steps:
    //   U1 = U0 - dt R(U0); U2 = 3/4 U0 + 1/4 (U1 - dt R(U1)); U3 = 1/3 U0 + 2/3 (U2 - dt R(U2))
    auto back = [&](std::vector<double *> &st, int cnt) -> int {
        int r;
        for (int j = cnt - 1; j >= 0; j--) {
            double *U0 = st[3 * j], *U1 = st[3 * j + 1], *U2 = st[3 * j + 2];
            // lam2 = 2/3 (lam3 - dt J(U2)^T lam3)
            if ((r = rhs_vjp(h, U2, lam, vjp_out(w, lam, 2.0 / 3.0, -2.0 / 3.0 * dt)))) return r;
            // lam1 = 1/4 (lam2 - dt J(U1)^T lam2); lam = lam3 / 3 + 3/4 lam2
            cfd::adj::VjpOut o1 = vjp_out(w2, w, 0.25, -0.25 * dt);
            o1.out2 = lam; o1.c = 1.0 / 3.0; o1.y = w; o1.d = 0.75;
            if ((r = rhs_vjp(h, U1, w, o1))) return r;
            // lam0 = lam + lam1 - dt J(U0)^T lam1
            if ((r = rhs_vjp(h, U0, w2, vjp_out(lam, lam, 1.0, -dt, w2, 1.0)))) return r;
        }
        return CFD_OK;
    };
    if (h->adj_graph_K != K || h->adj_graph_dt != dt) {
        drop_graphs(h);
        h->adj_graph_K = K;
        h->adj_graph_dt = dt;
    }
    cudaStream_t main_st = h->stream, aux = h->adj_aux;
    // the recomputation stream starts after everything queued so far
    CFD_CUDA(h, cudaEventRecord(h->adj_ev[2], main_st));
    CFD_CUDA(h, cudaStreamWaitEvent(aux, h->adj_ev[2], 0));
    auto launch_recompute = [&](int seg, int set) -> int {
        const int cnt = std::min(K, N - seg * K);
        std::vector<double *> &st = *sets[set];
        h->stream = aux;  // every launch of the recomputation goes to the second stream
        int r = CFD_OK;
        cudaError_t e = cudaMemcpyAsync(st[0], h->adj_ckpt[seg], state, cudaMemcpyDeviceToDevice, aux);
        if (e != cudaSuccess) r = cuda_fail(h, e, "checkpoint copy");
        if (!r && cnt == K) {
            if (!h->adj_recomp_graph[set])
                r = capture_graph(h, [&] { return recompute(st, K); }, &h->adj_recomp_graph[set]);
            if (!r && (e = cudaGraphLaunch(h->adj_recomp_graph[set], aux)) != cudaSuccess) r = cuda_fail(h, e, "graph");
            if (!r) h->launches += 3ULL * h->dim * K;
        } else if (!r) {
            r = recompute(st, cnt);
        }
        h->stream = main_st;
        if (!r && (e = cudaEventRecord(h->adj_ev[set], aux)) != cudaSuccess) r = cuda_fail(h, e, "event");
        return r;
    };
    auto launch_back = [&](int seg, int set) -> int {
        const int cnt = std::min(K, N - seg * K);
        std::vector<double *> &st = *sets[set];
        cudaError_t e = cudaStreamWaitEvent(main_st, h->adj_ev[set], 0);
        if (e != cudaSuccess) return cuda_fail(h, e, "event wait");
        int r;
        if (cnt == K) {
            if (!h->adj_back_graph[set] && (r = capture_graph(h, [&] { return back(st, K); }, &h->adj_back_graph[set])))
                return r;
            if ((e = cudaGraphLaunch(h->adj_back_graph[set], main_st)) != cudaSuccess) return cuda_fail(h, e, "graph");
            h->launches += 9ULL * K;
        } else if ((r = back(st, cnt))) {
            return r;
        }
        if ((e = cudaEventRecord(h->adj_ev[2 + set], main_st)) != cudaSuccess) return cuda_fail(h, e, "event");
        return CFD_OK;
    };
    bool used[2] = {false, false};
    if (have_last) CFD_CUDA(h, cudaEventRecord(h->adj_ev[0], main_st));
    else if ((rc = launch_recompute(nseg - 1, 0))) return rc;
    for (int seg = nseg - 1; seg >= 0; seg--) {
        const int set = (nseg - 1 - seg) & 1, other = set ^ 1;
        if (seg > 0) {
            // the other set is free once the reverse sweep that read it is done
            if (used[other]) CFD_CUDA(h, cudaStreamWaitEvent(aux, h->adj_ev[2 + other], 0));
            if ((rc = launch_recompute(seg - 1, other))) return rc;
        }
        if ((rc = launch_back(seg, set))) return rc;
        used[set] = true;
    }
    if ((rc = launch_soa_to_aos(h, lam, h->stage, 0))) return rc;
    CFD_CUDA(h, cudaMemcpyAsync(dJ_dU0_aos, h->stage, state, cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    return CFD_OK;
}

// ------------------------------------------------------------------ slab decomposition

int cfd_enable_halo(cfd_handle *h, int side, double **buf, long long *count)
{
    if (!h || !buf || !count || (side != 0 && side != 1) || h->dim < 2) return CFD_ERR_CONFIG;
    if (h->ng != kGhost) return fail(h, CFD_ERR_UNSUPPORTED, "slab halos carry 4 rows (MND6 only)");
    const int d = h->dim - 1;
    const long long nl = nlines(h, d);
    const long long n = (long long)h->nv * 4 * nl;
    if (!h->halo[side]) {
        CFD_CUDA(h, cudaMalloc(&h->halo[side], sizeof(double) * n));
        CFD_CUDA(h, cudaMemsetAsync(h->halo[side], 0, sizeof(double) * n, h->stream));
    }
    for (long long lid = 0; lid < nl; lid++) {
        BcLine b;
        std::memset(&b, 0, sizeof(b));
        b.type = cfd::BND_HALO;
        b.i0 = lid;
        b.offset = side;
        b.slot = -1;
        (side == 0 ? h->bc_lo[d] : h->bc_hi[d])[lid] = b;
    }
    h->bc_dirty = true;
    drop_graphs(h);
    *buf = h->halo[side];
    *count = n;
    return CFD_OK;
}

int cfd_stage_state(cfd_handle *h, int stage, double **state)
{
    if (!h || !state || stage < 1 || stage > 3) return CFD_ERR_CONFIG;
    *state = h->u[(h->cur + stage - 1) % 3];
    return CFD_OK;
}

int cfd_rk3_stage(cfd_handle *h, int stage, double dt, double t)
{
    if (!h || stage < 1 || stage > 3) return CFD_ERR_CONFIG;
    int rc = sync_bc(h);
    if (rc) return rc;
    double *U0 = h->u[h->cur], *U1 = h->u[(h->cur + 1) % 3], *U2 = h->u[(h->cur + 2) % 3];
    // stage times follow info->t in RK3_SSP: t, t + dt, (t + dt) - dt/2
    const double t2 = t + dt, t3 = t2 - dt / 2;
    if (stage == 1) {
        CFD_CUDA(h, cudaMemsetAsync(h->err, 0, sizeof(unsigned), h->stream));
        return rk_stage(h, 1, U0, U0, U1, 1.0, dt, 0.0, t, false);
    }
    if (stage == 2) return rk_stage(h, 2, U1, U0, U2, 0.75, 0.25 * dt, 0.25, t2, false);
    CFD_CUDA(h, cudaMemsetAsync(h->red, 0, 4 * sizeof(unsigned long long), h->stream));
    if ((rc = rk_stage(h, 3, U2, U0, U1, 1.0 / 3.0, 2.0 / 3.0 * dt, 2.0 / 3.0, t3, true))) return rc;
    h->cur = (h->cur + 1) % 3;
    h->ws_valid = true;
    unsigned err;
    CFD_CUDA(h, cudaMemcpyAsync(&err, h->err, sizeof(err), cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    return check_err(h, err);
}

int cfd_max_wave_speeds(cfd_handle *h, double *lam)
{
    if (!h || !lam) return CFD_ERR_CONFIG;
    unsigned long long r[4];
    if (!h->ws_valid) {
        int rc = launch_wave_speed(h);
        if (rc) return rc;
    }
    CFD_CUDA(h, cudaMemcpyAsync(r, h->red, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    for (int d = 0; d < 3; d++) {
        double l = 0.0;
        if (d < h->dim) std::memcpy(&l, &r[1 + d], sizeof(double));
        lam[d] = l;
    }
    return CFD_OK;
}

int cfd_loop_begin(cfd_handle *h, double cfl, double t)
{
    if (!h || !(cfl > 0.0)) return CFD_ERR_CONFIG;
    int rc;
    if ((rc = sync_bc(h)) || (rc = ensure_run_buffers(h, 1))) return rc;
    if (!h->ws_valid && (rc = launch_wave_speed(h))) return rc;
    cfd::StepCtl *c = h->ctl_host;
    std::memset(c, 0, sizeof(*c));
    c->t = t;
    c->outputDt = 1e300;  // no output clipping: every step takes dt = CFL / sum_d lambda_d
    c->cfl = cfl;
    c->endStep = 1;
    c->maxSteps = 0x7fffffff;
    CFD_CUDA(h, cudaMemcpyAsync(h->ctl, c, sizeof(*c), cudaMemcpyHostToDevice, h->stream));
    CFD_CUDA(h, cudaMemsetAsync(h->err, 0, sizeof(unsigned), h->stream));
    return CFD_OK;
}

int cfd_reduction_words(cfd_handle *h, unsigned long long **words)
{
    if (!h || !words) return CFD_ERR_CONFIG;
    *words = h->red;
    return CFD_OK;
}

int cfd_loop_step_begin(cfd_handle *h)
{
    if (!h || !h->ctl) return CFD_ERR_CONFIG;
    step_begin_kernel<<<1, 1, 0, h->stream>>>(h->ctl, h->red, h->dim, nullptr);
    CFD_CUDA(h, cudaGetLastError());
    h->launches++;
    return CFD_OK;
}

int cfd_loop_stage(cfd_handle *h, int stage)
{
    if (!h || !h->ctl || stage < 1 || stage > 3) return CFD_ERR_CONFIG;
    double *U0 = h->u[h->cur], *U1 = h->u[(h->cur + 1) % 3], *U2 = h->u[(h->cur + 2) % 3];
    // dt and stage time come from the device step control (the coefficients
    // of the host form, cfd_rk3_stage, with Bdt taken from ctl->bdt[stage])
    if (stage == 1) return rk_stage(h, 1, U0, U0, U1, 1.0, 0.0, 0.0, 0.0, false, h->ctl);
    if (stage == 2) return rk_stage(h, 2, U1, U0, U2, 0.75, 0.0, 0.25, 0.0, false, h->ctl);
    return rk_stage(h, 3, U2, U0, U1, 1.0 / 3.0, 0.0, 2.0 / 3.0, 0.0, true, h->ctl);
}

int cfd_loop_step_end(cfd_handle *h)
{
    if (!h || !h->ctl) return CFD_ERR_CONFIG;
    step_end_kernel<<<1, 1, 0, h->stream>>>(h->ctl, h->red, nullptr);
    CFD_CUDA(h, cudaGetLastError());
    h->launches++;
    h->cur = (h->cur + 1) % 3;
    h->ws_valid = true;  // stage 3 left this handle's wave speeds in the reduction words
    return CFD_OK;
}

int cfd_loop_end(cfd_handle *h, double *t, int *nsteps)
{
    if (!h || !h->ctl) return CFD_ERR_CONFIG;
    CFD_CUDA(h, cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(cfd::StepCtl), cudaMemcpyDeviceToHost, h->stream));
    unsigned err = 0;
    CFD_CUDA(h, cudaMemcpyAsync(&err, h->err, sizeof(err), cudaMemcpyDeviceToHost, h->stream));
    CFD_CUDA(h, cudaStreamSynchronize(h->stream));
    if (t) *t = h->ctl_host->t;
    if (nsteps) *nsteps = h->ctl_host->k;
    return check_err(h, err);
}

// ------------------------------------------------------------------ checkpoint / restart

namespace {

// FNV-1a, 64 bit, over the header and the payload
uint64_t fnv1a(const void *data, size_t n, uint64_t hsh)
{
    const unsigned char *p = static_cast<const unsigned char *>(data);
    for (size_t i = 0; i < n; i++) {
        hsh ^= p[i];
        hsh *= 1099511628211ull;
    }
    return hsh;
}

struct CkptHeader {
    char magic[8];         // "CFDGPUCK"
    uint32_t version;      // 1
    uint32_t dim;
    int64_t n[3];
    uint32_t nvar;
    int32_t inter_method;
    int32_t flux_method;
    int32_t pad;
    double gamma;
    double h[3];
    double t;
    int64_t step;
};
static_assert(sizeof(CkptHeader) == 104, "checkpoint header layout");

} // namespace

int cfd_save_checkpoint(cfd_handle *h, const char *path, double t, long long step)
{
    if (!h || !path) return CFD_ERR_CONFIG;
    const size_t n = (size_t)h->ncell * h->nv;
    std::vector<double> cons(n);
    int rc = cfd_download_cons(h, cons.data());
    if (rc) return rc;
    CkptHeader hd;
    std::memset(&hd, 0, sizeof(hd));
    std::memcpy(hd.magic, "CFDGPUCK", 8);
    hd.version = 1;
    hd.dim = (uint32_t)h->dim;
    for (int d = 0; d < 3; d++) {
        hd.n[d] = h->cfg.n[d];
        hd.h[d] = h->cfg.h[d];
    }
    hd.nvar = (uint32_t)h->nv;
    hd.inter_method = h->cfg.inter_method;
    hd.flux_method = h->cfg.flux_method;
    hd.gamma = h->cfg.gamma;
    hd.t = t;
    hd.step = step;
    uint64_t sum = fnv1a(&hd, sizeof(hd), 14695981039346656037ull);
    sum = fnv1a(cons.data(), n * sizeof(double), sum);
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(h, CFD_ERR_CONFIG, std::string("cannot open ") + path + " for writing");
    bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1 && std::fwrite(cons.data(), sizeof(double), n, f) == n &&
              std::fwrite(&sum, sizeof(sum), 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(h, CFD_ERR_CONFIG, std::string("short write to ") + path);
    return CFD_OK;
}

int cfd_load_checkpoint(cfd_handle *h, const char *path, double *t, long long *step)
{
    if (!h || !path) return CFD_ERR_CONFIG;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(h, CFD_ERR_CONFIG, std::string("cannot open ") + path);
    CkptHeader hd;
    const size_t n = (size_t)h->ncell * h->nv;
    std::vector<double> cons(n);
    uint64_t stored = 0;
    bool ok = std::fread(&hd, sizeof(hd), 1, f) == 1;
    if (ok && (std::memcmp(hd.magic, "CFDGPUCK", 8) != 0 || hd.version != 1)) {
        std::fclose(f);
        return fail(h, CFD_ERR_CONFIG, std::string(path) + " is not a version-1 checkpoint");
    }
    if (ok && (hd.dim != (uint32_t)h->dim || hd.nvar != (uint32_t)h->nv || hd.n[0] != h->cfg.n[0] ||
               hd.n[1] != h->cfg.n[1] || hd.n[2] != h->cfg.n[2])) {
        std::fclose(f);
        return fail(h, CFD_ERR_CONFIG, std::string(path) + " holds a grid of another shape");
    }
    ok = ok && std::fread(cons.data(), sizeof(double), n, f) == n && std::fread(&stored, sizeof(stored), 1, f) == 1;
    std::fclose(f);
    if (!ok) return fail(h, CFD_ERR_CONFIG, std::string(path) + " is truncated");
    uint64_t sum = fnv1a(&hd, sizeof(hd), 14695981039346656037ull);
    sum = fnv1a(cons.data(), n * sizeof(double), sum);
    if (sum != stored) return fail(h, CFD_ERR_CONFIG, std::string(path) + ": checksum mismatch");
    int rc = cfd_upload_cons(h, cons.data());
    if (rc) return rc;
    if (t) *t = hd.t;
    if (step) *step = hd.step;
    return CFD_OK;
}
