// Allocation-free right-hand side: cfd_rhs_noalloc (include/cfdgpu.h).
//
// For callers that must not allocate device memory themselves or let a
// library do it: code running inside another framework's memory pool or
// arena, or a host program that has reserved all device memory up front. They
// pass device buffers for the input state and the output RHS; the only scratch
// this entry point needs, the ghost-cell wiring of every line end, lives in a
// fixed file-scope device array that every GPU loading the library holds until
// the process exits.
//
// Compiled with --fmad=false like api.cu.
#include "cfdgpu.h"
#include "euler_math.cuh"
#include "sweep_dispatch.h"

#include <cstdio>
#include <cstring>
#include <mutex>

namespace cfd {
bool map_inter_method_for(int inter_method, int dim, int *fam, double *c);
int default_seg_len_for(const cfd_config *cfg, int fam, bool strict, int d);
bool config_bc_ok(const cfd_config *cfg, const char **why);
}

namespace {

// Scratch: one BcLine (48 bytes) per line end, x/y/z lines, low then high end.
// 16384 entries = 768 KiB per device, enough for 2D grids up to 4096 x 4096.
constexpr int kMaxLineEnds = CFD_NOALLOC_MAX_LINE_ENDS;
static __device__ __align__(256) cfd::BcLine g_noalloc_bc[kMaxLineEnds];

// Device address of g_noalloc_bc per device, looked up once per device. In
// host code the symbol is only a host-side stand-in and must never be handed
// to a kernel.
constexpr int kMaxDevices = 64;
cfd::BcLine *g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Default ghost wiring of one line end (the rules of cfd_create's tables:
// Initializer::initBnds wiring, PERIODIC_WRAP as a true wrap, DoubleMachUp
// coordinates as OneDBnd::setCoor receives them).
struct WireArgs {
    int dim;
    int n[3];
    long long stride[3];
    int bc[3][2];
    double x0, h;
    long long base_index[3];  // first table entry of each direction (low ends, then high ends)
};

__device__ double cell_coor_dev(const WireArgs &w, long long cell, int idim)
{
    long long idx[3];
    idx[0] = cell % w.n[0];
    idx[1] = (cell / w.n[0]) % w.n[1];
    idx[2] = cell / ((long long)w.n[0] * w.n[1]);
    return w.x0 + (idx[idim] + 0.5) * w.h;
}

__global__ void noalloc_wire_kernel(WireArgs w, cfd::BcLine *tab)
{
    for (int d = 0; d < w.dim; d++) {
        const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
        const long long nl = (long long)w.n[t0] * w.n[t1];
        for (long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x; lid < nl;
             lid += (long long)gridDim.x * blockDim.x) {
            long long a = lid % w.n[t0], bb = lid / w.n[t0];
            long long base = a * w.stride[t0] + bb * w.stride[t1];
            long long last = base + (long long)(w.n[d] - 1) * w.stride[d];
            for (int side = 0; side < 2; side++) {
                cfd::BcLine b;
                b.slot = -1;
                b.pad = 0;
                b.coor_x = 0.0;
                b.dh_y = 0.0;
                int type = w.bc[d][side];
                if (type == CFD_BND_PERIODIC_WRAP) {
                    b.type = cfd::BND_PERIODIC1D;
                    b.i0 = side == 0 ? last : base;
                    b.offset = side == 0 ? -(int)w.stride[d] : (int)w.stride[d];
                } else {
                    b.type = type;
                    b.i0 = side == 0 ? base : last;
                    b.offset = side == 0 ? (int)w.stride[d] : -(int)w.stride[d];
                }
                if (b.type == cfd::BND_DOUBLEMACHUP) {
                    b.coor_x = cell_coor_dev(w, b.i0, 0);
                    b.dh_y = cell_coor_dev(w, b.i0, 1) - cell_coor_dev(w, b.i0 + b.offset, 1);
                }
                tab[w.base_index[d] + side * nl + lid] = b;
            }
        }
    }
}

} // namespace

extern "C" int cfd_rhs_noalloc(const cfd_config *cfg, const double *cons_soa, double *rhs_soa, double t,
                               void *stream)
{
    if (!cfg || !cons_soa || !rhs_soa) return CFD_ERR_CONFIG;
    if (cfg->dim < 1 || cfg->dim > 3) return CFD_ERR_CONFIG;
    if (cfg->n_ghost != 4 || cfg->gamma != 1.4 || cfg->diff_method != CFD_DIFF_MND6 ||
        cfg->precision != CFD_PREC_FP64)
        return CFD_ERR_UNSUPPORTED;
    if (cfg->flux_method != CFD_FLUX_HLLC && cfg->flux_method != CFD_FLUX_ROE) return CFD_ERR_CONFIG;
    if (cfg->positivity != 0 && cfg->positivity != 1) return CFD_ERR_CONFIG;
    if (cfg->source_type != 0 && !(cfg->source_type == 1 && cfg->dim == 2)) return CFD_ERR_UNSUPPORTED;
    for (int d = 0; d < 3; d++) {
        if (d < cfg->dim && (cfg->n[d] < 5 || !(cfg->h[d] > 0.0))) return CFD_ERR_CONFIG;
        if (d >= cfg->dim && cfg->n[d] != 1) return CFD_ERR_CONFIG;
    }
    int fam;
    double icst;
    if (!cfd::map_inter_method_for(cfg->inter_method, cfg->dim, &fam, &icst)) return CFD_ERR_UNSUPPORTED;
    const char *why = nullptr;
    if (!cfd::config_bc_ok(cfg, &why)) {
        fprintf(stderr, "cfd_rhs_noalloc: %s\n", why);
        return CFD_ERR_CONFIG;
    }
    // An error left pending by earlier, unrelated work on this thread is not
    // ours to report or to clear: refuse to queue anything behind it.
    {
        cudaError_t pending = cudaPeekAtLastError();
        if (pending != cudaSuccess) {
            fprintf(stderr, "cfd_rhs_noalloc: an earlier CUDA error is pending (%s); nothing was queued\n",
                    cudaGetErrorString(pending));
            return CFD_ERR_CUDA;
        }
    }

    const long long ncell = (long long)cfg->n[0] * cfg->n[1] * cfg->n[2];
    WireArgs w;
    std::memset(&w, 0, sizeof(w));
    w.dim = cfg->dim;
    w.stride[0] = 1;
    w.stride[1] = cfg->n[0];
    w.stride[2] = (long long)cfg->n[0] * cfg->n[1];
    w.x0 = cfg->x0[0];
    w.h = cfg->h[0];
    long long ends = 0;
    for (int d = 0; d < 3; d++) {
        w.n[d] = cfg->n[d];
        w.bc[d][0] = cfg->bc[d][0];
        w.bc[d][1] = cfg->bc[d][1];
    }
    for (int d = 0; d < cfg->dim; d++) {
        w.base_index[d] = ends;
        ends += 2 * (ncell / cfg->n[d]);
    }
    if (ends > kMaxLineEnds) {
        fprintf(stderr,
                "cfd_rhs_noalloc: the grid has %lld line ends; the allocation-free path holds at most %d "
                "(use cfd_create/cfd_rhs for larger grids)\n",
                ends, kMaxLineEnds);
        return CFD_ERR_CONFIG;
    }

    int old_dev = 0;
    if (cudaGetDevice(&old_dev) != cudaSuccess) return CFD_ERR_CUDA;
    if (cfg->device < 0 || cfg->device >= kMaxDevices) return CFD_ERR_CONFIG;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return CFD_ERR_CUDA;
    int rc = CFD_OK;
    cfd::BcLine *tab = nullptr;
    {
        // one-time set-up per device, with that device current
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_ptr[cfg->device]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_bc);
            if (e != cudaSuccess) {
                fprintf(stderr, "cfd_rhs_noalloc: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
                rc = CFD_ERR_CUDA;
            } else {
                g_scratch_ptr[cfg->device] = (cfd::BcLine *)p;
            }
        }
        tab = g_scratch_ptr[cfg->device];
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (rc == CFD_OK) {
        noalloc_wire_kernel<<<64, 256, 0, st>>>(w, tab);
        if (cudaGetLastError() != cudaSuccess) rc = CFD_ERR_CUDA;
    }
    for (int d = 0; d < cfg->dim && rc == CFD_OK; d++) {
        cfd::SweepParams p;
        std::memset(&p, 0, sizeof(p));
        p.u = cons_soa;
        p.rhs = rhs_soa;
        p.ncell = ncell;
        for (int k = 0; k < 3; k++) {
            p.n[k] = cfg->n[k];
            p.stride[k] = w.stride[k];
            p.hdir[k] = cfg->h[k];
        }
        p.h = cfg->h[d];
        p.mode = cfd::MODE_WRITE;
        p.first = (d == 0);
        p.bc_lo = tab + w.base_index[d];
        p.bc_hi = tab + w.base_index[d] + ncell / cfg->n[d];
        p.bc_vals = nullptr;
        p.t = t;
        p.icst = icst;
        p.icst_k = (fam == cfd::FAM_TENOZ) ? cfd::teno_kappa(icst) : 0.0;
        p.seg_len = cfg->seg_len[d] > 0 ? cfg->seg_len[d] : cfd::default_seg_len_for(cfg, fam, cfg->strict != 0, d);
        p.dm_u = 8.25 * std::cos(M_PI / 6);
        p.dm_v = -8.25 * std::sin(M_PI / 6);
        p.gravity = (cfg->source_type == 1 && d == cfg->dim - 1) ? 1 : 0;
        p.posl = cfg->positivity;
        if (cfd::launch_sweep_any(cfg->strict != 0, cfg->dim + 2, fam, d, cfg->flux_method, p, st) != cudaSuccess)
            rc = CFD_ERR_CUDA;
    }
    cudaSetDevice(old_dev);
    return rc;
}
