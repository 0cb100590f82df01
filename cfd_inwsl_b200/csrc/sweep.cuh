// Fused per-direction line sweep of the zone_FD right-hand side.
//
// Replaces SpDistributor::rhsSolve (zone_FD/src/src/sp_distributor.cpp:3-79)
// for one direction together with Equation::consToPrim (equation.cpp:8-93)
// and OneDBnd::update (oneDBnd.cpp:31-114) for the lines it touches, and
// optionally the RK3 stage combination of BlockSolver::RK3_SSP
// (blockSolver.cpp:58-86) plus the reductions for the log value and the next
// CFL step.
//
// Work decomposition. A CTA owns W neighbouring lines along the sweep axis AX
// and one segment [s_begin, s_end) of them. It marches through the segment in
// chunks of S cells. Per chunk it
//   1. loads the S new cells (cons -> prim on the fly, ghost cells from the
//      line's boundary wiring) into a shared-memory ring of S+8 positions
//      (S+10 with the TRAD6 difference),
//   2. computes the S new face fluxes (one face per thread) into a ring of
//      S+3 faces (S+5); the faces shared with the previous chunk are reused,
//   3. applies the MND6 difference (node fluxes recomputed from the prim ring)
//      or the TRAD6 one, and the epilogue for S cells.
// Face values and face fluxes never leave shared memory, and every cell is
// read from HBM once per sweep plus 8 (10) halo cells per line segment.
//
// Thread layout: along x (AX = 0) consecutive threads take consecutive cells
// of a line; along y/z consecutive threads take neighbouring lines (adjacent
// x), so every global access is coalesced along x in all three sweeps.
#pragma once
#include <cuda_pipeline.h>

#include "euler_math.cuh"
#include "mixed.cuh"
#include "sweep_params.h"

namespace cfd {
namespace CFD_NS {

template <int NV>
__device__ __forceinline__ void load_cons_prim(const double *__restrict__ u, long long ncell, long long cell,
                                               double *pr)
{
    double c[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) c[v] = __ldg(u + v * ncell + cell);
    cons_to_prim<NV>(c, pr);
}

// Ghost cell k (0 = nearest the boundary) of a line end, as OneDBnd::update
// leaves it after Bnds::update (oneDBnd.cpp:31-114).
template <int NV, int NG>
__device__ __forceinline__ void ghost_prim(const SweepParams &p, const BcLine &bl, int k, double tstage, double *pr)
{
    switch (bl.type) {
    case BND_PERIODIC1D:
        load_cons_prim<NV>(p.u, p.ncell, bl.i0 + (long long)k * bl.offset, pr);
        return;
    case BND_SUPERSONICOUTLET:
        load_cons_prim<NV>(p.u, p.ncell, bl.i0, pr);
        return;
    case BND_SYMMETRYX:
    case BND_SYMMETRYY:
    case BND_SYMMETRYZ:
    case BND_SYMMETRY1D: {
        load_cons_prim<NV>(p.u, p.ncell, bl.i0 + (long long)k * bl.offset, pr);
        int neg = (bl.type == BND_SYMMETRYY) ? 2 : (bl.type == BND_SYMMETRYZ) ? 3 : 1;
        if (neg < NV - 1) pr[neg] = -pr[neg];
        if (bl.type == BND_SYMMETRY1D) {
            // SYMMETRY1D writes only the first three values of each ghost cell.
            for (int v = 3; v < NV; v++) pr[v] = (bl.slot >= 0) ? p.bc_vals[((long long)bl.slot * NG + k) * NV + v] : 0.0;
        }
        return;
    }
    case BND_DOUBLEMACHUP: {
        // oneDBnd.cpp:87-108: exact post- or pre-shock state at the stage time.
        // As in the reference, ghost k is placed at y = -dh/2 + k*dh (measured
        // from 0, not from the line end) and x is the edge cell's centre.
        double x = bl.coor_x;
        double y = -bl.dh_y / 2 + k * bl.dh_y;
        double gt = 1.0 / 6.0 + sqrt(3.0) / 3.0 * (1.0 + 20 * tstage);
        if (y > sqrt(3.0) * (x - gt)) {
            pr[0] = 8.0; pr[1] = p.dm_u; pr[2] = p.dm_v; pr[NV - 1] = 116.5;
        } else {
            pr[0] = 1.4; pr[1] = 0; pr[2] = 0; pr[NV - 1] = 1.0;
        }
        if (NV == 5) pr[3] = 0.0;
        return;
    }
    case BND_HALO: {
        // rows of the neighbouring slab, ascending: the low side's nearest
        // ghost is the neighbour's last row, the high side's its first
        const int kk = k > 3 ? 3 : k;  // four halo rows (MND6 only)
        const int r = (bl.offset == 0) ? 3 - kk : kk;
        const double *hb = (bl.offset == 0) ? p.halo_lo : p.halo_hi;
        double c[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) c[v] = hb[((long long)v * 4 + r) * p.halo_nl + bl.i0];
        cons_to_prim<NV>(c, pr);
        return;
    }
    default:
        // DIRICLET and every type whose update() is a no-op keep their static data.
        for (int v = 0; v < NV; v++) pr[v] = (bl.slot >= 0) ? p.bc_vals[((long long)bl.slot * NG + k) * NV + v] : 0.0;
        return;
    }
}

template <int NV>
struct PrimVals {
    double v[NV];
};

// The same out of line, returned by value: boundary ghosts are a few cells
// per line end, and one copy of this code instead of one per cell-loader call
// site keeps the sweep's instruction footprint small.
template <int NV, int NG>
__device__ __noinline__ PrimVals<NV> ghost_prim_ool(const SweepParams &p, const BcLine &bl, int k, double tstage)
{
    PrimVals<NV> r;
    ghost_prim<NV, NG>(p, bl, k, tstage, r.v);
    return r;
}

#ifndef CFD_SWEEP_MINB
#define CFD_SWEEP_MINB 2
#endif
#ifndef CFD_SWEEP_MINB128
#define CFD_SWEEP_MINB128 4  // resident 128-thread CTAs per SM (2D/3D)
#endif

#if defined(CFD_FAST)
constexpr bool kStrictFlavour = false;
#else
constexpr bool kStrictFlavour = true;
#endif

constexpr int pow2_ceil(int x)
{
    int r = 1;
    while (r < x) r <<= 1;
    return r;
}

template <int NV, int AX, int FAM, int FLUX, int S, int W, int PREC = 0, int DIFF = 0>
struct SweepShape {
    static constexpr int NT = S * W;
    // Halo cells per side: MND6 differences faces x_{i-3/2}..x_{i+3/2} (cells
    // i-4..i+4), TRAD6 faces x_{i-5/2}..x_{i+5/2} (cells i-5..i+5). A chunk
    // shares FC = 2 HG - 5 faces with the previous one.
    static constexpr int HG = DIFF ? 5 : 4;
    static constexpr int FC = 2 * HG - 5;
    // ring sizes are powers of two so that ring positions are bit masks
    static constexpr int R = pow2_ceil(S + 2 * HG);  // prim ring positions (S + 2 HG used)
    static constexpr int RF = pow2_ceil(S + FC);     // face ring positions (S + FC used)
    static constexpr int LSP = R | 1;         // odd line strides avoid bank conflicts
    static constexpr int LSF = RF | 1;
    // The 3D mixed y/z sweeps keep no FP64 cons ring: they read the cons as
    // hi + lo from the FP32 split (within 2^-48 of the cons), which leaves room
    // for the cp.async staging below (the x sweep stages less and has room).
    static constexpr bool HL_CS = (PREC == 1 && NV == 5 && AX != 0 && FAM != FAM_RESEARCH);
    static constexpr int SMEM_DOUBLES0 = (HL_CS ? 1 : 2) * NV * W * LSP + NV * W * LSF;
    // mixed form: FP32 hi/lo split of the cons ring (exact FP32 increments)
    static constexpr int SMEM_FLOATS = PREC ? 2 * NV * W * LSP : 0;
    // Resident CTAs per SM the launch bounds ask for: 512 threads per SM in
    // 2D/3D (two CTAs of 256 threads or four of 128), 128 registers a thread;
    // or three 128-thread CTAs (168 registers, fewer spills), which measured
    // faster for the FP64 y sweep (2D), every FP64 3D sweep (the x sweep
    // spilled 880 / 576 bytes per thread at 128 registers in the strict /
    // fast flavour: 3.35 -> 3.23 and 1.90 -> 1.78 ms per 256^3 launch at
    // three CTAs), the FP64 TENO-Z x sweep and the 3D mixed TENO-Z sweeps.
    static constexpr bool THREE = ((FAM == FAM_TENOZ) && (PREC == 0 ? AX == 0 : NV == 5)) ||
                                  (CFD_FP64_3D_YZ16 && PREC == 0 && NV == 5) ||
                                  (CFD_FP64_2D_Y16 && PREC == 0 && NV == 4 && AX == 1);
    // The strict flavour's 3D z sweep (the stage-closing one) measured 7%
    // faster at two CTAs per SM (255 registers) than at three.
    static constexpr bool TWO = kStrictFlavour && PREC == 0 && NV == 5 && AX == 2;
    static constexpr int MINB128 = TWO ? 2 : THREE ? 3 : CFD_SWEEP_MINB128;
    static constexpr int MINB = (NT <= 256) ? (NV >= 4 ? (NT == 128 ? MINB128 : CFD_SWEEP_MINB * (256 / NT))
                                                       : CFD_SWEEP_MINB)
                                            : 1;
    // Asynchronous staging (cp.async) of each thread's global operands: the next
    // chunk's cell and the epilogue's rhs / U^0 / U^k, so that their latency
    // hides behind the face phase. Only where MINB CTAs per SM still fit in the
    // 228 KB of an SM (1 KB of it reserved per CTA).
    // The x sweep of a 2D/3D step is always the first direction (no epilogue
    // operands to stage), so it stages only the next chunk's cells.
    static constexpr int NSTG = (AX == 0 && NV >= 4) ? 1 : 4;
    static constexpr size_t SMEM_STAGE = sizeof(double) * NSTG * NV * NT;
    static constexpr size_t SMEM_LIMIT = (size_t)(MINB > 2 ? 224 / MINB : 112) * 1024;
    // FP64 multi-dimensional sweeps keep each cell's Roe weights (sqrt(rho),
    // sqrt(rho) v, sqrt(rho) H) beside its prim: formed once per cell instead
    // of once for each of the cell's two faces; where the ring fits beside the
    // staging buffers
    static constexpr bool RW = (PREC == 0 && NV >= 4) &&
                               sizeof(double) * (SMEM_DOUBLES0 + NV * W * LSP) + SMEM_STAGE <= SMEM_LIMIT;
    static constexpr int SMEM_DOUBLES = SMEM_DOUBLES0 + (RW ? NV * W * LSP : 0);
    static constexpr size_t SMEM_RINGS = sizeof(double) * SMEM_DOUBLES + sizeof(float) * SMEM_FLOATS;
    static constexpr bool PF = SMEM_RINGS + SMEM_STAGE <= SMEM_LIMIT;
    static constexpr bool PF_EPI = PF && NSTG == 4;
    static constexpr size_t SMEM_BYTES = SMEM_RINGS + (PF ? SMEM_STAGE : 0);
};

template <int NV, int AX, int FAM, int FLUX, int S, int W, int PREC, int DIFF>
__device__ __forceinline__ void sweep_tile(const SweepParams &p, int block_id)
{
    using SH = SweepShape<NV, AX, FAM, FLUX, S, W, PREC, DIFF>;
    constexpr int NT = SH::NT, R = SH::R, RF = SH::RF, LSP = SH::LSP, LSF = SH::LSF;
    constexpr int HG = SH::HG, FC = SH::FC, FO = HG - 3;  // face j sits at face-ring position j - s_begin + FO
    // device-resident loop: the whole launch is a no-op once the loop is done
    if (p.ctl && p.ctl->done) return;
    const double tstage = p.ctl ? p.ctl->tst[p.rk_stage] : p.t;
    const double inv_h = 1.0 / p.h;
    // RN(1/h_d) for the correctly rounded wave-speed quotients of the epilogue
    double inv_hdir[3] = {0.0, 0.0, 0.0};
    if (p.mode == MODE_RK && p.want_reduce)
        for (int d = 0; d < NV - 2; d++) inv_hdir[d] = 1.0 / p.hdir[d];
    // ring positions (R and RF are powers of two; arguments are never negative)
    auto ring = [](int x) { return (int)((unsigned)x & (unsigned)(R - 1)); };
    auto fring = [](int x) { return (int)((unsigned)x & (unsigned)(RF - 1)); };
    const double rkBdt = p.ctl ? p.ctl->bdt[p.rk_stage] : p.rkBdt;
    extern __shared__ double smem[];
    double *sp = smem;                   // [NV][W][LSP] prim
    double *sc = sp + NV * W * LSP;      // [NV][W][LSP] cons re-derived from prim (primToChar prologue); absent with HL_CS
    double *sf = SH::HL_CS ? sc : sc + NV * W * LSP;  // [NV][W][LSF] face flux
    // mixed form: [NV][W][LSP] (hi, lo) = ((float)cons, (float)(cons - hi))
    float2 *shl = reinterpret_cast<float2 *>(sf + NV * W * LSF);
    // FP64 form: [NV][W][LSP] Roe weights of each cell (in place of the mixed form's split)
    double *skw = sf + NV * W * LSF;
    // staging: [0] next chunk's cons, [1] rhs, [2] U^0, [3] U^k; [NV][NT] each
    double *stg = reinterpret_cast<double *>(reinterpret_cast<char *>(smem) + SH::SMEM_RINGS);
    constexpr bool PF = SH::PF, PF_EPI = SH::PF_EPI;

    constexpr int T0 = (AX == 0) ? 1 : 0;  // transverse axis with neighbouring lines in a CTA
    constexpr int T1 = (AX == 2) ? 1 : 2;
    const int nd = p.n[AX];
    const int nt0 = p.n[T0];
    const int nseg = (nd + p.seg_len - 1) / p.seg_len;
    const int nblk0 = (nt0 + W - 1) / W;
    int bid = block_id;
    int seg;
    if (p.seg_outer) {  // segments outermost (partial sweeps along the last dimension)
        const int per = nblk0 * p.n[T1];
        seg = bid / per;
        bid -= seg * per;
    } else {
        seg = bid % nseg;
        bid /= nseg;
    }
    const int a0 = (bid % nblk0) * W;
    const int bb = bid / nblk0;
    const int s_begin = seg * p.seg_len;
    const int s_end = min(s_begin + p.seg_len, nd);

    const int tid = threadIdx.x;
    const int tl = (AX == 0) ? tid / S : tid % W;   // line within the CTA
    const int tp = (AX == 0) ? tid % S : tid / W;   // position within the chunk
    const long long sAX = p.stride[AX];

    auto line_of = [&](int l, bool &ok, long long &base, int &lid) {
        int a = a0 + l;
        ok = a < nt0;
        base = (long long)a * p.stride[T0] + (long long)bb * p.stride[T1];
        lid = a + nt0 * bb;
    };
    // the thread's own line, fixed for the whole tile: held in registers by
    // the mixed form, recomputed where needed by the FP64 form (whose kernels
    // have no registers to spare)
    bool my_ok = false; long long my_base = 0; int my_lid = 0;
    if constexpr (PREC == 1) line_of(tl, my_ok, my_base, my_lid);
    auto own_line = [&](bool &ok, long long &base, int &lid) {
        if constexpr (PREC == 1) {
            ok = my_ok; base = my_base; lid = my_lid;
        } else {
            line_of(tl, ok, base, lid);
        }
    };

    // Stage cell P (global index along AX, may be a ghost) of line l; staged:
    // its cons already sit in stg[0] (interior cells of the thread's own line).
    auto load_pos = [&](int l, int P, bool staged = false) {
        bool ok; long long base; int lid;
        if (PREC == 1 && l == tl) own_line(ok, base, lid);
        else line_of(l, ok, base, lid);
        double pr[NV];
        double cs[NV];
        bool have_cs = false;  // the mixed form takes interior cells' cons as loaded
        if (!ok) {
            pr[0] = 1.0;
            for (int v = 1; v < NV - 1; v++) pr[v] = 0.0;
            pr[NV - 1] = 1.0;
        } else if (P >= 0 && P < nd) {
            if (staged) {
#pragma unroll
                for (int v = 0; v < NV; v++) cs[v] = stg[v * NT + threadIdx.x];
            } else {
#pragma unroll
                for (int v = 0; v < NV; v++) cs[v] = __ldg(p.u + v * p.ncell + base + (long long)P * sAX);
            }
            cons_to_prim<NV>(cs, pr);
            have_cs = (PREC == 1);
        } else if (P < 0) {
            int k = -P - 1;
            const PrimVals<NV> g = ghost_prim_ool<NV, HG>(p, p.bc_lo[lid], k > HG - 1 ? HG - 1 : k, tstage);
#pragma unroll
            for (int v = 0; v < NV; v++) pr[v] = g.v[v];
        } else {
            int k = P - nd;
            const PrimVals<NV> g = ghost_prim_ool<NV, HG>(p, p.bc_hi[lid], k > HG - 1 ? HG - 1 : k, tstage);
#pragma unroll
            for (int v = 0; v < NV; v++) pr[v] = g.v[v];
        }
        if (!have_cs) prim_to_cons<NV>(pr, cs);  // as the reference's primToChar re-derives them
        int slot = ring(P - s_begin + HG);
        if constexpr (SH::RW) {
            double kw[NV];
            EigenBase<NV, AX>::roe_weights(pr, kw);
#pragma unroll
            for (int v = 0; v < NV; v++) skw[(v * W + l) * LSP + slot] = kw[v];
        }
#pragma unroll
        for (int v = 0; v < NV; v++) {
            sp[(v * W + l) * LSP + slot] = pr[v];
            if constexpr (!SH::HL_CS) sc[(v * W + l) * LSP + slot] = cs[v];
            if constexpr (PREC == 1) {
                const float hi = (float)cs[v];
                shl[(v * W + l) * LSP + slot] = make_float2(hi, (float)(cs[v] - (double)hi));
            }
        }
    };

    // Face j lies between cells j-1 and j (x_{j-1/2}); stencil cells j-3..j+2.
    auto face = [&](int l, int j) {
        int slot[6];
#pragma unroll
        for (int m = 0; m < 6; m++) slot[m] = ring(j - 3 + m - s_begin + HG);
        double fl[NV], fr[NV], fx[NV];
        if constexpr (NV == 3) {
            double pr6[6][NV], cs6[6][NV];
#pragma unroll
            for (int m = 0; m < 6; m++) {
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    pr6[m][v] = sp[(v * W + l) * LSP + slot[m]];
                    cs6[m][v] = sc[(v * W + l) * LSP + slot[m]];
                }
            }
            reconstruct_face<NV, AX, FAM>(pr6, cs6, p.icst, p.icst_k, fl, fr);
        } else {
            const double *spl = sp + l * LSP, *scl = sc + l * LSP;
            auto csacc = [&](int m, int v) { return scl[v * W * LSP + slot[m]]; };
            auto pracc = [&](int m, int v) { return spl[v * W * LSP + slot[m]]; };
            if constexpr (PREC == 1 && FAM != FAM_RESEARCH) {
                const float2 *hll = shl + l * LSP;
                // the FP32 hi/lo split of each stencil cell's cons
                auto hlacc = [&](int m, int v) {
                    return hll[v * W * LSP + slot[m]];
                };
                if constexpr (SH::HL_CS) {
                    auto hlcs = [&](int m, int v) {
                        const float2 t = hlacc(m, v);
                        return (double)t.x + (double)t.y;
                    };
                    reconstruct_face_mixed<NV, AX, FAM>(hlcs, pracc, hlacc, p.icst, p.icst_k, fl, fr);
                } else {
                    reconstruct_face_mixed<NV, AX, FAM>(csacc, pracc, hlacc, p.icst, p.icst_k, fl, fr);
                }
            } else if constexpr (SH::RW) {
                const double *kwl = skw + l * LSP;
                double kl[NV], kr[NV];
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    kl[v] = kwl[v * W * LSP + slot[2]];
                    kr[v] = kwl[v * W * LSP + slot[3]];
                }
                const EigenBase<NV, AX> eb(kl, kr);
                reconstruct_face_stream<NV, AX, FAM>(eb, csacc, pracc, p.icst, p.icst_k, fl, fr, p.posl);
            } else {
                reconstruct_face_stream<NV, AX, FAM>(csacc, pracc, p.icst, p.icst_k, fl, fr, p.posl);
            }
        }
        if constexpr (PREC == 1 && FLUX == FLUX_ROE && NV >= 4) roe_md_mixed<NV, AX>(fl, fr, fx);
        else if constexpr (PREC == 1 && FLUX == FLUX_HLLC && NV >= 4) hllc_md_mixed<NV, AX>(fl, fr, fx);
        else riemann<NV, AX, FLUX>(fl, fr, fx);
        int fslot = fring(j - s_begin + FO);
#pragma unroll
        for (int v = 0; v < NV; v++) sf[(v * W + l) * LSF + fslot] = fx[v];
    };

    // prologue: cells s_begin-HG .. s_begin+HG-1
    for (int idx = tid; idx < 2 * HG * W; idx += NT) {
        int l = (AX == 0) ? idx / (2 * HG) : idx % W;
        int q = (AX == 0) ? idx % (2 * HG) : idx / W;
        load_pos(l, s_begin - HG + q);
    }

    double red_rho = 0.0, red_lam[3] = {0.0, 0.0, 0.0};
    unsigned err = 0;

    // cp.async of this thread's interior cell at position P into stg[0]
    auto prefetch_cell = [&](int P) {
        bool ok; long long base; int lid;
        own_line(ok, base, lid);
        if (ok && P >= 0 && P < nd) {
            const long long cell = base + (long long)P * sAX;
#pragma unroll
            for (int v = 0; v < NV; v++) __pipeline_memcpy_async(stg + v * NT + tid, p.u + v * p.ncell + cell, 8);
        }
        __pipeline_commit();
    };
    // cp.async of the epilogue operands of this thread's cell i
    const bool need_rhs = PF_EPI && !p.first, need_u0 = PF_EPI && p.mode == MODE_RK,
               need_u = PF_EPI && p.mode == MODE_RK && p.rk_stage != 1;
    auto prefetch_epilogue = [&](int i) {
        bool ok; long long base; int lid;
        own_line(ok, base, lid);
        if (ok && i < s_end) {
            const long long cell = base + (long long)i * sAX;
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const long long gi = v * p.ncell + cell;
                if (need_rhs) __pipeline_memcpy_async(stg + (1 * NV + v) * NT + tid, p.rhs + gi, 8);
                if (need_u0) __pipeline_memcpy_async(stg + (2 * NV + v) * NT + tid, p.u0 + gi, 8);
                if (need_u) __pipeline_memcpy_async(stg + (3 * NV + v) * NT + tid, p.u + gi, 8);
            }
        }
        __pipeline_commit();
    };
    if constexpr (PF) prefetch_cell(s_begin + HG + tp);

    for (int c0 = s_begin; c0 < s_end; c0 += S) {
        if constexpr (PF) {
            __pipeline_wait_prior(0);
            load_pos(tl, c0 + HG + tp, true);
            prefetch_epilogue(c0 + tp);
            prefetch_cell(c0 + S + HG + tp);  // an empty group past the segment
        } else {
            load_pos(tl, c0 + HG + tp);
        }
        __syncthreads();
        {
            // the chunk's S new faces per line, and before the segment's first
            // chunk also the FC faces ahead of them, from one call site (the
            // face code is emitted once)
            const int nface = (c0 == s_begin) ? NT + FC * W : NT;
            for (int idx = tid; idx < nface; idx += NT) {
                int l, j;
                if (idx < NT) {
                    l = tl;
                    j = c0 + HG - 2 + tp;
                } else {
                    const int e = idx - NT;
                    l = (AX == 0) ? e / FC : e % W;
                    j = s_begin - FO + ((AX == 0) ? e % FC : e / W);
                }
                face(l, j);
            }
        }
        __syncthreads();

        const int i = c0 + tp;
        bool ok; long long base; int lid;
        own_line(ok, base, lid);
        if constexpr (PF) __pipeline_wait_prior(1);  // the epilogue operands; the next cell may still fly
        if (ok && i < s_end) {
            double fnm[NV], fnp[NV];
            if constexpr (DIFF == 0) {  // node fluxes of cells i-1 and i+1 (SolvePointSolver, nl = nr = 1)
                double pm[NV], pp[NV];
                int sm = ring(i - 1 - s_begin + HG), spp = ring(i + 1 - s_begin + HG);
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    pm[v] = sp[(v * W + tl) * LSP + sm];
                    pp[v] = sp[(v * W + tl) * LSP + spp];
                }
                node_flux<NV, AX>(pm, fnm);
                node_flux<NV, AX>(pp, fnp);
            }
            // faces j = i-(FC-1)/2 .. i+(FC+1)/2, face j being x_{j-1/2}
            int fs[FC + 1];
#pragma unroll
            for (int m = 0; m <= FC; m++) fs[m] = fring(i - (FC - 1) / 2 + m - s_begin + FO);
            const long long cell = base + (long long)i * sAX;
            // MND6 differences of the NV variables (strict: the NV quotients by
            // h formed together, one branch for the group)
            double dd[NV];
            if constexpr (DIFF == 0) {
#if defined(CFD_FAST)
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const double *fv = sf + (v * W + tl) * LSF;
                    dd[v] = mnd6(fnm[v], fnp[v], fv[fs[0]], fv[fs[1]], fv[fs[2]], fv[fs[3]], p.h, inv_h);
                }
#else
                double num[NV], hh[NV], ihh[NV];
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const double *fv = sf + (v * W + tl) * LSF;
                    num[v] = mnd6_num(fnm[v], fnp[v], fv[fs[0]], fv[fs[1]], fv[fs[2]], fv[fs[3]]);
                    hh[v] = p.h;
                    ihh[v] = inv_h;
                }
                divs_rn<NV>(num, hh, ihh, dd);
#endif
            }
            double uo[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const double *fv = sf + (v * W + tl) * LSF;
                double d;
                if constexpr (DIFF == 0) d = dd[v];
                else d = trad6(fv[fs[0]], fv[fs[1]], fv[fs[2]], fv[fs[3]], fv[fs[4]], fv[fs[5]], p.h, inv_h);
                const long long gi = v * p.ncell + cell;
                const double *sv = stg + v * NT + tid;
                double r = p.first ? (0.0 + d) : ((PF_EPI ? sv[1 * NV * NT] : p.rhs[gi]) + d);
                if constexpr (NV == 4) {
                    // SourceTerm::calGravitySource (sourceTerm.cpp:3-20) on the
                    // stage's prim: rhs(rho v) -= rho, rhs(rho E) -= rho v
                    if (p.gravity) {
                        const int sc0 = ring(i - s_begin + HG);
                        const double rho = sp[(0 * W + tl) * LSP + sc0];
                        if (v == 2) r -= rho;
                        if (v == 3) r -= rho * sp[(2 * W + tl) * LSP + sc0];
                    }
                }
                if (p.mode != MODE_RK) {
                    p.rhs[gi] = r;
                } else {
                    if (v == 0 && p.want_reduce) red_rho = fmax(red_rho, fabs(r));
                    double o;
                    const double u0v = PF_EPI ? sv[2 * NV * NT] : p.u0[gi];
                    if (p.rk_stage == 1) {
                        o = u0v - rkBdt * r;
                    } else {
                        o = p.rkA * u0v - rkBdt * r + p.rkC * (PF_EPI ? sv[3 * NV * NT] : p.u[gi]);
                    }
                    uo[v] = o;
                    p.u_out[gi] = o;
                }
            }
            if (p.mode == MODE_RK) {
                bool fin = true;
#pragma unroll
                for (int v = 0; v < NV; v++) fin = fin && isfinite(uo[v]);
                if (!fin) err |= ERR_NONFINITE;
                if (p.want_reduce) {
                    double pr[NV];
                    cons_to_prim<NV>(uo, pr);
                    if (!(pr[0] > 0.0) || !(pr[NV - 1] > 0.0)) err |= ERR_NEGATIVE;
                    double cs = sqrt(kGamma * pr[NV - 1] / pr[0]);
#pragma unroll
                    for (int d = 0; d < NV - 2; d++)
                        red_lam[d] = fmax(red_lam[d], div_rn(cs + fabs(pr[1 + d]), p.hdir[d], inv_hdir[d]));
                }
            }
        }
        __syncthreads();
    }

    if (p.mode == MODE_RK) {
        if (err) atomicOr(p.err, err);
        if (p.want_reduce) block_max_reduce<NT, 4>(red_rho, red_lam, p.red);
    }
}

template <int NV, int AX, int FAM, int FLUX, int S, int W, int PREC, int DIFF>
__global__ void __launch_bounds__(S *W, (SweepShape<NV, AX, FAM, FLUX, S, W, PREC, DIFF>::MINB))
    sweep_kernel(const __grid_constant__ SweepParams p)
{
    sweep_tile<NV, AX, FAM, FLUX, S, W, PREC, DIFF>(p, (int)(p.tile0 + blockIdx.x));
}

// Number of CTA tiles one case's sweep along AX needs.
template <int AX, int W>
__host__ __device__ inline long long sweep_tiles(const SweepParams &p)
{
    constexpr int T0 = (AX == 0) ? 1 : 0;
    constexpr int T1 = (AX == 2) ? 1 : 2;
    long long nseg = (p.n[AX] + p.seg_len - 1) / p.seg_len;
    return (long long)((p.n[T0] + W - 1) / W) * p.n[T1] * nseg;
}

// Persistent sweep over many independent cases: the tiles of all cases form
// one work list (tile_start[c] = first tile of case c, prefix sums); each CTA
// walks the list with a grid stride, copies its case's parameter block to
// shared memory and runs the same tile code as sweep_kernel. Cases whose
// device loop is done are skipped tile by tile.
template <int NV, int AX, int FAM, int FLUX, int S, int W, int PREC>
__global__ void __launch_bounds__(S *W, (SweepShape<NV, AX, FAM, FLUX, S, W, PREC>::MINB))
    sweep_batched_kernel(const SweepParams *__restrict__ cases, const long long *__restrict__ tile_start, int ncases)
{
    __shared__ SweepParams sp;
    __shared__ int s_case;
    const long long total = tile_start[ncases];
    for (long long item = blockIdx.x; item < total; item += gridDim.x) {
        __syncthreads();  // the previous tile is done with sp
        if (threadIdx.x == 0) {
            int lo = 0, hi = ncases - 1;  // last case with tile_start <= item
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if (tile_start[mid] <= item) lo = mid; else hi = mid - 1;
            }
            s_case = lo;
        }
        __syncthreads();
        const int c = s_case;
        {
            const int words = (int)(sizeof(SweepParams) / sizeof(int));
            const int *src = reinterpret_cast<const int *>(cases + c);
            int *dst = reinterpret_cast<int *>(&sp);
            for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
        }
        __syncthreads();
        sweep_tile<NV, AX, FAM, FLUX, S, W, PREC, 0>(sp, (int)(item - tile_start[c]));
    }
}

template <int NV, int AX, int FAM, int FLUX, int S, int W, int PREC, int DIFF>
static cudaError_t launch_sweep_shape_p(const SweepParams &p, cudaStream_t st)
{
    using SH = SweepShape<NV, AX, FAM, FLUX, S, W, PREC, DIFF>;
    auto kern = sweep_kernel<NV, AX, FAM, FLUX, S, W, PREC, DIFF>;
    // the dynamic shared-memory opt-in is per device
    static bool attr_set[64] = {};
    int dev = 0;
    cudaError_t e0 = cudaGetDevice(&dev);
    if (e0 != cudaSuccess) return e0;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SH::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_set[dev] = true;
    }
    constexpr int T0 = (AX == 0) ? 1 : 0;
    constexpr int T1 = (AX == 2) ? 1 : 2;
    long long nseg = (p.n[AX] + p.seg_len - 1) / p.seg_len;
    const long long nblk0 = (p.n[T0] + W - 1) / W;
    long long nblk = nblk0 * p.n[T1] * nseg;
    if (nblk > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    SweepParams q = p;
    q.tile0 = 0;
    if (p.part_lo < p.part_hi) {
        // the tiles covering [part_lo, part_hi) of the last dimension L
        const int L = (p.n[2] > 1) ? 2 : 1;
        if (AX == L) {  // whole segments, segments outermost
            if (!p.seg_outer) return cudaErrorInvalidValue;
            const long long s0 = p.part_lo / p.seg_len, s1 = (p.part_hi + p.seg_len - 1) / p.seg_len;
            q.tile0 = s0 * nblk0 * p.n[T1];
            nblk = (s1 - s0) * nblk0 * p.n[T1];
        } else if (T0 == L) {  // lines of L in blocks of W (2D)
            if (p.part_lo % W) return cudaErrorInvalidValue;
            const long long b0 = p.part_lo / W, b1 = (p.part_hi + W - 1) / W;
            q.tile0 = b0 * nseg;
            nblk = (b1 - b0) * nseg;
        } else {  // planes of L (3D)
            q.tile0 = (long long)p.part_lo * nblk0 * nseg;
            nblk = (long long)(p.part_hi - p.part_lo) * nblk0 * nseg;
        }
    } else if (p.seg_outer) {
        return cudaErrorInvalidValue;
    }
    if (nblk <= 0) return cudaSuccess;
    sweep_kernel<NV, AX, FAM, FLUX, S, W, PREC, DIFF><<<(unsigned)nblk, SH::NT, SH::SMEM_BYTES, st>>>(q);
    return cudaGetLastError();
}

template <int NV, int AX, int FAM, int FLUX, int S, int W, int PREC>
static cudaError_t launch_batched_shape_p(const BatchSweep &b, cudaStream_t st)
{
    using SH = SweepShape<NV, AX, FAM, FLUX, S, W, PREC>;
    auto kern = sweep_batched_kernel<NV, AX, FAM, FLUX, S, W, PREC>;
    static bool attr_set[64] = {};
    static int blocks_per_sm[64] = {};
    int dev = 0;
    cudaError_t e0 = cudaGetDevice(&dev);
    if (e0 != cudaSuccess) return e0;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SH::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm[dev], kern, SH::NT, SH::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        if (blocks_per_sm[dev] < 1) blocks_per_sm[dev] = 1;
        attr_set[dev] = true;
    }
    long long grid = (long long)b.num_sms * (b.one_cta ? 1 : blocks_per_sm[dev]);
    if (b.total_tiles < grid) grid = b.total_tiles;
    if (grid <= 0) return cudaSuccess;
    sweep_batched_kernel<NV, AX, FAM, FLUX, S, W, PREC>
        <<<(unsigned)grid, SH::NT, SH::SMEM_BYTES, st>>>(b.cases, b.tile_start, b.ncases);
    return cudaGetLastError();
}

template <int NV, int AX, int FAM, int FLUX, int S, int W>
static cudaError_t launch_batched_shape(const BatchSweep &b, cudaStream_t st)
{
    if (b.prec == 0) return launch_batched_shape_p<NV, AX, FAM, FLUX, S, W, 0>(b, st);
#if defined(CFD_FAST)
    if constexpr (NV >= 4 && FAM != FAM_RESEARCH) return launch_batched_shape_p<NV, AX, FAM, FLUX, S, W, 1>(b, st);
#endif
    return cudaErrorInvalidValue;
}

// FP64 or, in the fast flavour of the multi-dimensional kernels, mixed; the
// TRAD6 difference in FP64 only.
template <int NV, int AX, int FAM, int FLUX, int S, int W>
static cudaError_t launch_sweep_shape(const SweepParams &p, cudaStream_t st)
{
    if (p.diff == DIFF_TRAD6) return p.prec == 0 ? launch_sweep_shape_p<NV, AX, FAM, FLUX, S, W, 0, 1>(p, st)
                                                 : cudaErrorInvalidValue;
    if (p.prec == 0) return launch_sweep_shape_p<NV, AX, FAM, FLUX, S, W, 0, 0>(p, st);
#if defined(CFD_FAST)
    if constexpr (NV >= 4 && FAM != FAM_RESEARCH) return launch_sweep_shape_p<NV, AX, FAM, FLUX, S, W, 1, 0>(p, st);
#endif
    return cudaErrorInvalidValue;
}

// Tile shapes (sweep_params.h): kXSn x kXWn along x in 3D and for 2D FP64,
// kXS x kXW along x for the 2D mixed form; kYSm x kYWm along y and z for the
// single-grid sweeps; kXS x kXW and kYS x kYW for the TRAD6 difference and the
// batched kernel's default; k1S x k1W in 1D.
template <int NV, int FAM>
cudaError_t launch_sweep(int ax, int flux, const SweepParams &p, cudaStream_t st)
{
    if constexpr (NV == 3) {
        if (ax != 0) return cudaErrorInvalidValue;
        return flux == FLUX_HLLC ? launch_sweep_shape<3, 0, FAM, FLUX_HLLC, k1S, k1W>(p, st)
                                 : launch_sweep_shape<3, 0, FAM, FLUX_ROE, k1S, k1W>(p, st);
    } else {
        if (ax == 0) {
            // 16-cell chunks of 8 lines: faster in 3D (both forms) and for 2D FP64
            if (p.diff != DIFF_TRAD6 && (NV == 5 || p.prec == 0))
                return flux == FLUX_HLLC ? launch_sweep_shape<NV, 0, FAM, FLUX_HLLC, kXSn, kXWn>(p, st)
                                         : launch_sweep_shape<NV, 0, FAM, FLUX_ROE, kXSn, kXWn>(p, st);
            return flux == FLUX_HLLC ? launch_sweep_shape<NV, 0, FAM, FLUX_HLLC, kXS, kXW>(p, st)
                                     : launch_sweep_shape<NV, 0, FAM, FLUX_ROE, kXS, kXW>(p, st);
        }
        if (ax == 1) {
#if defined(CFD_FAST)
            if constexpr (FAM != FAM_RESEARCH) {
                if (p.prec == 1 && p.diff != DIFF_TRAD6)
                    return flux == FLUX_HLLC ? launch_sweep_shape_p<NV, 1, FAM, FLUX_HLLC, kYSm, kYWm, 1, 0>(p, st)
                                             : launch_sweep_shape_p<NV, 1, FAM, FLUX_ROE, kYSm, kYWm, 1, 0>(p, st);
            }
#endif
            if constexpr ((NV == 5 && CFD_FP64_3D_YZ16) || (NV == 4 && CFD_FP64_2D_Y16)) {
                if (p.prec == 0 && p.diff != DIFF_TRAD6)
                    return flux == FLUX_HLLC ? launch_sweep_shape_p<NV, 1, FAM, FLUX_HLLC, kYSm, kYWm, 0, 0>(p, st)
                                             : launch_sweep_shape_p<NV, 1, FAM, FLUX_ROE, kYSm, kYWm, 0, 0>(p, st);
            }
            return flux == FLUX_HLLC ? launch_sweep_shape<NV, 1, FAM, FLUX_HLLC, kYS, kYW>(p, st)
                                     : launch_sweep_shape<NV, 1, FAM, FLUX_ROE, kYS, kYW>(p, st);
        }
        if constexpr (NV == 5) {
            if (ax == 2) {
#if defined(CFD_FAST)
                if constexpr (FAM != FAM_RESEARCH && CFD_MIXED_Z16) {
                    if (p.prec == 1 && p.diff != DIFF_TRAD6)
                        return flux == FLUX_HLLC
                                   ? launch_sweep_shape_p<NV, 2, FAM, FLUX_HLLC, kYSm, kYWm, 1, 0>(p, st)
                                   : launch_sweep_shape_p<NV, 2, FAM, FLUX_ROE, kYSm, kYWm, 1, 0>(p, st);
                }
#endif
                if constexpr (CFD_FP64_3D_YZ16) {
                    if (p.prec == 0 && p.diff != DIFF_TRAD6)
                        return flux == FLUX_HLLC
                                   ? launch_sweep_shape_p<NV, 2, FAM, FLUX_HLLC, kYSm, kYWm, 0, 0>(p, st)
                                   : launch_sweep_shape_p<NV, 2, FAM, FLUX_ROE, kYSm, kYWm, 0, 0>(p, st);
                }
                return flux == FLUX_HLLC ? launch_sweep_shape<NV, 2, FAM, FLUX_HLLC, kYS, kYW>(p, st)
                                         : launch_sweep_shape<NV, 2, FAM, FLUX_ROE, kYS, kYW>(p, st);
            }
        }
        return cudaErrorInvalidValue;
    }
}

// Persistent batched sweep (1D, 2D and 3D; the tile shapes of launch_sweep or,
// for 2D/3D FP64 with b.shape = 1, the alternative shapes).
template <int NV, int FAM>
cudaError_t launch_sweep_batched(int ax, int flux, const BatchSweep &b, cudaStream_t st)
{
    if constexpr (NV == 3) {
        if (ax != 0) return cudaErrorInvalidValue;
        return flux == FLUX_HLLC ? launch_batched_shape<3, 0, FAM, FLUX_HLLC, k1S, k1W>(b, st)
                                 : launch_batched_shape<3, 0, FAM, FLUX_ROE, k1S, k1W>(b, st);
    } else {
        if (b.shape == 1) {
            if (b.prec != 0) return cudaErrorInvalidValue;
            if (ax == 0)
                return flux == FLUX_HLLC ? launch_batched_shape_p<NV, 0, FAM, FLUX_HLLC, kXS2, kXW2, 0>(b, st)
                                         : launch_batched_shape_p<NV, 0, FAM, FLUX_ROE, kXS2, kXW2, 0>(b, st);
            if (ax == 1)
                return flux == FLUX_HLLC ? launch_batched_shape_p<NV, 1, FAM, FLUX_HLLC, kYS2, kYW2, 0>(b, st)
                                         : launch_batched_shape_p<NV, 1, FAM, FLUX_ROE, kYS2, kYW2, 0>(b, st);
            if constexpr (NV == 5) {
                if (ax == 2)
                    return flux == FLUX_HLLC ? launch_batched_shape_p<NV, 2, FAM, FLUX_HLLC, kYS2, kYW2, 0>(b, st)
                                             : launch_batched_shape_p<NV, 2, FAM, FLUX_ROE, kYS2, kYW2, 0>(b, st);
            }
            return cudaErrorInvalidValue;
        }
        if (ax == 0)
            return flux == FLUX_HLLC ? launch_batched_shape<NV, 0, FAM, FLUX_HLLC, kXS, kXW>(b, st)
                                     : launch_batched_shape<NV, 0, FAM, FLUX_ROE, kXS, kXW>(b, st);
        if (ax == 1)
            return flux == FLUX_HLLC ? launch_batched_shape<NV, 1, FAM, FLUX_HLLC, kYS, kYW>(b, st)
                                     : launch_batched_shape<NV, 1, FAM, FLUX_ROE, kYS, kYW>(b, st);
        if constexpr (NV == 5) {
            if (ax == 2)
                return flux == FLUX_HLLC ? launch_batched_shape<NV, 2, FAM, FLUX_HLLC, kYS, kYW>(b, st)
                                         : launch_batched_shape<NV, 2, FAM, FLUX_ROE, kYS, kYW>(b, st);
        }
        return cudaErrorInvalidValue;
    }
}

} // namespace CFD_NS
} // namespace cfd

namespace cfd {
namespace CFD_NS {

// The RK stage combination of the last sweep's epilogue, applied by itself to
// a complete RHS in p.rhs (the last sweep having run with MODE_WRITE):
// U_out = (A U0 - Bdt R) + C U_k (stage 1: U0 - dt R) with the epilogue's
// non-finite check. Compiled in the flavour's own unit, so it rounds the
// expression as the fused epilogue does. No reductions: it serves stage 1.
template <int NV>
__global__ void __launch_bounds__(256) rk_combine_kernel(const __grid_constant__ SweepParams p)
{
    if (p.ctl && p.ctl->done) return;
    const double rkBdt = p.ctl ? p.ctl->bdt[p.rk_stage] : p.rkBdt;
    unsigned err = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < p.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        bool fin = true;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const long long gi = v * p.ncell + c;
            const double r = p.rhs[gi];
            double o;
            if (p.rk_stage == 1) o = p.u0[gi] - rkBdt * r;
            else o = p.rkA * p.u0[gi] - rkBdt * r + p.rkC * p.u[gi];
            p.u_out[gi] = o;
            fin = fin && isfinite(o);
        }
        if (!fin) err |= ERR_NONFINITE;
    }
    if (err) atomicOr(p.err, err);
}

template <int NV>
cudaError_t launch_rk_combine(const SweepParams &p, cudaStream_t st)
{
    long long g = (p.ncell + 255) / 256;
    if (g > 148LL * 16) g = 148LL * 16;
    if (g < 1) g = 1;
    rk_combine_kernel<NV><<<(unsigned)g, 256, 0, st>>>(p);
    return cudaGetLastError();
}

} // namespace CFD_NS
} // namespace cfd
