// Declarations of the explicitly instantiated sweep launchers
// (sweep_inst.cu is compiled once per flavour, NV and interpolator family).
#pragma once
#include "sweep_params.h"

namespace cfd {
namespace strict {
template <int NV, int FAM>
cudaError_t launch_sweep(int ax, int flux, const SweepParams &p, cudaStream_t st);
template <int NV, int FAM>
cudaError_t launch_sweep_batched(int ax, int flux, const BatchSweep &b, cudaStream_t st);
template <int NV>
cudaError_t launch_rk_combine(const SweepParams &p, cudaStream_t st);
}
namespace fast {
template <int NV, int FAM>
cudaError_t launch_sweep(int ax, int flux, const SweepParams &p, cudaStream_t st);
template <int NV, int FAM>
cudaError_t launch_sweep_batched(int ax, int flux, const BatchSweep &b, cudaStream_t st);
template <int NV>
cudaError_t launch_rk_combine(const SweepParams &p, cudaStream_t st);
}

#define CFD_FOR_EACH_FAMILY(X) X(0) X(1) X(2) X(3) X(4) X(5)

#define CFD_DECL_EXTERN(NS, NV, F) \
    namespace NS { extern template cudaError_t launch_sweep<NV, F>(int, int, const SweepParams &, cudaStream_t); }

// Runtime dispatch over (flavour, NV, family).
inline cudaError_t launch_sweep_any(bool strict_flavour, int nv, int fam, int ax, int flux, const SweepParams &p,
                                    cudaStream_t st)
{
#define CFD_CASE(NV, F)                                                                                       \
    if (nv == NV && fam == F)                                                                                 \
        return strict_flavour ? strict::launch_sweep<NV, F>(ax, flux, p, st) : fast::launch_sweep<NV, F>(ax, flux, p, st);
#define CFD_CASES_NV(F) CFD_CASE(3, F) CFD_CASE(4, F) CFD_CASE(5, F)
    CFD_FOR_EACH_FAMILY(CFD_CASES_NV)
#undef CFD_CASES_NV
#undef CFD_CASE
    return cudaErrorInvalidValue;
}

// The stage combination by itself (rk_combine_kernel), in the flavour's rounding.
inline cudaError_t launch_rk_combine_any(bool strict_flavour, int nv, const SweepParams &p, cudaStream_t st)
{
    if (nv == 3) return strict_flavour ? strict::launch_rk_combine<3>(p, st) : fast::launch_rk_combine<3>(p, st);
    if (nv == 4) return strict_flavour ? strict::launch_rk_combine<4>(p, st) : fast::launch_rk_combine<4>(p, st);
    if (nv == 5) return strict_flavour ? strict::launch_rk_combine<5>(p, st) : fast::launch_rk_combine<5>(p, st);
    return cudaErrorInvalidValue;
}

inline cudaError_t launch_sweep_batched_any(bool strict_flavour, int nv, int fam, int ax, int flux,
                                            const BatchSweep &b, cudaStream_t st)
{
#define CFD_CASE(NV, F)                                                                                        \
    if (nv == NV && fam == F)                                                                                  \
        return strict_flavour ? strict::launch_sweep_batched<NV, F>(ax, flux, b, st)                           \
                              : fast::launch_sweep_batched<NV, F>(ax, flux, b, st);
#define CFD_CASES_NV(F) CFD_CASE(3, F) CFD_CASE(4, F) CFD_CASE(5, F)
    CFD_FOR_EACH_FAMILY(CFD_CASES_NV)
#undef CFD_CASES_NV
#undef CFD_CASE
    return cudaErrorInvalidValue;
}

// Tile count of one case's sweep along ax (same shapes as the launchers;
// shape 1: the batched alternative shapes).
inline long long sweep_tile_count(int nv, int ax, const SweepParams &p, int shape = 0)
{
    int T0 = (nv == 3) ? 1 : ((ax == 0) ? 1 : 0);
    int T1 = (ax == 2) ? 1 : 2;
    int W = (nv == 3) ? k1W : ((ax == 0) ? (shape ? kXW2 : kXW) : (shape ? kYW2 : kYW));
    long long nseg = (p.n[ax] + p.seg_len - 1) / p.seg_len;
    return (long long)((p.n[T0] + W - 1) / W) * p.n[T1] * nseg;
}

} // namespace cfd
