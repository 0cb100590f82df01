// Declarations of the explicitly instantiated sweep launchers
// (sweep_inst.cu is compiled once per flavour, NV and interpolator family).
#pragma once
#include "sweep_params.h"

namespace cfd {
namespace strict {
template <int NV, int FAM>
cudaError_t launch_sweep(int ax, int flux, const SweepParams &p, cudaStream_t st);
}
namespace fast {
template <int NV, int FAM>
cudaError_t launch_sweep(int ax, int flux, const SweepParams &p, cudaStream_t st);
}

#define CFD_FOR_EACH_FAMILY(X) X(0) X(1) X(2) X(3) X(4)

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

} // namespace cfd
