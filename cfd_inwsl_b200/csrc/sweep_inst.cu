// Explicit instantiation of the sweep launcher for one (flavour, NV, family).
// The build compiles this file once per combination with -DCFD_NS=<strict|fast>,
// -DCFD_NV=<3|4|5>, -DCFD_FAM=<family>, and --fmad=false for the strict flavour.
#include "sweep.cuh"
namespace cfd {
namespace CFD_NS {
template cudaError_t launch_sweep<CFD_NV, CFD_FAM>(int ax, int flux, const SweepParams &p, cudaStream_t st);
template cudaError_t launch_sweep_batched<CFD_NV, CFD_FAM>(int ax, int flux, const BatchSweep &b, cudaStream_t st);
#if CFD_FAM == 0
template cudaError_t launch_rk_combine<CFD_NV>(const SweepParams &p, cudaStream_t st);
#endif
} // namespace CFD_NS
} // namespace cfd
