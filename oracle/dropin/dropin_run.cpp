// Test harness of the drop-in build (oracle/_ref/libcongfd_dropin.so).
//
// TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles this file with the
// reference sources (zone_FD/src/src/*.cpp), except that blockSolver.cpp and
// blockSolver.hpp are the copies patch_blocksolver.py writes with the GPU
// change of INTEGRATION.md applied, and links the result against
// libcfdgpu.so. dropin_run() then runs the reference's own driver,
// BlockSolver(Info*) and BlockSolver::stepsLoopCFL (blockSolver.cpp:24-41,
// 170-235), whose RK3_SSP and getTimeIntervalExplicit now call the GPU
// library; tests compare its final state with the unpatched reference.
#include <algorithm>
#include <array>
#include <cassert>
#include <chrono>
#include <cmath>
#include <concepts>
#include <cstring>
#include <filesystem>
#include <format>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <ranges>
#include <span>
#include <string>
#include <type_traits>
#include <variant>
#include <vector>
#include <omp.h>

#define private public
#define protected public
#include "blockSolver.hpp"
#undef private
#undef protected

extern "C" {

// One run of the reference driver with the GPU drop-in: an Info set up as
// the reference harness (oracle/ref_capi.cpp) sets it, one output interval of
// length t_end (endStep = 1, outputDt = t_end), BlockSolver::stepsLoopCFL.
// cons_out receives the final cons (AoS, ncell * nvar), *steps the RK3 steps.
int dropin_run(int dim, const int *n, const double *zone, int inter_method, int flux_method, int n_case, double cfl,
               int source_type, double t_end, double *cons_out, long long *steps)
{
    Info *info = new Info();
    info->eqType = EULER;
    info->spMethod = WCNS5;
    info->diffMethod = MND6;
    info->fluxMethod = (FluxMethod)flux_method;
    info->interMethod = (InterMethod)inter_method;
    info->nCase = n_case;
    info->CFL = cfl;
    info->sourceType = (SourceType)source_type;
    info->dim = dim;
    for (int i = 0; i < 6; i++) info->calZone[i] = zone[i];
    for (int d = 0; d < 3; d++) info->iMax[d] = (n[d] > 1) ? n[d] + 1 : 1;
    info->endStep = 1;
    info->outputDt = t_end;
    std::streambuf *old = std::cout.rdbuf(nullptr);  // progress lines of the constructor and the loop
    BlockSolver *bs = new BlockSolver(info);
    bs->stepsLoopCFL();
    std::cout.rdbuf(old);
    std::copy(bs->cons->begin(), bs->cons->end(), cons_out);
    *steps = bs->timesteps;
    cfd_destroy(bs->gpu);
    bs->gpu = nullptr;
    delete bs;
    return 0;
}

}  // extern "C"
