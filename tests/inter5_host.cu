// Host build of the device interpolators (cfd_inwsl_b200/csrc/euler_math.cuh)
// for tests/test_research_host.py: the research variants' cut-off decisions
// compiled by the host compiler, with the host libm, so that they can be held
// to the reference's own functions bit for bit on the CPU.
#include "euler_math.cuh"

extern "C" void h_research_inter5(int variant, const double *q, int n, double *out)
{
    for (int i = 0; i < n; i++)
        out[i] = cfd::inter5<cfd::FAM_RESEARCH>(q[5 * i], q[5 * i + 1], q[5 * i + 2], q[5 * i + 3], q[5 * i + 4],
                                                 (double)variant);
}
