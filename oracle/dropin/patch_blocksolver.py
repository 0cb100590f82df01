"""Generates the drop-in build of the reference's BlockSolver.

TEST INFRASTRUCTURE. Writes a patched copy of the reference's
zone_FD/src/include/blockSolver.hpp and zone_FD/src/src/blockSolver.cpp into an
output folder (oracle/_ref/dropin, git-ignored; nothing of the reference is
committed): the change a maintainer makes to hand the per-stage work of
BlockSolver::RK3_SSP (blockSolver.cpp:43-87) and the CFL step of
BlockSolver::getTimeIntervalExplicit (blockSolver.cpp:318-349) to the GPU
library through its C ABI (include/cfdgpu.h), as INTEGRATION.md describes:

  * blockSolver.hpp: #include "cfdgpu.h"; a cfd_handle member, gpuSetup(), and
    the CPU bodies kept under new names (RK3_SSP_cpu,
    getTimeIntervalExplicit_cpu);
  * blockSolver.cpp: both constructors end with gpuSetup(); the original
    RK3_SSP / getTimeIntervalExplicit are renamed, and GPU-backed ones are
    appended (GPU_CODE below, the same code INTEGRATION.md shows).

    python patch_blocksolver.py <reference zone_FD dir> <output dir>

Every edit is anchored on a line of the reference; a missing anchor is an error.
"""
import sys
from pathlib import Path

GPU_CODE = r'''
// ---- GPU drop-in (libcfdgpu.so): the per-stage work of RK3_SSP and the CFL
// step run on the device; everything else in BlockSolver is unchanged.
void BlockSolver::gpuSetup()
{
    cfd_config cfg;
    cfd_config_default(&cfg);
    const auto ic = info->icMax();
    cfg.dim = info->dim;
    for (int d = 0; d < 3; d++) {
        cfg.n[d] = d < info->dim ? ic[d] : 1;
        cfg.h[d] = info->geth(d);
        cfg.x0[d] = info->calZone[2 * d];
    }
    cfg.inter_method = info->interMethod;
    cfg.flux_method = info->fluxMethod;
    cfg.diff_method = info->diffMethod;
    cfg.n_ghost = info->nGhostCell();
    cfg.source_type = info->sourceType;
    cfg.strict = 1;  // the reference's operation order and roundings, bit for bit
    const int nv = info->nPrim(), ng = info->nGhostCell();
    // boundary types the configuration wires by itself for a whole side
    auto whole_side = [&](int t) {
        return t == PERIODIC1D || t == SUPERSONICOUTLET || t == SYMMETRYX || (t == SYMMETRY1D && info->dim == 1) ||
               (t == SYMMETRYY && info->dim >= 2) || (t == DoubleMachUp && info->dim == 2);
    };
    for (int d = 0; d < info->dim; d++)
        for (int side = 0; side < 2; side++) {
            const int t = bnds->getOneDBnd(d + 1, 0, 0)[side]->getType();
            cfg.bc[d][side] = whole_side(t) ? t : CFD_BND_SUPERSONICOUTLET;
        }
    if (cfd_create(&cfg, &gpu) != CFD_OK) {
        std::cout << "cfd_create failed\n";
        std::abort();
    }
    // every line end whose type differs from its side's default or that keeps
    // static ghost values (DIRICLET, ...), with the source cells of
    // calOffset / calOffsetInverse (macro.hpp:105-137)
    const long long stride[3] = {1, ic[0], (long long)ic[0] * ic[1]};
    for (int d = 0; d < info->dim; d++) {
        const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
        const int n0 = t0 < info->dim ? ic[t0] : 1, n1 = t1 < info->dim ? ic[t1] : 1;
        for (int j = 0; j < n1; j++)
            for (int i = 0; i < n0; i++) {
                auto ends = bnds->getOneDBnd(d + 1, i, j);
                for (int side = 0; side < 2; side++) {
                    const int t = ends[side]->getType();
                    if (t == cfg.bc[d][side] && whole_side(t)) continue;
                    const long long base = i * stride[t0] + (long long)j * stride[t1];
                    const long long last = base + (long long)(ic[d] - 1) * stride[d];
                    std::vector<double> vals;
                    if (!whole_side(t))
                        for (int k = 0; k < ng; k++)
                            for (int v = 0; v < nv; v++) vals.push_back((*ends[side])(k, v));
                    if (cfd_set_line_bc(gpu, d + 1, i, j, side, t, side == 0 ? base : last,
                                        side == 0 ? (int)stride[d] : -(int)stride[d],
                                        vals.empty() ? nullptr : vals.data()) != CFD_OK) {
                        std::cout << cfd_last_error(gpu) << '\n';
                        std::abort();
                    }
                }
            }
    }
}

void BlockSolver::RK3_SSP(real dt)
{
    cfd_upload_cons(gpu, &*cons->begin());  // Data is AoS, cell-major
    double rho_linf = 0.0;
    const int rc = cfd_rk3_step(gpu, dt, info->t, &rho_linf);  // stage times t, t+dt, t+dt/2
    cfd_download_cons(gpu, &*cons->begin());
    if (rc != CFD_OK) std::cout << cfd_last_error(gpu) << '\n';
    info->t = ((info->t + dt) - dt / 2) - dt / 2;  // where the reference's RK3_SSP leaves it
}

real BlockSolver::getTimeIntervalExplicit()
{
    double dt = 0.0;
    cfd_upload_cons(gpu, &*cons->begin());
    if (cfd_max_dt(gpu, info->CFL, &dt) != CFD_OK) std::cout << cfd_last_error(gpu) << '\n';
    return dt;
}
'''

HPP_MEMBERS = '''
    // GPU drop-in: device-side RHS / RK3 (libcfdgpu.so)
    cfd_handle *gpu = nullptr;
    void gpuSetup();
    void RK3_SSP_cpu(real);
    real getTimeIntervalExplicit_cpu();
'''


def edit(text, anchor, new, count=1, path=""):
    if text.count(anchor) != count:
        raise SystemExit(f"{path}: anchor {anchor!r} found {text.count(anchor)} times, expected {count}")
    return text.replace(anchor, new)


def main(ref_dir, out_dir):
    ref, out = Path(ref_dir), Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    hpp_path = ref / "src" / "include" / "blockSolver.hpp"
    cpp_path = ref / "src" / "src" / "blockSolver.cpp"
    hpp = hpp_path.read_text()
    hpp = edit(hpp, "#pragma once\n", '#pragma once\n#include "cfdgpu.h"\n', path=hpp_path)
    hpp = edit(hpp, "    TimeMethod timeMethod = RK3SSP;\n", "    TimeMethod timeMethod = RK3SSP;\n" + HPP_MEMBERS,
               path=hpp_path)
    cpp = cpp_path.read_text()
    cpp = edit(cpp, "    rhs = eqn->getRhs();\n}\n", "    rhs = eqn->getRhs();\n    gpuSetup();\n}\n", count=2,
               path=cpp_path)
    cpp = edit(cpp, "void BlockSolver::RK3_SSP(real dt)\n", "void BlockSolver::RK3_SSP_cpu(real dt)\n", path=cpp_path)
    cpp = edit(cpp, "real BlockSolver::getTimeIntervalExplicit()\n", "real BlockSolver::getTimeIntervalExplicit_cpu()\n",
               path=cpp_path)
    cpp = cpp + GPU_CODE
    (out / "blockSolver.hpp").write_text(hpp)
    (out / "blockSolver.cpp").write_text(cpp)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
