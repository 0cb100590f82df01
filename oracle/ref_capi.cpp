// Test-oracle harness around the reference zone_FD solver.
//
// ORACLE / TEST INFRASTRUCTURE ONLY. This file is compiled together with the
// unmodified reference sources (zone_FD/src/src/*.cpp) into
// oracle/_ref/libcongfd_ref.so by oracle/Makefile. Only tests, the smoke check
// and the CPU-baseline leg of bench.py load that library; the product
// (libcfdgpu.so) never links or calls it.
//
// It exposes a plain C interface so Python can drive the reference's own
// RHS evaluation, SSP-RK3 stepper and CFL time step on arbitrary states:
//   * the solver is built by the reference's public constructor
//     BlockSolver(Info*) (zone_FD/src/src/blockSolver.cpp:24-41), which runs
//     initUniformBlock / initEqution / initBnds / initSpDistributor;
//   * the private members are reached by compiling the reference headers with
//     `private`/`protected` mapped to `public` (standard headers are included
//     first so they are not affected);
//   * one RHS is rhs->setZeros; eqn->consToPrim; bnds->update;
//     spDis->rhsSolve; sourceTerm->calSource, the per-stage body of
//     BlockSolver::RK3_SSP (blockSolver.cpp:51-55);
//   * ref_run restates BlockSolver::stepsLoopCFL (blockSolver.cpp:170-235)
//     without its CGNS output and log-file side effects.
//   * ref_set_line_bc replaces one OneDBnd (oneDBnd.cpp:3-29) so tests can wire
//     any boundary type per line end, including a true periodic wrap that the
//     reference's own Euler wiring (initializer.cpp:806-862) does not produce.
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
#include "eigenSystem.hpp"
#include "fluxSchemes.hpp"
#include "interScheme.hpp"
#include "reconstructor5order.hpp"
#undef private
#undef protected

extern "C" {

struct ref_cfg {
    int dim;            // 1 or 2 (the reference has no 3D Euler path)
    int n[3];           // cells per direction (1 for unused directions)
    double zone[6];     // Info::calZone
    int inter_method;   // InterMethod enum value (macro.hpp:37-78)
    int flux_method;    // FluxMethod: HLLC=0, ROE=1
    int n_case;         // Info::nCase: selects the initial state and BC wiring
    double cfl;         // Info::CFL
    int source_type;    // Info::sourceType (0 SOURCENULL, 1 GRAVITY)
    int diff_method;    // Info::diffMethod (DiffMethod: HDS6 0, TRAD6 1, TRAD2 2, MND6 3)
};

struct ref_handle {
    Info *info;
    BlockSolver *bs;
};

void *ref_create(const ref_cfg *c)
{
    Info *info = new Info();
    info->eqType = EULER;
    info->spMethod = WCNS5;
    info->diffMethod = (DiffMethod)c->diff_method;
    info->fluxMethod = (FluxMethod)c->flux_method;
    info->interMethod = (InterMethod)c->inter_method;
    info->nCase = c->n_case;
    info->CFL = c->cfl;
    info->sourceType = (SourceType)c->source_type;
    info->dim = c->dim;
    for (int i = 0; i < 6; i++) info->calZone[i] = c->zone[i];
    // iMax counts vertices; Info::icMax() gives cells = iMax - 1 (info.cpp:120-129).
    for (int d = 0; d < 3; d++) info->iMax[d] = (c->n[d] > 1) ? c->n[d] + 1 : 1;
    info->endStep = 1;
    info->outputDt = 1e300;
    std::streambuf *old = std::cout.rdbuf(nullptr); // constructor prints progress lines
    BlockSolver *bs = new BlockSolver(info);
    std::cout.rdbuf(old);
    ref_handle *h = new ref_handle{info, bs};
    return h;
}

void ref_destroy(void *hp)
{
    ref_handle *h = (ref_handle *)hp;
    // BlockSolver's destructor deletes info and every owned object.
    delete h->bs;
    delete h;
}

int ref_ncells(void *hp) { return ((ref_handle *)hp)->bs->cons->getN(); }
int ref_nvar(void *hp) { return ((ref_handle *)hp)->bs->cons->getNVar(); }
double ref_h(void *hp, int idim) { return ((ref_handle *)hp)->info->geth(idim); }
double ref_time(void *hp) { return ((ref_handle *)hp)->info->t; }
void ref_set_time(void *hp, double t) { ((ref_handle *)hp)->info->t = t; }

void ref_set_cons(void *hp, const double *aos)
{
    Data *cons = ((ref_handle *)hp)->bs->cons;
    std::copy(aos, aos + cons->size(), cons->begin());
}
void ref_get_cons(void *hp, double *aos)
{
    Data *cons = ((ref_handle *)hp)->bs->cons;
    std::copy(cons->begin(), cons->end(), aos);
}
void ref_get_prim(void *hp, double *aos)
{
    ref_handle *h = (ref_handle *)hp;
    h->bs->eqn->consToPrim();
    Data *prim = h->bs->eqn->getPrim();
    std::copy(prim->begin(), prim->end(), aos);
}

// One RHS evaluation exactly as one stage of BlockSolver::RK3_SSP computes it.
void ref_rhs(void *hp, double *aos_rhs)
{
    ref_handle *h = (ref_handle *)hp;
    BlockSolver *bs = h->bs;
    bs->rhs->setZeros();
    bs->eqn->consToPrim();
    bs->bnds->update();
    bs->spDis->rhsSolve();
    bs->sourceTerm->calSource();
    if (aos_rhs) std::copy(bs->rhs->begin(), bs->rhs->end(), aos_rhs);
}

// BlockSolver::getTimeIntervalExplicit (blockSolver.cpp:318-349).
double ref_max_dt(void *hp) { return ((ref_handle *)hp)->bs->getTimeIntervalExplicit(); }

// BlockSolver::solve (blockSolver.cpp:120-124): RK3_SSP then t += dt.
void ref_rk3(void *hp, double dt) { ((ref_handle *)hp)->bs->solve(dt); }

// Data::getLinf(0) of the RHS after the last stage: the log value printed by
// stepsLoopCFL (blockSolver.cpp:204).
double ref_rho_linf(void *hp) { return ((ref_handle *)hp)->bs->rhs->getLinf(0); }

// Restatement of BlockSolver::stepsLoopCFL (blockSolver.cpp:170-235) without
// output: runs until `step` reaches end_step (step counts output intervals) or
// max_steps RK3 steps were taken. dts/linf (may be NULL) receive per-step
// values. Returns the number of RK3 steps taken.
int ref_run(void *hp, int end_step, double output_dt, int max_steps, double *dts, double *linf)
{
    ref_handle *h = (ref_handle *)hp;
    Info *info = h->info;
    BlockSolver *bs = h->bs;
    info->endStep = end_step;
    info->outputDt = output_dt;
    info->step = 0;
    info->outputT = 0.0;
    int k = 0;
    while (info->step < info->endStep && k < max_steps) {
        double dt = bs->getTimeIntervalExplicit();
        if (info->outputT + dt > info->outputDt) {
            dt = info->outputDt - info->outputT;
            info->outputT = 0.0;
            info->step++;
        } else
            info->outputT += dt;
        bs->solve(dt);
        if (dts) dts[k] = dt;
        if (linf) linf[k] = bs->rhs->getLinf(0);
        k++;
    }
    return k;
}

// Replace the ghost strip of one line end. idim is 1-based as in
// Bnds::getOneDBnd (bnds.cpp:3-21): 1 = x lines indexed (i=j-index, j=k-index),
// 2 = y lines (i=x-index, j=k-index). side 0 = low end, 1 = high end.
// i0/offset follow OneDBnd::setUpdate; values (nGhost*nPrim, may be NULL) follow
// OneDBnd::setValue.
int ref_set_line_bc(void *hp, int idim, int i, int j, int side, int type, int i0, int offset,
                    const double *values)
{
    ref_handle *h = (ref_handle *)hp;
    BlockSolver *bs = h->bs;
    Bnds *bnds = bs->bnds;
    int nG = h->info->nGhostCell(), nP = h->info->nPrim();
    auto iMax = bnds->iMax;
    int index;
    if (idim == 1)
        index = (i + j * iMax[2]) * 2;
    else if (idim == 2)
        index = (iMax[1] * iMax[2] + i + j * iMax[2]) * 2;
    else
        return -1;
    auto b = std::make_shared<OneDBnd>(nG, nP, (BndType)type);
    b->setUpdate(bs->eqn->getPrim(), i0, offset);
    if (values) b->setValue(std::vector<double>(values, values + nG * nP));
    b->setInfo(h->info);
    bnds->oneDBnds.at(index + side) = b;
    return 0;
}

// Pointwise kernels of the reference, exposed for known-answer tests.
double ref_inter5(int inter_method, const double *q5)
{
    std::array<real, 5> q = {q5[0], q5[1], q5[2], q5[3], q5[4]};
    switch (inter_method) {
    case WCNS5: return weno5_JSchen(q);
    case WCNSZ5: return weno5_Z(q);
    case TCNS5: return Teno5_Z(q);
    case TCNS5CT4: return Teno5_ZCT4(q);
    case TCNS5CT7: return Teno5_ZCT7(q);
    case WCNS5CONGZ: return Teno5_CongZ(q);
    case WCNS5CONGZCT4: return Teno5_CongZCT4(q);
    case WCNS5CONGZCT7: return Teno5_CongZCT7(q);
    case new_TCNS5: return new_Teno5_Z(q);
    case new_WCNS5CONGZ: return new_Teno5_CongZ(q);
    case congTCNS5CT5: return congTcns5_ZCT5(q);
    case congTCNS5CT10: return congTcns5_ZCT10(q);
    case MUCSLIN5: return musclIn5(q);
    // the research variants (solverType.cpp:262-388 / 445-576)
    case whfTCNSN: return whf_TcnsN(q);
    case whfTCNSNA: return whf_TcnsN_A(q);
    case whfTCNSNAS: return whf_TcnsN_AS(q);
    case whfTCNSNS: return whf_TcnsN_S(q);
    case whfTCNSNLAD: return whf_TcnsN_LAD(q);
    case whfAITCNSNS: return whf_ai_TcnsN_S_1(q);
    case whfAITCNSNA: return whf_ai_TcnsN_A_2(q);
    case whfAITCNSNAS_1: return whf_ai_TcnsN_AS_1(q);
    case whfAITCNSNAS_2: return whf_ai_TcnsN_AS_2(q);
    case whfAITCNSNLADS: return whf_ai_TcnsN_LADS_yuanbao(q);
    case whfAITCNSNAZS: return whf_ai_TcnsN_AZS_yuanbao(q);
    case whfAITCNSNmyASF002_1: return whf_ai_TcnsN_myASF002_1(q);
    case whfAITCNSNmyASF002_2: return whf_ai_TcnsN_myASF002_2(q);
    case whfAITCNSNmyASF002_ai1: return whf_ai_TcnsN_myASF002_ai1(q);
    case whfzycTCNSNmyASF002_1: return whf_zyc_TcnsN_myASF002_1(q);
    case whfCOMPARE: return whf_TcnsN_COMPARE(q);
    case new_WHFTCNSA: return new_whf_TCNS_A(q);
    case new_WHFTCNSASF203_NoS: return whf_TCNS_AS_myF203_NoS(q);
    case new_WHFTCNSASF202_NoS: return whf_TCNS_AS_myF202_NoS(q);
    case 1010: return Teno5_CongAA(q);  // WCNS5CONGZCT7 as the 1D selector maps it
    default: return NAN;
    }
}

void ref_flux2d(int flux_method, const double *lr8, int normal_y, double *out4)
{
    std::array<real, 8> in;
    std::copy(lr8, lr8 + 8, in.begin());
    std::array<real, 4> res;
    std::array<real, 3> norm = {normal_y ? 0.0 : 1.0, normal_y ? 1.0 : 0.0, 0.0};
    std::span<real, 8> si(in);
    std::span<real, 4> so(res);
    if (flux_method == HLLC)
        HLLCFlux2D2(si, so, norm);
    else
        roeFlux2DSym(si, so, norm);
    std::copy(res.begin(), res.end(), out4);
}

void ref_flux1d(int flux_method, const double *lr6, double *out3)
{
    std::array<real, 6> in;
    std::copy(lr6, lr6 + 6, in.begin());
    std::array<real, 3> res;
    std::array<real, 3> norm = {1.0, 0.0, 0.0};
    std::span<real, 6> si(in);
    std::span<real, 3> so(res);
    if (flux_method == HLLC)
        HLLCFlux1D(si, so, norm);
    else
        roeFlux1D2(si, so, norm);
    std::copy(res.begin(), res.end(), out3);
}

} // extern "C"

// One face of Recon5Order{1D,2D}EulerEig::reconI (reconstructor5order.hpp:233-429):
// prims6 = six stencil cells (nvar prims each), face between cells 2 and 3;
// out = left face prim | right face prim. normal_y selects the 2D normal.
template <InterpolationScheme5Order F>
static void recon_one(int dim, int normal_y, const double *prims6, double *out)
{
    int nv = dim + 2;
    std::vector<std::vector<real>> cells(6, std::vector<real>(nv));
    for (int j = 0; j < 6; j++)
        for (int v = 0; v < nv; v++) cells[j][v] = prims6[j * nv + v];
    std::array<std::vector<real>::iterator, 6> in;
    for (int j = 0; j < 6; j++) in[j] = cells[j].begin();
    auto run = [&](auto &rc) {
        rc.nvar = nv;
        rc.data = std::make_shared<Data>(1, 2 * nv);
        rc.iter = rc.data->begin();
        rc.norm = {normal_y ? 0.0 : 1.0, normal_y ? 1.0 : 0.0, 0.0};
        rc.reconI(in);
        std::copy(rc.data->begin(), rc.data->end(), out);
    };
    if (dim == 1) {
        Recon5Order1DEulerEig<F> rc;
        run(rc);
    } else {
        Recon5Order2DEulerEig<F> rc;
        run(rc);
    }
}

extern "C" int ref_recon_face(int inter_method, int dim, int normal_y, const double *prims6, double *out)
{
    switch (inter_method) {
    case WCNS5: recon_one<weno5_JSchen>(dim, normal_y, prims6, out); return 0;
    case WCNSZ5: recon_one<weno5_Z>(dim, normal_y, prims6, out); return 0;
    case TCNS5: recon_one<Teno5_Z>(dim, normal_y, prims6, out); return 0;
    case WCNS5CONGZ: recon_one<Teno5_CongZ>(dim, normal_y, prims6, out); return 0;
    case MUCSLIN5: recon_one<musclIn5>(dim, normal_y, prims6, out); return 0;
    default: return -1;
    }
}

extern "C" void ref_set_threads(int n) { omp_set_num_threads(n); }
