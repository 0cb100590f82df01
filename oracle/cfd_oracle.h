/* ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the zone_FD right-hand side and SSP-RK3 step
 * (1D/2D as in the reference, 3D as this project's extension), used only by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg. It is the
 * checker, never the product: libcfdgpu.so does not link it.
 *
 * Pinning: in 1D and 2D it reproduces the compiled reference
 * (oracle/_ref/libcongfd_ref.so) bit for bit on the golden cases under
 * tests/golden; in 3D it is pinned by the z-invariance cross-check against
 * its own (reference-pinned) 2D path.
 */
#ifndef CFD_ORACLE_H
#define CFD_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* interpolator families (same numbering as the library) */
enum { ORC_WCNS5 = 0, ORC_WENOZ = 1, ORC_TENOZ = 2, ORC_TENOCONG = 3, ORC_MUSCL = 4 };
/* boundary kinds, uniform per direction side */
enum { ORC_OUTLET = 7, ORC_SYMMETRY = 10, ORC_WRAP = 100, ORC_MIRRORCOPY = 1 };

typedef struct orc_cfg {
    int dim;          /* 1, 2, 3 */
    int n[3];         /* cells per direction */
    double h;         /* uniform spacing (Info::geth) */
    int fam;          /* interpolator family */
    double icst;      /* family constant (TENO cutoff) */
    int flux;         /* 0 HLLC, 1 Roe */
    int bc[3][2];     /* ORC_OUTLET / ORC_SYMMETRY (normal velocity negated) / ORC_WRAP /
                         ORC_MIRRORCOPY (PERIODIC1D with the reference's default wiring) */
    int threads;      /* OpenMP threads (0 = runtime default) */
    int diff;         /* 0: MND6 (4 ghosts), 1: TRAD6 (ExplicitDif6, 5 ghosts) */
    int posl;         /* 2D/3D: 1 = the 1D positivity limiter on the face states (the library's
                         cfd_config.positivity) instead of the reference's cell-state fallback */
} orc_cfg;

/* rhs (AoS, ncell*nvar) of cons (AoS) */
void orc_rhs(const orc_cfg *c, const double *cons, double *rhs);
/* getTimeIntervalExplicit */
double orc_max_dt(const orc_cfg *c, const double *cons, double cfl);
/* one RK3 step in place; returns max |R_rho| of stage 3 */
double orc_rk3(const orc_cfg *c, double *cons, double dt);
/* one interpolation (family, constant) */
double orc_inter5(int fam, double icst, const double *q5);

#ifdef __cplusplus
}
#endif
#endif
