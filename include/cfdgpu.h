/*
 * cfdgpu.h - C ABI of the B200 (sm_100a) right-hand-side evaluation and
 * SSP-RK3 time stepper for the zone_FD finite-difference Euler solver.
 *
 * The reference evaluates one RK stage inside BlockSolver::RK3_SSP
 * (zone_FD/src/src/blockSolver.cpp:43-87) as four member calls on host
 * objects:
 *     Equation::consToPrim()        equation.cpp:8-29
 *     Bnds::update()                bnds.cpp:23-27, oneDBnd.cpp:31-114
 *     SpDistributor::rhsSolve()     sp_distributor.cpp:3-79
 *     SourceTerm::calSource()       sourceTerm.cpp:50-52 (a no-op without gravity)
 * followed by an OpenMP stage combination, and computes the CFL step in
 * BlockSolver::getTimeIntervalExplicit (blockSolver.cpp:318-349). This
 * library replaces that whole per-stage body with GPU kernels behind the
 * plain C functions below. No C++ or CUDA types cross the interface.
 *
 * Ownership: a handle owns all device memory it allocates. Host pointers are
 * borrowed for the duration of a call only. Calls on one handle are ordered
 * on the handle's CUDA stream; a handle is not thread-safe.
 *
 * Status: every function returns CFD_OK (0) or a negative CFD_ERR_* code;
 * cfd_last_error() gives a message for the last failure on a handle. There is
 * no CPU fallback: if the CUDA kernels cannot run, calls fail.
 *
 * Array layout on the host side is the reference's Data layout
 * (zone_FD/src/src/data.cpp:63): cell-major AoS, data[cell * nvar + var],
 * cell = i + nx * (j + ny * k), nvar = 3 (1D), 4 (2D) or 5 (3D), conserved
 * variables (rho, rho*u, rho*v, [rho*w,] rho*E).
 */
#ifndef CFDGPU_H
#define CFDGPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define CFD_OK 0
#define CFD_ERR_CONFIG (-1)          /* invalid configuration or argument */
#define CFD_ERR_CUDA (-2)            /* a CUDA call failed (message in cfd_last_error) */
#define CFD_ERR_NONFINITE (-3)       /* a stage produced NaN/Inf in the state */
#define CFD_ERR_NEGATIVE_STATE (-4)  /* density or pressure <= 0 after a step */
#define CFD_ERR_TIMEOUT (-5)         /* a bounded device-side wait gave up */
#define CFD_ERR_UNSUPPORTED (-6)     /* option the library does not implement */
#define CFD_ERR_NOMEM (-7)           /* device allocation failed */

/* FluxMethod (zone_FD/src/include/macro.hpp:86). */
#define CFD_FLUX_HLLC 0
#define CFD_FLUX_ROE 1

/* DiffMethod (macro.hpp:82). MND6 (MidNodeAndNodeDif6, 4 ghosts) and TRAD6
 * (ExplicitDif6, differ.cpp:23-52, 5 ghosts) are implemented; HDS6 has no
 * differ in the reference (SolverType::initDiffer, solverType.cpp:657-681) and
 * TRAD2 no ghost count with a five-point interpolation (info.cpp:7-22). */
#define CFD_DIFF_TRAD6 1
#define CFD_DIFF_MND6 3

/* Arithmetic of the sweep kernels. */
#define CFD_PREC_FP64 0   /* FP64 everywhere */
#define CFD_PREC_MIXED 1  /* FP32 reconstruction and face flux, FP64 state/RK/differences */

/* Boundary types: BndType values of macro.hpp:33-34, plus two extensions. */
#define CFD_BND_TYPENULL 0
#define CFD_BND_PERIODIC1D 1        /* ghost k = prim(i0 + k*offset) */
#define CFD_BND_SYMMETRY1D 2        /* mirror, normal (x) velocity negated, 1D */
#define CFD_BND_DIRICLET 3          /* static ghost values */
#define CFD_BND_SUPERSONICOUTLET 7  /* ghost k = prim(i0) (zero gradient) */
#define CFD_BND_DOUBLEMACHUP 8      /* exact moving-shock state at the stage time */
#define CFD_BND_SYMMETRYX 10        /* mirror, u negated */
#define CFD_BND_SYMMETRYY 11        /* mirror, v negated */
#define CFD_BND_SYMMETRYZ 12        /* extension for 3D: mirror, w negated */
#define CFD_BND_PERIODIC_WRAP 100   /* extension: PERIODIC1D wired as a true wrap
                                       (low side copies the far end, high side the near end) */
#define CFD_BND_HALO 101            /* extension: ghosts from a neighbouring slab's rows
                                       (cfd_enable_halo; slab decomposition over GPUs) */

typedef struct cfd_config {
    int dim;            /* 1, 2 or 3 */
    int n[3];           /* cells per direction (Info::icMax()); 1 for unused directions */
    double h[3];        /* spacing per direction; the reference uses one h for all (Info::geth) */
    double x0[3];       /* lower corner of the domain (Info::calZone[0,2,4]) */
    int n_ghost;        /* Info::nGhostCell (info.cpp:7-22): 4 with MND6, 5 with TRAD6 */
    double gamma;       /* must be 1.4 (macro.hpp:28 GAMMA) */
    int inter_method;   /* InterMethod enum value (macro.hpp:37-78) */
    int flux_method;    /* CFD_FLUX_HLLC or CFD_FLUX_ROE */
    int diff_method;    /* CFD_DIFF_MND6 or CFD_DIFF_TRAD6 (TRAD6: FP64 only; not in batches,
                           slabs, the adjoint or cfd_rhs_noalloc) */
    int precision;      /* CFD_PREC_FP64 or CFD_PREC_MIXED */
    int strict;         /* 1: reference operation order, no FMA contraction (bitwise parity build) */
    int bc[3][2];       /* default boundary type per direction and side (0 = low, 1 = high),
                           wired per line like Initializer::initBnds (initializer.cpp:743-870):
                           low side i0 = first cell, offset = +stride (calOffset);
                           high side i0 = last cell, offset = -stride (calOffsetInverse).
                           Accepted here (CFD_ERR_CONFIG otherwise, before any device work):
                           PERIODIC1D, SUPERSONICOUTLET, PERIODIC_WRAP, SYMMETRYX, SYMMETRY1D (1D),
                           SYMMETRYY (2D/3D), SYMMETRYZ (3D), DOUBLEMACHUP (2D). Static types such
                           as DIRICLET need ghost values: wire those lines with cfd_set_line_bc.
                           HALO ends are wired by cfd_enable_halo. */
    int device;         /* CUDA device ordinal */
    int seg_len[3];     /* cells per CTA segment along each sweep (0 = autotuned default) */
    int source_type;    /* SourceType (macro.hpp:90): 0 none, 1 GRAVITY (2D; SourceTerm::calGravitySource,
                           sourceTerm.cpp:3-20: rhs_(rho v) -= rho, rhs_(rho E) -= rho v) */
    int positivity;     /* face states of 2D/3D reconstruction: 0 = the reference's fallback to the cell
                           state when rho or p < 0 (reconstructor5order.hpp:380-381); 1 = the limiter
                           the reference applies in 1D (variable_positive_limiter,
                           positive_preserving.hpp:13-46, on rho then gamma p, as in
                           reconstructor5order.hpp:227-232), extended to the 2D/3D cons
                           (FP64 only; not in the adjoint) */
} cfd_config;

typedef struct cfd_handle cfd_handle;

/* Fills *cfg with the reference's defaults (2D, 4 ghosts, gamma 1.4, WCNS5,
 * HLLC, MND6, FP64, supersonic outlets on every side). */
void cfd_config_default(cfd_config *cfg);

/* Replaces BlockSolver(Info*)'s setup (blockSolver.cpp:24-41) for the device
 * side: allocates the state, RHS and boundary tables. */
int cfd_create(const cfd_config *cfg, cfd_handle **out);
void cfd_destroy(cfd_handle *h);
const char *cfd_last_error(const cfd_handle *h);

/* Rewires one ghost strip, mirroring OneDBnd (oneDBnd.cpp:3-29):
 * idim 1/2/3 selects x/y/z lines as in Bnds::getOneDBnd (bnds.cpp:3-21), (i, j)
 * are the line's transverse indices, side 0/1 = low/high end. i0/offset are
 * OneDBnd::setUpdate's source cell and stride; ghost_prim (n_ghost*nvar
 * primitive values, may be NULL) is OneDBnd::setValue's static data. */
int cfd_set_line_bc(cfd_handle *h, int idim, int i, int j, int side, int bnd_type, long long i0, int offset,
                    const double *ghost_prim);

/* Host <-> device state copies in the reference AoS layout (Data). */
int cfd_upload_cons(cfd_handle *h, const double *aos);
int cfd_download_cons(cfd_handle *h, double *aos);
/* Primitive variables of the current state (Equation::consToPrim). */
int cfd_download_prim(cfd_handle *h, double *aos);

/* One RHS evaluation on the current state at time t (one stage body of
 * RK3_SSP: consToPrim, Bnds::update, rhsSolve), written to aos_rhs in the
 * reference layout. */
int cfd_rhs(cfd_handle *h, double t, double *aos_rhs);

/* CFL step of BlockSolver::getTimeIntervalExplicit: cfl / sum_d max_i
 * ((sqrt(gamma p / rho) + |u_d|) / h_d) on the current state. */
int cfd_max_dt(cfd_handle *h, double cfl, double *dt);

/* One SSP-RK3 step of size dt starting at time t (BlockSolver::RK3_SSP; the
 * stage times are t, t + dt, t + dt/2). If rho_linf is not NULL it receives
 * max |R_rho| of the third stage (the reference's log value). */
int cfd_rk3_step(cfd_handle *h, double dt, double t, double *rho_linf);

/* Device-resident time loop of BlockSolver::stepsLoopCFL
 * (blockSolver.cpp:170-235): from time *t, takes CFL steps clipped to the
 * output interval until end_step output intervals are done or max_steps RK3
 * steps were taken. dt and the clipping stay on the device; steps are launched
 * as captured CUDA graphs. *t and *nsteps receive the final time and step
 * count; dts/linf (length max_steps, may be NULL) receive per-step dt and
 * max |R_rho|. */
int cfd_run(cfd_handle *h, double cfl, int end_step, double output_dt, int max_steps, double *t, int *nsteps,
            double *dts, double *linf);

/* One CFL step from a host state to a host state, both in the reference's
 * AoS layout (BlockSolver::RK3_SSP with getTimeIntervalExplicit's dt, as one
 * step of stepsLoopCFL, blockSolver.cpp:43-87 and :170-235, for host code
 * that keeps its Data on the host between steps): equal bit for bit to
 * cfd_upload_cons(in_aos) + cfd_run(h, cfl, 1, output_dt, 1, t, ...) +
 * cfd_download_cons(out_aos). The copies overlap the step: the upload runs in
 * chunks along the last dimension, each chunk transposed, its wave speeds
 * reduced and its lines of stage 1's leading sweeps computed while the next
 * one copies, stage 1's last sweep as a partial RHS as soon as its segments'
 * cells are in; the last sweep of stage 3 runs in chunks of whole segments,
 * each downloaded while the next is computed. in_aos and out_aos may be the same
 * buffer; pinned host memory lets the copies run asynchronously. *t is
 * advanced; *dt (may be NULL) receives the step size. 1D grids and grids of
 * fewer than 64 cells along the last dimension take the three calls in turn.
 * A handle with slab halos (cfd_enable_halo) is refused (CFD_ERR_UNSUPPORTED):
 * its stages need halo exchanges in between. */
int cfd_step_host(cfd_handle *h, double cfl, double output_dt, const double *in_aos, double *out_aos, double *t,
                  double *dt);

/* Device pointers and CUDA stream of the handle, for callers that keep the
 * state resident (e.g. a framework tensor sharing the buffer). state receives
 * the current conserved state in the device layout: planar SoA
 * state[var * ncell + cell]. */
int cfd_device_state(cfd_handle *h, double **state, long long *ncell, void **stream);
/* Uploads/downloads a planar SoA device buffer (same layout as above). */
int cfd_set_state_device(cfd_handle *h, const double *soa_dev);

/* Runs the handle's work on a caller-provided CUDA stream (cudaStream_t passed
 * as void*; NULL restores the handle's own stream). The caller keeps ownership. */
int cfd_set_stream(cfd_handle *h, void *stream);

/* Number of kernels this library launched for the handle so far (every kernel
 * of a captured step graph counts once per graph launch). */
unsigned long long cfd_launch_count(const cfd_handle *h);

/* One direction's line sweep alone, stream-ordered and not synchronised (the
 * per-kernel timing hook of the benchmark). idim is 1-based. mode 0: RHS of
 * this direction into the RHS buffer; 1: added to the RHS buffer; 2: added and
 * combined like RK stage 2 (dt = 0) into a spare state slot, as the last sweep
 * of a stage runs. The current state is not changed. */
int cfd_sweep(cfd_handle *h, int idim, int mode, double t);

/* FP64 peak probe: enqueues on `stream` (a cudaStream_t, NULL = legacy
 * default stream) one launch of eight independent DFMA chains of `iters`
 * steps per thread, eight 256-thread CTAs per SM, and returns in *flops the
 * floating-point operations it performs (2 per DFMA). Timing it with events
 * on the same stream gives the device's FP64 throughput, the denominator of
 * the sweeps' FP64 roofline. No counterpart in the reference. */
int cfd_fp64_peak_probe(long long iters, void *stream, double *flops);

/* Self-check of the strict flavour's correctly rounded division by a shared
 * reciprocal (Markstein's correction) against the device's IEEE division on n
 * seeded operand pairs (random, next to rounding midpoints, physical ranges,
 * signed zeros, tiny and huge dividends), each also in the grouped form
 * (three dividends over one divisor of either sign); *mismatches counts
 * quotients or reciprocals whose bits differ. No counterpart in the reference: it
 * backs the strict flavour's bit-for-bit parity. */
int cfd_check_division(long long n, unsigned long long seed, unsigned long long *mismatches);

/* Pointwise known-answer hooks: evaluate the device interpolator for
 * inter_method on n five-point stencils (q[5*i..5*i+4] -> out[i]), and the
 * device Riemann flux on n face pairs (lr[2*nvar*i ...] = left prim | right
 * prim -> out[nvar*i ...]) for sweep axis ax. Host pointers; used by tests. */
int cfd_eval_inter5(int inter_method, int strict, const double *q, int n, double *out);
int cfd_eval_flux(int dim, int ax, int flux_method, int strict, const double *lr, int n, double *out);
/* Face reconstruction known-answer hook (Recon5Order{1D,2D}EulerEig::reconI,
 * reconstructor5order.hpp:233-429): n stencils of six cells' prims
 * (prims6[(6*i + j)*nvar + v]) -> left | right face prims (out[2*nvar*i ...]),
 * in the reference's operation order (precision 0) or the mixed form (1). */
int cfd_eval_face(int dim, int ax, int inter_method, int precision, const double *prims6, int n, double *out);

/* Allocation-free RHS evaluation (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory: code that runs inside
 * another framework's memory pool, or a program that reserved all device
 * memory before loading this library. It takes the caller's device buffers,
 * cons_soa (input state) and rhs_soa (output), both planar SoA
 * [var * ncell + cell] with ncell = n[0]*n[1]*n[2], evaluates one RHS exactly
 * as cfd_rhs does for the same cfg (default boundary wiring from cfg->bc), and
 * enqueues everything on `stream` (a cudaStream_t; NULL = legacy default
 * stream) without synchronising. It calls no cudaMalloc/cudaFree and no
 * allocating library routine.
 *
 * Its only scratch, the ghost wiring of every line end, lives in a file-scope
 * device array of CFD_NOALLOC_MAX_LINE_ENDS entries (768 KiB) that each GPU
 * loading the library holds until the process exits. Grids with more line
 * ends than that (sum over directions of 2 * ncell / n[d]; 2D grids up to
 * 4096 x 4096 fit) are rejected with CFD_ERR_CONFIG and a message on stderr.
 * The first call on a device looks up the array's device address (once per
 * device, with cfg->device made current); make that first call before any
 * stream capture. The address is kept until the process exits: after
 * cudaDeviceReset, or anything else that destroys the device's primary
 * context, this entry point must not be called on that device again in the
 * same process. cfg->bc takes the same types as in cfd_create. A CUDA error
 * already pending on the calling thread is left in place and the call
 * returns CFD_ERR_CUDA without queueing anything. Every call rewrites the part of the array it uses, and all
 * calls share it: calls that overlap on the GPU (different streams, or other
 * threads) race on the array and must be serialised by the caller. */
#define CFD_NOALLOC_MAX_LINE_ENDS 16384
int cfd_rhs_noalloc(const cfd_config *cfg, const double *cons_soa, double *rhs_soa, double t, void *stream);

/* Order-of-accuracy hook (the reference's AccuracyTest, CongFD1.0/AccuracyTest.cpp:14-83):
 * d q / d x at n cells of spacing h for a unit-speed scalar, face values by the
 * left-biased five-point interpolation of inter_method, node values = q, MND6
 * difference. q holds n + 8 values: 4 ghosts, the n cells, 4 ghosts. */
int cfd_accuracy_test(int inter_method, int n, double h, const double *q, double *dqdx);

/* Batched mode: many independent cases of uneven grid sizes advanced
 * together. The configurations must share dim, inter_method, flux_method,
 * strict, precision and device; grid sizes, spacing and boundaries may differ.
 * Each step is one persistent sweep launch per direction and stage over the
 * tiles of every unfinished case and one control kernel for all cases; steps
 * are captured in CUDA graphs. Each case keeps its own dt, output clipping and
 * step count (BlockSolver::stepsLoopCFL per case). */
typedef struct cfd_batch cfd_batch;
int cfd_batch_create(const cfd_config *cfgs, int ncases, cfd_batch **out);
void cfd_batch_destroy(cfd_batch *b);
const char *cfd_batch_last_error(const cfd_batch *b);
/* The handle of case c, for cfd_upload_cons / cfd_download_cons /
 * cfd_set_line_bc on that case (owned by the batch). */
int cfd_batch_case(cfd_batch *b, int c, cfd_handle **h);
int cfd_batch_set_stream(cfd_batch *b, void *stream);
unsigned long long cfd_batch_launch_count(const cfd_batch *b);
/* Runs every case until it finished end_step output intervals of
 * output_dt[c] or max_steps steps; t[c] is each case's start time on entry
 * and end time on return; nsteps[c] its step count. */
int cfd_batch_run(cfd_batch *b, double cfl, int end_step, const double *output_dt, int max_steps, double *t,
                  int *nsteps);

/* Autotuner of the batched sweeps (no counterpart in the reference). For each
 * direction it times the persistent first-stage sweep of the whole batch over
 * the tilings it can run: tile shape in cells per chunk x lines per CTA
 * (0: 32 x 4 along x, 8 x 32 along y and z; 1: 32 x 8 along x, 8 x 16 along
 * y and z, 2D and 3D FP64 only), lines cut into 1 or 2 segments, and one or
 * as many persistent CTAs per SM as fit; keeps the
 * fastest. Results are bit for bit those of any other tiling. The tuning runs
 * sweeps on the cases' current states and touches only scratch buffers (RHS,
 * stage state); call it between runs. choice (may be NULL) receives per
 * direction {shape, segments, one CTA per SM}, ms (may be NULL) the chosen
 * sweep's time per direction. */
int cfd_batch_autotune(cfd_batch *b, int *choice, double *ms);
/* Sets the tiling of the sweeps along idim (1/2/3) by hand: shape 0/1,
 * segments per line (1..64), one_cta 0/1, as cfd_batch_autotune reports it. */
int cfd_batch_set_tiling(cfd_batch *b, int idim, int shape, int segments, int one_cta);

/* Frozen-dt time loop: nsteps SSP-RK3 steps of one fixed dt (no CFL step,
 * no output clipping), replayed from captured CUDA graphs of steps_per_graph
 * steps (the forward steps of cfd_adjoint_record, without its checkpoints).
 * Stage times stay at 0, so time-dependent boundaries (DoubleMachUp) are
 * refused with CFD_ERR_UNSUPPORTED. Returns after the steps finished, with
 * CFD_ERR_NONFINITE / CFD_ERR_NEGATIVE_STATE as cfd_rk3_step. The loop the
 * reference runs with a fixed step is BlockSolver::solve's RK3_SSP sequence
 * (blockSolver.cpp:43-87). */
int cfd_run_fixed(cfd_handle *h, double dt, int nsteps, int steps_per_graph);

/* Discrete adjoint. The reference has no adjoint; these entry points serve
 * gradient studies of the same discretisation (sensitivity of a functional of
 * the final state to the initial state). They cover 2D handles with WCNS5
 * (weno5_JSchen), TENO-Z (Teno5_Z family) or TENO-Cong reconstruction, the
 * Roe flux, MND6, FP64, no source term and CFD_BND_PERIODIC_WRAP on every side
 * (CFD_ERR_UNSUPPORTED otherwise); the positivity fallback is differentiated
 * where it fires. TENO's cut-off decisions are frozen: each face interpolates
 * with the fixed stencil its forward state selects, and the derivative is
 * that stencil's.
 *
 * cfd_rhs_vjp: lam = (dR/dU)^T mu at the handle's current state, R the RHS of
 * cfd_rhs (SpDistributor::rhsSolve, sp_distributor.cpp:3-79); mu and lam are
 * host AoS arrays like the state.
 *
 * cfd_adjoint_record: from the current state U^0, runs nsteps SSP-RK3 steps
 * with the fixed step dt (BlockSolver::RK3_SSP, blockSolver.cpp:43-87, dt
 * frozen so that the map U^0 -> U^N is differentiable) and keeps the state of
 * every ckpt_every-th step on the device. The handle's state is U^N afterwards.
 *
 * cfd_adjoint_reverse: given dJ/dU^N (host AoS), returns dJ/dU^0 (host AoS):
 * segment by segment backwards, it recomputes the segment's steps from its
 * checkpoint (keeping the three stage states of each step) and applies the
 * transposed stage Jacobians. Device memory: nsteps / ckpt_every + 3 *
 * ckpt_every + 9 states. */
int cfd_rhs_vjp(cfd_handle *h, const double *mu, double *lam);
int cfd_adjoint_record(cfd_handle *h, double dt, int nsteps, int ckpt_every);
int cfd_adjoint_reverse(cfd_handle *h, const double *dJ_dUN, double *dJ_dU0);

/* Slab decomposition of one grid over several GPUs (no counterpart in the
 * reference, which runs one block on one host). Each rank's handle holds a
 * slab along the last direction (y in 2D, z in 3D) and takes the ghost cells
 * of that direction's slab interfaces from halo buffers that the caller fills
 * with the neighbouring slab's four boundary rows (planes) before every stage:
 *
 * cfd_enable_halo: wires every line end of `side` (0 low, 1 high) of the last
 *   direction as CFD_BND_HALO and returns the device halo buffer, planar
 *   [var][row][line] with 4 rows in ascending coordinate order and
 *   n[0] (2D) or n[0]*n[1] (3D) lines; *count = nvar * 4 * lines doubles.
 * cfd_stage_state: device pointer of stage `stage`'s input state (1: U^n,
 *   2: U^(1), 3: U^(2)), planar SoA; its first and last four rows (planes) of
 *   the last direction are what the neighbours need.
 * cfd_rk3_stage: one stage of cfd_rk3_step (stage 3 completes the step and
 *   makes U^(n+1) the current state); t is the step's start time.
 * cfd_max_wave_speeds: max over cells of (c + |u_d|) / h_d per direction d
 *   (the terms of getTimeIntervalExplicit's sum, blockSolver.cpp:318-349), so
 *   that ranks can take the maximum over slabs before dt = CFL / sum_d. */
int cfd_enable_halo(cfd_handle *h, int side, double **buf, long long *count);
int cfd_stage_state(cfd_handle *h, int stage, double **state);
int cfd_rk3_stage(cfd_handle *h, int stage, double dt, double t);
int cfd_max_wave_speeds(cfd_handle *h, double *lam);

/* Device-controlled steps for callers that act between the stages (the slab
 * decomposition: halo exchange before each stage, wave speeds reduced over
 * ranks before each step) without a host round trip per step. No counterpart
 * in the reference; one step is the sequence
 *     [reduce the 4 words of cfd_reduction_words over ranks with MAX]
 *     cfd_loop_step_begin; for stage 1..3: [halos], cfd_loop_stage; cfd_loop_step_end
 * enqueued on the handle's stream, dt = CFL / sum_d lambda_d as
 * getTimeIntervalExplicit (blockSolver.cpp:318-349) and the stage times of
 * RK3_SSP kept on the device.
 * cfd_loop_begin: starts at time t with the given CFL number (no output
 *   clipping) and makes sure the reduction words hold the current state's wave
 *   speeds.
 * cfd_reduction_words: device pointer of 4 words: max |R_rho| of the last
 *   step and the per-direction maximum wave speeds (c + |u_d|) / h_d, as the
 *   IEEE bit patterns of non-negative doubles, whose order is that of the
 *   64-bit integers: a MAX reduction over ranks as int64 gives the global ones.
 * cfd_loop_end: waits for the stream and returns the time and the steps taken
 *   since cfd_loop_begin (CFD_ERR_NONFINITE / NEGATIVE as cfd_rk3_step). */
int cfd_loop_begin(cfd_handle *h, double cfl, double t);
int cfd_reduction_words(cfd_handle *h, unsigned long long **words);
int cfd_loop_step_begin(cfd_handle *h);
int cfd_loop_stage(cfd_handle *h, int stage);
int cfd_loop_step_end(cfd_handle *h);
int cfd_loop_end(cfd_handle *h, double *t, int *nsteps);

/* Binary checkpoint / restart of the state (the reference writes its output
 * through CGNS, cgnsio.cpp:3-101, and has no restart; libcgns is not part of
 * this library). Little-endian file: a 104-byte header (magic "CFDGPUCK",
 * version 1, dim, n[3], nvar, inter_method, flux_method, gamma, h[3], t, step),
 * the cons in the reference's AoS Data layout (ncell * nvar doubles), and a
 * 64-bit FNV-1a checksum of header and payload. Loading checks the magic, the
 * version, the grid shape and the checksum (CFD_ERR_CONFIG and a message
 * otherwise); t and step may be NULL. */
int cfd_save_checkpoint(cfd_handle *h, const char *path, double t, long long step);
int cfd_load_checkpoint(cfd_handle *h, const char *path, double *t, long long *step);

/* Library version string. */
const char *cfd_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CFDGPU_H */
