/*
 * pcc.h -- C ABI of the B200 Newton-shooting engine for discretely
 * self-similar critical collapse (the hot path of
 * tobjec/parallel-critical-collapse: the finite-difference Jacobian whose
 * columns are independent two-sided IRK shoots, and the dense Newton solve).
 *
 * Plain C: pointers and sizes only.  Host pointers are caller-owned; device
 * buffers are owned by a pcc_solve.  Every call is ordered on the context's
 * single CUDA stream and the host-pointer variants synchronise before they
 * return.  No call exits the process: failures come back as pcc_status, with
 * the failing column, side and grid index in pcc_stats.
 *
 * Conventions shared with the reference (all arrays FP64):
 *   Ntau        collocation points per echoing period (power of two, 128..2048)
 *   Nnewton     3*Ntau/4 Newton unknowns; in0[2*Nnewton/3+2] holds Delta
 *   state Y     Ntau/2 complex Fourier modes stored as Ntau interleaved reals,
 *               Re Y[2] = Delta (ODEStepper.cpp:92-136)
 *   J           Nnewton x Nnewton, row-major, J[row*Nnewton + col]
 *               = (F(in0 + eps e_col)[row] - out0[row]) / eps
 */
#ifndef PCC_H
#define PCC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PCC_OK = 0,
    PCC_ERR_INVALID_ARG = 1,
    PCC_ERR_CUDA = 2,
    PCC_ERR_OOM = 3,
    PCC_ERR_IRK_NO_CONVERGENCE = 4, /* ShootingSolver.cpp:69-82,112-125 exit */
    PCC_ERR_DELTA_MISMATCH = 5,     /* ShootingSolver.cpp:167-178 exit */
    PCC_ERR_NAN = 6,                /* non-finite free data given to a host-pointer entry point */
    PCC_ERR_LU_SINGULAR = 7,        /* NewtonSolver.cpp:751-755 exit */
    PCC_ERR_IR_STALL = 8,
    PCC_ERR_UNSUPPORTED = 9,
    PCC_ERR_NEWTON_NO_CONVERGENCE = 10, /* NewtonSolver.cpp:368-372 exit */
    PCC_ERR_BUSY = 11,
    PCC_ERR_TIMEOUT = 12            /* pcc_wait: the solve had not ended by the deadline */
} pcc_status;

typedef enum {
    PCC_PREC_FP64 = 0,  /* LU with partial pivoting in FP64 (LAPACKE_dgesv semantics) */
    PCC_PREC_MIXED = 1  /* FP32 LU + FP64 iterative refinement */
} pcc_precision;

typedef struct pcc_ctx pcc_ctx;
typedef struct pcc_solve pcc_solve;

typedef struct {
    int reserved; /* must be 0 */
} pcc_ctx_opts;

/* The numeric fields of the reference's SimulationConfig
 * (include/SimulationConfig.hpp:37-50) that the shooting path reads. */
typedef struct {
    int ntau;            /* Ntau */
    double dim;          /* Dim (D) */
    double xl, xm, xr;   /* XLeft, XMid, XRight */
    double eps_newton;   /* EpsNewton */
    int nl, nr;          /* NLeft, NRight */
    double prec_irk;     /* PrecisionIRK */
    int scheme;          /* SchemeIRK: 1, 2 or 3 Gauss-Legendre stages */
    int max_irk;         /* MaxIterIRK */
    double prec_newton;  /* PrecisionNewton */
    double slow_error;   /* SlowError (Newton damping) */
    int max_newton;      /* MaxIterNewton */
    int irk_predictor;   /* start of each step's stage iteration: 0 = y, as the reference
                          * (ODEStepper.cpp:202-212); 1 = the previous step's collocation
                          * polynomial, extrapolated (not in the reference: the same fixed
                          * point to round-off, fewer iterations) */
    int shoot_both_sides; /* 0 (default): a Jacobian column marches only the sides that read
                          * its free datum (U_p modes: the right side; psi_c and f_c modes:
                          * the left side; Delta: both) and takes the other side's final
                          * state from the base shoot, which marched the same boundary
                          * state bit for bit, so J and the statuses are those of full
                          * shoots; 1: every column marches both sides, as the reference's
                          * NewtonSolver::assembleJacobian (NewtonSolver.cpp:615-650, a
                          * full shoot per column at :639) */
} pcc_solve_desc;

typedef struct {
    long long rhs_evals;      /* RHS evaluations performed on the device */
    long long irk_iterations; /* fixed-point iterations summed over all steps */
    long long irk_steps;      /* grid steps marched */
    long long shoots;         /* shoot results delivered (Jacobian columns + base); with side reuse a
                               * column marches one side (see irk_steps for the sweeps' work) */
    double ms_prologue;       /* boundary data kernel (device time) */
    double ms_sweep;          /* IRK march kernel (device time) */
    double ms_epilogue;       /* mismatch/pack/difference kernels (device time) */
    double ms_total;          /* whole call incl. copies (device time) */
    int fail_column;          /* first failing column (-1: none; Nnewton: base) */
    int fail_side;            /* 0 left sweep, 1 right sweep */
    int fail_grid_index;      /* grid index the failing IRK step started from */
    int sweep_ctas;           /* persistent CTAs of the march kernel */
} pcc_stats;

typedef struct {
    double rel_err_vs_fp64; /* ||dx - dx_fp64|| / ||dx_fp64|| when checked, else -1 */
    double residual_norm;   /* ||b - A dx||_inf / (||A||_inf ||dx||_inf) after refinement */
    int refinement_steps;
    int fell_back_to_fp64;
    double ms;
} pcc_refine_report;

/* Context: one CUDA device, one stream.  NewtonSolver.hpp:150 (ctor) owner.
 * Destroying a context also destroys the solves still alive in it; their
 * handles must not be used afterwards. */
pcc_status pcc_ctx_create(int device, const pcc_ctx_opts* opts, pcc_ctx** out);
pcc_status pcc_ctx_destroy(pcc_ctx* ctx);
const char* pcc_status_string(pcc_status s);
const char* pcc_last_error(pcc_ctx* ctx);

/* Solve: device buffers, grid and tables for one SimulationConfig
 * (NewtonSolver.cpp:18-52 ctor + generateGrid :477-519). */
pcc_status pcc_solve_create(pcc_ctx* ctx, const pcc_solve_desc* desc, pcc_solve** out);
pcc_status pcc_solve_destroy(pcc_solve* s);
pcc_status pcc_solve_grid(pcc_solve* s, double* grid_out /* nl+nr+1 */);

/* The sweeps that a Jacobian or Newton pipeline over columns [c0, c1) (column
 * Nnewton = 3 Ntau/4 is the base shoot) of a solve with this Ntau marches, as
 * slots 2 column + side (0 left, 1 right): right sides first, each side in
 * column order; with shoot_both_sides = 0 only the sides that read each
 * column's free datum, plus the base shoot's sides that other columns take
 * (see pcc_solve_desc.shoot_both_sides).  Writes min(count, cap) slots and
 * returns the count, or -1 for an invalid Ntau or range.  Needs no device. */
int pcc_sweep_plan(int ntau, int shoot_both_sides, int c0, int c1, int* slots, int cap);

/* NewtonSolver::shoot (NewtonSolver.cpp:403-423): in0 -> out0, host arrays. */
pcc_status pcc_shoot(pcc_solve* s, const double* in0, double* out0, pcc_stats* stats);

/* pcc_shoot with the reference's Debug field export (ShootingSolver.cpp:
 * 85-97, 128-138): the state at the start of every step from grid index i
 * with i % debug_nx == 0, and at the ends of each sweep (left sweep ascending,
 * then right sweep descending, the reference's order), converted to A =
 * 1/sqrt(IA2), U, V, f on Ntau points.  *count gets the number of snapshots;
 * grid_idx[count] and fields[count][4][Ntau] are filled when count <=
 * max_snaps (else PCC_ERR_INVALID_ARG and nothing runs). */
pcc_status pcc_shoot_debug(pcc_solve* s, const double* in0, double* out0, int debug_nx, int max_snaps, int* count,
                           int* grid_idx, double* fields, pcc_stats* stats);

/* NewtonSolver::assembleJacobian (NewtonSolver.cpp:615-702): all Nnewton
 * columns in one persistent launch; host arrays, J row-major. */
pcc_status pcc_jacobian(pcc_solve* s, const double* in0, const double* out0, double* J, pcc_stats* stats);

/* The same on device pointers (inputs already resident in HBM); asynchronous
 * on the context stream, stats filled after pcc_solve_sync. */
pcc_status pcc_jacobian_device(pcc_solve* s, const double* d_in0, const double* d_out0, double* d_J);
pcc_status pcc_solve_sync(pcc_solve* s, pcc_stats* stats);

/* Columns [c0, c1) of J on device pointers, written column-major
 * (d_cols[(c - c0) * Nnewton + row] = J[row][c]), so that the blocks of a
 * column partition concatenate into J^T: the building block of a Jacobian
 * sharded over several GPUs and gathered with one all-gather.  Asynchronous
 * on the context stream; stats after pcc_solve_sync. */
pcc_status pcc_jacobian_columns_device(pcc_solve* s, const double* d_in0, const double* d_out0, int c0, int c1,
                                       double* d_cols);

/* Columns [c0, c1) only (c1 may be Nnewton+1 to include the base shoot, whose
 * output then lands in out_base).  cols is column-major (c1-c0) x Nnewton. */
pcc_status pcc_jacobian_columns(pcc_solve* s, const double* in0, const double* out0, int c0, int c1,
                                double* cols, pcc_stats* stats);

/* NewtonSolver::solveLinearSystem (NewtonSolver.cpp:739-757): A x = rhs,
 * A row-major n x n, n <= 3128 (a factorisation panel of n rows lives in
 * shared memory; every Newton system here has n = 3 Ntau / 4 <= 1536).  FP64
 * LU (LAPACKE_dgesv semantics), or PCC_PREC_MIXED: an FP32 LU whose trailing
 * updates run on the tensor cores (TF32 with a high/low split of each FP32
 * operand, FP32 accumulation; $PCC_LU_TC=0 keeps them on the CUDA cores),
 * refined to FP64 with FP64 residuals as LAPACK dsgesv does, falling back to
 * the FP64 LU if the refinement does not converge in 30 sweeps. */
pcc_status pcc_lu_solve(pcc_ctx* ctx, int n, const double* A, const double* rhs, double* x, pcc_precision prec,
                        pcc_refine_report* report);

/* One iteration of NewtonSolver::run's loop (NewtonSolver.cpp:279-366):
 * shoot, Jacobian, solve, damped update of in0 (in place).  err_out gets the
 * RMS mismatch before the update. */
pcc_status pcc_newton_step(pcc_solve* s, double* in0, double* err_out, pcc_precision prec, pcc_stats* stats,
                           pcc_refine_report* report);

/* ---- batches of solves and the device-resident Newton loop --------------
 * Several solves of one context (different Dim, Ntau and grid sizes) share
 * ONE persistent march launch: every sweep of every listed solve is an item
 * of that launch.  Solves with Ntau 128..1024 and 2 IRK stages batch; others
 * run their own launch inside the same call.  The result of a solve does not
 * depend on what it is batched with: each sweep is computed by one sweep slot
 * with the same arithmetic. */

/* assembleJacobian for count solves at once (host arrays, J[i] row-major
 * Nnewton_i x Nnewton_i).  Every solve must batch (PCC_ERR_UNSUPPORTED). */
pcc_status pcc_jacobian_batch(pcc_ctx* ctx, int count, pcc_solve* const* solves, const double* const* in0,
                              const double* const* out0, double* const* J, pcc_stats* stats);

/* Newton state codes: how NewtonSolver::run (NewtonSolver.cpp:279-372) ends. */
typedef enum {
    PCC_NEWTON_RUNNING = 0,
    PCC_NEWTON_CONVERGED = 1,      /* mismatch RMS < PrecisionNewton (:303-309) */
    PCC_NEWTON_STOPPED = 2,        /* mismatch grew 5 times: result = last improving iterate (:312-325) */
    PCC_NEWTON_MAX_ITER = 3,       /* MaxIterNewton iterations without convergence (:368-372) */
    PCC_NEWTON_IRK_FAILED = 4,     /* a sweep's IRK iteration failed (ShootingSolver.cpp:69-82) */
    PCC_NEWTON_DELTA_MISMATCH = 5, /* ShootingSolver.cpp:167-178 */
    PCC_NEWTON_SINGULAR = 6        /* zero pivot (NewtonSolver.cpp:751-755) */
} pcc_newton_code;

typedef struct {
    int iterations;          /* base shoots evaluated */
    int code;                /* pcc_newton_code */
    double err;              /* mismatch RMS of the last base shoot */
    double err_old;          /* of the one before */
    int fail_column, fail_side, fail_grid_index; /* IRK failure location, else -1 */
    int lu_refinement_steps; /* last mixed-precision solve's refinement sweeps (-1: FP64 solve) */
    int lu_fell_back;        /* last mixed-precision solve fell back to the FP64 factorisation */
} pcc_newton_state;

/* Starts NewtonSolver::run's loop on the device from in0 (host, Nnewton):
 * err = errOld = 1, no increases, in0old = in0 (NewtonSolver.cpp:268-277). */
pcc_status pcc_newton_begin(pcc_solve* s, const double* in0);

/* One loop iteration for every listed solve still running: base shoot and
 * all Jacobian columns of all of them in one batch launch, then per solve on
 * the device the convergence test and divergence safeguard, J, the Newton
 * solve (prec) and the damped update.  states[i] (optional) is solve i's
 * state afterwards; stats (optional) describes the launch. */
pcc_status pcc_newton_iterate(pcc_ctx* ctx, int count, pcc_solve* const* solves, pcc_precision prec,
                              pcc_newton_state* states, pcc_stats* stats);

/* The solve's result: the converged (or last) iterate, or for
 * PCC_NEWTON_STOPPED the last improving one; Delta at in0_out[2N/3+2]. */
pcc_status pcc_newton_result(pcc_solve* s, double* in0_out, pcc_newton_state* state);

/* begin + iterate until no solve is running + result, in0[i] in place. */
pcc_status pcc_newton_solve(pcc_ctx* ctx, int count, pcc_solve* const* solves, double* const* in0,
                            pcc_precision prec, pcc_newton_state* states, pcc_stats* stats);

/* ---- serving: whole Newton solves submitted over time --------------------
 * A request is one NewtonSolver::run of its own SimulationConfig.  A
 * scheduler thread inside the library admits requests in arrival order while
 * the device bytes of the admitted solves fit the HBM budget (and the cap on
 * concurrent solves), keeps each solve's Newton state on the device, and
 * batches the sweeps of all admitted solves as they become ready into shared
 * persistent launches, so that requests arriving while others run overlap
 * with them on the device.  Each launch is filled shortest work first (the
 * longest-waiting solve always gets a share), so small solves finish early.  Each result equals the one the same request gives
 * alone.  Ntau 128..1024 with 2 IRK stages.  While serving runs, the context
 * takes only pcc_submit / pcc_poll / pcc_wait / pcc_serve_stats, from any
 * thread; results can be read until pcc_serve_stop. */
typedef struct {
    size_t hbm_budget_bytes; /* device bytes admitted solves may hold (0: 3/4 of the free memory at start) */
    int max_active;          /* solves admitted at once (0: limited by the budget only) */
} pcc_serve_opts;

typedef struct {
    pcc_solve_desc desc;     /* the request's SimulationConfig */
    const double* in0;       /* Nnewton initial unknowns (Delta at 2N/3+2), copied by pcc_submit */
    pcc_precision precision; /* of its Newton solves */
} pcc_request;

typedef struct {
    int done;                /* 1 once the solve has ended; the fields below are then final */
    pcc_status status;       /* PCC_OK (converged, or stopped by the divergence safeguard) or why it failed */
    pcc_newton_state newton; /* how the Newton loop ended */
    double ms_queued;        /* submit -> admission (host clock) */
    double ms_latency;       /* submit -> result available */
    size_t footprint_bytes;  /* device bytes the solve held */
} pcc_result;

typedef struct {
    long long submitted, completed, launches, sweeps;
    int active, waiting;
    size_t bytes_in_use, budget_bytes;
} pcc_serve_info;

/* Starts the loop (pcc_submit starts it with defaults when needed). */
pcc_status pcc_serve_start(pcc_ctx* ctx, const pcc_serve_opts* opts);
/* Queues a request; ticket identifies it in pcc_poll / pcc_wait. */
pcc_status pcc_submit(pcc_ctx* ctx, const pcc_request* req, uint64_t* ticket);
/* Non-blocking: out->done tells whether the solve has ended; x_out (optional,
 * Nnewton) receives the result iterate once it has.  A finished result is
 * handed out once: the pcc_poll or pcc_wait call that returns it with
 * done = 1 releases its record, and later calls with that ticket return
 * PCC_ERR_INVALID_ARG (so a long-running service holds no memory for results
 * it has delivered). */
pcc_status pcc_poll(pcc_ctx* ctx, uint64_t ticket, pcc_result* out, double* x_out);
/* As pcc_poll, waiting up to timeout_s seconds for the solve to end;
 * PCC_ERR_TIMEOUT (out filled, out->done = 0) if it has not ended by then,
 * PCC_ERR_BUSY if serving was shut down (context destroyed) meanwhile. */
pcc_status pcc_wait(pcc_ctx* ctx, uint64_t ticket, double timeout_s, pcc_result* out, double* x_out);
pcc_status pcc_serve_stats(pcc_ctx* ctx, pcc_serve_info* out);
/* Finishes every submitted request (callers blocked in pcc_wait receive their
 * results meanwhile), then stops the loop and drops the undelivered results.
 * It may overlap pcc_poll / pcc_wait / pcc_submit on other threads: those
 * return PCC_ERR_INVALID_ARG or PCC_ERR_BUSY once the loop has stopped, and
 * the server is freed only after the last of them has returned.  A second
 * concurrent pcc_serve_stop returns at once. */
pcc_status pcc_serve_stop(pcc_ctx* ctx);

/* ---- lower-level entry points (the reference's inner class methods) ---- */

/* ODEStepper::computeDerivatives (ODEStepper.cpp:92-136) for `count` states:
 * y and dy are count x Ntau, x has count entries. */
pcc_status pcc_rhs_eval(pcc_ctx* ctx, int ntau, double dim, int count, const double* y, const double* x,
                        double* dy);

/* ODEStepper::stepIRK (ODEStepper.cpp:163-292) for `count` independent states
 * (x_in, x_out per state).  its_out (count ints, may be NULL) receives the
 * fixed-point iterations used, negated when the step did not converge. */
pcc_status pcc_irk_step(pcc_ctx* ctx, int ntau, double dim, int scheme, double precision, int max_its, int count,
                        const double* y_in, const double* x_in, const double* x_out, double* y_out, int* its_out);

/* InitialConditionGenerator::computeLeftExpansion / computeRightExpansion after
 * unpackSpectralFields, as NewtonSolver::shoot performs them (:408-415):
 * y_left and y_right are Ntau reals each. */
pcc_status pcc_boundary_data(pcc_solve* s, const double* in0, double* y_left, double* y_right);

/* ShootingSolver::integrateToMatchPoint (ShootingSolver.cpp:53-145) for
 * `count` states on the solve's grid; side 0 marches x_L -> x_M, side 1
 * x_R -> x_M. */
pcc_status pcc_sweep(pcc_solve* s, int count, const int* sides, const double* y_init, double* y_final,
                     pcc_stats* stats);

/* computeLeftExpansion / computeRightExpansion from time-domain fields
 * (InitialConditionGenerator.cpp:37-239, 252-667): y_left from (fc, psic),
 * y_right from up, at x_l / x_r with period delta.  Pass NULL to skip a side. */
pcc_status pcc_expansions(pcc_ctx* ctx, int ntau, double dim, double delta, double x_l, double x_r,
                          const double* fc, const double* psic, const double* up, double* y_left, double* y_right);

/* Allocation-free variant of pcc_expansions; it has no counterpart in the
 * reference.  For callers that may not allocate device memory once they are
 * running (a service that reserves its whole device-memory pool at start-up,
 * a library that must not trigger the device synchronisation cudaFree can
 * cause): the caller passes device pointers for the inputs (fc, psic, up:
 * Ntau doubles each) and outputs (y_left, y_right: Ntau doubles each; NULL
 * skips a side), and the work arrays live in a static device array compiled
 * into the library (1.3 MiB, kept by every GPU that loads the library until
 * the process exits), so Ntau is limited to 2048; larger values are rejected
 * with PCC_ERR_INVALID_ARG.  The call is asynchronous on the context stream
 * and allocates nothing.  It makes the context's device current for its
 * duration and restores the calling thread's current device before it
 * returns.  Its first call on a device looks up the array's device address;
 * make that first call before any stream capture.  All calls share the one
 * array, so calls that overlap on the GPU race. */
pcc_status pcc_expansions_static(pcc_ctx* ctx, int ntau, double dim, double delta, double x_l, double x_r,
                                 const double* d_fc, const double* d_psic, const double* d_up, double* d_y_left,
                                 double* d_y_right);

/* Spectral refinement of periodic fields for convergence studies (the
 * reference's scripts/create_simulation_data.py:37-58, double): count fields
 * of ntau_in samples (row-major) -> count x ntau_out samples, doubling
 * log2(ntau_out/ntau_in) times; powers of two, 4 <= ntau_in <= ntau_out <= 4096. */
pcc_status pcc_resample_fields(pcc_ctx* ctx, int ntau_in, int ntau_out, int count, const double* in, double* out);

/* The IRK march kernel's transform schedule for (Ntau, stages) on the
 * context's device, picked by this library's autotuner (no counterpart in the
 * reference): 1 = the independent transforms of an RHS evaluation run in
 * pairs, 0 = one at a time, 2 (Ntau 1024, 2 stages) = pairs of length-512
 * transforms with one of their two data exchanges inside a warp.  The first
 * solve of a shape times the schedules on a short single-RHS probe, keeps
 * pairs unless another schedule is more than 3 % faster, and caches the
 * choice ($PCC_AUTOTUNE_CACHE, default ~/.cache/pcc_b200/autotune.txt;
 * $PCC_AUTOTUNE=0 keeps pairs; $PCC_MARCH_SCHEDULE=0|1|2 forces a schedule
 * wherever the shape has it); this call tunes now if needed.
 * ms_pair/ms_single: probe times, 0 when read from the cache. */
pcc_status pcc_march_tuning(pcc_ctx* ctx, int ntau, int stages, int* pair, double* ms_pair, double* ms_single);

/* Replaces the solve's x-grid (NewtonSolver::generateGrid output) by grid,
 * NLeft + NRight + 1 points, as ShootingSolver::shoot accepts any gridX. */
pcc_status pcc_solve_set_grid(pcc_solve* s, const double* grid);

/* FFTW-convention DFT of `count` complex series of length n (power of two,
 * 2..4096), interleaved re/im: out[k] = sum_j in[j] exp(sign 2 pi i jk/n),
 * unscaled (SpectralTransformer.cpp:22-40 uses sign +1 as "forward"). */
pcc_status pcc_dft(pcc_ctx* ctx, int n, int count, int sign, const double* in, double* out);

/* InitialConditionGenerator::packSpectralFields / unpackSpectralFields
 * (InitialConditionGenerator.cpp:678-758): three Ntau-point series <-> the
 * Nnewton packed Fourier coefficients.  unpack reads z as given (the caller
 * zeroes the Delta slot as NewtonSolver::shoot does, :408-412). */
pcc_status pcc_pack_fields(pcc_ctx* ctx, int ntau, const double* up, const double* psic, const double* fc,
                           double* z);
pcc_status pcc_unpack_fields(pcc_ctx* ctx, int ntau, const double* z, double* up, double* psic, double* fc);

/* Measured FP64 FMA throughput of this device in TFLOP/s (a short probe). */
pcc_status pcc_fp64_peak(pcc_ctx* ctx, double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* PCC_H */
