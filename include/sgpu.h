/*
 * sgpu.h — C ABI of the B200 (sm_100a) SIMPLE solver for the 2D lid-driven cavity.
 *
 * This is the drop-in boundary for simple-hpc's `backend = gpu` path. In the reference that path is
 * the C++ class `HipSolver` and the function `run_simple_hip` (include/simple/solver_hip.hpp:11-40,
 * src/hip/solver_hip.hip:369-550), called from src/main.cpp:40-46. Every entry point below names the
 * reference member or function it replaces.
 *
 * Conventions
 *  - Plain C: ints, doubles, pointers and sizes. No C++ or CUDA types cross this boundary.
 *  - Every function returns an int status: SGPU_OK (0) or a negative SGPU_E* code. Nothing throws.
 *    sgpu_last_error() returns the message of the last failure on the calling host thread. The
 *    reference throws std::runtime_error("GPU error: ...") from HIP_CHECK (solver_hip.hip:17-23) and
 *    "backend = gpu supports ..." from the HipSolver constructor (solver_hip.hip:373-377); the host
 *    driver turns a non-zero status back into that exception so `simple` still exits 1.
 *  - Host fields are full-grid row-major arrays of nrows x ncols doubles (nrows = NX + 2H + 1,
 *    ncols = NY + 2H + 1), element (i, j) at i * ncols + j, halos included: the layout of the
 *    reference's Field2D (include/simple/field2d.hpp:36-65).
 *  - A handle owns all of its device memory and one CUDA stream. One handle per host thread.
 */
#ifndef SGPU_H
#define SGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
enum {
    SGPU_OK = 0,
    SGPU_E_INVALID = -1,     /* bad argument, unsupported solver combination, bad config */
    SGPU_E_CUDA = -2,        /* a CUDA runtime call failed (message holds cudaGetErrorString) */
    SGPU_E_NOMEM = -3,       /* a device allocation failed */
    SGPU_E_TIMEOUT = -4,     /* a bounded device-side wait ran out (persistent kernels; the mixed
                                mode's correction sweep waiting for its record copies) */
    SGPU_E_NONFINITE = -5,   /* a residual became NaN or Inf: sgpu_run stopped the diverged run */
    SGPU_E_NODEVICE = -6     /* no CUDA device is visible */
};

/* ---- enumerations: the values of the reference's config keys (include/simple/params.hpp:9-13) ---- */
enum { SGPU_UDS = 0, SGPU_QUICK = 1 };                                   /* convection_scheme */
enum { SGPU_NORM_ABSOLUTE = 0, SGPU_NORM_RUNNING_MAX = 1 };              /* residual_normalisation */
enum { SGPU_BACKEND_SERIAL = 0, SGPU_BACKEND_OPENMP = 1, SGPU_BACKEND_GPU = 2 };
enum { SGPU_MOM_GS_LEX = 0, SGPU_MOM_JACOBI = 1, SGPU_MOM_GS_MULTICOLOUR = 2 };
enum { SGPU_P_GS_LEX = 0, SGPU_P_JACOBI = 1, SGPU_P_GS_REDBLACK = 2, SGPU_P_CG = 3, SGPU_P_MG = 4 };
/* Keys of this build only (the reference rejects them as unknown keys). */
enum { SGPU_PREC_FP64 = 0, SGPU_PREC_MIXED = 1 };                        /* precision */
enum { SGPU_MG_FIXED = 0, SGPU_MG_TOLERANCE = 1 };                       /* mg_mode */

/*
 * Parameters: the reference's struct Params (include/simple/params.hpp:15-58) as plain data.
 * Fill it with sgpu_params_from_config(), which applies make_params (src/params.cpp:50-180):
 * the same keys, defaults, validation and error messages, and the same derived values.
 */
typedef struct sgpu_params {
    int NX, NY;                 /* N_cells_x (rows), N_cells_y (columns) */
    int H, N_halo_x, N_halo_y;
    double Re;
    int maxit_inner_u, maxit_inner_v, maxit_inner_p;
    double error_tolerance;
    int maxit;
    double relaxation_factor_u, relaxation_factor_v, relaxation_factor_p;
    int convection_scheme;      /* SGPU_UDS / SGPU_QUICK */
    int diffusion_order;        /* 2 or 4 */
    int hybrid_switch;          /* always 0: the reference rejects True */
    int residual_normalisation; /* SGPU_NORM_* */
    int backend;                /* SGPU_BACKEND_* */
    int momentum_solver;        /* SGPU_MOM_* */
    int pressure_solver;        /* SGPU_P_* */
    double pressure_tolerance;  /* cg: ||r|| / ||b|| target; mg_mode = tolerance: the same for MG */
    int pressure_maxit;         /* cg iteration cap; mg_mode = tolerance: V-cycle cap */
    int mg_cycles, mg_pre, mg_post;
    double mg_omega;
    int halo_overlap, write_fields;
    int grid_rows_cfg, grid_cols_cfg; /* mpi_grid (accepted and stored; one GPU has one block) */
    /* keys of this build */
    int precision;              /* SGPU_PREC_FP64 (default) or SGPU_PREC_MIXED */
    int mg_mode;                /* SGPU_MG_FIXED (default: the reference) or SGPU_MG_TOLERANCE */
    int warm_start;             /* 0: p' starts at 0 (reference); 1: learned warm start (sgpu_cnn_*) */
    int graph_batch;            /* outer iterations per CUDA-graph launch in sgpu_run (0 = auto) */
    /* derived (make_params, src/params.cpp:174-178) */
    int nrows, ncols;
    double dx, dy, nu;
    char output_dir[512];
    char cnn_weights[512];      /* key cnn_weights: path of a trained warm-start network */
    char restart_from[512];     /* key restart_from: directory of u.csv, v.csv, p.csv to start from */
} sgpu_params_t;

/*
 * Parse config text ("key = value" lines, '#' comments; src/config.cpp:16-39) and build the
 * parameters (src/params.cpp:50-180). On failure returns SGPU_E_INVALID and the reference's
 * message (e.g. "config line 3: duplicate key 'Re'", "unknown config key: foo").
 */
int sgpu_params_from_config(const char* text, sgpu_params_t* out);
/* Defaults of struct Params with the derived values filled (NX = NY = 80). */
int sgpu_params_default(sgpu_params_t* out);
/* Recompute nrows, ncols, dx, dy, nu and validate (the tail of make_params). */
int sgpu_params_finalize(sgpu_params_t* p);

const char* sgpu_last_error(void);
const char* sgpu_version(void);

/* ---- field identifiers for sgpu_download / sgpu_upload (every array of the reference's State) ---- */
enum {
    SGPU_F_U = 0, SGPU_F_V = 1, SGPU_F_P = 2,
    /* u-momentum coefficients, reference order AE AW AN AS AEE AWW ANN ASS AP (coefficients.hpp:5-7) */
    SGPU_F_CU_AE = 3, SGPU_F_CU_AW, SGPU_F_CU_AN, SGPU_F_CU_AS, SGPU_F_CU_AEE, SGPU_F_CU_AWW,
    SGPU_F_CU_ANN, SGPU_F_CU_ASS, SGPU_F_CU_AP,
    SGPU_F_CV_AE = 12, SGPU_F_CV_AW, SGPU_F_CV_AN, SGPU_F_CV_AS, SGPU_F_CV_AEE, SGPU_F_CV_AWW,
    SGPU_F_CV_ANN, SGPU_F_CV_ASS, SGPU_F_CV_AP,
    /* PressureWork (include/simple/pressure.hpp:7-11) */
    SGPU_F_AEP = 21, SGPU_F_AWP, SGPU_F_ANP, SGPU_F_ASP, SGPU_F_APP, SGPU_F_B, SGPU_F_PC,
    SGPU_F_COUNT = 28
};

/* Phases of the reference's PhaseTimers (include/simple/timer.hpp:6-20). */
enum {
    SGPU_PH_ASSEMBLE_U = 0, SGPU_PH_BC_U, SGPU_PH_RESIDUAL_U, SGPU_PH_SWEEP_U,
    SGPU_PH_ASSEMBLE_V, SGPU_PH_BC_V, SGPU_PH_RESIDUAL_V, SGPU_PH_SWEEP_V,
    SGPU_PH_ASSEMBLE_P, SGPU_PH_SOLVE_P, SGPU_PH_CORRECT, SGPU_PH_OUTPUT, SGPU_PH_COUNT
};

typedef struct sgpu_handle sgpu_handle;

/*
 * Create a solver: allocate every device array and upload u, v, p (each may be NULL = zeros).
 * Replaces HipSolver::HipSolver (solver_hip.hip:369-408). Accepted combinations: momentum_solver
 * gs_multicolour or jacobi with pressure_solver gs_redblack, jacobi, cg or mg (the reference GPU
 * accepts gs_multicolour + gs_redblack only); gs_lex is rejected with the reference's message.
 */
int sgpu_create(const sgpu_params_t* p, const double* u, const double* v, const double* pf,
                sgpu_handle** out);
/* Free the handle and its device memory. Replaces HipSolver::~HipSolver (solver_hip.hip:410-415). */
int sgpu_destroy(sgpu_handle* h);

/*
 * Per-phase entry points: same order and semantics as the CPU functions the reference's
 * outer_iteration calls (src/solver.cpp:27-93) and as HipSolver's members (solver_hip.hip:417-499).
 * They run the reference-shaped kernels, which also materialise the 9 + 9 coefficient arrays, so a
 * per-phase test can download and compare every array. Each call completes before it returns.
 */
int sgpu_assemble_u(sgpu_handle* h);                /* HipSolver::assemble_u / assemble_u (momentum_u.cpp:8) */
int sgpu_bc_u(sgpu_handle* h);                      /* HipSolver::bc_u / apply_bc_u (momentum_u.cpp:24) */
int sgpu_residual_u(sgpu_handle* h, double* res);   /* HipSolver::residual_u / residual_u (momentum_u.cpp:43) */
int sgpu_sweep_u(sgpu_handle* h, int nsweeps);      /* HipSolver::sweep_u / sweep_u_batch (momentum_u.cpp:162) */
int sgpu_assemble_v(sgpu_handle* h);                /* assemble_v (momentum_v.cpp:9) */
int sgpu_bc_v(sgpu_handle* h);                      /* apply_bc_v (momentum_v.cpp:24) */
int sgpu_residual_v(sgpu_handle* h, double* res);   /* residual_v (momentum_v.cpp:36) */
int sgpu_sweep_v(sgpu_handle* h, int nsweeps);      /* sweep_v_batch (momentum_v.cpp:164) */
int sgpu_assemble_p(sgpu_handle* h, double* res);   /* HipSolver::assemble_p / assemble_p (pressure.cpp:14) */
int sgpu_solve_p(sgpu_handle* h);                   /* HipSolver::solve_p / solve_pc_* (solver.cpp:65-76) */
int sgpu_correct(sgpu_handle* h);                   /* HipSolver::correct / correct (pressure.cpp:136) */

/*
 * One outer iteration on the fused fast path (bit-identical to the per-phase path in FP64).
 * res[3] = res_u, res_v, res_p. phase_seconds (may be NULL) accumulates per-phase device time
 * (SGPU_PH_COUNT doubles) measured with CUDA events. Replaces HipSolver::outer_iteration
 * (solver_hip.hip:501-523).
 */
int sgpu_outer_iteration(sgpu_handle* h, double res[3], double* phase_seconds);

/* Result of sgpu_run: the reference's RunResult (include/simple/solver.hpp:32-45). */
typedef struct sgpu_result {
    int iterations;
    int converged;
    double seconds;                  /* wall time of the loop, like run_outer_loop's steady_clock */
    double phase_seconds[SGPU_PH_COUNT];
    long long cg_iterations;         /* pressure_solver = cg: CG iterations over all outer iterations */
    long long mg_vcycles;            /* pressure_solver = mg: V-cycles over all outer iterations */
} sgpu_result_t;

/*
 * Run the outer loop with the reference's stopping rule (run_outer_loop, src/solver.cpp:106-132):
 * stop when max(res_u, res_v, res_p) (running_max-normalised if configured) <= error_tolerance and
 * iter > 1, or at maxit. log (may be NULL) receives 4 doubles per iteration
 * [iter, res_u, res_v, res_p] and must hold 4 * maxit doubles. If print_every > 0, the
 * reference's "iter k  res_u ..." lines are printed at iteration 1 and every print_every
 * iterations. Replaces run_simple_hip's loop (solver_hip.hip:538-550).
 * A residual that becomes NaN or Inf stops the run after that iteration: *result and log cover the
 * iterations run, and the call returns SGPU_E_NONFINITE (the reference has no such test and runs a
 * diverged case on to maxit).
 */
int sgpu_run(sgpu_handle* h, int maxit, double* log, int print_every, sgpu_result_t* result);

/* Copy one device array to a host nrows x ncols buffer. Replaces HipSolver::download. */
int sgpu_download(sgpu_handle* h, int field_id, double* host);
/* Copy a host nrows x ncols buffer into one device array (tests, restarts). */
int sgpu_upload(sgpu_handle* h, int field_id, const double* host);
/* Device bytes held by the handle. */
int sgpu_memory_bytes(sgpu_handle* h, size_t* bytes);
/* Diagnostic of the device-side failure detection (no counterpart in the reference): one warp on the
 * current device waits, at most `polls` polls (1 .. 1 << 20), on an mbarrier that nothing completes,
 * through the same bounded-wait helper the mixed mode's correction sweep uses. *gave_up = 1 when the
 * wait ended by giving up and reported it, as it must; the GPU context stays usable. */
int sgpu_selftest_bounded_wait(int polls, int* gave_up);
/* Number of multigrid levels and the dims of level l (mg_level_dims, multigrid.cpp:143-151). */
int sgpu_mg_levels(int NX, int NY, int* nlevels, int* dims /* 2 * 64 ints, may be NULL */);
/* Statistics of the last solve_p: CG iterations, MG V-cycles, coarsest-level sweeps. */
int sgpu_last_solve_stats(sgpu_handle* h, int* cg_iterations, int* mg_vcycles,
                          int* coarse_sweeps, double* rel_residual);

/*
 * Ordered sum on the device: sum of values[r * ncols_v + c] over r < nrows_v, c < ncols_v, each row
 * added left to right from 0.0, then the row sums top to bottom from 0.0: the fixed order of the
 * reference's CellSums (src/decomp.cpp:176-205) and det_sum (src/multigrid.cpp:18-34). values is a
 * host array; the call copies it to the device, sums there and returns the sum in *out.
 */
int sgpu_ordered_sum(const double* values, int nrows_v, int ncols_v, double* out);

/*
 * The same ordered sum for callers that cannot allocate device memory (no counterpart in the
 * reference). values and out are DEVICE pointers: nrows_v rows of ncols_v doubles, row k starting
 * at values + k * ld; *out receives the sum. stream is a cudaStream_t (NULL = legacy default). The
 * call allocates nothing: its scratch is a fixed array inside the library (16384 rows at most;
 * larger blocks are refused with SGPU_E_INVALID), fetched per device by the first call made on that
 * device, which should come before any stream capture. That address is kept for the life of the
 * process: a cudaDeviceReset after the first call on a device is not supported. The call is
 * asynchronous on stream; calls that overlap on the GPU (other streams, other host threads) share
 * that scratch and race, so serialise them.
 */
int sgpu_ordered_sum_noalloc(const double* values, int nrows_v, int ncols_v, int ld, double* out,
                             void* stream);

/*
 * Instrumentation. With profiling on, every outer iteration records CUDA events between its phases
 * on the handle's stream and accumulates the device time per phase (sgpu_phase_seconds, indexed by
 * SGPU_PH_*), the way the reference's PhaseTimers accumulate wall time (include/simple/timer.hpp).
 * sgpu_stream returns the handle's cudaStream_t (as void*) so a caller can time on it.
 * sgpu_launch_count returns the number of kernel launches this library has issued in the process.
 * sgpu_sweep_seconds returns the device time of the streaming momentum sweep kernels alone (the
 * FP64 sweep, or the FP32 correction sweep with precision = mixed) and how many were launched, both
 * accumulated over the profiled iterations: the per-launch time of the dominant kernel.
 */
/* on: 0 off; 1 every iteration host-issued between events (exact per-phase device times, slower);
 * 2 sampled: sgpu_run times the phases of its first 10 iterations that way, replays the captured
 * graph for the rest (the fast path; same iterations and bits) and scales the sampled phase times
 * to the whole run. 2 is what a drop-in caller that writes timing.csv should use. */
int sgpu_set_profiling(sgpu_handle* h, int on);
int sgpu_phase_seconds(sgpu_handle* h, double* out /* SGPU_PH_COUNT */);
int sgpu_sweep_seconds(sgpu_handle* h, double* seconds, long long* launches);
int sgpu_stream(sgpu_handle* h, void** stream);
long long sgpu_launch_count(void);

/*
 * Write the reference's output files into p->output_dir from host arrays: u.csv, v.csv, p.csv,
 * ux_centre.csv, uy_centre.csv (when write_fields), alog.csv, timing.csv, run_info.json, in the
 * reference's formats (write_outputs, src/io.cpp:43-151; cell_centre, :22-31). log holds
 * 4 doubles per iteration as sgpu_run writes it. Runs on the host only.
 */
int sgpu_write_outputs(const sgpu_params_t* p, const double* u, const double* v, const double* pf,
                       const double* log, int iterations, const sgpu_result_t* result,
                       const char* cfg_path, const char* git_hash, const char* compiler);

/*
 * Restart (key restart_from; the reference always starts from u = v = p = 0): read u.csv, v.csv and
 * p.csv from dir into host arrays of nrows x ncols, the files sgpu_write_outputs writes (full arrays,
 * halos included, %.18e: the values round-trip exactly). A run restarted from the files of a run of
 * k iterations continues with the fields of iteration k. Runs on the host only; a file with the
 * wrong shape or an unparsable value is an SGPU_E_INVALID error naming it.
 */
int sgpu_read_fields(const sgpu_params_t* p, const char* dir, double* u, double* v, double* pf);

/* ---- learned warm start for p' (keys warm_start, cnn_weights) ----
 *
 * The reference has no learned part: p' starts at zero before every solve (multigrid.cpp:349-354,
 * pressure.cpp:114-134). With a network attached (warm_start = cnn, sgpu_cnn_load or
 * sgpu_attach_cnn) and pressure_solver = mg, each p' solve first runs the network on the finest
 * multigrid level of at most max_size x max_size cells (inputs: that level's restricted b and its
 * diagonal AP), injects the guess down to the fine grid and starts the V-cycles from it. The
 * multigrid is unchanged: with mg_mode = tolerance it iterates to the same tolerance as from zero.
 * A guess whose residual is not below ||b|| is discarded (the cycles start from zero, counted as a
 * fallback).
 *
 * Network: U-Net of `levels` levels, `base` channels on the finest (doubling per level), 3x3
 * convolutions with ReLU, 2x2 average pooling, nearest upsampling with skip concatenation, 1x1
 * head; BF16 weights and activations, FP32 accumulation on the tensor cores; FP32 master weights
 * trained with Adam on the mean-squared error. Images are n x height x width with 2 FP32 input
 * channels interleaved per pixel (b / rms(b), AP / mean(AP) - 1) and 1 FP32 output channel (p' *
 * mean(AP) / rms(b)); height and width must be multiples of 2^(levels-1).
 */
typedef struct sgpu_cnn sgpu_cnn;
/* Load or replace the network of a handle from a weights file (sgpu_cnn_write), cnn_max 256. */
int sgpu_cnn_load(sgpu_handle* h, const char* path);
int sgpu_cnn_create(int base, int levels, unsigned seed, sgpu_cnn** out);
int sgpu_cnn_read(const char* path, sgpu_cnn** out);
int sgpu_cnn_write(sgpu_cnn* c, const char* path);
int sgpu_cnn_destroy(sgpu_cnn* c);
int sgpu_cnn_info(sgpu_cnn* c, int* base, int* levels, long long* num_params, double* flops_per_pixel);
/* FP32 master parameters: per convolution W[cout][9][cin] then bias[cout], in network order (encoder
 * levels finest first, two convolutions each; decoder levels coarsest first, the first of each pair
 * with cin = its upsampled input + the skip); then the head's base weights and its bias. */
int sgpu_cnn_get_params(sgpu_cnn* c, float* host);
int sgpu_cnn_set_params(sgpu_cnn* c, const float* host);
int sgpu_cnn_forward(sgpu_cnn* c, const float* in, int n, int height, int width, float* out);
/* Loss (mean-squared error against target) and, if grads is not null, its gradient with respect to
 * every parameter (layout of sgpu_cnn_get_params). */
int sgpu_cnn_loss_grad(sgpu_cnn* c, const float* in, const float* target, int n, int height, int width,
                       float* loss, float* grads);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on one batch; *loss = the batch loss before the step. */
int sgpu_cnn_train_step(sgpu_cnn* c, const float* in, const float* target, int n, int height, int width,
                        float lr, float* loss);
/* Attach a network to a handle (not owned: keep it alive while attached; NULL detaches). */
int sgpu_attach_cnn(sgpu_handle* h, sgpu_cnn* c, int max_size);
/* Switch the handle's multigrid stopping mode (keys mg_mode, pressure_tolerance, pressure_maxit)
 * between outer iterations, e.g. to solve p' tightly only where a training pair is sampled. */
int sgpu_set_mg_mode(sgpu_handle* h, int mg_mode, double pressure_tolerance, int pressure_maxit);
/* Warm starts applied, guesses discarded, and the residual ||b - A p'|| / ||b|| after the first
 * V-cycle from the last guess. */
int sgpu_warm_start_stats(sgpu_handle* h, long long* used, long long* fallbacks, double* rel_initial);
/* Training pair from the handle's last p' solve (precision = fp64, pressure_solver = mg): the
 * network input of the finest level of at most max_size x max_size cells (nx x ny x 2) and the
 * normalised block mean of the solved p' on it (nx x ny). With in or target NULL only *nx, *ny and
 * *level are returned. Run the solves with mg_mode = tolerance and a tight pressure_tolerance so
 * the target is the converged p'. */
int sgpu_cnn_sample(sgpu_handle* h, int max_size, float* in, float* target, int* nx, int* ny, int* level);

/* ---- batched cavities (sgpu_batch_*) ----
 *
 * Many independent cavities, each with its own parameters (size, Re, schemes, precision), solved in
 * one graph launch: a WHILE node repeats one batch iteration while any cavity is active; inside it
 * each cavity's outer iteration (captured from its own solver) sits under an IF node that runs it
 * only while that cavity is active, and a final kernel applies the reference's stopping rule
 * (run_outer_loop, solver.cpp:117-129) to every cavity on the device. A cavity therefore stops at
 * exactly the iteration a single sgpu_run would, with the same fields. Supported per cavity: every
 * momentum solver; pressure_solver gs_redblack, jacobi or mg with mg_mode = fixed; no warm start.
 * The reference has no batched mode; a batch of one behaves like sgpu_run.
 */
typedef struct sgpu_batch sgpu_batch;
int sgpu_batch_create(const sgpu_params_t* params /* count */, int count, sgpu_batch** out);
int sgpu_batch_destroy(sgpu_batch* b);
int sgpu_batch_count(sgpu_batch* b, int* count);
/* Autotuner: per distinct grid, times the candidate row-segment heights of the streaming momentum
 * sweep and keeps the fastest (chosen[count], 0 for cavities without that sweep; may be NULL). The
 * segment height changes no result bit. Call before sgpu_batch_run. */
int sgpu_batch_autotune(sgpu_batch* b, int* chosen);
/* Run every cavity to its tolerance or maxit iterations from its current fields. log_cap > 0 keeps
 * the first log_cap (iteration, res_u, res_v, res_p) rows of every cavity (sgpu_batch_log).
 * *seconds = device time of the launch. */
int sgpu_batch_run(sgpu_batch* b, int maxit, int log_cap, double* seconds);
/* Per cavity: iterations run, converged flag (1 converged, 0 not, -1 stopped because a residual became
 * NaN or Inf), last res_u, res_v, res_p (3 per cavity). */
int sgpu_batch_results(sgpu_batch* b, int* iterations, int* converged, double* residuals);
/* count x log_cap x 4 doubles; rows past a cavity's iteration count are zero. */
int sgpu_batch_log(sgpu_batch* b, double* host);
int sgpu_batch_download(sgpu_batch* b, int index, int field_id, double* host);

#ifdef __cplusplus
}
#endif
#endif /* SGPU_H */
