/*
 * qa_gpu.h -- C ABI of the B200 Monte Carlo sweep engine (libqa_gpu.so).
 *
 * This is the drop-in boundary for qanneal's sweep engine.  In qanneal every
 * annealer drives a model through the per-flip Backend interface
 * (include/qanneal/backend.hpp:39-53); BackendKind::CUDA is parsed
 * (backend.hpp:19-27) but make_backend() throws "CUDA backend stub: kernels
 * not wired yet." (backend.hpp:97-102).  A per-flip virtual call cannot cross
 * to a device, so the boundary sits one level up: each entry point below runs
 * one whole annealer run*() call -- for ALL reads of a solve() at once -- and
 * returns the same result fields as the annealer's result struct.
 *
 * Conventions: plain C types, caller-owned host buffers, int status codes
 * (QA_OK == 0), the message of the last failure on this thread through
 * qa_last_error().  No exception crosses this boundary.  One qa_ctx per host
 * thread; calls on one context are serialised by the caller (qanneal's
 * annealers are not re-entrant either: rng_ is a member).
 *
 * Randomness: read r of a call uses the stream keyed by (seed + r), as
 * solve() seeds read r with set_seed(seed + r) (python/qanneal/solver.py:679-681).
 */
#ifndef QA_GPU_H
#define QA_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define QA_API __attribute__((visibility("default")))
#else
#define QA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    QA_OK = 0,
    QA_ERR_ARG = 1,         /* invalid argument (qanneal: std::invalid_argument -> ValueError) */
    QA_ERR_CUDA = 2,        /* CUDA runtime failure */
    QA_ERR_OOM = 3,         /* device allocation failed */
    QA_ERR_TIMEOUT = 4,     /* a bounded device wait ran out */
    QA_ERR_DRIFT = 5,       /* incremental fields drifted from a float64 recompute */
    QA_ERR_UNSUPPORTED = 6  /* option outside the engine (cluster sweeps, observers) */
};

typedef struct qa_ctx qa_ctx;
typedef struct qa_problem qa_problem;

/* Library identity and errors. */
QA_API const char *qa_version(void);
/* Copies the last error message of the calling thread into buf (NUL-terminated). */
QA_API int qa_last_error(char *buf, size_t len);
QA_API int qa_device_count(int *count);

/* Context: one device, one stream, a cached device workspace.
 * Replaces make_backend(BackendKind::CUDA, ham) (backend.hpp:92-105). */
QA_API int qa_create(qa_ctx **out, int device);
QA_API int qa_destroy(qa_ctx *ctx);

/* Field-drift check of the incremental local-field updates (the property
 * tests/test_higher_order_ising.cpp:149-167 checks for the reference's float64
 * cache).  tolerance > 0: every later SA, SQA and SQA-PT call on this context
 * recomputes the float32 field caches in float64 after the run, reports the
 * largest deviation in qa_stats.max_field_drift and returns QA_ERR_DRIFT when
 * it exceeds the tolerance (outputs are written either way).  Kernels with
 * exact integer fields (+-1 dense, integer sparse) report 0.  tolerance <= 0
 * (the default): off. */
QA_API int qa_set_drift_check(qa_ctx *ctx, double tolerance);

/* Update order of the SQA and SQA-PT sweeps (qa_sqa_run, qa_sqa_opt_run,
 * qa_sqapt_run, qa_sqapt_opt_run and the traced SQA run).
 * QA_ORDER_REFERENCE (the default) is qanneal's order: before every slice,
 * cluster and worldline sweep of a replica a fresh uniformly random spin
 * order (the std::shuffle of sqa_annealer.cpp:181,216,295 and
 * sqa_parallel_tempering.cpp:209,224,281), the Trotter slices swept one after
 * another, t = 0 .. P-1, each in that order; the engine then samples the
 * reference's Markov chain, so finite-time statistics (best-energy
 * distributions, ground-state probabilities) match the reference's.
 * QA_ORDER_CHECKERBOARD sweeps the slices in parity phases (even, odd) with
 * the spins ascending, the order qanneal's SQAChiAnnealer uses
 * (sqa_chi_annealer.cpp:68-140): the same stationary distribution, faster on
 * the GPU, different finite-time dynamics.  SQA-Chi always keeps its
 * checkerboard, SA and classical parallel tempering their ascending order.
 * A pipeline wait that runs out (it cannot in a correct run) makes the call
 * return QA_ERR_TIMEOUT. */
enum { QA_ORDER_CHECKERBOARD = 0, QA_ORDER_REFERENCE = 1 };
QA_API int qa_set_update_order(qa_ctx *ctx, int order);
QA_API int qa_get_update_order(const qa_ctx *ctx, int *order);

/* Launch-shape overrides of a context, for the autotuner (no counterpart in
 * the reference: its loops have no launch shape).  Every choice leaves the
 * results unchanged bit for bit; it moves only time.  0 / -1 is automatic.
 *   warps_per_ring: warps of a ring's CTA (1..32, at most P; automatic:
 *                   ceil(P/2));
 *   field_form:     the dense +-1 kernel's ring state: 0 int32 fields and the
 *                   coupling bits in shared memory, 1 int16 fields and the
 *                   bits in shared memory, 2 int16 fields and the bits read
 *                   through L2 (a form that does not fit falls back to the
 *                   automatic order of the three);
 *   rotate:         0 whole-grid launches, 1 rotated ring groups whenever the
 *                   rings outnumber the SMs, -1 when whole-grid waves would
 *                   leave slots idle;
 *   rot_steps:      steps per rotated launch;
 *   rot_group:      rings per rotated group (at most 128 groups). */
typedef struct {
    int warps_per_ring;
    int field_form;
    int rotate;
    int rot_steps;
    int rot_group;
} qa_tuning;
QA_API int qa_set_tuning(qa_ctx *ctx, const qa_tuning *tuning);  /* NULL: all automatic */
QA_API int qa_get_tuning(const qa_ctx *ctx, qa_tuning *tuning);

/* ---- problems (device copies of one model instance) ------------------- */

/* DenseIsing(h, J, n, c) (dense_ising.hpp:17-21): E = c + sum h s + sum_{i<j} J_ij s_i s_j.
 * J is n*n row-major float64; the couplings read are the upper triangle, as in
 * DenseIsing::energy (dense_ising.cpp:29-44). */
QA_API int qa_problem_dense(qa_ctx *ctx, int n, const double *h, const double *J, double c, qa_problem **out);

/* QUBO(Q, n).to_ising() (qubo.cpp:33-69) built on the device: Q is the n*n
 * row-major float64 matrix on the host; W = (Q + Q^T)/2, J = W/2, h = W.1/2
 * are formed by device kernels straight into the problem's device block, the
 * constant c = tr(W)/4 + 1^T W 1/4 (one running sum, the reference's order) on
 * the host meanwhile.  The result is the DenseIsing the reference converts to,
 * bit for bit.  h_out [n] and c_out (either may be NULL) receive h and c. */
QA_API int qa_problem_qubo(qa_ctx *ctx, int n, const double *Q, double *h_out, double *c_out, qa_problem **out);

/* SparseIsing(h, edges, n, c) (sparse_ising.hpp:22-25); edge e couples ei[e], ej[e]
 * with weight w[e]; self-edges are rejected (sparse_ising.cpp:29-31). */
QA_API int qa_problem_sparse(qa_ctx *ctx, int n, const double *h, int m, const int64_t *ei, const int64_t *ej,
                      const double *w, double c, qa_problem **out);

/* HigherOrderIsing after its constructor's consolidation (higher_order_ising.cpp:10-90):
 * h[n] holds the folded degree-1 terms, c the folded constant, and term t
 * (0 <= t < n_terms) couples term_vars[term_ptr[t] .. term_ptr[t+1]) -- strictly
 * increasing indices, degree >= 2 -- with coefficient coeff[t]. */
QA_API int qa_problem_hubo(qa_ctx *ctx, int n, const double *h, int n_terms, const int64_t *term_ptr,
                    const int32_t *term_vars, const double *coeff, double c, qa_problem **out);

QA_API int qa_problem_free(qa_problem *p);
QA_API int qa_problem_size(const qa_problem *p, int *n);

/* ---- results ------------------------------------------------------------
 * One qa_run_out per problem of a call; every pointer is a caller-owned host
 * array and may be NULL when the field is not wanted. */
typedef struct {
    int8_t *best_spins;      /* [reads][n]   best_state per read (+1/-1) */
    double *best_energy;     /* [reads]      float64 energy of best_state */
    double *energy_trace;    /* [reads][steps] energy_trace (SA: energy after the step;
                                SQA: mean over replicas x slices) */
} qa_run_out;

/* Totals of one call, for measurement.  May be NULL. */
typedef struct {
    int64_t slice_attempts, slice_accepts;          /* SA: spin attempts / accepts */
    int64_t worldline_attempts, worldline_accepts;  /* proposals (each covers P sites) */
    double sweep_ms;                                /* device time of the sweep kernels (CUDA events) */
    double total_ms;                                /* device time of the whole call */
    int64_t launches;                               /* kernels launched by the call */
    int64_t sweep_launches;                         /* of which sweep-kernel launches */
    int64_t h2d_bytes, d2h_bytes;                   /* host<->device bytes moved by the call */
    double max_field_drift;                         /* with a drift check on (qa_set_drift_check): the
                                                       largest |cached float32 local field - float64
                                                       recompute from the same couplings| over every
                                                       replica, slice and spin after the run; else 0 */
} qa_stats;

/* ---- SA: Annealer::run (annealer.cpp:33-75) ------------------------------ */
typedef struct {
    const double *betas;     /* [steps]  AnnealSchedule::betas */
    int steps;
    int sweeps_per_beta;     /* > 0 */
    int reads;               /* independent reads per problem */
    uint64_t seed;           /* read r keyed by seed + r */
} qa_sa_params;

QA_API int qa_sa_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sa_params *params,
              qa_run_out *outs, qa_stats *stats);

/* ---- SA replicas: ReplicaAnnealer::run (replica_annealer.cpp:46-142) -------
 * params->reads = replicas; replica r is SA read r (keyed seed + r).  Besides
 * qa_sa_run's outputs: the magnetisation after each step and the step whose
 * sweeps last lowered each replica's best energy (-1: the starting state),
 * from which the caller picks the global best as the reference does (lowest
 * energy, then earliest step, then lowest replica). */
typedef struct {
    int8_t *best_spins;              /* [replicas][n] */
    double *best_energy;             /* [replicas] */
    double *energy_trace;            /* [replicas][steps] */
    double *magnetization_trace;     /* [replicas][steps] */
    int32_t *best_step;              /* [replicas] */
} qa_replica_out;

QA_API int qa_replica_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems,
                          const qa_sa_params *params, qa_replica_out *outs, qa_stats *stats);

/* ---- SQA: SQAAnnealer::run (sqa_annealer.cpp:87-477) ---------------------- */
typedef struct {
    const double *betas;     /* [steps]  SQASchedule */
    const double *gammas;    /* [steps] */
    int steps;
    int trotter_slices;      /* P > 0 */
    int replicas;            /* K > 0 rings per read */
    int sweeps_per_beta;     /* slice sweeps per step */
    int worldline_sweeps;    /* worldline sweeps per step */
    int cluster_sweeps;      /* imaginary-time cluster sweeps per step (P <= 64) */
    int continuous_time_slices; /* slices = max(P, this) when larger, as in the reference */
    int reads;
    uint64_t seed;
} qa_sqa_params;

QA_API int qa_sqa_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sqa_params *params,
               qa_run_out *outs, qa_stats *stats);

/* ---- SQA with the calibrated chi_B schedule: SQAAnnealer::run_optimal
 *      (sqa_annealer.cpp:499-952) ---------------------------------------------
 * Phase 1: beta ramped from beta_ramp_start to beta over beta_ramp_fraction
 * of the steps at J_perp = j_perp_start.  Then, when eps_tilde <= 0, a
 * calibration pilot (calib_probes probes of calib_sweeps sweeps from the
 * post-ramp state, which is restored afterwards) measures chi_B(J_perp) =
 * Var(bond sum) and sets the J_perp trajectory of phase 2 (inverse of the
 * integral of chi_B^alpha); with eps_tilde > 0, J_perp advances online by
 * eps_tilde * chi_B^-alpha after every step.  Phase 2 runs at the cold beta.
 * The slices' Trotter coupling is J_perp itself (no Gamma). */
typedef struct {
    int trotter_slices;
    int replicas;
    double beta;
    double j_perp_start;
    double j_perp_end;             /* > j_perp_start */
    double eps_tilde;              /* <= 0: calibrate */
    double alpha;
    int num_steps;
    int sweeps_per_step;
    int worldline_sweeps;
    int cluster_sweeps;            /* P <= 64 when > 0 */
    int calib_probes;
    int calib_sweeps;
    double beta_ramp_fraction;
    double beta_ramp_start;
    int reads;
    uint64_t seed;
} qa_sqaopt_params;

typedef struct {
    int8_t *best_spins;        /* [reads][n] */
    double *best_energy;       /* [reads] */
    double *energy_trace;      /* [reads][num_steps] average energy over replicas and slices */
    double *j_perp_trace;      /* [reads][num_steps] */
    double *chi_B_trace;       /* [reads][num_steps] the chi_B that drove each step */
    double *scalars;           /* [reads][4] calibrated_eps_tilde, j_perp_start, resolved_j_perp_end, final_j_perp */
} qa_sqaopt_out;

QA_API int qa_sqa_opt_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems,
                          const qa_sqaopt_params *params, qa_sqaopt_out *outs, qa_stats *stats);

/* ---- observers: Annealer::run / SQAAnnealer::run with an observer
 *      (annealer.cpp:48-71, sqa_annealer.cpp:318-473) --------------------------
 * The run is the same as qa_sa_run / qa_sqa_run (identical results); the sweep
 * kernels also write a strided trace into a device buffer, read back once at
 * the end.  A sweep is recorded when its index within its phase of the step is
 * a multiple of stride.  Every output pointer may be NULL (not recorded). */
typedef struct {
    int stride;              /* >= 1 */
    int8_t *states;          /* [reads][steps][rps][n] the state after each recorded sweep, rps = ceil(sweeps_per_beta/stride) */
    double *energies;        /* [reads][steps][rps] the running energy after each recorded sweep */
    int8_t *step_states;     /* [reads][steps][n] the state at each step end */
    double *magnetization;   /* [reads][steps] mean spin at each step end */
} qa_sa_trace;

QA_API int qa_sa_trace_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sa_params *params,
                           const qa_sa_trace *traces, qa_run_out *outs, qa_stats *stats);

/* rps = ceil(sweeps_per_beta/stride) + ceil(cluster_sweeps/stride) + ceil(worldline_sweeps/stride); the
 * records of a step are the slice, then the cluster, then the worldline sweeps. */
typedef struct {
    int stride;              /* >= 1 */
    int8_t *ring_states;     /* [reads][replicas][steps][rps][P][n] each replica after each recorded sweep */
    double *ring_energies;   /* [reads][replicas][steps][rps][P] its slice energies */
    int8_t *step_states;     /* [reads][replicas][steps + 1][P][n] each replica at the start (0) and each step end */
    double *step_energies;   /* [reads][replicas][steps + 1][P] */
    double *magnetization;   /* [reads][steps] mean spin over replicas, slices and spins at each step end */
} qa_sqa_trace;

QA_API int qa_sqa_trace_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems,
                            const qa_sqa_params *params, const qa_sqa_trace *traces, qa_run_out *outs,
                            qa_stats *stats);

/* ---- SQA parallel tempering: SQAParallelTemperingAnnealer::run
 *      (sqa_parallel_tempering.cpp:81-346) ----------------------------------
 * rungs (beta_r, Gamma_r) pairs, one Trotter ring per rung, swaps of
 * neighbouring rungs every swap_interval steps. */
typedef struct {
    const double *betas;     /* [rungs] */
    const double *gammas;    /* [rungs] */
    int rungs;               /* >= 2 */
    int trotter_slices;
    int sweeps_per_step;     /* slice sweeps per step */
    int worldline_sweeps;
    int steps;               /* pt_steps */
    int swap_interval;       /* > 0 */
    int cluster_sweeps;      /* imaginary-time cluster sweeps per step (P <= 64) */
    int continuous_time_slices;
    int reads;
    uint64_t seed;
} qa_sqapt_params;

typedef struct {
    int8_t *best_spins;              /* [reads][n] */
    double *best_energy;             /* [reads] */
    int8_t *final_spins;             /* [reads][rungs][n]  final_states */
    double *final_energies;          /* [reads][rungs]     projected energies (min over slices) */
    double *average_energy_trace;    /* [reads][steps] */
    double *swap_acceptance_trace;   /* [reads][steps] */
} qa_sqapt_out;

QA_API int qa_sqapt_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems,
                        const qa_sqapt_params *params, qa_sqapt_out *outs, qa_stats *stats);

/* ---- SQA-PT adaptive schedule: SQAParallelTemperingAnnealer::run_optimal
 *      (sqa_parallel_tempering.cpp:348-882) ----------------------------------
 * Every rung keeps its beta_r and runs at one schedule J_perp per step,
 * starting at the hottest rung's coupling J(beta_0, Gamma_0).  eps_tilde <= 0:
 * calib_probes chi_B probes from the starting states fix eps_tilde and a
 * J_perp trajectory spanning num_steps; eps_tilde > 0: J += eps_tilde *
 * chi_B^-alpha after every step.  Swaps use the classical action (the shared
 * Trotter terms cancel).  Outputs as qa_sqapt_out plus the schedule traces. */
typedef struct {
    const double *betas;     /* [rungs] */
    const double *gammas;    /* [rungs] (J_start and the default J_end only) */
    int rungs;               /* >= 2 */
    int trotter_slices;
    int continuous_time_slices;
    int sweeps_per_step;
    int worldline_sweeps;
    int cluster_sweeps;      /* P <= 64 when > 0 */
    int num_steps;           /* > 0 */
    int swap_interval;       /* > 0 */
    double eps_tilde;        /* <= 0: calibrate */
    double alpha;
    double j_perp_end;       /* <= 0: the coldest rung's coupling */
    int calib_probes;
    int calib_sweeps;
    int reads;
    uint64_t seed;
} qa_sqaptopt_params;

typedef struct {
    qa_sqapt_out pt;           /* best / final states and energies, average energy and swap traces */
    double *j_perp_trace;      /* [reads][num_steps] */
    double *chi_B_trace;       /* [reads][num_steps] */
    double *scalars;           /* [reads][4] calibrated_eps_tilde, j_perp_start, resolved_j_perp_end, final_j_perp */
} qa_sqaptopt_out;

QA_API int qa_sqapt_opt_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems,
                            const qa_sqaptopt_params *params, qa_sqaptopt_out *outs, qa_stats *stats);

/* ---- classical parallel tempering: ParallelTemperingAnnealer::run
 *      (parallel_tempering.cpp:36-122) --------------------------------------
 * One replica per beta, Metropolis sweeps, swaps of neighbouring replicas
 * every swap_interval steps.  Outputs as qa_sqapt_out (final energies are the
 * replicas' energies). */
typedef struct {
    const double *betas;     /* [rungs] */
    int rungs;               /* >= 2 */
    int sweeps_per_step;     /* > 0 */
    int steps;               /* > 0 */
    int swap_interval;       /* > 0 */
    int reads;
    uint64_t seed;
} qa_pt_params;

QA_API int qa_pt_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_pt_params *params,
                     qa_sqapt_out *outs, qa_stats *stats);

/* ---- SQA-Chi: SQAChiAnnealer::run_chi (sqa_chi_annealer.cpp:146-438) -----
 * Stage 1, the pilot chi_B scan (scan_points fresh worldlines per read, all
 * reads and points in one launch); Stage 2, the schedule built from the curve
 * (host, float64, as the reference does); Stage 3, the production anneal.
 * With scan_chi_in != NULL, Stage 1 is skipped and scan_chi_in
 * [reads][scan_points] is used as the chi_B curve of each read (a predicted
 * curve; the learned-schedule path). */
typedef struct {
    int trotter_slices;
    int replicas;
    double beta, gamma_start, gamma_end;
    int num_steps;            /* >= 2 */
    int sweeps_per_step;      /* > 0 */
    int scan_points;          /* >= 4 */
    int scan_sweeps;          /* > 0 */
    int scan_burn;
    double chi_floor_fraction;
    double driver_A0;         /* <= 0: gamma_start */
    double beta_ramp_fraction;
    double beta_ramp_start;
    int reads;
    uint64_t seed;
    const double *scan_chi_in;
} qa_chi_params;

typedef struct {
    int8_t *best_spins;       /* [reads][n] */
    double *best_energy;      /* [reads] */
    double *energy_trace;     /* [reads][num_steps] mean slice energy per step */
    double *beta_schedule;    /* [reads][num_steps] */
    double *gamma_schedule;   /* [reads][num_steps] */
    double *s_schedule;       /* [reads][num_steps] */
    double *scan_s;           /* [reads][scan_points] */
    double *scan_gamma;       /* [reads][scan_points] */
    double *scan_chi_B;       /* [reads][scan_points] */
    double *scalars;          /* [reads][5]: s_star, gamma_star, j_perp_star, chi_floor, driver_A0 */
} qa_chi_out;

QA_API int qa_chi_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_chi_params *params,
                      qa_chi_out *outs, qa_stats *stats);

/* Stage 1 alone (sqa_chi_annealer.cpp:217-281): scan_chi[(problem*reads + read)*scan_points + point]
 * (the training curves of the chi_B MLP).  num_steps, sweeps_per_step and the
 * schedule fields of params are ignored. */
QA_API int qa_chi_pilot(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_chi_params *params,
                        double *scan_chi, qa_stats *stats);

/* ---- chi_B-curve MLP (no counterpart in the reference: it replaces Stage 1
 * of run_chi, sqa_chi_annealer.cpp:217-281, with a predicted curve) --------
 * dims[0] -> ... -> dims[n_dims-1], ReLU between layers; bfloat16 weights,
 * float32 accumulation and float32 Adam masters.  The output holds M means and
 * M log-variances (dims[last] = 2M) of a Gaussian over the M-point target; the
 * loss is the mean Gaussian negative log-likelihood.  Inputs X [batch][dims[0]],
 * targets T [batch][M], outputs Y [batch][2M] are host float32 arrays.
 * Parameters: per layer W[d_l][d_l+1] row-major, then b[d_l+1]. */
typedef struct qa_mlp qa_mlp;
QA_API int qa_mlp_create(qa_ctx *ctx, const int *dims, int n_dims, uint64_t seed, qa_mlp **out);
QA_API int qa_mlp_free(qa_mlp *m);
QA_API int qa_mlp_num_params(const qa_mlp *m, int64_t *count);
QA_API int qa_mlp_get_params(qa_mlp *m, float *params, int64_t count);
QA_API int qa_mlp_set_params(qa_mlp *m, const float *params, int64_t count);  /* also resets Adam */
QA_API int qa_mlp_forward(qa_mlp *m, const float *X, int batch, float *Y);
/* loss of (X, T) and its gradient w.r.t. every parameter (grads may be NULL) */
QA_API int qa_mlp_loss_grad(qa_mlp *m, const float *X, const float *T, int batch, float *loss, float *grads);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the batch; loss before the step */
QA_API int qa_mlp_train_step(qa_mlp *m, const float *X, const float *T, int batch, float lr, float *loss);

/* ---- SA on a dense model without any allocation by this library --------
 * No counterpart in the reference.  For callers that cannot let a library
 * call cudaMalloc/cudaFree: their device memory belongs to a framework
 * allocator (PyTorch's caching allocator, JAX/XLA reserving most of HBM) or
 * to a fixed serving budget, so an allocation inside the call could fail or
 * stall them.  The caller passes device pointers: d_h[n], d_J[n*n] (float64,
 * as for qa_problem_dense) and the outputs d_best_spins[reads*n] (int8),
 * d_best_energy[reads], d_energy_trace[reads*steps]; params->betas stays a
 * host array.  The run is the same as qa_sa_run's (bit for bit) and uses a
 * 16 MiB static device array as scratch (held by every GPU that loads the
 * library until exit); runs needing more (about 4 n^2 + 8 reads n +
 * 4 steps bytes) are rejected with QA_ERR_ARG.  The first call on a device
 * looks up that array's device address: make it before any stream capture.
 * With CUDA's default lazy module loading that first call is also when the
 * 16 MiB are reserved on the device: make it (a small warm-up run) before a
 * framework claims most of the memory, or set CUDA_MODULE_LOADING=EAGER.
 * The call runs on `device` and restores the caller's current device before
 * it returns.
 * Calls share the array, so calls that overlap on the GPU race; serialise
 * them.  stream may be NULL (the legacy default stream); the call returns
 * after the run has finished on it.  stats may be NULL (counters only). */
QA_API int qa_sa_dense_run_noalloc(int device, void *stream, int n, const double *d_h, const double *d_J, double c,
                                   const qa_sa_params *params, int8_t *d_best_spins, double *d_best_energy,
                                   double *d_energy_trace, qa_stats *stats);

/* ---- measurement ---------------------------------------------------------
 * No counterpart in the reference: the L2 read bandwidth of `device`, the
 * denominator of the sweep kernels' L2 roofline.  A buffer of `bytes`
 * (1 MiB .. 96 MiB, small enough to stay in L2) is read `passes` times with
 * 16-byte L2-only loads by a grid of eight 256-thread CTAs per SM after one
 * warm pass; *gbs = bytes * passes / device time (CUDA events).  Allocates
 * and frees its own buffer; restores the caller's current device. */
QA_API int qa_probe_l2_read(int device, size_t bytes, int passes, double *gbs);

#ifdef __cplusplus
}
#endif

#endif /* QA_GPU_H */
