/* msgpu.h -- C ABI of the B200 HSGeneral stochastic propagation library.
 *
 * This library replaces, for the stochastic static case, the body of the
 * HSGeneral time loop of MolSpin (RunSection/General/HS/TaskHSGeneral.cpp:
 * 471-560): per step the observable evaluation
 * (HSObservableCollector::Evaluate, HSObservableCollector.cpp:276-288), the
 * symmetric stochastic split (HSPropagator::StepStochastic,
 * HSPropagator.cpp:131-140) with its fixed-dimension Krylov step
 * (HSPropagator::Step Krylov branch, HSPropagator.cpp:64-78, i.e.
 * SpinSpace::KrylovExpmGeneral / ArnoldiProcess,
 * SpinAPI/SpinSpace/SpinSpace_operators.cpp:1257-1408) and the
 * singlet-triplet random-unitary noise (SpinAPI::ApplyStochasticRelaxationHilbert,
 * SpinAPI/SpinSpace/SpinSpace_relaxation.cpp:1211-1254), and afterwards the
 * trapezoid integration (HSObservableCollector::IntegrateFiniteTime,
 * HSObservableCollector.cpp:304-326).
 *
 * Everything the host side of MolSpin still builds -- the Hamiltonian
 * (HSHamiltonianBuilder), the Haberkorn operator K (HSReactionRelaxation),
 * the trace-sampled factors (HSStatePreparation) and the time grid -- is
 * handed over as plain arrays.  Complex numbers are interleaved (re, im)
 * doubles.  Every function returns MSGPU_OK (0) or an error code and fills
 * the context's message (msgpu_last_error), mirroring the reference's
 * bool + std::string &error convention (e.g. HSPropagator.cpp:51-102).
 *
 * Units follow the reference: H in rad/ns, rates in 1/ns, times in ns.
 */
#ifndef MSGPU_H
#define MSGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MSGPU_OK 0
#define MSGPU_ERR_INVALID 1   /* bad argument or missing input */
#define MSGPU_ERR_BUDGET 2    /* device memory budget of the context exceeded */
#define MSGPU_ERR_NONFINITE 3 /* a non-finite value appeared on the device */
#define MSGPU_ERR_EXPM 4      /* small matrix exponential failed (singular Pade denominator) */
#define MSGPU_ERR_CUDA 6      /* CUDA runtime error */
#define MSGPU_ERR_STATE 7     /* call out of order (e.g. run before upload) */

/* Precision forms. */
#define MSGPU_PREC_C128 0 /* plain form: complex128 everywhere (reference parity) */
#define MSGPU_PREC_C64 1  /* precision form: complex64 vectors and H, FP64 reductions, expm and sums */

/* Krylov recurrences. */
#define MSGPU_REC_AUTO 0    /* Arnoldi for C128; for C64 Lanczos with scalar K, else Arnoldi */
#define MSGPU_REC_ARNOLDI 1 /* Arnoldi on G = -iH - K (as SpinSpace::ArnoldiProcess).  C64
                               takes it when K acts on the electron pair only (K = I x K4,
                               e.g. unequal sinks on the pair's states: CGS2 with FP64 dots,
                               FP32 storage); any other K needs C128 */
#define MSGPU_REC_LANCZOS 2 /* Lanczos on H; valid only when K is a scalar */

/* Propagators. */
#define MSGPU_PROP_KRYLOV 0
/* Dense propagator for a static H of dimension <= 4096 (the reference's
 * "normal" expmat branch, HSPropagator.cpp:92-100): U = expm(dt(-iH-K)) is
 * built once in FP64 on the device and applied every step as a real
 * interleaved GEMM on the tensor cores (tcgen05, BF16 split operands, FP32
 * accumulation).  Precision must be MSGPU_PREC_BF16X3 (two-part split, three
 * products) or MSGPU_PREC_BF16X6 (three-part split, six products). */
#define MSGPU_PROP_DENSE 1
/* propagationmethod=autoexpm (HSPropagator.cpp:58-62 -> SpinSpace::HighamProp,
 * SpinSpace_operators.cpp:1028-1134): truncated Taylor series of
 * exp(dt(G - mu I)), G = -iH - K, mu = trace(G)/D, on s sub-steps with
 * s = ceil(dt ||G - mu I||_1 / 4) and the a-priori degree for the tolerance
 * MSGPU_OPT_TAYLOR_TOL; complex128 only, any K.  The reference picks (m, s)
 * from a random norm estimate; this choice is deterministic and no less
 * accurate. */
#define MSGPU_PROP_TAYLOR 2
/* propagationmethod=rk4 (HSPropagator.cpp:80-90): one classical RK4 step of
 * dB/dt = (-iH - K) B per time step, complex128, time-independent H; the
 * explicit method needs dt small against 1/||H||. */
#define MSGPU_PROP_RK4 3
#define MSGPU_PREC_BF16X3 2
#define MSGPU_PREC_BF16X6 3
/* Dense propagator with exact accumulation: U and the state are cut into four
 * int8 slices each (a power-of-two scale per row of U and per trajectory),
 * the ten slice products up to the fourth level run as tcgen05.mma kind::i8
 * with int32 accumulators (exact), and the levels are combined in FP64 into
 * an FP64 state.  No FP32 rounding enters the step. */
#define MSGPU_PREC_INT8X4 4

/* Options (msgpu_set_option). */
#define MSGPU_OPT_DENSE_RENORMALIZE 1 /* 1 (default): the dense form restores the exact
                                        Haberkorn survival |psi|^2 e^{-2 kappa t} of each
                                        trajectory every step (scalar K only); 0: off */
#define MSGPU_OPT_SPMM_VARIANT 3      /* -1 (default): the autotuner picks the complex64 SpMM
                                        variant and tile; k >= 0: tune the tile of variant k
                                        only (0-3 register-gather variants, 4-5 the variants
                                        that stage the tile's own quartets in shared memory,
                                        6-7 two trajectory pairs per thread, 8-9 the
                                        tensor-core SpMM over cubes of 16 / 8 quartets, 10
                                        the TMEM-staged SpMM (persistent, cubes of 8
                                        quartets x 256 trajectories, inputs through TMA,
                                        tcgen05.cp and tcgen05.ld); 8-10 need radical pairs
                                        whose other spins are all spin-1/2 and whose second
                                        electron stride is a multiple of the cube, and are
                                        refused with MSGPU_ERR_INVALID at the run
                                        otherwise);
                                        a forced variant also keeps the four-kernel Lanczos
                                        iteration */
#define MSGPU_OPT_TAYLOR_TOL 2        /* truncation tolerance of MSGPU_PROP_TAYLOR: 2^-53
                                        (default, "double"), 2^-24 ("single"), 2^-10 ("half") */
#define MSGPU_OPT_LANCZOS_CLUSTER 4   /* complex64 streamed form.  0 (default): per Krylov
                                        iteration one SpMM, one update and two reductions.
                                        -1: the whole Lanczos recurrence of a step as one
                                        cluster-resident launch (two trajectory pairs per
                                        thread-block cluster, their vectors in shared memory)
                                        with the smallest cluster of at most 16 CTAs that
                                        holds them (not while MSGPU_OPT_SPMM_VARIANT forces a
                                        variant); 1, 2, 4, 8 or 16: that cluster size only.
                                        Same results to FP32 rounding; at D=16384 with 1024
                                        trajectories on a B200 it is the slower of the two
                                        (latency-bound at one 512-thread CTA per SM) */
#define MSGPU_OPT_TRAJ_GROUPS 5       /* complex64 streamed form: 0 (default) splits a block of
                                        512 or more trajectories into 2 groups whose step
                                        sequences run on two streams, so that one group's SpMM
                                        (held by the SM's load pipe) overlaps the other's
                                        memory-bound update and combine; 1: one group; 2 or 4:
                                        that many groups when each is a multiple of 128
                                        trajectories.  Results do not depend on it. */
#define MSGPU_OPT_COMBINE_TILE 6      /* streamed forms: quartets per CTA of the evaluation and
                                        Krylov-combination kernels (and so the number of
                                        per-tile partial sums of the yields); 0 (default) picks
                                        it from the dimension.  Ensemble and per-trajectory
                                        yields change only by FP64 summation order. */

/* Execution forms (msgpu_set_form).  AUTO picks RESIDENT for small
 * dimensions (the whole time loop in one launch, one warp per trajectory,
 * Krylov basis in shared memory) and STREAMED otherwise (one kernel sequence
 * per step over the trajectory block, vectors in HBM). */
#define MSGPU_FORM_AUTO 0
#define MSGPU_FORM_STREAMED 1
#define MSGPU_FORM_RESIDENT 2

/* Noise modes for the singlet-triplet dephasing Operator. */
#define MSGPU_NOISE_NONE 0
#define MSGPU_NOISE_REPLAY 1 /* host-supplied flip bits (e.g. the reference's mt19937 stream) */
#define MSGPU_NOISE_PHILOX 2 /* on-device Philox4x32-10 keyed by (seed, trajectory, step, half) */

typedef struct msgpu_ctx msgpu_ctx;

typedef struct msgpu_run_params {
    const double *times;   /* time points t_0 < t_1 < ... (ns); one step per interval */
    int ntimes;            /* number of time points (steps = ntimes - 1) */
    int krylov_dim;        /* krylovsize (reference default 16, HSExecutionPlan.h:63); 1..32 */
    int precision;         /* MSGPU_PREC_* */
    int recurrence;        /* MSGPU_REC_* */
    int propagator;        /* MSGPU_PROP_KRYLOV */
    long long step_offset; /* global index of the first step (noise counters / replay bits) */
    int accumulate;        /* 0: start new yield integrals at times[0]; 1: continue the previous run */
} msgpu_run_params;

/* Create a context on CUDA device `device`; all device memory it allocates is
 * charged against hbm_budget_bytes (0 = no limit).  Returns NULL on failure. */
msgpu_ctx *msgpu_create(int device, size_t hbm_budget_bytes);
void msgpu_destroy(msgpu_ctx *ctx);
const char *msgpu_last_error(const msgpu_ctx *ctx);
/* Bytes of device memory currently held by the context. */
size_t msgpu_device_bytes(const msgpu_ctx *ctx);

/* Use an external cudaStream_t (NULL restores the context's own stream). */
int msgpu_set_stream(msgpu_ctx *ctx, void *cuda_stream);

/* Hamiltonian H (rad/ns) as CSR with int32 indices; val holds nnz complex
 * values.  Replaces the sp_cx_mat passed to HSPropagator::Step (HSPropagator.h:40-41). */
int msgpu_upload_hamiltonian_csr(msgpu_ctx *ctx, int dim, const int *rowptr, const int *col, const double *val);


/* H as a fixed-pattern linear combination H = sum_k coef_k H_k, 1 <= nterms
 * <= 16 (for example H_hf + Bx Zx + By Zy + Bz Zz: a new field direction or
 * strength changes only the coefficients -- the per-orientation Hamiltonian
 * of TaskHSGeneral.cpp:371-379 and SpinSpace_hamiltonians.cpp:780-1043 with
 * a sparsity pattern that does not change).  The terms share one CSR pattern
 * (rowptr, col; a term stores explicit zeros where the others have entries);
 * vals holds nterms blocks of nnz interleaved complex values.  The derived
 * device forms (complex64 copy, quartet blocks) are built once from the
 * pattern; msgpu_set_hamiltonian_coefficients then updates H on the device,
 * without host assembly or re-upload, and drops a cached dense propagator.
 * msgpu_upload_hamiltonian_csr leaves this mode. */
int msgpu_upload_hamiltonian_terms(msgpu_ctx *ctx, int dim, const int *rowptr, const int *col, int nterms,
                                   const double *vals, const double *coef);
int msgpu_set_hamiltonian_coefficients(msgpu_ctx *ctx, const double *coef);
/* Time-dependent H (dynamic interactions, TaskHSGeneral.cpp:486-560 with
 * HSHamiltonianBuilder::BuildAtTime): coef holds nsteps rows of nterms
 * coefficients, row j for global step first_step + j, evaluated by the caller
 * at that step's midpoint; each step of msgpu_run then propagates with
 * sum_k coef_k H_k, combined on the device.  Streamed Krylov and Taylor
 * propagators (RK4 takes msgpu_set_hamiltonian_schedule_rk4); the dense
 * propagator and the resident form need a static H.
 * nsteps = 0 clears the schedule. */
int msgpu_set_hamiltonian_schedule(msgpu_ctx *ctx, const double *coef, long long first_step, long long nsteps);
/* Time-dependent H for the RK4 propagator (HSPropagator::StepDynamicRK4,
 * HSPropagator.cpp:104-128, and StepDynamicRK4Stochastic, :142-150): RK4 on
 * dB/dt = G(t) B needs G at the start, midpoint and end of each step.  coef
 * holds 2 nsteps + 1 rows of nterms coefficients: row 2j at the start of
 * global step first_step + j, row 2j + 1 at its midpoint, row 2j + 2 at its
 * end (the next step's start).  The Krylov and Taylor propagators use the
 * midpoint rows of the same schedule.  K stays time-independent.  nsteps = 0
 * clears the schedule. */
int msgpu_set_hamiltonian_schedule_rk4(msgpu_ctx *ctx, const double *coef, long long first_step, long long nsteps);

/* K = kappa * I (symmetric recombination: kappa = k/2,
 * HSReactionRelaxation::BuildReactionForOrientation, HSReactionRelaxation.cpp:134-164). */
int msgpu_set_reaction_scalar(msgpu_ctx *ctx, double kappa);
/* General K as CSR (dimension of the uploaded H). */
int msgpu_upload_reaction_csr(msgpu_ctx *ctx, const int *rowptr, const int *col, const double *val);

/* Kronecker strides of the two spin-1/2 spins of the singlet-triplet pair in
 * the basis index (index = sum_k digit_k * stride_k, digit 0 = m=+1/2).  The
 * reference's basis follows the SpinSpace spin order (SpinSpace_management.cpp:37). */
int msgpu_set_electron_pair(msgpu_ctx *ctx, int stride1, int stride2);

/* Observables O = op (4x4, row-major, pair basis |e1 e2> = uu, ud, du, dd) on
 * the pair, identity elsewhere; each value is multiplied by `rate`
 * (transition yields rate * P_source, HSObservableCollector.cpp:101-127).
 * At most 8. */
int msgpu_clear_observables(msgpu_ctx *ctx);
int msgpu_add_pair_observable(msgpu_ctx *ctx, const double *op4x4, double rate);

/* Singlet-triplet dephasing Operator with rate st_rate (1/ns); the random
 * unitary U = PS - PT is applied with per-half-step probability
 * -expm1(-st_rate*h)/2 (SpinSpace_relaxation.cpp:1233).  For
 * MSGPU_NOISE_REPLAY, bits holds one bit per (step, half, trajectory) at
 * index (step*2 + half)*ntraj + t for nsteps steps.  Several dephasing
 * Operators on the same pair: st_rate = the sum of their rates.  Every
 * channel applies P_S - P_T, so the superposed-Poisson branch
 * (SpinSpace_relaxation.cpp:1239-1252) acts through the parity of its event
 * count alone, and the odd-parity probability at the summed rate is the
 * one-channel formula: MSGPU_NOISE_PHILOX then draws it on the device, and
 * msgpu_host_reference_flip_bits_multi gives the reference's own bits for
 * MSGPU_NOISE_REPLAY. */
int msgpu_set_st_noise(msgpu_ctx *ctx, double st_rate, int mode, unsigned long long seed,
                       const unsigned char *bits, long long nsteps, int ntraj);

/* Trajectory block: D x ntraj column-major complex (HSPreparedState factors,
 * HSStatePreparation.h:31-56, usually already scaled by 1/sqrt(M)). */
int msgpu_upload_factors(msgpu_ctx *ctx, int dim, int ntraj, const double *factors);
/* Same, from device memory (interleaved complex128, column-major D x ntraj). */
int msgpu_upload_factors_device(msgpu_ctx *ctx, int dim, int ntraj, const void *factors_device);
int msgpu_download_factors(msgpu_ctx *ctx, double *factors);

/* Run the stochastic finite-time loop over params->times (one orientation). */
int msgpu_run(msgpu_ctx *ctx, const msgpu_run_params *params);

/* Yield integrals so far: per trajectory (ntraj x nobs, trajectory-major) and
 * ensemble (sum over trajectories, nobs).  Either pointer may be NULL. */
int msgpu_fetch_yields(msgpu_ctx *ctx, double *per_traj, double *ensemble);
/* Ensemble observable values at each time point of the last run
 * ((ntimes) x nobs), the rows of orientationValues in TaskHSGeneral.cpp:470-482. */
int msgpu_fetch_values(msgpu_ctx *ctx, double *values);

/* Kernel timing with CUDA events on the launch stream.  Classes:
 * 0 apply (SpMM), 1 orth/update, 2 reductions, 3 expm, 4 combine, 5 yield,
 * 6 dense GEMM (tensor cores), 7 cluster-resident Lanczos recurrence (one
 * launch per step, MSGPU_OPT_LANCZOS_CLUSTER).  enable: 0 off; 1 every launch; 2 sampled --
 * every launch of every 32nd time step of the streamed step loop (whose
 * trajectory groups then run back to back, so each launch is timed alone),
 * and every 8th dense GEMM (events between kernels cost them their overlap,
 * so timing every launch slows a many-launch step by 10 % or more; the
 * sampled mode costs about 1 %).  msgpu_profile_read returns the total time and the
 * number of launches that time covers. */
int msgpu_profile_enable(msgpu_ctx *ctx, int enable);
int msgpu_profile_read(msgpu_ctx *ctx, int kernel_class, double *total_ms, long long *launches);

/* Select the execution form (MSGPU_FORM_*); RESIDENT falls back to an error
 * at run time if the Krylov basis of one trajectory does not fit shared memory. */
int msgpu_set_form(msgpu_ctx *ctx, int form);

/* Set an option (MSGPU_OPT_*). */
int msgpu_set_option(msgpu_ctx *ctx, int key, double value);
/* Read an option back; for MSGPU_OPT_TRAJ_GROUPS the number of groups the
 * current trajectory block runs in (once factors are uploaded). */
int msgpu_get_option(msgpu_ctx *ctx, int key, double *value);

/* ---------------------------------------------------------------- batching
 * Many spin systems of uneven dimension and trajectory count propagated by
 * ONE persistent launch (replayed from a CUDA graph): the loop over
 * orientations / field values / systems of a powder or sweep run
 * (TaskHSGeneral.cpp:347 orientation loop, RunSection::Step sweeps) with each
 * system's HSGeneral time loop inside the launch.  Precision form
 * (complex64 vectors, FP64 reductions and yield sums), Lanczos recurrence,
 * K = kappa I, Philox noise keyed by (seed, trajectory, step, half).
 * Systems with dimension >= the team threshold get a whole CTA per
 * trajectory, smaller ones a warp; msgpu_batch_tune picks the threshold and
 * the persistent grid size by timing the batch itself.  Systems of dimension
 * >= 2048 instead run the streamed single-system path (all trajectories in
 * lockstep through the quartet-block SpMM) on their own context and stream,
 * concurrently with the persistent launch; msgpu_batch_run returns when all
 * are done and its stats report the wall time of the whole run. */
typedef struct msgpu_batch msgpu_batch;
msgpu_batch *msgpu_batch_create(int device, size_t hbm_budget_bytes);
void msgpu_batch_destroy(msgpu_batch *batch);
const char *msgpu_batch_last_error(const msgpu_batch *batch);
/* Returns the system index (>= 0) or -MSGPU_ERR_*.  ops: nobs 4x4 pair
 * observables (as msgpu_add_pair_observable), factors: dim x ntraj
 * column-major complex (HSPreparedState factors). */
int msgpu_batch_add_system(msgpu_batch *batch, int dim, const int *rowptr, const int *col, const double *val,
                           double kappa, int stride1, int stride2, int nobs, const double *ops, const double *rates,
                           double st_rate, unsigned long long seed, int ntraj, const double *factors);
/* Drops every system of the batch (the team threshold and CTAs per SM of a
 * previous tune stay).  The device buffers of persistent-route systems are
 * kept and serve the next msgpu_batch_add_system calls, so a pooled batch
 * runs one group of systems after another without allocating or freeing
 * device memory; a streamed system's context is destroyed.  Waits for the
 * batch's stream.  Replaces nothing in the reference: its orientation and
 * RunSection loops hold no device state. */
int msgpu_batch_clear(msgpu_batch *batch);
int msgpu_batch_tune(msgpu_batch *batch, const double *times, int ntimes, int krylov_dim);
int msgpu_batch_run(msgpu_batch *batch, const double *times, int ntimes, int krylov_dim, long long step_offset,
                    int accumulate);
int msgpu_batch_fetch_yields(msgpu_batch *batch, int system, double *per_traj, double *ensemble);
int msgpu_batch_stats(const msgpu_batch *batch, double *last_run_ms, int *team_threshold, int *ctas_per_sm);
/* Kernels launched by the batch since creation (graph replays of the
 * persistent launch count once each), streamed systems included. */
long long msgpu_batch_launch_count(const msgpu_batch *batch);

/* Number of kernels this context launched since creation. */
long long msgpu_launch_count(const msgpu_ctx *ctx);

/* The complex64 SpMM this context's autotuner picked for its current
 * trajectory block: *variant in the numbering of MSGPU_OPT_SPMM_VARIANT,
 * *tile the quartets per CTA, *groups the trajectory groups of the step;
 * all -1 before the first complex64 streamed run.  No counterpart in the
 * reference (a tuning report). */
int msgpu_spmm_choice(const msgpu_ctx *ctx, int *variant, int *tile, int *groups);

/* System i of a batch: *streamed = 1 when it runs the streamed single-system
 * path on its own context (dimension >= 2048), 0 inside the persistent
 * launch; for a streamed system the SpMM its own tuner picked
 * (msgpu_spmm_choice), else -1.  No counterpart in the reference. */
int msgpu_batch_system_info(const msgpu_batch *batch, int system, int *streamed, int *variant, int *tile, int *groups);

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (for example an embedding host framework whose memory pool owns
 * all device memory, or code on a latency-critical path that must not take
 * the implicit device synchronisation of cudaMalloc / cudaFree): one Krylov step psi_out = exp(dt (-iH - kappa I)) psi_in for
 * every trajectory column, computed with the complex128 Arnoldi kernels of
 * msgpu_run, using only the caller's buffers and a fixed static scratch area
 * of MSGPU_NOALLOC_SCRATCH_BYTES compiled into this library (held on every
 * GPU that loads it, until the process exits).  It calls no cudaMalloc or
 * cudaFree.
 *   - rowptr/col/val (CSR of H in rad/ns, val interleaved complex128),
 *     psi_in and psi_out (dim x ntraj column-major complex128) are DEVICE
 *     pointers; psi_in and psi_out must not overlap.  dim must be a multiple
 *     of 4 (a radical pair is always present).
 *   - Problems whose working set does not fit the scratch area are rejected
 *     with MSGPU_ERR_SCRATCH before any work is queued; with krylov_dim 16 the
 *     area holds, e.g., dim 64 with up to 512 trajectories.
 *   - No call can be captured into a CUDA graph: every call copies its status
 *     to the host and waits on `stream` (cudaStreamSynchronize) before it
 *     returns, which a capturing stream refuses (and the capture is lost).
 *   - The first call on a device looks up the scratch address on that device
 *     (cudaGetSymbolAddress).  Later calls reuse the address and look it up
 *     again only when it no longer names live device memory (after a
 *     cudaDeviceReset).
 *   - A CUDA error that is already pending when the call starts is left in
 *     place for the caller and reported as MSGPU_ERR_CUDA; nothing is queued.
 *   - All calls share the one scratch area: calls that may overlap on the GPU
 *     (different streams, or several host threads) race and must be
 *     serialised by the caller.
 * Work is queued on `stream` (a cudaStream_t; NULL = legacy default stream)
 * and the call waits for it to finish. */
#define MSGPU_ERR_SCRATCH 8
#define MSGPU_NOALLOC_SCRATCH_BYTES (16u << 20)
int msgpu_krylov_step_noalloc(int dim, const int *rowptr, const int *col, const double *val, double kappa,
                              int ntraj, const double *psi_in, double *psi_out, double dt, int krylov_dim,
                              void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MSGPU_H */
