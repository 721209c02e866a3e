/*
 * tmnb: C ABI of the B200 (sm_100a) nonbonded potential.
 *
 * Drop-in boundary for timemachine's Nonbonded hot path. Each entry point
 * below names the reference interface it replaces (paths relative to the
 * timemachine source tree). Conventions shared by all entry points:
 *
 *  - Device pointers are plain CUDA device addresses; `stream` is a
 *    cudaStream_t passed as void* (0 = legacy default stream).
 *  - A NULL output pointer means "do not compute" that output; it selects the
 *    kernel variant (timemachine/cpp/src/nonbonded_all_pairs.cu:375-379).
 *  - Outputs ACCUMULATE (+=) in the reference's int64 fixed-point encoding
 *    (du_dx, u, du_dl and du_dcharge at 2^36; du_dsigma at 2^37; du_depsilon
 *    at 2^38; timemachine/cpp/src/fixed_point.hpp:3-8). The caller zeroes
 *    them (timemachine/cpp/src/potential.cu:141-157).
 *  - du_dl and u are per-atom buffers of length N whose SUM is the result
 *    (timemachine/cpp/src/wrap_kernels.cpp:596-601); the per-atom split itself is
 *    not part of the contract.
 *  - Parameters are [N,3] (or [2N,3] for interpolated potentials, lambda=0
 *    block first) doubles: charge * sqrt(138.935456), sigma/2, sqrt(epsilon).
 *  - Every call returns a tmnb_status; tmnb_last_error() gives the message of
 *    the last failing call on the calling thread. No call aborts the process
 *    (the reference calls exit() on CUDA errors, timemachine/cpp/src/gpu_utils.cuh:12-20).
 *  - A handle is not thread-safe (timemachine/cpp/src/potential.hpp:7): use
 *    one handle per stream/thread.
 */
#ifndef TMNB_H
#define TMNB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tmnb_potential tmnb_potential;

/* Lambda windows evaluated together by one multi-window call. */
#define TMNB_MAX_WINDOWS 32

typedef enum tmnb_status {
    TMNB_OK = 0,
    TMNB_ERR_INVALID_ARGUMENT = 1,
    TMNB_ERR_CUDA = 2,
    TMNB_ERR_NONORTHO_BOX = 3,  /* "Provided non-ortholinear box, unable to compute nonbonded energy" */
    TMNB_ERR_BOX_TOO_SMALL = 4, /* "Cutoff with padding is more than half of the box width, ..." */
    TMNB_ERR_UNSUPPORTED = 5,
    TMNB_ERR_INTERNAL = 6
} tmnb_status;

/* Message of the last failing call on this thread ("" if none). */
const char *tmnb_last_error(void);

/* Library version string. */
const char *tmnb_version(void);

/*
 * NonbondedAllPairs: every pair of the atom set (all N atoms, or the subset
 * atom_idxs[0..K) when atom_idxs != NULL) within cutoff, through a tile
 * neighbour list. Replaces the constructor
 * timemachine/cpp/src/nonbonded_all_pairs.cu:16-141 as bound at
 * timemachine/cpp/src/wrap_kernels.cpp:835-893 (NonbondedAllPairs_f32 and
 * NonbondedAllPairsInterpolated_f32, and the _f64 forms). precision: 32
 * (FP32 pair arithmetic, bit-exact to the reference's _f32 kernels) or 64
 * (FP64 pair arithmetic, the reference's _f64 kernels; 16-row tiles only).
 * The lambda transforms start as the identity ("lambda"), the reference
 * default; tmnb_potential_set_lambda_transforms sets others. The same
 * precision values apply to every nonbonded constructor below.
 */
tmnb_status tmnb_all_pairs_create(
    int N,
    const int32_t *lambda_plane_idxs,  /* [N] host */
    const int32_t *lambda_offset_idxs, /* [N] host */
    double beta,
    double cutoff,
    const int32_t *atom_idxs, /* [K] host, unique, or NULL */
    int K,
    int interpolated,
    int precision,
    tmnb_potential **out);

/*
 * NonbondedPairList / NonbondedPairListNegated: the listed pairs only, each
 * scaled by (charge_scale, lj_scale), subtracted when negated != 0. Replaces
 * timemachine/cpp/src/nonbonded_pair_list.cu:10-75 as bound at
 * timemachine/cpp/src/wrap_kernels.cpp:962-1013.
 */
tmnb_status tmnb_pair_list_create(
    int N,
    const int32_t *pair_idxs, /* [M,2] host */
    const double *scales,     /* [M,2] host: (charge_scale, lj_scale) */
    int M,
    const int32_t *lambda_plane_idxs,  /* [N] host */
    const int32_t *lambda_offset_idxs, /* [N] host */
    double beta,
    double cutoff,
    int negated,
    int interpolated,
    int precision,
    tmnb_potential **out);

/*
 * Nonbonded: all pairs minus the scaled exclusions, in ONE device pipeline
 * (one neighbour list, the exclusion pairs fused into the pair kernel's
 * launch). Replaces timemachine/lib/potentials.py:269-301, i.e.
 * FanoutSummedPotential([NonbondedAllPairs, NonbondedPairListNegated]),
 * and its interpolated form (timemachine/lib/potentials.py:333-344).
 */
tmnb_status tmnb_nonbonded_create(
    int N,
    const int32_t *exclusion_idxs, /* [M,2] host */
    const double *scales,          /* [M,2] host */
    int M,
    const int32_t *lambda_plane_idxs,  /* [N] host */
    const int32_t *lambda_offset_idxs, /* [N] host */
    double beta,
    double cutoff,
    int interpolated,
    int precision,
    tmnb_potential **out);

/* Releases all device memory of the handle (NULL is a no-op). */
tmnb_status tmnb_potential_destroy(tmnb_potential *pot);

/*
 * Device entry: replaces the virtual Potential::execute_device
 * (timemachine/cpp/src/potential.hpp:51-62). No host synchronisation and no
 * allocation happen inside; the neighbour-list rebuild decision is taken on
 * the device, so the call can be captured in a CUDA graph. Box errors are
 * recorded on the device; read them with tmnb_potential_check_device_error.
 */
tmnb_status tmnb_potential_execute_device(
    tmnb_potential *pot,
    int N,
    int P,
    const double *d_x,   /* [N,3] */
    const double *d_p,   /* [P] */
    const double *d_box, /* [3,3] */
    double lambda,
    unsigned long long *d_du_dx, /* [N,3] or NULL */
    unsigned long long *d_du_dp, /* [P] or NULL */
    unsigned long long *d_du_dl, /* [N] or NULL */
    unsigned long long *d_u,     /* [N] or NULL */
    void *stream);

/*
 * Host entry: replaces Potential::execute_host
 * (timemachine/cpp/src/potential.cu:110-185): copies the host inputs in,
 * zeroes and computes the selected outputs, copies them out and
 * synchronises. Outputs are OVERWRITTEN (not accumulated), as in the
 * reference. Device staging buffers are owned by the handle and reused.
 */
tmnb_status tmnb_potential_execute_host(
    tmnb_potential *pot,
    int N,
    int P,
    const double *h_x,
    const double *h_p,
    const double *h_box,
    double lambda,
    unsigned long long *h_du_dx,
    unsigned long long *h_du_dp,
    unsigned long long *h_du_dl,
    unsigned long long *h_u);

/*
 * Replaces the NonbondedInteractionGroup constructors
 * (timemachine/cpp/src/wrap_kernels.cpp:895-960,
 * timemachine/cpp/src/nonbonded_interaction_group.cu:19-158): pairs (i, j)
 * with i among the NR row atoms and j among the other N - NR atoms, no
 * exclusions. row_atom_idxs must be non-empty, unique, < N and fewer than N
 * ("row_atom_idxs must be nonempty", "atom indices must be unique", "number
 * of idxs must be less than N", "indices values must be less than N").
 * interpolated != 0: P = 2*N*3 (NonbondedInteractionGroupInterpolated).
 */
tmnb_status tmnb_interaction_group_create(
    int N,
    const int32_t *row_atom_idxs, /* [NR] */
    int NR,
    const int32_t *lambda_plane_idxs,  /* [N] */
    const int32_t *lambda_offset_idxs, /* [N] */
    double beta,
    double cutoff,
    int interpolated,
    int precision,
    tmnb_potential **out);

/*
 * Multi-window device entry (no single reference counterpart: replaces the
 * loop over lambda windows that execute_selective_batch
 * (timemachine/cpp/src/wrap_kernels.cpp:381-551) and multiple_steps_U
 * (timemachine/cpp/src/context.cu:139-234) run with one execute_device per
 * window). Evaluates K lambda windows (1 <= K <= TMNB_MAX_WINDOWS) of the same coordinates
 * and parameters in one launch sequence; window k's outputs start at
 * d_du_dx + 3*N*k, d_du_dp + P*k, d_du_dl + N*k, d_u + N*k and ACCUMULATE
 * (+=), as execute_device does. Each window's result equals that of
 * tmnb_potential_execute_device at lambdas[k], bit for bit. `lambdas` is a
 * HOST array.
 */
tmnb_status tmnb_potential_execute_windows_device(
    tmnb_potential *pot,
    int N,
    int P,
    const double *d_x,
    const double *d_p,
    const double *d_box,
    int K,
    const double *lambdas,       /* [K], host memory */
    unsigned long long *d_du_dx, /* [K,N,3] or NULL */
    unsigned long long *d_du_dp, /* [K,P] or NULL */
    unsigned long long *d_du_dl, /* [K,N] or NULL */
    unsigned long long *d_u,     /* [K,N] or NULL */
    void *stream);

/*
 * Host form of tmnb_potential_execute_windows_device, with the copy-in /
 * overwrite / copy-out / synchronise behaviour of tmnb_potential_execute_host.
 */
tmnb_status tmnb_potential_execute_windows_host(
    tmnb_potential *pot,
    int N,
    int P,
    const double *h_x,
    const double *h_p,
    const double *h_box,
    int K,
    const double *lambdas,       /* [K] */
    unsigned long long *h_du_dx, /* [K,N,3] or NULL */
    unsigned long long *h_du_dp, /* [K,P] or NULL */
    unsigned long long *h_du_dl, /* [K,N] or NULL */
    unsigned long long *h_u);    /* [K,N] or NULL */

/*
 * Batched host entry: replaces Potential::execute_batch_host behind
 * execute_selective_batch (timemachine/cpp/src/wrap_kernels.cpp:381-551).
 * Executes every (coords, params, lambda) combination; outputs have the
 * leading shape [coord_batches, param_batches, lambda_batches]. The lambda
 * windows of one (coords, params) pair run as one multi-window evaluation
 * (32 windows at a time).
 */
tmnb_status tmnb_potential_execute_batch_host(
    tmnb_potential *pot,
    int coord_batches,
    int N,
    int param_batches,
    int P,
    int lambda_batches,
    const double *h_x,       /* [coord_batches,N,3] */
    const double *h_p,       /* [param_batches,P] */
    const double *h_boxes,   /* [coord_batches,3,3] */
    const double *h_lambdas, /* [lambda_batches] */
    unsigned long long *h_du_dx,
    unsigned long long *h_du_dp,
    unsigned long long *h_du_dl,
    unsigned long long *h_u);

/* Fixed-point du_dp to float with per-column exponents
 * (timemachine/cpp/src/nonbonded_all_pairs.cu:435-450). */
tmnb_status tmnb_potential_du_dp_fixed_to_float(
    tmnb_potential *pot, int N, int P, const unsigned long long *du_dp, double *du_dp_float);

/* timemachine/cpp/src/nonbonded_all_pairs.cu:180-187 */
tmnb_status tmnb_potential_set_nblist_padding(tmnb_potential *pot, double padding);
tmnb_status tmnb_potential_disable_hilbert_sort(tmnb_potential *pot);

/* Synchronises `stream`, returns (and clears) a box error recorded by the
 * device since the last check. */
tmnb_status tmnb_potential_check_device_error(tmnb_potential *pot, void *stream);

/* Diagnostics of the last neighbour-list build (synchronises `stream`):
 * tiles, work items and the number of rebuilds so far. */
tmnb_status tmnb_potential_nblist_stats(
    tmnb_potential *pot, void *stream, int *n_tiles, int *n_items, int *n_rebuilds);

/* Neighbour-list introspection (timemachine/cpp/src/neighborlist.cu:81-124
 * get_nblist_host serves the same tests): S slots, RB = ceil(S/32) row
 * blocks, tile storage of tile_capacity tiles. copy_nblist synchronises and
 * copies the slot order perm[S] (slot -> atom), the tile count of every row
 * block [RB] and the column slots of all tiles [tile_capacity*32]; row block
 * rb owns the tiles starting at rb*RB - rb*(rb-1)/2. Any pointer may be NULL. */
tmnb_status tmnb_potential_nblist_shape(tmnb_potential *pot, int *S, int *RB, long long *tile_capacity);

/*
 * Rows per tile of the neighbour list (no reference counterpart; the
 * reference's tiles are 32 rows x 32 columns): 16 (default), 32 or 8 slots per
 * row group. A tile is always 32 column atoms; smaller row groups occupy
 * smaller regions and list fewer out-of-range pairs, at more tiles. The
 * results are identical; the next call rebuilds the list. nblist_rows reports
 * the row-group size and the number of 32-slot column blocks, with which row
 * group g owns the tiles from
 *   m * (b*CB - b*(b-1)/2) + (g - b*m) * (CB - b),  m = 32/rows, b = g/m
 * (interaction groups: g * (CB - NR/32)); nblist_shape's RB is then the number
 * of row groups and copy_nblist's row_block_ntiles has one entry per group.
 */
tmnb_status tmnb_potential_set_tile_rows(tmnb_potential *pot, int rows);
tmnb_status tmnb_potential_nblist_rows(tmnb_potential *pot, int *rows, int *column_blocks);
tmnb_status tmnb_potential_copy_nblist(
    tmnb_potential *pot, void *stream, unsigned *perm, int *row_block_ntiles, unsigned *tile_cols);

/* Instrumentation (no reference counterpart): CUDA events around every
 * stage of a call on the launching stream, and the duration of the stage's
 * last launch (synchronises on its end event). Stages: */
#define TMNB_STAGE_PREPARE 0  /* rebuild check, box checks, staging (k_check_prepare) */
#define TMNB_STAGE_REBUILD 1  /* neighbour-list rebuild chain (returns at once when none is due) */
#define TMNB_STAGE_PAIR 2     /* pair kernel */
#define TMNB_STAGE_FINALIZE 3 /* scatter into the caller's outputs and accumulator reset */
tmnb_status tmnb_potential_enable_timing(tmnb_potential *pot, int on);
tmnb_status tmnb_potential_last_stage_ms(tmnb_potential *pot, int stage, float *ms);
tmnb_status tmnb_potential_last_pair_kernel_ms(tmnb_potential *pot, float *ms);

/* Measured FP32 FMA throughput of the current device in TFLOP/s (the
 * denominator of the pair kernel's FP32 roofline; no reference counterpart). */
tmnb_status tmnb_probe_fp32_peak(double *tflops);

/*
 * MD context: replaces timemachine's Context (timemachine/cpp/src/context.hpp:12-45)
 * with its LangevinIntegrator (timemachine/cpp/src/integrator.hpp:29) and
 * MonteCarloBarostat (timemachine/cpp/src/barostat.hpp:26-33). The context
 * copies x0/v0/box0 and the parameters to the device; the potentials stay
 * owned by the caller and must outlive the context. ca/cbs/ccs are the
 * reference's Langevin coefficients (timemachine/integrator.py:32-46 with
 * cbs = -dt/m, timemachine/lib/__init__.py:13-17).
 */
typedef struct tmnb_context tmnb_context;

tmnb_status tmnb_context_create(
    int N,
    const double *x0,   /* [N,3] host */
    const double *v0,   /* [N,3] host */
    const double *box0, /* [3,3] host */
    double dt,
    double ca,
    const double *cbs, /* [N] host */
    const double *ccs, /* [N] host */
    unsigned long long seed,
    int n_potentials,
    tmnb_potential *const *potentials,
    const double *const *params, /* per potential, host */
    const int *param_sizes,
    tmnb_context **out);

/* Isotropic MC barostat every `interval` steps; group_of[i] is the molecule
 * of atom i (-1: not rescaled). */
tmnb_status tmnb_context_set_barostat(
    tmnb_context *ctx, double pressure_bar, double temperature_k, const int32_t *group_of, int interval,
    unsigned long long seed);

/* Context::multiple_steps (timemachine/cpp/src/context.cu:55-137): runs
 * n_steps steps at lambda_schedule[i]; du_dl is stored every
 * store_du_dl_interval steps into du_dl_out[n_steps/interval] (host),
 * coordinates/box every store_x_interval steps into x_out/box_out (host);
 * intervals <= 0 store nothing. use_graphs != 0 replays each step as a CUDA
 * graph (one per distinct lambda). */
tmnb_status tmnb_context_multiple_steps(
    tmnb_context *ctx,
    int n_steps,
    const double *lambda_schedule,
    int store_du_dl_interval,
    double *du_dl_out,
    int store_x_interval,
    double *x_out,
    double *box_out,
    int use_graphs);

/* Context::multiple_steps_U (timemachine/cpp/src/context.cu:139-234): runs
 * n_steps steps at `lambda`; every store_u_interval steps stores the total
 * potential energy at each of the n_windows lambda_windows into
 * u_out[n_steps/store_u_interval][n_windows] (host), computed with one
 * multi-window evaluation per potential (TMNB_MAX_WINDOWS windows at a time);
 * coordinates/box every store_x_interval steps into x_out/box_out (host).
 * Both intervals must be positive ("store_u_interval <= 0" /
 * "store_x_interval <= 0" otherwise, as the reference throws). */
tmnb_status tmnb_context_multiple_steps_U(
    tmnb_context *ctx,
    double lambda,
    int n_steps,
    int n_windows,
    const double *lambda_windows,
    int store_u_interval,
    int store_x_interval,
    double *u_out,
    double *x_out,
    double *box_out,
    int use_graphs);

/* State accessors (timemachine/cpp/src/context.cu:284-304). */
tmnb_status tmnb_context_get_x(tmnb_context *ctx, double *out);
tmnb_status tmnb_context_get_v(tmnb_context *ctx, double *out);
tmnb_status tmnb_context_get_box(tmnb_context *ctx, double *out);
tmnb_status tmnb_context_set_x(tmnb_context *ctx, const double *in);
tmnb_status tmnb_context_set_v(tmnb_context *ctx, const double *in);
tmnb_status tmnb_context_set_box(tmnb_context *ctx, const double *in);
tmnb_status tmnb_context_barostat_stats(tmnb_context *ctx, int *accepted, int *attempted, double *volume_scale);
/* MonteCarloBarostat::set_pressure / set_interval
 * (timemachine/cpp/src/barostat.cu:386-397, bound in wrap_kernels.cpp):
 * the pressure in bar; a new interval restarts the move counter. */
tmnb_status tmnb_context_barostat_set_pressure(tmnb_context *ctx, double pressure_bar);
tmnb_status tmnb_context_barostat_set_interval(tmnb_context *ctx, int interval);
/* The last barostat move (inspection, no reference counterpart):
 * values[8] = rand0, rand1, proposal volume scale, volume delta, length
 * scale, accepted (1/0), volume scale after adaptation, pressure
 * (kJ/mol/nm^3); energies[2] = fixed-point total energy before the move and
 * at the trial coordinates. */
tmnb_status tmnb_context_barostat_last_move(tmnb_context *ctx, double *values, unsigned long long *energies);
tmnb_status tmnb_context_destroy(tmnb_context *ctx);

/*
 * Bonded terms the MD drivers need alongside the nonbonded potential:
 * HarmonicBond (timemachine/cpp/src/harmonic_bond.cu, U = kb/2 (r - b0)^2,
 * params [B,2]) and HarmonicAngle (timemachine/cpp/src/harmonic_angle.cu,
 * U = ka/2 (cos theta - cos a0)^2, params [A,2], angle_idxs [A,3] with the
 * vertex in the middle). Each term is scaled by lambda_offset + lambda_mult *
 * lambda (NULL: offset 1, mult 0).
 */
tmnb_status tmnb_harmonic_bond_create(
    int N, int B, const int32_t *bond_idxs, const int32_t *lambda_mult, const int32_t *lambda_offset, tmnb_potential **out);
tmnb_status tmnb_harmonic_angle_create(
    int N, int A, const int32_t *angle_idxs, const int32_t *lambda_mult, const int32_t *lambda_offset, tmnb_potential **out);

/* Expected parameter count P (N*3, or 2*N*3 when interpolated). */
int tmnb_potential_num_params(const tmnb_potential *pot);
int tmnb_potential_num_atoms(const tmnb_potential *pot);

/*
 * Lambda transforms of a nonbonded handle: the four C-expression schedules
 * in `lambda` that the reference constructors take as their last four
 * arguments (transform_lambda_charge, _sigma, _epsilon, _w;
 * timemachine/cpp/src/wrap_kernels.cpp:843-893, :901-958, :962-1013) and
 * compile at run time (timemachine/cpp/src/kernels/k_lambda_transformer_jit.cuh).
 * Here each expression is parsed once and evaluated on the host per call
 * (value and exact derivative), so nothing is compiled at run time. NULL
 * keeps "lambda". Non-interpolated handles use only the w schedule, as the
 * reference's do. Supported: numeric literals (C integer rules), lambda, PI,
 * + - * / % (unary + - !), comparisons, && ||, ?:, parentheses, and sin cos
 * tan asin acos atan atan2 sinh cosh tanh exp log log10 sqrt pow fabs abs
 * fmin fmax min max floor ceil. A parse error returns TMNB_ERR_INVALID_ARGUMENT
 * with the offending position. The replica batch and the allocation-free
 * entry point use the identity only; the adjoint needs the identity w schedule.
 */
tmnb_status tmnb_potential_set_lambda_transforms(
    tmnb_potential *pot, const char *charge, const char *sigma, const char *epsilon, const char *w);

/* Value f and derivative df/dlambda of one lambda-transform expression at
 * lambda, as the staging uses them (host only, no GPU needed; no reference
 * counterpart -- the reference evaluates its compiled transforms on the
 * device). TMNB_ERR_INVALID_ARGUMENT on a parse error. */
tmnb_status tmnb_lambda_transform_eval(const char *expression, double lambda, double *f, double *df);

/*
 * Adjoint (no reference counterpart: the reference differentiates its jax
 * potential, timemachine/potentials/nonbonded.py, with jax.grad). For the
 * potential at (x, params, lambda) and upstream gradients g_du_dx [N,3]
 * (of du_dx, as float64) and g_du_dl (of the summed du_dl), ADDS the
 * vector-Jacobian product to d_grad_p [P] (d/d charge, sigma/2, sqrt(eps))
 * and d_grad_w [N] (d/d the per-atom lambda offset, treated as a continuous
 * coefficient of w = cutoff * (plane + offset * lambda)). Pair terms are
 * recomputed in FP64; nothing from the forward pass is stored. Non-interpolated
 * AllPairs, PairList and Nonbonded handles (TMNB_ERR_UNSUPPORTED otherwise).
 */
tmnb_status tmnb_potential_adjoint_device(
    tmnb_potential *pot,
    int N,
    int P,
    const double *d_x,
    const double *d_p,
    const double *d_box,
    double lambda,
    const double *d_g_du_dx, /* [N,3] */
    double g_du_dl,
    double *d_grad_p, /* [P] += */
    double *d_grad_w, /* [N] += */
    void *stream);

/*
 * Replica batch (no single reference counterpart: it replaces the loops in
 * which the reference evaluates or simulates replicas one at a time, one
 * Potential::execute_device / one Context per replica and lambda). Holds any
 * number of independent systems, each at its own lambda, with its nonbonded
 * potential (all pairs minus the scaled exclusions), harmonic bonds and
 * angles; one launch sequence per step serves every replica. Each replica's
 * outputs equal a single-system evaluation of the same inputs bit for bit,
 * whatever else is in the batch. Replicas can be added and removed between
 * calls (each owns one device arena; tmnb_batch_footprint gives its size).
 */
typedef struct tmnb_batch tmnb_batch;

tmnb_status tmnb_batch_create(tmnb_batch **out);
tmnb_status tmnb_batch_destroy(tmnb_batch *b);

/* Adds one replica (host arrays, copied). v, cbs, ccs may be NULL (no MD;
 * v = 0). ca, cbs, ccs, dt: Langevin coefficients as in tmnb_context_create.
 * id receives the replica's handle within the batch. */
tmnb_status tmnb_batch_add(
    tmnb_batch *b,
    int N,
    const double *x,      /* [N,3] */
    const double *v,      /* [N,3] or NULL */
    const double *box,    /* [3,3] */
    const double *params, /* [N,3] */
    const int32_t *lambda_plane_idxs,
    const int32_t *lambda_offset_idxs,
    int M,
    const int32_t *exclusion_idxs, /* [M,2] */
    const double *scales,          /* [M,2] */
    int B,
    const int32_t *bond_idxs, /* [B,2] */
    const double *bond_params,
    int A,
    const int32_t *angle_idxs, /* [A,3] */
    const double *angle_params,
    double beta,
    double cutoff,
    double lambda,
    double dt,
    double ca,
    const double *cbs, /* [N] or NULL */
    const double *ccs, /* [N] or NULL */
    unsigned long long seed,
    int *id);

tmnb_status tmnb_batch_remove(tmnb_batch *b, int id);

/* Device bytes a replica of N atoms, M exclusions, B bonds, A angles holds
 * (admission control by HBM footprint), and the bytes all replicas hold. */
tmnb_status tmnb_batch_footprint(tmnb_batch *b, int N, int M, int B, int A, unsigned long long *bytes);
tmnb_status tmnb_batch_bytes_in_use(tmnb_batch *b, unsigned long long *bytes);

/* Schedule of the tile work: tiles per work item, neighbour-list padding (nm),
 * Hilbert grid resolution offset (-2..2), pair-kernel CTAs per SM (0: by
 * occupancy). Applies to every replica (re-laid out, list rebuilt). */
tmnb_status tmnb_batch_set_tuning(tmnb_batch *b, int chunk, double padding, int grid_bits_offset, int pair_ctas_per_sm);

/* Rows per neighbour-list tile of every replica: 16 (default), 32 or 8 slots
 * (identical results; as tmnb_potential_set_tile_rows). Every replica is
 * re-laid out and rebuilds its list. */
tmnb_status tmnb_batch_set_tile_rows(tmnb_batch *b, int rows);

/* One evaluation of every replica (outputs overwritten; read them with
 * tmnb_batch_get). Asynchronous on the batch's stream. */
tmnb_status tmnb_batch_evaluate(tmnb_batch *b, int compute_du_dx, int compute_du_dp, int compute_du_dl, int compute_u);

/* n_steps Langevin steps of every replica; use_graph != 0 replays a CUDA
 * graph of `chunk` steps. Asynchronous on the batch's stream. */
tmnb_status tmnb_batch_md(tmnb_batch *b, int n_steps, int chunk, int use_graph);

tmnb_status tmnb_batch_synchronize(tmnb_batch *b);

/* Copies (synchronising) replica id's x [N,3] (which 0), v (1), box (2) as
 * doubles, or its outputs du_dx [N,3] (3), du_dp [N,3] (4), per-atom du_dl
 * [N] (5), per-atom u [N] (6) as int64 fixed point. */
tmnb_status tmnb_batch_get(tmnb_batch *b, int id, int which, void *out);
/* Overwrites replica id's x (0), v (1) or box (2). */
tmnb_status tmnb_batch_set(tmnb_batch *b, int id, int which, const double *in);
/* Sticky device error of replica id (TMNB_ERR_* value, 0 = none), cleared. */
tmnb_status tmnb_batch_error(tmnb_batch *b, int id, int *code);
tmnb_status tmnb_batch_stats(tmnb_batch *b, int id, int *tiles, int *items, int *rebuilds);
/* The batch's CUDA stream (every batch call is ordered on it), e.g. to record
 * events around tmnb_batch_evaluate / tmnb_batch_md. */
tmnb_status tmnb_batch_stream(tmnb_batch *b, void **stream);
/* Scheduling priority of the batch's stream (CUDA stream priority, clamped to
 * the device's range; lower numbers are scheduled first when blocks of
 * several streams wait for SMs). Waits for the batch's work; its stream
 * handle changes. */
tmnb_status tmnb_batch_set_priority(tmnb_batch *b, int priority);
int tmnb_batch_size(const tmnb_batch *b);

/* Largest N accepted by tmnb_pair_list_execute_static (3.16 MiB of static
 * device scratch). */
#define TMNB_STATIC_MAX_ATOMS 32768

/*
 * Allocation-free pair-list evaluation. NO REFERENCE COUNTERPART: it has the
 * arguments of tmnb_pair_list_create (interpolated = 0, precision 32)
 * followed by those of tmnb_potential_execute_device, with every array in
 * device memory, and gives the same outputs (accumulated, +=).
 *
 * For callers that must not allocate device memory: processes that hand all
 * of HBM to their own fixed arena or caching allocator up front (a raw
 * cudaMalloc then fails or fragments it), and loops that cannot afford the
 * device-wide synchronisation that cudaFree implies. It calls no cudaMalloc,
 * cudaFree or allocating library routine: its slot staging, accumulators and
 * device state live in a file-scope static device array of fixed size.
 *
 * Limit: 1 <= N <= TMNB_STATIC_MAX_ATOMS; larger N returns
 * TMNB_ERR_INVALID_ARGUMENT ("N=... exceeds the static scratch capacity").
 * The scratch must start at zero: it is zero at module load and every call
 * leaves it at zero. The FIRST call on each device performs a one-time
 * set-up with that device current (loads the kernels, looks up the scratch
 * with cudaGetSymbolAddress, writes the identity slot order, synchronises
 * the device); make that first call before any stream capture. Every call
 * synchronises `stream` before returning, to report pair indices outside
 * [0, N) or with src == dst (TMNB_ERR_INVALID_ARGUMENT; outputs unchanged).
 * The scratch is shared by all calls on a device: calls that overlap in time
 * (other host threads, or other streams still running) race on it and give
 * wrong results; serialise them.
 */
tmnb_status tmnb_pair_list_execute_static(
    int N,
    int M,
    const int32_t *d_pair_idxs,          /* [M,2] */
    const double *d_scales,              /* [M,2] */
    const int32_t *d_lambda_plane_idxs,  /* [N] */
    const int32_t *d_lambda_offset_idxs, /* [N] */
    double beta,
    double cutoff,
    int negated,
    const double *d_x,           /* [N,3] */
    const double *d_p,           /* [N,3] */
    const double *d_box,         /* [3,3] */
    double lambda,
    unsigned long long *d_du_dx, /* [N,3] or NULL */
    unsigned long long *d_du_dp, /* [N,3] or NULL */
    unsigned long long *d_du_dl, /* [N] or NULL */
    unsigned long long *d_u,     /* [N] or NULL */
    void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TMNB_H */
