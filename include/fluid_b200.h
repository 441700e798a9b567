/* fluid_b200.h — C ABI of the B200 particle-fluid library (libfluid_b200.so).
 *
 * Drop-in replacement for the hot path of SParksLz/fluid_simulation: the
 * warp-lang 1.17.0 hash grid (`wp.HashGrid`) and the per-particle kernels of
 * SolverWCSPH / SolverDFSPH / SolverPBF behind
 * `SolverBase.step(state_in, state_out, control, contacts, dt)`.
 *
 * Conventions
 *  - Every array is a raw DEVICE pointer into caller-owned memory laid out as
 *    the reference's Newton arrays: vec3 arrays are float[n][3] (AoS), scalars
 *    float[n], flags/masks/worlds/counts int32[n], all in ORIGINAL particle
 *    order.  The library never frees caller memory.
 *  - Scratch (cell tables, cell-sorted copies, reductions) belongs to an
 *    fs_context, which is bound to one device and sized for `capacity`
 *    particles at creation.
 *  - Every call is asynchronous on `stream` (a cudaStream_t; NULL = legacy
 *    default stream) and returns an int status: FS_OK or one of FS_ERR_*.
 *    Kernel-side conditions are recorded in the context's status word
 *    (FS_STATUS_* bits) and read with fs_status_read.
 *  - Errors never trap or hang the device.
 */
#ifndef FLUID_B200_H
#define FLUID_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* fs_stream_t; /* == cudaStream_t */
typedef struct fs_context fs_context;

/* return codes */
#define FS_OK 0
#define FS_ERR_INVALID 1   /* null pointer, negative size, bad config */
#define FS_ERR_CUDA 2      /* a CUDA runtime call failed (fs_last_error_string) */
#define FS_ERR_CAPACITY 3  /* n exceeds the context capacity */
#define FS_ERR_NOGRID 4    /* a pass needs a grid that was not built for this n */
#define FS_ERR_NONFINITE 5 /* fs_wcsph_density_noalloc only: a position was not finite */

/* device status word bits (sticky until fs_status_clear) */
#define FS_STATUS_NONFINITE 1u      /* a non-finite position reached the grid build */
#define FS_STATUS_GRID_OVERFLOW 2u  /* more particles than the grid was reserved for */
#define FS_STATUS_BOUNDS 4u         /* a checked index fell outside its array */
#define FS_STATUS_TIMEOUT 8u        /* a bounded device-side wait gave up */

/* Hash-grid geometry.  The reference uses wp.HashGrid(128, 128, 128)
 * (solver_wcsph.py:398-402) with cell width = support radius h and warp's
 * truncating float-to-int conversion (rounding = 0).  rounding = 1 selects
 * floor.  Cell coords wrap modulo the dims (shifted by 2^20 first). */
typedef struct {
  int32_t dim_x, dim_y, dim_z;
  int32_t rounding;
} fs_grid_config;

/* Model arrays (Newton Model + the `sph` custom-attribute namespace).
 * Unused fields may be NULL (stiffness/exponent are WCSPH only). */
typedef struct {
  int64_t n;                      /* Model.particle_count */
  int32_t n_worlds;               /* rows of gravity */
  const int32_t* particle_flags;  /* Model.particle_flags (bit 0 = ParticleFlags.ACTIVE) */
  const int32_t* particle_mask;   /* Model.sph.particle_mask (non-zero = not dynamic) */
  const int32_t* particle_world;  /* Model.particle_world (may be NULL = world 0) */
  const float* particle_mass;     /* Model.particle_mass */
  const float* gravity;           /* Model.gravity [n_worlds][3] */
  const float* rest_density;      /* Model.sph.rest_density */
  const float* surface_tension;   /* Model.sph.surface_tension (cohesion coefficient) */
  const float* viscosity;         /* Model.sph.viscosity */
  const float* stiffness;         /* Model.sph.stiffness (WCSPH) */
  const float* exponent;          /* Model.sph.exponent (WCSPH) */
} fs_model;

/* One Newton State: particle_q / particle_qd plus the `sph` STATE attributes.
 * Fields a solver does not write may be NULL. */
typedef struct {
  float* particle_q;      /* [n][3] */
  float* particle_qd;     /* [n][3] */
  float* rho;             /* all solvers */
  float* pressure;        /* WCSPH */
  float* factor;          /* DFSPH */
  float* rho_star;        /* DFSPH */
  float* d_rho_dt;        /* DFSPH */
  float* kappa;           /* DFSPH */
  float* kappa_v;         /* DFSPH */
  int32_t* neighbor_count;/* DFSPH, PBF */
  float* v_star;          /* DFSPH [n][3] */
  float* pbf_lambda;      /* PBF */
  float* delta_p;         /* PBF [n][3] */
} fs_state;

/* Scalars of one WCSPH substep (SolverWCSPH.SphConfig, solver_wcsph.py:309-318). */
typedef struct {
  float dt;
  float smoothing_length;  /* h = particle_length * smoothing_length_coff */
  float particle_radius;   /* config radius, or Model.particle_max_radius when <= 0 */
  float bound_width, bound_height, bound_length;
  float boundary_damping;
  int32_t clamp_negative_pressure;
} fs_wcsph_params;

/* Scalars of one DFSPH substep (SolverDFSPH.SphConfig, solver_dfsph.py:446-463). */
typedef struct {
  float dt;
  float smoothing_length;
  float particle_radius;
  float bound_width, bound_height, bound_length;
  float boundary_damping;
  int32_t max_rho_iterations, max_vel_iterations, warm_start, min_neighbors_for_factor;
  float eta_density, eta_divergence, max_kappa, max_kappa_v;
} fs_dfsph_params;

/* Scalars of one PBF substep (SolverPBF.PbfConfig, solver_pbf.py:521-539). */
typedef struct {
  float dt;
  float smoothing_length;
  float particle_radius;
  float bound_width, bound_height, bound_length;
  float boundary_damping, boundary_epsilon;
  int32_t max_iterations, min_neighbors_for_lambda, rebuild_grid_each_iteration;
  float lambda_epsilon, scorr_k, scorr_n, scorr_w_delta_q, max_delta_position, xsph_c;
} fs_pbf_params;

/* SolverAPIC particle separation (solver_apic.py:1003-1064): the kernel
 * arguments of accumulate_particle_separation / apply_particle_separation_delta
 * (193-266) and the iteration count. */
typedef struct {
  float rest_dist;     /* pushes act below this distance */
  float query_radius;  /* grid cell width and query radius (max(rest_dist, 1e-5)) */
  float strength;      /* separation_strength */
  float bound_lo[3], bound_hi[3];
  float wall_band;     /* into-wall push components removed within this band */
  float wall_margin;   /* positions clamped to the bounds inset by this margin */
  int32_t iterations;  /* separation_iterations (at least 1) */
} fs_separation_params;

/* Per-step DFSPH solver record (read back on demand; not needed to step). */
typedef struct {
  int32_t rho_iterations;       /* density iterations entered */
  int32_t vel_iterations;       /* divergence iterations entered */
  double density_residual;      /* last computed mean max(rho*-rho0, 0) */
  double divergence_residual;   /* last computed mean max(drho/dt, 0) */
} fs_dfsph_info;

/* ---- context / grid ---------------------------------------------------
 * Replaces `wp.HashGrid(128,128,128)` + `.reserve(N)` done by every solver
 * constructor (solver_wcsph.py:398-402, solver_dfsph.py:541-545,
 * solver_pbf.py:634-638) and the solvers' private scratch arrays. */
int fs_context_create(fs_context** out, int64_t capacity, const fs_grid_config* grid, int32_t device);
int fs_context_destroy(fs_context* ctx);
int64_t fs_context_capacity(const fs_context* ctx);

/* Launch tuning of a context's neighbour kernels (no counterpart in the
 * reference, whose kernels Warp launches one thread per point).  Chosen by
 * the autotuner (fluid_simulation_b200.autotune) from measured substeps.
 *   block_size            threads per block: 64, 128 (default) or 256
 *   particles_per_thread  1 (default), 2 or 4: each thread walks that many
 *                         cell-sorted particles (grid-stride)
 *   cell_ratio            WCSPH grid cell width / h: 1 (default, the
 *                         reference's grid: candidates in its order) or 0.5
 *                         (125 half-width cells per query instead of 27;
 *                         same neighbours, sums in another order).  PBF and
 *                         DFSPH always bin at h: PBF queries the grid from
 *                         moved positions and DFSPH counts candidates, so
 *                         the cell width is part of their results.
 *   list_skin             PBF: the first density pass records its neighbour
 *                         lists out to h (1 + list_skin) (default 0.02, at
 *                         most 0.25), so that the first lambda pass, after
 *                         the non-pressure update moved every particle by
 *                         less than list_skin h / 2, reuses them instead of
 *                         scanning the grid; 0 always scans.
 * block_size, particles_per_thread and list_skin change no result (DFSPH
 * sums its residual per block, so its last bits follow block_size). */
typedef struct {
  int32_t block_size;
  int32_t particles_per_thread;
  float cell_ratio;
  float list_skin;
} fs_tuning;
int fs_context_set_tuning(fs_context* ctx, const fs_tuning* tuning);
int fs_context_get_tuning(const fs_context* ctx, fs_tuning* tuning);

/* `grid.build(points, radius)` (solver_wcsph.py:456, solver_dfsph.py:624,783,
 * solver_pbf.py:737,858): cell keys, stable sort by cell, cell ranges. */
int fs_grid_build(fs_context* ctx, const float* x, int64_t n, float radius, fs_stream_t stream);

/* Copies of the last build's tables into caller device arrays (tests):
 * point_ids[n] (`hash_grid_point_id`), point_cells[n] (sorted cell keys),
 * cell_starts/cell_ends[dim_x*dim_y*dim_z] (empty cells: start == end). */
int fs_grid_tables(fs_context* ctx, int32_t* point_ids, int32_t* point_cells, int32_t* cell_starts,
                   int32_t* cell_ends, fs_stream_t stream);

/* Candidate enumeration of `wp.hash_grid_query(grid, q[i], r)` against the
 * last build (tests): counts[i], and when cand != NULL the candidates in
 * visiting order at cand[offsets[i]...]. */
int fs_grid_candidates(fs_context* ctx, const float* q, int64_t nq, float r, int64_t* counts,
                       const int64_t* offsets, int32_t* cand, fs_stream_t stream);

/* ---- batched worlds (no counterpart in the reference) ------------------
 * Many independent scenes (Newton worlds, Model.particle_world) advance in
 * one model: one launch per pass covers every scene.  The reference puts all
 * worlds of a model into one hash grid, so scenes that overlap in space
 * would interact; a batched context instead gives each world its own box of
 * cells keyed (world, cell): per axis cell = clamp(c - cell_lo, 0, dims - 1)
 * with c the reference's truncating cell coordinate int(x / h), no hashing,
 * and a query never leaves its world.  Inside its box a world sees the cells,
 * candidate order and results of the hash grid of that world alone.  Each
 * world also
 * has its own tank: the walls of the step parameters are replaced by
 * fs_world_box.bound_* of the particle's world.  particle_world is required;
 * an index outside [0, nworlds) is clamped and raises FS_STATUS_BOUNDS.
 * Every substep and separate pass accepts a batched context.  The DFSPH
 * substep takes its iteration decisions per world (each world iterates until
 * the mean residual of its own dynamic particles passes, as that scene would
 * alone); fs_dfsph_info_worlds reads them.  fs_grid_build / fs_grid_candidates on a batched context
 * (and the *_worlds forms on a hash-grid context) return FS_ERR_INVALID. */
typedef struct {
  int32_t cell_lo[3];  /* cell coordinate int(x / h) of the box's first cell per axis */
  int32_t dims[3];     /* cells per axis */
  float bound_width, bound_height, bound_length;  /* tank [-W,W]x[-H,H]x[0,2L] */
} fs_world_box;

int fs_context_create_worlds(fs_context** out, int64_t capacity, const fs_world_box* worlds, int32_t nworlds,
                             int32_t device);
int32_t fs_context_worlds(const fs_context* ctx); /* 0 for a hash-grid context */
int64_t fs_context_cells(const fs_context* ctx);  /* cells of the grid (the size of cell_starts) */
/* grid.build for a batched context: world[n] = Model.particle_world. */
int fs_grid_build_worlds(fs_context* ctx, const float* x, const int32_t* world, int64_t n, float radius,
                         fs_stream_t stream);
/* fs_grid_candidates of queries that belong to world qworld[i]. */
int fs_grid_candidates_worlds(fs_context* ctx, const float* q, const int32_t* qworld, int64_t nq, float r,
                              int64_t* counts, const int64_t* offsets, int32_t* cand, fs_stream_t stream);

/* ---- whole substeps --------------------------------------------------- */
/* SolverWCSPH.step (solver_wcsph.py:431-535).  accel = solver._particle_accel [n][3]. */
int fs_wcsph_substep(fs_context* ctx, const fs_model* model, const fs_state* state_in, fs_state* state_out,
                     const fs_wcsph_params* params, float* accel, fs_stream_t stream);
/* SolverDFSPH.step (solver_dfsph.py:598-898).  Iteration decisions are taken
 * on the device (no host synchronisation inside the step). */
int fs_dfsph_substep(fs_context* ctx, const fs_model* model, const fs_state* state_in, fs_state* state_out,
                     const fs_dfsph_params* params, float* accel, fs_stream_t stream);
int fs_dfsph_info_read(fs_context* ctx, fs_dfsph_info* info); /* synchronises the context's last stream */
/* Per-world decisions of the last DFSPH substep of a batched context:
 * info[w] for w < nworlds (nworlds = fs_context_worlds(ctx)); on a batched
 * context fs_dfsph_info_read gives the largest iteration counts and residuals
 * over the worlds.  Synchronises the context's last stream. */
int fs_dfsph_info_worlds(fs_context* ctx, fs_dfsph_info* info, int32_t nworlds);
/* SolverPBF.step (solver_pbf.py:676-954).  x_pred may be NULL (solver._x_pred [n][3]). */
/* SolverAPIC._apply_particle_separation (solver_apic.py:1003-1064): per
 * iteration, a grid build over x with cell width query_radius, the mean push
 * of each active particle's active neighbours closer than rest_dist (wall-band
 * components removed), and x += push clamped to the inset bounds.  x [n][3]
 * is updated in place; flags[n] = Model.particle_flags; delta [n][3] receives
 * the last iteration's pushes (solver._sep_delta).  ctx: a hash-grid context
 * with the reference's dims for this pass, max(4, ceil(extent / query_radius))
 * per axis, and capacity >= n.  Results equal the reference's bit for bit. */
int fs_apic_separation(fs_context* ctx, float* x, const int32_t* flags, int64_t n, const fs_separation_params* params,
                       float* delta, fs_stream_t stream);
int fs_pbf_substep(fs_context* ctx, const fs_model* model, const fs_state* state_in, fs_state* state_out,
                   const fs_pbf_params* params, float* accel, float* x_pred, fs_stream_t stream);

/* ---- WCSPH adjoint (no counterpart in the reference, which differentiates
 * nothing; the reference project's archive took gradients through Warp's
 * tape) ----------------------------------------------------------------
 * Reverse-mode derivative of one fs_wcsph_substep with the step's neighbour
 * set held fixed.  Inputs: the step's input state (particle_q/qd of
 * state_in), what the forward step wrote (rho, pressure: state_out.sph; accel),
 * and the adjoints of its outputs (adj_x_out = dL/d particle_q out, adj_v_out =
 * dL/d particle_qd out, [n][3]).  Writes adj_x_in / adj_v_in (dL/d particle_q
 * and particle_qd in, [n][3]) and ADDS dL/d stiffness, viscosity and
 * rest_density per particle into adj_stiffness / adj_viscosity /
 * adj_rest_density (each may be NULL).  Builds the grid of state_in itself;
 * uses the context's scratch like a substep. */
int fs_wcsph_substep_adjoint(fs_context* ctx, const fs_model* model, const fs_state* state_in, const float* rho,
                             const float* pressure, const float* accel, const float* adj_x_out, const float* adj_v_out,
                             float* adj_x_in, float* adj_v_in, float* adj_stiffness, float* adj_viscosity,
                             float* adj_rest_density, const fs_wcsph_params* params, fs_stream_t stream);

/* ---- separate passes (each needs fs_grid_build(positions, h) first) --------
 * WCSPH compute_density_pressure (solver_wcsph.py:120-158). */
int fs_wcsph_density(fs_context* ctx, const fs_model* model, const float* x, float h, int32_t clamp_negative,
                     float* rho, float* pressure, fs_stream_t stream);
/* WCSPH acceleration_wcsph + integrate_velocity + integrate_positions +
 * apply_bounds (solver_wcsph.py:162-305), fused. */
int fs_wcsph_force_integrate(fs_context* ctx, const fs_model* model, const fs_state* state_in, fs_state* state_out,
                             const fs_wcsph_params* params, float* accel, fs_stream_t stream);
/* DFSPH compute_density + compute_factor_dfsph (solver_dfsph.py:107-174), fused. */
int fs_dfsph_density_factor(fs_context* ctx, const fs_model* model, const float* x, float h,
                            int32_t min_neighbors_for_factor, float* rho, float* factor, int32_t* neighbor_count,
                            fs_stream_t stream);
/* DFSPH acceleration_non_pressure + predict_velocity (solver_dfsph.py:178-242),
 * fused: accel [n][3] (gravity included, 0 for non-dynamic particles) and
 * v_star = v + dt * accel [n][3]; rho [n] is the density of the step. */
int fs_dfsph_nonpressure_predict(fs_context* ctx, const fs_model* model, const float* x, const float* v,
                                 const float* rho, float h, float particle_radius, float dt, float* accel,
                                 float* v_star, fs_stream_t stream);
/* DFSPH compute_density_change_rate (solver_dfsph.py:246-272). */
int fs_dfsph_divergence(fs_context* ctx, const fs_model* model, const float* x, const float* v, float h,
                        float* d_rho_dt, fs_stream_t stream);
/* DFSPH apply_constant_density_correction / apply_divergence_free_correction
 * (solver_dfsph.py:310-337, 376-403): v_star[i] -= dt * sum(...), in place. */
int fs_dfsph_correct(fs_context* ctx, const fs_model* model, const float* x, float* v_star, const float* rho,
                     const float* kappa, float h, float dt, fs_stream_t stream);
/* DFSPH residual (solver_dfsph.py:579-596): mean over dynamic particles of
 * max(a - b, 0) (b may be NULL), written as one double to *out (device). */
int fs_dfsph_residual(fs_context* ctx, const fs_model* model, const float* a, const float* b, double* out,
                      fs_stream_t stream);
/* PBF predict_velocity_with_gravity + predict_positions + apply_position_bounds
 * (solver_pbf.py:193-224, 367-399): v_pred = v + dt g, x_pred = x + dt v_pred
 * clamped into the walls inset by particle_radius + boundary_epsilon (dynamic
 * particles; the others copy x and v).  Needs no grid; a batched context
 * takes each particle's walls from its world. */
int fs_pbf_predict(fs_context* ctx, const fs_model* model, const float* x, const float* v,
                   const fs_pbf_params* params, float* x_pred, float* v_pred, fs_stream_t stream);
/* PBF compute_density (poly6, solver_pbf.py:115-141). */
int fs_pbf_density(fs_context* ctx, const fs_model* model, const float* x, float h, float* rho, fs_stream_t stream);
/* PBF compute_pbf_lambda (solver_pbf.py:246-302). */
int fs_pbf_lambda(fs_context* ctx, const fs_model* model, const float* x_pred, const fs_pbf_params* params,
                  float* pbf_lambda, float* rho, int32_t* neighbor_count, fs_stream_t stream);
/* PBF compute_delta_position + compute_scorr (solver_pbf.py:306-350, 91-101). */
int fs_pbf_delta(fs_context* ctx, const fs_model* model, const float* x_pred, const float* pbf_lambda,
                 const fs_pbf_params* params, float* delta_p, fs_stream_t stream);
/* PBF apply_xsph_viscosity (solver_pbf.py:435-463). */
int fs_pbf_xsph(fs_context* ctx, const fs_model* model, const float* x_pred, const float* v_in, const float* rho,
                float h, float xsph_c, float* v_out, fs_stream_t stream);

/* ---- dam-break harness reductions (examples/dam_break/simulation.py) -----
 * particle_norm_maxima (19-36): out[0] = max |v|^2 over nv rows, out[1] =
 * max |a|^2 over na rows (a non-finite vector counts as +inf); out is a
 * device float[2] and is zeroed by the call. */
int fs_norm_maxima(const float* v, int64_t nv, const float* a, int64_t na, float* out, fs_stream_t stream);
/* check_particle_finite (39-53): *invalid (device int32) = 1 if any of x[n],
 * v[n], rho[nrho] is non-finite, else 0. */
int fs_check_finite(const float* x, const float* v, int64_t n, const float* rho, int64_t nrho, int32_t* invalid,
                    fs_stream_t stream);

/* ---- device-side harness loop (no counterpart in the reference, whose
 * harness reads the CFL maxima back to the host before every substep:
 * simulation.py:140-196) -------------------------------------------------
 * A frame clock in device memory (caller-owned, 32 bytes) carries the time
 * left in the frame and the dt of the next substep.  fs_frame_clock_advance
 * evaluates the harness's substep rule on the device (simulation.py:167-182,
 * in double precision like the Python harness) from max |v|^2 and |a|^2;
 * fs_wcsph_substep_clocked then runs with that dt, or, once the frame is
 * complete, copies state_in to state_out.  A frame thus records as a CUDA
 * graph of [advance, clocked substep] pairs with one read of the clock per
 * replay instead of one host round trip per substep. */
typedef struct {
  double remaining;      /* time left in the frame (s) */
  float dt;              /* dt of the next substep; 0 once the frame is complete */
  int32_t active;        /* 1: the next clocked substep runs */
  int32_t substeps;      /* substeps taken in this frame */
  int32_t run_substeps;  /* substeps taken since the clock was zeroed (the
                            acceleration bound applies from the second on) */
  int32_t fault;         /* sticky: 1 non-finite maxima, 2 dt below 1e-10 */
  float maxima[2];       /* |v|^2, |a|^2 of the last evaluation */
  int32_t pad;
} fs_frame_clock;        /* zero it (e.g. cudaMemset) before the first frame */

typedef struct {
  double frame_dt;       /* 1 / fps */
  double substep_limit;  /* frame_dt / base substeps */
  int32_t method;        /* 0: WCSPH rule (sound speed, acceleration, viscosity), 1: DFSPH rule (0.4 spacing / |v|) */
  int32_t use_accel;     /* WCSPH: include the acceleration bound (after the first substep of a run) */
  double h, sound_speed, viscosity, spacing;
} fs_cfl_rule;

int fs_frame_clock_start(fs_frame_clock* clock, double frame_dt, fs_stream_t stream);
int fs_frame_clock_advance(fs_frame_clock* clock, const fs_cfl_rule* rule, const float* v, int64_t nv,
                           const float* accel, int64_t na, fs_stream_t stream);
/* fs_wcsph_substep at dt = clock->dt; when clock->active == 0 it copies
 * particle_q, particle_qd (and rho, pressure when both states give them)
 * from state_in to state_out and leaves accel as it is. */
int fs_wcsph_substep_clocked(fs_context* ctx, const fs_model* model, const fs_state* state_in, fs_state* state_out,
                             const fs_wcsph_params* params, float* accel, const fs_frame_clock* clock,
                             fs_stream_t stream);
/* fs_dfsph_substep at dt = clock->dt (rule method 1); once the frame is
 * complete it copies state_in to state_out (every field both give). */
int fs_dfsph_substep_clocked(fs_context* ctx, const fs_model* model, const fs_state* state_in, fs_state* state_out,
                             const fs_dfsph_params* params, float* accel, const fs_frame_clock* clock,
                             fs_stream_t stream);

/* Frame metrics of the dam-break harness (simulation.py:198-225) reduced on
 * the device into out[14] (device doubles): [0] non-finite x or v, [1]
 * non-finite rho, [2] non-finite pressure (1/0), [3] max |v| (float32 norm,
 * as numpy.linalg.norm), [4..6] mean / min / max of z, [7..9] mean / min /
 * max of rho, [10] the k-th and [11] the (k+1)-th smallest rho (the (k)-th
 * again when k = nrho - 1: the percentile's interpolation ends), [12..13]
 * min / max of pressure (NULL pressure: 0).  Minima, maxima and the order
 * statistics are exact; means are double sums in a fixed order.  Uses the
 * context's scratch (n, nrho <= capacity); no grid is needed. */
int fs_frame_metrics(fs_context* ctx, const float* x, const float* v, int64_t n, const float* rho,
                     const float* pressure, int64_t nrho, int64_t k, double* out, fs_stream_t stream);

/* ---- instrumentation (no counterpart in the reference, which only times
 * whole frames with wall clocks: examples/dam_break/benchmark.py:63-72) ----
 * Per-pass CUDA-event timer: while enabled, every pass launched through the
 * context is bracketed by an event pair on its stream (up to `capacity`
 * passes).  fs_timer_read synchronises, sums the elapsed time per pass id
 * (names from fs_pass_name) and disables the timer. */
int32_t fs_pass_count(void);
const char* fs_pass_name(int32_t pass);
int fs_timer_enable(fs_context* ctx, int32_t capacity); /* capacity 0 frees the events */
int fs_timer_read(fs_context* ctx, float* ms_per_pass, int32_t* launches_per_pass, int32_t npass, int32_t* dropped);
int64_t fs_launch_count(const fs_context* ctx);           /* kernels launched through ctx so far */
/* Neighbour-list counters (synchronises): [0] particles whose current list
 * is usable, [1] particles whose current list overflowed (kNbMax entries;
 * their later passes scan the grid), both tallied from the lists now held;
 * [2] PBF first-lambda passes that reused the first density's list instead
 * of scanning, since the last reset and only while enabled
 * (fs_list_stats_enable, off by default). */
int fs_list_stats(fs_context* ctx, int64_t* counters, int32_t ncounters, int32_t reset);
int fs_list_stats_enable(fs_context* ctx, int32_t on);

/* ---- allocation-free density (no counterpart in the reference) ----------
 * For callers that cannot allocate device memory (hosts whose allocator
 * forbids cudaMalloc, plugins inside a runtime that owns all device memory):
 * grid build + WCSPH density and EOS, the results of fs_grid_build +
 * fs_wcsph_density (up to summation order), in a fixed scratch area compiled
 * into the library (about 1 MB per GPU that loads it, held until exit)
 * instead of an fs_context.  At most fs_noalloc_max_particles() particles;
 * larger n returns FS_ERR_CAPACITY.  The scratch address is looked up
 * (cudaGetSymbolAddress) on the first call in each CUDA context and cached
 * under that context; make that first call before any stream capture.  The
 * call waits for its stream: it reads back a status word and returns
 * FS_ERR_NONFINITE when a position is not finite (that particle's density
 * is 0 and it adds nothing to the others).  All calls share the one scratch
 * area: calls whose work overlaps on the GPU (other streams, other host
 * threads) race and give wrong results. */
int32_t fs_noalloc_max_particles(void);
int fs_wcsph_density_noalloc(const fs_model* model, const float* x, float h, int32_t clamp_negative, float* rho,
                             float* pressure, fs_stream_t stream);

/* ---- status ------------------------------------------------------------ */
int fs_status_read(fs_context* ctx, uint32_t* status); /* synchronises the context's last stream */
int fs_status_clear(fs_context* ctx, fs_stream_t stream);
const char* fs_last_error_string(void);
const char* fs_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FLUID_B200_H */
