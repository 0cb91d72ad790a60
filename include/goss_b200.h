/*
 * goss_b200 -- C ABI of the B200 (sm_100a) multi-node ODE solve path.
 *
 * This is the drop-in boundary that replaces the execution of
 * goss::ODESystemSolver (reference cpp/goss/ODESystemSolver.h:43-124) and of
 * the per-node solvers it drives (ExplicitEuler, RK2, RK4, RL1, RL2, GRL1,
 * GRL2, ImplicitEuler, ThetaSolver, ESDIRK23a).  Only plain C types cross it: pointers, sizes,
 * doubles and integer status codes.  Host arrays are borrowed for the
 * duration of a call and the call is complete on return (the reference is
 * synchronous), except for the *_async entry points.
 *
 * Every entry point returns 0 (GOSS_OK) on success or a positive status
 * code; goss_system_last_error() gives the message.  Status codes map to the
 * reference's exceptions (std::runtime_error -> RuntimeError in Python).
 *
 * Layout conventions
 *   tangled   = 1 : user arrays are node-major  [num_nodes][k]
 *   tangled   = 0 : user arrays are component-major [k][num_nodes]
 *   (the reference's tangled_storage flag, ODESystemSolver.h:238-312)
 * On the device states live component-major: states[i*ld + node], FP64.
 */
#ifndef GOSS_B200_H
#define GOSS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GOSS_API __attribute__((visibility("default")))
#else
#define GOSS_API
#endif

#define GOSS_B200_ABI_VERSION 4u

/* Solver kinds: the reference solver classes on this path. */
enum goss_solver_kind {
    GOSS_EXPLICIT_EULER = 0, /* cpp/goss/ExplicitEuler.cpp:64-87 */
    GOSS_RK4 = 1,            /* cpp/goss/RK4.cpp:68-102 */
    GOSS_GRL1 = 2,           /* cpp/goss/GRL1.cpp:61-82 */
    GOSS_GRL2 = 3,           /* cpp/goss/GRL2.cpp:63-86 */
    GOSS_THETA = 4,          /* cpp/goss/ThetaSolver.cpp:49-155 */
    GOSS_ESDIRK23A = 5,      /* cpp/goss/ESDIRK23a.cpp:280-316 */
    GOSS_RL1 = 6,            /* cpp/goss/RL1.cpp:60-80, RL1.h:68-77 */
    GOSS_RL2 = 7,            /* cpp/goss/RL2.cpp:64-87 */
    GOSS_RK2 = 8,            /* cpp/goss/RK2.cpp:62-92 */
    GOSS_IMPLICIT_EULER = 9, /* cpp/goss/ImplicitEuler.cpp:57-152 */
    GOSS_NUM_SOLVERS = 10
};

/* Arithmetic of the right-hand side.  States are always stored and
 * accumulated in FP64; GOSS_FP32 evaluates the model and the explicit
 * update in FP32.  The implicit solvers (ThetaSolver, ImplicitEuler,
 * ESDIRK23a) in GOSS_FP32 evaluate only the Newton matrix's Jacobian in FP32,
 * from the model's analytic Jacobian (models generated with it); right-hand
 * sides, residuals, LU and updates stay FP64.  GOSS_FP64
 * evaluates the model's split program (every distinct exponential and
 * reciprocal once); GOSS_FP64_PRINTED evaluates it in the printed operation
 * order of the reference's generated model code (GRL1 only: the plain FP64
 * path the FP32 kernels are compared with). */
enum goss_precision { GOSS_FP64 = 0, GOSS_FP32 = 1, GOSS_FP64_PRINTED = 2 };

enum goss_status {
    GOSS_OK = 0,
    GOSS_ERR_ARGUMENT = 1,    /* invalid argument (std::invalid_argument / ValueError) */
    GOSS_ERR_CUDA = 2,        /* CUDA runtime failure */
    GOSS_ERR_NEWTON = 3,      /* ThetaSolver: dt fell below min_dt (ThetaSolver.cpp:133-149) */
    GOSS_ERR_UNSUPPORTED = 4, /* solver / model combination not available */
    GOSS_ERR_TIMEOUT = 5,     /* a bounded device loop hit its iteration cap */
    GOSS_ERR_NOT_ATTACHED = 6
};

/* Bits of the device status word (goss_system_status). */
enum goss_flag_bits {
    GOSS_FLAG_NONFINITE = 1u,     /* a node produced a non-finite state */
    GOSS_FLAG_NEWTON_FAILED = 2u, /* a node's step size fell below min_dt */
    GOSS_FLAG_ITERATION_CAP = 4u  /* a node exhausted the loop guard */
};

/* Solver parameters: the public members of the reference solver classes.
 * goss_solver_default_params() fills the reference defaults. */
typedef struct goss_solver_params {
    double ldt;                     /* ODESolver::_ldt, <= 0: one step per interval (ODESolver.h:137) */
    double delta;                   /* GRL1::delta (GRL1.h:39) */
    double eta_0;                   /* ImplicitODESolver.h:36 */
    double kappa;                   /* ImplicitODESolver.h:37 */
    double relative_tolerance;      /* ImplicitODESolver.h:38 */
    double max_relative_previous_residual; /* ImplicitODESolver.h:40 */
    int32_t max_iterations;         /* ImplicitODESolver.h:39 */
    int32_t always_recompute_jacobian; /* ImplicitODESolver.h:41 */
    int32_t num_refinements_without_always_recomputing_jacobian; /* ThetaSolver.h:35, ESDIRK23a.h:37 */
    double min_dt;                  /* ThetaSolver.h:36, ESDIRK23a.h:38 */
    double theta;                   /* ThetaSolver.h:37 */
} goss_solver_params;

/* One kernel launch of a solver over a node range (filled by the runtime,
 * consumed by a model module's launch function). */
typedef struct goss_launch {
    int32_t solver;
    int32_t precision;
    uint32_t num_nodes;
    uint32_t block;          /* threads per block, 0 = module default */
    uint64_t ld;             /* row stride of the device arrays, >= num_nodes */
    double* states;          /* device [num_states][ld] */
    const double* field_params; /* device [num_field_parameters][ld] (may be NULL if none) */
    double* solver_state;    /* device, solver specific (goss_model_desc.solver_state_rows) */
    uint32_t* flags;         /* device status word */
    uint8_t* node_status;    /* device [ld] per-node flag bits */
    const double* params;    /* host [num_parameters] uniform parameter values */
    const goss_solver_params* solver_params; /* host */
    double t;
    double interval;
    uint64_t max_loop;       /* guard for adaptive loops (0 = default) */
    void* stream;            /* cudaStream_t */
} goss_launch;

/* Batched evaluation of the model on device arrays (used by ODE.eval and the
 * tests): out = rhs (what = 0), [linear; rhs] (what = 1), the monitored values
 * (what = 2) or, for a model with has_jacobian, the analytic Jacobian
 * [num_states * num_states][ld], entry (i, j) = d f_i / d y_j in row
 * i * num_states + j (what = 3). */
typedef struct goss_eval_launch {
    int32_t what;
    int32_t precision;
    uint32_t num_nodes;
    uint64_t ld;
    const double* states;       /* device [num_states][ld] */
    const double* field_params; /* device [nfp][ld] or NULL */
    const double* times;        /* device [num_nodes] */
    double* out;                /* device [rows][ld], rows as listed above */
    const double* params;       /* host [num_parameters] */
    void* stream;
} goss_eval_launch;

/* Adjoint of a GRL1 trajectory (no counterpart in the reference).  The
 * trajectory is the reference's user loop: for j < num_intervals,
 * forward(t0 + j*interval, interval) with steps_per_interval GRL1 steps, the
 * state trace_state sampled after every interval.
 *   mode 0 (record): states (in: initial, out: final) -> trace [J][ld] and a
 *     checkpoint every checkpoint_every steps (a multiple of
 *     steps_per_interval) in checkpoints: FP32 [C][2n][ld] floats (hi, lo),
 *     FP64 [C][n][ld] doubles, C = ceil(J*S/K).
 *   mode 1 (backward): trace_bar [J][ld] = dLoss/dtrace -> field_params_bar
 *     [nfp][ld] = dLoss/dfield_params and states_bar [n][ld] = dLoss/dstates
 *     (initial); scratch holds [K][n][round_up(num_nodes, 256) + 256] values
 *     of the arithmetic type (K = checkpoint_every).
 *   tape (both modes, may be NULL with taped_segments 0): the input state of
 *     every step of the last taped_segments checkpoint segments, written by
 *     the record and read by the backward in place of recomputing those
 *     segments; [taped_segments][K][n][round_up(num_nodes, 256) + 256]
 *     values of the arithmetic type (the scratch layout per segment). */
typedef struct goss_adjoint_launch {
    int32_t mode;
    int32_t solver;           /* GOSS_GRL1 */
    int32_t precision;
    uint32_t num_nodes;
    uint32_t block;           /* backward threads per block: 0 = chosen from the
                                 node count, else a multiple of 32 <= 128 (FP32)
                                 or <= 256 (FP64) */
    uint64_t ld;
    double* states;
    const double* field_params;
    const double* params;     /* host [num_parameters] */
    double t0;
    double interval;
    uint32_t num_intervals;
    uint32_t steps_per_interval;
    uint32_t checkpoint_every;
    uint32_t trace_state;
    void* checkpoints;
    double* trace;
    const double* trace_bar;
    void* scratch;
    double* field_params_bar;
    double* states_bar;
    uint32_t* flags;
    void* stream;
    void* tape;
    uint32_t taped_segments;  /* <= C */
    int32_t reverse_precision; /* arithmetic of the backward's step VJPs: the
                                  record's precision, or GOSS_FP64 with precision
                                  GOSS_FP32 (GRL1): the FP32 trajectory (its
                                  checkpoints, tape and recomputed steps)
                                  differentiated in FP64 */
} goss_adjoint_launch;

/* A compiled model: produced by the code generator for one .ode model and one
 * choice of field parameters; replaces the goss::ParameterizedODE plugin and
 * its extern "C" create_<Name>() factory (python/goss/codegeneration.py:109-112). */
typedef struct goss_model_desc {
    uint32_t abi_version;
    const char* name;
    uint32_t num_states;
    uint32_t num_parameters;
    uint32_t num_field_parameters;
    uint32_t num_monitored;
    const char* const* state_names;
    const char* const* parameter_names;
    const char* const* field_parameter_names;
    const uint32_t* field_parameter_indices;
    const double* initial_conditions;
    const double* default_parameters;
    const uint8_t* linear_terms;
    uint32_t supported_solvers;   /* bit i set: solver kind i compiled */
    int (*launch)(const goss_launch* launch);
    int (*eval)(const goss_eval_launch* launch);
    /* rows of FP64 per node that solver kind s needs in solver_state */
    uint32_t (*solver_state_rows)(int32_t solver);
    /* static FP operation census of one linearized evaluation and one rhs
     * evaluation: add, mul, div, exp, log, sqrt, pow, cmp, misc */
    const uint32_t* op_census_linearized;
    const uint32_t* op_census_rhs;
    /* GRL1 trajectory adjoint (goss_adjoint_launch) */
    int (*adjoint)(const goss_adjoint_launch* launch);
    /* 1: generated with the analytic Jacobian (the reference's code_params
     * "generate_jacobian", python/goss/codegeneration.py:622-641): eval what=3
     * returns it and ThetaSolver/ImplicitEuler/ESDIRK23a use it in place of
     * forward differences (ODE::compute_jacobian, ODE.cpp:47-67) */
    uint32_t has_jacobian;
    /* packed entries of the implicit solvers' Newton matrix: the Jacobian's
     * structural non-zeros, the diagonal and the LU fill-in */
    uint32_t lu_nnz;
} goss_model_desc;

/* One population of a heterogeneous batch (filled by the runtime). */
typedef struct goss_batch_pop {
    int32_t kind;            /* index into the batch module's kinds */
    uint32_t num_nodes;
    uint64_t ld;
    double* states;          /* device [num_states][ld] */
    const double* field_params;
    uint8_t* node_status;
    uint32_t* flags;
    const double* params;    /* host [num_parameters] */
    const goss_solver_params* solver_params; /* host */
} goss_batch_pop;

/* One launch of a batch module over all populations. */
typedef struct goss_batch_launch {
    int32_t precision;
    uint32_t num_pops;
    const goss_batch_pop* pops;
    const uint32_t* order;   /* tile order of the populations (NULL: as given) */
    uint32_t block;          /* nodes per tile = threads per block */
    uint32_t grid;           /* persistent grid size (0: one block per tile) */
    uint32_t schedule;       /* 0: round-robin tiles, 1: tiles claimed from an atomic counter,
                                2: persistent CTAs staging the next tile's rows in shared memory
                                   with bulk asynchronous copies (grid 0: all resident CTAs) */
    uint32_t* counters;      /* device [2], zero before the first launch */
    double t;                /* forward f of this launch runs on */
    double interval;         /* [t + (first_forward + f) * interval, + interval) */
    uint64_t first_forward;
    uint32_t forwards;       /* consecutive forwards in this launch (0 or 1: one), the
                                states kept on chip in between */
    void* stream;
} goss_batch_launch;

/* A compiled batch module: the kernels of several (model variant, explicit
 * solver) kinds in one persistent kernel.  No counterpart in the reference,
 * which runs one ODESystemSolver per population in sequence. */
typedef struct goss_batch_desc {
    uint32_t abi_version;
    const char* name;
    uint32_t num_kinds;
    const char* const* kind_variants; /* model variant of each kind */
    const int32_t* kind_solvers;      /* solver kind of each kind */
    const uint32_t* kind_num_states;
    int (*launch)(const goss_batch_launch* launch);
} goss_batch_desc;

typedef struct goss_system goss_system;
typedef struct goss_batch goss_batch;

/* ODESystemSolver(uint nodes, shared_ptr<ODESolver>, shared_ptr<ParameterizedODE>)
 * (ODESystemSolver.cpp:45-59): allocates device state, sets the initial
 * conditions and default field parameters (reset_default). */
GOSS_API int goss_system_create(const goss_model_desc* model, int32_t solver, const goss_solver_params* params,
                                uint32_t num_nodes, int32_t precision, int32_t device, goss_system** out);
GOSS_API int goss_system_destroy(goss_system* sys);

/* reference defaults of a solver kind */
GOSS_API int goss_solver_default_params(int32_t solver, goss_solver_params* out);
GOSS_API int goss_system_set_solver_params(goss_system* sys, const goss_solver_params* params);
GOSS_API int goss_system_get_solver_params(const goss_system* sys, goss_solver_params* out);

/* ODESystemSolver::forward(t, interval) (ODESystemSolver.cpp:67-79) */
GOSS_API int goss_system_forward(goss_system* sys, double t, double interval);
/* ODESystemSolver::solve (ODESystemSolver.cpp:81-99): field_states is
 * [num_timesteps][num_nodes][nfs] (tangled) or [num_timesteps][nfs][num_nodes];
 * row 0 is left untouched, row i holds the field states after the step to t[i]. */
GOSS_API int goss_system_solve(goss_system* sys, double* field_states, const double* t, uint64_t num_timesteps,
                               int32_t tangled);

/* Field states: the states named by field_state_indices (ParameterizedODE.h:147-150). */
GOSS_API int goss_system_set_field_state_indices(goss_system* sys, const uint32_t* indices, uint32_t count);
GOSS_API int goss_system_get_field_states(const goss_system* sys, double* values, int32_t tangled);
GOSS_API int goss_system_set_field_states(goss_system* sys, const double* values, int32_t tangled);
GOSS_API int goss_system_get_field_state_components(const goss_system* sys, double* values,
                                                    uint32_t num_components, const uint32_t* components,
                                                    int32_t tangled);
GOSS_API int goss_system_set_field_state_components(goss_system* sys, const double* values,
                                                    uint32_t num_components, const uint32_t* components,
                                                    int32_t tangled);
GOSS_API int goss_system_get_field_parameters(const goss_system* sys, double* values, int32_t tangled);
GOSS_API int goss_system_set_field_parameters(goss_system* sys, const double* values, int32_t tangled);

/* All states, node-major [num_nodes][num_states] (ODESystemSolver::states()). */
GOSS_API int goss_system_get_states(const goss_system* sys, double* states);
GOSS_API int goss_system_set_states(goss_system* sys, const double* states);

/* Uniform model parameters (ParameterizedODE::set_parameter/get_parameter by index). */
GOSS_API int goss_system_set_parameter(goss_system* sys, uint32_t index, double value);
GOSS_API int goss_system_get_parameter(const goss_system* sys, uint32_t index, double* value);

/* reset_default() (ODESystemSolver.cpp:192-216); also resets implicit solver state */
GOSS_API int goss_system_reset_default(goss_system* sys);

/* set_num_threads/get_num_threads keep their API; the device ignores them. */
GOSS_API int goss_system_set_num_threads(goss_system* sys, uint32_t num_threads);
GOSS_API uint32_t goss_system_get_num_threads(const goss_system* sys);
GOSS_API uint32_t goss_system_num_nodes(const goss_system* sys);

/* Launch configuration (threads per block, a multiple of 32; 0 = the default:
 * 128 for the explicit solvers, 256 for the implicit ones, whose blocks run in
 * lockstep; the kernels take at most 128 and 256). */
GOSS_API int goss_system_set_block_size(goss_system* sys, uint32_t block);

/* Status word accumulated since the last clear (goss_flag_bits). */
GOSS_API int goss_system_status(goss_system* sys, uint32_t* flags, int32_t clear);
/* Per-node flag bits [num_nodes]. */
GOSS_API int goss_system_node_status(const goss_system* sys, uint8_t* out);
/* Counters of the implicit solvers per node: jacobian computations,
 * rejected steps, accepted steps (any pointer may be NULL). */
GOSS_API int goss_system_counters(const goss_system* sys, int64_t* jac_comp, int64_t* rejected, int64_t* accepted);

/* Device-resident access for callers that keep data on the GPU. */
GOSS_API int goss_system_device_states(goss_system* sys, double** states, uint64_t* ld);
GOSS_API int goss_system_device_field_params(goss_system* sys, double** field_params, uint64_t* ld);
GOSS_API int goss_system_set_stream(goss_system* sys, void* stream);
GOSS_API int goss_system_forward_async(goss_system* sys, double t, double interval);
GOSS_API int goss_system_synchronize(goss_system* sys);

/* Batched model evaluation on host arrays: states [count][n], times [count],
 * field_params [count][nfp] (may be NULL), out [count][n] (what=0),
 * [count][2n] = (linear, rhs) (what=1), [count][num_monitored] (what=2) or
 * [count][n*n] = the analytic Jacobian, row-major (what=3, has_jacobian). */
GOSS_API int goss_model_eval(const goss_model_desc* model, int32_t what, int32_t precision, const double* params,
                             const double* states, const double* field_params, const double* times, uint64_t count,
                             double* out, int32_t device);

/* CUDA graphs of forward loops.  goss_system_capture records num_steps
 * consecutive forward(t0 + k*interval, interval) launches into a graph;
 * goss_system_replay launches it (solver and model parameters are those at
 * capture time) and synchronises; a new capture replaces the old graph. */
GOSS_API int goss_system_capture(goss_system* sys, double t0, double interval, uint32_t num_steps);
GOSS_API int goss_system_replay(goss_system* sys);

/* Heterogeneous batches: the populations are existing systems (their states,
 * field parameters, solver and model parameters); kinds[i] selects the
 * batch module's kind for systems[i] (it must match the system's model
 * variant name and solver).  One goss_batch_forward launches one kernel for
 * all populations; capture/replay record num_steps forwards in a CUDA graph.
 * goss_batch_time measures num_steps forwards (graph or direct launches)
 * with CUDA events on the batch stream, leaving the states advanced. */
GOSS_API int goss_batch_create(const goss_batch_desc* desc, goss_system* const* systems, const int32_t* kinds,
                               uint32_t count, int32_t precision, goss_batch** out);
GOSS_API int goss_batch_destroy(goss_batch* batch);
GOSS_API int goss_batch_set_config(goss_batch* batch, uint32_t block, uint32_t grid, uint32_t schedule,
                                   const uint32_t* order);
GOSS_API int goss_batch_forward(goss_batch* batch, double t, double interval);
GOSS_API int goss_batch_capture(goss_batch* batch, double t0, double interval, uint32_t num_steps);
/* Forwards one launch of a captured graph performs (0, the default: all
 * num_steps of the capture in one launch; 1: one launch per forward).  Every
 * node's states stay in registers across the forwards of a launch; forward k
 * still runs on [t0 + k*interval, t0 + (k+1)*interval) with the solver's
 * internal steps, so the results do not depend on this setting. */
GOSS_API int goss_batch_set_forwards_per_launch(goss_batch* batch, uint32_t forwards);
GOSS_API int goss_batch_replay(goss_batch* batch);
GOSS_API int goss_batch_time(goss_batch* batch, double t0, double interval, uint32_t num_steps, int32_t use_graph,
                             float* ms);
GOSS_API const char* goss_batch_last_error(const goss_batch* batch);

/* Batched model evaluation that allocates no device memory.  No counterpart
 * in the reference: it exists for callers that must not have a library call
 * cudaMalloc -- a process whose GPU memory belongs to another allocator (a
 * framework's caching allocator that reserved the device, or a fixed memory
 * budget), where an allocation would fail, stall on that allocator or
 * fragment its pool.
 *
 * Same arithmetic as goss_model_eval, but every pointer is DEVICE memory on
 * the current device: states [count][n], field_params [count][nfp] (NULL:
 * the parameter values), times [count], out [count][width] with width n
 * (what = 0), 2n (what = 1: linear then rhs), num_monitored (what = 2) or
 * n*n (what = 3: the analytic Jacobian of a model with has_jacobian).
 * params is a HOST array of num_parameters values (NULL: defaults).
 *
 * Working arrays live in one fixed file-scope device array of
 * goss_model_eval_noalloc_capacity() doubles (16 MiB) that every GPU using
 * this library keeps until the process exits; (n + nfp + width) * count,
 * with count rounded up to 32, must fit or the call fails with
 * GOSS_ERR_ARGUMENT.  The first call on a device, and the first after the
 * device's context was reset, looks up that array's device address.  All
 * calls share the array and it keeps the last call's contents, so calls that
 * overlap on the GPU (other streams, other threads) race; the call
 * synchronises `stream` before it returns.  A CUDA error left pending by earlier work is reported
 * (GOSS_ERR_CUDA) and left pending. */
GOSS_API int goss_model_eval_noalloc(const goss_model_desc* model, int32_t what, int32_t precision,
                                     const double* params, const double* states, const double* field_params,
                                     const double* times, uint64_t count, double* out, void* stream);
GOSS_API uint64_t goss_model_eval_noalloc_capacity(void);

/* Single-matrix helpers of the ODE plugin interface, on the host (the
 * reference's ODE::lu_factorize / ODE::forward_backward_subst, ODE.cpp:69-132):
 * in-place LU without pivoting of a row-major n x n matrix, and the solve
 * with that factorisation (b and x may alias). */
GOSS_API int goss_lu_factorize(uint32_t n, double* mat);
GOSS_API int goss_forward_backward_subst(uint32_t n, const double* mat, const double* b, double* x);

GOSS_API const char* goss_system_last_error(const goss_system* sys);
GOSS_API const char* goss_last_error(void);
GOSS_API uint32_t goss_abi_version(void);

/* No counterpart in the reference: the CUDA-core peaks the model kernels'
 * rooflines are measured against, on `device`: XU-pipe results per second
 * (independent ex2/lg2 chains, the pipe of the models' exponentials and
 * reciprocals) and FP32 fused multiply-adds per second (one op each), each the
 * best of three timed launches filling every SM.  Takes a few milliseconds. */
GOSS_API int goss_measure_peaks(int32_t device, double* xu_ops_per_s, double* fp32_ops_per_s);
/* No counterpart in the reference: FP64 fused multiply-adds per second on
 * `device` (independent fma.rn.f64 chains, 2048 threads per SM, best of three
 * timed launches), the FP64-pipe peak of the FP64 model kernels' roofline. */
GOSS_API int goss_measure_fp64_peak(int32_t device, double* fp64_fma_per_s);

#ifdef __cplusplus
}
#endif
#endif
