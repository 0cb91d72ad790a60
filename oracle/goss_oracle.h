/*
 * Test infrastructure -- NOT part of the product path.
 *
 * CPU restatement (plain C, FP64) of goss's multi-node solve path,
 * ODESystemSolver::forward (reference cpp/goss/ODESystemSolver.cpp:67-79)
 * stepping one model at every node with ExplicitEuler, RK4, GRL1, GRL2,
 * ThetaSolver or ESDIRK23a.  It is the checker the parity tests, smoke()
 * and the CPU-baseline leg of bench.py compare the CUDA kernels against.
 *
 * Layout follows the reference: node-major (AoS) states[node*n + i] and
 * field_params[node*nfp + k] (ODESystemSolver.h:173-176).
 *
 * Semantics that differ from a single shared reference solver object:
 * implicit solvers keep their adaptive state (eta, dt history, Jacobian)
 * per node, i.e. every node behaves as if it were solved by its own
 * solver instance.  The reference shares one solver object across the node
 * loop (ODESystemSolver.cpp:76-77), which leaks that state from node to
 * node and makes results depend on the OpenMP schedule.
 */
#ifndef GOSS_ORACLE_H
#define GOSS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_model {
    const char* name;
    int num_states;
    int num_params;
    int num_field_params;
    const unsigned* field_param_index; /* index of each field parameter in params[] */
    void (*rhs)(const double* states, double time, const double* params, double* values);
    void (*linearized)(const double* states, double time, const double* params, double* linear,
                       double* rhs, int only_linear);
    const double* ic;
    const double* default_params;
    const unsigned char* linear_terms;
    /* analytic Jacobian jac[i*n + j] = d f_i / d y_j, the generated override
     * of ODE::compute_jacobian (ODE.h:71); NULL: forward differences */
    void (*jacobian)(const double* states, double time, const double* params, double* jac);
} oracle_model;

enum {
    ORACLE_EXPLICIT_EULER = 0,
    ORACLE_RK4 = 1,
    ORACLE_GRL1 = 2,
    ORACLE_GRL2 = 3,
    ORACLE_THETA = 4,
    ORACLE_ESDIRK23A = 5,
    ORACLE_RL1 = 6,
    ORACLE_RL2 = 7,
    ORACLE_RK2 = 8,
    ORACLE_IMPLICIT_EULER = 9
};

/* solver parameters (public members of the reference solver classes) */
typedef struct oracle_solver_params {
    double ldt;            /* ODESolver::_ldt, <= 0 means one step per interval */
    double delta;          /* GRL1::delta (GRL1.h:39) */
    /* ImplicitODESolver (ImplicitODESolver.h:36-41) */
    double eta_0, kappa, relative_tolerance, max_relative_previous_residual;
    int max_iterations;
    int always_recompute_jacobian;
    /* ThetaSolver (ThetaSolver.h:35-37) */
    int num_refinements_without_always_recomputing_jacobian;
    double min_dt;
    double theta;
} oracle_solver_params;

void oracle_default_solver_params(int solver, oracle_solver_params* p);

typedef struct oracle_system oracle_system;

/* Create a system of num_nodes nodes; states start at the model's initial
 * conditions and field parameters at the model's default values
 * (ODESystemSolver::reset_default, ODESystemSolver.cpp:192-216). */
oracle_system* oracle_system_create(const oracle_model* model, int solver, const oracle_solver_params* sp,
                                    uint32_t num_nodes);
void oracle_system_destroy(oracle_system* s);
double* oracle_system_states(oracle_system* s);        /* [N][n] */
double* oracle_system_field_params(oracle_system* s);  /* [N][nfp] */
double* oracle_system_params(oracle_system* s);        /* [num_params], uniform values */
/* Advance every node by `interval` starting at t.  Returns 0, or the number
 * of nodes whose Newton solve failed below min_dt (ThetaSolver.cpp:133-149). */
int oracle_system_forward(oracle_system* s, double t, double interval, int num_threads);
/* Per-node counters of the implicit solvers: jacobian computations,
 * rejected steps, accepted steps (may be NULL). */
void oracle_system_counters(oracle_system* s, int64_t* jac_comp, int64_t* rejected, int64_t* accepted);

/* Single-node building blocks, exposed for the tests. */
void oracle_compute_jacobian(const oracle_model* m, const double* params, double* states, double time,
                             double* jac, double* f1, double* f2);
void oracle_lu_factorize(int n, double* mat);
void oracle_forward_backward_subst(int n, const double* mat, const double* b, double* x);

#ifdef __cplusplus
}
#endif
#endif
