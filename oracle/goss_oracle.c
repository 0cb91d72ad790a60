/*
 * Test infrastructure -- NOT part of the product path.
 *
 * CPU restatement (FP64) of the goss per-node solvers and the multi-node
 * driver.  Each routine cites the reference file:line it restates; the
 * operation order of every floating-point expression follows the reference
 * so results agree with the reference solvers bit for bit when compiled with
 * the same flags (no FMA contraction, -O2/-O3 without fast-math).
 */
#include "goss_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define GOSS_EPS 3.0e-16 /* cpp/goss/constants.h:25 */

/* std::max / std::min semantics (first argument wins ties and NaNs) */
static double std_max(double a, double b) { return (a < b) ? b : a; }
static double std_min(double a, double b) { return (b < a) ? b : a; }

/* ---------------------------------------------------------------------- */
/* per-node solver state                                                  */
/* ---------------------------------------------------------------------- */
typedef struct node_state {
    /* ImplicitODESolver members (ImplicitODESolver.h:81-99) */
    double eta;
    int recompute_jacobian;
    int newton_iterations;
    int always_recompute_jacobian;
    int64_t jac_comp, rejects, accepted;
    /* ESDIRK23a members (ESDIRK23a.h:92-112) */
    double e_eta, loc_error, prev_dt, dt;
    int first_step, new_jacobian;
    int justrefined; /* ThetaSolver::_justrefined (ThetaSolver.h:68), kept across calls */
    double* jac;  /* [n*n] */
    double* jfac; /* [n*n] */
} node_state;

struct oracle_system {
    const oracle_model* m;
    int solver;
    oracle_solver_params sp;
    uint32_t N;
    double* states;
    double* fparams;
    double* params;
    node_state* ns;
};

void oracle_default_solver_params(int solver, oracle_solver_params* p)
{
    memset(p, 0, sizeof(*p));
    p->ldt = -1.0;                       /* ODESolver.h:137 */
    p->delta = 1e-8;                     /* GRL1.h:39 */
    p->eta_0 = 1.0;                      /* ImplicitODESolver.h:36 */
    p->kappa = 0.1;                      /* :37 */
    p->relative_tolerance = 1e-12;       /* :38 */
    p->max_iterations = 30;              /* :39 */
    p->max_relative_previous_residual = 0.01; /* :40 */
    p->always_recompute_jacobian = 0;    /* :41 */
    p->num_refinements_without_always_recomputing_jacobian = 2; /* ThetaSolver.h:35, ImplicitEuler.h:35 */
    p->min_dt = solver == ORACLE_ESDIRK23A ? 0.001 : 0.0001;   /* ESDIRK23a.h:38, ThetaSolver.h:36, ImplicitEuler.h:36 */
    p->theta = 0.5;                      /* ThetaSolver.h:37 */
}

static void node_reset(oracle_system* s, node_state* st)
{
    int n = s->m->num_states;
    /* ImplicitODESolver::reset (ImplicitODESolver.cpp:80-90) */
    st->eta = s->sp.eta_0;
    st->recompute_jacobian = 1;
    st->newton_iterations = 0;
    st->always_recompute_jacobian = s->sp.always_recompute_jacobian;
    st->jac_comp = st->rejects = st->accepted = 0;
    /* ESDIRK23a constructor values (ESDIRK23a.cpp:27-39) */
    st->e_eta = 1.0;
    st->loc_error = 1e9;
    st->prev_dt = 0.1;
    st->dt = 0.1; /* AdaptiveImplicitSolver.cpp:20 (_dt(.1)) */
    st->first_step = 1;
    st->new_jacobian = 1;
    st->justrefined = 0;
    if (s->solver == ORACLE_THETA || s->solver == ORACLE_ESDIRK23A || s->solver == ORACLE_IMPLICIT_EULER) {
        st->jac = (double*)calloc((size_t)n * n, sizeof(double));
        st->jfac = (double*)calloc((size_t)n * n, sizeof(double));
    } else {
        st->jac = st->jfac = NULL;
    }
}

oracle_system* oracle_system_create(const oracle_model* m, int solver, const oracle_solver_params* sp,
                                    uint32_t N)
{
    oracle_system* s = (oracle_system*)calloc(1, sizeof(oracle_system));
    int n = m->num_states, nfp = m->num_field_params;
    s->m = m;
    s->solver = solver;
    if (sp)
        s->sp = *sp;
    else
        oracle_default_solver_params(solver, &s->sp);
    s->N = N;
    s->states = (double*)malloc(sizeof(double) * (size_t)N * n);
    s->fparams = (double*)malloc(sizeof(double) * (size_t)N * (nfp > 0 ? nfp : 1));
    s->params = (double*)malloc(sizeof(double) * (size_t)(m->num_params > 0 ? m->num_params : 1));
    memcpy(s->params, m->default_params, sizeof(double) * (size_t)m->num_params);
    s->ns = (node_state*)calloc(N, sizeof(node_state));
    /* reset_default (ODESystemSolver.cpp:192-216) */
    for (uint32_t node = 0; node < N; ++node) {
        for (int i = 0; i < n; ++i)
            s->states[(size_t)node * n + i] = m->ic[i];
        for (int k = 0; k < nfp; ++k)
            s->fparams[(size_t)node * nfp + k] = m->default_params[m->field_param_index[k]];
        node_reset(s, &s->ns[node]);
    }
    return s;
}

void oracle_system_destroy(oracle_system* s)
{
    if (!s)
        return;
    for (uint32_t i = 0; i < s->N; ++i) {
        free(s->ns[i].jac);
        free(s->ns[i].jfac);
    }
    free(s->ns);
    free(s->states);
    free(s->fparams);
    free(s->params);
    free(s);
}

double* oracle_system_states(oracle_system* s) { return s->states; }
double* oracle_system_field_params(oracle_system* s) { return s->fparams; }
double* oracle_system_params(oracle_system* s) { return s->params; }

void oracle_system_counters(oracle_system* s, int64_t* jac_comp, int64_t* rejected, int64_t* accepted)
{
    for (uint32_t i = 0; i < s->N; ++i) {
        if (jac_comp)
            jac_comp[i] = s->ns[i].jac_comp;
        if (rejected)
            rejected[i] = s->ns[i].rejects;
        if (accepted)
            accepted[i] = s->ns[i].accepted;
    }
}

/* ---------------------------------------------------------------------- */
/* linear algebra: ODE::compute_jacobian / lu_factorize / fbs            */
/* ---------------------------------------------------------------------- */

/* ODE::compute_jacobian (ODE.cpp:47-67): forward differences, column i
 * perturbed by sqrt(1e-15*max(1e-5,|y_i|)), stored row-major jac[j*n+i];
 * a model generated with the analytic Jacobian overrides it (the plugin's
 * compute_jacobian, which leaves f1 untouched). */
void oracle_compute_jacobian(const oracle_model* m, const double* params, double* states, double time,
                             double* jac, double* f1, double* f2)
{
    int n = m->num_states;
    if (m->jacobian) {
        m->jacobian(states, time, params, jac);
        return;
    }
    m->rhs(states, time, params, f1);
    for (int i = 0; i < n; ++i) {
        double ysafe = states[i];
        double max = 1e-5 > fabs(ysafe) ? 1e-5 : fabs(ysafe);
        double delta = sqrt(1e-15 * max);
        states[i] += delta;
        m->rhs(states, time, params, f2);
        for (int j = 0; j < n; ++j)
            jac[j * n + i] = (f2[j] - f1[j]) / delta;
        states[i] = ysafe;
    }
}

/* ODE::lu_factorize (ODE.cpp:69-100): in-place Doolittle LU, no pivoting. */
void oracle_lu_factorize(int n, double* mat)
{
    double sum;
    int i, k, r;
    for (k = 1; k < n; k++) {
        for (i = 0; i <= k - 1; ++i) {
            sum = 0.0;
            for (r = 0; r <= i - 1; r++)
                sum += mat[i * n + r] * mat[r * n + k];
            mat[i * n + k] -= sum;
            sum = 0.0;
            for (r = 0; r <= i - 1; r++)
                sum += mat[k * n + r] * mat[r * n + i];
            mat[k * n + i] = (mat[k * n + i] - sum) / mat[i * n + i];
        }
        sum = 0.0;
        for (r = 0; r <= k - 1; r++)
            sum += mat[k * n + r] * mat[r * n + k];
        mat[k * n + k] -= sum;
    }
}

/* ODE::forward_backward_subst (ODE.cpp:102-132).  b and x may alias. */
void oracle_forward_backward_subst(int n, const double* mat, const double* b, double* dx)
{
    double sum;
    dx[0] = b[0];
    for (int i = 1; i < n; ++i) {
        sum = 0.0;
        for (int j = 0; j <= i - 1; ++j)
            sum = sum + mat[i * n + j] * dx[j];
        dx[i] = b[i] - sum;
    }
    dx[n - 1] = dx[n - 1] / mat[(n - 1) * n + (n - 1)];
    for (int i = n - 2; i >= 0; i--) {
        sum = 0;
        for (int j = i + 1; j < n; ++j)
            sum = sum + mat[i * n + j] * dx[j];
        dx[i] = (dx[i] - sum) / mat[i * n + i];
    }
}

/* ImplicitODESolver::norm (ImplicitODESolver.cpp:247-256) */
static double l2norm(int n, const double* v)
{
    double s = 0;
    for (int i = 0; i < n; ++i)
        s += v[i] * v[i];
    return sqrt(s);
}

/* ---------------------------------------------------------------------- */
/* explicit solvers                                                       */
/* ---------------------------------------------------------------------- */
static unsigned long num_steps(double ldt_0, double dt)
{
    /* e.g. GRL1.cpp:66: ldt_0 > 0 ? ceil(dt/ldt_0 - 1e-12) : 1 */
    return ldt_0 > 0 ? (unsigned long)ceil(dt / ldt_0 - 1.0E-12) : 1UL;
}

typedef struct scratch {
    double *a, *b, *c, *d, *e, *f, *g, *h, *i, *j, *k, *l;
} scratch;

/* ExplicitEuler::forward (ExplicitEuler.cpp:64-87) */
static void fwd_euler(const oracle_model* m, const double* P, double* y, double t, double dt, double ldt_0,
                      scratch* w)
{
    int n = m->num_states;
    unsigned long nsteps = num_steps(ldt_0, dt);
    double ldt = dt / nsteps, lt = t;
    for (unsigned long s = 0; s < nsteps; ++s) {
        m->rhs(y, lt, P, w->a);
        for (int i = 0; i < n; ++i)
            y[i] += ldt * w->a[i];
        lt += ldt;
    }
}

/* RK4::forward (RK4.cpp:68-102) with RK4::axpy (RK4.h:70-74) */
static void fwd_rk4(const oracle_model* m, const double* P, double* y, double t, double dt, double ldt_0,
                    scratch* w)
{
    int n = m->num_states;
    double *k1 = w->a, *k2 = w->b, *k3 = w->c, *k4 = w->d, *tmp = w->e;
    unsigned long nsteps = num_steps(ldt_0, dt);
    double ldt = dt / nsteps, lt = t;
    for (unsigned long j = 0; j < nsteps; ++j) {
        m->rhs(y, lt, P, k1);
        for (int i = 0; i < n; ++i)
            tmp[i] = y[i] + 0.5 * ldt * k1[i];
        m->rhs(tmp, lt + 0.5 * ldt, P, k2);
        for (int i = 0; i < n; ++i)
            tmp[i] = y[i] + 0.5 * ldt * k2[i];
        m->rhs(tmp, lt + 0.5 * ldt, P, k3);
        for (int i = 0; i < n; ++i)
            tmp[i] = y[i] + ldt * k3[i];
        m->rhs(tmp, lt + ldt, P, k4);
        for (int i = 0; i < n; ++i)
            y[i] += ldt * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]) / 6.0;
        lt += ldt;
    }
}

/* GRL1::_one_step (GRL1.h:72-84) */
static void grl_one_step(const oracle_model* m, const double* P, double* y2, const double* y, const double* y0,
                         double t, double dt, double delta, scratch* w)
{
    int n = m->num_states;
    double *lin = w->a, *rhs = w->b;
    m->linearized(y, t, P, lin, rhs, 0);
    for (int i = 0; i < n; ++i)
        y2[i] = (fabs(lin[i]) > delta) ? y0[i] + rhs[i] / lin[i] * (exp(lin[i] * dt) - 1.0)
                                       : y0[i] + rhs[i] * dt;
}

/* GRL1::forward (GRL1.cpp:61-82) */
static void fwd_grl1(const oracle_model* m, const double* P, double* y, double t, double dt, double ldt_0,
                     double delta, scratch* w)
{
    unsigned long nsteps = num_steps(ldt_0, dt);
    double ldt = dt / nsteps, lt = t;
    for (unsigned long s = 0; s < nsteps; ++s) {
        grl_one_step(m, P, y, y, y, lt, ldt, delta, w);
        lt += ldt;
    }
}

/* GRL2::forward (GRL2.cpp:63-86): half step to y2 linearised at y, then a
 * full step from y linearised at y2, both at time lt.  The reference's
 * `const double delta = delta;` (GRL2.cpp:67) reads an uninitialised local;
 * its g++ -O3 build takes the exponential branch whenever the linear term is
 * non-zero (bit-identical results to a threshold of 0, and different ones
 * for 1e-8), so GRL2 uses a threshold of 0 and ignores the delta parameter. */
static void fwd_grl2(const oracle_model* m, const double* P, double* y, double t, double dt, double ldt_0,
                     double delta, scratch* w)
{
    unsigned long nsteps = num_steps(ldt_0, dt);
    double ldt = dt / nsteps, lt = t;
    double* y2 = w->c;
    (void)delta;
    delta = 0.0;
    for (unsigned long s = 0; s < nsteps; ++s) {
        grl_one_step(m, P, y2, y, y, lt, ldt * 0.5, delta, w);
        grl_one_step(m, P, y, y2, y, lt, ldt, delta, w);
        lt += ldt;
    }
}

/* RL1::_one_step (RL1.h:68-77): linearized_eval with only_linear = true, then
 * the exponential update for the model's linear-term states (no threshold:
 * a zero linear coefficient gives the reference's 0/0) and Euler otherwise */
static void rl_one_step(const oracle_model* m, const double* P, double* y2, const double* y, const double* y0,
                        double t, double dt, scratch* w)
{
    int n = m->num_states;
    double *lin = w->a, *rhs = w->b;
    m->linearized(y, t, P, lin, rhs, 1);
    for (int i = 0; i < n; ++i)
        y2[i] = m->linear_terms[i] ? y0[i] + rhs[i] / lin[i] * (exp(lin[i] * dt) - 1.0) : y0[i] + rhs[i] * dt;
}

/* RL1::forward (RL1.cpp:60-80) */
static void fwd_rl1(const oracle_model* m, const double* P, double* y, double t, double dt, double ldt_0,
                    scratch* w)
{
    unsigned long nsteps = num_steps(ldt_0, dt);
    double ldt = dt / nsteps, lt = t;
    for (unsigned long s = 0; s < nsteps; ++s) {
        rl_one_step(m, P, y, y, y, lt, ldt, w);
        lt += ldt;
    }
}

/* RL2::forward (RL2.cpp:64-87): half step to y2 linearised at y, then a full
 * step from y linearised at y2, both at time lt */
static void fwd_rl2(const oracle_model* m, const double* P, double* y, double t, double dt, double ldt_0,
                    scratch* w)
{
    unsigned long nsteps = num_steps(ldt_0, dt);
    double ldt = dt / nsteps, lt = t;
    double* y2 = w->c;
    for (unsigned long s = 0; s < nsteps; ++s) {
        rl_one_step(m, P, y2, y, y, lt, ldt * 0.5, w);
        rl_one_step(m, P, y, y2, y, lt, ldt, w);
        lt += ldt;
    }
}

/* RK2::forward (RK2.cpp:62-92) with RK2::axpy (RK2.h:70-74): the midpoint rule */
static void fwd_rk2(const oracle_model* m, const double* P, double* y, double t, double dt, double ldt_0,
                    scratch* w)
{
    int n = m->num_states;
    double *k1 = w->a, *tmp = w->b;
    unsigned long nsteps = num_steps(ldt_0, dt);
    double ldt = dt / nsteps, lt = t;
    for (unsigned long j = 0; j < nsteps; ++j) {
        m->rhs(y, lt, P, k1);
        for (int i = 0; i < n; ++i)
            tmp[i] = y[i] + 0.5 * ldt * k1[i];
        m->rhs(tmp, lt + 0.5 * ldt, P, k1);
        for (int i = 0; i < n; ++i)
            y[i] += ldt * k1[i];
        lt += ldt;
    }
}

/* ---------------------------------------------------------------------- */
/* ThetaSolver                                                            */
/* ---------------------------------------------------------------------- */

/* ImplicitODESolver::compute_factorized_jacobian (ImplicitODESolver.cpp:92-105)
 * followed by mult (:107-112) and add_mass_matrix (:258-262); every state
 * is differential for the ODEs on this path. */
static void compute_factorized_jacobian(const oracle_model* m, const double* P, node_state* st, double* y,
                                        double t, double dt, double alpha, scratch* w)
{
    int n = m->num_states;
    oracle_compute_jacobian(m, P, y, t, st->jac, w->k, w->l);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            st->jac[i * n + j] *= (-dt * alpha);
    for (int i = 0; i < n; ++i)
        st->jac[i * n + i] += 1.0 * 1.0;
    oracle_lu_factorize(n, st->jac);
    st->jac_comp += 1;
}

/* ImplicitODESolver::newton_solve (ImplicitODESolver.cpp:114-245) */
static int newton_solve(const oracle_model* m, const double* P, const oracle_solver_params* sp, node_state* st,
                        double* z, const double* prev, const double* y0, double t, double dt, double alpha,
                        int always_recompute_jacobian, scratch* w)
{
    int n = m->num_states;
    double *yz = w->f, *f1 = w->g, *b = w->h, *dz = w->i;
    int step_ok = 1;
    st->newton_iterations = 0;
    double relative_previous_residual = 1.0, relative_residual = 1.0, previous_residual = 1.0;
    double initial_residual = 1.0, residual;
    do {
        for (int i = 0; i < n; ++i)
            yz[i] = y0[i] + z[i];
        m->rhs(yz, t, P, f1);
        for (int i = 0; i < n; ++i)
            b[i] = -z[i] * 1.0 + dt * (prev[i] + alpha * f1[i]);
        residual = l2norm(n, b);
        if (relative_residual < sp->relative_tolerance)
            break;
        if (st->recompute_jacobian || always_recompute_jacobian) {
            compute_factorized_jacobian(m, P, st, yz, t, dt, alpha, w);
            st->recompute_jacobian = 0;
        }
        oracle_forward_backward_subst(n, st->jac, b, dz);
        if (st->newton_iterations == 0) {
            initial_residual = residual;
            st->eta = st->eta > GOSS_EPS ? st->eta : GOSS_EPS;
            st->eta = pow(st->eta, 0.8);
        } else {
            relative_previous_residual = residual / previous_residual;
            st->recompute_jacobian = relative_previous_residual >= sp->max_relative_previous_residual;
            if (relative_previous_residual >= 1) {
                step_ok = 0;
                st->rejects++;
                st->recompute_jacobian = 1;
                break;
            }
            const double scaled =
                std_max(pow(relative_previous_residual, sp->max_iterations - st->newton_iterations), GOSS_EPS);
            if (residual > (sp->kappa * sp->relative_tolerance * (1 - relative_previous_residual) / scaled))
                st->recompute_jacobian = 1;
            st->eta = relative_previous_residual / (1.0 - relative_previous_residual);
        }
        if (st->newton_iterations > sp->max_iterations) {
            st->recompute_jacobian = 1;
            st->rejects++;
            step_ok = 0;
            break;
        }
        for (int i = 0; i < n; ++i)
            z[i] += dz[i];
        relative_residual = residual / initial_residual;
        previous_residual = residual;
        st->newton_iterations++;
    } while (st->eta * relative_residual >= sp->kappa * sp->relative_tolerance);
    return step_ok;
}

/* ThetaSolver::forward (ThetaSolver.cpp:49-155).  Returns 0 on success and
 * 1 when the step size fell below min_dt (the reference throws). */
static int fwd_theta(const oracle_model* m, const double* P, const oracle_solver_params* sp, node_state* st,
                     double* y, double t, double dt, scratch* w)
{
    int n = m->num_states;
    double *z1 = w->a, *ft1 = w->b, *prev = w->c;
    const double t_end = t + dt;
    const double ldt_0 = sp->ldt;
    double ldt = ldt_0 > 0 ? ldt_0 : dt;
    int num_refinements = 0;
    const double eps = GOSS_EPS * 1000;
    for (int i = 0; i < n; ++i)
        prev[i] = 0.0;
    while (1) {
        for (int i = 0; i < n; ++i)
            z1[i] = 0.0;
        if (fabs(sp->theta - 1.0) > GOSS_EPS) {
            m->rhs(y, t, P, ft1);
            for (int i = 0; i < n; ++i)
                prev[i] = (1 - sp->theta) * ft1[i];
        }
        if (num_refinements <= sp->num_refinements_without_always_recomputing_jacobian)
            st->always_recompute_jacobian = 1;
        int step_ok = newton_solve(m, P, sp, st, z1, prev, y, t + sp->theta * ldt, ldt, sp->theta,
                                   st->always_recompute_jacobian, w);
        if (step_ok) {
            for (int i = 0; i < n; ++i)
                y[i] += z1[i];
            t += ldt;
            st->accepted++;
            if (fabs(t - t_end) < eps)
                break;
            if (!st->justrefined) {
                const double tmp = 2.0 * ldt;
                if (ldt_0 > 0. && tmp >= ldt_0)
                    ldt = ldt_0;
                else
                    ldt = tmp;
            } else {
                st->justrefined = 0;
            }
            if ((t + ldt + GOSS_EPS) > t_end)
                ldt = t_end - t;
        } else {
            ldt /= 2.0;
            if (ldt < sp->min_dt)
                return 1;
            st->justrefined = 1;
            num_refinements += 1;
        }
    }
    return 0;
}

/* ImplicitEuler::forward (ImplicitEuler.cpp:57-152): the theta loop at
 * theta = 1 (no explicit part, stage time t + ldt), except that the Jacobian
 * is always recomputed once more than num_refinements_without_always_
 * recomputing_jacobian refinements happened (ThetaSolver: up to that many),
 * and a failed step also requests a new Jacobian.  Returns 0 on success and
 * 1 when the step size fell below min_dt (the reference throws). */
static int fwd_implicit_euler(const oracle_model* m, const double* P, const oracle_solver_params* sp,
                              node_state* st, double* y, double t, double dt, scratch* w)
{
    int n = m->num_states;
    double *z1 = w->a, *prev = w->c;
    const double t_end = t + dt;
    const double ldt_0 = sp->ldt;
    double ldt = ldt_0 > 0 ? ldt_0 : dt;
    int num_refinements = 0;
    const double eps = GOSS_EPS * 1000;
    for (int i = 0; i < n; ++i)
        prev[i] = 0.0;
    while (1) {
        for (int i = 0; i < n; ++i)
            z1[i] = 0.0;
        if (num_refinements > sp->num_refinements_without_always_recomputing_jacobian)
            st->always_recompute_jacobian = 1;
        int step_ok = newton_solve(m, P, sp, st, z1, prev, y, t + ldt, ldt, 1.0, st->always_recompute_jacobian, w);
        if (step_ok) {
            for (int i = 0; i < n; ++i)
                y[i] += z1[i];
            t += ldt;
            st->accepted++;
            if (fabs(t - t_end) < eps)
                break;
            if (!st->justrefined) {
                const double tmp = 2.0 * ldt;
                if (ldt_0 > 0. && tmp >= ldt_0)
                    ldt = ldt_0;
                else
                    ldt = tmp;
            } else {
                st->justrefined = 0;
            }
            if ((t + ldt + GOSS_EPS) > t_end)
                ldt = t_end - t;
        } else {
            ldt /= 2.0;
            if (ldt < sp->min_dt)
                return 1;
            st->recompute_jacobian = 1;
            st->justrefined = 1;
            num_refinements += 1;
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* ESDIRK23a                                                              */
/* ---------------------------------------------------------------------- */
typedef struct esdirk_coef {
    double gamma, a21, a22, a31, a32, a33, a41, a42, a43, a44, b1, b2, b3, b4, bh1, bh2, bh3, c2, c3, c4;
    double s_fac, tol, etamin, kappa;
} esdirk_coef;

/* coefficients of the ESDIRK23a constructor (ESDIRK23a.cpp:27-39) */
static void esdirk_coefficients(esdirk_coef* c)
{
    double gamma = 0.43586652150845899942;
    c->gamma = gamma;
    c->a21 = gamma;
    c->a22 = gamma;
    c->a31 = (-4 * gamma * gamma + 6 * gamma - 1) / (4 * gamma);
    c->a32 = (-2 * gamma + 1) / (4 * gamma);
    c->a33 = gamma;
    c->a41 = (6 * gamma - 1) / (12 * gamma);
    c->a42 = -1 / ((24 * gamma - 12) * gamma);
    c->a43 = (-6 * gamma * gamma + 6 * gamma - 1) / (6 * gamma - 3);
    c->a44 = gamma;
    c->b1 = c->a41;
    c->b2 = c->a42;
    c->b3 = c->a43;
    c->b4 = c->a44;
    c->bh1 = c->a31;
    c->bh2 = c->a32;
    c->bh3 = c->a33;
    c->c2 = 2.0 * gamma;
    c->c3 = 1.0;
    c->c4 = 1.0;
    c->s_fac = 0.9;
    c->tol = 1.0e-5;
    c->etamin = 1.0e-10;
    c->kappa = 1.0e-1;
}

/* ESDIRK23a::compute_ode_jacobian (ESDIRK23a.h:58-63) */
static void esdirk_ode_jacobian(const oracle_model* m, const double* P, node_state* st, double* y, double t,
                                scratch* w)
{
    oracle_compute_jacobian(m, P, y, t, st->jac, w->k, w->l);
    st->jac_comp++;
    st->new_jacobian = 1;
}

/* ESDIRK23a::compute_factorized_jacobian(dt) (ESDIRK23a.cpp:101-115) */
static void esdirk_factorize(int n, const esdirk_coef* c, node_state* st, double dt)
{
    memcpy(st->jfac, st->jac, sizeof(double) * (size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            st->jfac[i * n + j] *= (-dt * c->a22);
    for (int i = 0; i < n; ++i)
        st->jfac[i * n + i] += 1.0 * 1.0;
    oracle_lu_factorize(n, st->jfac);
}

/* ESDIRK23a::compute_stage_val (ESDIRK23a.cpp:201-258) */
static int esdirk_stage(const oracle_model* m, const double* P, const oracle_solver_params* sp,
                        const esdirk_coef* c, node_state* st, double* z, const double* y, const double* prev,
                        double t_s, double dt, scratch* w)
{
    int n = m->num_states;
    double *y_int = w->f, *z_int = w->g, *b = w->h, *dz = w->i, *prev_dz = w->j;
    int conv_ok = 1;
    double theta;
    st->newton_iterations = 0;
    for (int i = 0; i < n; ++i)
        dz[i] = 0.0, prev_dz[i] = 0.0;
    st->e_eta = pow(std_max(st->e_eta, c->etamin), 0.8);
    do {
        for (int i = 0; i < n; i++)
            y_int[i] = y[i] + dt * prev[i] + c->gamma * dt * z[i];
        m->rhs(y_int, t_s, P, z_int);
        for (int i = 0; i < n; i++)
            b[i] = -z[i] + z_int[i];
        memcpy(prev_dz, dz, sizeof(double) * (size_t)n);
        oracle_forward_backward_subst(n, st->jfac, b, dz);
        if (st->newton_iterations >= 1) {
            theta = l2norm(n, dz) / l2norm(n, prev_dz);
            if (!(theta <= 1)) {
                st->rejects++;
                conv_ok = 0;
                break;
            }
            st->e_eta = theta / (1.0 - theta);
        }
        if (st->newton_iterations > sp->max_iterations) {
            st->rejects++;
            conv_ok = 0;
            break;
        }
        for (int i = 0; i < n; i++)
            z[i] += dz[i];
        st->newton_iterations++;
    } while (st->e_eta * l2norm(n, dz) > c->kappa * c->tol);
    return conv_ok;
}

/* ESDIRK23a::do_step (ESDIRK23a.cpp:134-199) */
static int esdirk_do_step(const oracle_model* m, const double* P, const oracle_solver_params* sp,
                          const esdirk_coef* c, node_state* st, double* y, double t0, double delta_t, scratch* w)
{
    int n = m->num_states;
    double *z1 = w->a, *z2 = w->b, *z3 = w->c, *z4 = w->d, *prev = w->e, *yh = w->l;
    int step_ok;
    m->rhs(y, t0, P, z1);
    for (int i = 0; i < n; i++) {
        z2[i] = z1[i];
        prev[i] = z1[i] * c->a21;
    }
    step_ok = esdirk_stage(m, P, sp, c, st, z2, y, prev, t0 + c->c2 * delta_t, delta_t, w);
    if (step_ok) {
        for (int i = 0; i < n; i++) {
            z3[i] = z2[i];
            prev[i] = z1[i] * c->bh1 + z2[i] * c->bh2;
        }
        step_ok = esdirk_stage(m, P, sp, c, st, z3, y, prev, t0 + c->c3 * delta_t, delta_t, w);
    }
    if (step_ok) {
        for (int i = 0; i < n; i++) {
            z4[i] = z3[i];
            prev[i] = z1[i] * c->b1 + z2[i] * c->b2 + z3[i] * c->b3;
        }
        step_ok = esdirk_stage(m, P, sp, c, st, z4, y, prev, t0 + c->c4 * delta_t, delta_t, w);
    }
    if (step_ok) {
        for (int i = 0; i < n; i++)
            yh[i] = delta_t * ((c->b1 - c->bh1) * z1[i] + (c->b2 - c->bh2) * z2[i] + (c->b3 - c->gamma) * z3[i] +
                               c->gamma * z4[i]);
        oracle_forward_backward_subst(n, st->jfac, yh, yh);
        st->loc_error = l2norm(n, yh);
        if (st->loc_error > c->tol) {
            st->rejects++;
            step_ok = 0;
        } else {
            for (int i = 0; i < n; i++)
                y[i] = y[i] + delta_t * (c->b1 * z1[i] + c->b2 * z2[i] + c->b3 * z3[i] + c->gamma * z4[i]);
            st->accepted++;
        }
    }
    return step_ok;
}

/* ESDIRK23a::reduce_time_step (ESDIRK23a.cpp:260-278) */
static void esdirk_reduce(const esdirk_coef* c, const oracle_solver_params* sp, const node_state* st,
                          double* delta_t)
{
    double reduction_factor = 1.0, e = st->loc_error;
    do {
        reduction_factor *= 0.6;
        e *= 0.1;
    } while (e > c->tol);
    *delta_t = std_max(reduction_factor * (*delta_t), sp->min_dt);
}

/* ESDIRK23a::advance_one_step (ESDIRK23a.cpp:117-132) */
static void esdirk_advance(const oracle_model* m, const double* P, const oracle_solver_params* sp,
                           const esdirk_coef* c, node_state* st, double* y, double t0, double* dt, scratch* w)
{
    int n = m->num_states;
    int accepted = esdirk_do_step(m, P, sp, c, st, y, t0, *dt, w);
    while (!accepted && *dt > sp->min_dt) {
        if (!st->new_jacobian)
            esdirk_ode_jacobian(m, P, st, y, t0, w);
        esdirk_reduce(c, sp, st, dt);
        esdirk_factorize(n, c, st, *dt);
        accepted = esdirk_do_step(m, P, sp, c, st, y, t0, *dt, w);
    }
    st->new_jacobian = 0;
}


/* ESDIRK23a::forward (ESDIRK23a.cpp:280-316) */
static void fwd_esdirk(const oracle_model* m, const double* P, const oracle_solver_params* sp, node_state* st,
                       double* y, double t0, double interval, scratch* w)
{
    int n = m->num_states;
    esdirk_coef c;
    esdirk_coefficients(&c);
    double local_t = 0;
    st->dt = std_max(c.s_fac * st->prev_dt * pow((c.tol / st->loc_error), 0.25), sp->min_dt);
    st->dt = std_min(st->dt, interval);
    if (st->first_step) {
        st->prev_dt = st->dt;
        esdirk_ode_jacobian(m, P, st, y, t0, w);
    }
    while (local_t < interval) {
        if (st->dt * 1.1 >= interval - local_t)
            st->dt = interval - local_t;
        if (st->newton_iterations >= 2)
            esdirk_ode_jacobian(m, P, st, y, t0 + local_t, w);
        if (fabs((st->dt - st->prev_dt) / st->prev_dt) > 0.2 || st->new_jacobian)
            esdirk_factorize(n, &c, st, st->dt);
        esdirk_advance(m, P, sp, &c, st, y, t0 + local_t, &st->dt, w);
        st->prev_dt = st->dt;
        local_t += st->dt;
        st->dt = std_max(c.s_fac * st->prev_dt * pow((c.tol / st->loc_error), 0.25), sp->min_dt);
    }
    st->first_step = 0;
}

/* ---------------------------------------------------------------------- */
/* multi-node driver: ODESystemSolver::forward / _forward_node            */
/* ---------------------------------------------------------------------- */
int oracle_system_forward(oracle_system* s, double t, double interval, int num_threads)
{
    const oracle_model* m = s->m;
    int n = m->num_states, nfp = m->num_field_params, np = m->num_params;
    int failures = 0;
    long N = (long)s->N;
#ifdef _OPENMP
    if (num_threads <= 0)
        num_threads = 1;
#pragma omp parallel num_threads(num_threads) reduction(+ : failures)
#endif
    {
        double* buf = (double*)malloc(sizeof(double) * (size_t)(12 * n + np + 1));
        scratch w;
        w.a = buf;
        w.b = w.a + n;
        w.c = w.b + n;
        w.d = w.c + n;
        w.e = w.d + n;
        w.f = w.e + n;
        w.g = w.f + n;
        w.h = w.g + n;
        w.i = w.h + n;
        w.j = w.i + n;
        w.k = w.j + n;
        w.l = w.k + n;
        double* P = w.l + n;
        memcpy(P, s->params, sizeof(double) * (size_t)np);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (long node = 0; node < N; ++node) {
            /* _forward_node (ODESystemSolver.h:213-236): set field params, then forward */
            for (int k = 0; k < nfp; ++k)
                P[m->field_param_index[k]] = s->fparams[(size_t)node * nfp + k];
            double* y = s->states + (size_t)node * n;
            node_state* st = &s->ns[node];
            switch (s->solver) {
            case ORACLE_EXPLICIT_EULER:
                fwd_euler(m, P, y, t, interval, s->sp.ldt, &w);
                break;
            case ORACLE_RK4:
                fwd_rk4(m, P, y, t, interval, s->sp.ldt, &w);
                break;
            case ORACLE_GRL1:
                fwd_grl1(m, P, y, t, interval, s->sp.ldt, s->sp.delta, &w);
                break;
            case ORACLE_GRL2:
                fwd_grl2(m, P, y, t, interval, s->sp.ldt, s->sp.delta, &w);
                break;
            case ORACLE_THETA:
                failures += fwd_theta(m, P, &s->sp, st, y, t, interval, &w);
                break;
            case ORACLE_ESDIRK23A:
                fwd_esdirk(m, P, &s->sp, st, y, t, interval, &w);
                break;
            case ORACLE_RL1:
                fwd_rl1(m, P, y, t, interval, s->sp.ldt, &w);
                break;
            case ORACLE_RL2:
                fwd_rl2(m, P, y, t, interval, s->sp.ldt, &w);
                break;
            case ORACLE_RK2:
                fwd_rk2(m, P, y, t, interval, s->sp.ldt, &w);
                break;
            case ORACLE_IMPLICIT_EULER:
                failures += fwd_implicit_euler(m, P, &s->sp, st, y, t, interval, &w);
                break;
            default:
                break;
            }
        }
        free(buf);
    }
    return failures;
}
