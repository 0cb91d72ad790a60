// Test infrastructure -- NOT part of the product path.
//
// C entry points around the reference's own compiled solvers
// (goss::ODESystemSolver and the solver classes, built from the reference
// sources into oracle/_ref/libgoss_ref.so by oracle/Makefile), so the tests
// and the CPU baseline of bench.py can run the real reference on the same
// inputs as the CUDA kernels.  Models are goss::ParameterizedODE plugins
// emitted by goss_b200's code generator and loaded with dlopen, exactly like
// the reference loads gotran-generated plugins (python/goss/compilemodule.py:63-82).
//
// Explicit solvers run through one goss::ODESystemSolver over all nodes (the
// reference's OpenMP node loop, ODESystemSolver.cpp:67-79).  Implicit solvers
// carry adaptive state in the solver object, which the reference shares
// between nodes; to give every node its own solver state they run as one
// single-node goss::ODESystemSolver per node.
#include <dlfcn.h>
#include <omp.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "goss/ESDIRK23a.h"
#include "goss/ExplicitEuler.h"
#include "goss/GRL1.h"
#include "goss/GRL2.h"
#include "goss/ImplicitEuler.h"
#include "goss/ODESystemSolver.h"
#include "goss/ParameterizedODE.h"
#include "goss/RK2.h"
#include "goss/RK4.h"
#include "goss/RL1.h"
#include "goss/RL2.h"
#include "goss/ThetaSolver.h"

namespace {

struct RefParams {  // same layout as goss_solver_params in include/goss_b200.h
    double ldt, delta, eta_0, kappa, relative_tolerance, max_relative_previous_residual;
    int32_t max_iterations, always_recompute_jacobian, num_refinements_without_always_recomputing_jacobian;
    double min_dt, theta;
};

std::shared_ptr<goss::ODESolver> make_solver(int kind, const RefParams& p)
{
    std::shared_ptr<goss::ODESolver> s;
    switch (kind) {
    case 0:
        s = std::make_shared<goss::ExplicitEuler>();
        break;
    case 1:
        s = std::make_shared<goss::RK4>();
        break;
    case 2: {
        auto g = std::make_shared<goss::GRL1>();
        g->delta = p.delta;
        s = g;
        break;
    }
    case 3: {
        auto g = std::make_shared<goss::GRL2>();
        g->delta = p.delta;
        s = g;
        break;
    }
    case 4: {
        auto th = std::make_shared<goss::ThetaSolver>();
        th->eta_0 = p.eta_0;
        th->kappa = p.kappa;
        th->relative_tolerance = p.relative_tolerance;
        th->max_iterations = p.max_iterations;
        th->max_relative_previous_residual = p.max_relative_previous_residual;
        th->always_recompute_jacobian = p.always_recompute_jacobian != 0;
        th->num_refinements_without_always_recomputing_jacobian =
            p.num_refinements_without_always_recomputing_jacobian;
        th->min_dt = p.min_dt;
        th->theta = p.theta;
        s = th;
        break;
    }
    case 5: {
        auto es = std::make_shared<goss::ESDIRK23a>();
        // ESDIRK23a's own kappa (ESDIRK23a.h:109) is private and fixed at 0.1
        es->eta_0 = p.eta_0;
        es->relative_tolerance = p.relative_tolerance;
        es->max_iterations = p.max_iterations;
        es->max_relative_previous_residual = p.max_relative_previous_residual;
        es->always_recompute_jacobian = p.always_recompute_jacobian != 0;
        es->num_refinements_without_always_recomputing_jacobian =
            p.num_refinements_without_always_recomputing_jacobian;
        es->min_dt = p.min_dt;
        s = es;
        break;
    }
    case 6:
        s = std::make_shared<goss::RL1>();
        break;
    case 7:
        s = std::make_shared<goss::RL2>();
        break;
    case 8:
        s = std::make_shared<goss::RK2>();
        break;
    case 9: {
        auto ie = std::make_shared<goss::ImplicitEuler>();
        ie->eta_0 = p.eta_0;
        ie->kappa = p.kappa;
        ie->relative_tolerance = p.relative_tolerance;
        ie->max_iterations = p.max_iterations;
        ie->max_relative_previous_residual = p.max_relative_previous_residual;
        ie->always_recompute_jacobian = p.always_recompute_jacobian != 0;
        ie->num_refinements_without_always_recomputing_jacobian =
            p.num_refinements_without_always_recomputing_jacobian;
        ie->min_dt = p.min_dt;
        s = ie;
        break;
    }
    default:
        return nullptr;
    }
    s->set_internal_time_step(p.ldt);
    return s;
}

struct RefSystem {
    void* plugin = nullptr;
    int kind = 0;
    RefParams params{};
    uint32_t N = 0, n = 0, nfp = 0;
    std::shared_ptr<goss::ParameterizedODE> ode;
    // explicit: one system over all nodes
    std::shared_ptr<goss::ODESystemSolver> system;
    // implicit: one single-node system per node
    std::vector<std::shared_ptr<goss::ODESystemSolver>> nodes;
    std::string error;
    uint32_t threads = 0;
};

bool implicit(int kind) { return kind == 4 || kind == 5 || kind == 9; }

}  // namespace

extern "C" {

__attribute__((visibility("default"))) void* ref_create(const char* plugin_path, const char* class_name, int kind,
                                                        const RefParams* params, uint32_t N)
{
    void* lib = dlopen(plugin_path, RTLD_NOW | RTLD_LOCAL);
    if (!lib)
        return nullptr;
    std::string fn = std::string("create_") + class_name;
    auto create = reinterpret_cast<goss::ParameterizedODE* (*)()>(dlsym(lib, fn.c_str()));
    if (!create)
        return nullptr;
    auto* r = new RefSystem();
    r->plugin = lib;
    r->kind = kind;
    r->params = *params;
    r->N = N;
    r->ode.reset(create());
    r->n = r->ode->num_states();
    r->nfp = r->ode->num_field_parameters();
    if (!implicit(kind)) {
        r->system = std::make_shared<goss::ODESystemSolver>(N, make_solver(kind, *params), r->ode);
    } else {
        r->nodes.resize(N);
        for (uint32_t i = 0; i < N; ++i) {
            auto ode = std::dynamic_pointer_cast<goss::ParameterizedODE>(r->ode->copy());
            r->nodes[i] = std::make_shared<goss::ODESystemSolver>(1, make_solver(kind, *params), ode);
        }
    }
    return r;
}

__attribute__((visibility("default"))) void ref_destroy(void* h)
{
    auto* r = static_cast<RefSystem*>(h);
    if (!r)
        return;
    r->system.reset();
    r->nodes.clear();
    r->ode.reset();
    // the plugin stays loaded: destructors of objects it created have run
    delete r;
}

__attribute__((visibility("default"))) int ref_num_states(void* h) { return (int)static_cast<RefSystem*>(h)->n; }

__attribute__((visibility("default"))) int ref_set_parameter(void* h, const char* name, double value)
{
    auto* r = static_cast<RefSystem*>(h);
    try {
        if (r->system) {
            r->system->ode()->set_parameter(name, value);
        } else {
            for (auto& s : r->nodes)
                s->ode()->set_parameter(name, value);
        }
        r->ode->set_parameter(name, value);
    } catch (const std::exception& e) {
        r->error = e.what();
        return 1;
    }
    return 0;
}

// states: [N][n] node-major
__attribute__((visibility("default"))) void ref_set_states(void* h, const double* states)
{
    auto* r = static_cast<RefSystem*>(h);
    if (r->system) {
        std::memcpy(r->system->states(), states, sizeof(double) * r->N * r->n);
    } else {
        for (uint32_t i = 0; i < r->N; ++i)
            std::memcpy(r->nodes[i]->states(), states + (size_t)i * r->n, sizeof(double) * r->n);
    }
}

__attribute__((visibility("default"))) void ref_get_states(void* h, double* states)
{
    auto* r = static_cast<RefSystem*>(h);
    if (r->system) {
        std::memcpy(states, r->system->states(), sizeof(double) * r->N * r->n);
    } else {
        for (uint32_t i = 0; i < r->N; ++i)
            std::memcpy(states + (size_t)i * r->n, r->nodes[i]->states(), sizeof(double) * r->n);
    }
}

// field parameters: [N][nfp] node-major
__attribute__((visibility("default"))) void ref_set_field_parameters(void* h, const double* fp)
{
    auto* r = static_cast<RefSystem*>(h);
    if (!r->nfp)
        return;
    if (r->system) {
        r->system->set_field_parameters(fp, true);
    } else {
        for (uint32_t i = 0; i < r->N; ++i)
            r->nodes[i]->set_field_parameters(fp + (size_t)i * r->nfp, true);
    }
}

// ODESystemSolver::set_num_threads (ODESystemSolver.cpp:218-250)
__attribute__((visibility("default"))) void ref_set_num_threads(void* h, uint32_t threads)
{
    auto* r = static_cast<RefSystem*>(h);
    r->threads = threads;
    if (r->system && threads > 0)
        r->system->set_num_threads(threads);
}

__attribute__((visibility("default"))) int ref_forward(void* h, double t, double interval)
{
    auto* r = static_cast<RefSystem*>(h);
    int failures = 0;
    if (r->system) {
        try {
            r->system->forward(t, interval);
        } catch (const std::exception& e) {
            r->error = e.what();
            return 1;
        }
        return 0;
    }
    const int threads = r->threads > 0 ? (int)r->threads : 1;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 16) reduction(+ : failures)
    for (long i = 0; i < (long)r->N; ++i) {
        try {
            r->nodes[i]->forward(t, interval);
        } catch (const std::exception&) {
            failures += 1;
        }
    }
    if (failures)
        r->error = "Newtons solver failed to converge as dt become smaller than 'min_dt'";
    return failures;
}

// ODESystemSolver::solve (ODESystemSolver.cpp:81-99) of an explicit solver
// over all nodes: field states of the plugin model at the times t[1..nt-1]
// ([nt][N][nfs] tangled, [nt][nfs][N] untangled; row 0 is not written).
__attribute__((visibility("default"))) int ref_solve(void* h, double* field_states, double* t, uint64_t nt,
                                                    int tangled)
{
    auto* r = static_cast<RefSystem*>(h);
    if (!r->system)
        return 1;
    try {
        r->system->solve(field_states, t, nt, tangled != 0);
    } catch (const std::exception& e) {
        r->error = e.what();
        return 1;
    }
    return 0;
}

__attribute__((visibility("default"))) uint32_t ref_num_field_states(void* h)
{
    return static_cast<RefSystem*>(h)->ode->num_field_states();
}

__attribute__((visibility("default"))) const char* ref_last_error(void* h)
{
    return static_cast<RefSystem*>(h)->error.c_str();
}

__attribute__((visibility("default"))) int ref_num_jac_comp(void* h, int64_t* out)
{
    auto* r = static_cast<RefSystem*>(h);
    if (!implicit(r->kind))
        return 1;
    for (uint32_t i = 0; i < r->N; ++i) {
        auto s = std::dynamic_pointer_cast<goss::ImplicitODESolver>(r->nodes[i]->solver());
        out[i] = s ? s->num_jac_comp() : -1;
    }
    return 0;
}

// AdaptiveImplicitSolver::get_num_rejected (AdaptiveImplicitSolver.h:63-66)
// of every node's ESDIRK23a solver (the other solvers have no such counter).
__attribute__((visibility("default"))) int ref_num_rejected(void* h, int64_t* out)
{
    auto* r = static_cast<RefSystem*>(h);
    if (r->kind != 5)
        return 1;
    for (uint32_t i = 0; i < r->N; ++i) {
        auto s = std::dynamic_pointer_cast<goss::AdaptiveImplicitSolver>(r->nodes[i]->solver());
        out[i] = s ? s->get_num_rejected() : -1;
    }
    return 0;
}

// ODE::compute_jacobian (ODE.h:71) of the plugin model with its default
// parameters: the generated analytic override when the plugin has one, else
// the reference's forward differences (ODE.cpp:47-67); jac is row-major n x n.
__attribute__((visibility("default"))) void ref_compute_jacobian(void* h, double* states, double time, double* jac)
{
    auto* r = static_cast<RefSystem*>(h);
    auto ode = std::dynamic_pointer_cast<goss::ParameterizedODE>(r->ode->copy());
    ode->compute_jacobian(states, time, jac);
}

// ODE::lu_factorize (ODE.cpp:69-100) and ODE::forward_backward_subst
// (ODE.cpp:102-132) of the plugin model, in place on a row-major n x n matrix.
__attribute__((visibility("default"))) void ref_lu_factorize(void* h, double* mat)
{
    static_cast<RefSystem*>(h)->ode->lu_factorize(mat);
}

__attribute__((visibility("default"))) void ref_forward_backward_subst(void* h, const double* mat, const double* b,
                                                                      double* x)
{
    static_cast<RefSystem*>(h)->ode->forward_backward_subst(mat, b, x);
}

}  // extern "C"
