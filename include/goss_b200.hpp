/*
 * goss_b200.hpp -- header-only C++ drop-in over the C ABI of goss_b200.h.
 *
 * C++ callers of goss's multi-node solve path keep their code: the classes
 * below carry the signatures of the reference's
 *   goss::ODESystemSolver          (cpp/goss/ODESystemSolver.h:43-124)
 *   goss::ParameterizedODE          (cpp/goss/ParameterizedODE.h:60-160, ODE.h:43-92)
 *   goss::ExplicitEuler, RK2, RK4, RL1, RL2, GRL1, GRL2, ThetaSolver,
 *   ImplicitEuler, ESDIRK23a       (their public parameter members,
 *                                   ODESolver.h:36-153, GRL1.h:39,
 *                                   ImplicitODESolver.h:36-41, ThetaSolver.h:35-37,
 *                                   ImplicitEuler.h:35-36, ESDIRK23a.h:37-38)
 * in namespace goss_b200, so switching is a change of namespace (or a
 * `namespace goss = goss_b200;`) and of how the model is loaded: a model is a
 * compiled goss_b200 model library (libgoss_model.so from the project's code
 * generator) instead of a gotran plugin with create_<Name>().
 *
 * Semantics follow the reference: calls are synchronous, host arrays are
 * borrowed for the duration of a call, errors throw std::runtime_error with
 * the reference's text (a goss_b200::Error carrying the status code).
 * Solver members are read at every forward/solve, as the reference reads its
 * shared solver object.  States live on the GPU; states() returns a host
 * copy refreshed by each call of states() (writes to it reach the device
 * only through set_states()).
 *
 * Link with -lgoss_b200 (goss_b200/_lib) and -ldl.
 */
#ifndef GOSS_B200_HPP
#define GOSS_B200_HPP

#include <dlfcn.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "goss_b200.h"

namespace goss_b200 {

typedef unsigned int uint;
typedef unsigned long ulong;

class Error : public std::runtime_error {
  public:
    Error(int status, const std::string& what) : std::runtime_error(what), _status(status) {}
    int status() const { return _status; }

  private:
    int _status;
};

namespace detail {
inline void check(int rc, const char* msg)
{
    if (rc != GOSS_OK)
        throw Error(rc, msg && *msg ? msg : "goss_b200 call failed");
}
inline goss_solver_params defaults(int32_t kind)
{
    goss_solver_params p;
    check(goss_solver_default_params(kind, &p), goss_last_error());
    return p;
}
}  // namespace detail

// ---------------------------------------------------------------------------
// ParameterizedODE: one compiled model variant (goss_model_desc) plus the
// uniform parameter values and the choice of field states.
// ---------------------------------------------------------------------------
class ParameterizedODE {
  public:
    // A model whose library is linked into the program (its factory called).
    explicit ParameterizedODE(const goss_model_desc* desc) : _desc(desc)
    {
        if (!desc || desc->abi_version != GOSS_B200_ABI_VERSION)
            throw Error(GOSS_ERR_ARGUMENT, "model descriptor missing or built for another ABI version");
        for (uint i = 0; i < desc->num_states; ++i)
            _state_names.push_back(desc->state_names[i]);
        for (uint i = 0; i < desc->num_parameters; ++i) {
            _parameter_names.push_back(desc->parameter_names[i]);
            _params.push_back(desc->default_parameters[i]);
        }
        for (uint i = 0; i < desc->num_field_parameters; ++i)
            _field_parameter_names.push_back(desc->field_parameter_names[i]);
    }

    // A model library loaded at run time: `library` is a libgoss_model.so and
    // `variant` its variant name (the factory goss_b200_model_<variant>); the
    // counterpart of loading a gotran plugin and calling create_<Name>().
    static std::shared_ptr<ParameterizedODE> load(const std::string& library, const std::string& variant)
    {
        void* h = dlopen(library.c_str(), RTLD_NOW | RTLD_LOCAL);
        if (!h)
            throw Error(GOSS_ERR_ARGUMENT, std::string("cannot load model library: ") + dlerror());
        const std::string sym = "goss_b200_model_" + variant;
        typedef const goss_model_desc* (*factory)(void);
        factory f = reinterpret_cast<factory>(dlsym(h, sym.c_str()));
        if (!f)
            throw Error(GOSS_ERR_ARGUMENT, "model library has no " + sym);
        auto ode = std::make_shared<ParameterizedODE>(f());
        ode->_library = std::shared_ptr<void>(h, [](void* p) { dlclose(p); });
        return ode;
    }

    uint num_states() const { return _desc->num_states; }
    uint num_parameters() const { return _desc->num_parameters; }
    uint num_field_parameters() const { return _desc->num_field_parameters; }
    uint num_monitored() const { return _desc->num_monitored; }
    uint num_field_states() const { return (uint)_field_state_indices.size(); }
    bool has_jacobian() const { return _desc->has_jacobian != 0; }
    unsigned char linear_term(uint i) const { return _desc->linear_terms[i]; }

    const std::vector<std::string>& get_state_names() const { return _state_names; }
    const std::vector<std::string>& get_parameter_names() const { return _parameter_names; }
    const std::vector<std::string>& get_field_parameter_names() const { return _field_parameter_names; }
    const std::vector<std::string>& get_field_state_names() const { return _field_state_names; }
    const std::vector<uint>& get_field_state_indices() const { return _field_state_indices; }

    // The reference fixes the field states when the plugin is generated
    // (gotran's field_states); here they are chosen on the compiled model.
    void set_field_states(const std::vector<std::string>& names)
    {
        std::vector<uint> idx;
        for (const auto& nm : names)
            idx.push_back(state_index(nm));
        _field_state_indices = idx;
        _field_state_names = names;
    }

    // ParameterizedODE::set_parameter / get_parameter (ParameterizedODE.h:111-121)
    void set_parameter(std::string name, double value) { _params[parameter_index(name)] = value; }
    double get_parameter(std::string name) const { return _params[parameter_index(name)]; }

    void get_ic(double* values) const
    {
        for (uint i = 0; i < num_states(); ++i)
            values[i] = _desc->initial_conditions[i];
    }

    // ODE::eval / linearized_eval / compute_jacobian (ODE.h:55-71) of one state
    // vector, evaluated on the GPU with the current parameter values; field
    // parameters at their current uniform values.
    void eval(const double* states, double time, double* values) const { evaluate(0, states, time, values); }
    void linearized_eval(const double* states, double time, double* linearized, double* rhs,
                         bool only_linear = false) const
    {
        std::vector<double> out(2 * num_states());
        evaluate(1, states, time, out.data());
        for (uint i = 0; i < num_states(); ++i) {
            linearized[i] = out[i];
            if (!only_linear)
                rhs[i] = out[num_states() + i];
        }
    }
    void eval_monitored(const double* states, double time, double* monitored) const
    {
        evaluate(2, states, time, monitored);
    }
    // analytic Jacobian of a model generated with code_params generate_jacobian
    void compute_jacobian(double* states, double time, double* jac) const { evaluate(3, states, time, jac); }
    void lu_factorize(double* mat) const { detail::check(goss_lu_factorize(num_states(), mat), goss_last_error()); }
    void forward_backward_subst(const double* mat, const double* b, double* x) const
    {
        detail::check(goss_forward_backward_subst(num_states(), mat, b, x), goss_last_error());
    }

    const goss_model_desc* desc() const { return _desc; }
    const std::vector<double>& parameter_values() const { return _params; }

  private:
    uint state_index(const std::string& name) const
    {
        for (uint i = 0; i < _state_names.size(); ++i)
            if (_state_names[i] == name)
                return i;
        throw Error(GOSS_ERR_ARGUMENT, "'" + name + "' is not a state in the " + _desc->name + " ODE");
    }
    uint parameter_index(const std::string& name) const
    {
        for (uint i = 0; i < _parameter_names.size(); ++i)
            if (_parameter_names[i] == name)
                return i;
        // the reference's message (ParameterizedODE.h:190-192)
        throw Error(GOSS_ERR_ARGUMENT, "'" + name + "' is not a parameter in the " + _desc->name + " ODE");
    }
    void evaluate(int what, const double* states, double time, double* out) const
    {
        std::vector<double> fp(num_field_parameters());
        for (uint k = 0; k < fp.size(); ++k)
            fp[k] = _params[_desc->field_parameter_indices[k]];
        detail::check(goss_model_eval(_desc, what, GOSS_FP64, _params.data(), states, fp.empty() ? nullptr : fp.data(),
                                      &time, 1, out, 0),
                      goss_last_error());
    }

    const goss_model_desc* _desc;
    std::shared_ptr<void> _library;
    std::vector<std::string> _state_names, _parameter_names, _field_parameter_names, _field_state_names;
    std::vector<uint> _field_state_indices;
    std::vector<double> _params;
};

// ---------------------------------------------------------------------------
// Solvers: the reference's classes with their public parameter members
// (defaults from goss_solver_default_params, i.e. the reference's).
// ---------------------------------------------------------------------------
class ODESolver {
  public:
    virtual ~ODESolver() {}
    virtual int32_t kind() const = 0;
    virtual bool is_adaptive() const { return false; }
    virtual void attach(std::shared_ptr<ParameterizedODE> ode) { _ode = ode; }
    std::shared_ptr<ParameterizedODE> get_ode() { return _ode; }
    uint num_states() const { return _ode ? _ode->num_states() : 0; }
    double get_internal_time_step() const { return _ldt; }
    void set_internal_time_step(double ldt) { _ldt = ldt; }
    // the members as the C ABI's parameter block
    virtual goss_solver_params params() const
    {
        goss_solver_params p = detail::defaults(kind());
        p.ldt = _ldt;
        return p;
    }

  protected:
    double _ldt = -1.0;  // ODESolver.h:137
    std::shared_ptr<ParameterizedODE> _ode;
};

#define GOSS_B200_PLAIN_SOLVER(Name, Kind)                                        \
    class Name : public ODESolver {                                               \
      public:                                                                     \
        Name() {}                                                                 \
        explicit Name(std::shared_ptr<ParameterizedODE> ode) { attach(ode); }     \
        int32_t kind() const override { return Kind; }                            \
    };
GOSS_B200_PLAIN_SOLVER(ExplicitEuler, GOSS_EXPLICIT_EULER)
GOSS_B200_PLAIN_SOLVER(RK2, GOSS_RK2)
GOSS_B200_PLAIN_SOLVER(RK4, GOSS_RK4)
GOSS_B200_PLAIN_SOLVER(RL1, GOSS_RL1)
GOSS_B200_PLAIN_SOLVER(RL2, GOSS_RL2)
GOSS_B200_PLAIN_SOLVER(GRL2, GOSS_GRL2)
#undef GOSS_B200_PLAIN_SOLVER

class GRL1 : public ODESolver {
  public:
    GRL1() : delta(detail::defaults(GOSS_GRL1).delta) {}
    explicit GRL1(std::shared_ptr<ParameterizedODE> ode) : GRL1() { attach(ode); }
    int32_t kind() const override { return GOSS_GRL1; }
    goss_solver_params params() const override
    {
        goss_solver_params p = ODESolver::params();
        p.delta = delta;
        return p;
    }
    double delta;  // GRL1.h:39
};

class ImplicitODESolver : public ODESolver {
  public:
    goss_solver_params params() const override
    {
        goss_solver_params p = ODESolver::params();
        p.eta_0 = eta_0;
        p.kappa = kappa;
        p.relative_tolerance = relative_tolerance;
        p.max_iterations = max_iterations;
        p.max_relative_previous_residual = max_relative_previous_residual;
        p.always_recompute_jacobian = always_recompute_jacobian ? 1 : 0;
        p.num_refinements_without_always_recomputing_jacobian = num_refinements_without_always_recomputing_jacobian;
        p.min_dt = min_dt;
        p.theta = _theta;
        return p;
    }
    // ImplicitODESolver.h:36-41
    double eta_0, kappa, relative_tolerance;
    int max_iterations;
    double max_relative_previous_residual;
    bool always_recompute_jacobian;
    // ThetaSolver.h:35-36, ImplicitEuler.h:35-36, ESDIRK23a.h:37-38
    int num_refinements_without_always_recomputing_jacobian;
    double min_dt;

  protected:
    explicit ImplicitODESolver(int32_t k)
    {
        const goss_solver_params p = detail::defaults(k);
        eta_0 = p.eta_0;
        kappa = p.kappa;
        relative_tolerance = p.relative_tolerance;
        max_iterations = p.max_iterations;
        max_relative_previous_residual = p.max_relative_previous_residual;
        always_recompute_jacobian = p.always_recompute_jacobian != 0;
        num_refinements_without_always_recomputing_jacobian = p.num_refinements_without_always_recomputing_jacobian;
        min_dt = p.min_dt;
        _theta = p.theta;
    }
    double _theta;
};

class ThetaSolver : public ImplicitODESolver {
  public:
    ThetaSolver() : ImplicitODESolver(GOSS_THETA), theta(_theta) {}
    explicit ThetaSolver(std::shared_ptr<ParameterizedODE> ode) : ThetaSolver() { attach(ode); }
    int32_t kind() const override { return GOSS_THETA; }
    goss_solver_params params() const override
    {
        goss_solver_params p = ImplicitODESolver::params();
        p.theta = theta;
        return p;
    }
    double theta;  // ThetaSolver.h:37
};

class ImplicitEuler : public ImplicitODESolver {
  public:
    ImplicitEuler() : ImplicitODESolver(GOSS_IMPLICIT_EULER) {}
    explicit ImplicitEuler(std::shared_ptr<ParameterizedODE> ode) : ImplicitEuler() { attach(ode); }
    int32_t kind() const override { return GOSS_IMPLICIT_EULER; }
};

class ESDIRK23a : public ImplicitODESolver {
  public:
    ESDIRK23a() : ImplicitODESolver(GOSS_ESDIRK23A) {}
    explicit ESDIRK23a(std::shared_ptr<ParameterizedODE> ode) : ESDIRK23a() { attach(ode); }
    int32_t kind() const override { return GOSS_ESDIRK23A; }
    bool is_adaptive() const override { return true; }
};

// ---------------------------------------------------------------------------
// ODESystemSolver (ODESystemSolver.h:43-124)
// ---------------------------------------------------------------------------
class ODESystemSolver {
  public:
    ODESystemSolver(uint nodes, std::shared_ptr<ODESolver> solver, std::shared_ptr<ParameterizedODE> ode,
                    int32_t precision = GOSS_FP64, int32_t device = 0)
        : _solver(solver), _ode(ode), _num_nodes(nodes)
    {
        if (!solver || !ode)
            throw Error(GOSS_ERR_ARGUMENT, "ODESystemSolver needs a solver and an ODE");
        solver->attach(ode);  // ODESystemSolver.cpp:55
        const goss_solver_params p = solver->params();
        goss_system* h = nullptr;
        detail::check(goss_system_create(ode->desc(), solver->kind(), &p, nodes, precision, device, &h),
                      goss_last_error());
        _h = std::shared_ptr<goss_system>(h, [](goss_system* s) { goss_system_destroy(s); });
        const auto& fsi = ode->get_field_state_indices();
        check(goss_system_set_field_state_indices(_h.get(), fsi.empty() ? nullptr : fsi.data(), (uint32_t)fsi.size()));
        sync();
    }

    // Step all nodes an interval of time forward (ODESystemSolver.cpp:67-79)
    void forward(double t, double interval)
    {
        sync();
        check(goss_system_forward(_h.get(), t, interval));
    }

    // Step all nodes through the times t[1..num_timesteps-1], storing the field
    // states after each (ODESystemSolver.cpp:81-99)
    void solve(double* field_states, double* t, const ulong num_timesteps, bool tangled_storage = true)
    {
        sync();
        check(goss_system_solve(_h.get(), field_states, t, num_timesteps, tangled_storage ? 1 : 0));
    }

    void get_field_state_components(double* component_field_states, uint num_components, const uint* components,
                                    bool tangled_storage = true) const
    {
        check(goss_system_get_field_state_components(_h.get(), component_field_states, num_components, components,
                                                     tangled_storage ? 1 : 0));
    }
    void set_field_state_components(const double* component_field_states, uint num_components, const uint* components,
                                    bool tangled_storage = true)
    {
        check(goss_system_set_field_state_components(_h.get(), component_field_states, num_components, components,
                                                     tangled_storage ? 1 : 0));
    }
    void get_field_states(double* system_field_states, bool tangled_storage = true) const
    {
        check(goss_system_get_field_states(_h.get(), system_field_states, tangled_storage ? 1 : 0));
    }
    void set_field_states(const double* system_field_states, bool tangled_storage = true)
    {
        check(goss_system_set_field_states(_h.get(), system_field_states, tangled_storage ? 1 : 0));
    }
    void get_field_parameters(double* system_field_params, bool tangled_storage = true) const
    {
        check(goss_system_get_field_parameters(_h.get(), system_field_params, tangled_storage ? 1 : 0));
    }
    void set_field_parameters(const double* system_field_params, bool tangled_storage = true)
    {
        check(goss_system_set_field_parameters(_h.get(), system_field_params, tangled_storage ? 1 : 0));
    }

    // Initial conditions and default field parameters (ODESystemSolver.cpp:192-216)
    void reset_default() { check(goss_system_reset_default(_h.get())); }

    void set_num_threads(uint num_threads) { check(goss_system_set_num_threads(_h.get(), num_threads)); }
    uint get_num_threads() const { return goss_system_get_num_threads(_h.get()); }

    // All states, node-major [num_nodes][num_states]: a host copy refreshed by
    // every call (the device holds the states; write through set_states)
    const double* states() const
    {
        _host.resize((size_t)_num_nodes * _ode->num_states());
        check(goss_system_get_states(_h.get(), _host.data()));
        return _host.data();
    }
    const double* states(uint node) const { return states() + (size_t)node * _ode->num_states(); }
    void set_states(const double* states) { check(goss_system_set_states(_h.get(), states)); }

    std::shared_ptr<ParameterizedODE> ode() { return _ode; }
    std::shared_ptr<ODESolver> solver() { return _solver; }
    uint num_nodes() { return _num_nodes; }
    goss_system* handle() { return _h.get(); }

  private:
    void check(int rc) const { detail::check(rc, goss_system_last_error(_h.get())); }
    // the reference reads the shared solver and ODE objects at every step
    void sync()
    {
        const goss_solver_params p = _solver->params();
        check(goss_system_set_solver_params(_h.get(), &p));
        const auto& v = _ode->parameter_values();
        for (uint i = 0; i < v.size(); ++i)
            check(goss_system_set_parameter(_h.get(), i, v[i]));
    }

    std::shared_ptr<ODESolver> _solver;
    std::shared_ptr<ParameterizedODE> _ode;
    std::shared_ptr<goss_system> _h;
    uint _num_nodes;
    mutable std::vector<double> _host;
};

}  // namespace goss_b200
#endif
