// Generated by goss_b200.codegen from the 'oscilator' model; do not edit.
// goss::ParameterizedODE plugin consumed by the oracle build of the reference solvers.
#ifndef OSCILATOR_GOSS_PLUGIN_H
#define OSCILATOR_GOSS_PLUGIN_H
#include <cmath>
#include <memory>
#include <stdexcept>
#include "goss/ParameterizedODE.h"

namespace goss {
class Oscilator : public ParameterizedODE
{
  public:
    Oscilator() : ParameterizedODE(2, 2, 0, 2, 0), a(1.0), b(1.0)
    {
        _state_names[0] = "x";
        _state_names[1] = "y";
        _parameter_names[0] = "a";
        _parameter_names[1] = "b";
        _field_parameter_names[0] = "a";
        _field_parameter_names[1] = "b";
        _param_to_value["a"] = &a;
        _param_to_value["b"] = &b;
    }
    Oscilator(const Oscilator& ode) : ParameterizedODE(ode), a(ode.a), b(ode.b) {}

    void eval(const double* states, double time, double* values)
    {
        const double x = states[0];
        const double y = states[1];
        values[0] = (-(a*y));
        values[1] = (b*x);
    }

    void linearized_eval(const double* states, double time, double* linear, double* rhs,
                         bool only_linear) const
    {
        const double x = states[0];
        const double y = states[1];
        rhs[0] = (-(a*y));
        rhs[1] = (b*x);
        if (only_linear) return;
        linear[0] = 0.0;
        linear[1] = 0.0;
    }

    void get_ic(goss::DoubleVector* values) const
    {
        values->n = _num_states;
        values->data.reset(new double[_num_states]);
        values->data[0] = 1.0;
        values->data[1] = 0.0;
    }

    std::shared_ptr<ODE> copy() const { return std::make_shared<Oscilator>(*this); }

    void eval_monitored(const double* states, double time, double* monitored) const
    {
        throw std::runtime_error("No monitored in the \'Oscilator\' model.");
    }

    void set_field_parameters(const double* field_params)
    {
        a = field_params[0];
        b = field_params[1];
    }

  private:
    double a, b;
};
}  // namespace goss

extern "C" __attribute__((visibility("default"))) goss::ParameterizedODE* create_Oscilator()
{
    return new goss::Oscilator;
}
#endif
