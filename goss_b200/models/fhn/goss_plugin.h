// Generated by goss_b200.codegen from the 'fhn' model; do not edit.
// goss::ParameterizedODE plugin consumed by the oracle build of the reference solvers.
#ifndef FHN_GOSS_PLUGIN_H
#define FHN_GOSS_PLUGIN_H
#include <cmath>
#include <memory>
#include <stdexcept>
#include "goss/ParameterizedODE.h"

namespace goss {
class Fhn : public ParameterizedODE
{
  public:
    Fhn() : ParameterizedODE(2, 11, 0, 0, 0), a(0.13), b(0.013), c_1(0.26), c_2(0.1), c_3(1.0), stim_amplitude(50.0), stim_duration(1.0), stim_period(1000.0), stim_start(1.0), v_peak(40.0), v_rest(-85.0)
    {
        _state_names[0] = "v";
        _state_names[1] = "s";
        _parameter_names[0] = "a";
        _parameter_names[1] = "b";
        _parameter_names[2] = "c_1";
        _parameter_names[3] = "c_2";
        _parameter_names[4] = "c_3";
        _parameter_names[5] = "stim_amplitude";
        _parameter_names[6] = "stim_duration";
        _parameter_names[7] = "stim_period";
        _parameter_names[8] = "stim_start";
        _parameter_names[9] = "v_peak";
        _parameter_names[10] = "v_rest";
        _param_to_value["a"] = &a;
        _param_to_value["b"] = &b;
        _param_to_value["c_1"] = &c_1;
        _param_to_value["c_2"] = &c_2;
        _param_to_value["c_3"] = &c_3;
        _param_to_value["stim_amplitude"] = &stim_amplitude;
        _param_to_value["stim_duration"] = &stim_duration;
        _param_to_value["stim_period"] = &stim_period;
        _param_to_value["stim_start"] = &stim_start;
        _param_to_value["v_peak"] = &v_peak;
        _param_to_value["v_rest"] = &v_rest;
        _linear_terms[1] = 1;
    }
    Fhn(const Fhn& ode) : ParameterizedODE(ode), a(ode.a), b(ode.b), c_1(ode.c_1), c_2(ode.c_2), c_3(ode.c_3), stim_amplitude(ode.stim_amplitude), stim_duration(ode.stim_duration), stim_period(ode.stim_period), stim_start(ode.stim_start), v_peak(ode.v_peak), v_rest(ode.v_rest) {}

    void eval(const double* states, double time, double* values)
    {
        const double v = states[0];
        const double s = states[1];
        const double v_amp = (v_peak - ((v_rest)));
        const double v_th = (v_rest + (a*v_amp));
        const double I = ((-(c_2*s*(v - ((v_rest)))/v_amp)) + (c_1*(v - ((v_rest)))*(v - ((v_th)))*(v_peak - ((v)))/(v_amp*v_amp)));
        const double i_Stim = (stim_amplitude*(1.0 - ((1.0/(1.0 + std::exp(((5.0*time) - ((5.0*stim_start))))))))/(1.0 + std::exp(((5.0*time) - ((5.0*stim_duration)) - ((5.0*stim_start))))));
        values[0] = (I + i_Stim);
        values[1] = (b*(v - ((v_rest)) - ((c_3*s))));
    }

    void linearized_eval(const double* states, double time, double* linear, double* rhs,
                         bool only_linear) const
    {
        const double v = states[0];
        const double s = states[1];
        const double v_amp = (v_peak - ((v_rest)));
        const double v_th = (v_rest + (a*v_amp));
        const double I = ((-(c_2*s*(v - ((v_rest)))/v_amp)) + (c_1*(v - ((v_rest)))*(v - ((v_th)))*(v_peak - ((v)))/(v_amp*v_amp)));
        const double i_Stim = (stim_amplitude*(1.0 - ((1.0/(1.0 + std::exp(((5.0*time) - ((5.0*stim_start))))))))/(1.0 + std::exp(((5.0*time) - ((5.0*stim_duration)) - ((5.0*stim_start))))));
        rhs[0] = (I + i_Stim);
        rhs[1] = (b*(v - ((v_rest)) - ((c_3*s))));
        linear[1] = (-(b*c_3));
        if (only_linear) return;
        const double dI_dv = ((-(c_2*s/v_amp)) + (c_1*(v - ((v_rest)))*(v_peak - ((v)))/(v_amp*v_amp)) + (c_1*(v - ((v_th)))*(v_peak - ((v)))/(v_amp*v_amp)) - ((c_1*(v - ((v_rest)))*(v - ((v_th)))/(v_amp*v_amp))));
        linear[0] = dI_dv;
    }

    void get_ic(goss::DoubleVector* values) const
    {
        values->n = _num_states;
        values->data.reset(new double[_num_states]);
        values->data[0] = -85.0;
        values->data[1] = 0.0;
    }

    std::shared_ptr<ODE> copy() const { return std::make_shared<Fhn>(*this); }

    void eval_monitored(const double* states, double time, double* monitored) const
    {
        throw std::runtime_error("No monitored in the \'Fhn\' model.");
    }

    void set_field_parameters(const double* field_params)
    {
        (void)field_params;
    }

  private:
    double a, b, c_1, c_2, c_3, stim_amplitude, stim_duration, stim_period, stim_start, v_peak, v_rest;
};
}  // namespace goss

extern "C" __attribute__((visibility("default"))) goss::ParameterizedODE* create_Fhn()
{
    return new goss::Fhn;
}
#endif
