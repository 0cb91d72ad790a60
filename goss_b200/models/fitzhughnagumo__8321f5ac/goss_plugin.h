// Generated by goss_b200.codegen from the 'fitzhughnagumo' model; do not edit.
// goss::ParameterizedODE plugin consumed by the oracle build of the reference solvers.
#ifndef FITZHUGHNAGUMO_GOSS_PLUGIN_H
#define FITZHUGHNAGUMO_GOSS_PLUGIN_H
#include <cmath>
#include <memory>
#include <stdexcept>
#include "goss/ParameterizedODE.h"

namespace goss {
class Fitzhughnagumo : public ParameterizedODE
{
  public:
    Fitzhughnagumo() : ParameterizedODE(2, 11, 0, 0, 2), V_peak(40.0), V_rest(-85.0), a(0.13), b(0.013), c_1(0.26), c_2(0.1), c_3(1.0), stim_amplitude(50.0), stim_duration(1.0), stim_period(1000.0), stim_start(1.0)
    {
        _state_names[0] = "V";
        _state_names[1] = "s";
        _parameter_names[0] = "V_peak";
        _parameter_names[1] = "V_rest";
        _parameter_names[2] = "a";
        _parameter_names[3] = "b";
        _parameter_names[4] = "c_1";
        _parameter_names[5] = "c_2";
        _parameter_names[6] = "c_3";
        _parameter_names[7] = "stim_amplitude";
        _parameter_names[8] = "stim_duration";
        _parameter_names[9] = "stim_period";
        _parameter_names[10] = "stim_start";
        _monitored_names[0] = "p_42";
        _monitored_names[1] = "p_V";
        _param_to_value["V_peak"] = &V_peak;
        _param_to_value["V_rest"] = &V_rest;
        _param_to_value["a"] = &a;
        _param_to_value["b"] = &b;
        _param_to_value["c_1"] = &c_1;
        _param_to_value["c_2"] = &c_2;
        _param_to_value["c_3"] = &c_3;
        _param_to_value["stim_amplitude"] = &stim_amplitude;
        _param_to_value["stim_duration"] = &stim_duration;
        _param_to_value["stim_period"] = &stim_period;
        _param_to_value["stim_start"] = &stim_start;
        _linear_terms[1] = 1;
    }
    Fitzhughnagumo(const Fitzhughnagumo& ode) : ParameterizedODE(ode), V_peak(ode.V_peak), V_rest(ode.V_rest), a(ode.a), b(ode.b), c_1(ode.c_1), c_2(ode.c_2), c_3(ode.c_3), stim_amplitude(ode.stim_amplitude), stim_duration(ode.stim_duration), stim_period(ode.stim_period), stim_start(ode.stim_start) {}

    void eval(const double* states, double time, double* values)
    {
        const double V = states[0];
        const double s = states[1];
        const double V_amp = (V_peak - ((V_rest)));
        const double V_th = (V_rest + (V_amp*a));
        const double I = ((-(c_2*s*(V - ((V_rest)))/V_amp)) + (c_1*(V - ((V_rest)))*(V - ((V_th)))*(V_peak - ((V)))/(V_amp*V_amp)));
        const double i_Stim = (stim_amplitude*(1.0 - ((1.0/(1.0 + std::exp(((5.0*time) - ((5.0*stim_start))))))))/(1.0 + std::exp(((5.0*time) - ((5.0*stim_duration)) - ((5.0*stim_start))))));
        values[0] = (I + i_Stim);
        values[1] = (b*(V - ((V_rest)) - ((c_3*s))));
    }

    void linearized_eval(const double* states, double time, double* linear, double* rhs,
                         bool only_linear) const
    {
        const double V = states[0];
        const double s = states[1];
        const double V_amp = (V_peak - ((V_rest)));
        const double V_th = (V_rest + (V_amp*a));
        const double I = ((-(c_2*s*(V - ((V_rest)))/V_amp)) + (c_1*(V - ((V_rest)))*(V - ((V_th)))*(V_peak - ((V)))/(V_amp*V_amp)));
        const double i_Stim = (stim_amplitude*(1.0 - ((1.0/(1.0 + std::exp(((5.0*time) - ((5.0*stim_start))))))))/(1.0 + std::exp(((5.0*time) - ((5.0*stim_duration)) - ((5.0*stim_start))))));
        rhs[0] = (I + i_Stim);
        rhs[1] = (b*(V - ((V_rest)) - ((c_3*s))));
        linear[1] = (-(b*c_3));
        if (only_linear) return;
        const double dI_dV = ((-(c_2*s/V_amp)) + (c_1*(V - ((V_rest)))*(V_peak - ((V)))/(V_amp*V_amp)) + (c_1*(V - ((V_th)))*(V_peak - ((V)))/(V_amp*V_amp)) - ((c_1*(V - ((V_rest)))*(V - ((V_th)))/(V_amp*V_amp))));
        linear[0] = dI_dV;
    }

    void get_ic(goss::DoubleVector* values) const
    {
        values->n = _num_states;
        values->data.reset(new double[_num_states]);
        values->data[0] = -85.0;
        values->data[1] = 0.0;
    }

    std::shared_ptr<ODE> copy() const { return std::make_shared<Fitzhughnagumo>(*this); }

    void eval_monitored(const double* states, double time, double* monitored) const
    {
        const double V = states[0];
        const double s = states[1];
        const double p_42 = 42.0;
        const double p_V = V;
        monitored[0] = p_42;
        monitored[1] = p_V;
    }

    void set_field_parameters(const double* field_params)
    {
        (void)field_params;
    }

  private:
    double V_peak, V_rest, a, b, c_1, c_2, c_3, stim_amplitude, stim_duration, stim_period, stim_start;
};
}  // namespace goss

extern "C" __attribute__((visibility("default"))) goss::ParameterizedODE* create_Fitzhughnagumo()
{
    return new goss::Fitzhughnagumo;
}
#endif
