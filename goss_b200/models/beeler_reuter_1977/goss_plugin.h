// Generated by goss_b200.codegen from the 'beeler_reuter_1977' model; do not edit.
// goss::ParameterizedODE plugin consumed by the oracle build of the reference solvers.
#ifndef BEELER_REUTER_1977_GOSS_PLUGIN_H
#define BEELER_REUTER_1977_GOSS_PLUGIN_H
#include <cmath>
#include <memory>
#include <stdexcept>
#include "goss/ParameterizedODE.h"

namespace goss {
class Beeler_reuter_1977 : public ParameterizedODE
{
  public:
    Beeler_reuter_1977() : ParameterizedODE(8, 10, 0, 0, 0), E_Na(50.0), g_Na(0.04), g_Nac(3e-05), g_s(0.0005), IstimAmplitude(0.5), IstimEnd(50000.0), IstimPeriod(1000.0), IstimPulseDuration(1.0), IstimStart(10.0), C(0.01)
    {
        _state_names[0] = "m";
        _state_names[1] = "h";
        _state_names[2] = "j";
        _state_names[3] = "Cai";
        _state_names[4] = "d";
        _state_names[5] = "f";
        _state_names[6] = "x1";
        _state_names[7] = "V";
        _parameter_names[0] = "E_Na";
        _parameter_names[1] = "g_Na";
        _parameter_names[2] = "g_Nac";
        _parameter_names[3] = "g_s";
        _parameter_names[4] = "IstimAmplitude";
        _parameter_names[5] = "IstimEnd";
        _parameter_names[6] = "IstimPeriod";
        _parameter_names[7] = "IstimPulseDuration";
        _parameter_names[8] = "IstimStart";
        _parameter_names[9] = "C";
        _param_to_value["E_Na"] = &E_Na;
        _param_to_value["g_Na"] = &g_Na;
        _param_to_value["g_Nac"] = &g_Nac;
        _param_to_value["g_s"] = &g_s;
        _param_to_value["IstimAmplitude"] = &IstimAmplitude;
        _param_to_value["IstimEnd"] = &IstimEnd;
        _param_to_value["IstimPeriod"] = &IstimPeriod;
        _param_to_value["IstimPulseDuration"] = &IstimPulseDuration;
        _param_to_value["IstimStart"] = &IstimStart;
        _param_to_value["C"] = &C;
        _linear_terms[0] = 1;
        _linear_terms[1] = 1;
        _linear_terms[2] = 1;
        _linear_terms[4] = 1;
        _linear_terms[5] = 1;
        _linear_terms[6] = 1;
    }
    Beeler_reuter_1977(const Beeler_reuter_1977& ode) : ParameterizedODE(ode), E_Na(ode.E_Na), g_Na(ode.g_Na), g_Nac(ode.g_Nac), g_s(ode.g_s), IstimAmplitude(ode.IstimAmplitude), IstimEnd(ode.IstimEnd), IstimPeriod(ode.IstimPeriod), IstimPulseDuration(ode.IstimPulseDuration), IstimStart(ode.IstimStart), C(ode.C) {}

    void eval(const double* states, double time, double* values)
    {
        const double m = states[0];
        const double h = states[1];
        const double j = states[2];
        const double Cai = states[3];
        const double d = states[4];
        const double f = states[5];
        const double x1 = states[6];
        const double V = states[7];
        const double i_Na = ((V - ((E_Na)))*(g_Nac + (g_Na*h*j*(m*m*m))));
        const double V_eff_0 = ((std::fabs((47.0 + V)) < 0.01) ? 0.01 : (47.0 + V));
        const double alpha_m = (((-47.0) - ((V)))/((-1.0) + std::exp((-(0.1*V_eff_0)))));
        const double beta_m = (0.7095526727489909*std::exp((-(0.056*V))));
        const double alpha_h = (5.497962438709065e-10*std::exp((-(0.25*V))));
        const double beta_h = (1.7/(1.0 + (0.1580253208896478*std::exp((-(0.082*V))))));
        const double alpha_j = (1.8690473007222892e-10*std::exp((-(0.25*V)))/(1.0 + (1.6788275299956603e-07*std::exp((-(0.2*V))))));
        const double beta_j = (0.3/(1.0 + (0.040762203978366204*std::exp((-(0.1*V))))));
        const double E_s = ((-82.3) - ((13.0287*std::log((0.001*Cai)))));
        const double i_s = (d*f*g_s*(V - ((E_s))));
        const double alpha_d = (0.095*std::exp((0.05 - ((0.01*V))))/(1.0 + (1.4332881385696572*std::exp((-(0.07199424046076314*V))))));
        const double beta_d = (0.07*std::exp(((-0.7457627118644068) - ((0.01694915254237288*V))))/(1.0 + std::exp((2.2 + (0.05*V)))));
        const double alpha_f = (0.012*std::exp(((-0.224) - ((0.008*V))))/(1.0 + (66.5465065250986*std::exp((0.14992503748125938*V)))));
        const double beta_f = (0.0065*std::exp(((-0.6) - ((0.02*V))))/(1.0 + std::exp(((-6.0) - ((0.2*V))))));
        const double i_x1 = (0.0019727757115328517*x1*((-1.0) + (21.75840239619708*std::exp((0.04*V))))*std::exp((-(0.04*V))));
        const double alpha_x1 = (0.031158410986342627*std::exp((0.08264462809917356*V))/(1.0 + (17.41170806332765*std::exp((0.05714285714285714*V)))));
        const double beta_x1 = (0.0003916464405623223*std::exp((-(0.05998800239952009*V)))/(1.0 + std::exp(((-0.8) - ((0.04*V))))));
        const double V_eff_1 = ((std::fabs((23.0 + V)) < 0.01) ? 0.01 : (23.0 + V));
        const double i_K1 = ((0.0035*(4.6000000000000005 + (0.2*V))/(1.0 - ((std::exp((-(0.04*V_eff_1))))))) + (0.0035*((-4.0) + (119.85640018958804*std::exp((0.04*V))))/((8.331137487687693*std::exp((0.04*V))) + (69.4078518387552*std::exp((0.08*V))))));
        const double Istim = (((time >= IstimStart) && (time <= IstimEnd) && ((time - ((IstimStart)) - ((IstimPeriod*std::floor(((time - ((IstimStart)))/IstimPeriod))))) <= IstimPulseDuration)) ? IstimAmplitude : 0.0);
        values[0] = ((alpha_m*(1.0 - ((m)))) - ((beta_m*m)));
        values[1] = ((alpha_h*(1.0 - ((h)))) - ((beta_h*h)));
        values[2] = ((alpha_j*(1.0 - ((j)))) - ((beta_j*j)));
        values[3] = (7.000000000000001e-06 - ((0.07*Cai)) - ((0.01*i_s)));
        values[4] = ((alpha_d*(1.0 - ((d)))) - ((beta_d*d)));
        values[5] = ((alpha_f*(1.0 - ((f)))) - ((beta_f*f)));
        values[6] = ((alpha_x1*(1.0 - ((x1)))) - ((beta_x1*x1)));
        values[7] = ((Istim - ((i_K1)) - ((i_Na)) - ((i_s)) - ((i_x1)))/C);
    }

    void linearized_eval(const double* states, double time, double* linear, double* rhs,
                         bool only_linear) const
    {
        const double m = states[0];
        const double h = states[1];
        const double j = states[2];
        const double Cai = states[3];
        const double d = states[4];
        const double f = states[5];
        const double x1 = states[6];
        const double V = states[7];
        const double i_Na = ((V - ((E_Na)))*(g_Nac + (g_Na*h*j*(m*m*m))));
        const double V_eff_0 = ((std::fabs((47.0 + V)) < 0.01) ? 0.01 : (47.0 + V));
        const double alpha_m = (((-47.0) - ((V)))/((-1.0) + std::exp((-(0.1*V_eff_0)))));
        const double beta_m = (0.7095526727489909*std::exp((-(0.056*V))));
        const double alpha_h = (5.497962438709065e-10*std::exp((-(0.25*V))));
        const double beta_h = (1.7/(1.0 + (0.1580253208896478*std::exp((-(0.082*V))))));
        const double alpha_j = (1.8690473007222892e-10*std::exp((-(0.25*V)))/(1.0 + (1.6788275299956603e-07*std::exp((-(0.2*V))))));
        const double beta_j = (0.3/(1.0 + (0.040762203978366204*std::exp((-(0.1*V))))));
        const double E_s = ((-82.3) - ((13.0287*std::log((0.001*Cai)))));
        const double i_s = (d*f*g_s*(V - ((E_s))));
        const double alpha_d = (0.095*std::exp((0.05 - ((0.01*V))))/(1.0 + (1.4332881385696572*std::exp((-(0.07199424046076314*V))))));
        const double beta_d = (0.07*std::exp(((-0.7457627118644068) - ((0.01694915254237288*V))))/(1.0 + std::exp((2.2 + (0.05*V)))));
        const double alpha_f = (0.012*std::exp(((-0.224) - ((0.008*V))))/(1.0 + (66.5465065250986*std::exp((0.14992503748125938*V)))));
        const double beta_f = (0.0065*std::exp(((-0.6) - ((0.02*V))))/(1.0 + std::exp(((-6.0) - ((0.2*V))))));
        const double i_x1 = (0.0019727757115328517*x1*((-1.0) + (21.75840239619708*std::exp((0.04*V))))*std::exp((-(0.04*V))));
        const double alpha_x1 = (0.031158410986342627*std::exp((0.08264462809917356*V))/(1.0 + (17.41170806332765*std::exp((0.05714285714285714*V)))));
        const double beta_x1 = (0.0003916464405623223*std::exp((-(0.05998800239952009*V)))/(1.0 + std::exp(((-0.8) - ((0.04*V))))));
        const double V_eff_1 = ((std::fabs((23.0 + V)) < 0.01) ? 0.01 : (23.0 + V));
        const double i_K1 = ((0.0035*(4.6000000000000005 + (0.2*V))/(1.0 - ((std::exp((-(0.04*V_eff_1))))))) + (0.0035*((-4.0) + (119.85640018958804*std::exp((0.04*V))))/((8.331137487687693*std::exp((0.04*V))) + (69.4078518387552*std::exp((0.08*V))))));
        const double Istim = (((time >= IstimStart) && (time <= IstimEnd) && ((time - ((IstimStart)) - ((IstimPeriod*std::floor(((time - ((IstimStart)))/IstimPeriod))))) <= IstimPulseDuration)) ? IstimAmplitude : 0.0);
        rhs[0] = ((alpha_m*(1.0 - ((m)))) - ((beta_m*m)));
        rhs[1] = ((alpha_h*(1.0 - ((h)))) - ((beta_h*h)));
        rhs[2] = ((alpha_j*(1.0 - ((j)))) - ((beta_j*j)));
        rhs[3] = (7.000000000000001e-06 - ((0.07*Cai)) - ((0.01*i_s)));
        rhs[4] = ((alpha_d*(1.0 - ((d)))) - ((beta_d*d)));
        rhs[5] = ((alpha_f*(1.0 - ((f)))) - ((beta_f*f)));
        rhs[6] = ((alpha_x1*(1.0 - ((x1)))) - ((beta_x1*x1)));
        rhs[7] = ((Istim - ((i_K1)) - ((i_Na)) - ((i_s)) - ((i_x1)))/C);
        linear[0] = ((-(alpha_m)) - ((beta_m)));
        linear[1] = ((-(alpha_h)) - ((beta_h)));
        linear[2] = ((-(alpha_j)) - ((beta_j)));
        linear[4] = ((-(alpha_d)) - ((beta_d)));
        linear[5] = ((-(alpha_f)) - ((beta_f)));
        linear[6] = ((-(alpha_x1)) - ((beta_x1)));
        if (only_linear) return;
        const double dE_s_dCai = (-(13.0287/Cai));
        const double di_s_dCai = (-(d*dE_s_dCai*f*g_s));
        const double dV_eff_1_dV = ((std::fabs((23.0 + V)) < 0.01) ? 0.0 : 1.0);
        const double di_K1_dV = ((0.0007000000000000001/(1.0 - ((std::exp((-(0.04*V_eff_1))))))) + (0.016779896026542326*std::exp((0.04*V))/((8.331137487687693*std::exp((0.04*V))) + (69.4078518387552*std::exp((0.08*V))))) + (0.0035*((-4.0) + (119.85640018958804*std::exp((0.04*V))))*((-(0.3332454995075077*std::exp((0.04*V)))) - ((5.552628147100417*std::exp((0.08*V)))))/(((8.331137487687693*std::exp((0.04*V))) + (69.4078518387552*std::exp((0.08*V))))*((8.331137487687693*std::exp((0.04*V))) + (69.4078518387552*std::exp((0.08*V)))))) - ((0.00028000000000000003*dV_eff_1_dV*(4.6000000000000005 + (0.2*V))*std::exp((-(0.04*V_eff_1)))/((1.0 - ((std::exp((-(0.04*V_eff_1))))))*(1.0 - ((std::exp((-(0.04*V_eff_1))))))))));
        const double di_Na_dV = (g_Nac + (g_Na*h*j*(m*m*m)));
        const double di_s_dV = (d*f*g_s);
        const double di_x1_dV = ((0.0017169779107590322*x1) - ((7.891102846131407e-05*x1*((-1.0) + (21.75840239619708*std::exp((0.04*V))))*std::exp((-(0.04*V))))));
        linear[3] = ((-0.07) - ((0.01*di_s_dCai)));
        linear[7] = ((-(di_K1_dV/C)) - ((di_Na_dV/C)) - ((di_s_dV/C)) - ((di_x1_dV/C)));
    }

    void get_ic(goss::DoubleVector* values) const
    {
        values->n = _num_states;
        values->data.reset(new double[_num_states]);
        values->data[0] = 0.011;
        values->data[1] = 0.988;
        values->data[2] = 0.975;
        values->data[3] = 0.0001;
        values->data[4] = 0.003;
        values->data[5] = 0.994;
        values->data[6] = 0.0001;
        values->data[7] = -84.624;
    }

    std::shared_ptr<ODE> copy() const { return std::make_shared<Beeler_reuter_1977>(*this); }

    void eval_monitored(const double* states, double time, double* monitored) const
    {
        throw std::runtime_error("No monitored in the \'Beeler_reuter_1977\' model.");
    }

    void set_field_parameters(const double* field_params)
    {
        (void)field_params;
    }

  private:
    double E_Na, g_Na, g_Nac, g_s, IstimAmplitude, IstimEnd, IstimPeriod, IstimPulseDuration, IstimStart, C;
};
}  // namespace goss

extern "C" __attribute__((visibility("default"))) goss::ParameterizedODE* create_Beeler_reuter_1977()
{
    return new goss::Beeler_reuter_1977;
}
#endif
