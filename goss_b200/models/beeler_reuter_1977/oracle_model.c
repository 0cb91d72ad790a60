/* Generated by goss_b200.codegen from the 'beeler_reuter_1977' model; do not edit. */
/* Test infrastructure: C restatement of the model consumed by the oracle. */
#include <math.h>
#include "goss_oracle.h"

#if defined(__GNUC__)
#pragma GCC diagnostic ignored "-Wunused-variable"
#pragma GCC diagnostic ignored "-Wunused-parameter"
#endif

static void beeler_reuter_1977_rhs(const double* states, double time, const double* params, double* values)
{
  const double s_m = states[0];
  const double s_h = states[1];
  const double s_j = states[2];
  const double s_Cai = states[3];
  const double s_d = states[4];
  const double s_f = states[5];
  const double s_x1 = states[6];
  const double s_V = states[7];
  const double p_E_Na = params[0];
  const double p_g_Na = params[1];
  const double p_g_Nac = params[2];
  const double p_g_s = params[3];
  const double p_IstimAmplitude = params[4];
  const double p_IstimEnd = params[5];
  const double p_IstimPeriod = params[6];
  const double p_IstimPulseDuration = params[7];
  const double p_IstimStart = params[8];
  const double p_C = params[9];
  const double v_i_Na = ((s_V - ((p_E_Na)))*(p_g_Nac + (p_g_Na*s_h*s_j*(s_m*s_m*s_m))));
  const double v_V_eff_0 = ((fabs((47.0 + s_V)) < 0.01) ? 0.01 : (47.0 + s_V));
  const double v_alpha_m = (((-47.0) - ((s_V)))/((-1.0) + exp((-(0.1*v_V_eff_0)))));
  const double v_beta_m = (0.7095526727489909*exp((-(0.056*s_V))));
  const double v_alpha_h = (5.497962438709065e-10*exp((-(0.25*s_V))));
  const double v_beta_h = (1.7/(1.0 + (0.1580253208896478*exp((-(0.082*s_V))))));
  const double v_alpha_j = (1.8690473007222892e-10*exp((-(0.25*s_V)))/(1.0 + (1.6788275299956603e-07*exp((-(0.2*s_V))))));
  const double v_beta_j = (0.3/(1.0 + (0.040762203978366204*exp((-(0.1*s_V))))));
  const double v_E_s = ((-82.3) - ((13.0287*log((0.001*s_Cai)))));
  const double v_i_s = (s_d*s_f*p_g_s*(s_V - ((v_E_s))));
  const double v_alpha_d = (0.095*exp((0.05 - ((0.01*s_V))))/(1.0 + (1.4332881385696572*exp((-(0.07199424046076314*s_V))))));
  const double v_beta_d = (0.07*exp(((-0.7457627118644068) - ((0.01694915254237288*s_V))))/(1.0 + exp((2.2 + (0.05*s_V)))));
  const double v_alpha_f = (0.012*exp(((-0.224) - ((0.008*s_V))))/(1.0 + (66.5465065250986*exp((0.14992503748125938*s_V)))));
  const double v_beta_f = (0.0065*exp(((-0.6) - ((0.02*s_V))))/(1.0 + exp(((-6.0) - ((0.2*s_V))))));
  const double v_i_x1 = (0.0019727757115328517*s_x1*((-1.0) + (21.75840239619708*exp((0.04*s_V))))*exp((-(0.04*s_V))));
  const double v_alpha_x1 = (0.031158410986342627*exp((0.08264462809917356*s_V))/(1.0 + (17.41170806332765*exp((0.05714285714285714*s_V)))));
  const double v_beta_x1 = (0.0003916464405623223*exp((-(0.05998800239952009*s_V)))/(1.0 + exp(((-0.8) - ((0.04*s_V))))));
  const double v_V_eff_1 = ((fabs((23.0 + s_V)) < 0.01) ? 0.01 : (23.0 + s_V));
  const double v_i_K1 = ((0.0035*(4.6000000000000005 + (0.2*s_V))/(1.0 - ((exp((-(0.04*v_V_eff_1))))))) + (0.0035*((-4.0) + (119.85640018958804*exp((0.04*s_V))))/((8.331137487687693*exp((0.04*s_V))) + (69.4078518387552*exp((0.08*s_V))))));
  const double v_Istim = (((time >= p_IstimStart) && (time <= p_IstimEnd) && ((time - ((p_IstimStart)) - ((p_IstimPeriod*floor(((time - ((p_IstimStart)))/p_IstimPeriod))))) <= p_IstimPulseDuration)) ? p_IstimAmplitude : 0.0);
  values[0] = ((v_alpha_m*(1.0 - ((s_m)))) - ((v_beta_m*s_m)));
  values[1] = ((v_alpha_h*(1.0 - ((s_h)))) - ((v_beta_h*s_h)));
  values[2] = ((v_alpha_j*(1.0 - ((s_j)))) - ((v_beta_j*s_j)));
  values[3] = (7.000000000000001e-06 - ((0.07*s_Cai)) - ((0.01*v_i_s)));
  values[4] = ((v_alpha_d*(1.0 - ((s_d)))) - ((v_beta_d*s_d)));
  values[5] = ((v_alpha_f*(1.0 - ((s_f)))) - ((v_beta_f*s_f)));
  values[6] = ((v_alpha_x1*(1.0 - ((s_x1)))) - ((v_beta_x1*s_x1)));
  values[7] = ((v_Istim - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1)))/p_C);
}

static void beeler_reuter_1977_linearized(const double* states, double time, const double* params,
    double* linear, double* rhs, int only_linear)
{
  const double s_m = states[0];
  const double s_h = states[1];
  const double s_j = states[2];
  const double s_Cai = states[3];
  const double s_d = states[4];
  const double s_f = states[5];
  const double s_x1 = states[6];
  const double s_V = states[7];
  const double p_E_Na = params[0];
  const double p_g_Na = params[1];
  const double p_g_Nac = params[2];
  const double p_g_s = params[3];
  const double p_IstimAmplitude = params[4];
  const double p_IstimEnd = params[5];
  const double p_IstimPeriod = params[6];
  const double p_IstimPulseDuration = params[7];
  const double p_IstimStart = params[8];
  const double p_C = params[9];
  const double v_i_Na = ((s_V - ((p_E_Na)))*(p_g_Nac + (p_g_Na*s_h*s_j*(s_m*s_m*s_m))));
  const double v_V_eff_0 = ((fabs((47.0 + s_V)) < 0.01) ? 0.01 : (47.0 + s_V));
  const double v_alpha_m = (((-47.0) - ((s_V)))/((-1.0) + exp((-(0.1*v_V_eff_0)))));
  const double v_beta_m = (0.7095526727489909*exp((-(0.056*s_V))));
  const double v_alpha_h = (5.497962438709065e-10*exp((-(0.25*s_V))));
  const double v_beta_h = (1.7/(1.0 + (0.1580253208896478*exp((-(0.082*s_V))))));
  const double v_alpha_j = (1.8690473007222892e-10*exp((-(0.25*s_V)))/(1.0 + (1.6788275299956603e-07*exp((-(0.2*s_V))))));
  const double v_beta_j = (0.3/(1.0 + (0.040762203978366204*exp((-(0.1*s_V))))));
  const double v_E_s = ((-82.3) - ((13.0287*log((0.001*s_Cai)))));
  const double v_i_s = (s_d*s_f*p_g_s*(s_V - ((v_E_s))));
  const double v_alpha_d = (0.095*exp((0.05 - ((0.01*s_V))))/(1.0 + (1.4332881385696572*exp((-(0.07199424046076314*s_V))))));
  const double v_beta_d = (0.07*exp(((-0.7457627118644068) - ((0.01694915254237288*s_V))))/(1.0 + exp((2.2 + (0.05*s_V)))));
  const double v_alpha_f = (0.012*exp(((-0.224) - ((0.008*s_V))))/(1.0 + (66.5465065250986*exp((0.14992503748125938*s_V)))));
  const double v_beta_f = (0.0065*exp(((-0.6) - ((0.02*s_V))))/(1.0 + exp(((-6.0) - ((0.2*s_V))))));
  const double v_i_x1 = (0.0019727757115328517*s_x1*((-1.0) + (21.75840239619708*exp((0.04*s_V))))*exp((-(0.04*s_V))));
  const double v_alpha_x1 = (0.031158410986342627*exp((0.08264462809917356*s_V))/(1.0 + (17.41170806332765*exp((0.05714285714285714*s_V)))));
  const double v_beta_x1 = (0.0003916464405623223*exp((-(0.05998800239952009*s_V)))/(1.0 + exp(((-0.8) - ((0.04*s_V))))));
  const double v_V_eff_1 = ((fabs((23.0 + s_V)) < 0.01) ? 0.01 : (23.0 + s_V));
  const double v_i_K1 = ((0.0035*(4.6000000000000005 + (0.2*s_V))/(1.0 - ((exp((-(0.04*v_V_eff_1))))))) + (0.0035*((-4.0) + (119.85640018958804*exp((0.04*s_V))))/((8.331137487687693*exp((0.04*s_V))) + (69.4078518387552*exp((0.08*s_V))))));
  const double v_Istim = (((time >= p_IstimStart) && (time <= p_IstimEnd) && ((time - ((p_IstimStart)) - ((p_IstimPeriod*floor(((time - ((p_IstimStart)))/p_IstimPeriod))))) <= p_IstimPulseDuration)) ? p_IstimAmplitude : 0.0);
  rhs[0] = ((v_alpha_m*(1.0 - ((s_m)))) - ((v_beta_m*s_m)));
  rhs[1] = ((v_alpha_h*(1.0 - ((s_h)))) - ((v_beta_h*s_h)));
  rhs[2] = ((v_alpha_j*(1.0 - ((s_j)))) - ((v_beta_j*s_j)));
  rhs[3] = (7.000000000000001e-06 - ((0.07*s_Cai)) - ((0.01*v_i_s)));
  rhs[4] = ((v_alpha_d*(1.0 - ((s_d)))) - ((v_beta_d*s_d)));
  rhs[5] = ((v_alpha_f*(1.0 - ((s_f)))) - ((v_beta_f*s_f)));
  rhs[6] = ((v_alpha_x1*(1.0 - ((s_x1)))) - ((v_beta_x1*s_x1)));
  rhs[7] = ((v_Istim - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1)))/p_C);
  linear[0] = ((-(v_alpha_m)) - ((v_beta_m)));
  linear[1] = ((-(v_alpha_h)) - ((v_beta_h)));
  linear[2] = ((-(v_alpha_j)) - ((v_beta_j)));
  linear[4] = ((-(v_alpha_d)) - ((v_beta_d)));
  linear[5] = ((-(v_alpha_f)) - ((v_beta_f)));
  linear[6] = ((-(v_alpha_x1)) - ((v_beta_x1)));
  if (only_linear) return;
  const double v_dE_s_dCai = (-(13.0287/s_Cai));
  const double v_di_s_dCai = (-(s_d*v_dE_s_dCai*s_f*p_g_s));
  const double v_dV_eff_1_dV = ((fabs((23.0 + s_V)) < 0.01) ? 0.0 : 1.0);
  const double v_di_K1_dV = ((0.0007000000000000001/(1.0 - ((exp((-(0.04*v_V_eff_1))))))) + (0.016779896026542326*exp((0.04*s_V))/((8.331137487687693*exp((0.04*s_V))) + (69.4078518387552*exp((0.08*s_V))))) + (0.0035*((-4.0) + (119.85640018958804*exp((0.04*s_V))))*((-(0.3332454995075077*exp((0.04*s_V)))) - ((5.552628147100417*exp((0.08*s_V)))))/(((8.331137487687693*exp((0.04*s_V))) + (69.4078518387552*exp((0.08*s_V))))*((8.331137487687693*exp((0.04*s_V))) + (69.4078518387552*exp((0.08*s_V)))))) - ((0.00028000000000000003*v_dV_eff_1_dV*(4.6000000000000005 + (0.2*s_V))*exp((-(0.04*v_V_eff_1)))/((1.0 - ((exp((-(0.04*v_V_eff_1))))))*(1.0 - ((exp((-(0.04*v_V_eff_1))))))))));
  const double v_di_Na_dV = (p_g_Nac + (p_g_Na*s_h*s_j*(s_m*s_m*s_m)));
  const double v_di_s_dV = (s_d*s_f*p_g_s);
  const double v_di_x1_dV = ((0.0017169779107590322*s_x1) - ((7.891102846131407e-05*s_x1*((-1.0) + (21.75840239619708*exp((0.04*s_V))))*exp((-(0.04*s_V))))));
  linear[3] = ((-0.07) - ((0.01*v_di_s_dCai)));
  linear[7] = ((-(v_di_K1_dV/p_C)) - ((v_di_Na_dV/p_C)) - ((v_di_s_dV/p_C)) - ((v_di_x1_dV/p_C)));
}

static const double beeler_reuter_1977_ic[8] = {0.011, 0.988, 0.975, 0.0001, 0.003, 0.994, 0.0001, -84.624};
static const double beeler_reuter_1977_defaults[10] = {50.0, 0.04, 3e-05, 0.0005, 0.5, 50000.0, 1000.0, 1.0, 10.0, 0.01};
static const unsigned char beeler_reuter_1977_linear_terms[8] = {1, 1, 1, 0, 1, 1, 1, 0};
static const unsigned beeler_reuter_1977_field_param_index[1] = {0};

const oracle_model* oracle_model_beeler_reuter_1977(void)
{
  static oracle_model model;
  model.name = "beeler_reuter_1977";
  model.num_states = 8;
  model.num_params = 10;
  model.num_field_params = 0;
  model.field_param_index = beeler_reuter_1977_field_param_index;
  model.rhs = beeler_reuter_1977_rhs;
  model.linearized = beeler_reuter_1977_linearized;
  model.ic = beeler_reuter_1977_ic;
  model.default_params = beeler_reuter_1977_defaults;
  model.linear_terms = beeler_reuter_1977_linear_terms;
  model.jacobian = 0;
  return &model;
}
