/* Generated by goss_b200.codegen from the 'fitzhughnagumo' model; do not edit. */
/* Test infrastructure: C restatement of the model consumed by the oracle. */
#include <math.h>
#include "goss_oracle.h"

#if defined(__GNUC__)
#pragma GCC diagnostic ignored "-Wunused-variable"
#pragma GCC diagnostic ignored "-Wunused-parameter"
#endif

static void fitzhughnagumo_rhs(const double* states, double time, const double* params, double* values)
{
  const double s_V = states[0];
  const double s_s = states[1];
  const double p_V_peak = params[0];
  const double p_V_rest = params[1];
  const double p_a = params[2];
  const double p_b = params[3];
  const double p_c_1 = params[4];
  const double p_c_2 = params[5];
  const double p_c_3 = params[6];
  const double p_stim_amplitude = params[7];
  const double p_stim_duration = params[8];
  const double p_stim_period = params[9];
  const double p_stim_start = params[10];
  const double v_V_amp = (p_V_peak - ((p_V_rest)));
  const double v_V_th = (p_V_rest + (v_V_amp*p_a));
  const double v_I = ((-(p_c_2*s_s*(s_V - ((p_V_rest)))/v_V_amp)) + (p_c_1*(s_V - ((p_V_rest)))*(s_V - ((v_V_th)))*(p_V_peak - ((s_V)))/(v_V_amp*v_V_amp)));
  const double v_i_Stim = (p_stim_amplitude*(1.0 - ((1.0/(1.0 + exp(((5.0*time) - ((5.0*p_stim_start))))))))/(1.0 + exp(((5.0*time) - ((5.0*p_stim_duration)) - ((5.0*p_stim_start))))));
  values[0] = (v_I + v_i_Stim);
  values[1] = (p_b*(s_V - ((p_V_rest)) - ((p_c_3*s_s))));
}

static void fitzhughnagumo_linearized(const double* states, double time, const double* params,
    double* linear, double* rhs, int only_linear)
{
  const double s_V = states[0];
  const double s_s = states[1];
  const double p_V_peak = params[0];
  const double p_V_rest = params[1];
  const double p_a = params[2];
  const double p_b = params[3];
  const double p_c_1 = params[4];
  const double p_c_2 = params[5];
  const double p_c_3 = params[6];
  const double p_stim_amplitude = params[7];
  const double p_stim_duration = params[8];
  const double p_stim_period = params[9];
  const double p_stim_start = params[10];
  const double v_V_amp = (p_V_peak - ((p_V_rest)));
  const double v_V_th = (p_V_rest + (v_V_amp*p_a));
  const double v_I = ((-(p_c_2*s_s*(s_V - ((p_V_rest)))/v_V_amp)) + (p_c_1*(s_V - ((p_V_rest)))*(s_V - ((v_V_th)))*(p_V_peak - ((s_V)))/(v_V_amp*v_V_amp)));
  const double v_i_Stim = (p_stim_amplitude*(1.0 - ((1.0/(1.0 + exp(((5.0*time) - ((5.0*p_stim_start))))))))/(1.0 + exp(((5.0*time) - ((5.0*p_stim_duration)) - ((5.0*p_stim_start))))));
  rhs[0] = (v_I + v_i_Stim);
  rhs[1] = (p_b*(s_V - ((p_V_rest)) - ((p_c_3*s_s))));
  linear[1] = (-(p_b*p_c_3));
  if (only_linear) return;
  const double v_dI_dV = ((-(p_c_2*s_s/v_V_amp)) + (p_c_1*(s_V - ((p_V_rest)))*(p_V_peak - ((s_V)))/(v_V_amp*v_V_amp)) + (p_c_1*(s_V - ((v_V_th)))*(p_V_peak - ((s_V)))/(v_V_amp*v_V_amp)) - ((p_c_1*(s_V - ((p_V_rest)))*(s_V - ((v_V_th)))/(v_V_amp*v_V_amp))));
  linear[0] = v_dI_dV;
}

static void fitzhughnagumo_monitored(const double* states, double time, const double* params, double* monitored)
{
  const double s_V = states[0];
  const double s_s = states[1];
  const double p_V_peak = params[0];
  const double p_V_rest = params[1];
  const double p_a = params[2];
  const double p_b = params[3];
  const double p_c_1 = params[4];
  const double p_c_2 = params[5];
  const double p_c_3 = params[6];
  const double p_stim_amplitude = params[7];
  const double p_stim_duration = params[8];
  const double p_stim_period = params[9];
  const double p_stim_start = params[10];
  const double v_p_42 = 42.0;
  const double v_p_V = s_V;
  monitored[0] = v_p_42;
  monitored[1] = v_p_V;
}

static const double fitzhughnagumo_ic[2] = {-85.0, 0.0};
static const double fitzhughnagumo_defaults[11] = {40.0, -85.0, 0.13, 0.013, 0.26, 0.1, 1.0, 50.0, 1.0, 1000.0, 1.0};
static const unsigned char fitzhughnagumo_linear_terms[2] = {0, 1};
static const unsigned fitzhughnagumo_field_param_index[1] = {0};

const oracle_model* oracle_model_fitzhughnagumo(void)
{
  static oracle_model model;
  model.name = "fitzhughnagumo";
  model.num_states = 2;
  model.num_params = 11;
  model.num_field_params = 0;
  model.field_param_index = fitzhughnagumo_field_param_index;
  model.rhs = fitzhughnagumo_rhs;
  model.linearized = fitzhughnagumo_linearized;
  model.ic = fitzhughnagumo_ic;
  model.default_params = fitzhughnagumo_defaults;
  model.linear_terms = fitzhughnagumo_linear_terms;
  model.jacobian = 0;
  return &model;
}
