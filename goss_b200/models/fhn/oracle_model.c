/* Generated by goss_b200.codegen from the 'fhn' model; do not edit. */
/* Test infrastructure: C restatement of the model consumed by the oracle. */
#include <math.h>
#include "goss_oracle.h"

#if defined(__GNUC__)
#pragma GCC diagnostic ignored "-Wunused-variable"
#pragma GCC diagnostic ignored "-Wunused-parameter"
#endif

static void fhn_rhs(const double* states, double time, const double* params, double* values)
{
  const double s_v = states[0];
  const double s_s = states[1];
  const double p_a = params[0];
  const double p_b = params[1];
  const double p_c_1 = params[2];
  const double p_c_2 = params[3];
  const double p_c_3 = params[4];
  const double p_stim_amplitude = params[5];
  const double p_stim_duration = params[6];
  const double p_stim_period = params[7];
  const double p_stim_start = params[8];
  const double p_v_peak = params[9];
  const double p_v_rest = params[10];
  const double v_v_amp = (p_v_peak - ((p_v_rest)));
  const double v_v_th = (p_v_rest + (p_a*v_v_amp));
  const double v_I = ((-(p_c_2*s_s*(s_v - ((p_v_rest)))/v_v_amp)) + (p_c_1*(s_v - ((p_v_rest)))*(s_v - ((v_v_th)))*(p_v_peak - ((s_v)))/(v_v_amp*v_v_amp)));
  const double v_i_Stim = (p_stim_amplitude*(1.0 - ((1.0/(1.0 + exp(((5.0*time) - ((5.0*p_stim_start))))))))/(1.0 + exp(((5.0*time) - ((5.0*p_stim_duration)) - ((5.0*p_stim_start))))));
  values[0] = (v_I + v_i_Stim);
  values[1] = (p_b*(s_v - ((p_v_rest)) - ((p_c_3*s_s))));
}

static void fhn_linearized(const double* states, double time, const double* params,
    double* linear, double* rhs, int only_linear)
{
  const double s_v = states[0];
  const double s_s = states[1];
  const double p_a = params[0];
  const double p_b = params[1];
  const double p_c_1 = params[2];
  const double p_c_2 = params[3];
  const double p_c_3 = params[4];
  const double p_stim_amplitude = params[5];
  const double p_stim_duration = params[6];
  const double p_stim_period = params[7];
  const double p_stim_start = params[8];
  const double p_v_peak = params[9];
  const double p_v_rest = params[10];
  const double v_v_amp = (p_v_peak - ((p_v_rest)));
  const double v_v_th = (p_v_rest + (p_a*v_v_amp));
  const double v_I = ((-(p_c_2*s_s*(s_v - ((p_v_rest)))/v_v_amp)) + (p_c_1*(s_v - ((p_v_rest)))*(s_v - ((v_v_th)))*(p_v_peak - ((s_v)))/(v_v_amp*v_v_amp)));
  const double v_i_Stim = (p_stim_amplitude*(1.0 - ((1.0/(1.0 + exp(((5.0*time) - ((5.0*p_stim_start))))))))/(1.0 + exp(((5.0*time) - ((5.0*p_stim_duration)) - ((5.0*p_stim_start))))));
  rhs[0] = (v_I + v_i_Stim);
  rhs[1] = (p_b*(s_v - ((p_v_rest)) - ((p_c_3*s_s))));
  linear[1] = (-(p_b*p_c_3));
  if (only_linear) return;
  const double v_dI_dv = ((-(p_c_2*s_s/v_v_amp)) + (p_c_1*(s_v - ((p_v_rest)))*(p_v_peak - ((s_v)))/(v_v_amp*v_v_amp)) + (p_c_1*(s_v - ((v_v_th)))*(p_v_peak - ((s_v)))/(v_v_amp*v_v_amp)) - ((p_c_1*(s_v - ((p_v_rest)))*(s_v - ((v_v_th)))/(v_v_amp*v_v_amp))));
  linear[0] = v_dI_dv;
}

static const double fhn_ic[2] = {-85.0, 0.0};
static const double fhn_defaults[11] = {0.13, 0.013, 0.26, 0.1, 1.0, 50.0, 1.0, 1000.0, 1.0, 40.0, -85.0};
static const unsigned char fhn_linear_terms[2] = {0, 1};
static const unsigned fhn_field_param_index[1] = {0};

const oracle_model* oracle_model_fhn(void)
{
  static oracle_model model;
  model.name = "fhn";
  model.num_states = 2;
  model.num_params = 11;
  model.num_field_params = 0;
  model.field_param_index = fhn_field_param_index;
  model.rhs = fhn_rhs;
  model.linearized = fhn_linearized;
  model.ic = fhn_ic;
  model.default_params = fhn_defaults;
  model.linear_terms = fhn_linear_terms;
  model.jacobian = 0;
  return &model;
}
