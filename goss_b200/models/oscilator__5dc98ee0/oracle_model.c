/* Generated by goss_b200.codegen from the 'oscilator' model; do not edit. */
/* Test infrastructure: C restatement of the model consumed by the oracle. */
#include <math.h>
#include "goss_oracle.h"

#if defined(__GNUC__)
#pragma GCC diagnostic ignored "-Wunused-variable"
#pragma GCC diagnostic ignored "-Wunused-parameter"
#endif

static void oscilator_rhs(const double* states, double time, const double* params, double* values)
{
  const double s_x = states[0];
  const double s_y = states[1];
  const double p_a = params[0];
  const double p_b = params[1];
  values[0] = (-(p_a*s_y));
  values[1] = (p_b*s_x);
}

static void oscilator_linearized(const double* states, double time, const double* params,
    double* linear, double* rhs, int only_linear)
{
  const double s_x = states[0];
  const double s_y = states[1];
  const double p_a = params[0];
  const double p_b = params[1];
  rhs[0] = (-(p_a*s_y));
  rhs[1] = (p_b*s_x);
  if (only_linear) return;
  linear[0] = 0.0;
  linear[1] = 0.0;
}

static const double oscilator_ic[2] = {1.0, 0.0};
static const double oscilator_defaults[2] = {1.0, 1.0};
static const unsigned char oscilator_linear_terms[2] = {0, 0};
static const unsigned oscilator_field_param_index[2] = {0, 1};

const oracle_model* oracle_model_oscilator(void)
{
  static oracle_model model;
  model.name = "oscilator";
  model.num_states = 2;
  model.num_params = 2;
  model.num_field_params = 2;
  model.field_param_index = oscilator_field_param_index;
  model.rhs = oscilator_rhs;
  model.linearized = oscilator_linearized;
  model.ic = oscilator_ic;
  model.default_params = oscilator_defaults;
  model.linear_terms = oscilator_linear_terms;
  model.jacobian = 0;
  return &model;
}
