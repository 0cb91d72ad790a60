// Generated by goss_b200.codegen from the 'fitzhughnagumo' model; do not edit.
// Device-side model: rhs and linearised rhs templated on the arithmetic type T.
#ifndef FITZHUGHNAGUMO_DEVICE_CUH
#define FITZHUGHNAGUMO_DEVICE_CUH
#include "goss_device_math.cuh"

namespace goss_b200 { namespace models {

struct Fitzhughnagumo {
  static constexpr const char* name = "fitzhughnagumo";
  static constexpr int num_states = 2;
  static constexpr int num_params = 11;
  static constexpr int num_field_params = 2;
  static constexpr int num_monitored = 0;

  // values = f(y, time)
  template <typename T>
  __device__ static __forceinline__ void rhs(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ values)
  {
    const T s_V = y[0];
    const T s_s = y[1];
    const T v_V_amp = (P[0] - ((P[1])));
    const T v_V_th = (P[1] + (v_V_amp*F[0]));
    const T v_I = ((-(P[5]*s_s*(s_V - ((P[1])))/v_V_amp)) + (P[4]*(s_V - ((P[1])))*(s_V - ((v_V_th)))*(P[0] - ((s_V)))/(v_V_amp*v_V_amp)));
    const double v_i_Stim = (PD[7]*(1.0 - ((1.0/(1.0 + exp(((5.0*time) - ((5.0*PD[10]))))))))/(1.0 + exp(((5.0*time) - ((5.0*PD[8])) - ((5.0*PD[10]))))));
    values[0] = (v_I + T(v_i_Stim));
    values[1] = (F[1]*(s_V - ((P[1])) - ((P[6]*s_s))));
    (void)time; (void)P; (void)PD; (void)F;
  }

  // rhs = f(y, time), linear[i] = d f_i / d y_i
  template <typename T>
  __device__ static __forceinline__ void linearized(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ linear, T* __restrict__ rhs)
  {
    const T s_V = y[0];
    const T s_s = y[1];
    const T v_V_amp = (P[0] - ((P[1])));
    const T v_V_th = (P[1] + (v_V_amp*F[0]));
    const T v_I = ((-(P[5]*s_s*(s_V - ((P[1])))/v_V_amp)) + (P[4]*(s_V - ((P[1])))*(s_V - ((v_V_th)))*(P[0] - ((s_V)))/(v_V_amp*v_V_amp)));
    const double v_i_Stim = (PD[7]*(1.0 - ((1.0/(1.0 + exp(((5.0*time) - ((5.0*PD[10]))))))))/(1.0 + exp(((5.0*time) - ((5.0*PD[8])) - ((5.0*PD[10]))))));
    rhs[0] = (v_I + T(v_i_Stim));
    rhs[1] = (F[1]*(s_V - ((P[1])) - ((P[6]*s_s))));
    linear[1] = (-(F[1]*P[6]));
    const T v_dI_dV = ((-(P[5]*s_s/v_V_amp)) + (P[4]*(s_V - ((P[1])))*(P[0] - ((s_V)))/(v_V_amp*v_V_amp)) + (P[4]*(s_V - ((v_V_th)))*(P[0] - ((s_V)))/(v_V_amp*v_V_amp)) - ((P[4]*(s_V - ((P[1])))*(s_V - ((v_V_th)))/(v_V_amp*v_V_amp))));
    linear[0] = v_dI_dV;
    (void)time; (void)P; (void)PD; (void)F;
  }
};

}}  // namespace goss_b200::models
#endif
