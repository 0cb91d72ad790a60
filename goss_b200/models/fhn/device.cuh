// Generated by goss_b200.codegen from the 'fhn' model; do not edit.
// Device-side model: rhs and linearised rhs templated on the arithmetic type T.
#ifndef FHN_DEVICE_CUH
#define FHN_DEVICE_CUH
#include "goss_device_math.cuh"

namespace goss_b200 { namespace models {

struct Fhn {
  static constexpr const char* name = "fhn";
  static constexpr int num_states = 2;
  static constexpr int num_params = 11;
  static constexpr int num_field_params = 0;
  static constexpr int num_monitored = 0;

  // values = f(y, time)
  template <typename T>
  __device__ static __forceinline__ void rhs(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ values)
  {
    const T s_v = y[0];
    const T s_s = y[1];
    const T v_v_amp = (P[9] - ((P[10])));
    const T v_v_th = (P[10] + (P[0]*v_v_amp));
    const T v_I = ((-(P[3]*s_s*(s_v - ((P[10])))/v_v_amp)) + (P[2]*(s_v - ((P[10])))*(s_v - ((v_v_th)))*(P[9] - ((s_v)))/(v_v_amp*v_v_amp)));
    const double v_i_Stim = (PD[5]*(1.0 - ((1.0/(1.0 + exp(((5.0*time) - ((5.0*PD[8]))))))))/(1.0 + exp(((5.0*time) - ((5.0*PD[6])) - ((5.0*PD[8]))))));
    values[0] = (v_I + T(v_i_Stim));
    values[1] = (P[1]*(s_v - ((P[10])) - ((P[4]*s_s))));
    (void)time; (void)P; (void)PD; (void)F;
  }

  // rhs = f(y, time), linear[i] = d f_i / d y_i
  template <typename T>
  __device__ static __forceinline__ void linearized(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ linear, T* __restrict__ rhs)
  {
    const T s_v = y[0];
    const T s_s = y[1];
    const T v_v_amp = (P[9] - ((P[10])));
    const T v_v_th = (P[10] + (P[0]*v_v_amp));
    const T v_I = ((-(P[3]*s_s*(s_v - ((P[10])))/v_v_amp)) + (P[2]*(s_v - ((P[10])))*(s_v - ((v_v_th)))*(P[9] - ((s_v)))/(v_v_amp*v_v_amp)));
    const double v_i_Stim = (PD[5]*(1.0 - ((1.0/(1.0 + exp(((5.0*time) - ((5.0*PD[8]))))))))/(1.0 + exp(((5.0*time) - ((5.0*PD[6])) - ((5.0*PD[8]))))));
    rhs[0] = (v_I + T(v_i_Stim));
    rhs[1] = (P[1]*(s_v - ((P[10])) - ((P[4]*s_s))));
    linear[1] = (-(P[1]*P[4]));
    const T v_dI_dv = ((-(P[3]*s_s/v_v_amp)) + (P[2]*(s_v - ((P[10])))*(P[9] - ((s_v)))/(v_v_amp*v_v_amp)) + (P[2]*(s_v - ((v_v_th)))*(P[9] - ((s_v)))/(v_v_amp*v_v_amp)) - ((P[2]*(s_v - ((P[10])))*(s_v - ((v_v_th)))/(v_v_amp*v_v_amp))));
    linear[0] = v_dI_dv;
    (void)time; (void)P; (void)PD; (void)F;
  }
};

}}  // namespace goss_b200::models
#endif
