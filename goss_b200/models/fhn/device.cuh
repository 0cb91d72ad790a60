// Generated by goss_b200.codegen from the 'fhn' model; do not edit.
// Device-side model: rhs and linearised rhs templated on the arithmetic type T.
#ifndef M_FHN_DEVICE_CUH
#define M_FHN_DEVICE_CUH
#include "goss_device_math.cuh"

namespace goss_b200 { namespace models {

struct M_fhn {
  static constexpr const char* name = "fhn";
  static constexpr int num_states = 2;
  static constexpr int num_params = 11;
  static constexpr int num_field_params = 0;
  static constexpr int num_monitored = 0;
  static constexpr int num_derived = 9;

  // values = f(y, time)
  template <typename T>
  __device__ static __forceinline__ void rhs(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ values)
  {
    const T s_v = y[0];
    const T s_s = y[1];
    const T v_I = ((P[12]*s_s*(P[11] + s_v)) + (P[14]*(P[11] + s_v)*(P[13] + s_v)*(P[9] - ((s_v)))));
    const double v_i_Stim = (PD[5]*(1.0 - ((1.0/(1.0 + exp((PD[16] + (5.0*time)))))))/(1.0 + exp((PD[15] + (5.0*time)))));
    values[0] = (v_I + T(v_i_Stim));
    values[1] = (P[1]*(P[11] + s_v + (P[17]*s_s)));
    (void)time; (void)P; (void)PD; (void)F;
  }

  // derived constants: parameter-only sub-expressions, evaluated once per
  // launch on the host in FP64 and stored after the parameters
  static void derived(const double* P, double* C)
  {
    const double v_v_amp = (P[9] - ((P[10])));
    const double v_v_th = (P[10] + (P[0]*v_v_amp));
    C[0] = (-(P[10]));
    C[1] = (-(P[3]/v_v_amp));
    C[2] = (-(v_v_th));
    C[3] = (P[2]/(v_v_amp*v_v_amp));
    C[4] = ((-(5.0*P[6])) - ((5.0*P[8])));
    C[5] = (-(5.0*P[8]));
    C[6] = (-(P[4]));
    C[7] = (-(P[1]*P[4]));
    C[8] = (-(P[2]/(v_v_amp*v_v_amp)));
    (void)P; (void)C;
  }

  // rhs = f(y, time), linear[i] = d f_i / d y_i
  template <typename T>
  __device__ static __forceinline__ void linearized(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ linear, T* __restrict__ rhs)
  {
    const T s_v = y[0];
    const T s_s = y[1];
    const T v_I = ((P[12]*s_s*(P[11] + s_v)) + (P[14]*(P[11] + s_v)*(P[13] + s_v)*(P[9] - ((s_v)))));
    const double v_i_Stim = (PD[5]*(1.0 - ((1.0/(1.0 + exp((PD[16] + (5.0*time)))))))/(1.0 + exp((PD[15] + (5.0*time)))));
    rhs[0] = (v_I + T(v_i_Stim));
    rhs[1] = (P[1]*(P[11] + s_v + (P[17]*s_s)));
    linear[1] = P[18];
    const T v_dI_dv = ((P[12]*s_s) + (P[14]*(P[11] + s_v)*(P[9] - ((s_v)))) + (P[14]*(P[13] + s_v)*(P[9] - ((s_v)))) + (P[19]*(P[11] + s_v)*(P[13] + s_v)));
    linear[0] = v_dI_dv;
    (void)time; (void)P; (void)PD; (void)F;
  }
};

}}  // namespace goss_b200::models
#endif
