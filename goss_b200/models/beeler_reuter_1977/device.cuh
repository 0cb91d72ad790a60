// Generated by goss_b200.codegen from the 'beeler_reuter_1977' model; do not edit.
// Device-side model: rhs and linearised rhs templated on the arithmetic type T.
#ifndef M_BEELER_REUTER_1977_DEVICE_CUH
#define M_BEELER_REUTER_1977_DEVICE_CUH
#include "goss_device_math.cuh"

namespace goss_b200 { namespace models {

struct M_beeler_reuter_1977 {
  static constexpr const char* name = "beeler_reuter_1977";
  static constexpr int num_states = 8;
  static constexpr int num_params = 10;
  static constexpr int num_field_params = 0;
  static constexpr int num_monitored = 0;
  static constexpr int num_derived = 7;
  // the reference generator's linear-term flags (RL1/RL2 use the exponential update for these)
  __host__ __device__ static constexpr bool linear_term(int i) { return i == 0 || i == 1 || i == 2 || i == 4 || i == 5 || i == 6; }

  // values = f(y, time)
  template <typename T>
  __device__ static __forceinline__ void rhs(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ values)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v_alpha_m = (((-T(47.0)) - ((s_V)))/((-T(1.0)) + gexp((-(T(0.1)*v_V_eff_0)))));
    const T v_beta_m = (T(0.7095526727489909)*gexp((-(T(0.056)*s_V))));
    const T v_alpha_h = (T(5.497962438709065e-10)*gexp((-(T(0.25)*s_V))));
    const T v_beta_h = (T(1.7)/(T(1.0) + (T(0.1580253208896478)*gexp((-(T(0.082)*s_V))))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*gexp((-(T(0.25)*s_V)))/(T(1.0) + (T(1.6788275299956603e-07)*gexp((-(T(0.2)*s_V))))));
    const T v_beta_j = (T(0.3)/(T(1.0) + (T(0.040762203978366204)*gexp((-(T(0.1)*s_V))))));
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*glog((T(0.001)*s_Cai)))));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v_alpha_d = (T(0.095)*gexp((T(0.05) - ((T(0.01)*s_V))))/(T(1.0) + (T(1.4332881385696572)*gexp((-(T(0.07199424046076314)*s_V))))));
    const T v_beta_d = (T(0.07)*gexp(((-T(0.7457627118644068)) - ((T(0.01694915254237288)*s_V))))/(T(1.0) + gexp((T(2.2) + (T(0.05)*s_V)))));
    const T v_alpha_f = (T(0.012)*gexp(((-T(0.224)) - ((T(0.008)*s_V))))/(T(1.0) + (T(66.5465065250986)*gexp((T(0.14992503748125938)*s_V)))));
    const T v_beta_f = (T(0.0065)*gexp(((-T(0.6)) - ((T(0.02)*s_V))))/(T(1.0) + gexp(((-T(6.0)) - ((T(0.2)*s_V))))));
    const T v_i_x1 = (T(0.0019727757115328517)*s_x1*((-T(1.0)) + (T(21.75840239619708)*gexp((T(0.04)*s_V))))*gexp((-(T(0.04)*s_V))));
    const T v_alpha_x1 = (T(0.031158410986342627)*gexp((T(0.08264462809917356)*s_V))/(T(1.0) + (T(17.41170806332765)*gexp((T(0.05714285714285714)*s_V)))));
    const T v_beta_x1 = (T(0.0003916464405623223)*gexp((-(T(0.05998800239952009)*s_V)))/(T(1.0) + gexp(((-T(0.8)) - ((T(0.04)*s_V))))));
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v_i_K1 = ((T(0.0035)*(T(4.6000000000000005) + (T(0.2)*s_V))/(T(1.0) - ((gexp((-(T(0.04)*v_V_eff_1))))))) + (T(0.0035)*((-T(4.0)) + (T(119.85640018958804)*gexp((T(0.04)*s_V))))/((T(8.331137487687693)*gexp((T(0.04)*s_V))) + (T(69.4078518387552)*gexp((T(0.08)*s_V))))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    values[0] = ((v_alpha_m*(T(1.0) - ((s_m)))) - ((v_beta_m*s_m)));
    values[1] = ((v_alpha_h*(T(1.0) - ((s_h)))) - ((v_beta_h*s_h)));
    values[2] = ((v_alpha_j*(T(1.0) - ((s_j)))) - ((v_beta_j*s_j)));
    values[3] = (T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s)));
    values[4] = ((v_alpha_d*(T(1.0) - ((s_d)))) - ((v_beta_d*s_d)));
    values[5] = ((v_alpha_f*(T(1.0) - ((s_f)))) - ((v_beta_f*s_f)));
    values[6] = ((v_alpha_x1*(T(1.0) - ((s_x1)))) - ((v_beta_x1*s_x1)));
    values[7] = (P[14]*(T(v_Istim) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    (void)time; (void)P; (void)PD; (void)F;
  }

  // Newton matrix: 24 packed entries (the Jacobian's 24 structural
  // non-zeros, the diagonal and the LU fill-in; row-major over the structure)
  static constexpr int lu_nnz = 24;
  static constexpr bool has_jacobian = false;
  // J := scale*J + I
  template <class A>
  __device__ static __forceinline__ void lu_shift(A J, const double scale)
  {
    for (int k = 0; k < 24; ++k) J[k] = J[k] * scale;
    J[0] = J[0] + 1.0 * 1.0;
    J[2] = J[2] + 1.0 * 1.0;
    J[4] = J[4] + 1.0 * 1.0;
    J[6] = J[6] + 1.0 * 1.0;
    J[10] = J[10] + 1.0 * 1.0;
    J[12] = J[12] + 1.0 * 1.0;
    J[14] = J[14] + 1.0 * 1.0;
    J[23] = J[23] + 1.0 * 1.0;
  }
  // D := scale*S + I
  template <class A, class B>
  __device__ static __forceinline__ void lu_copy_shift(A S, B D, const double scale)
  {
    for (int k = 0; k < 24; ++k) D[k] = S[k] * scale;
    D[0] = D[0] + 1.0 * 1.0;
    D[2] = D[2] + 1.0 * 1.0;
    D[4] = D[4] + 1.0 * 1.0;
    D[6] = D[6] + 1.0 * 1.0;
    D[10] = D[10] + 1.0 * 1.0;
    D[12] = D[12] + 1.0 * 1.0;
    D[14] = D[14] + 1.0 * 1.0;
    D[23] = D[23] + 1.0 * 1.0;
  }
  // in-place Doolittle LU without pivoting over the structure
  template <class A>
  __device__ static __forceinline__ void lu_factorize(A J)
  {
    { const double s = 0.0; J[16] = (J[16] - s) / J[0]; }
    { const double s = 0.0; J[17] = (J[17] - s) / J[2]; }
    { const double s = 0.0; J[18] = (J[18] - s) / J[4]; }
    { const double s = 0.0; J[19] = (J[19] - s) / J[6]; }
    { double s = 0.0; s = s + J[19] * J[7]; J[20] = (J[20] - s) / J[10]; }
    { double s = 0.0; s = s + J[19] * J[8]; J[21] = (J[21] - s) / J[12]; }
    { const double s = 0.0; J[22] = (J[22] - s) / J[14]; }
    { double s = 0.0; s = s + J[16] * J[1]; s = s + J[17] * J[3]; s = s + J[18] * J[5]; s = s + J[19] * J[9]; s = s + J[20] * J[11]; s = s + J[21] * J[13]; s = s + J[22] * J[15]; J[23] -= s; }
  }
  // x = (LU)^-1 b, forward then backward substitution; b and x may alias
  template <class A>
  __device__ static __forceinline__ void lu_solve(A J, const double* b, double* x)
  {
    x[0] = b[0];
    x[1] = b[1] - 0.0;
    x[2] = b[2] - 0.0;
    x[3] = b[3] - 0.0;
    x[4] = b[4] - 0.0;
    x[5] = b[5] - 0.0;
    x[6] = b[6] - 0.0;
    { double s = 0.0; s = s + J[16] * x[0]; s = s + J[17] * x[1]; s = s + J[18] * x[2]; s = s + J[19] * x[3]; s = s + J[20] * x[4]; s = s + J[21] * x[5]; s = s + J[22] * x[6]; x[7] = b[7] - s; }
    x[7] = x[7] / J[23];
    { double s = 0.0; s = s + J[15] * x[7]; x[6] = (x[6] - s) / J[14]; }
    { double s = 0.0; s = s + J[13] * x[7]; x[5] = (x[5] - s) / J[12]; }
    { double s = 0.0; s = s + J[11] * x[7]; x[4] = (x[4] - s) / J[10]; }
    { double s = 0.0; s = s + J[7] * x[4]; s = s + J[8] * x[5]; s = s + J[9] * x[7]; x[3] = (x[3] - s) / J[6]; }
    { double s = 0.0; s = s + J[5] * x[7]; x[2] = (x[2] - s) / J[4]; }
    { double s = 0.0; s = s + J[3] * x[7]; x[1] = (x[1] - s) / J[2]; }
    { double s = 0.0; s = s + J[1] * x[7]; x[0] = (x[0] - s) / J[0]; }
  }
  // forward differences: zero the entries outside the Jacobian's structure, then
  // column i = (f2 - f1) / delta at its structural rows
  template <class A>
  __device__ static __forceinline__ void fd_clear(A J)
  {
    (void)J;
  }
  template <class A>
  __device__ static __forceinline__ void fd_column(const int i, const double* f1, const double* f2,
                                                   const double delta, A J)
  {
    switch (i) {
    case 0: J[0] = (f2[0] - f1[0]) / delta; J[16] = (f2[7] - f1[7]) / delta; break;
    case 1: J[2] = (f2[1] - f1[1]) / delta; J[17] = (f2[7] - f1[7]) / delta; break;
    case 2: J[4] = (f2[2] - f1[2]) / delta; J[18] = (f2[7] - f1[7]) / delta; break;
    case 3: J[6] = (f2[3] - f1[3]) / delta; J[19] = (f2[7] - f1[7]) / delta; break;
    case 4: J[7] = (f2[3] - f1[3]) / delta; J[10] = (f2[4] - f1[4]) / delta; J[20] = (f2[7] - f1[7]) / delta; break;
    case 5: J[8] = (f2[3] - f1[3]) / delta; J[12] = (f2[5] - f1[5]) / delta; J[21] = (f2[7] - f1[7]) / delta; break;
    case 6: J[14] = (f2[6] - f1[6]) / delta; J[22] = (f2[7] - f1[7]) / delta; break;
    case 7: J[1] = (f2[0] - f1[0]) / delta; J[3] = (f2[1] - f1[1]) / delta; J[5] = (f2[2] - f1[2]) / delta; J[9] = (f2[3] - f1[3]) / delta; J[11] = (f2[4] - f1[4]) / delta; J[13] = (f2[5] - f1[5]) / delta; J[15] = (f2[6] - f1[6]) / delta; J[23] = (f2[7] - f1[7]) / delta; break;
    default: break;
    }
  }
  // dense row-major copy: out(r*n + c, value) for every entry
  template <typename T, class Out>
  __device__ static __forceinline__ void lu_unpack(const T* J, Out&& out)
  {
    out(0, J[0]);
    out(1, T(0.0));
    out(2, T(0.0));
    out(3, T(0.0));
    out(4, T(0.0));
    out(5, T(0.0));
    out(6, T(0.0));
    out(7, J[1]);
    out(8, T(0.0));
    out(9, J[2]);
    out(10, T(0.0));
    out(11, T(0.0));
    out(12, T(0.0));
    out(13, T(0.0));
    out(14, T(0.0));
    out(15, J[3]);
    out(16, T(0.0));
    out(17, T(0.0));
    out(18, J[4]);
    out(19, T(0.0));
    out(20, T(0.0));
    out(21, T(0.0));
    out(22, T(0.0));
    out(23, J[5]);
    out(24, T(0.0));
    out(25, T(0.0));
    out(26, T(0.0));
    out(27, J[6]);
    out(28, J[7]);
    out(29, J[8]);
    out(30, T(0.0));
    out(31, J[9]);
    out(32, T(0.0));
    out(33, T(0.0));
    out(34, T(0.0));
    out(35, T(0.0));
    out(36, J[10]);
    out(37, T(0.0));
    out(38, T(0.0));
    out(39, J[11]);
    out(40, T(0.0));
    out(41, T(0.0));
    out(42, T(0.0));
    out(43, T(0.0));
    out(44, T(0.0));
    out(45, J[12]);
    out(46, T(0.0));
    out(47, J[13]);
    out(48, T(0.0));
    out(49, T(0.0));
    out(50, T(0.0));
    out(51, T(0.0));
    out(52, T(0.0));
    out(53, T(0.0));
    out(54, J[14]);
    out(55, J[15]);
    out(56, J[16]);
    out(57, J[17]);
    out(58, J[18]);
    out(59, J[19]);
    out(60, J[20]);
    out(61, J[21]);
    out(62, J[22]);
    out(63, J[23]);
  }

  // derived constants: parameter-only sub-expressions, evaluated once per
  // launch on the host in FP64 and stored after the parameters
  static void derived(const double* P, double* C)
  {
    C[0] = (-(P[0]));
    C[1] = (-(P[8]));
    C[2] = (1.0/P[6]);
    C[3] = (-(P[6]));
    C[4] = (1.0/P[9]);
    C[5] = (-(P[3]));
    C[6] = (-(1.0/P[9]));
    (void)P; (void)C;
  }

  // rhs = f(y, time), linear[i] = d f_i / d y_i
  template <typename T>
  __device__ static __forceinline__ void linearized(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ linear, T* __restrict__ rhs)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v_alpha_m = (((-T(47.0)) - ((s_V)))/((-T(1.0)) + gexp((-(T(0.1)*v_V_eff_0)))));
    const T v_beta_m = (T(0.7095526727489909)*gexp((-(T(0.056)*s_V))));
    const T v_alpha_h = (T(5.497962438709065e-10)*gexp((-(T(0.25)*s_V))));
    const T v_beta_h = (T(1.7)/(T(1.0) + (T(0.1580253208896478)*gexp((-(T(0.082)*s_V))))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*gexp((-(T(0.25)*s_V)))/(T(1.0) + (T(1.6788275299956603e-07)*gexp((-(T(0.2)*s_V))))));
    const T v_beta_j = (T(0.3)/(T(1.0) + (T(0.040762203978366204)*gexp((-(T(0.1)*s_V))))));
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*glog((T(0.001)*s_Cai)))));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v_alpha_d = (T(0.095)*gexp((T(0.05) - ((T(0.01)*s_V))))/(T(1.0) + (T(1.4332881385696572)*gexp((-(T(0.07199424046076314)*s_V))))));
    const T v_beta_d = (T(0.07)*gexp(((-T(0.7457627118644068)) - ((T(0.01694915254237288)*s_V))))/(T(1.0) + gexp((T(2.2) + (T(0.05)*s_V)))));
    const T v_alpha_f = (T(0.012)*gexp(((-T(0.224)) - ((T(0.008)*s_V))))/(T(1.0) + (T(66.5465065250986)*gexp((T(0.14992503748125938)*s_V)))));
    const T v_beta_f = (T(0.0065)*gexp(((-T(0.6)) - ((T(0.02)*s_V))))/(T(1.0) + gexp(((-T(6.0)) - ((T(0.2)*s_V))))));
    const T v_i_x1 = (T(0.0019727757115328517)*s_x1*((-T(1.0)) + (T(21.75840239619708)*gexp((T(0.04)*s_V))))*gexp((-(T(0.04)*s_V))));
    const T v_alpha_x1 = (T(0.031158410986342627)*gexp((T(0.08264462809917356)*s_V))/(T(1.0) + (T(17.41170806332765)*gexp((T(0.05714285714285714)*s_V)))));
    const T v_beta_x1 = (T(0.0003916464405623223)*gexp((-(T(0.05998800239952009)*s_V)))/(T(1.0) + gexp(((-T(0.8)) - ((T(0.04)*s_V))))));
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v_i_K1 = ((T(0.0035)*(T(4.6000000000000005) + (T(0.2)*s_V))/(T(1.0) - ((gexp((-(T(0.04)*v_V_eff_1))))))) + (T(0.0035)*((-T(4.0)) + (T(119.85640018958804)*gexp((T(0.04)*s_V))))/((T(8.331137487687693)*gexp((T(0.04)*s_V))) + (T(69.4078518387552)*gexp((T(0.08)*s_V))))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    rhs[0] = ((v_alpha_m*(T(1.0) - ((s_m)))) - ((v_beta_m*s_m)));
    rhs[1] = ((v_alpha_h*(T(1.0) - ((s_h)))) - ((v_beta_h*s_h)));
    rhs[2] = ((v_alpha_j*(T(1.0) - ((s_j)))) - ((v_beta_j*s_j)));
    rhs[3] = (T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s)));
    rhs[4] = ((v_alpha_d*(T(1.0) - ((s_d)))) - ((v_beta_d*s_d)));
    rhs[5] = ((v_alpha_f*(T(1.0) - ((s_f)))) - ((v_beta_f*s_f)));
    rhs[6] = ((v_alpha_x1*(T(1.0) - ((s_x1)))) - ((v_beta_x1*s_x1)));
    rhs[7] = (P[14]*(T(v_Istim) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    linear[0] = ((-(v_alpha_m)) - ((v_beta_m)));
    linear[1] = ((-(v_alpha_h)) - ((v_beta_h)));
    linear[2] = ((-(v_alpha_j)) - ((v_beta_j)));
    linear[4] = ((-(v_alpha_d)) - ((v_beta_d)));
    linear[5] = ((-(v_alpha_f)) - ((v_beta_f)));
    linear[6] = ((-(v_alpha_x1)) - ((v_beta_x1)));
    const T v_dE_s_dCai = (-(T(13.0287)/s_Cai));
    const T v_di_s_dCai = (P[15]*s_d*v_dE_s_dCai*s_f);
    const T v_dV_eff_1_dV = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.0) : T(1.0));
    const T v_di_K1_dV = ((T(0.0007000000000000001)/(T(1.0) - ((gexp((-(T(0.04)*v_V_eff_1))))))) + (T(0.016779896026542326)*gexp((T(0.04)*s_V))/((T(8.331137487687693)*gexp((T(0.04)*s_V))) + (T(69.4078518387552)*gexp((T(0.08)*s_V))))) + (T(0.0035)*((-T(4.0)) + (T(119.85640018958804)*gexp((T(0.04)*s_V))))*((-(T(0.3332454995075077)*gexp((T(0.04)*s_V)))) - ((T(5.552628147100417)*gexp((T(0.08)*s_V)))))/(((T(8.331137487687693)*gexp((T(0.04)*s_V))) + (T(69.4078518387552)*gexp((T(0.08)*s_V))))*((T(8.331137487687693)*gexp((T(0.04)*s_V))) + (T(69.4078518387552)*gexp((T(0.08)*s_V)))))) - ((T(0.00028000000000000003)*v_dV_eff_1_dV*(T(4.6000000000000005) + (T(0.2)*s_V))*gexp((-(T(0.04)*v_V_eff_1)))/((T(1.0) - ((gexp((-(T(0.04)*v_V_eff_1))))))*(T(1.0) - ((gexp((-(T(0.04)*v_V_eff_1))))))))));
    const T v_di_Na_dV = (P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m)));
    const T v_di_s_dV = (s_d*s_f*P[3]);
    const T v_di_x1_dV = ((T(0.0017169779107590322)*s_x1) - ((T(7.891102846131407e-05)*s_x1*((-T(1.0)) + (T(21.75840239619708)*gexp((T(0.04)*s_V))))*gexp((-(T(0.04)*s_V))))));
    linear[3] = ((-T(0.07)) - ((T(0.01)*v_di_s_dCai)));
    linear[7] = ((P[16]*v_di_K1_dV) + (P[16]*v_di_Na_dV) + (P[16]*v_di_s_dV) + (P[16]*v_di_x1_dV));
    (void)time; (void)P; (void)PD; (void)F;
  }

  // linearized with every distinct transcendental and reciprocal of a state-dependent
  // operand evaluated once (the FP32 kernels' form; FP64 keeps the reference's operations)
  template <typename T>
  __device__ static __forceinline__ void linearized_split(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ linear, T* __restrict__ rhs)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v___t0 = gexp2((-T(0.14426950408889636))*v_V_eff_0);
    const T v___t1 = (T(1.0)/((-T(1.0)) + v___t0));
    const T v_alpha_m = (v___t1*((-T(47.0)) - ((s_V))));
    const T v___t2 = gexp2((-T(0.08079092228978195))*s_V);
    const T v_beta_m = (T(0.7095526727489909)*v___t2);
    const T v___t3 = gexp2((-T(0.36067376022224085))*s_V);
    const T v_alpha_h = (T(5.497962438709065e-10)*v___t3);
    const T v___t4 = gexp2((-T(0.118300993352895))*s_V);
    const T v___t5 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4)));
    const T v_beta_h = (T(1.7)*v___t5);
    const T v___t6 = gexp2((-T(0.14426950408889636))*s_V);
    const T v___t7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6*v___t6))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*v___t3*v___t7);
    const T v___t8 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6)));
    const T v_beta_j = (T(0.3)*v___t8);
    const T v___t9 = glog((T(0.001)*s_Cai));
    const T v___t10 = (T(1.0)/s_Cai);
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*v___t9)));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v___t11 = gexp2((-T(0.10386573368531053))*s_V);
    const T v___t12 = gexp2((-T(0.014426950408889635))*s_V);
    const T v___t13 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11)));
    const T v_alpha_d = (T(0.09987075415572229)*v___t12*v___t13);
    const T v___t14 = gexp2(T(0.07213475204444818)*s_V);
    const T v___t15 = gexp2((-T(0.024452458320151922))*s_V);
    const T v___t16 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14)));
    const T v_beta_d = (T(0.03320606467536786)*v___t15*v___t16);
    const T v___t17 = gexp2(T(0.21629610807930486)*s_V);
    const T v___t18 = gexp2((-T(0.011541560327111707))*s_V);
    const T v___t19 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17)));
    const T v_alpha_f = (T(0.009591781612432381)*v___t18*v___t19);
    const T v___t20 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6*v___t6))));
    const T v_beta_f = (T(0.0035672756346111717)*v___t20*(v___t12*v___t12));
    const T v___t21 = gexp2(T(0.05770780163555854)*s_V);
    const T v___t22 = gexp2((-T(0.05770780163555854))*s_V);
    const T v_i_x1 = (T(0.0019727757115328517)*v___t22*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
    const T v___t23 = gexp2(T(0.08243971662222647)*s_V);
    const T v___t24 = gexp2(T(0.11923099511479036)*s_V);
    const T v___t25 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23)));
    const T v_alpha_x1 = (T(0.031158410986342627)*v___t24*v___t25);
    const T v___t26 = gexp2((-T(0.08654439357462287))*s_V);
    const T v___t27 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22)));
    const T v_beta_x1 = (T(0.0003916464405623223)*v___t26*v___t27);
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v___t28 = gexp2((-T(0.05770780163555854))*v_V_eff_1);
    const T v___t29 = (T(1.0)/(T(1.0) - ((v___t28))));
    const T v___t30 = (T(1.0)/(v___t21*(T(8.331137487687693) + (T(69.4078518387552)*v___t21))));
    const T v_i_K1 = (T(0.0035)*((v___t29*(T(4.6000000000000005) + (T(0.2)*s_V))) + (v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21)))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    const T v_dE_s_dCai = (-(T(13.0287)*v___t10));
    const T v_di_s_dCai = (P[15]*s_d*v_dE_s_dCai*s_f);
    const T v_dV_eff_1_dV = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.0) : T(1.0));
    const T v_di_K1_dV = ((v___t30*(v___t21*(T(0.016779896026542326) + (T(0.0035)*v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21))*((-T(0.3332454995075077)) - ((T(5.552628147100417)*v___t21))))))) + (v___t29*(T(0.0007000000000000001) - ((T(0.00028000000000000003)*v___t28*v___t29*v_dV_eff_1_dV*(T(4.6000000000000005) + (T(0.2)*s_V)))))));
    const T v_di_Na_dV = (P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m)));
    const T v_di_s_dV = (s_d*s_f*P[3]);
    const T v_di_x1_dV = (s_x1*(T(0.0017169779107590322) - ((T(7.891102846131407e-05)*v___t22*((-T(1.0)) + (T(21.75840239619708)*v___t21))))));
    rhs[0] = ((v_alpha_m*(T(1.0) - ((s_m)))) - ((v_beta_m*s_m)));
    rhs[1] = ((v_alpha_h*(T(1.0) - ((s_h)))) - ((v_beta_h*s_h)));
    rhs[2] = ((v_alpha_j*(T(1.0) - ((s_j)))) - ((v_beta_j*s_j)));
    rhs[3] = (T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s)));
    rhs[4] = ((v_alpha_d*(T(1.0) - ((s_d)))) - ((v_beta_d*s_d)));
    rhs[5] = ((v_alpha_f*(T(1.0) - ((s_f)))) - ((v_beta_f*s_f)));
    rhs[6] = ((v_alpha_x1*(T(1.0) - ((s_x1)))) - ((v_beta_x1*s_x1)));
    rhs[7] = (P[14]*(T(v_Istim) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    linear[0] = ((-(v_alpha_m)) - ((v_beta_m)));
    linear[1] = ((-(v_alpha_h)) - ((v_beta_h)));
    linear[2] = ((-(v_alpha_j)) - ((v_beta_j)));
    linear[4] = ((-(v_alpha_d)) - ((v_beta_d)));
    linear[5] = ((-(v_alpha_f)) - ((v_beta_f)));
    linear[6] = ((-(v_alpha_x1)) - ((v_beta_x1)));
    linear[3] = ((-T(0.07)) - ((T(0.01)*v_di_s_dCai)));
    linear[7] = (P[16]*(v_di_K1_dV + v_di_Na_dV + v_di_s_dV + v_di_x1_dV));
    (void)time; (void)P; (void)PD; (void)F;
  }

  // rhs in the same split form
  template <typename T>
  __device__ static __forceinline__ void rhs_split(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ values)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v___t0 = gexp2((-T(0.14426950408889636))*v_V_eff_0);
    const T v___t1 = (T(1.0)/((-T(1.0)) + v___t0));
    const T v_alpha_m = (v___t1*((-T(47.0)) - ((s_V))));
    const T v___t2 = gexp2((-T(0.08079092228978195))*s_V);
    const T v_beta_m = (T(0.7095526727489909)*v___t2);
    const T v___t3 = gexp2((-T(0.36067376022224085))*s_V);
    const T v_alpha_h = (T(5.497962438709065e-10)*v___t3);
    const T v___t4 = gexp2((-T(0.118300993352895))*s_V);
    const T v___t5 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4)));
    const T v_beta_h = (T(1.7)*v___t5);
    const T v___t6 = gexp2((-T(0.14426950408889636))*s_V);
    const T v___t7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6*v___t6))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*v___t3*v___t7);
    const T v___t8 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6)));
    const T v_beta_j = (T(0.3)*v___t8);
    const T v___t9 = glog((T(0.001)*s_Cai));
    const T v___t10 = (T(1.0)/s_Cai);
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*v___t9)));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v___t11 = gexp2((-T(0.10386573368531053))*s_V);
    const T v___t12 = gexp2((-T(0.014426950408889635))*s_V);
    const T v___t13 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11)));
    const T v_alpha_d = (T(0.09987075415572229)*v___t12*v___t13);
    const T v___t14 = gexp2(T(0.07213475204444818)*s_V);
    const T v___t15 = gexp2((-T(0.024452458320151922))*s_V);
    const T v___t16 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14)));
    const T v_beta_d = (T(0.03320606467536786)*v___t15*v___t16);
    const T v___t17 = gexp2(T(0.21629610807930486)*s_V);
    const T v___t18 = gexp2((-T(0.011541560327111707))*s_V);
    const T v___t19 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17)));
    const T v_alpha_f = (T(0.009591781612432381)*v___t18*v___t19);
    const T v___t20 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6*v___t6))));
    const T v_beta_f = (T(0.0035672756346111717)*v___t20*(v___t12*v___t12));
    const T v___t21 = gexp2(T(0.05770780163555854)*s_V);
    const T v___t22 = gexp2((-T(0.05770780163555854))*s_V);
    const T v_i_x1 = (T(0.0019727757115328517)*v___t22*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
    const T v___t23 = gexp2(T(0.08243971662222647)*s_V);
    const T v___t24 = gexp2(T(0.11923099511479036)*s_V);
    const T v___t25 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23)));
    const T v_alpha_x1 = (T(0.031158410986342627)*v___t24*v___t25);
    const T v___t26 = gexp2((-T(0.08654439357462287))*s_V);
    const T v___t27 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22)));
    const T v_beta_x1 = (T(0.0003916464405623223)*v___t26*v___t27);
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v___t28 = gexp2((-T(0.05770780163555854))*v_V_eff_1);
    const T v___t29 = (T(1.0)/(T(1.0) - ((v___t28))));
    const T v___t30 = (T(1.0)/(v___t21*(T(8.331137487687693) + (T(69.4078518387552)*v___t21))));
    const T v_i_K1 = (T(0.0035)*((v___t29*(T(4.6000000000000005) + (T(0.2)*s_V))) + (v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21)))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    values[0] = ((v_alpha_m*(T(1.0) - ((s_m)))) - ((v_beta_m*s_m)));
    values[1] = ((v_alpha_h*(T(1.0) - ((s_h)))) - ((v_beta_h*s_h)));
    values[2] = ((v_alpha_j*(T(1.0) - ((s_j)))) - ((v_beta_j*s_j)));
    values[3] = (T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s)));
    values[4] = ((v_alpha_d*(T(1.0) - ((s_d)))) - ((v_beta_d*s_d)));
    values[5] = ((v_alpha_f*(T(1.0) - ((s_f)))) - ((v_beta_f*s_f)));
    values[6] = ((v_alpha_x1*(T(1.0) - ((s_x1)))) - ((v_beta_x1*s_x1)));
    values[7] = (P[14]*(T(v_Istim) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    (void)time; (void)P; (void)PD; (void)F;
  }

  // forward-difference Jacobian of rhs_split at y into the packed Newton matrix (structural
  // entries; fd_clear sets the others): f1 = f(y, time); column i recomputes only the
  // statements of its rows that depend on state i
  template <typename T, class A>
  __device__ static __forceinline__ void fd_jacobian(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, const T* __restrict__ f1, A J)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v___t0 = gexp2((-T(0.14426950408889636))*v_V_eff_0);
    const T v___t1 = (T(1.0)/((-T(1.0)) + v___t0));
    const T v_alpha_m = (v___t1*((-T(47.0)) - ((s_V))));
    const T v___t2 = gexp2((-T(0.08079092228978195))*s_V);
    const T v_beta_m = (T(0.7095526727489909)*v___t2);
    const T v___t3 = gexp2((-T(0.36067376022224085))*s_V);
    const T v_alpha_h = (T(5.497962438709065e-10)*v___t3);
    const T v___t4 = gexp2((-T(0.118300993352895))*s_V);
    const T v___t5 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4)));
    const T v_beta_h = (T(1.7)*v___t5);
    const T v___t6 = gexp2((-T(0.14426950408889636))*s_V);
    const T v___t7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6*v___t6))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*v___t3*v___t7);
    const T v___t8 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6)));
    const T v_beta_j = (T(0.3)*v___t8);
    const T v___t9 = glog((T(0.001)*s_Cai));
    const T v___t10 = (T(1.0)/s_Cai);
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*v___t9)));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v___t11 = gexp2((-T(0.10386573368531053))*s_V);
    const T v___t12 = gexp2((-T(0.014426950408889635))*s_V);
    const T v___t13 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11)));
    const T v_alpha_d = (T(0.09987075415572229)*v___t12*v___t13);
    const T v___t14 = gexp2(T(0.07213475204444818)*s_V);
    const T v___t15 = gexp2((-T(0.024452458320151922))*s_V);
    const T v___t16 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14)));
    const T v_beta_d = (T(0.03320606467536786)*v___t15*v___t16);
    const T v___t17 = gexp2(T(0.21629610807930486)*s_V);
    const T v___t18 = gexp2((-T(0.011541560327111707))*s_V);
    const T v___t19 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17)));
    const T v_alpha_f = (T(0.009591781612432381)*v___t18*v___t19);
    const T v___t20 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6*v___t6))));
    const T v_beta_f = (T(0.0035672756346111717)*v___t20*(v___t12*v___t12));
    const T v___t21 = gexp2(T(0.05770780163555854)*s_V);
    const T v___t22 = gexp2((-T(0.05770780163555854))*s_V);
    const T v_i_x1 = (T(0.0019727757115328517)*v___t22*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
    const T v___t23 = gexp2(T(0.08243971662222647)*s_V);
    const T v___t24 = gexp2(T(0.11923099511479036)*s_V);
    const T v___t25 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23)));
    const T v_alpha_x1 = (T(0.031158410986342627)*v___t24*v___t25);
    const T v___t26 = gexp2((-T(0.08654439357462287))*s_V);
    const T v___t27 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22)));
    const T v_beta_x1 = (T(0.0003916464405623223)*v___t26*v___t27);
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v___t28 = gexp2((-T(0.05770780163555854))*v_V_eff_1);
    const T v___t29 = (T(1.0)/(T(1.0) - ((v___t28))));
    const T v___t30 = (T(1.0)/(v___t21*(T(8.331137487687693) + (T(69.4078518387552)*v___t21))));
    const T v_i_K1 = (T(0.0035)*((v___t29*(T(4.6000000000000005) + (T(0.2)*s_V))) + (v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21)))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[0])) ? 1e-5 : fabs(double(y[0]))));
      const T v___yp0 = T(double(y[0]) + d);
      const T v_i_Na__k0 = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(v___yp0*v___yp0*v___yp0))));
      J[0] = ((((v_alpha_m*(T(1.0) - ((v___yp0)))) - ((v___yp0*v_beta_m)))) - f1[0]) / d;
      J[16] = (((P[14]*(T(v_Istim) - ((v_i_Na__k0)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[1])) ? 1e-5 : fabs(double(y[1]))));
      const T v___yp1 = T(double(y[1]) + d);
      const T v_i_Na__k1 = ((s_V + P[10])*(P[2] + (v___yp1*P[1]*s_j*(s_m*s_m*s_m))));
      J[2] = ((((v_alpha_h*(T(1.0) - ((v___yp1)))) - ((v___yp1*v_beta_h)))) - f1[1]) / d;
      J[17] = (((P[14]*(T(v_Istim) - ((v_i_Na__k1)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[2])) ? 1e-5 : fabs(double(y[2]))));
      const T v___yp2 = T(double(y[2]) + d);
      const T v_i_Na__k2 = ((s_V + P[10])*(P[2] + (v___yp2*P[1]*s_h*(s_m*s_m*s_m))));
      J[4] = ((((v_alpha_j*(T(1.0) - ((v___yp2)))) - ((v___yp2*v_beta_j)))) - f1[2]) / d;
      J[18] = (((P[14]*(T(v_Istim) - ((v_i_Na__k2)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[3])) ? 1e-5 : fabs(double(y[3]))));
      const T v___yp3 = T(double(y[3]) + d);
      const T v___t9__k3 = glog((T(0.001)*v___yp3));
      const T v_E_s__k3 = ((-T(82.3)) - ((T(13.0287)*v___t9__k3)));
      const T v_i_s__k3 = (s_d*s_f*P[3]*(s_V - ((v_E_s__k3))));
      J[6] = (((T(7.000000000000001e-06) - ((T(0.07)*v___yp3)) - ((T(0.01)*v_i_s__k3)))) - f1[3]) / d;
      J[19] = (((P[14]*(T(v_Istim) - ((v_i_s__k3)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[4])) ? 1e-5 : fabs(double(y[4]))));
      const T v___yp4 = T(double(y[4]) + d);
      const T v_i_s__k4 = (v___yp4*s_f*P[3]*(s_V - ((v_E_s))));
      J[7] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k4)))) - f1[3]) / d;
      J[10] = ((((v_alpha_d*(T(1.0) - ((v___yp4)))) - ((v___yp4*v_beta_d)))) - f1[4]) / d;
      J[20] = (((P[14]*(T(v_Istim) - ((v_i_s__k4)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[5])) ? 1e-5 : fabs(double(y[5]))));
      const T v___yp5 = T(double(y[5]) + d);
      const T v_i_s__k5 = (v___yp5*s_d*P[3]*(s_V - ((v_E_s))));
      J[8] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k5)))) - f1[3]) / d;
      J[12] = ((((v_alpha_f*(T(1.0) - ((v___yp5)))) - ((v___yp5*v_beta_f)))) - f1[5]) / d;
      J[21] = (((P[14]*(T(v_Istim) - ((v_i_s__k5)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[6])) ? 1e-5 : fabs(double(y[6]))));
      const T v___yp6 = T(double(y[6]) + d);
      const T v_i_x1__k6 = (T(0.0019727757115328517)*v___yp6*v___t22*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
      J[14] = ((((v_alpha_x1*(T(1.0) - ((v___yp6)))) - ((v___yp6*v_beta_x1)))) - f1[6]) / d;
      J[22] = (((P[14]*(T(v_Istim) - ((v_i_x1__k6)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[7])) ? 1e-5 : fabs(double(y[7]))));
      const T v___yp7 = T(double(y[7]) + d);
      const T v_i_Na__k7 = ((v___yp7 + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
      const T v_V_eff_0__k7 = ((gfabs((T(47.0) + v___yp7)) < T(0.01)) ? T(0.01) : (T(47.0) + v___yp7));
      const T v___t0__k7 = gexp2((-T(0.14426950408889636))*v_V_eff_0__k7);
      const T v___t1__k7 = (T(1.0)/((-T(1.0)) + v___t0__k7));
      const T v_alpha_m__k7 = (v___t1__k7*((-T(47.0)) - ((v___yp7))));
      const T v___t2__k7 = gexp2((-T(0.08079092228978195))*v___yp7);
      const T v_beta_m__k7 = (T(0.7095526727489909)*v___t2__k7);
      const T v___t3__k7 = gexp2((-T(0.36067376022224085))*v___yp7);
      const T v_alpha_h__k7 = (T(5.497962438709065e-10)*v___t3__k7);
      const T v___t4__k7 = gexp2((-T(0.118300993352895))*v___yp7);
      const T v___t5__k7 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4__k7)));
      const T v_beta_h__k7 = (T(1.7)*v___t5__k7);
      const T v___t6__k7 = gexp2((-T(0.14426950408889636))*v___yp7);
      const T v___t7__k7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6__k7*v___t6__k7))));
      const T v_alpha_j__k7 = (T(1.8690473007222892e-10)*v___t3__k7*v___t7__k7);
      const T v___t8__k7 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6__k7)));
      const T v_beta_j__k7 = (T(0.3)*v___t8__k7);
      const T v_i_s__k7 = (s_d*s_f*P[3]*(v___yp7 - ((v_E_s))));
      const T v___t11__k7 = gexp2((-T(0.10386573368531053))*v___yp7);
      const T v___t12__k7 = gexp2((-T(0.014426950408889635))*v___yp7);
      const T v___t13__k7 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11__k7)));
      const T v_alpha_d__k7 = (T(0.09987075415572229)*v___t12__k7*v___t13__k7);
      const T v___t14__k7 = gexp2(T(0.07213475204444818)*v___yp7);
      const T v___t15__k7 = gexp2((-T(0.024452458320151922))*v___yp7);
      const T v___t16__k7 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14__k7)));
      const T v_beta_d__k7 = (T(0.03320606467536786)*v___t15__k7*v___t16__k7);
      const T v___t17__k7 = gexp2(T(0.21629610807930486)*v___yp7);
      const T v___t18__k7 = gexp2((-T(0.011541560327111707))*v___yp7);
      const T v___t19__k7 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17__k7)));
      const T v_alpha_f__k7 = (T(0.009591781612432381)*v___t18__k7*v___t19__k7);
      const T v___t20__k7 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6__k7*v___t6__k7))));
      const T v_beta_f__k7 = (T(0.0035672756346111717)*v___t20__k7*(v___t12__k7*v___t12__k7));
      const T v___t21__k7 = gexp2(T(0.05770780163555854)*v___yp7);
      const T v___t22__k7 = gexp2((-T(0.05770780163555854))*v___yp7);
      const T v_i_x1__k7 = (T(0.0019727757115328517)*v___t22__k7*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21__k7)));
      const T v___t23__k7 = gexp2(T(0.08243971662222647)*v___yp7);
      const T v___t24__k7 = gexp2(T(0.11923099511479036)*v___yp7);
      const T v___t25__k7 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23__k7)));
      const T v_alpha_x1__k7 = (T(0.031158410986342627)*v___t24__k7*v___t25__k7);
      const T v___t26__k7 = gexp2((-T(0.08654439357462287))*v___yp7);
      const T v___t27__k7 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22__k7)));
      const T v_beta_x1__k7 = (T(0.0003916464405623223)*v___t26__k7*v___t27__k7);
      const T v_V_eff_1__k7 = ((gfabs((T(23.0) + v___yp7)) < T(0.01)) ? T(0.01) : (T(23.0) + v___yp7));
      const T v___t28__k7 = gexp2((-T(0.05770780163555854))*v_V_eff_1__k7);
      const T v___t29__k7 = (T(1.0)/(T(1.0) - ((v___t28__k7))));
      const T v___t30__k7 = (T(1.0)/(v___t21__k7*(T(8.331137487687693) + (T(69.4078518387552)*v___t21__k7))));
      const T v_i_K1__k7 = (T(0.0035)*((v___t29__k7*(T(4.6000000000000005) + (T(0.2)*v___yp7))) + (v___t30__k7*((-T(4.0)) + (T(119.85640018958804)*v___t21__k7)))));
      J[1] = ((((v_alpha_m__k7*(T(1.0) - ((s_m)))) - ((v_beta_m__k7*s_m)))) - f1[0]) / d;
      J[3] = ((((v_alpha_h__k7*(T(1.0) - ((s_h)))) - ((v_beta_h__k7*s_h)))) - f1[1]) / d;
      J[5] = ((((v_alpha_j__k7*(T(1.0) - ((s_j)))) - ((v_beta_j__k7*s_j)))) - f1[2]) / d;
      J[9] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k7)))) - f1[3]) / d;
      J[11] = ((((v_alpha_d__k7*(T(1.0) - ((s_d)))) - ((v_beta_d__k7*s_d)))) - f1[4]) / d;
      J[13] = ((((v_alpha_f__k7*(T(1.0) - ((s_f)))) - ((v_beta_f__k7*s_f)))) - f1[5]) / d;
      J[15] = ((((v_alpha_x1__k7*(T(1.0) - ((s_x1)))) - ((v_beta_x1__k7*s_x1)))) - f1[6]) / d;
      J[23] = (((P[14]*(T(v_Istim) - ((v_i_K1__k7)) - ((v_i_Na__k7)) - ((v_i_s__k7)) - ((v_i_x1__k7))))) - f1[7]) / d;
    }
    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;
  }

  // the same, also writing f1 = f(y, time) (rhs_split) from its unperturbed statements
  template <typename T, class A>
  __device__ static __forceinline__ void rhs_fd_jacobian(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ f1, A J)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v___t0 = gexp2((-T(0.14426950408889636))*v_V_eff_0);
    const T v___t1 = (T(1.0)/((-T(1.0)) + v___t0));
    const T v_alpha_m = (v___t1*((-T(47.0)) - ((s_V))));
    const T v___t2 = gexp2((-T(0.08079092228978195))*s_V);
    const T v_beta_m = (T(0.7095526727489909)*v___t2);
    const T v___t3 = gexp2((-T(0.36067376022224085))*s_V);
    const T v_alpha_h = (T(5.497962438709065e-10)*v___t3);
    const T v___t4 = gexp2((-T(0.118300993352895))*s_V);
    const T v___t5 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4)));
    const T v_beta_h = (T(1.7)*v___t5);
    const T v___t6 = gexp2((-T(0.14426950408889636))*s_V);
    const T v___t7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6*v___t6))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*v___t3*v___t7);
    const T v___t8 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6)));
    const T v_beta_j = (T(0.3)*v___t8);
    const T v___t9 = glog((T(0.001)*s_Cai));
    const T v___t10 = (T(1.0)/s_Cai);
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*v___t9)));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v___t11 = gexp2((-T(0.10386573368531053))*s_V);
    const T v___t12 = gexp2((-T(0.014426950408889635))*s_V);
    const T v___t13 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11)));
    const T v_alpha_d = (T(0.09987075415572229)*v___t12*v___t13);
    const T v___t14 = gexp2(T(0.07213475204444818)*s_V);
    const T v___t15 = gexp2((-T(0.024452458320151922))*s_V);
    const T v___t16 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14)));
    const T v_beta_d = (T(0.03320606467536786)*v___t15*v___t16);
    const T v___t17 = gexp2(T(0.21629610807930486)*s_V);
    const T v___t18 = gexp2((-T(0.011541560327111707))*s_V);
    const T v___t19 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17)));
    const T v_alpha_f = (T(0.009591781612432381)*v___t18*v___t19);
    const T v___t20 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6*v___t6))));
    const T v_beta_f = (T(0.0035672756346111717)*v___t20*(v___t12*v___t12));
    const T v___t21 = gexp2(T(0.05770780163555854)*s_V);
    const T v___t22 = gexp2((-T(0.05770780163555854))*s_V);
    const T v_i_x1 = (T(0.0019727757115328517)*v___t22*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
    const T v___t23 = gexp2(T(0.08243971662222647)*s_V);
    const T v___t24 = gexp2(T(0.11923099511479036)*s_V);
    const T v___t25 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23)));
    const T v_alpha_x1 = (T(0.031158410986342627)*v___t24*v___t25);
    const T v___t26 = gexp2((-T(0.08654439357462287))*s_V);
    const T v___t27 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22)));
    const T v_beta_x1 = (T(0.0003916464405623223)*v___t26*v___t27);
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v___t28 = gexp2((-T(0.05770780163555854))*v_V_eff_1);
    const T v___t29 = (T(1.0)/(T(1.0) - ((v___t28))));
    const T v___t30 = (T(1.0)/(v___t21*(T(8.331137487687693) + (T(69.4078518387552)*v___t21))));
    const T v_i_K1 = (T(0.0035)*((v___t29*(T(4.6000000000000005) + (T(0.2)*s_V))) + (v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21)))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    f1[0] = ((v_alpha_m*(T(1.0) - ((s_m)))) - ((v_beta_m*s_m)));
    f1[1] = ((v_alpha_h*(T(1.0) - ((s_h)))) - ((v_beta_h*s_h)));
    f1[2] = ((v_alpha_j*(T(1.0) - ((s_j)))) - ((v_beta_j*s_j)));
    f1[3] = (T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s)));
    f1[4] = ((v_alpha_d*(T(1.0) - ((s_d)))) - ((v_beta_d*s_d)));
    f1[5] = ((v_alpha_f*(T(1.0) - ((s_f)))) - ((v_beta_f*s_f)));
    f1[6] = ((v_alpha_x1*(T(1.0) - ((s_x1)))) - ((v_beta_x1*s_x1)));
    f1[7] = (P[14]*(T(v_Istim) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[0])) ? 1e-5 : fabs(double(y[0]))));
      const T v___yp0 = T(double(y[0]) + d);
      const T v_i_Na__k0 = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(v___yp0*v___yp0*v___yp0))));
      J[0] = ((((v_alpha_m*(T(1.0) - ((v___yp0)))) - ((v___yp0*v_beta_m)))) - f1[0]) / d;
      J[16] = (((P[14]*(T(v_Istim) - ((v_i_Na__k0)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[1])) ? 1e-5 : fabs(double(y[1]))));
      const T v___yp1 = T(double(y[1]) + d);
      const T v_i_Na__k1 = ((s_V + P[10])*(P[2] + (v___yp1*P[1]*s_j*(s_m*s_m*s_m))));
      J[2] = ((((v_alpha_h*(T(1.0) - ((v___yp1)))) - ((v___yp1*v_beta_h)))) - f1[1]) / d;
      J[17] = (((P[14]*(T(v_Istim) - ((v_i_Na__k1)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[2])) ? 1e-5 : fabs(double(y[2]))));
      const T v___yp2 = T(double(y[2]) + d);
      const T v_i_Na__k2 = ((s_V + P[10])*(P[2] + (v___yp2*P[1]*s_h*(s_m*s_m*s_m))));
      J[4] = ((((v_alpha_j*(T(1.0) - ((v___yp2)))) - ((v___yp2*v_beta_j)))) - f1[2]) / d;
      J[18] = (((P[14]*(T(v_Istim) - ((v_i_Na__k2)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[3])) ? 1e-5 : fabs(double(y[3]))));
      const T v___yp3 = T(double(y[3]) + d);
      const T v___t9__k3 = glog((T(0.001)*v___yp3));
      const T v_E_s__k3 = ((-T(82.3)) - ((T(13.0287)*v___t9__k3)));
      const T v_i_s__k3 = (s_d*s_f*P[3]*(s_V - ((v_E_s__k3))));
      J[6] = (((T(7.000000000000001e-06) - ((T(0.07)*v___yp3)) - ((T(0.01)*v_i_s__k3)))) - f1[3]) / d;
      J[19] = (((P[14]*(T(v_Istim) - ((v_i_s__k3)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[4])) ? 1e-5 : fabs(double(y[4]))));
      const T v___yp4 = T(double(y[4]) + d);
      const T v_i_s__k4 = (v___yp4*s_f*P[3]*(s_V - ((v_E_s))));
      J[7] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k4)))) - f1[3]) / d;
      J[10] = ((((v_alpha_d*(T(1.0) - ((v___yp4)))) - ((v___yp4*v_beta_d)))) - f1[4]) / d;
      J[20] = (((P[14]*(T(v_Istim) - ((v_i_s__k4)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[5])) ? 1e-5 : fabs(double(y[5]))));
      const T v___yp5 = T(double(y[5]) + d);
      const T v_i_s__k5 = (v___yp5*s_d*P[3]*(s_V - ((v_E_s))));
      J[8] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k5)))) - f1[3]) / d;
      J[12] = ((((v_alpha_f*(T(1.0) - ((v___yp5)))) - ((v___yp5*v_beta_f)))) - f1[5]) / d;
      J[21] = (((P[14]*(T(v_Istim) - ((v_i_s__k5)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[6])) ? 1e-5 : fabs(double(y[6]))));
      const T v___yp6 = T(double(y[6]) + d);
      const T v_i_x1__k6 = (T(0.0019727757115328517)*v___yp6*v___t22*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
      J[14] = ((((v_alpha_x1*(T(1.0) - ((v___yp6)))) - ((v___yp6*v_beta_x1)))) - f1[6]) / d;
      J[22] = (((P[14]*(T(v_Istim) - ((v_i_x1__k6)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[7])) ? 1e-5 : fabs(double(y[7]))));
      const T v___yp7 = T(double(y[7]) + d);
      const T v_i_Na__k7 = ((v___yp7 + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
      const T v_V_eff_0__k7 = ((gfabs((T(47.0) + v___yp7)) < T(0.01)) ? T(0.01) : (T(47.0) + v___yp7));
      const T v___t0__k7 = gexp2((-T(0.14426950408889636))*v_V_eff_0__k7);
      const T v___t1__k7 = (T(1.0)/((-T(1.0)) + v___t0__k7));
      const T v_alpha_m__k7 = (v___t1__k7*((-T(47.0)) - ((v___yp7))));
      const T v___t2__k7 = gexp2((-T(0.08079092228978195))*v___yp7);
      const T v_beta_m__k7 = (T(0.7095526727489909)*v___t2__k7);
      const T v___t3__k7 = gexp2((-T(0.36067376022224085))*v___yp7);
      const T v_alpha_h__k7 = (T(5.497962438709065e-10)*v___t3__k7);
      const T v___t4__k7 = gexp2((-T(0.118300993352895))*v___yp7);
      const T v___t5__k7 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4__k7)));
      const T v_beta_h__k7 = (T(1.7)*v___t5__k7);
      const T v___t6__k7 = gexp2((-T(0.14426950408889636))*v___yp7);
      const T v___t7__k7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6__k7*v___t6__k7))));
      const T v_alpha_j__k7 = (T(1.8690473007222892e-10)*v___t3__k7*v___t7__k7);
      const T v___t8__k7 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6__k7)));
      const T v_beta_j__k7 = (T(0.3)*v___t8__k7);
      const T v_i_s__k7 = (s_d*s_f*P[3]*(v___yp7 - ((v_E_s))));
      const T v___t11__k7 = gexp2((-T(0.10386573368531053))*v___yp7);
      const T v___t12__k7 = gexp2((-T(0.014426950408889635))*v___yp7);
      const T v___t13__k7 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11__k7)));
      const T v_alpha_d__k7 = (T(0.09987075415572229)*v___t12__k7*v___t13__k7);
      const T v___t14__k7 = gexp2(T(0.07213475204444818)*v___yp7);
      const T v___t15__k7 = gexp2((-T(0.024452458320151922))*v___yp7);
      const T v___t16__k7 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14__k7)));
      const T v_beta_d__k7 = (T(0.03320606467536786)*v___t15__k7*v___t16__k7);
      const T v___t17__k7 = gexp2(T(0.21629610807930486)*v___yp7);
      const T v___t18__k7 = gexp2((-T(0.011541560327111707))*v___yp7);
      const T v___t19__k7 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17__k7)));
      const T v_alpha_f__k7 = (T(0.009591781612432381)*v___t18__k7*v___t19__k7);
      const T v___t20__k7 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6__k7*v___t6__k7))));
      const T v_beta_f__k7 = (T(0.0035672756346111717)*v___t20__k7*(v___t12__k7*v___t12__k7));
      const T v___t21__k7 = gexp2(T(0.05770780163555854)*v___yp7);
      const T v___t22__k7 = gexp2((-T(0.05770780163555854))*v___yp7);
      const T v_i_x1__k7 = (T(0.0019727757115328517)*v___t22__k7*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21__k7)));
      const T v___t23__k7 = gexp2(T(0.08243971662222647)*v___yp7);
      const T v___t24__k7 = gexp2(T(0.11923099511479036)*v___yp7);
      const T v___t25__k7 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23__k7)));
      const T v_alpha_x1__k7 = (T(0.031158410986342627)*v___t24__k7*v___t25__k7);
      const T v___t26__k7 = gexp2((-T(0.08654439357462287))*v___yp7);
      const T v___t27__k7 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22__k7)));
      const T v_beta_x1__k7 = (T(0.0003916464405623223)*v___t26__k7*v___t27__k7);
      const T v_V_eff_1__k7 = ((gfabs((T(23.0) + v___yp7)) < T(0.01)) ? T(0.01) : (T(23.0) + v___yp7));
      const T v___t28__k7 = gexp2((-T(0.05770780163555854))*v_V_eff_1__k7);
      const T v___t29__k7 = (T(1.0)/(T(1.0) - ((v___t28__k7))));
      const T v___t30__k7 = (T(1.0)/(v___t21__k7*(T(8.331137487687693) + (T(69.4078518387552)*v___t21__k7))));
      const T v_i_K1__k7 = (T(0.0035)*((v___t29__k7*(T(4.6000000000000005) + (T(0.2)*v___yp7))) + (v___t30__k7*((-T(4.0)) + (T(119.85640018958804)*v___t21__k7)))));
      J[1] = ((((v_alpha_m__k7*(T(1.0) - ((s_m)))) - ((v_beta_m__k7*s_m)))) - f1[0]) / d;
      J[3] = ((((v_alpha_h__k7*(T(1.0) - ((s_h)))) - ((v_beta_h__k7*s_h)))) - f1[1]) / d;
      J[5] = ((((v_alpha_j__k7*(T(1.0) - ((s_j)))) - ((v_beta_j__k7*s_j)))) - f1[2]) / d;
      J[9] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k7)))) - f1[3]) / d;
      J[11] = ((((v_alpha_d__k7*(T(1.0) - ((s_d)))) - ((v_beta_d__k7*s_d)))) - f1[4]) / d;
      J[13] = ((((v_alpha_f__k7*(T(1.0) - ((s_f)))) - ((v_beta_f__k7*s_f)))) - f1[5]) / d;
      J[15] = ((((v_alpha_x1__k7*(T(1.0) - ((s_x1)))) - ((v_beta_x1__k7*s_x1)))) - f1[6]) / d;
      J[23] = (((P[14]*(T(v_Istim) - ((v_i_K1__k7)) - ((v_i_Na__k7)) - ((v_i_s__k7)) - ((v_i_x1__k7))))) - f1[7]) / d;
    }
    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;
  }

  // f1 = f(y, time), and the forward-difference Jacobian only if want_jac (J is left as it
  // is otherwise): rhs_fd_jacobian with its columns selected at run time
  template <typename T, class A>
  __device__ static __forceinline__ void rhs_fd_jacobian_sel(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, const bool want_jac,
      T* __restrict__ f1, A J)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v___t0 = gexp2((-T(0.14426950408889636))*v_V_eff_0);
    const T v___t1 = (T(1.0)/((-T(1.0)) + v___t0));
    const T v_alpha_m = (v___t1*((-T(47.0)) - ((s_V))));
    const T v___t2 = gexp2((-T(0.08079092228978195))*s_V);
    const T v_beta_m = (T(0.7095526727489909)*v___t2);
    const T v___t3 = gexp2((-T(0.36067376022224085))*s_V);
    const T v_alpha_h = (T(5.497962438709065e-10)*v___t3);
    const T v___t4 = gexp2((-T(0.118300993352895))*s_V);
    const T v___t5 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4)));
    const T v_beta_h = (T(1.7)*v___t5);
    const T v___t6 = gexp2((-T(0.14426950408889636))*s_V);
    const T v___t7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6*v___t6))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*v___t3*v___t7);
    const T v___t8 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6)));
    const T v_beta_j = (T(0.3)*v___t8);
    const T v___t9 = glog((T(0.001)*s_Cai));
    const T v___t10 = (T(1.0)/s_Cai);
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*v___t9)));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v___t11 = gexp2((-T(0.10386573368531053))*s_V);
    const T v___t12 = gexp2((-T(0.014426950408889635))*s_V);
    const T v___t13 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11)));
    const T v_alpha_d = (T(0.09987075415572229)*v___t12*v___t13);
    const T v___t14 = gexp2(T(0.07213475204444818)*s_V);
    const T v___t15 = gexp2((-T(0.024452458320151922))*s_V);
    const T v___t16 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14)));
    const T v_beta_d = (T(0.03320606467536786)*v___t15*v___t16);
    const T v___t17 = gexp2(T(0.21629610807930486)*s_V);
    const T v___t18 = gexp2((-T(0.011541560327111707))*s_V);
    const T v___t19 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17)));
    const T v_alpha_f = (T(0.009591781612432381)*v___t18*v___t19);
    const T v___t20 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6*v___t6))));
    const T v_beta_f = (T(0.0035672756346111717)*v___t20*(v___t12*v___t12));
    const T v___t21 = gexp2(T(0.05770780163555854)*s_V);
    const T v___t22 = gexp2((-T(0.05770780163555854))*s_V);
    const T v_i_x1 = (T(0.0019727757115328517)*v___t22*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
    const T v___t23 = gexp2(T(0.08243971662222647)*s_V);
    const T v___t24 = gexp2(T(0.11923099511479036)*s_V);
    const T v___t25 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23)));
    const T v_alpha_x1 = (T(0.031158410986342627)*v___t24*v___t25);
    const T v___t26 = gexp2((-T(0.08654439357462287))*s_V);
    const T v___t27 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22)));
    const T v_beta_x1 = (T(0.0003916464405623223)*v___t26*v___t27);
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v___t28 = gexp2((-T(0.05770780163555854))*v_V_eff_1);
    const T v___t29 = (T(1.0)/(T(1.0) - ((v___t28))));
    const T v___t30 = (T(1.0)/(v___t21*(T(8.331137487687693) + (T(69.4078518387552)*v___t21))));
    const T v_i_K1 = (T(0.0035)*((v___t29*(T(4.6000000000000005) + (T(0.2)*s_V))) + (v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21)))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    f1[0] = ((v_alpha_m*(T(1.0) - ((s_m)))) - ((v_beta_m*s_m)));
    f1[1] = ((v_alpha_h*(T(1.0) - ((s_h)))) - ((v_beta_h*s_h)));
    f1[2] = ((v_alpha_j*(T(1.0) - ((s_j)))) - ((v_beta_j*s_j)));
    f1[3] = (T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s)));
    f1[4] = ((v_alpha_d*(T(1.0) - ((s_d)))) - ((v_beta_d*s_d)));
    f1[5] = ((v_alpha_f*(T(1.0) - ((s_f)))) - ((v_beta_f*s_f)));
    f1[6] = ((v_alpha_x1*(T(1.0) - ((s_x1)))) - ((v_beta_x1*s_x1)));
    f1[7] = (P[14]*(T(v_Istim) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    if (want_jac) {
    fd_clear(J);
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[0])) ? 1e-5 : fabs(double(y[0]))));
      const T v___yp0 = T(double(y[0]) + d);
      const T v_i_Na__k0 = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(v___yp0*v___yp0*v___yp0))));
      J[0] = ((((v_alpha_m*(T(1.0) - ((v___yp0)))) - ((v___yp0*v_beta_m)))) - f1[0]) / d;
      J[16] = (((P[14]*(T(v_Istim) - ((v_i_Na__k0)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[1])) ? 1e-5 : fabs(double(y[1]))));
      const T v___yp1 = T(double(y[1]) + d);
      const T v_i_Na__k1 = ((s_V + P[10])*(P[2] + (v___yp1*P[1]*s_j*(s_m*s_m*s_m))));
      J[2] = ((((v_alpha_h*(T(1.0) - ((v___yp1)))) - ((v___yp1*v_beta_h)))) - f1[1]) / d;
      J[17] = (((P[14]*(T(v_Istim) - ((v_i_Na__k1)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[2])) ? 1e-5 : fabs(double(y[2]))));
      const T v___yp2 = T(double(y[2]) + d);
      const T v_i_Na__k2 = ((s_V + P[10])*(P[2] + (v___yp2*P[1]*s_h*(s_m*s_m*s_m))));
      J[4] = ((((v_alpha_j*(T(1.0) - ((v___yp2)))) - ((v___yp2*v_beta_j)))) - f1[2]) / d;
      J[18] = (((P[14]*(T(v_Istim) - ((v_i_Na__k2)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[3])) ? 1e-5 : fabs(double(y[3]))));
      const T v___yp3 = T(double(y[3]) + d);
      const T v___t9__k3 = glog((T(0.001)*v___yp3));
      const T v_E_s__k3 = ((-T(82.3)) - ((T(13.0287)*v___t9__k3)));
      const T v_i_s__k3 = (s_d*s_f*P[3]*(s_V - ((v_E_s__k3))));
      J[6] = (((T(7.000000000000001e-06) - ((T(0.07)*v___yp3)) - ((T(0.01)*v_i_s__k3)))) - f1[3]) / d;
      J[19] = (((P[14]*(T(v_Istim) - ((v_i_s__k3)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[4])) ? 1e-5 : fabs(double(y[4]))));
      const T v___yp4 = T(double(y[4]) + d);
      const T v_i_s__k4 = (v___yp4*s_f*P[3]*(s_V - ((v_E_s))));
      J[7] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k4)))) - f1[3]) / d;
      J[10] = ((((v_alpha_d*(T(1.0) - ((v___yp4)))) - ((v___yp4*v_beta_d)))) - f1[4]) / d;
      J[20] = (((P[14]*(T(v_Istim) - ((v_i_s__k4)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[5])) ? 1e-5 : fabs(double(y[5]))));
      const T v___yp5 = T(double(y[5]) + d);
      const T v_i_s__k5 = (v___yp5*s_d*P[3]*(s_V - ((v_E_s))));
      J[8] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k5)))) - f1[3]) / d;
      J[12] = ((((v_alpha_f*(T(1.0) - ((v___yp5)))) - ((v___yp5*v_beta_f)))) - f1[5]) / d;
      J[21] = (((P[14]*(T(v_Istim) - ((v_i_s__k5)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[6])) ? 1e-5 : fabs(double(y[6]))));
      const T v___yp6 = T(double(y[6]) + d);
      const T v_i_x1__k6 = (T(0.0019727757115328517)*v___yp6*v___t22*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
      J[14] = ((((v_alpha_x1*(T(1.0) - ((v___yp6)))) - ((v___yp6*v_beta_x1)))) - f1[6]) / d;
      J[22] = (((P[14]*(T(v_Istim) - ((v_i_x1__k6)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[7])) ? 1e-5 : fabs(double(y[7]))));
      const T v___yp7 = T(double(y[7]) + d);
      const T v_i_Na__k7 = ((v___yp7 + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
      const T v_V_eff_0__k7 = ((gfabs((T(47.0) + v___yp7)) < T(0.01)) ? T(0.01) : (T(47.0) + v___yp7));
      const T v___t0__k7 = gexp2((-T(0.14426950408889636))*v_V_eff_0__k7);
      const T v___t1__k7 = (T(1.0)/((-T(1.0)) + v___t0__k7));
      const T v_alpha_m__k7 = (v___t1__k7*((-T(47.0)) - ((v___yp7))));
      const T v___t2__k7 = gexp2((-T(0.08079092228978195))*v___yp7);
      const T v_beta_m__k7 = (T(0.7095526727489909)*v___t2__k7);
      const T v___t3__k7 = gexp2((-T(0.36067376022224085))*v___yp7);
      const T v_alpha_h__k7 = (T(5.497962438709065e-10)*v___t3__k7);
      const T v___t4__k7 = gexp2((-T(0.118300993352895))*v___yp7);
      const T v___t5__k7 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4__k7)));
      const T v_beta_h__k7 = (T(1.7)*v___t5__k7);
      const T v___t6__k7 = gexp2((-T(0.14426950408889636))*v___yp7);
      const T v___t7__k7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6__k7*v___t6__k7))));
      const T v_alpha_j__k7 = (T(1.8690473007222892e-10)*v___t3__k7*v___t7__k7);
      const T v___t8__k7 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6__k7)));
      const T v_beta_j__k7 = (T(0.3)*v___t8__k7);
      const T v_i_s__k7 = (s_d*s_f*P[3]*(v___yp7 - ((v_E_s))));
      const T v___t11__k7 = gexp2((-T(0.10386573368531053))*v___yp7);
      const T v___t12__k7 = gexp2((-T(0.014426950408889635))*v___yp7);
      const T v___t13__k7 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11__k7)));
      const T v_alpha_d__k7 = (T(0.09987075415572229)*v___t12__k7*v___t13__k7);
      const T v___t14__k7 = gexp2(T(0.07213475204444818)*v___yp7);
      const T v___t15__k7 = gexp2((-T(0.024452458320151922))*v___yp7);
      const T v___t16__k7 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14__k7)));
      const T v_beta_d__k7 = (T(0.03320606467536786)*v___t15__k7*v___t16__k7);
      const T v___t17__k7 = gexp2(T(0.21629610807930486)*v___yp7);
      const T v___t18__k7 = gexp2((-T(0.011541560327111707))*v___yp7);
      const T v___t19__k7 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17__k7)));
      const T v_alpha_f__k7 = (T(0.009591781612432381)*v___t18__k7*v___t19__k7);
      const T v___t20__k7 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6__k7*v___t6__k7))));
      const T v_beta_f__k7 = (T(0.0035672756346111717)*v___t20__k7*(v___t12__k7*v___t12__k7));
      const T v___t21__k7 = gexp2(T(0.05770780163555854)*v___yp7);
      const T v___t22__k7 = gexp2((-T(0.05770780163555854))*v___yp7);
      const T v_i_x1__k7 = (T(0.0019727757115328517)*v___t22__k7*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21__k7)));
      const T v___t23__k7 = gexp2(T(0.08243971662222647)*v___yp7);
      const T v___t24__k7 = gexp2(T(0.11923099511479036)*v___yp7);
      const T v___t25__k7 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23__k7)));
      const T v_alpha_x1__k7 = (T(0.031158410986342627)*v___t24__k7*v___t25__k7);
      const T v___t26__k7 = gexp2((-T(0.08654439357462287))*v___yp7);
      const T v___t27__k7 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22__k7)));
      const T v_beta_x1__k7 = (T(0.0003916464405623223)*v___t26__k7*v___t27__k7);
      const T v_V_eff_1__k7 = ((gfabs((T(23.0) + v___yp7)) < T(0.01)) ? T(0.01) : (T(23.0) + v___yp7));
      const T v___t28__k7 = gexp2((-T(0.05770780163555854))*v_V_eff_1__k7);
      const T v___t29__k7 = (T(1.0)/(T(1.0) - ((v___t28__k7))));
      const T v___t30__k7 = (T(1.0)/(v___t21__k7*(T(8.331137487687693) + (T(69.4078518387552)*v___t21__k7))));
      const T v_i_K1__k7 = (T(0.0035)*((v___t29__k7*(T(4.6000000000000005) + (T(0.2)*v___yp7))) + (v___t30__k7*((-T(4.0)) + (T(119.85640018958804)*v___t21__k7)))));
      J[1] = ((((v_alpha_m__k7*(T(1.0) - ((s_m)))) - ((v_beta_m__k7*s_m)))) - f1[0]) / d;
      J[3] = ((((v_alpha_h__k7*(T(1.0) - ((s_h)))) - ((v_beta_h__k7*s_h)))) - f1[1]) / d;
      J[5] = ((((v_alpha_j__k7*(T(1.0) - ((s_j)))) - ((v_beta_j__k7*s_j)))) - f1[2]) / d;
      J[9] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k7)))) - f1[3]) / d;
      J[11] = ((((v_alpha_d__k7*(T(1.0) - ((s_d)))) - ((v_beta_d__k7*s_d)))) - f1[4]) / d;
      J[13] = ((((v_alpha_f__k7*(T(1.0) - ((s_f)))) - ((v_beta_f__k7*s_f)))) - f1[5]) / d;
      J[15] = ((((v_alpha_x1__k7*(T(1.0) - ((s_x1)))) - ((v_beta_x1__k7*s_x1)))) - f1[6]) / d;
      J[23] = (((P[14]*(T(v_Istim) - ((v_i_K1__k7)) - ((v_i_Na__k7)) - ((v_i_s__k7)) - ((v_i_x1__k7))))) - f1[7]) / d;
    }
    }
    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;
  }

  // the same, also writing f0 = f(y, t0) (only the time-dependent statements again)
  template <typename T, class A>
  __device__ static __forceinline__ void rhs2_fd_jacobian(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, const double t0,
      T* __restrict__ f0, T* __restrict__ f1, A J)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v___t0 = gexp2((-T(0.14426950408889636))*v_V_eff_0);
    const T v___t1 = (T(1.0)/((-T(1.0)) + v___t0));
    const T v_alpha_m = (v___t1*((-T(47.0)) - ((s_V))));
    const T v___t2 = gexp2((-T(0.08079092228978195))*s_V);
    const T v_beta_m = (T(0.7095526727489909)*v___t2);
    const T v___t3 = gexp2((-T(0.36067376022224085))*s_V);
    const T v_alpha_h = (T(5.497962438709065e-10)*v___t3);
    const T v___t4 = gexp2((-T(0.118300993352895))*s_V);
    const T v___t5 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4)));
    const T v_beta_h = (T(1.7)*v___t5);
    const T v___t6 = gexp2((-T(0.14426950408889636))*s_V);
    const T v___t7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6*v___t6))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*v___t3*v___t7);
    const T v___t8 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6)));
    const T v_beta_j = (T(0.3)*v___t8);
    const T v___t9 = glog((T(0.001)*s_Cai));
    const T v___t10 = (T(1.0)/s_Cai);
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*v___t9)));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v___t11 = gexp2((-T(0.10386573368531053))*s_V);
    const T v___t12 = gexp2((-T(0.014426950408889635))*s_V);
    const T v___t13 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11)));
    const T v_alpha_d = (T(0.09987075415572229)*v___t12*v___t13);
    const T v___t14 = gexp2(T(0.07213475204444818)*s_V);
    const T v___t15 = gexp2((-T(0.024452458320151922))*s_V);
    const T v___t16 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14)));
    const T v_beta_d = (T(0.03320606467536786)*v___t15*v___t16);
    const T v___t17 = gexp2(T(0.21629610807930486)*s_V);
    const T v___t18 = gexp2((-T(0.011541560327111707))*s_V);
    const T v___t19 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17)));
    const T v_alpha_f = (T(0.009591781612432381)*v___t18*v___t19);
    const T v___t20 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6*v___t6))));
    const T v_beta_f = (T(0.0035672756346111717)*v___t20*(v___t12*v___t12));
    const T v___t21 = gexp2(T(0.05770780163555854)*s_V);
    const T v___t22 = gexp2((-T(0.05770780163555854))*s_V);
    const T v_i_x1 = (T(0.0019727757115328517)*v___t22*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
    const T v___t23 = gexp2(T(0.08243971662222647)*s_V);
    const T v___t24 = gexp2(T(0.11923099511479036)*s_V);
    const T v___t25 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23)));
    const T v_alpha_x1 = (T(0.031158410986342627)*v___t24*v___t25);
    const T v___t26 = gexp2((-T(0.08654439357462287))*s_V);
    const T v___t27 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22)));
    const T v_beta_x1 = (T(0.0003916464405623223)*v___t26*v___t27);
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v___t28 = gexp2((-T(0.05770780163555854))*v_V_eff_1);
    const T v___t29 = (T(1.0)/(T(1.0) - ((v___t28))));
    const T v___t30 = (T(1.0)/(v___t21*(T(8.331137487687693) + (T(69.4078518387552)*v___t21))));
    const T v_i_K1 = (T(0.0035)*((v___t29*(T(4.6000000000000005) + (T(0.2)*s_V))) + (v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21)))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    f1[0] = ((v_alpha_m*(T(1.0) - ((s_m)))) - ((v_beta_m*s_m)));
    f1[1] = ((v_alpha_h*(T(1.0) - ((s_h)))) - ((v_beta_h*s_h)));
    f1[2] = ((v_alpha_j*(T(1.0) - ((s_j)))) - ((v_beta_j*s_j)));
    f1[3] = (T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s)));
    f1[4] = ((v_alpha_d*(T(1.0) - ((s_d)))) - ((v_beta_d*s_d)));
    f1[5] = ((v_alpha_f*(T(1.0) - ((s_f)))) - ((v_beta_f*s_f)));
    f1[6] = ((v_alpha_x1*(T(1.0) - ((s_x1)))) - ((v_beta_x1*s_x1)));
    f1[7] = (P[14]*(T(v_Istim) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    const double v___tzero = t0;
    const double v_Istim__tz = (((PD[5] >= v___tzero) && (PD[8] <= v___tzero) && (PD[7] >= (v___tzero + PD[11] + (PD[13]*floor((PD[12]*(v___tzero + PD[11]))))))) ? PD[4] : 0.0);
    f0[0] = f1[0];
    f0[1] = f1[1];
    f0[2] = f1[2];
    f0[3] = f1[3];
    f0[4] = f1[4];
    f0[5] = f1[5];
    f0[6] = f1[6];
    f0[7] = (P[14]*(v_Istim__tz - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[0])) ? 1e-5 : fabs(double(y[0]))));
      const T v___yp0 = T(double(y[0]) + d);
      const T v_i_Na__k0 = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(v___yp0*v___yp0*v___yp0))));
      J[0] = ((((v_alpha_m*(T(1.0) - ((v___yp0)))) - ((v___yp0*v_beta_m)))) - f1[0]) / d;
      J[16] = (((P[14]*(T(v_Istim) - ((v_i_Na__k0)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[1])) ? 1e-5 : fabs(double(y[1]))));
      const T v___yp1 = T(double(y[1]) + d);
      const T v_i_Na__k1 = ((s_V + P[10])*(P[2] + (v___yp1*P[1]*s_j*(s_m*s_m*s_m))));
      J[2] = ((((v_alpha_h*(T(1.0) - ((v___yp1)))) - ((v___yp1*v_beta_h)))) - f1[1]) / d;
      J[17] = (((P[14]*(T(v_Istim) - ((v_i_Na__k1)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[2])) ? 1e-5 : fabs(double(y[2]))));
      const T v___yp2 = T(double(y[2]) + d);
      const T v_i_Na__k2 = ((s_V + P[10])*(P[2] + (v___yp2*P[1]*s_h*(s_m*s_m*s_m))));
      J[4] = ((((v_alpha_j*(T(1.0) - ((v___yp2)))) - ((v___yp2*v_beta_j)))) - f1[2]) / d;
      J[18] = (((P[14]*(T(v_Istim) - ((v_i_Na__k2)) - ((v_i_K1)) - ((v_i_s)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[3])) ? 1e-5 : fabs(double(y[3]))));
      const T v___yp3 = T(double(y[3]) + d);
      const T v___t9__k3 = glog((T(0.001)*v___yp3));
      const T v_E_s__k3 = ((-T(82.3)) - ((T(13.0287)*v___t9__k3)));
      const T v_i_s__k3 = (s_d*s_f*P[3]*(s_V - ((v_E_s__k3))));
      J[6] = (((T(7.000000000000001e-06) - ((T(0.07)*v___yp3)) - ((T(0.01)*v_i_s__k3)))) - f1[3]) / d;
      J[19] = (((P[14]*(T(v_Istim) - ((v_i_s__k3)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[4])) ? 1e-5 : fabs(double(y[4]))));
      const T v___yp4 = T(double(y[4]) + d);
      const T v_i_s__k4 = (v___yp4*s_f*P[3]*(s_V - ((v_E_s))));
      J[7] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k4)))) - f1[3]) / d;
      J[10] = ((((v_alpha_d*(T(1.0) - ((v___yp4)))) - ((v___yp4*v_beta_d)))) - f1[4]) / d;
      J[20] = (((P[14]*(T(v_Istim) - ((v_i_s__k4)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[5])) ? 1e-5 : fabs(double(y[5]))));
      const T v___yp5 = T(double(y[5]) + d);
      const T v_i_s__k5 = (v___yp5*s_d*P[3]*(s_V - ((v_E_s))));
      J[8] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k5)))) - f1[3]) / d;
      J[12] = ((((v_alpha_f*(T(1.0) - ((v___yp5)))) - ((v___yp5*v_beta_f)))) - f1[5]) / d;
      J[21] = (((P[14]*(T(v_Istim) - ((v_i_s__k5)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_x1))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[6])) ? 1e-5 : fabs(double(y[6]))));
      const T v___yp6 = T(double(y[6]) + d);
      const T v_i_x1__k6 = (T(0.0019727757115328517)*v___yp6*v___t22*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
      J[14] = ((((v_alpha_x1*(T(1.0) - ((v___yp6)))) - ((v___yp6*v_beta_x1)))) - f1[6]) / d;
      J[22] = (((P[14]*(T(v_Istim) - ((v_i_x1__k6)) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s))))) - f1[7]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[7])) ? 1e-5 : fabs(double(y[7]))));
      const T v___yp7 = T(double(y[7]) + d);
      const T v_i_Na__k7 = ((v___yp7 + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
      const T v_V_eff_0__k7 = ((gfabs((T(47.0) + v___yp7)) < T(0.01)) ? T(0.01) : (T(47.0) + v___yp7));
      const T v___t0__k7 = gexp2((-T(0.14426950408889636))*v_V_eff_0__k7);
      const T v___t1__k7 = (T(1.0)/((-T(1.0)) + v___t0__k7));
      const T v_alpha_m__k7 = (v___t1__k7*((-T(47.0)) - ((v___yp7))));
      const T v___t2__k7 = gexp2((-T(0.08079092228978195))*v___yp7);
      const T v_beta_m__k7 = (T(0.7095526727489909)*v___t2__k7);
      const T v___t3__k7 = gexp2((-T(0.36067376022224085))*v___yp7);
      const T v_alpha_h__k7 = (T(5.497962438709065e-10)*v___t3__k7);
      const T v___t4__k7 = gexp2((-T(0.118300993352895))*v___yp7);
      const T v___t5__k7 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4__k7)));
      const T v_beta_h__k7 = (T(1.7)*v___t5__k7);
      const T v___t6__k7 = gexp2((-T(0.14426950408889636))*v___yp7);
      const T v___t7__k7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6__k7*v___t6__k7))));
      const T v_alpha_j__k7 = (T(1.8690473007222892e-10)*v___t3__k7*v___t7__k7);
      const T v___t8__k7 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6__k7)));
      const T v_beta_j__k7 = (T(0.3)*v___t8__k7);
      const T v_i_s__k7 = (s_d*s_f*P[3]*(v___yp7 - ((v_E_s))));
      const T v___t11__k7 = gexp2((-T(0.10386573368531053))*v___yp7);
      const T v___t12__k7 = gexp2((-T(0.014426950408889635))*v___yp7);
      const T v___t13__k7 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11__k7)));
      const T v_alpha_d__k7 = (T(0.09987075415572229)*v___t12__k7*v___t13__k7);
      const T v___t14__k7 = gexp2(T(0.07213475204444818)*v___yp7);
      const T v___t15__k7 = gexp2((-T(0.024452458320151922))*v___yp7);
      const T v___t16__k7 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14__k7)));
      const T v_beta_d__k7 = (T(0.03320606467536786)*v___t15__k7*v___t16__k7);
      const T v___t17__k7 = gexp2(T(0.21629610807930486)*v___yp7);
      const T v___t18__k7 = gexp2((-T(0.011541560327111707))*v___yp7);
      const T v___t19__k7 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17__k7)));
      const T v_alpha_f__k7 = (T(0.009591781612432381)*v___t18__k7*v___t19__k7);
      const T v___t20__k7 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6__k7*v___t6__k7))));
      const T v_beta_f__k7 = (T(0.0035672756346111717)*v___t20__k7*(v___t12__k7*v___t12__k7));
      const T v___t21__k7 = gexp2(T(0.05770780163555854)*v___yp7);
      const T v___t22__k7 = gexp2((-T(0.05770780163555854))*v___yp7);
      const T v_i_x1__k7 = (T(0.0019727757115328517)*v___t22__k7*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21__k7)));
      const T v___t23__k7 = gexp2(T(0.08243971662222647)*v___yp7);
      const T v___t24__k7 = gexp2(T(0.11923099511479036)*v___yp7);
      const T v___t25__k7 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23__k7)));
      const T v_alpha_x1__k7 = (T(0.031158410986342627)*v___t24__k7*v___t25__k7);
      const T v___t26__k7 = gexp2((-T(0.08654439357462287))*v___yp7);
      const T v___t27__k7 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22__k7)));
      const T v_beta_x1__k7 = (T(0.0003916464405623223)*v___t26__k7*v___t27__k7);
      const T v_V_eff_1__k7 = ((gfabs((T(23.0) + v___yp7)) < T(0.01)) ? T(0.01) : (T(23.0) + v___yp7));
      const T v___t28__k7 = gexp2((-T(0.05770780163555854))*v_V_eff_1__k7);
      const T v___t29__k7 = (T(1.0)/(T(1.0) - ((v___t28__k7))));
      const T v___t30__k7 = (T(1.0)/(v___t21__k7*(T(8.331137487687693) + (T(69.4078518387552)*v___t21__k7))));
      const T v_i_K1__k7 = (T(0.0035)*((v___t29__k7*(T(4.6000000000000005) + (T(0.2)*v___yp7))) + (v___t30__k7*((-T(4.0)) + (T(119.85640018958804)*v___t21__k7)))));
      J[1] = ((((v_alpha_m__k7*(T(1.0) - ((s_m)))) - ((v_beta_m__k7*s_m)))) - f1[0]) / d;
      J[3] = ((((v_alpha_h__k7*(T(1.0) - ((s_h)))) - ((v_beta_h__k7*s_h)))) - f1[1]) / d;
      J[5] = ((((v_alpha_j__k7*(T(1.0) - ((s_j)))) - ((v_beta_j__k7*s_j)))) - f1[2]) / d;
      J[9] = (((T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s__k7)))) - f1[3]) / d;
      J[11] = ((((v_alpha_d__k7*(T(1.0) - ((s_d)))) - ((v_beta_d__k7*s_d)))) - f1[4]) / d;
      J[13] = ((((v_alpha_f__k7*(T(1.0) - ((s_f)))) - ((v_beta_f__k7*s_f)))) - f1[5]) / d;
      J[15] = ((((v_alpha_x1__k7*(T(1.0) - ((s_x1)))) - ((v_beta_x1__k7*s_x1)))) - f1[6]) / d;
      J[23] = (((P[14]*(T(v_Istim) - ((v_i_K1__k7)) - ((v_i_Na__k7)) - ((v_i_s__k7)) - ((v_i_x1__k7))))) - f1[7]) / d;
    }
    (void)time; (void)t0; (void)P; (void)PD; (void)F; (void)f0; (void)f1; (void)J;
  }

  // vector-Jacobian product of linearized (reverse mode, generated): after the forward
  // sweep seed(linear, rhs, abar, bbar) supplies the cotangents of the outputs, then
  // ybar = abar^T d(linear)/dy + bbar^T d(rhs)/dy and Fbar likewise for the field parameters
  template <typename T, class Seed>
  __device__ static __forceinline__ void linearized_vjp(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, Seed&& seed,
      T* __restrict__ ybar, T* __restrict__ Fbar)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v___t0 = gexp2((-T(0.14426950408889636))*v_V_eff_0);
    const T v___t1 = (T(1.0)/((-T(1.0)) + v___t0));
    const T v_alpha_m = (v___t1*((-T(47.0)) - ((s_V))));
    const T v___t2 = gexp2((-T(0.08079092228978195))*s_V);
    const T v_beta_m = (T(0.7095526727489909)*v___t2);
    const T v___t3 = gexp2((-T(0.36067376022224085))*s_V);
    const T v_alpha_h = (T(5.497962438709065e-10)*v___t3);
    const T v___t4 = gexp2((-T(0.118300993352895))*s_V);
    const T v___t5 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4)));
    const T v_beta_h = (T(1.7)*v___t5);
    const T v___t6 = gexp2((-T(0.14426950408889636))*s_V);
    const T v___t7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6*v___t6))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*v___t3*v___t7);
    const T v___t8 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6)));
    const T v_beta_j = (T(0.3)*v___t8);
    const T v___t9 = glog((T(0.001)*s_Cai));
    const T v___t10 = (T(1.0)/s_Cai);
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*v___t9)));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v___t11 = gexp2((-T(0.10386573368531053))*s_V);
    const T v___t12 = gexp2((-T(0.014426950408889635))*s_V);
    const T v___t13 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11)));
    const T v_alpha_d = (T(0.09987075415572229)*v___t12*v___t13);
    const T v___t14 = gexp2(T(0.07213475204444818)*s_V);
    const T v___t15 = gexp2((-T(0.024452458320151922))*s_V);
    const T v___t16 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14)));
    const T v_beta_d = (T(0.03320606467536786)*v___t15*v___t16);
    const T v___t17 = gexp2(T(0.21629610807930486)*s_V);
    const T v___t18 = gexp2((-T(0.011541560327111707))*s_V);
    const T v___t19 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17)));
    const T v_alpha_f = (T(0.009591781612432381)*v___t18*v___t19);
    const T v___t20 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6*v___t6))));
    const T v_beta_f = (T(0.0035672756346111717)*v___t20*(v___t12*v___t12));
    const T v___t21 = gexp2(T(0.05770780163555854)*s_V);
    const T v___t22 = gexp2((-T(0.05770780163555854))*s_V);
    const T v_i_x1 = (T(0.0019727757115328517)*v___t22*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
    const T v___t23 = gexp2(T(0.08243971662222647)*s_V);
    const T v___t24 = gexp2(T(0.11923099511479036)*s_V);
    const T v___t25 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23)));
    const T v_alpha_x1 = (T(0.031158410986342627)*v___t24*v___t25);
    const T v___t26 = gexp2((-T(0.08654439357462287))*s_V);
    const T v___t27 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22)));
    const T v_beta_x1 = (T(0.0003916464405623223)*v___t26*v___t27);
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v___t28 = gexp2((-T(0.05770780163555854))*v_V_eff_1);
    const T v___t29 = (T(1.0)/(T(1.0) - ((v___t28))));
    const T v___t30 = (T(1.0)/(v___t21*(T(8.331137487687693) + (T(69.4078518387552)*v___t21))));
    const T v_i_K1 = (T(0.0035)*((v___t29*(T(4.6000000000000005) + (T(0.2)*s_V))) + (v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21)))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    const T v_dE_s_dCai = (-(T(13.0287)*v___t10));
    const T v_di_s_dCai = (P[15]*s_d*v_dE_s_dCai*s_f);
    const T v_dV_eff_1_dV = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.0) : T(1.0));
    const T v_di_K1_dV = ((v___t30*(v___t21*(T(0.016779896026542326) + (T(0.0035)*v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21))*((-T(0.3332454995075077)) - ((T(5.552628147100417)*v___t21))))))) + (v___t29*(T(0.0007000000000000001) - ((T(0.00028000000000000003)*v___t28*v___t29*v_dV_eff_1_dV*(T(4.6000000000000005) + (T(0.2)*s_V)))))));
    const T v_di_Na_dV = (P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m)));
    const T v_di_s_dV = (s_d*s_f*P[3]);
    const T v_di_x1_dV = (s_x1*(T(0.0017169779107590322) - ((T(7.891102846131407e-05)*v___t22*((-T(1.0)) + (T(21.75840239619708)*v___t21))))));
    T lin_v[8], abar[8], rhs_v[8], bbar[8];
    rhs_v[0] = ((v_alpha_m*(T(1.0) - ((s_m)))) - ((v_beta_m*s_m)));
    rhs_v[1] = ((v_alpha_h*(T(1.0) - ((s_h)))) - ((v_beta_h*s_h)));
    rhs_v[2] = ((v_alpha_j*(T(1.0) - ((s_j)))) - ((v_beta_j*s_j)));
    rhs_v[3] = (T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s)));
    rhs_v[4] = ((v_alpha_d*(T(1.0) - ((s_d)))) - ((v_beta_d*s_d)));
    rhs_v[5] = ((v_alpha_f*(T(1.0) - ((s_f)))) - ((v_beta_f*s_f)));
    rhs_v[6] = ((v_alpha_x1*(T(1.0) - ((s_x1)))) - ((v_beta_x1*s_x1)));
    rhs_v[7] = (P[14]*(T(v_Istim) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    lin_v[0] = ((-(v_alpha_m)) - ((v_beta_m)));
    lin_v[1] = ((-(v_alpha_h)) - ((v_beta_h)));
    lin_v[2] = ((-(v_alpha_j)) - ((v_beta_j)));
    lin_v[4] = ((-(v_alpha_d)) - ((v_beta_d)));
    lin_v[5] = ((-(v_alpha_f)) - ((v_beta_f)));
    lin_v[6] = ((-(v_alpha_x1)) - ((v_beta_x1)));
    lin_v[3] = ((-T(0.07)) - ((T(0.01)*v_di_s_dCai)));
    lin_v[7] = (P[16]*(v_di_K1_dV + v_di_Na_dV + v_di_s_dV + v_di_x1_dV));
    seed(lin_v, rhs_v, abar, bbar);
    const T a_di_x1_dV = (P[16]*abar[7]);
    const T a_di_s_dV = (P[16]*abar[7]);
    const T a_di_Na_dV = (P[16]*abar[7]);
    const T a_di_K1_dV = (P[16]*abar[7]);
    const T a_dV_eff_1_dV = (-(T(0.00028000000000000003)*a_di_K1_dV*v___t28*(v___t29*v___t29)*(T(4.6000000000000005) + (T(0.2)*s_V))));
    const T a_di_s_dCai = (-(T(0.01)*abar[3]));
    const T a_dE_s_dCai = (a_di_s_dCai*P[15]*s_d*s_f);
    const T a_i_K1 = (-(P[14]*bbar[7]));
    const T a___t30 = ((a_di_K1_dV*((T(0.016779896026542326)*v___t21) + (T(0.007)*v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21))*(v___t21*((-T(0.3332454995075077)) - ((T(5.552628147100417)*v___t21))))))) + (a_i_K1*((-T(0.014)) + (T(0.4194974006635582)*v___t21))));
    const T a___t29 = ((a_di_K1_dV*(T(0.0007000000000000001) - ((T(0.0005600000000000001)*v___t28*v___t29*v_dV_eff_1_dV*(T(4.6000000000000005) + (T(0.2)*s_V)))))) + (a_i_K1*(T(0.016100000000000003) + (T(0.0007000000000000001)*s_V))));
    const T a___t28 = (v___t29*(v___t29*(a___t29 - ((T(0.00028000000000000003)*a_di_K1_dV*v_dV_eff_1_dV*(T(4.6000000000000005) + (T(0.2)*s_V)))))));
    const T a_V_eff_1 = (-(T(0.04)*a___t28*v___t28));
    const T a_beta_x1 = ((-(abar[6])) - ((bbar[6]*s_x1)));
    const T a___t27 = (T(0.0003916464405623223)*a_beta_x1*v___t26);
    const T a___t26 = (T(0.0003916464405623223)*a_beta_x1*v___t27);
    const T a_alpha_x1 = ((-(abar[6])) + (bbar[6]*(T(1.0) - ((s_x1)))));
    const T a___t25 = (T(0.031158410986342627)*a_alpha_x1*v___t24);
    const T a___t24 = (T(0.031158410986342627)*a_alpha_x1*v___t25);
    const T a___t23 = (-(T(17.41170806332765)*a___t25*(v___t25*v___t25)));
    const T a_i_x1 = (-(P[14]*bbar[7]));
    const T a___t22 = ((s_x1*(((-T(1.0)) + (T(21.75840239619708)*v___t21))*((T(0.0019727757115328517)*a_i_x1) - ((T(7.891102846131407e-05)*a_di_x1_dV))))) - ((T(0.4493289641172216)*a___t27*(v___t27*v___t27))));
    const T a___t21 = ((s_x1*(v___t22*((T(0.042924447768975804)*a_i_x1) - ((T(0.001716977910759032)*a_di_x1_dV))))) + ((v___t30*((T(0.4194974006635582)*a_i_K1) - ((a___t30*v___t30*(T(8.331137487687693) + (T(138.8157036775104)*v___t21)))))) + (a_di_K1_dV*(v___t30*((v___t30*((T(0.0035)*((-T(4.0)) + (T(119.85640018958804)*v___t21))*((-T(0.3332454995075077)) - ((T(11.105256294200833)*v___t21)))) + (T(0.4194974006635582)*v___t21*((-T(0.3332454995075077)) - ((T(5.552628147100417)*v___t21)))))) + T(0.016779896026542326))))));
    const T a_beta_f = ((-(abar[5])) - ((bbar[5]*s_f)));
    const T a___t20 = (T(0.0035672756346111717)*a_beta_f*(v___t12*v___t12));
    const T a_alpha_f = ((-(abar[5])) + (bbar[5]*(T(1.0) - ((s_f)))));
    const T a___t19 = (T(0.009591781612432381)*a_alpha_f*v___t18);
    const T a___t18 = (T(0.009591781612432381)*a_alpha_f*v___t19);
    const T a___t17 = (-(T(66.5465065250986)*a___t19*(v___t19*v___t19)));
    const T a_beta_d = ((-(abar[4])) - ((bbar[4]*s_d)));
    const T a___t16 = (T(0.03320606467536786)*a_beta_d*v___t15);
    const T a___t15 = (T(0.03320606467536786)*a_beta_d*v___t16);
    const T a___t14 = (-(T(9.02501349943412)*a___t16*(v___t16*v___t16)));
    const T a_alpha_d = ((-(abar[4])) + (bbar[4]*(T(1.0) - ((s_d)))));
    const T a___t13 = (T(0.09987075415572229)*a_alpha_d*v___t12);
    const T a___t12 = ((T(0.09987075415572229)*a_alpha_d*v___t13) + (T(0.0071345512692223435)*a_beta_f*v___t12*v___t20));
    const T a___t11 = (-(T(1.4332881385696572)*a___t13*(v___t13*v___t13)));
    const T a_i_s = ((-(T(0.01)*bbar[3])) - ((P[14]*bbar[7])));
    const T a_E_s = (-(a_i_s*s_d*s_f*P[3]));
    const T a___t10 = (-(T(13.0287)*a_dE_s_dCai));
    const T a___t9 = (-(T(13.0287)*a_E_s));
    const T a_beta_j = ((-(abar[2])) - ((bbar[2]*s_j)));
    const T a___t8 = (T(0.3)*a_beta_j);
    const T a_alpha_j = ((-(abar[2])) + (bbar[2]*(T(1.0) - ((s_j)))));
    const T a___t7 = (T(1.8690473007222892e-10)*a_alpha_j*v___t3);
    const T a___t6 = ((v___t6*((-(T(3.3576550599913205e-07)*a___t7*(v___t7*v___t7))) - ((T(0.004957504353332717)*a___t20*(v___t20*v___t20))))) - ((T(0.040762203978366204)*a___t8*(v___t8*v___t8))));
    const T a_beta_h = ((-(abar[1])) - ((bbar[1]*s_h)));
    const T a___t5 = (T(1.7)*a_beta_h);
    const T a___t4 = (-(T(0.1580253208896478)*a___t5*(v___t5*v___t5)));
    const T a_alpha_h = ((-(abar[1])) + (bbar[1]*(T(1.0) - ((s_h)))));
    const T a___t3 = ((T(5.497962438709065e-10)*a_alpha_h) + (T(1.8690473007222892e-10)*a_alpha_j*v___t7));
    const T a_beta_m = ((-(abar[0])) - ((bbar[0]*s_m)));
    const T a___t2 = (T(0.7095526727489909)*a_beta_m);
    const T a_alpha_m = ((-(abar[0])) + (bbar[0]*(T(1.0) - ((s_m)))));
    const T a___t1 = (a_alpha_m*((-T(47.0)) - ((s_V))));
    const T a___t0 = (-(a___t1*(v___t1*v___t1)));
    const T a_V_eff_0 = (-(T(0.1)*a___t0*v___t0));
    const T a_i_Na = (-(P[14]*bbar[7]));
    ybar[0] = ((s_m*(s_m*(s_j*(s_h*(P[1]*(T(3.0)*(a_di_Na_dV + (a_i_Na*(s_V + P[10]))))))))) + (bbar[0]*((-(v_alpha_m)) - ((v_beta_m)))));
    ybar[1] = ((s_m*(s_m*(s_m*(s_j*(P[1]*(a_di_Na_dV + (a_i_Na*(s_V + P[10])))))))) + (bbar[1]*((-(v_alpha_h)) - ((v_beta_h)))));
    ybar[2] = ((s_m*(s_m*(s_m*(s_h*(P[1]*(a_di_Na_dV + (a_i_Na*(s_V + P[10])))))))) + (bbar[2]*((-(v_alpha_j)) - ((v_beta_j)))));
    ybar[3] = ((v___t10*((T(1.0)*a___t9) - ((a___t10*v___t10)))) - ((T(0.07)*bbar[3])));
    ybar[4] = ((s_f*((P[3]*(a_di_s_dV + (a_i_s*(s_V - ((v_E_s)))))) + (a_di_s_dCai*P[15]*v_dE_s_dCai))) + (bbar[4]*((-(v_alpha_d)) - ((v_beta_d)))));
    ybar[5] = ((s_d*((P[3]*(a_di_s_dV + (a_i_s*(s_V - ((v_E_s)))))) + (a_di_s_dCai*P[15]*v_dE_s_dCai))) + (bbar[5]*((-(v_alpha_f)) - ((v_beta_f)))));
    ybar[6] = ((a_di_x1_dV*(T(0.0017169779107590322) - ((T(7.891102846131407e-05)*v___t22*((-T(1.0)) + (T(21.75840239619708)*v___t21)))))) + (bbar[6]*((-(v_alpha_x1)) - ((v_beta_x1)))) + (T(0.0019727757115328517)*a_i_x1*v___t22*((-T(1.0)) + (T(21.75840239619708)*v___t21))));
    ybar[7] = ((v___t29*((T(0.0007000000000000001)*a_i_K1) - ((T(5.6000000000000006e-05)*a_di_K1_dV*v___t28*v___t29*v_dV_eff_1_dV)))) + ((T(0.04)*((a___t21*v___t21) - ((a___t22*v___t22)))) + ((a_V_eff_0*((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.0) : T(1.0))) + (a_V_eff_1*((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.0) : T(1.0))) + (a_i_Na*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m)))) - ((a_alpha_m*v___t1)) + (T(0.08264462809917356)*a___t24*v___t24) + (T(0.05)*a___t14*v___t14) + (T(0.14992503748125938)*a___t17*v___t17) + (T(0.05714285714285714)*a___t23*v___t23) - ((T(0.25)*a___t3*v___t3)) - ((T(0.008)*a___t18*v___t18)) - ((T(0.07199424046076314)*a___t11*v___t11)) - ((T(0.1)*a___t6*v___t6)) - ((T(0.01694915254237288)*a___t15*v___t15)) - ((T(0.01)*a___t12*v___t12)) - ((T(0.082)*a___t4*v___t4)) - ((T(0.056)*a___t2*v___t2)) - ((T(0.05998800239952009)*a___t26*v___t26)) + (a_i_s*s_d*s_f*P[3]))));
    (void)time; (void)P; (void)PD; (void)F; (void)abar; (void)bbar; (void)Fbar;
  }

  // vector-Jacobian product of rhs (reverse mode, generated): after the forward sweep
  // seed(values, bbar) supplies the cotangents of the values, then ybar = bbar^T df/dy
  // and Fbar = bbar^T df/dF
  template <typename T, class Seed>
  __device__ static __forceinline__ void rhs_vjp(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, Seed&& seed,
      T* __restrict__ ybar, T* __restrict__ Fbar)
  {
    const T s_m = y[0];
    const T s_h = y[1];
    const T s_j = y[2];
    const T s_Cai = y[3];
    const T s_d = y[4];
    const T s_f = y[5];
    const T s_x1 = y[6];
    const T s_V = y[7];
    const T v_i_Na = ((s_V + P[10])*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m))));
    const T v_V_eff_0 = ((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.01) : (T(47.0) + s_V));
    const T v___t0 = gexp2((-T(0.14426950408889636))*v_V_eff_0);
    const T v___t1 = (T(1.0)/((-T(1.0)) + v___t0));
    const T v_alpha_m = (v___t1*((-T(47.0)) - ((s_V))));
    const T v___t2 = gexp2((-T(0.08079092228978195))*s_V);
    const T v_beta_m = (T(0.7095526727489909)*v___t2);
    const T v___t3 = gexp2((-T(0.36067376022224085))*s_V);
    const T v_alpha_h = (T(5.497962438709065e-10)*v___t3);
    const T v___t4 = gexp2((-T(0.118300993352895))*s_V);
    const T v___t5 = (T(1.0)/(T(1.0) + (T(0.1580253208896478)*v___t4)));
    const T v_beta_h = (T(1.7)*v___t5);
    const T v___t6 = gexp2((-T(0.14426950408889636))*s_V);
    const T v___t7 = (T(1.0)/(T(1.0) + (T(1.6788275299956603e-07)*(v___t6*v___t6))));
    const T v_alpha_j = (T(1.8690473007222892e-10)*v___t3*v___t7);
    const T v___t8 = (T(1.0)/(T(1.0) + (T(0.040762203978366204)*v___t6)));
    const T v_beta_j = (T(0.3)*v___t8);
    const T v___t9 = glog((T(0.001)*s_Cai));
    const T v___t10 = (T(1.0)/s_Cai);
    const T v_E_s = ((-T(82.3)) - ((T(13.0287)*v___t9)));
    const T v_i_s = (s_d*s_f*P[3]*(s_V - ((v_E_s))));
    const T v___t11 = gexp2((-T(0.10386573368531053))*s_V);
    const T v___t12 = gexp2((-T(0.014426950408889635))*s_V);
    const T v___t13 = (T(1.0)/(T(1.0) + (T(1.4332881385696572)*v___t11)));
    const T v_alpha_d = (T(0.09987075415572229)*v___t12*v___t13);
    const T v___t14 = gexp2(T(0.07213475204444818)*s_V);
    const T v___t15 = gexp2((-T(0.024452458320151922))*s_V);
    const T v___t16 = (T(1.0)/(T(1.0) + (T(9.02501349943412)*v___t14)));
    const T v_beta_d = (T(0.03320606467536786)*v___t15*v___t16);
    const T v___t17 = gexp2(T(0.21629610807930486)*s_V);
    const T v___t18 = gexp2((-T(0.011541560327111707))*s_V);
    const T v___t19 = (T(1.0)/(T(1.0) + (T(66.5465065250986)*v___t17)));
    const T v_alpha_f = (T(0.009591781612432381)*v___t18*v___t19);
    const T v___t20 = (T(1.0)/(T(1.0) + (T(0.0024787521766663585)*(v___t6*v___t6))));
    const T v_beta_f = (T(0.0035672756346111717)*v___t20*(v___t12*v___t12));
    const T v___t21 = gexp2(T(0.05770780163555854)*s_V);
    const T v___t22 = gexp2((-T(0.05770780163555854))*s_V);
    const T v_i_x1 = (T(0.0019727757115328517)*v___t22*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21)));
    const T v___t23 = gexp2(T(0.08243971662222647)*s_V);
    const T v___t24 = gexp2(T(0.11923099511479036)*s_V);
    const T v___t25 = (T(1.0)/(T(1.0) + (T(17.41170806332765)*v___t23)));
    const T v_alpha_x1 = (T(0.031158410986342627)*v___t24*v___t25);
    const T v___t26 = gexp2((-T(0.08654439357462287))*s_V);
    const T v___t27 = (T(1.0)/(T(1.0) + (T(0.4493289641172216)*v___t22)));
    const T v_beta_x1 = (T(0.0003916464405623223)*v___t26*v___t27);
    const T v_V_eff_1 = ((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.01) : (T(23.0) + s_V));
    const T v___t28 = gexp2((-T(0.05770780163555854))*v_V_eff_1);
    const T v___t29 = (T(1.0)/(T(1.0) - ((v___t28))));
    const T v___t30 = (T(1.0)/(v___t21*(T(8.331137487687693) + (T(69.4078518387552)*v___t21))));
    const T v_i_K1 = (T(0.0035)*((v___t29*(T(4.6000000000000005) + (T(0.2)*s_V))) + (v___t30*((-T(4.0)) + (T(119.85640018958804)*v___t21)))));
    const double v_Istim = (((time >= PD[8]) && (time <= PD[5]) && ((PD[11] + time + (PD[13]*floor((PD[12]*(PD[11] + time))))) <= PD[7])) ? PD[4] : 0.0);
    T f_v[8], bbar[8];
    f_v[0] = ((v_alpha_m*(T(1.0) - ((s_m)))) - ((v_beta_m*s_m)));
    f_v[1] = ((v_alpha_h*(T(1.0) - ((s_h)))) - ((v_beta_h*s_h)));
    f_v[2] = ((v_alpha_j*(T(1.0) - ((s_j)))) - ((v_beta_j*s_j)));
    f_v[3] = (T(7.000000000000001e-06) - ((T(0.07)*s_Cai)) - ((T(0.01)*v_i_s)));
    f_v[4] = ((v_alpha_d*(T(1.0) - ((s_d)))) - ((v_beta_d*s_d)));
    f_v[5] = ((v_alpha_f*(T(1.0) - ((s_f)))) - ((v_beta_f*s_f)));
    f_v[6] = ((v_alpha_x1*(T(1.0) - ((s_x1)))) - ((v_beta_x1*s_x1)));
    f_v[7] = (P[14]*(T(v_Istim) - ((v_i_K1)) - ((v_i_Na)) - ((v_i_s)) - ((v_i_x1))));
    seed(f_v, bbar);
    const T a_i_K1 = (-(P[14]*bbar[7]));
    const T a___t30 = (a_i_K1*((-T(0.014)) + (T(0.4194974006635582)*v___t21)));
    const T a___t29 = (a_i_K1*(T(0.016100000000000003) + (T(0.0007000000000000001)*s_V)));
    const T a___t28 = (a___t29*(v___t29*v___t29));
    const T a_V_eff_1 = (-(T(0.04)*a___t28*v___t28));
    const T a_beta_x1 = (-(bbar[6]*s_x1));
    const T a___t27 = (T(0.0003916464405623223)*a_beta_x1*v___t26);
    const T a___t26 = (T(0.0003916464405623223)*a_beta_x1*v___t27);
    const T a_alpha_x1 = (bbar[6]*(T(1.0) - ((s_x1))));
    const T a___t25 = (T(0.031158410986342627)*a_alpha_x1*v___t24);
    const T a___t24 = (T(0.031158410986342627)*a_alpha_x1*v___t25);
    const T a___t23 = (-(T(17.41170806332765)*a___t25*(v___t25*v___t25)));
    const T a_i_x1 = (-(P[14]*bbar[7]));
    const T a___t22 = ((-(T(0.4493289641172216)*a___t27*(v___t27*v___t27))) + (T(0.0019727757115328517)*a_i_x1*s_x1*((-T(1.0)) + (T(21.75840239619708)*v___t21))));
    const T a___t21 = ((v___t30*((T(0.4194974006635582)*a_i_K1) - ((a___t30*v___t30*(T(8.331137487687693) + (T(138.8157036775104)*v___t21)))))) + (T(0.042924447768975804)*a_i_x1*v___t22*s_x1));
    const T a_beta_f = (-(bbar[5]*s_f));
    const T a___t20 = (T(0.0035672756346111717)*a_beta_f*(v___t12*v___t12));
    const T a_alpha_f = (bbar[5]*(T(1.0) - ((s_f))));
    const T a___t19 = (T(0.009591781612432381)*a_alpha_f*v___t18);
    const T a___t18 = (T(0.009591781612432381)*a_alpha_f*v___t19);
    const T a___t17 = (-(T(66.5465065250986)*a___t19*(v___t19*v___t19)));
    const T a_beta_d = (-(bbar[4]*s_d));
    const T a___t16 = (T(0.03320606467536786)*a_beta_d*v___t15);
    const T a___t15 = (T(0.03320606467536786)*a_beta_d*v___t16);
    const T a___t14 = (-(T(9.02501349943412)*a___t16*(v___t16*v___t16)));
    const T a_alpha_d = (bbar[4]*(T(1.0) - ((s_d))));
    const T a___t13 = (T(0.09987075415572229)*a_alpha_d*v___t12);
    const T a___t12 = ((T(0.09987075415572229)*a_alpha_d*v___t13) + (T(0.0071345512692223435)*a_beta_f*v___t12*v___t20));
    const T a___t11 = (-(T(1.4332881385696572)*a___t13*(v___t13*v___t13)));
    const T a_i_s = ((-(T(0.01)*bbar[3])) - ((P[14]*bbar[7])));
    const T a_E_s = (-(a_i_s*s_d*s_f*P[3]));
    const T a___t9 = (-(T(13.0287)*a_E_s));
    const T a_beta_j = (-(bbar[2]*s_j));
    const T a___t8 = (T(0.3)*a_beta_j);
    const T a_alpha_j = (bbar[2]*(T(1.0) - ((s_j))));
    const T a___t7 = (T(1.8690473007222892e-10)*a_alpha_j*v___t3);
    const T a___t6 = ((v___t6*((-(T(3.3576550599913205e-07)*a___t7*(v___t7*v___t7))) - ((T(0.004957504353332717)*a___t20*(v___t20*v___t20))))) - ((T(0.040762203978366204)*a___t8*(v___t8*v___t8))));
    const T a_beta_h = (-(bbar[1]*s_h));
    const T a___t5 = (T(1.7)*a_beta_h);
    const T a___t4 = (-(T(0.1580253208896478)*a___t5*(v___t5*v___t5)));
    const T a_alpha_h = (bbar[1]*(T(1.0) - ((s_h))));
    const T a___t3 = ((T(5.497962438709065e-10)*a_alpha_h) + (T(1.8690473007222892e-10)*a_alpha_j*v___t7));
    const T a_beta_m = (-(bbar[0]*s_m));
    const T a___t2 = (T(0.7095526727489909)*a_beta_m);
    const T a_alpha_m = (bbar[0]*(T(1.0) - ((s_m))));
    const T a___t1 = (a_alpha_m*((-T(47.0)) - ((s_V))));
    const T a___t0 = (-(a___t1*(v___t1*v___t1)));
    const T a_V_eff_0 = (-(T(0.1)*a___t0*v___t0));
    const T a_i_Na = (-(P[14]*bbar[7]));
    ybar[0] = ((bbar[0]*((-(v_alpha_m)) - ((v_beta_m)))) + (T(3.0)*a_i_Na*P[1]*s_h*s_j*(s_m*s_m)*(s_V + P[10])));
    ybar[1] = ((bbar[1]*((-(v_alpha_h)) - ((v_beta_h)))) + (a_i_Na*P[1]*s_j*(s_m*s_m*s_m)*(s_V + P[10])));
    ybar[2] = ((bbar[2]*((-(v_alpha_j)) - ((v_beta_j)))) + (a_i_Na*P[1]*s_h*(s_m*s_m*s_m)*(s_V + P[10])));
    ybar[3] = ((-(T(0.07)*bbar[3])) + (T(1.0)*a___t9*v___t10));
    ybar[4] = ((bbar[4]*((-(v_alpha_d)) - ((v_beta_d)))) + (a_i_s*s_f*P[3]*(s_V - ((v_E_s)))));
    ybar[5] = ((bbar[5]*((-(v_alpha_f)) - ((v_beta_f)))) + (a_i_s*s_d*P[3]*(s_V - ((v_E_s)))));
    ybar[6] = ((bbar[6]*((-(v_alpha_x1)) - ((v_beta_x1)))) + (T(0.0019727757115328517)*a_i_x1*v___t22*((-T(1.0)) + (T(21.75840239619708)*v___t21))));
    ybar[7] = ((T(0.04)*((a___t21*v___t21) - ((a___t22*v___t22)))) + ((a_V_eff_0*((gfabs((T(47.0) + s_V)) < T(0.01)) ? T(0.0) : T(1.0))) + (a_V_eff_1*((gfabs((T(23.0) + s_V)) < T(0.01)) ? T(0.0) : T(1.0))) + (a_i_Na*(P[2] + (P[1]*s_h*s_j*(s_m*s_m*s_m)))) - ((a_alpha_m*v___t1)) + (T(0.0007000000000000001)*a_i_K1*v___t29) + (T(0.08264462809917356)*a___t24*v___t24) + (T(0.05)*a___t14*v___t14) + (T(0.14992503748125938)*a___t17*v___t17) + (T(0.05714285714285714)*a___t23*v___t23) - ((T(0.25)*a___t3*v___t3)) - ((T(0.008)*a___t18*v___t18)) - ((T(0.07199424046076314)*a___t11*v___t11)) - ((T(0.1)*a___t6*v___t6)) - ((T(0.01694915254237288)*a___t15*v___t15)) - ((T(0.01)*a___t12*v___t12)) - ((T(0.082)*a___t4*v___t4)) - ((T(0.056)*a___t2*v___t2)) - ((T(0.05998800239952009)*a___t26*v___t26)) + (a_i_s*s_d*s_f*P[3])));
    (void)time; (void)P; (void)PD; (void)F; (void)bbar; (void)Fbar;
  }
};

}}  // namespace goss_b200::models
#endif
