// Generated by goss_b200.codegen from the 'oscilator' model; do not edit.
// Device-side model: rhs and linearised rhs templated on the arithmetic type T.
#ifndef M_OSCILATOR_DEVICE_CUH
#define M_OSCILATOR_DEVICE_CUH
#include "goss_device_math.cuh"

namespace goss_b200 { namespace models {

struct M_oscilator {
  static constexpr const char* name = "oscilator";
  static constexpr int num_states = 2;
  static constexpr int num_params = 2;
  static constexpr int num_field_params = 0;
  static constexpr int num_monitored = 0;
  static constexpr int num_derived = 1;
  // the reference generator's linear-term flags (RL1/RL2 use the exponential update for these)
  __host__ __device__ static constexpr bool linear_term(int i) { return false; }

  // values = f(y, time)
  template <typename T>
  __device__ static __forceinline__ void rhs(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ values)
  {
    const T s_x = y[0];
    const T s_y = y[1];
    values[0] = (P[2]*s_y);
    values[1] = (P[1]*s_x);
    (void)time; (void)P; (void)PD; (void)F;
  }

  // Newton matrix: 4 packed entries (the Jacobian's 2 structural
  // non-zeros, the diagonal and the LU fill-in; row-major over the structure)
  static constexpr int lu_nnz = 4;
  static constexpr bool has_jacobian = false;
  // J := scale*J + I
  template <class A>
  __device__ static __forceinline__ void lu_shift(A J, const double scale)
  {
    for (int k = 0; k < 4; ++k) J[k] = J[k] * scale;
    J[0] = J[0] + 1.0 * 1.0;
    J[3] = J[3] + 1.0 * 1.0;
  }
  // D := scale*S + I
  template <class A, class B>
  __device__ static __forceinline__ void lu_copy_shift(A S, B D, const double scale)
  {
    for (int k = 0; k < 4; ++k) D[k] = S[k] * scale;
    D[0] = D[0] + 1.0 * 1.0;
    D[3] = D[3] + 1.0 * 1.0;
  }
  // in-place Doolittle LU without pivoting over the structure
  template <class A>
  __device__ static __forceinline__ void lu_factorize(A J)
  {
    { const double s = 0.0; J[2] = (J[2] - s) / J[0]; }
    { double s = 0.0; s = s + J[2] * J[1]; J[3] -= s; }
  }
  // x = (LU)^-1 b, forward then backward substitution; b and x may alias
  template <class A>
  __device__ static __forceinline__ void lu_solve(A J, const double* b, double* x)
  {
    x[0] = b[0];
    { double s = 0.0; s = s + J[2] * x[0]; x[1] = b[1] - s; }
    x[1] = x[1] / J[3];
    { double s = 0.0; s = s + J[1] * x[1]; x[0] = (x[0] - s) / J[0]; }
  }
  // forward differences: zero the entries outside the Jacobian's structure, then
  // column i = (f2 - f1) / delta at its structural rows
  template <class A>
  __device__ static __forceinline__ void fd_clear(A J)
  {
    J[0] = 0.0;
    J[3] = 0.0;
    (void)J;
  }
  template <class A>
  __device__ static __forceinline__ void fd_column(const int i, const double* f1, const double* f2,
                                                   const double delta, A J)
  {
    switch (i) {
    case 0: J[2] = (f2[1] - f1[1]) / delta; break;
    case 1: J[1] = (f2[0] - f1[0]) / delta; break;
    default: break;
    }
  }
  // dense row-major copy: out(r*n + c, value) for every entry
  template <typename T, class Out>
  __device__ static __forceinline__ void lu_unpack(const T* J, Out&& out)
  {
    out(0, J[0]);
    out(1, J[1]);
    out(2, J[2]);
    out(3, J[3]);
  }

  // derived constants: parameter-only sub-expressions, evaluated once per
  // launch on the host in FP64 and stored after the parameters
  static void derived(const double* P, double* C)
  {
    C[0] = (-(P[0]));
    (void)P; (void)C;
  }

  // rhs = f(y, time), linear[i] = d f_i / d y_i
  template <typename T>
  __device__ static __forceinline__ void linearized(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ linear, T* __restrict__ rhs)
  {
    const T s_x = y[0];
    const T s_y = y[1];
    rhs[0] = (P[2]*s_y);
    rhs[1] = (P[1]*s_x);
    linear[0] = T(0.0);
    linear[1] = T(0.0);
    (void)time; (void)P; (void)PD; (void)F;
  }

  // linearized with every distinct transcendental and reciprocal of a state-dependent
  // operand evaluated once (the FP32 kernels' form; FP64 keeps the reference's operations)
  template <typename T>
  __device__ static __forceinline__ void linearized_split(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ linear, T* __restrict__ rhs)
  {
    const T s_x = y[0];
    const T s_y = y[1];
    rhs[0] = (P[2]*s_y);
    rhs[1] = (P[1]*s_x);
    linear[0] = T(0.0);
    linear[1] = T(0.0);
    (void)time; (void)P; (void)PD; (void)F;
  }

  // rhs in the same split form
  template <typename T>
  __device__ static __forceinline__ void rhs_split(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ values)
  {
    const T s_x = y[0];
    const T s_y = y[1];
    values[0] = (P[2]*s_y);
    values[1] = (P[1]*s_x);
    (void)time; (void)P; (void)PD; (void)F;
  }

  // forward-difference Jacobian of rhs_split at y into the packed Newton matrix (structural
  // entries; fd_clear sets the others): f1 = f(y, time); column i recomputes only the
  // statements of its rows that depend on state i
  template <typename T, class A>
  __device__ static __forceinline__ void fd_jacobian(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, const T* __restrict__ f1, A J)
  {
    const T s_x = y[0];
    const T s_y = y[1];
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[0])) ? 1e-5 : fabs(double(y[0]))));
      const T v___yp0 = T(double(y[0]) + d);
      J[2] = (((v___yp0*P[1])) - f1[1]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[1])) ? 1e-5 : fabs(double(y[1]))));
      const T v___yp1 = T(double(y[1]) + d);
      J[1] = (((v___yp1*P[2])) - f1[0]) / d;
    }
    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;
  }

  // the same, also writing f1 = f(y, time) (rhs_split) from its unperturbed statements
  template <typename T, class A>
  __device__ static __forceinline__ void rhs_fd_jacobian(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, T* __restrict__ f1, A J)
  {
    const T s_x = y[0];
    const T s_y = y[1];
    f1[0] = (P[2]*s_y);
    f1[1] = (P[1]*s_x);
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[0])) ? 1e-5 : fabs(double(y[0]))));
      const T v___yp0 = T(double(y[0]) + d);
      J[2] = (((v___yp0*P[1])) - f1[1]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[1])) ? 1e-5 : fabs(double(y[1]))));
      const T v___yp1 = T(double(y[1]) + d);
      J[1] = (((v___yp1*P[2])) - f1[0]) / d;
    }
    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;
  }

  // f1 = f(y, time), and the forward-difference Jacobian only if want_jac (J is left as it
  // is otherwise): rhs_fd_jacobian with its columns selected at run time
  template <typename T, class A>
  __device__ static __forceinline__ void rhs_fd_jacobian_sel(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, const bool want_jac,
      T* __restrict__ f1, A J)
  {
    const T s_x = y[0];
    const T s_y = y[1];
    f1[0] = (P[2]*s_y);
    f1[1] = (P[1]*s_x);
    if (want_jac) {
    fd_clear(J);
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[0])) ? 1e-5 : fabs(double(y[0]))));
      const T v___yp0 = T(double(y[0]) + d);
      J[2] = (((v___yp0*P[1])) - f1[1]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[1])) ? 1e-5 : fabs(double(y[1]))));
      const T v___yp1 = T(double(y[1]) + d);
      J[1] = (((v___yp1*P[2])) - f1[0]) / d;
    }
    }
    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;
  }

  // the same, also writing f0 = f(y, t0) (only the time-dependent statements again)
  template <typename T, class A>
  __device__ static __forceinline__ void rhs2_fd_jacobian(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, const double t0,
      T* __restrict__ f0, T* __restrict__ f1, A J)
  {
    const T s_x = y[0];
    const T s_y = y[1];
    f1[0] = (P[2]*s_y);
    f1[1] = (P[1]*s_x);
    const double v___tzero = t0;
    f0[0] = f1[0];
    f0[1] = f1[1];
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[0])) ? 1e-5 : fabs(double(y[0]))));
      const T v___yp0 = T(double(y[0]) + d);
      J[2] = (((v___yp0*P[1])) - f1[1]) / d;
    }
    {
      const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[1])) ? 1e-5 : fabs(double(y[1]))));
      const T v___yp1 = T(double(y[1]) + d);
      J[1] = (((v___yp1*P[2])) - f1[0]) / d;
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
    const T s_x = y[0];
    const T s_y = y[1];
    T lin_v[2], abar[2], rhs_v[2], bbar[2];
    rhs_v[0] = (P[2]*s_y);
    rhs_v[1] = (P[1]*s_x);
    lin_v[0] = T(0.0);
    lin_v[1] = T(0.0);
    seed(lin_v, rhs_v, abar, bbar);
    ybar[0] = (bbar[1]*P[1]);
    ybar[1] = (P[2]*bbar[0]);
    (void)time; (void)P; (void)PD; (void)F; (void)abar; (void)bbar; (void)Fbar;
  }

  // vector-Jacobian product of rhs (reverse mode, generated): after the forward sweep
  // seed(values, bbar) supplies the cotangents of the values, then ybar = bbar^T df/dy
  // and Fbar = bbar^T df/dF
  template <typename T, class Seed>
  __device__ static __forceinline__ void rhs_vjp(const T* __restrict__ y, const double time, const T* __restrict__ P, const double* __restrict__ PD, const T* __restrict__ F, Seed&& seed,
      T* __restrict__ ybar, T* __restrict__ Fbar)
  {
    const T s_x = y[0];
    const T s_y = y[1];
    T f_v[2], bbar[2];
    f_v[0] = (P[2]*s_y);
    f_v[1] = (P[1]*s_x);
    seed(f_v, bbar);
    ybar[0] = (bbar[1]*P[1]);
    ybar[1] = (P[2]*bbar[0]);
    (void)time; (void)P; (void)PD; (void)F; (void)bbar; (void)Fbar;
  }
};

}}  // namespace goss_b200::models
#endif
