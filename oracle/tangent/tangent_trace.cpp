// Test infrastructure -- NOT part of the product path.
//
// FP64 forward-mode tangent-linear reference for GRL1 and RK4 traces: the
// reference user loop forward(t0 + j*interval, interval), j < J, with S
// internal steps per interval -- GRL1::forward (GRL1.cpp:61-82; the step
// GRL1::_one_step, GRL1.h:72-84, threshold delta = 1e-8 of GRL1.h:39) or
// RK4::forward (RK4.cpp:68-102 with RK4::axpy, RK4.h:70-74) -- sampling one
// state after every interval, run in dual numbers.
// Each node carries up to D tangent directions, each the unit perturbation
// of one initial state or one field parameter, so the result is the exact
// Jacobian d trace[j] / d input (up to FP64 rounding) along the same branch
// of every conditional as the primal run.  It checks the reverse-mode
// adjoint kernels, whose transposed products must agree with it to rounding;
// central finite differences cannot, because conditionals such as the
// sodium-gate rates of ten Tusscher-Panfilov switch branches discontinuously.
//
// Compiled per model variant by oracle/pyoracle.py:
//   g++ -O2 -fopenmp -I oracle/tangent -I <variant dir>
//       -DGOSS_TANGENT_MODEL=M_<variant> -shared tangent_trace.cpp
// (oracle/tangent/goss_device_math.cuh stands in for the CUDA header, so the
// generated device.cuh compiles as host C++).
#include <cstdint>
#include <vector>

#include "goss_device_math.cuh"
#include "device.cuh"

#ifndef GOSS_TANGENT_MODEL
#error "compile with -DGOSS_TANGENT_MODEL=<device struct of the variant>"
#endif

namespace {

using namespace goss_b200::models;
using Model = GOSS_TANGENT_MODEL;

constexpr int kStates = Model::num_states;
constexpr int kFields = Model::num_field_params > 0 ? Model::num_field_params : 1;
constexpr int kParams = Model::num_params + Model::num_derived;

struct TraceArgs {
    uint32_t num_nodes;
    const double* states0;       // [N][n] node-major
    const double* field_params;  // [N][nfp] node-major (unused without fields)
    const double* params;        // [num_params + num_derived]: parameters then derived constants
    double t0, interval;
    uint32_t steps_per_interval, num_intervals, trace_state;
    uint32_t num_dirs;
    const uint32_t* dirs;        // direction k perturbs input dirs[k]: < n a state, else field dirs[k]-n
    int solver;                  // 0 GRL1, 1 RK4
    double delta;
    double* trace;               // [J][N]
    double* jacobian;            // [J][N][num_dirs]
};

template <int D>
void node_trace(const TraceArgs& a, uint32_t node)
{
    using T = Dual<D>;
    T y[kStates], F[kFields], lin[kStates], rhs[kStates];
    std::vector<T> P(kParams);
    for (int i = 0; i < kParams; ++i)
        P[i] = T(a.params[i]);
    for (int i = 0; i < kStates; ++i)
        y[i] = T(a.states0[(uint64_t)node * kStates + i]);
    for (int f = 0; f < Model::num_field_params; ++f)
        F[f] = T(a.field_params[(uint64_t)node * Model::num_field_params + f]);
    for (uint32_t k = 0; k < a.num_dirs; ++k) {
        const uint32_t d = a.dirs[k];
        if (d < (uint32_t)kStates)
            y[d].d[k] = 1.0;
        else
            F[d - kStates].d[k] = 1.0;
    }
    const uint32_t S = a.steps_per_interval;
    const double ldt = a.interval / S;
    for (uint32_t j = 0; j < a.num_intervals; ++j) {
        double lt = a.t0 + j * a.interval;
        for (uint32_t s = 0; s < S; ++s) {
            if (a.solver == 0) {
                for (int i = 0; i < kStates; ++i)
                    lin[i] = T(0.0);
                Model::template linearized<T>(y, lt, P.data(), a.params, F, lin, rhs);
                for (int i = 0; i < kStates; ++i)
                    y[i] = (gfabs(lin[i]) > a.delta) ? y[i] + rhs[i] / lin[i] * (gexp(lin[i] * ldt) - 1.0)
                                                     : y[i] + rhs[i] * ldt;
            } else {
                T k1[kStates], k2[kStates], k3[kStates], k4[kStates], tmp[kStates];
                Model::template rhs<T>(y, lt, P.data(), a.params, F, k1);
                for (int i = 0; i < kStates; ++i)
                    tmp[i] = y[i] + 0.5 * ldt * k1[i];
                Model::template rhs<T>(tmp, lt + 0.5 * ldt, P.data(), a.params, F, k2);
                for (int i = 0; i < kStates; ++i)
                    tmp[i] = y[i] + 0.5 * ldt * k2[i];
                Model::template rhs<T>(tmp, lt + 0.5 * ldt, P.data(), a.params, F, k3);
                for (int i = 0; i < kStates; ++i)
                    tmp[i] = y[i] + ldt * k3[i];
                Model::template rhs<T>(tmp, lt + ldt, P.data(), a.params, F, k4);
                for (int i = 0; i < kStates; ++i)
                    y[i] = y[i] + ldt * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]) / 6.0;
            }
            lt += ldt;
        }
        const T& v = y[a.trace_state];
        const uint64_t row = (uint64_t)j * a.num_nodes + node;
        a.trace[row] = v.v;
        for (uint32_t k = 0; k < a.num_dirs; ++k)
            a.jacobian[row * a.num_dirs + k] = v.d[k];
    }
}

template <int D>
void run(const TraceArgs& a)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t node = 0; node < (int64_t)a.num_nodes; ++node)
        node_trace<D>(a, (uint32_t)node);
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) int tangent_num_states() { return kStates; }
__attribute__((visibility("default"))) int tangent_num_field_params() { return Model::num_field_params; }
__attribute__((visibility("default"))) int tangent_num_params() { return Model::num_params; }
__attribute__((visibility("default"))) int tangent_num_derived() { return Model::num_derived; }

// solver: 0 GRL1, 1 RK4.  params: the model's num_params parameters followed
// by room for num_derived derived constants, which this call fills in.
// Returns 0, or -1 for bad arguments (more than 32 directions, a direction
// out of range, an unknown solver).
__attribute__((visibility("default"))) int tangent_trace(
    int solver, uint32_t num_nodes, const double* states0, const double* field_params, double* params, double t0,
    double interval, uint32_t steps_per_interval, uint32_t num_intervals, uint32_t trace_state,
    uint32_t num_dirs, const uint32_t* dirs, double delta, double* trace, double* jacobian)
{
    if (num_dirs > 32 || steps_per_interval == 0 || trace_state >= (uint32_t)kStates || solver < 0 || solver > 1)
        return -1;
    for (uint32_t k = 0; k < num_dirs; ++k)
        if (dirs[k] >= (uint32_t)(kStates + Model::num_field_params))
            return -1;
    Model::derived(params, params + Model::num_params);
    const TraceArgs a{num_nodes, states0, field_params, params, t0, interval, steps_per_interval,
                      num_intervals, trace_state, num_dirs, dirs, solver, delta, trace, jacobian};
    if (num_dirs <= 1) run<1>(a);
    else if (num_dirs <= 4) run<4>(a);
    else if (num_dirs <= 8) run<8>(a);
    else if (num_dirs <= 16) run<16>(a);
    else run<32>(a);
    return 0;
}

}  // extern "C"

// Single-evaluation checks of the generated model code (one state, one time):
//   tangent_jvp: (linear, rhs) and their directional derivatives along
//                (ydot, Fdot), by dual numbers through `linearized`;
//   tangent_vjp: ybar = abar^T d(linear)/dy + bbar^T d(rhs)/dy and Fbar, by
//                the generated reverse sweep `linearized_vjp` in FP64.
// A dot-product test <abar, lin_dot> + <bbar, rhs_dot> = <ybar, ydot> +
// <Fbar, Fdot> then checks the reverse sweep against forward mode.
// params as for tangent_trace (derived constants filled in here).
extern "C" {

__attribute__((visibility("default"))) int tangent_jvp(const double* y, const double* F, double* params,
                                                       double time, const double* ydot, const double* Fdot,
                                                       double* lin, double* rhs, double* lin_dot, double* rhs_dot)
{
    using T = Dual<1>;
    Model::derived(params, params + Model::num_params);
    std::vector<T> P(kParams);
    for (int i = 0; i < kParams; ++i)
        P[i] = T(params[i]);
    T yd[kStates], Fd[kFields], l[kStates], r[kStates];
    for (int i = 0; i < kStates; ++i) {
        yd[i] = T(y[i]);
        yd[i].d[0] = ydot[i];
        l[i] = T(0.0);
        r[i] = T(0.0);
    }
    for (int f = 0; f < Model::num_field_params; ++f) {
        Fd[f] = T(F[f]);
        Fd[f].d[0] = Fdot[f];
    }
    Model::template linearized<T>(yd, time, P.data(), params, Fd, l, r);
    for (int i = 0; i < kStates; ++i) {
        lin[i] = l[i].v;
        rhs[i] = r[i].v;
        lin_dot[i] = l[i].d[0];
        rhs_dot[i] = r[i].d[0];
    }
    return 0;
}

__attribute__((visibility("default"))) int tangent_vjp(const double* y, const double* F, double* params,
                                                       double time, const double* abar, const double* bbar,
                                                       double* ybar, double* Fbar)
{
    Model::derived(params, params + Model::num_params);
    double Fl[kFields] = {0.0};
    for (int f = 0; f < Model::num_field_params; ++f)
        Fl[f] = F[f];
    double yb[kStates], Fb[kFields];
    auto seed = [&](const double*, const double*, double* ab, double* bb) {
        for (int i = 0; i < kStates; ++i) {
            ab[i] = abar[i];
            bb[i] = bbar[i];
        }
    };
    Model::template linearized_vjp<double>(y, time, params, params, Fl, seed, yb, Fb);
    for (int i = 0; i < kStates; ++i)
        ybar[i] = yb[i];
    for (int f = 0; f < Model::num_field_params; ++f)
        Fbar[f] = Fb[f];
    return 0;
}

}  // extern "C"
