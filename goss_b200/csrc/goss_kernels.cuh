// sm_100a solver kernels of the multi-node solve path.
//
// One CUDA thread owns one mesh node for the whole call: its states are
// loaded once from the component-major FP64 arrays (states[i*ld + node],
// coalesced across the warp), kept in registers across every internal step
// of the interval, and stored once at the end.  Uniform model parameters
// travel in the kernel's parameter block (constant bank, read as free
// operands); per-node field parameters are loaded once into registers.
//
// Each kernel restates the arithmetic of one reference solver; the FP64
// instantiation follows the reference operation order so that it agrees with
// the FP64 CPU oracle to rounding.
//
//   explicit_kernel<M, T, ExplicitEuler>  cpp/goss/ExplicitEuler.cpp:64-87
//   explicit_kernel<M, T, RK4>            cpp/goss/RK4.cpp:68-102
//   explicit_kernel<M, T, GRL1>           cpp/goss/GRL1.cpp:61-82, GRL1.h:72-84
//   explicit_kernel<M, T, GRL2>           cpp/goss/GRL2.cpp:63-86
//   theta_kernel<M>                       cpp/goss/ThetaSolver.cpp:49-155,
//                                         ImplicitODESolver.cpp:92-262, ODE.cpp:47-132
//   esdirk_kernel<M>                      cpp/goss/ESDIRK23a.cpp:101-316
#ifndef GOSS_KERNELS_CUH
#define GOSS_KERNELS_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "goss_b200.h"
#include "goss_device_math.cuh"

namespace goss_b200 {

constexpr double kGossEps = 3.0e-16;  // GOSS_EPS, cpp/goss/constants.h:25

template <class M>
struct Dims {
    static constexpr int n = M::num_states;
    // parameter block: the model parameters followed by the derived constants
    static constexpr int npd = M::num_params + M::num_derived;
    static constexpr int np = npd > 0 ? npd : 1;
    static constexpr int nfp = M::num_field_params > 0 ? M::num_field_params : 1;
};

// Fill the FP64 parameter block: parameters, then the model's derived
// constants computed from them (once per launch, on the host).
template <class M>
inline void parameter_block(const double* params, double (&out)[Dims<M>::np])
{
    for (int i = 0; i < Dims<M>::np; ++i)
        out[i] = i < M::num_params ? params[i] : 0.0;
    if (M::num_derived > 0)
        M::derived(out, out + M::num_params);
}

// std::max / std::min semantics (first argument wins ties and NaNs)
__device__ __forceinline__ double std_max(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double std_min(double a, double b) { return (b < a) ? b : a; }

// ---------------------------------------------------------------------------
// kernel argument blocks (passed by value; __grid_constant__ keeps them in the
// parameter bank so indexing them costs no local-memory copy)
// ---------------------------------------------------------------------------
template <class M, typename T>
struct ExplicitArgs {
    double* states;
    const double* fparams;
    uint32_t* flags;
    uint8_t* node_status;
    uint64_t ld;
    uint64_t nsteps;
    double t;
    double ldt;
    double delta;
    uint32_t N;
    T P[Dims<M>::np];
    double PD[Dims<M>::np];
};

template <class M>
struct ImplicitArgs {
    double* states;
    const double* fparams;
    double* sstate;  // per-node solver state, [rows][ld]
    uint32_t* flags;
    uint8_t* node_status;
    uint64_t ld;
    uint64_t max_loop;
    double t;
    double interval;
    goss_solver_params sp;
    uint32_t N;
    double P[Dims<M>::np];
    float P32[Dims<M>::np];  // the same block in FP32 (the FP32 Jacobian of GOSS_FP32)
};

template <class M, typename T>
struct EvalArgs {
    const double* states;
    const double* fparams;
    const double* times;
    double* out;
    uint64_t ld;
    uint32_t N;
    int32_t what;
    T P[Dims<M>::np];
    double PD[Dims<M>::np];
};

// ---------------------------------------------------------------------------
// explicit solvers
// ---------------------------------------------------------------------------
// GRL1Printed: GRL1 with the model evaluated in its printed operation order
// (the arithmetic of the reference's generated model code), FP64 only.
enum class Explicit { Euler, RK4, GRL1, GRL2, RL1, RL2, RK2, GRL1Printed };

template <class M, typename T>
__device__ __forceinline__ void load_field(const double* __restrict__ fp, uint64_t ld, uint32_t node,
                                           T (&F)[Dims<M>::nfp])
{
#pragma unroll
    for (int k = 0; k < Dims<M>::nfp; ++k)
        F[k] = (k < M::num_field_params) ? T(fp[k * ld + node]) : T(0);
}

// GRL increment of one state, FP64: the reference expression
// b/a*(exp(a*h) - 1.0) or b*h (GRL1.h:80-83)
__device__ __forceinline__ double grl_increment(double a, double b, double h, double delta)
{
    return (fabs(a) > delta) ? b / a * (exp(a * h) - 1.0) : b * h;
}

// GRL increment of one state, FP32: b*h*phi1(a*h), algebraically identical
// and free of the cancellation in exp(a*h) - 1 (see phi1f).  (h phi1 with
// the polynomial's coefficients scaled by h, one multiply fewer per state,
// measured 1.4 % slower on B200: TP06, 1,048,576 nodes, 162 registers
// instead of 150.)
__device__ __forceinline__ float grl_increment(float a, float b, float h, float /*delta*/)
{
    return b * h * phi1f(a * h);
}

// RL increment of one state (RL1.h:68-77): the exponential form for the model's
// linear-term states whatever the coefficient (the reference divides by it),
// the Euler increment otherwise
__device__ __forceinline__ double rl_increment(bool linear, double a, double b, double h)
{
    return linear ? b / a * (exp(a * h) - 1.0) : b * h;
}
__device__ __forceinline__ float rl_increment(bool linear, float a, float b, float h)
{
    return linear ? b * h * phi1f(a * h) : b * h;
}

// State accumulators.  FP64 kernels hold each state as a double and update it
// exactly as the reference does (y = y + increment).  FP32 kernels hold each
// state as an unevaluated sum hi + lo of two floats with compensated (Kahan)
// updates: the model reads hi, lo carries what hi could not absorb, so
// increments far below one float ulp of the state (K_i ~ 138 mM changes by
// less than one ulp per step) still accumulate.  Four FP32 adds per update,
// no FP32<->FP64 conversions (those would compete with the model's
// exponentials and reciprocals for the XU pipe on every step).
template <typename T>
struct Acc;

template <>
struct Acc<double> {
    double y;
    __device__ __forceinline__ void load(double v) { y = v; }
    __device__ __forceinline__ double store() const { return y; }
    __device__ __forceinline__ double value() const { return y; }
    __device__ __forceinline__ double plus(double d) const { return y + d; }
    __device__ __forceinline__ void add(double d) { y = y + d; }
    __device__ __forceinline__ void renormalize() {}
};

template <>
struct Acc<float> {
    float hi, lo;
    __device__ __forceinline__ void load(double v)
    {
        hi = float(v);
        lo = float(v - double(hi));
    }
    __device__ __forceinline__ double store() const { return double(hi) + double(lo); }
    __device__ __forceinline__ float value() const { return hi; }
    __device__ __forceinline__ float plus(float d) const { return hi + (lo + d); }
    __device__ __forceinline__ void add(float d)
    {
        // hi + lo + d: the sum goes to hi, its rounding error (exact when
        // |hi| >= |y|, Fast2Sum) back to lo
        const float y = __fadd_rn(d, lo);
        const float t = __fadd_rn(hi, y);
        lo = __fsub_rn(y, __fsub_rn(t, hi));
        hi = t;
    }
    // between two forwards of one launch: bit for bit what store() to the
    // FP64 state array and load() by the next launch do, in FP32 arithmetic
    // (five FP64 conversions per state would double the XU pipe's work on a
    // one-step forward).  hi' = hi + lo rounded to FP32 and e its exact error
    // (two-sum); the FP64 round trip keeps e only to the FP64 grid of hi + lo,
    // g = 2^(floor(log2|hi + lo|) - 52), so e is rounded to a multiple of g
    // (ties to even) by adding and subtracting P = 2^23 g with e's sign, which
    // is exact for |e| < P; larger e are multiples of g already.  The binade
    // of hi + lo is that of hi' + e rounded toward zero (one below hi' when
    // hi' is a power of two and e has the opposite sign).  Sums below 2^-72
    // (where flushed FP32 subnormals would differ from the FP64 grid) and
    // non-finite sums take the FP64 round trip itself.
    __device__ __forceinline__ void renormalize()
    {
        const float t = __fadd_rn(hi, lo);
        const float at = fabsf(t);
        if (!(at >= 0x1p-72f && at <= 3.402823466e38f)) {
            load(store());
            return;
        }
        const float bp = __fsub_rn(t, hi);
        const float ap = __fsub_rn(t, bp);
        const float e = __fadd_rn(__fsub_rn(hi, ap), __fsub_rn(lo, bp));
        const float pow2 = __uint_as_float(__float_as_uint(__fadd_rz(t, e)) & 0x7f800000u);
        const float P = __fmul_rn(pow2, 0x1p-29f);
        const float C = copysignf(P, e);
        const float r = __fsub_rn(__fadd_rn(e, C), C);
        lo = fabsf(e) < P ? r : e;
        hi = t;
    }
};

// Where one node's explicit solve reads and writes (shared by the
// single-population kernel and the batched kernel of goss_batch.cuh).
struct NodeIO {
    double* states;         // [n][ld]
    const double* fparams;  // [nfp][ld]
    uint8_t* node_status;   // [ld]
    uint32_t* flags;
    uint64_t ld;
    uint64_t nsteps;        // internal steps of one forward
    double t;
    double ldt;
    double delta;
    // consecutive forwards of one launch: forward f starts at
    // t + (first + f) * interval (the host loop's t0 + k * interval)
    uint32_t forwards = 1;
    uint64_t first = 0;
    double interval = 0.0;
};

// The model evaluations the explicit steps use: the split forms (every
// distinct transcendental and reciprocal of a state-dependent operand
// evaluated once), in FP32 and in FP64.  The split FP64 programs change the
// reference's results by re-association only; they stay within 1e-10 of the
// reference over 10^5 TP06 GRL1 steps.  Printed = true takes the programs in
// the printed operation order of the model (one exp per occurrence, divisions
// as written), the arithmetic of the reference's own generated code.
template <class M, typename T, bool Printed = false>
__device__ __forceinline__ void model_linearized(const T* y, double t, const T* P, const double* PD, const T* F,
                                                 T* lin, T* rhs)
{
    if constexpr (Printed)
        M::template linearized<T>(y, t, P, PD, F, lin, rhs);
    else
        M::template linearized_split<T>(y, t, P, PD, F, lin, rhs);
}
template <class M, typename T>
__device__ __forceinline__ void model_rhs(const T* y, double t, const T* P, const double* PD, const T* F, T* f)
{
    M::template rhs_split<T>(y, t, P, PD, F, f);
}

// One internal step of an explicit solver at time lt with step ldt, in place
// on the accumulated states (shared by the solver kernels and the adjoint
// kernels' record and recompute passes, so all take identical arithmetic).
template <class M, typename T, Explicit S>
__device__ __forceinline__ void explicit_step(Acc<T>* y, const double lt, const double ldt, const T* __restrict__ P,
                                              const double* __restrict__ PD, const T* __restrict__ F, const T delta)
{
    constexpr int n = M::num_states;
    const T h = T(ldt);
    const T hh = T(0.5 * ldt);
    T yt[n];
#pragma unroll
    for (int i = 0; i < n; ++i)
        yt[i] = y[i].value();
    if constexpr (S == Explicit::Euler) {
        // ExplicitEuler.cpp:80-81
        T f[n];
        model_rhs<M, T>(yt, lt, P, PD, F, f);
#pragma unroll
        for (int i = 0; i < n; ++i)
            y[i].add(h * f[i]);
    } else if constexpr (S == Explicit::RK4) {
        // RK4.cpp:79-98 with RK4::axpy (RK4.h:70-74); the weighted sum is
        // accumulated in the order k1 + 2 k2 + 2 k3 + k4 of the reference.
        T k[n], sum[n], tmp[n];
        model_rhs<M, T>(yt, lt, P, PD, F, k);
#pragma unroll
        for (int i = 0; i < n; ++i) {
            sum[i] = k[i];
            tmp[i] = y[i].plus(hh * k[i]);
        }
        model_rhs<M, T>(tmp, lt + 0.5 * ldt, P, PD, F, k);
#pragma unroll
        for (int i = 0; i < n; ++i) {
            sum[i] = sum[i] + T(2.0) * k[i];
            tmp[i] = y[i].plus(hh * k[i]);
        }
        model_rhs<M, T>(tmp, lt + 0.5 * ldt, P, PD, F, k);
#pragma unroll
        for (int i = 0; i < n; ++i) {
            sum[i] = sum[i] + T(2.0) * k[i];
            tmp[i] = y[i].plus(h * k[i]);
        }
        model_rhs<M, T>(tmp, lt + ldt, P, PD, F, k);
#pragma unroll
        for (int i = 0; i < n; ++i) {
            sum[i] = sum[i] + k[i];
            y[i].add(h * sum[i] / T(6.0));
        }
    } else if constexpr (S == Explicit::GRL1) {
        // GRL1.h:72-84
        T lin[n], rhs[n];
        model_linearized<M, T>(yt, lt, P, PD, F, lin, rhs);
#pragma unroll
        for (int i = 0; i < n; ++i)
            y[i].add(grl_increment(lin[i], rhs[i], h, delta));
    } else if constexpr (S == Explicit::GRL1Printed) {
        // GRL1.h:72-84 over the printed model program
        T lin[n], rhs[n];
        model_linearized<M, T, true>(yt, lt, P, PD, F, lin, rhs);
#pragma unroll
        for (int i = 0; i < n; ++i)
            y[i].add(grl_increment(lin[i], rhs[i], h, delta));
    } else if constexpr (S == Explicit::GRL2) {
        // GRL2: GRL2.cpp:78-82.  The reference's branch threshold is a
        // self-initialised local (GRL2.cpp:67) whose -O3 build behaves as 0:
        // the exponential form is used whenever the linear term is non-zero.
        T lin[n], rhs[n], y2[n];
        model_linearized<M, T>(yt, lt, P, PD, F, lin, rhs);
#pragma unroll
        for (int i = 0; i < n; ++i)
            y2[i] = y[i].plus(grl_increment(lin[i], rhs[i], hh, T(0)));
        model_linearized<M, T>(y2, lt, P, PD, F, lin, rhs);
#pragma unroll
        for (int i = 0; i < n; ++i)
            y[i].add(grl_increment(lin[i], rhs[i], h, T(0)));
    } else if constexpr (S == Explicit::RL1) {
        // RL1.h:68-77
        T lin[n], rhs[n];
        model_linearized<M, T>(yt, lt, P, PD, F, lin, rhs);
#pragma unroll
        for (int i = 0; i < n; ++i)
            y[i].add(rl_increment(M::linear_term(i), lin[i], rhs[i], h));
    } else if constexpr (S == Explicit::RL2) {
        // RL2.cpp:78-83: a half step to y2 linearised at y, then the full step
        // from y linearised at y2, both at time lt
        T lin[n], rhs[n], y2[n];
        model_linearized<M, T>(yt, lt, P, PD, F, lin, rhs);
#pragma unroll
        for (int i = 0; i < n; ++i)
            y2[i] = y[i].plus(rl_increment(M::linear_term(i), lin[i], rhs[i], hh));
        model_linearized<M, T>(y2, lt, P, PD, F, lin, rhs);
#pragma unroll
        for (int i = 0; i < n; ++i)
            y[i].add(rl_increment(M::linear_term(i), lin[i], rhs[i], h));
    } else {
        // RK2: RK2.cpp:78-89 with RK2::axpy (RK2.h:70-74), the midpoint rule
        static_assert(S == Explicit::RK2, "unhandled explicit solver");
        T k[n], tmp[n];
        model_rhs<M, T>(yt, lt, P, PD, F, k);
#pragma unroll
        for (int i = 0; i < n; ++i)
            tmp[i] = y[i].plus(hh * k[i]);
        model_rhs<M, T>(tmp, lt + 0.5 * ldt, P, PD, F, k);
#pragma unroll
        for (int i = 0; i < n; ++i)
            y[i].add(h * k[i]);
    }
}

// Advance one node over nsteps internal steps of one explicit solver, from
// its accumulated states and field parameters, and store the result.
template <class M, typename T, Explicit S>
__device__ __forceinline__ void explicit_node_core(const NodeIO& a, uint32_t node, const T* __restrict__ P,
                                                   const double* __restrict__ PD, Acc<T>* y, const T* F)
{
    constexpr int n = M::num_states;
    const double ldt = a.ldt;
    const T delta = T(a.delta);
    for (uint32_t f = 0; f < a.forwards; ++f) {
        if (f) {
#pragma unroll
            for (int i = 0; i < n; ++i)
                y[i].renormalize();
        }
        // rounded like the host's t0 + k * interval (no fused multiply-add)
        double lt = __dadd_rn(a.t, __dmul_rn(double(a.first + f), a.interval));
        for (uint64_t step = 0; step < a.nsteps; ++step) {
            explicit_step<M, T, S>(y, lt, ldt, P, PD, F, delta);
            lt += ldt;
        }
    }
    bool finite = true;
#pragma unroll
    for (int i = 0; i < n; ++i) {
        const double v = y[i].store();
        a.states[i * a.ld + node] = v;
        finite = finite && isfinite(v);
    }
    if (!finite) {
        a.node_status[node] |= GOSS_FLAG_NONFINITE;
        atomicOr(a.flags, GOSS_FLAG_NONFINITE);
    }
}

// ... reading the node's states and field parameters from global memory
template <class M, typename T, Explicit S>
__device__ __forceinline__ void explicit_node(const NodeIO& a, uint32_t node, const T* __restrict__ P,
                                              const double* __restrict__ PD)
{
    constexpr int n = M::num_states;
    Acc<T> y[n];
#pragma unroll
    for (int i = 0; i < n; ++i)
        y[i].load(a.states[i * a.ld + node]);
    T F[Dims<M>::nfp];
    load_field<M, T>(a.fparams, a.ld, node, F);
    explicit_node_core<M, T, S>(a, node, P, PD, y, F);
}

// ... reading them from rows[r * stride]: the n state rows, then the field
// parameter rows (a tile staged in shared memory by the batch kernel)
template <class M, typename T, Explicit S>
__device__ __forceinline__ void explicit_node_from(const NodeIO& a, uint32_t node, const T* __restrict__ P,
                                                   const double* __restrict__ PD, const double* rows,
                                                   uint32_t stride)
{
    constexpr int n = M::num_states;
    Acc<T> y[n];
#pragma unroll
    for (int i = 0; i < n; ++i)
        y[i].load(rows[i * stride]);
    T F[Dims<M>::nfp];
#pragma unroll
    for (int k = 0; k < Dims<M>::nfp; ++k)
        F[k] = (k < M::num_field_params) ? T(rows[(n + k) * stride]) : T(0);
    explicit_node_core<M, T, S>(a, node, P, PD, y, F);
}

// Resident blocks of 128 threads per SM the explicit kernels are compiled for
// (register cap 65536 / (128 * blocks)).  FP64: 3 for the one-evaluation
// steps (170 registers), 4 for those with two or more evaluations (128
// registers): measured on B200 (TP06, 1,048,576 nodes, four fields) against
// the uncapped 255 registers, GRL1 3.55e9 -> 4.10e9 cell-steps/s (4: 3.90e9),
// GRL2 1.09e9 -> 1.82e9 (3: 1.57e9); more warps hide the FP64 latencies
// better than the spills cost.  FP32: uncapped (150 registers for TP06 GRL1,
// 3 blocks per SM); capping it at 128 registers measured 2.77e10 against
// 2.91e10 cell-steps/s.
#ifndef GOSS_EXPLICIT_MIN_BLOCKS_FP32
#define GOSS_EXPLICIT_MIN_BLOCKS_FP32 1
#endif
template <typename T, Explicit S>
struct ExplicitMinBlocks {
    static constexpr bool one_eval = S == Explicit::Euler || S == Explicit::GRL1 || S == Explicit::RL1 ||
                                     S == Explicit::GRL1Printed;
    static constexpr int value = sizeof(T) == 4 ? GOSS_EXPLICIT_MIN_BLOCKS_FP32 : (one_eval ? 3 : 4);
};

template <class M, typename T, Explicit S>
__global__ void __launch_bounds__(128, (ExplicitMinBlocks<T, S>::value))
    explicit_kernel(const __grid_constant__ ExplicitArgs<M, T> a)
{
    const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= a.N)
        return;
    const NodeIO io{a.states, a.fparams, a.node_status, a.flags, a.ld, a.nsteps, a.t, a.ldt, a.delta};
    explicit_node<M, T, S>(io, node, a.P, a.PD);
}

// ---------------------------------------------------------------------------
// dense linear algebra on one node's n x n matrix
// ---------------------------------------------------------------------------
// Newton matrices of the implicit solvers are stored packed (the model's
// lu_nnz entries of the LU structure of I - h*alpha*J, generated with the
// structure-aware factorisation and solve that reproduce ODE::lu_factorize and
// ODE::forward_backward_subst, ODE.cpp:69-132): in a thread-local array, or in
// a node's slice of component-major solver-state rows (entry k of the node at
// base[k*ld + node]).
struct PackedRows {
    double* base;
    uint64_t ld;
    __device__ __forceinline__ double& operator[](int k) const { return base[(uint64_t)k * ld]; }
};

// ... or in a tiled region: the 32 nodes of a tile keep their entries together
// ([tile][k][32]), so a warp's lu_nnz entries are one contiguous block of
// 256-byte rows instead of lu_nnz rows ld apart (each 2 MiB apart at 262,144
// nodes, whose cost depended on how the allocation happened to be mapped)
struct PackedTile {
    double* base;
    __device__ __forceinline__ double& operator[](int k) const { return base[(uint64_t)k * 32]; }
};

__device__ __forceinline__ PackedTile packed_tile(double* region, uint32_t node, int nnz)
{
    return PackedTile{region + (((uint64_t)(node >> 5) * (uint64_t)nnz) << 5) + (node & 31u)};
}

template <int n>
__device__ __forceinline__ double l2norm(const double* v)
{
    double s = 0;
#pragma unroll
    for (int i = 0; i < n; ++i)
        s += v[i] * v[i];
    return sqrt(s);
}

// FP64 model right-hand side of the implicit solvers: the split form (every
// distinct exp and reciprocal once, common factors pulled out), whose values
// differ from the reference's operation order by rounding only; Newton
// iterates to the same states (the implicit parity tests hold at 1e-10), and
// the FD Jacobian, ~19 evaluations per Newton iteration, gets ~2x cheaper.
#ifndef GOSS_IMPLICIT_SPLIT
#define GOSS_IMPLICIT_SPLIT 1
#endif
// Inlined at every call site: on TT04 with the analytic Jacobian, called
// (__noinline__) versions of these two measured 1.3x slower, and capping the
// kernels at 128 or 170 registers (3 or 4 blocks of 128 per SM) 1.3-1.4x
// slower, than the 255-register inlined kernel.
template <class M>
__device__ __forceinline__ void rhs64(const double* y, double t, const double* P, const double* F, double* out)
{
    if constexpr (GOSS_IMPLICIT_SPLIT)
        M::template rhs_split<double>(y, t, P, P, F, out);
    else
        M::template rhs<double>(y, t, P, P, F, out);
}

template <class M, class A>
__device__ __forceinline__ void jacobian64(const double* y, double t, const double* P, const double* F, A J)
{
    M::template jacobian<double>(y, t, P, P, F, J);
}

// The analytic Jacobian evaluated in FP32 at the FP64 point (y, t) and stored
// into the FP64 packed Newton matrix: the implicit solvers' GOSS_FP32 mode.
// The matrix only steers the simplified Newton iteration (the residual, the
// right-hand sides, the LU and the updates stay FP64), so the iteration
// converges to the same tolerance with an FP32-accurate matrix.
template <class M, class A>
__device__ __forceinline__ void jacobian32(const double* y, double t, const float* P32, const double* PD,
                                           const double* F, A J)
{
    float yf[M::num_states];
#pragma unroll
    for (int i = 0; i < M::num_states; ++i)
        yf[i] = float(y[i]);
    float Ff[Dims<M>::nfp];
#pragma unroll
    for (int k = 0; k < Dims<M>::nfp; ++k)
        Ff[k] = float(F[k]);
    M::template jacobian<float>(yf, t, P32, PD, Ff, J);
}

// ODE::compute_jacobian (ODE.cpp:47-67) into the packed Newton matrix J:
// the model's analytic Jacobian when it was generated with one (the
// reference's generated override), else forward differences: column i is
// (f(y + delta_i e_i) - f(y)) / delta_i with delta_i = sqrt(1e-15 max(1e-5, |y_i|)),
// f1 = f(y, t) supplied by the caller (the reference evaluates it first with
// the same arguments), stored at the column's structural rows (the other
// rows are exactly 0 in the reference too).  The perturbed state is built by
// selects over compile-time indices, so y stays in registers (the reference
// perturbs y[i] in place and restores it: the same values).  With the split
// right-hand side, the generated fd_jacobian evaluates it once at y and, for
// each column i, recomputes only the statements of the column's structural
// rows that depend on state i (the others keep the values a full
// re-evaluation would give).  Measured on B200 (TT04, 262,144 nodes, 0.1 ms
// intervals): ThetaSolver 4.43 ms per interval with n full evaluations, 3.61
// with the rows of each column's structure, 1.62 with the cones; ESDIRK23a
// 258 -> 219 ms.
template <class M, class A>
__device__ __forceinline__ void compute_jacobian(const double* y, double t, const double* P, const double* F, A J,
                                                 const double* f1)
{
    constexpr int n = M::num_states;
    if constexpr (M::has_jacobian) {
        (void)f1;
        jacobian64<M>(y, t, P, F, J);
    } else if constexpr (GOSS_IMPLICIT_SPLIT) {
        M::fd_clear(J);
        M::template fd_jacobian<double>(y, t, P, P, F, f1, J);
    } else {
        M::fd_clear(J);
#pragma unroll 1
        for (int i = 0; i < n; ++i) {
            double ysafe = 0.0;
#pragma unroll
            for (int k = 0; k < n; ++k)
                ysafe = (k == i) ? y[k] : ysafe;
            const double max = 1e-5 > fabs(ysafe) ? 1e-5 : fabs(ysafe);
            const double delta = sqrt(1e-15 * max);
            double yp[n], f2[n];
#pragma unroll
            for (int k = 0; k < n; ++k)
                yp[k] = (k == i) ? ysafe + delta : y[k];
            rhs64<M>(yp, t, P, F, f2);
            M::fd_column(i, f1, f2, delta, J);
        }
    }
}

// ---------------------------------------------------------------------------
// ThetaSolver
// ---------------------------------------------------------------------------
// per-node solver state rows
enum ThetaRows { TH_ETA = 0, TH_RECOMPUTE, TH_ALWAYS, TH_JUSTREFINED, TH_JACCOMP, TH_REJECTS, TH_ACCEPTED, TH_ROWS };

// ThetaSolver::forward (ThetaSolver.cpp:49-155); with IE, ImplicitEuler::forward
// (ImplicitEuler.cpp:57-152): theta = 1 (no explicit part, stage time t + ldt),
// the Jacobian always recomputed once MORE than num_refinements_without_
// always_recomputing_jacobian refinements happened (Theta: up to that many),
// and a failed step requests a new Jacobian.
// Lockstep form: every pass of the block-uniform loop runs one Newton
// iteration of every node that is not done (starting its next step first
// when the previous one ended), then the block synchronises, so the block's
// warps walk the large inlined right-hand side, Jacobian and LU together and
// share instruction-cache lines.  The per-node arithmetic and its order are
// those of the nested loops of ThetaSolver::forward (the states equal the
// nested-loop kernel's bit for bit).  Measured on B200 (TT04, 262,144 nodes,
// 0.1 ms intervals, blocks of 256 against the nested loops in blocks of 64):
// ImplicitEuler with the analytic Jacobian 2.49 -> 1.53 ms, ThetaSolver with
// it 1.24 -> 1.16 ms, with forward differences unchanged (4.41 ms).  Again
// with one model evaluation site per iteration (below), against each warp
// looping on its own (__any_sync): ImplicitEuler 1.03 against 1.33 ms (1.56
// against 2.36 with forward differences), ThetaSolver within 2 %.  Blocks of
// up to 256 threads; __launch_bounds__(256, 1) keeps the 255-register budget
// (without the minimum of one block ptxas capped it at 128 and spilled more).
//
// Launch shape: at most GOSS_THETA_THREADS threads per block, compiled for
// GOSS_THETA_MIN_BLOCKS resident blocks per SM (register cap 65536 / product).
// Measured on B200 (TT04 with the analytic Jacobian, 262,144 nodes, 0.1 ms
// intervals): 256 x 1 with the Newton matrix, z1 and prev in registers and
// local memory 0.61 ms per interval; the same with them in dynamic shared
// memory 0.77 ms (the DRAM spill traffic disappears, but the shared memory
// takes the L1 capacity the remaining spills hit in); the matrix alone in
// shared memory 0.79 ms, and in blocks of 128 x 3 (168 registers) 0.92 ms.
#ifndef GOSS_THETA_THREADS
#define GOSS_THETA_THREADS 256
#endif
#ifndef GOSS_THETA_MIN_BLOCKS
#define GOSS_THETA_MIN_BLOCKS 1
#endif
#ifndef GOSS_THETA_ONE_EVAL
#define GOSS_THETA_ONE_EVAL 1
#endif
template <class M, bool IE, bool J32 = false>
__global__ void __launch_bounds__(GOSS_THETA_THREADS, GOSS_THETA_MIN_BLOCKS)
    theta_kernel(const __grid_constant__ ImplicitArgs<M> a)
{
    constexpr int n = M::num_states;
    // One inlined copy of the model evaluation where that is faster (an
    // instruction-cache effect: the per-node code is far larger than the
    // cache).  ImplicitEuler, which keeps its Jacobian and mostly evaluates
    // f alone: every iteration through rhs_jacobian_sel or rhs_fd_jacobian_sel
    // (the Jacobian's own statements under a run-time condition).
    // ThetaSolver with the analytic Jacobian, which refactorises in (nearly)
    // every iteration: every refactorising iteration through rhs2_jacobian,
    // f(y, t) used at a step's first iteration only (the time-dependent
    // statements are evaluated at t each time).  Measured (TT04, 262,144
    // nodes, 0.1 ms intervals, A/B in one process): ImplicitEuler 1.30 -> 1.04
    // ms per interval with the analytic Jacobian, 1.88 -> 1.54 ms with forward
    // differences; ThetaSolver with the analytic Jacobian 0.61 -> 0.55 ms
    // (through rhs_jacobian_sel instead: 0.69 ms, the Jacobian's statements no
    // longer interleave with f's; with forward differences through
    // rhs2_fd_jacobian: 1.5 % slower, not used).
    constexpr bool one_eval = GOSS_THETA_ONE_EVAL && GOSS_IMPLICIT_SPLIT && !J32 && IE;
    constexpr bool one_jac = GOSS_THETA_ONE_EVAL && GOSS_IMPLICIT_SPLIT && !J32 && !IE && M::has_jacobian;
    // ImplicitEuler with the FP32 Jacobian: one FP64 right-hand-side call
    // site for every iteration, the FP32 Jacobian when refactorising (1.22 ->
    // 0.77 ms per interval; for ThetaSolver, with f(y, t) of a step's first
    // iteration from the same call site, 0.57 -> 0.73 ms, not used)
    constexpr bool one_eval32 = GOSS_THETA_ONE_EVAL && GOSS_IMPLICIT_SPLIT && J32 && IE;
    const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = node < a.N;
    const uint32_t src = active ? node : a.N - 1;  // threads past the end only take part in the barriers
    const goss_solver_params& sp = a.sp;
    double y[n], z1[n], prev[n], yz[n], f1[n], b[n];
    double J[M::lu_nnz];
    for (int i = 0; i < n; ++i)
        y[i] = a.states[i * a.ld + src];
    double F[Dims<M>::nfp];
    load_field<M, double>(a.fparams, a.ld, src, F);
    double* ss = a.sstate + src;
    const uint64_t ld = a.ld;
    double eta = ss[TH_ETA * ld];
    int recompute = ss[TH_RECOMPUTE * ld] != 0.0;
    int always = ss[TH_ALWAYS * ld] != 0.0;
    int justrefined = ss[TH_JUSTREFINED * ld] != 0.0;
    double jac_comp = ss[TH_JACCOMP * ld], rejects = ss[TH_REJECTS * ld], accepted = ss[TH_ACCEPTED * ld];
    double* const jrows = ss + (uint64_t)TH_ROWS * ld;
    if constexpr (IE) {
#pragma unroll
        for (int k = 0; k < M::lu_nnz; ++k)
            J[k] = jrows[(uint64_t)k * ld];
    }

    double t = a.t;
    const double dt = a.interval;
    const double t_end = t + dt;
    const double ldt_0 = sp.ldt;
    double ldt = ldt_0 > 0 ? ldt_0 : dt;
    int num_refinements = 0;
    const double eps = kGossEps * 1000;
    uint8_t status = 0;
    for (int i = 0; i < n; ++i)
        prev[i] = 0.0;
    uint64_t guard = 0;
    // the step in progress and its Newton iteration state
    bool done = !active, in_step = false, step_ok = true, prev_pending = false;
    double tn = 0.0, alpha = 1.0;
    int newton_iterations = 0;
    double relative_previous_residual = 1.0, relative_residual = 1.0, previous_residual = 1.0;
    double initial_residual = 1.0, residual;
    while (__syncthreads_or(!done)) {
        if (done)
            continue;
        if (!in_step) {
            if (++guard > a.max_loop) {
                status |= GOSS_FLAG_ITERATION_CAP;
                done = true;
                continue;
            }
            for (int i = 0; i < n; ++i)
                z1[i] = 0.0;
            if (IE ? num_refinements > sp.num_refinements_without_always_recomputing_jacobian
                   : num_refinements <= sp.num_refinements_without_always_recomputing_jacobian)
                always = 1;
            tn = IE ? t + ldt : t + sp.theta * ldt;
            alpha = IE ? 1.0 : sp.theta;
            step_ok = true;
            newton_iterations = 0;
            relative_previous_residual = relative_residual = previous_residual = initial_residual = 1.0;
            // (1 - theta) f(y, t): when the step's first Newton iteration will
            // refactorise, its f(y, tn) evaluation writes f(y, t) as well
            prev_pending = false;
            if (!IE && fabs(sp.theta - 1.0) > kGossEps) {
                if (one_eval32 || (GOSS_IMPLICIT_SPLIT && !(relative_residual < sp.relative_tolerance) &&
                                   (recompute || always))) {
                    prev_pending = true;
                } else {
                    rhs64<M>(y, t, a.P, F, f1);
                    for (int i = 0; i < n; ++i)
                        prev[i] = (1 - sp.theta) * f1[i];
                }
            }
            in_step = true;
        }
        // one iteration of ImplicitODESolver::newton_solve (ImplicitODESolver.cpp:114-245)
        bool newton_done = false;
        for (int i = 0; i < n; ++i)
            yz[i] = y[i] + z1[i];
        // when this iteration will refactorise (both conditions are known
        // before f(yz) is evaluated), f(yz) and the Jacobian come from one
        // evaluation: the unperturbed statements of the forward differences,
        // or the statements the analytic Jacobian shares with f
        constexpr bool fused = GOSS_IMPLICIT_SPLIT;
        if constexpr (one_eval32) {
            const bool want_jac = !(relative_residual < sp.relative_tolerance) && (recompute || always);
            // at a step's first iteration (yz = y) f(y, t) for the explicit part, then f(yz, tn)
#pragma unroll 1
            for (int k = (!IE && prev_pending) ? 0 : 1; k < 2; ++k) {
                double g[n];
                rhs64<M>(yz, k == 0 ? t : tn, a.P, F, g);
#pragma unroll
                for (int i = 0; i < n; ++i) {
                    if (k == 0)
                        prev[i] = (1 - sp.theta) * g[i];
                    else
                        f1[i] = g[i];
                }
            }
            prev_pending = false;
            if (want_jac)
                jacobian32<M>(yz, tn, a.P32, a.P, F, J);
        } else if constexpr (one_eval) {
            // f(yz, tn), and the Jacobian when this iteration refactorises
            const bool want_jac = !(relative_residual < sp.relative_tolerance) && (recompute || always);
            if constexpr (M::has_jacobian)
                M::template rhs_jacobian_sel<double>(yz, tn, a.P, a.P, F, t, false, want_jac, b, f1, J);
            else
                M::template rhs_fd_jacobian_sel<double>(yz, tn, a.P, a.P, F, want_jac, f1, J);
        } else if (fused && !(relative_residual < sp.relative_tolerance) && (recompute || always)) {
            if constexpr (J32) {
                // FP64 right-hand sides, the FP32 Jacobian
                if (!IE && prev_pending) {
                    rhs64<M>(yz, t, a.P, F, b);
                    for (int i = 0; i < n; ++i)
                        prev[i] = (1 - sp.theta) * b[i];
                    prev_pending = false;
                }
                rhs64<M>(yz, tn, a.P, F, f1);
                jacobian32<M>(yz, tn, a.P32, a.P, F, J);
            } else if (!IE && (one_jac || prev_pending)) {
                // f(yz, t) into b: at the first iteration of the step (yz = y)
                // the explicit part
                if constexpr (M::has_jacobian) {
                    M::template rhs2_jacobian<double>(yz, tn, a.P, a.P, F, t, b, f1, J);
                } else {
                    M::fd_clear(J);
                    M::template rhs2_fd_jacobian<double>(yz, tn, a.P, a.P, F, t, b, f1, J);
                }
                if (prev_pending) {
                    for (int i = 0; i < n; ++i)
                        prev[i] = (1 - sp.theta) * b[i];
                    prev_pending = false;
                }
            } else if constexpr (M::has_jacobian) {
                M::template rhs_jacobian<double>(yz, tn, a.P, a.P, F, f1, J);
            } else {
                M::fd_clear(J);
                M::template rhs_fd_jacobian<double>(yz, tn, a.P, a.P, F, f1, J);
            }
        } else {
            rhs64<M>(yz, tn, a.P, F, f1);
        }
        for (int i = 0; i < n; ++i)
            b[i] = -z1[i] * 1.0 + ldt * (prev[i] + alpha * f1[i]);
        residual = l2norm<n>(b);
        if (relative_residual < sp.relative_tolerance) {
            newton_done = true;
        } else {
            if (recompute || always) {
                if constexpr (!fused)
                    compute_jacobian<M>(yz, tn, a.P, F, J, f1);
                M::lu_shift(J, -ldt * alpha);
                M::lu_factorize(J);
                jac_comp += 1;
                recompute = 0;
            }
            M::lu_solve(J, b, b);
            if (newton_iterations == 0) {
                initial_residual = residual;
                eta = eta > kGossEps ? eta : kGossEps;
                eta = pow(eta, 0.8);
            } else {
                relative_previous_residual = residual / previous_residual;
                recompute = relative_previous_residual >= sp.max_relative_previous_residual;
                if (relative_previous_residual >= 1) {
                    step_ok = false;
                    rejects += 1;
                    recompute = 1;
                    newton_done = true;
                } else {
                    const double scaled = std_max(
                        pow(relative_previous_residual, (double)(sp.max_iterations - newton_iterations)), kGossEps);
                    if (residual > (sp.kappa * sp.relative_tolerance * (1 - relative_previous_residual) / scaled))
                        recompute = 1;
                    eta = relative_previous_residual / (1.0 - relative_previous_residual);
                }
            }
            if (!newton_done && newton_iterations > sp.max_iterations) {
                recompute = 1;
                rejects += 1;
                step_ok = false;
                newton_done = true;
            }
            if (!newton_done) {
                for (int i = 0; i < n; ++i)
                    z1[i] += b[i];
                relative_residual = residual / initial_residual;
                previous_residual = residual;
                newton_iterations++;
                newton_done = !(eta * relative_residual >= sp.kappa * sp.relative_tolerance);
            }
        }
        if (!newton_done)
            continue;
        in_step = false;
        if (step_ok) {
            for (int i = 0; i < n; ++i)
                y[i] += z1[i];
            t += ldt;
            accepted += 1;
            if (fabs(t - t_end) < eps) {
                done = true;
                continue;
            }
            if (!justrefined) {
                const double tmp = 2.0 * ldt;
                if (ldt_0 > 0. && tmp >= ldt_0)
                    ldt = ldt_0;
                else
                    ldt = tmp;
            } else {
                justrefined = 0;
            }
            if ((t + ldt + kGossEps) > t_end)
                ldt = t_end - t;
        } else {
            ldt /= 2.0;
            if (ldt < sp.min_dt) {
                status |= GOSS_FLAG_NEWTON_FAILED;
                done = true;
                continue;
            }
            if (IE)
                recompute = 1;
            justrefined = 1;
            num_refinements += 1;
        }
    }
    if (!active)
        return;
    bool finite = true;
    for (int i = 0; i < n; ++i) {
        a.states[i * a.ld + node] = y[i];
        finite = finite && isfinite(y[i]);
    }
    if (!finite)
        status |= GOSS_FLAG_NONFINITE;
    if constexpr (IE) {
#pragma unroll
        for (int k = 0; k < M::lu_nnz; ++k)
            jrows[(uint64_t)k * ld] = J[k];
    }
    ss[TH_ETA * ld] = eta;
    ss[TH_RECOMPUTE * ld] = recompute;
    ss[TH_ALWAYS * ld] = always;
    ss[TH_JUSTREFINED * ld] = justrefined;
    ss[TH_JACCOMP * ld] = jac_comp;
    ss[TH_REJECTS * ld] = rejects;
    ss[TH_ACCEPTED * ld] = accepted;
    if (status) {
        a.node_status[node] |= status;
        atomicOr(a.flags, (uint32_t)status);
    }
}

// ---------------------------------------------------------------------------
// ESDIRK23a
// ---------------------------------------------------------------------------
enum EsdirkRows {
    ES_PREV_DT = 0, ES_LOC_ERROR, ES_ETA, ES_NEWTON_IT, ES_FIRST, ES_NEWJAC, ES_JACCOMP, ES_REJECTS, ES_ACCEPTED,
    ES_SCALARS  // then the packed jac and jfac, each lu_nnz x ld values tiled [ld/32][lu_nnz][32]
};

struct EsdirkCoef {
    double gamma, a21, a22, a31, a32, a33, a41, a42, a43, a44, b1, b2, b3, b4, bh1, bh2, bh3, c2, c3, c4;
    double s_fac, tol, etamin, kappa;
};

// ESDIRK23a constructor (ESDIRK23a.cpp:27-39)
__device__ __forceinline__ EsdirkCoef esdirk_coefficients()
{
    EsdirkCoef c;
    const double gamma = 0.43586652150845899942;
    c.gamma = gamma;
    c.a21 = gamma;
    c.a22 = gamma;
    c.a31 = (-4 * gamma * gamma + 6 * gamma - 1) / (4 * gamma);
    c.a32 = (-2 * gamma + 1) / (4 * gamma);
    c.a33 = gamma;
    c.a41 = (6 * gamma - 1) / (12 * gamma);
    c.a42 = -1 / ((24 * gamma - 12) * gamma);
    c.a43 = (-6 * gamma * gamma + 6 * gamma - 1) / (6 * gamma - 3);
    c.a44 = gamma;
    c.b1 = c.a41;
    c.b2 = c.a42;
    c.b3 = c.a43;
    c.b4 = c.a44;
    c.bh1 = c.a31;
    c.bh2 = c.a32;
    c.bh3 = c.a33;
    c.c2 = 2.0 * gamma;
    c.c3 = 1.0;
    c.c4 = 1.0;
    c.s_fac = 0.9;
    c.tol = 1.0e-5;
    c.etamin = 1.0e-10;
    c.kappa = 1.0e-1;
    return c;
}

// ESDIRK23a as one loop per node in which every pass evaluates the right-hand
// side at most once and runs at most one substitution with the factorised
// matrix, whatever phase of the method the node is in: the start of a step
// attempt (f(y, t), the first stage), a Newton iteration of stage 2, 3 or 4,
// or the error estimate.  The lanes of a warp drift apart in their Newton
// iteration and step counts; in the nested form each lane then runs a
// different inlined copy of the stage loop and the warp executes the copies
// one after the other, here they share one copy of the model code.  The
// Jacobian (at most once per pass) and the factorisation follow the same rule.
// Per node the operations and their order are the nested form's
// (ESDIRK23a::forward, advance_one_step, do_step, compute_stage_val,
// reduce_time_step; ESDIRK23a.cpp:101-316).
// The passes run in block lockstep (a block barrier after each pass, until
// every node of the block has finished the interval), so the block's warps
// walk the large straight-line pass code together and share its
// instruction-cache lines, at the cost of waiting for the block's slowest
// node.  Measured on B200 (TT04, 262,144 nodes, 0.1 ms intervals, the same
// states): with the analytic Jacobian 17.5 ms per interval without barriers,
// 14.4 / 11.8 / 10.2 ms in lockstep blocks of 64 / 128 / 256 where steps are
// accepted (min_dt 1e-4), 284 ms against 231 / 173 / 136 ms where every
// attempt is rejected (default min_dt); with forward differences 18.4 against
// 15.0 / 12.4 / 10.7 ms and 354 against 302 / 211 / 156 ms.
#ifndef GOSS_ESDIRK_THREADS
#define GOSS_ESDIRK_THREADS 256
#endif
#ifndef GOSS_ESDIRK_MIN_BLOCKS
#define GOSS_ESDIRK_MIN_BLOCKS 1
#endif
#ifndef GOSS_ESDIRK_REUSE_F
#define GOSS_ESDIRK_REUSE_F 1
#endif
template <class M, bool J32 = false>
__global__ void __launch_bounds__(GOSS_ESDIRK_THREADS, GOSS_ESDIRK_MIN_BLOCKS)
    esdirk_kernel(const __grid_constant__ ImplicitArgs<M> a)
{
    constexpr int n = M::num_states;
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = gid < a.N;
    // threads past the last node shadow it (reads only) and take part in the barriers
    const uint32_t node = active ? gid : a.N - 1;
    const uint64_t ld = a.ld;
    double y[n];
    for (int i = 0; i < n; ++i)
        y[i] = a.states[i * ld + node];
    double F[Dims<M>::nfp];
    load_field<M, double>(a.fparams, ld, node, F);
    double* ss = a.sstate + node;
    const EsdirkCoef c = esdirk_coefficients();
    const goss_solver_params& sp = a.sp;
    const PackedTile jac = packed_tile(a.sstate + (uint64_t)ES_SCALARS * ld, node, M::lu_nnz);
    const PackedTile jfac = packed_tile(a.sstate + (uint64_t)(ES_SCALARS + M::lu_nnz) * ld, node, M::lu_nnz);
    double prev_dt = ss[ES_PREV_DT * ld];
    double loc_error = ss[ES_LOC_ERROR * ld];
    double eta = ss[ES_ETA * ld];
    int newton_iterations = (int)ss[ES_NEWTON_IT * ld];
    int first_step = ss[ES_FIRST * ld] != 0.0;
    int new_jacobian = ss[ES_NEWJAC * ld] != 0.0;
    double jac_comp = ss[ES_JACCOMP * ld], rejects = ss[ES_REJECTS * ld], accepted = ss[ES_ACCEPTED * ld];

    // stage derivatives z1, z2, z3 and the current stage's z (z2, z3 or z4)
    double z1[n], z2[n], z3[n], z[n], prev[n];
    enum { PH_BEGIN = 0, PH_NEWTON = 1, PH_ERROR = 2 };
    int phase = PH_BEGIN, stage = 2;
    double t_step = 0.0, t_s = 0.0, dz_norm = 0.0;
    int newton_guard = 0, advance_guard = 0;
    int jac_pending = 0;  // Jacobians due at the top of the next pass (same y and t)
    double t_jac = 0.0;
    bool fact_pending = false;

    const double t0 = a.t, interval = a.interval;
    const double min_dt = sp.min_dt;
    double local_t = 0;
    uint8_t status = 0;
    uint64_t guard = 0;
    // ESDIRK23a::forward (ESDIRK23a.cpp:280-316)
    double h = std_max(c.s_fac * prev_dt * pow((c.tol / loc_error), 0.25), min_dt);
    h = std_min(h, interval);
    if (first_step) {
        prev_dt = h;
        jac_pending = 1;
        t_jac = t0;
    }
    // top of the while loop of forward: returns false when the interval is done
    auto outer_begin = [&]() -> bool {
        if (!(local_t < interval))
            return false;
        if (++guard > a.max_loop) {
            status |= GOSS_FLAG_ITERATION_CAP;
            return false;
        }
        if (h * 1.1 >= interval - local_t)
            h = interval - local_t;
        if (newton_iterations >= 2) {
            jac_pending += 1;
            t_jac = t0 + local_t;
        }
        if (fabs((h - prev_dt) / prev_dt) > 0.2 || new_jacobian || jac_pending)
            fact_pending = true;
        t_step = t0 + local_t;
        advance_guard = 0;
        phase = PH_BEGIN;
        return true;
    };
    // compute_stage_val's entry
    auto start_stage = [&](int st, double t_stage) {
        stage = st;
        t_s = t_stage;
        newton_iterations = 0;
        dz_norm = 0.0;
        newton_guard = 0;
        eta = pow(std_max(eta, c.etamin), 0.8);
        phase = PH_NEWTON;
    };
    // the end of advance_one_step and of the while loop's body
    auto end_advance = [&]() -> bool {
        new_jacobian = 0;
        prev_dt = h;
        local_t += h;
        h = std_max(c.s_fac * prev_dt * pow((c.tol / loc_error), 0.25), min_dt);
        return outer_begin();
    };
    // do_step returned false: advance_one_step's retry loop
    auto step_failed = [&]() -> bool {
        if (h > min_dt && ++advance_guard < 4096) {
            if (!new_jacobian) {
                jac_pending = 1;
                t_jac = t_step;
            }
            // reduce_time_step (ESDIRK23a.cpp:260-278)
            double reduction_factor = 1.0, e = loc_error;
            int g = 0;
            do {
                reduction_factor *= 0.6;
                e *= 0.1;
            } while (e > c.tol && ++g < 4096);
            h = std_max(reduction_factor * h, min_dt);
            fact_pending = true;
            phase = PH_BEGIN;
            return true;
        }
        return end_advance();
    };

    // block-uniform loop: every pass, a block barrier (see above)
    bool running = active && outer_begin();
    while (__syncthreads_or(running)) {
        if (!running)
            continue;
        // f(y, t_step) of an attempt's first stage, when this pass's Jacobian
        // evaluation produced it (then held in z1)
        bool f_known = false;
        if (jac_pending || fact_pending) {
            // both are due only before an attempt's first stage, which
            // rewrites z1, z and prev before reading them, and z2, z3 before
            // reading them: their old values are dead here, and saying so
            // keeps them out of the registers the Jacobian code needs
#pragma unroll
            for (int i = 0; i < n; i++)
                z1[i] = z2[i] = z3[i] = z[i] = prev[i] = 0.0;
        }
        // ESDIRK23a::compute_ode_jacobian (ESDIRK23a.h:58-63)
        if (jac_pending) {
            double g1[n];  // f(y), a by-product of the fused evaluations
            if constexpr (J32) {
                (void)g1;
                jacobian32<M>(y, t_jac, a.P32, a.P, F, jac);
            } else if constexpr (M::has_jacobian && GOSS_IMPLICIT_SPLIT) {
                M::template rhs_jacobian<double>(y, t_jac, a.P, a.P, F, g1, jac);
            } else if constexpr (GOSS_IMPLICIT_SPLIT) {
                M::fd_clear(jac);
                M::template rhs_fd_jacobian<double>(y, t_jac, a.P, a.P, F, g1, jac);
            } else {
                rhs64<M>(y, t_jac, a.P, F, g1);
                compute_jacobian<M>(y, t_jac, a.P, F, jac, g1);
            }
            jac_comp += jac_pending;
            jac_pending = 0;
            new_jacobian = 1;
            // The Jacobian is due only before an attempt's first stage and is
            // taken at that stage's (y, t_step); the evaluation that fused it
            // with f(y) leaves f(y, t_step), which do_step (ESDIRK23a.cpp:
            // 134-140) evaluates once more for z1.  Only the FP32 Jacobian
            // does not produce it.
            if constexpr (!J32 && GOSS_ESDIRK_REUSE_F) {
                if (phase == PH_BEGIN && t_jac == t_step) {
#pragma unroll
                    for (int i = 0; i < n; i++)
                        z1[i] = g1[i];
                    f_known = true;
                }
            }
        }
        // ESDIRK23a::compute_factorized_jacobian(dt) (ESDIRK23a.cpp:101-115)
        if (fact_pending) {
            M::lu_copy_shift(jac, jfac, -h * c.a22);
            M::lu_factorize(jfac);
            fact_pending = false;
        }
        // the pass's right-hand side: f(y, t) at an attempt's start, else
        // f(y + h prev + gamma h z, t_s) of a Newton iteration
        double f[n];
        if (phase != PH_ERROR && !f_known) {
            double x[n];
#pragma unroll
            for (int i = 0; i < n; i++)
                x[i] = phase == PH_BEGIN ? y[i] : y[i] + h * prev[i] + c.gamma * h * z[i];
            rhs64<M>(x, phase == PH_BEGIN ? t_step : t_s, a.P, F, f);
        }
        // the pass's substitution: the Newton update, or the error estimate
        double dz[n];
        if (phase != PH_BEGIN) {
            double v[n];
#pragma unroll
            for (int i = 0; i < n; i++)
                v[i] = phase == PH_NEWTON
                           ? -z[i] + f[i]
                           : h * ((c.b1 - c.bh1) * z1[i] + (c.b2 - c.bh2) * z2[i] + (c.b3 - c.gamma) * z3[i] +
                                  c.gamma * z[i]);
            M::lu_solve(jfac, v, dz);
        }
        if (phase == PH_BEGIN) {
            // do_step: z1 = f(y, t0), z2 = z1, prev = a21 z1
#pragma unroll
            for (int i = 0; i < n; i++) {
                const double fi = f_known ? z1[i] : f[i];
                z1[i] = fi;
                z[i] = fi;
                prev[i] = fi * c.a21;
            }
            start_stage(2, t_step + c.c2 * h);
        } else if (phase == PH_NEWTON) {
            // one iteration of compute_stage_val (ESDIRK23a.cpp:201-258)
            const double prev_dz_norm = dz_norm;
            dz_norm = l2norm<n>(dz);
            bool fail = false;
            if (newton_iterations >= 1) {
                const double theta = dz_norm / prev_dz_norm;
                if (!(theta <= 1)) {
                    rejects += 1;
                    fail = true;
                } else {
                    eta = theta / (1.0 - theta);
                }
            }
            if (!fail && (newton_iterations > sp.max_iterations || ++newton_guard > 100000)) {
                rejects += 1;
                fail = true;
            }
            if (fail) {
                running = step_failed();
                continue;
            }
#pragma unroll
            for (int i = 0; i < n; i++)
                z[i] += dz[i];
            newton_iterations++;
            if (!(eta * dz_norm > c.kappa * c.tol)) {
                if (stage == 2) {
#pragma unroll
                    for (int i = 0; i < n; i++) {
                        z2[i] = z[i];
                        prev[i] = z1[i] * c.bh1 + z2[i] * c.bh2;
                    }
                    start_stage(3, t_step + c.c3 * h);
                } else if (stage == 3) {
#pragma unroll
                    for (int i = 0; i < n; i++) {
                        z3[i] = z[i];
                        prev[i] = z1[i] * c.b1 + z2[i] * c.b2 + z3[i] * c.b3;
                    }
                    start_stage(4, t_step + c.c4 * h);
                } else {
                    phase = PH_ERROR;  // z holds z4
                }
            }
        } else {
            // do_step's error test (ESDIRK23a.cpp:180-196)
            loc_error = l2norm<n>(dz);
            if (loc_error > c.tol) {
                rejects += 1;
                running = step_failed();
            } else {
#pragma unroll
                for (int i = 0; i < n; i++)
                    y[i] = y[i] + h * (c.b1 * z1[i] + c.b2 * z2[i] + c.b3 * z3[i] + c.gamma * z[i]);
                accepted += 1;
                running = end_advance();
            }
        }
    }
    if (!active)
        return;
    first_step = 0;
    bool finite = true;
    for (int i = 0; i < n; ++i) {
        a.states[i * ld + node] = y[i];
        finite = finite && isfinite(y[i]);
    }
    if (!finite)
        status |= GOSS_FLAG_NONFINITE;
    ss[ES_PREV_DT * ld] = prev_dt;
    ss[ES_LOC_ERROR * ld] = loc_error;
    ss[ES_ETA * ld] = eta;
    ss[ES_NEWTON_IT * ld] = newton_iterations;
    ss[ES_FIRST * ld] = first_step;
    ss[ES_NEWJAC * ld] = new_jacobian;
    ss[ES_JACCOMP * ld] = jac_comp;
    ss[ES_REJECTS * ld] = rejects;
    ss[ES_ACCEPTED * ld] = accepted;
    if (status) {
        a.node_status[node] |= status;
        atomicOr(a.flags, (uint32_t)status);
    }
}

// ---------------------------------------------------------------------------
// batched model evaluation (ODE::eval / ODE::linearized_eval on many states)
// ---------------------------------------------------------------------------
template <class M, typename T>
__global__ void __launch_bounds__(128) eval_kernel(const __grid_constant__ EvalArgs<M, T> a)
{
    constexpr int n = M::num_states;
    const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= a.N)
        return;
    T y[n], o1[n], o2[n];
    for (int i = 0; i < n; ++i)
        y[i] = T(a.states[i * a.ld + node]);
    T F[Dims<M>::nfp];
    load_field<M, T>(a.fparams, a.ld, node, F);
    const double t = a.times[node];
    if (a.what == 0) {
        M::template rhs<T>(y, t, a.P, a.PD, F, o1);
        for (int i = 0; i < n; ++i)
            a.out[i * a.ld + node] = double(o1[i]);
    } else if (a.what == 1) {
        M::template linearized<T>(y, t, a.P, a.PD, F, o1, o2);
        for (int i = 0; i < n; ++i) {
            a.out[i * a.ld + node] = double(o1[i]);
            a.out[(n + i) * a.ld + node] = double(o2[i]);
        }
    } else if (a.what == 2) {
        if constexpr (M::num_monitored > 0) {
            T mon[M::num_monitored];
            M::template monitored_values<T>(y, t, a.P, a.PD, F, mon);
            for (int i = 0; i < M::num_monitored; ++i)
                a.out[i * a.ld + node] = double(mon[i]);
        }
    } else if constexpr (M::has_jacobian) {
        T J[M::lu_nnz];
        M::template jacobian<T>(y, t, a.P, a.PD, F, J);
        M::lu_unpack(J, [&](int k, T v) { a.out[(uint64_t)k * a.ld + node] = double(v); });
    }
}

// ---------------------------------------------------------------------------
// host-side launchers (called through goss_model_desc::launch / ::eval)
// ---------------------------------------------------------------------------
inline unsigned long explicit_num_steps(double ldt_0, double dt)
{
    // e.g. GRL1.cpp:66
    return ldt_0 > 0 ? (unsigned long)ceil(dt / ldt_0 - 1.0E-12) : 1UL;
}

template <class M>
inline uint32_t solver_state_rows(int32_t solver)
{
    if (solver == GOSS_THETA)
        return TH_ROWS;
    if (solver == GOSS_IMPLICIT_EULER)
        return TH_ROWS + M::lu_nnz;
    if (solver == GOSS_ESDIRK23A)
        return ES_SCALARS + 2 * M::lu_nnz;
    return 0;
}

template <class M, typename T, Explicit S>
inline int launch_explicit(const goss_launch* L)
{
    ExplicitArgs<M, T> a;
    a.states = L->states;
    a.fparams = L->field_params;
    a.flags = L->flags;
    a.node_status = L->node_status;
    a.ld = L->ld;
    a.N = L->num_nodes;
    const double ldt_0 = L->solver_params->ldt;
    const unsigned long nsteps = explicit_num_steps(ldt_0, L->interval);
    a.nsteps = nsteps;
    a.ldt = L->interval / nsteps;
    a.t = L->t;
    a.delta = L->solver_params->delta;
    parameter_block<M>(L->params, a.PD);
    for (int i = 0; i < Dims<M>::np; ++i)
        a.P[i] = T(a.PD[i]);
    const unsigned block = L->block ? L->block : 128;
    const unsigned grid = (L->num_nodes + block - 1) / block;
    if (grid == 0)
        return 0;
    explicit_kernel<M, T, S><<<grid, block, 0, (cudaStream_t)L->stream>>>(a);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : GOSS_ERR_CUDA;
}

template <class M>
inline int launch_implicit(const goss_launch* L)
{
    ImplicitArgs<M> a;
    a.states = L->states;
    a.fparams = L->field_params;
    a.sstate = L->solver_state;
    a.flags = L->flags;
    a.node_status = L->node_status;
    a.ld = L->ld;
    a.N = L->num_nodes;
    a.t = L->t;
    a.interval = L->interval;
    a.sp = *L->solver_params;
    a.max_loop = L->max_loop ? L->max_loop : (1ull << 24);
    parameter_block<M>(L->params, a.P);
    for (int i = 0; i < Dims<M>::np; ++i)
        a.P32[i] = float(a.P[i]);
    // GOSS_FP32: the analytic Jacobian in FP32 (models generated with it)
    const bool j32 = L->precision == GOSS_FP32;
    if (j32 && !M::has_jacobian)
        return GOSS_ERR_UNSUPPORTED;
    // lockstep blocks of 256 (the kernels' limit)
    const bool theta = L->solver == GOSS_THETA || L->solver == GOSS_IMPLICIT_EULER;
    const unsigned block = L->block ? L->block : (theta ? GOSS_THETA_THREADS : GOSS_ESDIRK_THREADS);
    if (block > (theta ? (unsigned)GOSS_THETA_THREADS : (unsigned)GOSS_ESDIRK_THREADS))
        return GOSS_ERR_ARGUMENT;
    const unsigned grid = (L->num_nodes + block - 1) / block;
    if (grid == 0)
        return 0;
    const cudaStream_t st = (cudaStream_t)L->stream;
    if (j32) {
        if constexpr (M::has_jacobian) {
            if (L->solver == GOSS_THETA)
                theta_kernel<M, false, true><<<grid, block, 0, st>>>(a);
            else if (L->solver == GOSS_IMPLICIT_EULER)
                theta_kernel<M, true, true><<<grid, block, 0, st>>>(a);
            else
                esdirk_kernel<M, true><<<grid, block, 0, st>>>(a);
        }
    } else if (L->solver == GOSS_THETA) {
        theta_kernel<M, false><<<grid, block, 0, st>>>(a);
    } else if (L->solver == GOSS_IMPLICIT_EULER) {
        theta_kernel<M, true><<<grid, block, 0, st>>>(a);
    } else {
        esdirk_kernel<M><<<grid, block, 0, st>>>(a);
    }
    return cudaPeekAtLastError() == cudaSuccess ? 0 : GOSS_ERR_CUDA;
}

template <class M>
inline int launch_solver(const goss_launch* L)
{
    const bool f32 = L->precision == GOSS_FP32;
    if (L->precision == GOSS_FP64_PRINTED)
        return L->solver == GOSS_GRL1 ? launch_explicit<M, double, Explicit::GRL1Printed>(L) : GOSS_ERR_UNSUPPORTED;
    switch (L->solver) {
    case GOSS_EXPLICIT_EULER:
        return f32 ? launch_explicit<M, float, Explicit::Euler>(L) : launch_explicit<M, double, Explicit::Euler>(L);
    case GOSS_RK4:
        return f32 ? launch_explicit<M, float, Explicit::RK4>(L) : launch_explicit<M, double, Explicit::RK4>(L);
    case GOSS_GRL1:
        return f32 ? launch_explicit<M, float, Explicit::GRL1>(L) : launch_explicit<M, double, Explicit::GRL1>(L);
    case GOSS_GRL2:
        return f32 ? launch_explicit<M, float, Explicit::GRL2>(L) : launch_explicit<M, double, Explicit::GRL2>(L);
    case GOSS_RL1:
        return f32 ? launch_explicit<M, float, Explicit::RL1>(L) : launch_explicit<M, double, Explicit::RL1>(L);
    case GOSS_RL2:
        return f32 ? launch_explicit<M, float, Explicit::RL2>(L) : launch_explicit<M, double, Explicit::RL2>(L);
    case GOSS_RK2:
        return f32 ? launch_explicit<M, float, Explicit::RK2>(L) : launch_explicit<M, double, Explicit::RK2>(L);
    case GOSS_THETA:
    case GOSS_ESDIRK23A:
    case GOSS_IMPLICIT_EULER:
        return launch_implicit<M>(L);
    default:
        return GOSS_ERR_ARGUMENT;
    }
}

template <class M, typename T>
inline int launch_eval_t(const goss_eval_launch* L)
{
    EvalArgs<M, T> a;
    a.states = L->states;
    a.fparams = L->field_params;
    a.times = L->times;
    a.out = L->out;
    a.ld = L->ld;
    a.N = L->num_nodes;
    a.what = L->what;
    parameter_block<M>(L->params, a.PD);
    for (int i = 0; i < Dims<M>::np; ++i)
        a.P[i] = T(a.PD[i]);
    const unsigned block = 128;
    const unsigned grid = (L->num_nodes + block - 1) / block;
    if (grid == 0)
        return 0;
    eval_kernel<M, T><<<grid, block, 0, (cudaStream_t)L->stream>>>(a);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : GOSS_ERR_CUDA;
}

template <class M>
inline int launch_eval(const goss_eval_launch* L)
{
    return L->precision == GOSS_FP32 ? launch_eval_t<M, float>(L) : launch_eval_t<M, double>(L);
}

}  // namespace goss_b200
#endif
