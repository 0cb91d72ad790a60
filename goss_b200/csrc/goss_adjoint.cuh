// Adjoint of GRL1 and RK4 trajectories with checkpointing (one thread per node).
//
// Forward (record_kernel): the reference's user loop
//     for j in 0..J-1:  forward(t0 + j*interval, interval)   (S internal
//                       steps, GRL1.cpp:61-82 / RK4.cpp:68-102)
// storing the traced state after every interval (the trace) and the full
// state every K internal steps (checkpoints; K a multiple of S).  Each step
// is explicit_step of goss_kernels.cuh, the solver kernels' own arithmetic.
//
// Backward (adjoint_kernel): given the cotangent of the trace, walk the
// checkpoint segments from last to first; recompute each segment's K states
// into per-node scratch, then apply the transposed Jacobian of every step in
// reverse, adding the trace cotangent to the traced state's lambda at every
// sample and accumulating the field-parameter gradient.
//
// GRL1:  Phi_i(y) = y_i + b_i h phi1(a_i h),   (a, b) = linearized(y, t)
//     lambda <- lambda + [abar^T d a/dy + bbar^T d b/dy]
//     abar_i = lambda_i b_i h^2 phi1'(a_i h),  bbar_i = lambda_i h phi1(a_i h)
// with the generated linearized_vjp for the bracket.  phi1(x) = (e^x - 1)/x
// is the same function as the reference's b/a (e^{a h} - 1); the derivative
// uses the smooth phi1 form.
//
// RK4:   y' = y + h/6 (k1 + 2 k2 + 2 k3 + k4),  k_s = f(u_s, t_s),
//        u_1 = y, u_2 = y + h/2 k1, u_3 = y + h/2 k2, u_4 = y + h k3
// reversed stage by stage with the generated rhs_vjp:
//     kbar_4 = h/6 lambda;  ubar_s = (df/du)(u_s)^T kbar_s;
//     kbar_{s-1} = w_{s-1} lambda + c_s ubar_s  (w = h/6, h/3, h/3; c = h/2, h/2, h)
//     lambda <- lambda + sum_s ubar_s
// after recomputing k1..k3 from the step's input state.
#ifndef GOSS_ADJOINT_CUH
#define GOSS_ADJOINT_CUH

#include "goss_kernels.cuh"

// Launch shape of the adjoint kernel per arithmetic type: the largest threads
// per block (a multiple of 32, at most 256) and the minimum resident blocks
// per SM it is compiled for (its register cap is 65536 / (threads * blocks)).
// With GOSS_ADJOINT_LOCKSTEP the warps of a block synchronise after every step
// of the recompute and reverse loops, so they walk the large straight-line
// step code together and share instruction-cache lines.  Measured on B200
// (ten Tusscher-Panfilov, 65,536 nodes x 2,000 steps, backward pass):
//   FP32: blocks of up to 128 threads, 2 per SM (255 registers), lockstep
//         28.0 ms; 256 x 1: 29.3 ms; register caps of 168 or 128 (3 or 4
//         blocks of 128) spill more than the extra warps gain: 37.5 ms; with
//         the record's tape (65,536 nodes x 40,000 steps, 368 of 400
//         segments taped) 2, 3, 4 blocks: 445, 650, 716 ms;
//   FP64: 256 x 1: 207 ms; 128 x 2: 215 ms.
// (the shape of the backward follows the arithmetic of its VJPs)
template <typename T>
struct AdjointShape {
    static constexpr unsigned block = sizeof(T) == 4 ? 128 : 256;
    static constexpr unsigned min_blocks = sizeof(T) == 4 ? 2 : 1;
};
#ifndef GOSS_ADJOINT_LOCKSTEP
#define GOSS_ADJOINT_LOCKSTEP 1
#endif

namespace goss_b200 {

// phi1(x) = (e^x - 1)/x and phi1'(x) = (e^x (x - 1) + 1)/x^2 in FP64:
// Taylor series sum_k x^k/(k+1)! and sum_k (k+1) x^k/(k+2)! for |x| < 0.1
// (truncation below 1e-17 relative), closed forms otherwise.
__device__ __forceinline__ double phi1d(double x)
{
    if (fabs(x) < 0.1) {
        double p = 1.0 / 362880.0;
        p = fma(p, x, 1.0 / 40320.0);
        p = fma(p, x, 1.0 / 5040.0);
        p = fma(p, x, 1.0 / 720.0);
        p = fma(p, x, 1.0 / 120.0);
        p = fma(p, x, 1.0 / 24.0);
        p = fma(p, x, 1.0 / 6.0);
        p = fma(p, x, 0.5);
        p = fma(p, x, 1.0);
        return p;
    }
    return expm1(x) / x;
}

__device__ __forceinline__ double dphi1d(double x)
{
    if (fabs(x) < 0.1) {
        // sum_{k=0}^{9} (k+1) x^k / (k+2)!
        double p = 10.0 / 39916800.0;
        p = fma(p, x, 9.0 / 3628800.0);
        p = fma(p, x, 8.0 / 362880.0);
        p = fma(p, x, 7.0 / 40320.0);
        p = fma(p, x, 6.0 / 5040.0);
        p = fma(p, x, 5.0 / 720.0);
        p = fma(p, x, 4.0 / 120.0);
        p = fma(p, x, 3.0 / 24.0);
        p = fma(p, x, 2.0 / 6.0);
        p = fma(p, x, 0.5);
        return p;
    }
    return (exp(x) * (x - 1.0) + 1.0) / (x * x);
}

// FP32: Taylor series to x^6 for |x| < 1/4 (truncation < 2e-9), closed forms otherwise
__device__ __forceinline__ float dphi1f(float x)
{
    if (fabsf(x) < 0.25f) {
        // sum_{k=0}^{7} (k+1) x^k / (k+2)!
        float p = 8.0f / 362880.0f;
        p = fmaf(p, x, 7.0f / 40320.0f);
        p = fmaf(p, x, 6.0f / 5040.0f);
        p = fmaf(p, x, 5.0f / 720.0f);
        p = fmaf(p, x, 4.0f / 120.0f);
        p = fmaf(p, x, 3.0f / 24.0f);
        p = fmaf(p, x, 2.0f / 6.0f);
        p = fmaf(p, x, 0.5f);
        return p;
    }
    return __fdividef(__expf(x) * (x - 1.0f) + 1.0f, x * x);
}

__device__ __forceinline__ double phi1t(double x) { return phi1d(x); }
__device__ __forceinline__ float phi1t(float x) { return phi1f(x); }
__device__ __forceinline__ double dphi1t(double x) { return dphi1d(x); }
__device__ __forceinline__ float dphi1t(float x) { return dphi1f(x); }

template <class M, typename T>
struct AdjointArgs {
    double* states;            // [n][ld] in: initial, out: final (record)
    const double* fparams;     // [nfp][ld]
    void* checkpoints;         // [C][2n][ld] float (FP32: hi, lo) or [C][n][ld] double
    double* trace;             // [J][ld]
    const double* trace_bar;   // [J][ld]
    T* scratch;                // [K][n][sld], sld = num_nodes rounded up to 256, plus 256
    T* tape;                   // [taped_segments][K][n][sld]: step inputs of the last segments
    double* fparams_bar;       // [nfp][ld]
    double* states_bar;        // [n][ld]
    uint32_t* flags;
    uint64_t ld;
    uint64_t sld;              // scratch row stride (>= grid * block)
    uint32_t N;
    uint32_t num_intervals;    // J
    uint32_t steps_per_interval;  // S
    uint32_t checkpoint_every;    // K (multiple of S)
    uint32_t trace_state;
    uint32_t taped_segments;
    double t0;
    double interval;
    T P[Dims<M>::np];
    double PD[Dims<M>::np];
};

// checkpoint I/O for the accumulators
__device__ __forceinline__ void cp_store(void* cp, uint64_t idx_hi, uint64_t idx_lo, const Acc<double>& a)
{
    static_cast<double*>(cp)[idx_hi] = a.y;
    (void)idx_lo;
}
__device__ __forceinline__ void cp_store(void* cp, uint64_t idx_hi, uint64_t idx_lo, const Acc<float>& a)
{
    static_cast<float*>(cp)[idx_hi] = a.hi;
    static_cast<float*>(cp)[idx_lo] = a.lo;
}
__device__ __forceinline__ void cp_load(const void* cp, uint64_t idx_hi, uint64_t idx_lo, Acc<double>& a)
{
    a.y = static_cast<const double*>(cp)[idx_hi];
    (void)idx_lo;
}
__device__ __forceinline__ void cp_load(const void* cp, uint64_t idx_hi, uint64_t idx_lo, Acc<float>& a)
{
    a.hi = static_cast<const float*>(cp)[idx_hi];
    a.lo = static_cast<const float*>(cp)[idx_lo];
}

// GRL1 threshold of the reference (GRL1.h:39) used by the traces
constexpr double kGrlDelta = 1e-8;

template <typename T>
__host__ __device__ constexpr int cp_rows(int n)
{
    return sizeof(T) == 4 ? 2 * n : n;
}

template <class M, typename T, Explicit S>
__global__ void __launch_bounds__(128) record_kernel(const __grid_constant__ AdjointArgs<M, T> a)
{
    constexpr int n = M::num_states;
    const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= a.N)
        return;
    Acc<T> y[n];
    for (int i = 0; i < n; ++i)
        y[i].load(a.states[i * a.ld + node]);
    T F[Dims<M>::nfp];
    load_field<M, T>(a.fparams, a.ld, node, F);
    const uint32_t S_ = a.steps_per_interval, K = a.checkpoint_every;
    const double ldt = a.interval / S_;
    constexpr int rows = cp_rows<T>(n);
    // the last taped_segments segments keep every step's input state: the
    // values the backward's recompute would write to its scratch
    const uint64_t total = (uint64_t)a.num_intervals * S_;
    const uint64_t num_cp = (total + K - 1) / K;
    const uint64_t tape_from = (num_cp - a.taped_segments) * K;
    T* const tape = a.tape + node;
    for (uint32_t j = 0; j < a.num_intervals; ++j) {
        const uint64_t g = (uint64_t)j * S_;
        if (g % K == 0) {
            const uint64_t c = g / K;
            for (int i = 0; i < n; ++i)
                cp_store(a.checkpoints, ((c * rows) + i) * a.ld + node, ((c * rows) + n + i) * a.ld + node, y[i]);
        }
        double lt = a.t0 + j * a.interval;
        for (uint32_t s = 0; s < S_; ++s) {
            if (g + s >= tape_from) {
                const uint64_t row = (g + s - tape_from) * n;
                for (int i = 0; i < n; ++i)
                    tape[(row + i) * a.sld] = y[i].value();
            }
            explicit_step<M, T, S>(y, lt, ldt, a.P, a.PD, F, T(kGrlDelta));
            lt += ldt;
        }
        a.trace[(uint64_t)j * a.ld + node] = y[a.trace_state].store();
    }
    bool finite = true;
    for (int i = 0; i < n; ++i) {
        const double v = y[i].store();
        a.states[i * a.ld + node] = v;
        finite = finite && isfinite(v);
    }
    if (!finite)
        atomicOr(a.flags, GOSS_FLAG_NONFINITE);
}

// lambda <- lambda + (dPhi/dy)(y)^T lambda - lambda for one GRL1 step, and the
// field-parameter part into gF
template <class M, typename T>
__device__ __forceinline__ void reverse_step_grl1(const T* yt, double lt, double ldt, const T* P, const double* PD,
                                                  const T* F, Acc<T>* lam, double* gF)
{
    constexpr int n = M::num_states;
    constexpr int nfp = Dims<M>::nfp;
    const T h = T(ldt);
    T lv[n], ybar[n], Fbar[nfp];
    for (int i = 0; i < n; ++i)
        lv[i] = lam[i].value();
    auto seed = [&](const T* lin, const T* rhs, T* abar, T* bbar) {
#pragma unroll
        for (int i = 0; i < n; ++i) {
            const T x = lin[i] * h;
            bbar[i] = lv[i] * h * phi1t(x);
            abar[i] = lv[i] * rhs[i] * h * h * dphi1t(x);
        }
    };
    M::template linearized_vjp<T>(yt, lt, P, PD, F, seed, ybar, Fbar);
    for (int i = 0; i < n; ++i)
        lam[i].add(ybar[i]);
    for (int q = 0; q < M::num_field_params; ++q)
        gF[q] += double(Fbar[q]);
}

// the same for one RK4 step; the stage loops are not unrolled, so rhs and
// rhs_vjp are instantiated once.  The stage inputs are formed from the step's
// input value (in FP32 its high word; the forward adds the low word as well,
// a difference of at most half an FP32 ulp of the state).
template <class M, typename T>
__device__ __forceinline__ void reverse_step_rk4(const T* yt, double lt, double ldt, const T* P, const double* PD,
                                                 const T* F, Acc<T>* lam, double* gF)
{
    constexpr int n = M::num_states;
    constexpr int nfp = Dims<M>::nfp;
    const T h = T(ldt), hh = T(0.5 * ldt);
    T k1[n], k2[n], k3[n], u[n];
#pragma unroll 1
    for (int st = 0; st < 3; ++st) {
        const double ts = st == 0 ? lt : lt + 0.5 * ldt;
        for (int i = 0; i < n; ++i)
            u[i] = st == 0 ? yt[i] : yt[i] + hh * (st == 1 ? k1[i] : k2[i]);
        T k[n];
        model_rhs<M, T>(u, ts, P, PD, F, k);
        for (int i = 0; i < n; ++i) {
            k1[i] = st == 0 ? k[i] : k1[i];
            k2[i] = st == 1 ? k[i] : k2[i];
            k3[i] = st == 2 ? k[i] : k3[i];
        }
    }
    T lv[n], kb[n], ysum[n];
    const T w6 = h / T(6.0), w3 = h / T(3.0);
    for (int i = 0; i < n; ++i) {
        lv[i] = lam[i].value();
        kb[i] = w6 * lv[i];
        ysum[i] = T(0.0);
    }
#pragma unroll 1
    for (int st = 3; st >= 0; --st) {
        const T c = st == 3 ? h : hh;
        const double ts = st == 3 ? lt + ldt : (st == 0 ? lt : lt + 0.5 * ldt);
        for (int i = 0; i < n; ++i)
            u[i] = st == 0 ? yt[i] : yt[i] + c * (st == 3 ? k3[i] : st == 2 ? k2[i] : k1[i]);
        T ub[n], Fb[nfp];
        auto seed = [&](const T*, T* bbar) {
#pragma unroll
            for (int i = 0; i < n; ++i)
                bbar[i] = kb[i];
        };
        M::template rhs_vjp<T>(u, ts, P, PD, F, seed, ub, Fb);
        const T w = st == 1 ? w6 : w3;
        for (int i = 0; i < n; ++i) {
            ysum[i] = ysum[i] + ub[i];
            kb[i] = w * lv[i] + c * ub[i];
        }
        for (int q = 0; q < M::num_field_params; ++q)
            gF[q] += double(Fb[q]);
    }
    for (int i = 0; i < n; ++i)
        lam[i].add(ysum[i]);
}

// R is the arithmetic of the step VJPs and of lambda: T, or double over an
// FP32 trajectory (the recompute keeps T, so the same trajectory is
// differentiated; only the VJP arithmetic changes).
template <class M, typename T, Explicit S, typename R = T>
__global__ void __launch_bounds__(AdjointShape<R>::block, AdjointShape<R>::min_blocks)
adjoint_kernel(const __grid_constant__ AdjointArgs<M, T> a)
{
    constexpr int n = M::num_states;
    constexpr int nfp = Dims<M>::nfp;
    static_assert(sizeof(R) >= sizeof(T), "the VJP arithmetic is at least the trajectory's");
    // Every thread runs every loop (block-wide barriers below); threads past
    // the last node shadow it (reads only) and keep their own scratch column.
    const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = node < a.N;
    const uint32_t src = active ? node : a.N - 1;
    extern __shared__ double s_time[];  // time of every step of a segment (same for all nodes)
    const uint32_t S_ = a.steps_per_interval, K = a.checkpoint_every;
    const double ldt = a.interval / S_;
    T F[nfp];
    load_field<M, T>(a.fparams, a.ld, src, F);
    R FR[nfp];
    load_field<M, R>(a.fparams, a.ld, src, FR);
    const R* PR;
    if constexpr (sizeof(R) == sizeof(T))
        PR = reinterpret_cast<const R*>(a.P);
    else
        PR = a.PD;
    Acc<R> lam[n];
    for (int i = 0; i < n; ++i)
        lam[i].load(0.0);
    double gF[nfp];
    for (int k = 0; k < nfp; ++k)
        gF[k] = 0.0;
    const uint64_t total = (uint64_t)a.num_intervals * S_;
    const uint32_t num_cp = (uint32_t)((total + K - 1) / K);
    constexpr int rows = cp_rows<T>(n);
    T* const scratch = a.scratch + node;
    for (int c = (int)num_cp - 1; c >= 0; --c) {
        const uint64_t g0 = (uint64_t)c * K;
        const uint32_t len = (uint32_t)((g0 + K <= total) ? K : total - g0);
        // times of the segment's steps, exactly as the forward accumulated them
        __syncthreads();
        if (threadIdx.x == 0) {
            double lt = 0.0;
            for (uint32_t k = 0; k < len; ++k) {
                const uint64_t g = g0 + k;
                if (g % S_ == 0)
                    lt = a.t0 + (g / S_) * a.interval;
                s_time[k] = lt;
                lt += ldt;
            }
        }
        __syncthreads();
        // the input state of every step of the segment: from the record's
        // tape, or recomputed from the checkpoint into scratch
        const T* seg = scratch;
        if ((uint32_t)c >= num_cp - a.taped_segments) {
            seg = a.tape + (uint64_t)(c - (num_cp - a.taped_segments)) * K * n * a.sld + src;
        } else {
            Acc<T> y[n];
            for (int i = 0; i < n; ++i)
                cp_load(a.checkpoints, ((uint64_t)c * rows + i) * a.ld + src,
                        ((uint64_t)c * rows + n + i) * a.ld + src, y[i]);
            for (uint32_t k = 0; k < len; ++k) {
                for (int i = 0; i < n; ++i)
                    scratch[((uint64_t)k * n + i) * a.sld] = y[i].value();
                if (k + 1 < len)
                    explicit_step<M, T, S>(y, s_time[k], ldt, a.P, a.PD, F, T(kGrlDelta));
#if GOSS_ADJOINT_LOCKSTEP
                __syncthreads();
#endif
            }
        }
        // reverse through the segment
        for (int k = (int)len - 1; k >= 0; --k) {
            const uint64_t g = g0 + k;  // step g maps state g to state g+1
            if ((g + 1) % S_ == 0) {
                const uint64_t j = (g + 1) / S_ - 1;
                lam[a.trace_state].add(R(a.trace_bar[j * a.ld + src]));
            }
            R yt[n];
            for (int i = 0; i < n; ++i)
                yt[i] = R(seg[((uint64_t)k * n + i) * a.sld]);
            if constexpr (S == Explicit::GRL1)
                reverse_step_grl1<M, R>(yt, s_time[k], ldt, PR, a.PD, FR, lam, gF);
            else
                reverse_step_rk4<M, R>(yt, s_time[k], ldt, PR, a.PD, FR, lam, gF);
#if GOSS_ADJOINT_LOCKSTEP
            __syncthreads();
#endif
        }
    }
    if (!active)
        return;
    for (int q = 0; q < M::num_field_params; ++q)
        a.fparams_bar[(uint64_t)q * a.ld + node] = gF[q];
    for (int i = 0; i < n; ++i)
        a.states_bar[(uint64_t)i * a.ld + node] = lam[i].store();
}

// Threads per block for the backward kernel: every thread carries one node
// through the whole trajectory, so the job runs in waves of (resident blocks
// x SMs) blocks and its time is about waves x resident warps per SM.  Choose
// the multiple of 32 (<= AdjointShape<T>::block) minimising that product (ties:
// the larger block) -- e.g. for 65,536 nodes on 148 SMs with two blocks per
// SM: 112 threads (two nearly full waves) instead of 128 (a second wave on
// 108 of 148 SMs).
template <class M, typename T, Explicit S, typename R = T>
inline unsigned adjoint_block(uint32_t num_nodes, size_t shm)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return AdjointShape<R>::block;
    unsigned best = AdjointShape<R>::block;
    uint64_t best_cost = ~0ull;
    for (unsigned b = AdjointShape<R>::block; b >= 32; b -= 32) {
        int active = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&active, adjoint_kernel<M, T, S, R>, (int)b, shm) !=
                cudaSuccess || active <= 0)
            continue;
        const uint64_t grid = (num_nodes + b - 1) / b;
        const uint64_t slots = (uint64_t)active * sms;
        const uint64_t waves = (grid + slots - 1) / slots;
        const uint64_t cost = waves * (uint64_t)active * b;
        if (cost < best_cost) {
            best_cost = cost;
            best = b;
        }
    }
    return best;
}

template <class M, typename T, Explicit S, typename R = T>
inline int launch_adjoint_t(const goss_adjoint_launch* L)
{
    AdjointArgs<M, T> a;
    a.states = L->states;
    a.fparams = L->field_params;
    a.checkpoints = L->checkpoints;
    a.trace = L->trace;
    a.trace_bar = L->trace_bar;
    a.scratch = static_cast<T*>(L->scratch);
    a.tape = static_cast<T*>(L->tape);
    a.taped_segments = L->taped_segments;
    a.fparams_bar = L->field_params_bar;
    a.states_bar = L->states_bar;
    a.flags = L->flags;
    a.ld = L->ld;
    a.N = L->num_nodes;
    a.num_intervals = L->num_intervals;
    a.steps_per_interval = L->steps_per_interval;
    a.checkpoint_every = L->checkpoint_every;
    a.trace_state = L->trace_state;
    a.t0 = L->t0;
    a.interval = L->interval;
    parameter_block<M>(L->params, a.PD);
    for (int i = 0; i < Dims<M>::np; ++i)
        a.P[i] = T(a.PD[i]);
    if (a.steps_per_interval == 0 || a.checkpoint_every == 0 || a.checkpoint_every % a.steps_per_interval ||
        a.trace_state >= (uint32_t)M::num_states)
        return GOSS_ERR_ARGUMENT;
    {
        const uint64_t total = (uint64_t)a.num_intervals * a.steps_per_interval;
        const uint64_t num_cp = (total + a.checkpoint_every - 1) / a.checkpoint_every;
        if (a.taped_segments > num_cp || (a.taped_segments && !a.tape))
            return GOSS_ERR_ARGUMENT;
    }
    // room for grid * block <= round_up(num_nodes, block) for any block <= 256
    a.sld = ((uint64_t)L->num_nodes + 255) / 256 * 256 + 256;
    if (L->num_nodes == 0)
        return 0;
    if (L->mode == 0) {
        const unsigned block = 128;
        const unsigned grid = (L->num_nodes + block - 1) / block;
        record_kernel<M, T, S><<<grid, block, 0, (cudaStream_t)L->stream>>>(a);
    } else {
        const size_t shm = sizeof(double) * a.checkpoint_every;
        if (shm > 48 * 1024)
            return GOSS_ERR_ARGUMENT;
        const unsigned block = L->block ? L->block : adjoint_block<M, T, S, R>(L->num_nodes, shm);
        if (block == 0 || block > AdjointShape<R>::block || block % 32)
            return GOSS_ERR_ARGUMENT;
        const unsigned grid = (L->num_nodes + block - 1) / block;
        adjoint_kernel<M, T, S, R><<<grid, block, shm, (cudaStream_t)L->stream>>>(a);
    }
    return cudaPeekAtLastError() == cudaSuccess ? 0 : GOSS_ERR_CUDA;
}

template <class M>
inline int launch_adjoint(const goss_adjoint_launch* L)
{
    const bool f32 = L->precision == GOSS_FP32;
    const bool rev64 = L->reverse_precision == GOSS_FP64;
    if (!(L->reverse_precision == L->precision || (f32 && rev64 && L->solver == GOSS_GRL1)))
        return GOSS_ERR_UNSUPPORTED;
    switch (L->solver) {
    case GOSS_GRL1:
        if (f32 && rev64)
            return launch_adjoint_t<M, float, Explicit::GRL1, double>(L);
        return f32 ? launch_adjoint_t<M, float, Explicit::GRL1>(L) : launch_adjoint_t<M, double, Explicit::GRL1>(L);
    case GOSS_RK4:
        return f32 ? launch_adjoint_t<M, float, Explicit::RK4>(L) : launch_adjoint_t<M, double, Explicit::RK4>(L);
    default:
        return GOSS_ERR_UNSUPPORTED;
    }
}

}  // namespace goss_b200
#endif
