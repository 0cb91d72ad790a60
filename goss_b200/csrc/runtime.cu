// Host runtime behind the C ABI of include/goss_b200.h.
//
// goss_system is the device-resident counterpart of goss::ODESystemSolver
// (reference cpp/goss/ODESystemSolver.{h,cpp}): it owns the FP64
// component-major state and field-parameter arrays, the per-node solver state
// of the implicit solvers, a stream and a status word, and it drives the
// model module's solver kernels through goss_model_desc::launch.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "goss_b200.h"

namespace {

thread_local std::string g_last_error;

int fail(std::string* where, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    if (where)
        *where = buf;
    return code;
}

#define CUDA_TRY(sys, call)                                                                              \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return fail((sys) ? &(sys)->last_error : nullptr, GOSS_ERR_CUDA, "CUDA error %s at %s:%d: %s", \
                        cudaGetErrorName(e_), __FILE__, __LINE__, cudaGetErrorString(e_));              \
    } while (0)

uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

// ---------------------------------------------------------------------------
// layout kernels
// ---------------------------------------------------------------------------
// Scatter a user array (tangled [N][k] or untangled [k][N]) into rows of a
// component-major array: dst[rows[c]*ld + node] = src(node, c).  rows may be
// NULL for the identity map.
__global__ void scatter_kernel(double* __restrict__ dst, uint64_t ld, const double* __restrict__ src, uint32_t N,
                               uint32_t k, const uint32_t* __restrict__ rows, int tangled)
{
    const uint64_t total = (uint64_t)N * k;
    for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t node, c;
        if (tangled) {
            node = (uint32_t)(idx / k);
            c = (uint32_t)(idx % k);
        } else {
            c = (uint32_t)(idx / N);
            node = (uint32_t)(idx % N);
        }
        const uint32_t r = rows ? rows[c] : c;
        dst[(uint64_t)r * ld + node] = src[idx];
    }
}

// Gather rows of a component-major array into a user layout:
// dst(node, c) = src[rows[c]*ld + node].
__global__ void gather_kernel(double* __restrict__ dst, const double* __restrict__ src, uint64_t ld, uint32_t N,
                              uint32_t k, const uint32_t* __restrict__ rows, int tangled)
{
    const uint64_t total = (uint64_t)N * k;
    for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t node, c;
        if (tangled) {
            node = (uint32_t)(idx / k);
            c = (uint32_t)(idx % k);
        } else {
            c = (uint32_t)(idx / N);
            node = (uint32_t)(idx % N);
        }
        const uint32_t r = rows ? rows[c] : c;
        dst[idx] = src[(uint64_t)r * ld + node];
    }
}

// dst[r*ld + node] = values[r] for every node < N (rows 0..k-1)
__global__ void fill_rows_kernel(double* __restrict__ dst, uint64_t ld, uint32_t N, uint32_t k,
                                 const double* __restrict__ values)
{
    const uint64_t total = (uint64_t)N * k;
    for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(idx / N), node = (uint32_t)(idx % N);
        dst[(uint64_t)r * ld + node] = values[r];
    }
}

unsigned grid_for(uint64_t total, unsigned block = 256)
{
    uint64_t g = (total + block - 1) / block;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 32));
}

}  // namespace

// ---------------------------------------------------------------------------
// system object
// ---------------------------------------------------------------------------
struct goss_system {
    const goss_model_desc* m = nullptr;
    int32_t solver = 0, precision = 0, device = 0;
    goss_solver_params sp{};
    uint32_t N = 0, n = 0, nfp = 0;
    uint64_t ld = 0;
    double* d_states = nullptr;
    double* d_fparams = nullptr;
    double* d_sstate = nullptr;
    uint32_t sstate_rows = 0;
    uint32_t* d_flags = nullptr;
    uint8_t* d_node_status = nullptr;
    double* d_stage = nullptr;  // staging for host transfers, max(n, nfp, 1) * ld doubles
    uint64_t stage_elems = 0;
    double* d_small = nullptr;  // row constants
    uint32_t* d_rows = nullptr; // row maps (field state indices / components)
    uint32_t rows_cap = 0;
    std::vector<double> params;
    std::vector<uint32_t> fsi;  // field state indices
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t block = 0;
    uint32_t num_threads = 0;
    uint32_t host_flags = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    std::string last_error;
};

struct goss_batch {
    const goss_batch_desc* d = nullptr;
    std::vector<goss_system*> systems;
    std::vector<int32_t> kinds;
    std::vector<uint32_t> order;
    int32_t precision = 0;
    int32_t device = 0;
    uint32_t block = 128, grid = 0, schedule = 1;
    uint32_t forwards_per_launch = 0;  // of a captured graph; 0: all
    uint32_t* d_counters = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    std::string last_error;
};

namespace {

int set_device(goss_system* s)
{
    CUDA_TRY(s, cudaSetDevice(s->device));
    return 0;
}

int ensure_rows(goss_system* s, const uint32_t* rows, uint32_t k)
{
    if (k > s->rows_cap) {
        if (s->d_rows)
            cudaFree(s->d_rows);
        s->d_rows = nullptr;
        CUDA_TRY(s, cudaMalloc(&s->d_rows, sizeof(uint32_t) * k));
        s->rows_cap = k;
    }
    if (k)
        CUDA_TRY(s, cudaMemcpyAsync(s->d_rows, rows, sizeof(uint32_t) * k, cudaMemcpyHostToDevice, s->stream));
    return 0;
}

// init the per-node solver state (the reference solver's reset()/constructor values)
int init_solver_state(goss_system* s)
{
    if (!s->sstate_rows)
        return 0;
    std::vector<double> v(s->sstate_rows, 0.0);
    if (s->solver == GOSS_THETA || s->solver == GOSS_IMPLICIT_EULER) {
        // TH_ETA, TH_RECOMPUTE, TH_ALWAYS, TH_JUSTREFINED, counters
        // (ImplicitODESolver::reset, ImplicitODESolver.cpp:80-90; ThetaSolver.cpp:37-45;
        // ImplicitEuler.cpp:14-21)
        v[0] = s->sp.eta_0;
        v[1] = 1.0;
        v[2] = s->sp.always_recompute_jacobian ? 1.0 : 0.0;
    } else if (s->solver == GOSS_ESDIRK23A) {
        // prev_dt(0.1), loc_error(1e9), eta(1.0), _newton_iterations(0),
        // first_step(true), new_jacobian(true) (ESDIRK23a.cpp:27-39)
        v[0] = 0.1;
        v[1] = 1e9;
        v[2] = 1.0;
        v[3] = 0.0;
        v[4] = 1.0;
        v[5] = 1.0;
    }
    double* d_v = nullptr;
    CUDA_TRY(s, cudaMalloc(&d_v, sizeof(double) * v.size()));
    CUDA_TRY(s, cudaMemcpyAsync(d_v, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, s->stream));
    fill_rows_kernel<<<grid_for((uint64_t)s->N * v.size()), 256, 0, s->stream>>>(s->d_sstate, s->ld, s->N,
                                                                                  (uint32_t)v.size(), d_v);
    CUDA_TRY(s, cudaGetLastError());
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    cudaFree(d_v);
    return 0;
}

int check_flags(goss_system* s)
{
    uint32_t f = 0;
    CUDA_TRY(s, cudaMemcpyAsync(&f, s->d_flags, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    const uint32_t fresh = f & ~s->host_flags;
    s->host_flags |= f;
    if (fresh & GOSS_FLAG_NEWTON_FAILED) {
        // the reference throws std::runtime_error (ThetaSolver.cpp:140-145)
        return fail(&s->last_error, GOSS_ERR_NEWTON,
                    "Newtons solver failed to converge as dt become smaller than 'min_dt' %g", s->sp.min_dt);
    }
    if (fresh & GOSS_FLAG_ITERATION_CAP)
        return fail(&s->last_error, GOSS_ERR_TIMEOUT, "a node exceeded the solver loop guard");
    return 0;
}

int launch_forward(goss_system* s, double t, double interval)
{
    goss_launch L{};
    L.solver = s->solver;
    L.precision = s->precision;
    L.num_nodes = s->N;
    L.block = s->block;
    L.ld = s->ld;
    L.states = s->d_states;
    L.field_params = s->d_fparams;
    L.solver_state = s->d_sstate;
    L.flags = s->d_flags;
    L.node_status = s->d_node_status;
    L.params = s->params.data();
    L.solver_params = &s->sp;
    L.t = t;
    L.interval = interval;
    L.max_loop = 0;
    L.stream = s->stream;
    int rc = s->m->launch(&L);
    if (rc == GOSS_ERR_UNSUPPORTED)
        return fail(&s->last_error, rc, "solver %d is not available in %s precision for model %s", s->solver,
                    s->precision == GOSS_FP32 ? "FP32" : s->precision == GOSS_FP64_PRINTED ? "printed FP64" : "FP64",
                    s->m->name);
    if (rc) {
        cudaError_t e = cudaGetLastError();
        return fail(&s->last_error, rc, "kernel launch failed: %s", cudaGetErrorString(e));
    }
    return 0;
}

}  // namespace

extern "C" {

GOSS_API uint32_t goss_abi_version(void) { return GOSS_B200_ABI_VERSION; }

// ---------------------------------------------------------------------------
// CUDA-core peaks for the rooflines of the model kernels: independent chains
// of ex2/lg2 (XU pipe, the exponentials and reciprocals of the models) and of
// FP32 fused multiply-adds, enough warps to fill every SM
// ---------------------------------------------------------------------------
namespace {
constexpr int kXuChains = 8, kFmaChains = 16;

__global__ void peak_xu_kernel(float* sink, int iters)
{
    float x[kXuChains];
#pragma unroll
    for (int c = 0; c < kXuChains; ++c)
        x[c] = 0.5f + 0.01f * (threadIdx.x & 7) + 0.05f * c;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int c = 0; c < kXuChains; ++c) {
            float y;
            asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x[c]));
            asm volatile("lg2.approx.ftz.f32 %0, %1;" : "=f"(x[c]) : "f"(y));
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kXuChains; ++c)
        s += x[c];
    if (s == 12345.0f)  // never true; keeps the chains live
        sink[blockIdx.x] = s;
}

__global__ void peak_fma_kernel(float* sink, int iters)
{
    float x[kFmaChains];
#pragma unroll
    for (int c = 0; c < kFmaChains; ++c)
        x[c] = 0.5f + 0.01f * (threadIdx.x & 7) + 0.05f * c;
    const float a = 0.999f, b = 0.001f;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int c = 0; c < kFmaChains; ++c)
            asm volatile("fma.rn.f32 %0, %0, %1, %2;" : "+f"(x[c]) : "f"(a), "f"(b));
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kFmaChains; ++c)
        s += x[c];
    if (s == 12345.0f)
        sink[blockIdx.x] = s;
}
}  // namespace

GOSS_API int goss_measure_peaks(int32_t device, double* xu_ops_per_s, double* fp32_ops_per_s)
{
    if (!xu_ops_per_s || !fp32_ops_per_s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL output");
    cudaError_t e = cudaSetDevice(device);
    int sms = 0;
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess)
        return fail(nullptr, GOSS_ERR_CUDA, "measure peaks: %s", cudaGetErrorString(e));
    const int block = 256, grid = sms * 8;  // 2048 threads per SM
    const int xu_iters = 2048, fma_iters = 8192;
    float* sink = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double best_xu = 0.0, best_fma = 0.0;
    e = cudaMalloc(&sink, sizeof(float) * grid);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaEventCreate(&e0);
    if (e == cudaSuccess)
        e = cudaEventCreate(&e1);
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {  // the first of each is a warm-up
        float ms = 0.0f;
        cudaEventRecord(e0, st);
        peak_xu_kernel<<<grid, block, 0, st>>>(sink, xu_iters);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && rep && ms > 0)
            best_xu = std::max(best_xu, (double)grid * block * xu_iters * 2 * kXuChains / (ms * 1e-3));
        if (e != cudaSuccess)
            break;
        cudaEventRecord(e0, st);
        peak_fma_kernel<<<grid, block, 0, st>>>(sink, fma_iters);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && rep && ms > 0)
            best_fma = std::max(best_fma, (double)grid * block * fma_iters * kFmaChains / (ms * 1e-3));
    }
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    if (st)
        cudaStreamDestroy(st);
    cudaFree(sink);
    if (e != cudaSuccess)
        return fail(nullptr, GOSS_ERR_CUDA, "measure peaks: %s", cudaGetErrorString(e));
    *xu_ops_per_s = best_xu;
    *fp32_ops_per_s = best_fma;
    return 0;
}

namespace {
constexpr int kDfmaChains = 8;

__global__ void peak_dfma_kernel(double* sink, int iters)
{
    double x[kDfmaChains];
#pragma unroll
    for (int c = 0; c < kDfmaChains; ++c)
        x[c] = 0.5 + 0.01 * (threadIdx.x & 7) + 0.05 * c;
    const double a = 0.999, b = 0.001;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int c = 0; c < kDfmaChains; ++c)
            asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(x[c]) : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kDfmaChains; ++c)
        s += x[c];
    if (s == 12345.0)
        sink[blockIdx.x] = s;
}
}  // namespace

GOSS_API int goss_measure_fp64_peak(int32_t device, double* fp64_fma_per_s)
{
    if (!fp64_fma_per_s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL output");
    cudaError_t e = cudaSetDevice(device);
    int sms = 0;
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess)
        return fail(nullptr, GOSS_ERR_CUDA, "measure FP64 peak: %s", cudaGetErrorString(e));
    const int block = 256, grid = sms * 8;  // 2048 threads per SM
    const int iters = 2048;
    double* sink = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double best = 0.0;
    e = cudaMalloc(&sink, sizeof(double) * grid);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaEventCreate(&e0);
    if (e == cudaSuccess)
        e = cudaEventCreate(&e1);
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {  // the first is a warm-up
        float ms = 0.0f;
        cudaEventRecord(e0, st);
        peak_dfma_kernel<<<grid, block, 0, st>>>(sink, iters);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && rep && ms > 0)
            best = std::max(best, (double)grid * block * iters * kDfmaChains / (ms * 1e-3));
    }
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    if (st)
        cudaStreamDestroy(st);
    cudaFree(sink);
    if (e != cudaSuccess)
        return fail(nullptr, GOSS_ERR_CUDA, "measure FP64 peak: %s", cudaGetErrorString(e));
    *fp64_fma_per_s = best;
    return 0;
}

GOSS_API const char* goss_last_error(void) { return g_last_error.c_str(); }
GOSS_API const char* goss_system_last_error(const goss_system* s) { return s ? s->last_error.c_str() : ""; }

GOSS_API int goss_solver_default_params(int32_t solver, goss_solver_params* p)
{
    if (!p || solver < 0 || solver >= GOSS_NUM_SOLVERS)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "invalid solver kind %d", solver);
    std::memset(p, 0, sizeof(*p));
    p->ldt = -1.0;                             // ODESolver.h:137
    p->delta = 1e-8;                           // GRL1.h:39
    p->eta_0 = 1.0;                            // ImplicitODESolver.h:36
    p->kappa = 0.1;                            // ImplicitODESolver.h:37
    p->relative_tolerance = 1e-12;             // ImplicitODESolver.h:38
    p->max_iterations = 30;                    // ImplicitODESolver.h:39
    p->max_relative_previous_residual = 0.01;  // ImplicitODESolver.h:40
    p->always_recompute_jacobian = 0;          // ImplicitODESolver.h:41
    p->num_refinements_without_always_recomputing_jacobian = 2;  // ThetaSolver.h:35, ImplicitEuler.h:35
    p->min_dt = solver == GOSS_ESDIRK23A ? 0.001 : 0.0001;      // ESDIRK23a.h:38, ThetaSolver.h:36, ImplicitEuler.h:36
    p->theta = 0.5;                                              // ThetaSolver.h:37
    return 0;
}

GOSS_API int goss_system_create(const goss_model_desc* m, int32_t solver, const goss_solver_params* params,
                                uint32_t num_nodes, int32_t precision, int32_t device, goss_system** out)
{
    if (!out)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    if (!m || m->abi_version != GOSS_B200_ABI_VERSION)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "model descriptor missing or built for another ABI version");
    if (solver < 0 || solver >= GOSS_NUM_SOLVERS || !(m->supported_solvers & (1u << solver)))
        return fail(nullptr, GOSS_ERR_UNSUPPORTED, "solver kind %d is not available for model %s", solver, m->name);
    if (precision != GOSS_FP64 && precision != GOSS_FP32 && precision != GOSS_FP64_PRINTED)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "invalid precision %d", precision);
    if ((solver == GOSS_THETA || solver == GOSS_ESDIRK23A || solver == GOSS_IMPLICIT_EULER) && precision == GOSS_FP32 &&
        !m->has_jacobian)
        return fail(nullptr, GOSS_ERR_UNSUPPORTED,
                    "implicit solvers in GOSS_FP32 evaluate the analytic Jacobian in FP32 (the residuals, LU and "
                    "updates stay FP64) and need a model generated with it (code_params generate_jacobian); "
                    "use GOSS_FP64 for model %s", m->name);
    if (precision == GOSS_FP64_PRINTED && solver != GOSS_GRL1)
        return fail(nullptr, GOSS_ERR_UNSUPPORTED, "GOSS_FP64_PRINTED is available for GRL1 only");
    auto* s = new goss_system();
    s->m = m;
    s->solver = solver;
    s->precision = precision;
    s->device = device;
    if (params)
        s->sp = *params;
    else
        goss_solver_default_params(solver, &s->sp);
    s->N = num_nodes;
    s->n = m->num_states;
    s->nfp = m->num_field_parameters;
    s->ld = round_up(std::max<uint64_t>(num_nodes, 1), 32);
    s->params.assign(m->default_parameters, m->default_parameters + m->num_parameters);
    if (s->params.empty())
        s->params.push_back(0.0);
    s->sstate_rows = m->solver_state_rows(solver);
    int rc = set_device(s);
    if (rc) {
        delete s;
        return rc;
    }
#define CREATE_TRY(call)                                                                                 \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            fail(nullptr, GOSS_ERR_CUDA, "CUDA error %s during create: %s", cudaGetErrorName(e_),        \
                 cudaGetErrorString(e_));                                                                \
            goss_system_destroy(s);                                                                      \
            return GOSS_ERR_CUDA;                                                                        \
        }                                                                                                \
    } while (0)
    CREATE_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
    CREATE_TRY(cudaMalloc(&s->d_states, sizeof(double) * s->n * s->ld));
    if (s->nfp)
        CREATE_TRY(cudaMalloc(&s->d_fparams, sizeof(double) * s->nfp * s->ld));
    if (s->sstate_rows)
        CREATE_TRY(cudaMalloc(&s->d_sstate, sizeof(double) * s->sstate_rows * s->ld));
    CREATE_TRY(cudaMalloc(&s->d_flags, sizeof(uint32_t)));
    CREATE_TRY(cudaMemsetAsync(s->d_flags, 0, sizeof(uint32_t), s->stream));
    CREATE_TRY(cudaMalloc(&s->d_node_status, s->ld));
    CREATE_TRY(cudaMemsetAsync(s->d_node_status, 0, s->ld, s->stream));
    s->stage_elems = (uint64_t)std::max<uint32_t>(std::max(s->n, s->nfp), 1) * s->ld;
    CREATE_TRY(cudaMalloc(&s->d_stage, sizeof(double) * s->stage_elems));
    CREATE_TRY(cudaMalloc(&s->d_small, sizeof(double) * std::max<uint32_t>(std::max(s->n, s->nfp), 64)));
#undef CREATE_TRY
    rc = goss_system_reset_default(s);
    if (!rc)
        rc = init_solver_state(s);
    if (rc) {
        goss_system_destroy(s);
        return rc;
    }
    *out = s;
    return 0;
}

GOSS_API int goss_system_destroy(goss_system* s)
{
    if (!s)
        return 0;
    cudaSetDevice(s->device);
    if (s->stream)
        cudaStreamSynchronize(s->stream);
    cudaFree(s->d_states);
    cudaFree(s->d_fparams);
    cudaFree(s->d_sstate);
    cudaFree(s->d_flags);
    cudaFree(s->d_node_status);
    cudaFree(s->d_stage);
    cudaFree(s->d_small);
    cudaFree(s->d_rows);
    if (s->graph_exec)
        cudaGraphExecDestroy(s->graph_exec);
    if (s->graph)
        cudaGraphDestroy(s->graph);
    if (s->own_stream && s->stream)
        cudaStreamDestroy(s->stream);
    delete s;
    return 0;
}

// ---------------------------------------------------------------------------
// CUDA graphs of forward loops
// ---------------------------------------------------------------------------
GOSS_API int goss_system_capture(goss_system* s, double t0, double interval, uint32_t num_steps)
{
    if (!s || num_steps == 0)
        return fail(s ? &s->last_error : nullptr, GOSS_ERR_ARGUMENT, "capture needs a system and num_steps > 0");
    int rc = set_device(s);
    if (rc)
        return rc;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (s->graph_exec) {
        cudaGraphExecDestroy(s->graph_exec);
        s->graph_exec = nullptr;
    }
    if (s->graph) {
        cudaGraphDestroy(s->graph);
        s->graph = nullptr;
    }
    CUDA_TRY(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    for (uint32_t k = 0; k < num_steps && !rc; ++k)
        rc = launch_forward(s, t0 + k * interval, interval);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc) {
        if (g)
            cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess)
        return fail(&s->last_error, GOSS_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
    s->graph = g;
    CUDA_TRY(s, cudaGraphInstantiate(&s->graph_exec, s->graph, 0));
    return 0;
}

GOSS_API int goss_system_replay(goss_system* s)
{
    if (!s || !s->graph_exec)
        return fail(s ? &s->last_error : nullptr, GOSS_ERR_ARGUMENT, "no captured graph");
    int rc = set_device(s);
    if (rc)
        return rc;
    CUDA_TRY(s, cudaGraphLaunch(s->graph_exec, s->stream));
    return check_flags(s);
}

// ---------------------------------------------------------------------------
// heterogeneous batches
// ---------------------------------------------------------------------------
namespace {

int batch_fail(goss_batch* b, int code, const char* msg)
{
    return fail(b ? &b->last_error : nullptr, code, "%s", msg);
}

// count consecutive forwards in one launch, forward f on
// [t + (first + f) * interval, + interval)
int batch_launch(goss_batch* b, double t, double interval, uint64_t first = 0, uint32_t count = 1)
{
    std::vector<goss_batch_pop> pops(b->systems.size());
    for (size_t i = 0; i < pops.size(); ++i) {
        goss_system* s = b->systems[i];
        goss_batch_pop& p = pops[i];
        p.kind = b->kinds[i];
        p.num_nodes = s->N;
        p.ld = s->ld;
        p.states = s->d_states;
        p.field_params = s->d_fparams;
        p.node_status = s->d_node_status;
        p.flags = s->d_flags;
        p.params = s->params.data();
        p.solver_params = &s->sp;
    }
    goss_batch_launch L{};
    L.precision = b->precision;
    L.num_pops = (uint32_t)pops.size();
    L.pops = pops.data();
    L.order = b->order.empty() ? nullptr : b->order.data();
    L.block = b->block;
    L.grid = b->grid;
    L.schedule = b->schedule;
    L.counters = b->d_counters;
    L.t = t;
    L.interval = interval;
    L.first_forward = first;
    L.forwards = count;
    L.stream = b->stream;
    const int rc = b->d->launch(&L);
    if (rc)
        return fail(&b->last_error, rc, "batch launch failed (%s)", cudaGetErrorString(cudaGetLastError()));
    return 0;
}

int batch_check(goss_batch* b)
{
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess)
        return fail(&b->last_error, GOSS_ERR_CUDA, "batch failed: %s", cudaGetErrorString(e));
    for (goss_system* s : b->systems) {
        const int rc = check_flags(s);
        if (rc)
            return fail(&b->last_error, rc, "%s", s->last_error.c_str());
    }
    return 0;
}

}  // namespace

GOSS_API const char* goss_batch_last_error(const goss_batch* b) { return b ? b->last_error.c_str() : ""; }

GOSS_API int goss_batch_create(const goss_batch_desc* d, goss_system* const* systems, const int32_t* kinds,
                               uint32_t count, int32_t precision, goss_batch** out)
{
    if (!out || !d || (count && (!systems || !kinds)))
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (d->abi_version != GOSS_B200_ABI_VERSION)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "batch module built for another ABI version");
    if (count > 16)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "a batch holds at most 16 populations");
    if (precision != GOSS_FP64 && precision != GOSS_FP32)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "invalid precision %d", precision);
    int device = count ? systems[0]->device : 0;
    for (uint32_t i = 0; i < count; ++i) {
        const goss_system* s = systems[i];
        if (!s || kinds[i] < 0 || (uint32_t)kinds[i] >= d->num_kinds)
            return fail(nullptr, GOSS_ERR_ARGUMENT, "population %u: invalid system or kind", i);
        if (s->solver != d->kind_solvers[kinds[i]] || s->n != d->kind_num_states[kinds[i]])
            return fail(nullptr, GOSS_ERR_ARGUMENT, "population %u: solver or model does not match kind %d (%s)", i,
                        kinds[i], d->kind_variants[kinds[i]]);
        if (s->device != device)
            return fail(nullptr, GOSS_ERR_ARGUMENT, "all populations must live on one device");
        for (uint32_t j = 0; j < i; ++j)
            if (systems[j] == s)
                return fail(nullptr, GOSS_ERR_ARGUMENT, "a system appears twice in the batch");
    }
    auto* b = new goss_batch();
    b->d = d;
    b->systems.assign(systems, systems + count);
    b->kinds.assign(kinds, kinds + count);
    b->precision = precision;
    b->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_counters, 2 * sizeof(uint32_t));
    if (e == cudaSuccess)
        e = cudaMemsetAsync(b->d_counters, 0, 2 * sizeof(uint32_t), b->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        goss_batch_destroy(b);
        return fail(nullptr, GOSS_ERR_CUDA, "batch create: %s", cudaGetErrorString(e));
    }
    // the populations are about to be touched from the batch stream
    for (goss_system* s : b->systems)
        cudaStreamSynchronize(s->stream);
    *out = b;
    return 0;
}

GOSS_API int goss_batch_destroy(goss_batch* b)
{
    if (!b)
        return 0;
    cudaSetDevice(b->device);
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    if (b->graph_exec)
        cudaGraphExecDestroy(b->graph_exec);
    if (b->graph)
        cudaGraphDestroy(b->graph);
    cudaFree(b->d_counters);
    if (b->stream)
        cudaStreamDestroy(b->stream);
    delete b;
    return 0;
}

GOSS_API int goss_batch_set_config(goss_batch* b, uint32_t block, uint32_t grid, uint32_t schedule,
                                   const uint32_t* order)
{
    if (!b)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL batch");
    if (block && (block % 32 || block > 128))
        return batch_fail(b, GOSS_ERR_ARGUMENT, "block must be a multiple of 32 and at most 128");
    if (schedule > 2)
        return batch_fail(b, GOSS_ERR_ARGUMENT,
                          "schedule must be 0 (round-robin), 1 (dynamic) or 2 (persistent with prefetch)");
    if (order) {
        std::vector<uint32_t> o(order, order + b->systems.size());
        std::vector<uint32_t> s(o);
        std::sort(s.begin(), s.end());
        for (size_t i = 0; i < s.size(); ++i)
            if (s[i] != i)
                return batch_fail(b, GOSS_ERR_ARGUMENT, "order must be a permutation of the populations");
        b->order = o;
    } else {
        b->order.clear();
    }
    b->block = block ? block : 128;
    b->grid = grid;
    b->schedule = schedule;
    return 0;
}

GOSS_API int goss_batch_forward(goss_batch* b, double t, double interval)
{
    if (!b)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL batch");
    CUDA_TRY((goss_system*)nullptr, cudaSetDevice(b->device));
    int rc = batch_launch(b, t, interval);
    return rc ? rc : batch_check(b);
}

GOSS_API int goss_batch_capture(goss_batch* b, double t0, double interval, uint32_t num_steps)
{
    if (!b || num_steps == 0)
        return fail(b ? &b->last_error : nullptr, GOSS_ERR_ARGUMENT, "capture needs a batch and num_steps > 0");
    CUDA_TRY((goss_system*)nullptr, cudaSetDevice(b->device));
    cudaStreamSynchronize(b->stream);
    if (b->graph_exec) {
        cudaGraphExecDestroy(b->graph_exec);
        b->graph_exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
        return fail(&b->last_error, GOSS_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
    int rc = 0;
    const uint32_t per = b->forwards_per_launch ? b->forwards_per_launch : num_steps;
    for (uint32_t k = 0; k < num_steps && !rc; k += per)
        rc = batch_launch(b, t0, interval, k, std::min(per, num_steps - k));
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g)
            cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess)
        return fail(&b->last_error, GOSS_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
    b->graph = g;
    e = cudaGraphInstantiate(&b->graph_exec, b->graph, 0);
    if (e != cudaSuccess)
        return fail(&b->last_error, GOSS_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return 0;
}

GOSS_API int goss_batch_set_forwards_per_launch(goss_batch* b, uint32_t forwards)
{
    if (!b)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL batch");
    b->forwards_per_launch = forwards;
    return 0;
}

GOSS_API int goss_batch_replay(goss_batch* b)
{
    if (!b || !b->graph_exec)
        return fail(b ? &b->last_error : nullptr, GOSS_ERR_ARGUMENT, "no captured graph");
    CUDA_TRY((goss_system*)nullptr, cudaSetDevice(b->device));
    cudaError_t e = cudaGraphLaunch(b->graph_exec, b->stream);
    if (e != cudaSuccess)
        return fail(&b->last_error, GOSS_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
    return batch_check(b);
}

GOSS_API int goss_batch_time(goss_batch* b, double t0, double interval, uint32_t num_steps, int32_t use_graph,
                             float* ms)
{
    if (!b || !ms || num_steps == 0)
        return fail(b ? &b->last_error : nullptr, GOSS_ERR_ARGUMENT, "NULL argument or num_steps == 0");
    CUDA_TRY((goss_system*)nullptr, cudaSetDevice(b->device));
    int rc = 0;
    if (use_graph) {
        rc = goss_batch_capture(b, t0, interval, num_steps);
        if (rc)
            return rc;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, b->stream);
    if (use_graph) {
        cudaGraphLaunch(b->graph_exec, b->stream);
    } else {
        for (uint32_t k = 0; k < num_steps && !rc; ++k)
            rc = batch_launch(b, t0 + k * interval, interval);
    }
    cudaEventRecord(e1, b->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    float v = 0.f;
    if (e == cudaSuccess)
        e = cudaEventElapsedTime(&v, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc)
        return rc;
    if (e != cudaSuccess)
        return fail(&b->last_error, GOSS_ERR_CUDA, "timing failed: %s", cudaGetErrorString(e));
    *ms = v;
    return batch_check(b);
}

GOSS_API int goss_system_set_solver_params(goss_system* s, const goss_solver_params* p)
{
    if (!s || !p)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    s->sp = *p;
    return 0;
}

GOSS_API int goss_system_get_solver_params(const goss_system* s, goss_solver_params* p)
{
    if (!s || !p)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    *p = s->sp;
    return 0;
}

GOSS_API int goss_system_reset_default(goss_system* s)
{
    if (!s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL system");
    int rc = set_device(s);
    if (rc)
        return rc;
    // states = initial conditions, field parameters = current parameter
    // values (ODESystemSolver::reset_default, ODESystemSolver.cpp:192-216)
    std::vector<double> fp(s->nfp);
    for (uint32_t k = 0; k < s->nfp; ++k)
        fp[k] = s->params[s->m->field_parameter_indices[k]];
    CUDA_TRY(s, cudaMemcpyAsync(s->d_small, s->m->initial_conditions, sizeof(double) * s->n, cudaMemcpyHostToDevice,
                                s->stream));
    fill_rows_kernel<<<grid_for((uint64_t)s->N * s->n), 256, 0, s->stream>>>(s->d_states, s->ld, s->N, s->n,
                                                                             s->d_small);
    CUDA_TRY(s, cudaGetLastError());
    if (s->nfp) {
        CUDA_TRY(s, cudaStreamSynchronize(s->stream));
        CUDA_TRY(s, cudaMemcpyAsync(s->d_small, fp.data(), sizeof(double) * s->nfp, cudaMemcpyHostToDevice,
                                    s->stream));
        fill_rows_kernel<<<grid_for((uint64_t)s->N * s->nfp), 256, 0, s->stream>>>(s->d_fparams, s->ld, s->N,
                                                                                   s->nfp, s->d_small);
        CUDA_TRY(s, cudaGetLastError());
    }
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return 0;
}

GOSS_API int goss_system_forward(goss_system* s, double t, double interval)
{
    if (!s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL system");
    int rc = set_device(s);
    if (!rc)
        rc = launch_forward(s, t, interval);
    if (!rc)
        rc = check_flags(s);
    return rc;
}

GOSS_API int goss_system_forward_async(goss_system* s, double t, double interval)
{
    if (!s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL system");
    int rc = set_device(s);
    return rc ? rc : launch_forward(s, t, interval);
}

GOSS_API int goss_system_synchronize(goss_system* s)
{
    if (!s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL system");
    int rc = set_device(s);
    return rc ? rc : check_flags(s);
}

GOSS_API int goss_system_set_stream(goss_system* s, void* stream)
{
    if (!s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL system");
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (s->own_stream)
        cudaStreamDestroy(s->stream);
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
    return 0;
}

namespace {

int to_device(goss_system* s, double* dst, const double* host, uint32_t k, const uint32_t* rows, int32_t tangled)
{
    if (!k || !s->N)
        return 0;
    const uint64_t count = (uint64_t)s->N * k;
    if (count > s->stage_elems)
        return fail(&s->last_error, GOSS_ERR_ARGUMENT, "transfer larger than staging buffer");
    int rc = set_device(s);
    if (rc)
        return rc;
    CUDA_TRY(s, cudaMemcpyAsync(s->d_stage, host, sizeof(double) * count, cudaMemcpyHostToDevice, s->stream));
    if (rows) {
        rc = ensure_rows(s, rows, k);
        if (rc)
            return rc;
    }
    scatter_kernel<<<grid_for(count), 256, 0, s->stream>>>(dst, s->ld, s->d_stage, s->N, k, rows ? s->d_rows : nullptr,
                                                           tangled);
    CUDA_TRY(s, cudaGetLastError());
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return 0;
}

int to_host(goss_system* s, double* host, const double* src, uint32_t k, const uint32_t* rows, int32_t tangled)
{
    if (!k || !s->N)
        return 0;
    const uint64_t count = (uint64_t)s->N * k;
    if (count > s->stage_elems)
        return fail(&s->last_error, GOSS_ERR_ARGUMENT, "transfer larger than staging buffer");
    int rc = set_device(s);
    if (rc)
        return rc;
    if (rows) {
        rc = ensure_rows(s, rows, k);
        if (rc)
            return rc;
    }
    gather_kernel<<<grid_for(count), 256, 0, s->stream>>>(s->d_stage, src, s->ld, s->N, k, rows ? s->d_rows : nullptr,
                                                          tangled);
    CUDA_TRY(s, cudaGetLastError());
    CUDA_TRY(s, cudaMemcpyAsync(host, s->d_stage, sizeof(double) * count, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return 0;
}

}  // namespace

GOSS_API int goss_system_set_field_state_indices(goss_system* s, const uint32_t* idx, uint32_t count)
{
    if (!s || (count && !idx))
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    for (uint32_t i = 0; i < count; ++i)
        if (idx[i] >= s->n)
            return fail(&s->last_error, GOSS_ERR_ARGUMENT, "field state index %u out of range", idx[i]);
    s->fsi.assign(idx, idx + count);
    return 0;
}

GOSS_API int goss_system_get_field_states(const goss_system* cs, double* values, int32_t tangled)
{
    auto* s = const_cast<goss_system*>(cs);
    if (!s || (!values && !s->fsi.empty()))
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    return to_host(s, values, s->d_states, (uint32_t)s->fsi.size(), s->fsi.data(), tangled);
}

GOSS_API int goss_system_set_field_states(goss_system* s, const double* values, int32_t tangled)
{
    if (!s || (!values && !s->fsi.empty()))
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    return to_device(s, s->d_states, values, (uint32_t)s->fsi.size(), s->fsi.data(), tangled);
}

// ODESystemSolver::get/set_field_state_components (ODESystemSolver.cpp:101-133):
// components index the field states; user arrays keep the full field-state
// shape and only the listed components are read or written.
GOSS_API int goss_system_get_field_state_components(const goss_system* cs, double* values, uint32_t nc,
                                                    const uint32_t* comps, int32_t tangled)
{
    auto* s = const_cast<goss_system*>(cs);
    if (!s || (nc && (!values || !comps)))
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    const uint32_t nfs = (uint32_t)s->fsi.size();
    for (uint32_t i = 0; i < nc; ++i)
        if (comps[i] >= nfs)
            return fail(&s->last_error, GOSS_ERR_ARGUMENT, "component %u out of range", comps[i]);
    if (!nc)
        return 0;
    std::vector<double> full((size_t)s->N * nfs);
    int rc = to_host(s, full.data(), s->d_states, nfs, s->fsi.data(), tangled);
    if (rc)
        return rc;
    for (uint32_t node = 0; node < s->N; ++node)
        for (uint32_t j = 0; j < nc; ++j) {
            const uint32_t c = comps[j];
            const size_t ind = tangled ? (size_t)node * nfs + c : (size_t)s->N * c + node;
            values[ind] = full[ind];
        }
    return 0;
}

GOSS_API int goss_system_set_field_state_components(goss_system* s, const double* values, uint32_t nc,
                                                    const uint32_t* comps, int32_t tangled)
{
    if (!s || (nc && (!values || !comps)))
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    const uint32_t nfs = (uint32_t)s->fsi.size();
    for (uint32_t i = 0; i < nc; ++i)
        if (comps[i] >= nfs)
            return fail(&s->last_error, GOSS_ERR_ARGUMENT, "component %u out of range", comps[i]);
    if (!nc)
        return 0;
    // stage only the selected components, component-major
    std::vector<double> sel((size_t)s->N * nc);
    std::vector<uint32_t> rows(nc);
    for (uint32_t j = 0; j < nc; ++j) {
        const uint32_t c = comps[j];
        rows[j] = s->fsi[c];
        for (uint32_t node = 0; node < s->N; ++node) {
            const size_t ind = tangled ? (size_t)node * nfs + c : (size_t)s->N * c + node;
            sel[(size_t)j * s->N + node] = values[ind];
        }
    }
    return to_device(s, s->d_states, sel.data(), nc, rows.data(), 0);
}

GOSS_API int goss_system_get_field_parameters(const goss_system* cs, double* values, int32_t tangled)
{
    auto* s = const_cast<goss_system*>(cs);
    if (!s || (!values && s->nfp))
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    return to_host(s, values, s->d_fparams, s->nfp, nullptr, tangled);
}

GOSS_API int goss_system_set_field_parameters(goss_system* s, const double* values, int32_t tangled)
{
    if (!s || (!values && s->nfp))
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    return to_device(s, s->d_fparams, values, s->nfp, nullptr, tangled);
}

GOSS_API int goss_system_get_states(const goss_system* cs, double* states)
{
    auto* s = const_cast<goss_system*>(cs);
    if (!s || !states)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    return to_host(s, states, s->d_states, s->n, nullptr, 1);
}

GOSS_API int goss_system_set_states(goss_system* s, const double* states)
{
    if (!s || !states)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    return to_device(s, s->d_states, states, s->n, nullptr, 1);
}

GOSS_API int goss_system_set_parameter(goss_system* s, uint32_t index, double value)
{
    if (!s || index >= s->m->num_parameters)
        return fail(s ? &s->last_error : nullptr, GOSS_ERR_ARGUMENT, "parameter index out of range");
    s->params[index] = value;
    return 0;
}

GOSS_API int goss_system_get_parameter(const goss_system* s, uint32_t index, double* value)
{
    if (!s || !value || index >= s->m->num_parameters)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "parameter index out of range");
    *value = s->params[index];
    return 0;
}

GOSS_API int goss_system_set_num_threads(goss_system* s, uint32_t num_threads)
{
    if (!s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL system");
    s->num_threads = num_threads;
    return 0;
}

GOSS_API uint32_t goss_system_get_num_threads(const goss_system* s) { return s ? s->num_threads : 0; }
GOSS_API uint32_t goss_system_num_nodes(const goss_system* s) { return s ? s->N : 0; }

GOSS_API int goss_system_set_block_size(goss_system* s, uint32_t block)
{
    if (!s || (block && (block % 32 || block > 1024)))
        return fail(s ? &s->last_error : nullptr, GOSS_ERR_ARGUMENT, "block size must be a multiple of 32 <= 1024");
    s->block = block;
    return 0;
}

GOSS_API int goss_system_status(goss_system* s, uint32_t* flags, int32_t clear)
{
    if (!s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL system");
    int rc = set_device(s);
    if (rc)
        return rc;
    uint32_t f = 0;
    CUDA_TRY(s, cudaMemcpyAsync(&f, s->d_flags, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (flags)
        *flags = f;
    if (clear) {
        CUDA_TRY(s, cudaMemsetAsync(s->d_flags, 0, sizeof(uint32_t), s->stream));
        CUDA_TRY(s, cudaMemsetAsync(s->d_node_status, 0, s->ld, s->stream));
        CUDA_TRY(s, cudaStreamSynchronize(s->stream));
        s->host_flags = 0;
    }
    return 0;
}

GOSS_API int goss_system_node_status(const goss_system* cs, uint8_t* out)
{
    auto* s = const_cast<goss_system*>(cs);
    if (!s || !out)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    int rc = set_device(s);
    if (rc)
        return rc;
    CUDA_TRY(s, cudaMemcpyAsync(out, s->d_node_status, s->N, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return 0;
}

GOSS_API int goss_system_counters(const goss_system* cs, int64_t* jac_comp, int64_t* rejected, int64_t* accepted)
{
    auto* s = const_cast<goss_system*>(cs);
    if (!s)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL system");
    uint32_t rows[3];
    if (s->solver == GOSS_THETA || s->solver == GOSS_IMPLICIT_EULER) {
        rows[0] = 4, rows[1] = 5, rows[2] = 6;  // TH_JACCOMP, TH_REJECTS, TH_ACCEPTED
    } else if (s->solver == GOSS_ESDIRK23A) {
        rows[0] = 6, rows[1] = 7, rows[2] = 8;  // ES_JACCOMP, ES_REJECTS, ES_ACCEPTED
    } else {
        for (uint32_t i = 0; i < s->N; ++i) {
            if (jac_comp)
                jac_comp[i] = 0;
            if (rejected)
                rejected[i] = 0;
            if (accepted)
                accepted[i] = 0;
        }
        return 0;
    }
    std::vector<double> buf((size_t)3 * s->N);
    int rc = to_host(s, buf.data(), s->d_sstate, 3, rows, 0);
    if (rc)
        return rc;
    for (uint32_t i = 0; i < s->N; ++i) {
        if (jac_comp)
            jac_comp[i] = (int64_t)buf[i];
        if (rejected)
            rejected[i] = (int64_t)buf[(size_t)s->N + i];
        if (accepted)
            accepted[i] = (int64_t)buf[(size_t)2 * s->N + i];
    }
    return 0;
}

GOSS_API int goss_system_device_states(goss_system* s, double** states, uint64_t* ld)
{
    if (!s || !states || !ld)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    *states = s->d_states;
    *ld = s->ld;
    return 0;
}

GOSS_API int goss_system_device_field_params(goss_system* s, double** fp, uint64_t* ld)
{
    if (!s || !fp || !ld)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    *fp = s->d_fparams;
    *ld = s->ld;
    return 0;
}

// ODESystemSolver::solve (ODESystemSolver.cpp:81-99).  The field states of
// every output time are gathered on the device into a chunk buffer and
// copied back once per chunk.
GOSS_API int goss_system_solve(goss_system* s, double* field_states, const double* t, uint64_t nt, int32_t tangled)
{
    if (!s || !t || (nt > 1 && !field_states && !s->fsi.empty()))
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    int rc = set_device(s);
    if (rc)
        return rc;
    const uint32_t nfs = (uint32_t)s->fsi.size();
    const uint64_t per = (uint64_t)s->N * nfs;
    if (nt < 2)
        return 0;
    uint64_t chunk = per ? std::max<uint64_t>(1, (256ull << 20) / (8 * per)) : 1;
    chunk = std::min<uint64_t>(chunk, nt - 1);
    double* d_out = nullptr;
    if (per) {
        CUDA_TRY(s, cudaMalloc(&d_out, sizeof(double) * per * chunk));
        rc = ensure_rows(s, s->fsi.data(), nfs);
        if (rc) {
            cudaFree(d_out);
            return rc;
        }
    }
    double t_current = t[0];
    uint64_t filled = 0, first = 1;
    for (uint64_t it = 1; it < nt; ++it) {
        const double t_next = t[it];
        rc = launch_forward(s, t_current, t_next - t_current);
        if (rc)
            break;
        if (per) {
            gather_kernel<<<grid_for(per), 256, 0, s->stream>>>(d_out + filled * per, s->d_states, s->ld, s->N, nfs,
                                                                s->d_rows, tangled);
            if (cudaGetLastError() != cudaSuccess) {
                rc = fail(&s->last_error, GOSS_ERR_CUDA, "gather launch failed");
                break;
            }
            ++filled;
            if (filled == chunk || it == nt - 1) {
                if (cudaMemcpyAsync(field_states + first * per, d_out, sizeof(double) * per * filled,
                                    cudaMemcpyDeviceToHost, s->stream) != cudaSuccess) {
                    rc = fail(&s->last_error, GOSS_ERR_CUDA, "copy of solve output failed");
                    break;
                }
                rc = check_flags(s);  // synchronises the stream
                if (rc)
                    break;
                first += filled;
                filled = 0;
            }
        }
        t_current = t_next;
    }
    if (!rc && !per)
        rc = check_flags(s);
    cudaStreamSynchronize(s->stream);
    cudaFree(d_out);
    return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched evaluation without any device allocation
// ---------------------------------------------------------------------------
// Some callers cannot let a library call cudaMalloc: a process whose GPU
// memory is owned by another allocator (a framework's caching allocator that
// has reserved the device, or a fixed memory budget) would see the call fail,
// block on the allocator's synchronisation, or fragment its pool.  For them
// goss_model_eval_noalloc keeps its working arrays (the component-major
// copies of the states, field parameters and results) in this fixed device
// array instead.  Every GPU on which this library is used holds the array
// until the process exits.
#define GOSS_NOALLOC_SCRATCH_DOUBLES (2u * 1024u * 1024u) /* 16 MiB */
static __device__ __align__(256) double g_eval_scratch[GOSS_NOALLOC_SCRATCH_DOUBLES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
struct ScratchAddress {
    unsigned long long context = 0;  // the context the address belongs to
    double* ptr = nullptr;
};
ScratchAddress g_scratch[kMaxDevices];

// Identifier of the calling thread's current CUDA context, 0 if it cannot be
// read.  The driver functions are reached through the runtime's entry-point
// query, so the library does not link the driver library itself.
unsigned long long current_context_id()
{
    typedef CUresult (*get_current_fn)(CUcontext*);
    typedef CUresult (*get_id_fn)(CUcontext, unsigned long long*);
    static get_current_fn get_current = nullptr;
    static get_id_fn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<get_current_fn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<get_id_fn>(f);
    });
    CUcontext ctx = nullptr;
    if (!get_current || get_current(&ctx) != CUDA_SUCCESS || !ctx)
        return 0;
    unsigned long long id = 0;
    if (get_id && get_id(ctx, &id) == CUDA_SUCCESS)
        return id;
    return (unsigned long long)(uintptr_t)ctx;
}

// Device address of g_eval_scratch on the current device.  In host code the
// symbol is only a host-side stand-in, so the address is looked up with the
// device current: once per device, and again when the device's context is
// no longer the one the cached address belongs to (after cudaDeviceReset the
// array lives in a new context at a new address).
int noalloc_scratch(double** out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaSetDevice(dev);  // makes the device's primary context current
    if (e != cudaSuccess)
        return fail(nullptr, GOSS_ERR_CUDA, "cannot make the current device's context current: %s",
                    cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "device ordinal %d out of range", dev);
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ScratchAddress& a = g_scratch[dev];
    if (!a.ptr || ctx == 0 || a.context != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_eval_scratch);
        if (e != cudaSuccess || !p)
            return fail(nullptr, GOSS_ERR_CUDA, "cudaGetSymbolAddress of the evaluation scratch failed: %s",
                        cudaGetErrorString(e));
        a.ptr = static_cast<double*>(p);
        a.context = ctx;
    }
    *out = a.ptr;
    return 0;
}

struct RowValues {
    double v[32];
};

// dst[r*ld + node] = vals.v[r] for every node < N (values passed by value)
__global__ void fill_rows_const_kernel(double* __restrict__ dst, uint64_t ld, uint32_t N, uint32_t k, RowValues vals)
{
    const uint64_t total = (uint64_t)N * k;
    for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(idx / N), node = (uint32_t)(idx % N);
        dst[(uint64_t)r * ld + node] = vals.v[r];
    }
}

}  // namespace

extern "C" {

GOSS_API uint64_t goss_model_eval_noalloc_capacity(void) { return GOSS_NOALLOC_SCRATCH_DOUBLES; }

// Output rows per state of goss_model_eval for `what`, 0 when the model has
// no such output (the caller reports it with eval_what_error).
static uint32_t eval_width(const goss_model_desc* m, int32_t what)
{
    switch (what) {
    case 0: return m->num_states;
    case 1: return 2 * m->num_states;
    case 2: return m->num_monitored;
    case 3: return m->has_jacobian ? m->num_states * m->num_states : 0;
    default: return 0;
    }
}

static int eval_what_error(const goss_model_desc* m, int32_t what)
{
    if (what == 2)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "No monitored in the '%s' model.", m->name);
    if (what == 3)
        return fail(nullptr, GOSS_ERR_ARGUMENT,
                    "the '%s' model was generated without the analytic Jacobian (generate_jacobian)", m->name);
    return fail(nullptr, GOSS_ERR_ARGUMENT,
                "what must be 0 (rhs), 1 (linearized), 2 (monitored) or 3 (analytic Jacobian)");
}

GOSS_API int goss_model_eval_noalloc(const goss_model_desc* m, int32_t what, int32_t precision, const double* params,
                                     const double* states, const double* field_params, const double* times,
                                     uint64_t count, double* out, void* stream)
{
    if (!m || !states || !times || !out)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    const uint32_t width = eval_width(m, what);
    if (!width)
        return eval_what_error(m, what);
    if (count == 0)
        return 0;
    const uint32_t n = m->num_states, nfp = m->num_field_parameters;
    if (nfp > 32 && !field_params)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "models with more than 32 field parameters need field_params");
    const uint64_t ld = round_up(count, 32);
    const uint64_t need = (uint64_t)(n + nfp + width) * ld;
    if (count > 0xffffffffull || need > GOSS_NOALLOC_SCRATCH_DOUBLES)
        return fail(nullptr, GOSS_ERR_ARGUMENT,
                    "goss_model_eval_noalloc: %llu states of model '%s' need %llu scratch doubles; the fixed "
                    "scratch holds %u (at most %llu states of this model)",
                    (unsigned long long)count, m->name, (unsigned long long)need, GOSS_NOALLOC_SCRATCH_DOUBLES,
                    (unsigned long long)(GOSS_NOALLOC_SCRATCH_DOUBLES / (n + nfp + width) / 32 * 32));
    // an error left by the caller's own earlier work is reported as such (and
    // left pending), not blamed on this call's kernels
    cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
        return fail(nullptr, GOSS_ERR_CUDA, "goss_model_eval_noalloc: a CUDA error from earlier work is pending: %s",
                    cudaGetErrorName(pending));
    double* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc)
        return rc;
    double* d_states = scratch;                       // [n][ld]
    double* d_fp = scratch + (uint64_t)n * ld;        // [nfp][ld]
    double* d_out = d_fp + (uint64_t)nfp * ld;        // [width][ld]
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t N = (uint32_t)count;
    scatter_kernel<<<grid_for(count * n), 256, 0, st>>>(d_states, ld, states, N, n, nullptr, 1);
    if (nfp) {
        if (field_params) {
            scatter_kernel<<<grid_for(count * nfp), 256, 0, st>>>(d_fp, ld, field_params, N, nfp, nullptr, 1);
        } else {
            RowValues vals{};
            for (uint32_t k = 0; k < nfp; ++k)
                vals.v[k] = params ? params[m->field_parameter_indices[k]]
                                   : m->default_parameters[m->field_parameter_indices[k]];
            fill_rows_const_kernel<<<grid_for(count * nfp), 256, 0, st>>>(d_fp, ld, N, nfp, vals);
        }
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(nullptr, GOSS_ERR_CUDA, "goss_model_eval_noalloc: layout kernel launch failed: %s (%s)",
                    cudaGetErrorName(e), cudaGetErrorString(e));
    goss_eval_launch L{};
    L.what = what;
    L.precision = precision;
    L.num_nodes = N;
    L.ld = ld;
    L.states = d_states;
    L.field_params = nfp ? d_fp : nullptr;
    L.times = times;
    L.out = d_out;
    L.params = params ? params : m->default_parameters;
    L.stream = stream;
    rc = m->eval(&L);
    if (rc)
        return fail(nullptr, rc, "model evaluation launch failed");
    gather_kernel<<<grid_for(count * width), 256, 0, st>>>(out, d_out, ld, N, width, nullptr, 1);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return fail(nullptr, GOSS_ERR_CUDA, "goss_model_eval_noalloc failed: %s", cudaGetErrorString(e));
    return 0;
}

// ODE::lu_factorize (ODE.cpp:69-100): Doolittle LU without pivoting.
GOSS_API int goss_lu_factorize(uint32_t un, double* mat)
{
    if (!mat && un)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL matrix");
    const int n = (int)un;
    for (int k = 1; k < n; k++) {
        for (int i = 0; i <= k - 1; ++i) {
            double sum = 0.0;
            for (int r = 0; r <= i - 1; r++)
                sum += mat[i * n + r] * mat[r * n + k];
            mat[i * n + k] -= sum;
            sum = 0.0;
            for (int r = 0; r <= i - 1; r++)
                sum += mat[k * n + r] * mat[r * n + i];
            mat[k * n + i] = (mat[k * n + i] - sum) / mat[i * n + i];
        }
        double sum = 0.0;
        for (int r = 0; r <= k - 1; r++)
            sum += mat[k * n + r] * mat[r * n + k];
        mat[k * n + k] -= sum;
    }
    return 0;
}

// ODE::forward_backward_subst (ODE.cpp:102-132)
GOSS_API int goss_forward_backward_subst(uint32_t un, const double* mat, const double* b, double* dx)
{
    if (!un)
        return 0;
    if (!mat || !b || !dx)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    const int n = (int)un;
    dx[0] = b[0];
    for (int i = 1; i < n; ++i) {
        double sum = 0.0;
        for (int j = 0; j <= i - 1; ++j)
            sum = sum + mat[i * n + j] * dx[j];
        dx[i] = b[i] - sum;
    }
    dx[n - 1] = dx[n - 1] / mat[(n - 1) * n + (n - 1)];
    for (int i = n - 2; i >= 0; i--) {
        double sum = 0;
        for (int j = i + 1; j < n; ++j)
            sum = sum + mat[i * n + j] * dx[j];
        dx[i] = (dx[i] - sum) / mat[i * n + i];
    }
    return 0;
}

// Batched model evaluation on host arrays (ODE::eval / linearized_eval).
GOSS_API int goss_model_eval(const goss_model_desc* m, int32_t what, int32_t precision, const double* params,
                             const double* states, const double* field_params, const double* times, uint64_t count,
                             double* out, int32_t device)
{
    if (!m || !states || !times || !out)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "NULL argument");
    const uint32_t rows_out = eval_width(m, what);
    if (!rows_out)
        return eval_what_error(m, what);
    if (count == 0)
        return 0;
    if (count > 0xffffffffull)
        return fail(nullptr, GOSS_ERR_ARGUMENT, "too many states");
    goss_system tmp;  // only for error plumbing
    goss_system* s = &tmp;
    CUDA_TRY(s, cudaSetDevice(device));
    const uint32_t n = m->num_states, nfp = m->num_field_parameters;
    const uint64_t ld = round_up(count, 32);
    double *d_states = nullptr, *d_fp = nullptr, *d_t = nullptr, *d_out = nullptr, *d_stage = nullptr;
    cudaStream_t st = nullptr;
    int rc = 0;
    auto cleanup = [&]() {
        cudaFree(d_states);
        cudaFree(d_fp);
        cudaFree(d_t);
        cudaFree(d_out);
        cudaFree(d_stage);
        if (st)
            cudaStreamDestroy(st);
    };
    std::vector<double> pv(m->default_parameters, m->default_parameters + m->num_parameters);
    if (params)
        pv.assign(params, params + m->num_parameters);
    if (pv.empty())
        pv.push_back(0.0);
#define EVAL_TRY(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            cleanup();                                                                   \
            return fail(nullptr, GOSS_ERR_CUDA, "CUDA error %s", cudaGetErrorString(e_)); \
        }                                                                                \
    } while (0)
    EVAL_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    EVAL_TRY(cudaMalloc(&d_states, sizeof(double) * n * ld));
    EVAL_TRY(cudaMalloc(&d_t, sizeof(double) * count));
    EVAL_TRY(cudaMalloc(&d_out, sizeof(double) * rows_out * ld));
    EVAL_TRY(cudaMalloc(&d_stage, sizeof(double) * std::max(rows_out, std::max(n, nfp)) * ld));
    EVAL_TRY(cudaMemcpyAsync(d_stage, states, sizeof(double) * n * count, cudaMemcpyHostToDevice, st));
    scatter_kernel<<<grid_for(count * n), 256, 0, st>>>(d_states, ld, d_stage, (uint32_t)count, n, nullptr, 1);
    EVAL_TRY(cudaGetLastError());
    if (nfp) {
        EVAL_TRY(cudaMalloc(&d_fp, sizeof(double) * nfp * ld));
        if (field_params) {
            EVAL_TRY(cudaStreamSynchronize(st));
            EVAL_TRY(cudaMemcpyAsync(d_stage, field_params, sizeof(double) * nfp * count, cudaMemcpyHostToDevice, st));
            scatter_kernel<<<grid_for(count * nfp), 256, 0, st>>>(d_fp, ld, d_stage, (uint32_t)count, nfp, nullptr, 1);
            EVAL_TRY(cudaGetLastError());
        } else {
            std::vector<double> fpv(nfp);
            for (uint32_t k = 0; k < nfp; ++k)
                fpv[k] = pv[m->field_parameter_indices[k]];
            double* d_v = nullptr;
            EVAL_TRY(cudaMalloc(&d_v, sizeof(double) * nfp));
            cudaMemcpy(d_v, fpv.data(), sizeof(double) * nfp, cudaMemcpyHostToDevice);
            fill_rows_kernel<<<grid_for(count * nfp), 256, 0, st>>>(d_fp, ld, (uint32_t)count, nfp, d_v);
            cudaStreamSynchronize(st);
            cudaFree(d_v);
        }
    }
    EVAL_TRY(cudaMemcpyAsync(d_t, times, sizeof(double) * count, cudaMemcpyHostToDevice, st));
    goss_eval_launch L{};
    L.what = what;
    L.precision = precision;
    L.num_nodes = (uint32_t)count;
    L.ld = ld;
    L.states = d_states;
    L.field_params = d_fp;
    L.times = d_t;
    L.out = d_out;
    L.params = pv.data();
    L.stream = st;
    rc = m->eval(&L);
    if (rc) {
        cleanup();
        return fail(nullptr, rc, "eval launch failed");
    }
    EVAL_TRY(cudaStreamSynchronize(st));
    gather_kernel<<<grid_for(count * rows_out), 256, 0, st>>>(d_stage, d_out, ld, (uint32_t)count, rows_out, nullptr,
                                                              1);
    EVAL_TRY(cudaGetLastError());
    EVAL_TRY(cudaMemcpyAsync(out, d_stage, sizeof(double) * rows_out * count, cudaMemcpyDeviceToHost, st));
    EVAL_TRY(cudaStreamSynchronize(st));
#undef EVAL_TRY
    cleanup();
    return 0;
}

}  // extern "C"
