// Heterogeneous batch: several node populations, each with its own model
// and explicit solver, advanced by ONE kernel launch.
//
// The reference runs one ODESystemSolver per population in sequence (or one
// per DOLFIN subdomain, python/goss/dolfinutils.py:519-530).  Here every
// population is cut into tiles of blockDim.x nodes; the tiles of all
// populations form one work list that a persistent grid walks either
// round-robin (schedule 0) or by claiming tiles from an atomic counter
// (schedule 1).  A generated dispatcher (batch.cu of a batch module) maps a
// population's kind to the inlined explicit_node<Model, T, Solver> of
// goss_kernels.cuh, so each node runs exactly the code of the
// single-population kernel.
#ifndef GOSS_BATCH_CUH
#define GOSS_BATCH_CUH

#include "goss_kernels.cuh"

namespace goss_b200 {

constexpr int kBatchMaxPops = 16;
constexpr int kBatchMaxParams = 768;

struct BatchPop {
    NodeIO io;
    int32_t kind;
    uint32_t num_nodes;
    uint32_t tile_begin;  // first tile of this population in the work list
    uint32_t poff;        // offset of its parameter block in P / PD
    uint32_t state_rows;  // rows staged per tile by the prefetching kernel
    uint32_t field_rows;
};

template <typename T>
struct BatchParamsT {
    T P[kBatchMaxParams];
};
template <>
struct BatchParamsT<double> {
};

template <typename T>
struct BatchArgs : BatchParamsT<T> {
    BatchPop pops[kBatchMaxPops];
    uint32_t num_pops;
    uint32_t total_tiles;
    uint32_t nodes_per_tile;
    uint32_t schedule;
    uint32_t* counters;  // [0] next tile, [1] blocks done (reset by the last block)
    double PD[kBatchMaxParams];
    __device__ __forceinline__ const T* params(uint32_t off) const
    {
        if constexpr (sizeof(T) == 8)
            return reinterpret_cast<const T*>(PD + off);
        else
            return this->P + off;
    }
};

// Resident 128-thread blocks per SM the batch kernel is compiled for.  FP32
// fits 4 blocks (128 registers): with a launch per forward it streams every
// population's states through HBM, and with all forwards in one launch it is
// bound by instruction issue, and in both cases warps in flight matter --
// measured on B200 (1.97M-node mix, 1000 fused one-step forwards): 2 blocks
// 128 ms, 3 blocks 98 ms, 4 blocks 90 ms, 5 blocks 92 ms, 6 blocks 99 ms.  FP64
// stays at the compiler's choice (its models spill heavily below ~240
// registers).
#ifndef GOSS_BATCH_MIN_BLOCKS_F32
#define GOSS_BATCH_MIN_BLOCKS_F32 4
#endif
template <typename T>
struct BatchShape {
    static constexpr int min_blocks = sizeof(T) == 4 ? GOSS_BATCH_MIN_BLOCKS_F32 : 1;
};

template <class Dispatch, typename T>
__global__ void __launch_bounds__(128, BatchShape<T>::min_blocks) batch_kernel(const __grid_constant__ BatchArgs<T> a)
{
    __shared__ uint32_t s_tile;
    uint32_t tile = blockIdx.x;
    for (;;) {
        if (a.schedule) {
            if (threadIdx.x == 0)
                s_tile = atomicAdd(&a.counters[0], 1u);
            __syncthreads();
            tile = s_tile;
            __syncthreads();
        }
        if (tile >= a.total_tiles)
            break;
        uint32_t p = 0;
        while (p + 1 < a.num_pops && tile >= a.pops[p + 1].tile_begin)
            ++p;
        const BatchPop& pop = a.pops[p];
        const uint32_t node = (tile - pop.tile_begin) * a.nodes_per_tile + threadIdx.x;
        if (node < pop.num_nodes)
            Dispatch::template run<T>(pop.kind, pop.io, node, a.params(pop.poff), a.PD + pop.poff);
        if (!a.schedule)
            tile += gridDim.x;
    }
    if (a.schedule && threadIdx.x == 0) {
        // every block has made its last claim before it counts itself done,
        // so the last one can reset the counters for the next launch
        __threadfence();
        const uint32_t done = atomicAdd(&a.counters[1], 1u);
        if (done == gridDim.x - 1) {
            atomicExch(&a.counters[0], 0u);
            atomicExch(&a.counters[1], 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// Prefetching batch kernel (schedule 2).  A launch of one or a few steps per
// node streams every population's FP64 states through HBM, so the plain kernel
// spends much of its time waiting for its loads.  Here a persistent CTA stages
// each tile's state and field-parameter rows in shared memory with bulk
// asynchronous copies (cp.async.bulk, completion on an mbarrier), one tile
// ahead: the copies of tile k+1 are in flight while tile k is computed.  Rows
// of a tile are contiguous in the component-major arrays ([row][ld], ld a
// multiple of 32, tiles a multiple of 32 nodes), so every copy starts on a
// 512-byte boundary; a ragged last tile copies an even node count (16-byte
// multiple), which stays inside the row's ld.  Waits are bounded: a CTA that
// gives up flags GOSS_FLAG_ITERATION_CAP, waits (bounded) for its copies in
// flight and returns.
// ---------------------------------------------------------------------------
constexpr uint32_t kBulkWaitLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// bounded wait for one phase of an mbarrier; false when the limit ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kBulkWaitLimit; ++i)
        if (mbar_try_wait(bar, parity))
            return true;
    return false;
}

template <typename T>
__device__ __forceinline__ uint32_t batch_pop_of(const BatchArgs<T>& a, uint32_t tile)
{
    uint32_t p = 0;
    while (p + 1 < a.num_pops && tile >= a.pops[p + 1].tile_begin)
        ++p;
    return p;
}

// thread 0: stage the rows of `tile` into dst ([rows][tn] doubles)
template <typename T>
__device__ __forceinline__ void batch_stage(const BatchArgs<T>& a, uint32_t tile, double* dst, uint32_t tn,
                                            uint64_t* bar)
{
    const BatchPop& pop = a.pops[batch_pop_of(a, tile)];
    const uint32_t start = (tile - pop.tile_begin) * tn;
    const uint32_t cnt = min(tn, pop.num_nodes - start);
    const uint32_t cnt2 = (cnt + 1u) & ~1u;  // even: a multiple of 16 bytes
    const uint32_t bytes = cnt2 * (uint32_t)sizeof(double);
    mbar_arrive_expect_tx(bar, bytes * (pop.state_rows + pop.field_rows));
    for (uint32_t r = 0; r < pop.state_rows; ++r)
        bulk_copy_g2s(dst + (uint64_t)r * tn, pop.io.states + (uint64_t)r * pop.io.ld + start, bytes, bar);
    for (uint32_t f = 0; f < pop.field_rows; ++f)
        bulk_copy_g2s(dst + (uint64_t)(pop.state_rows + f) * tn, pop.io.fparams + (uint64_t)f * pop.io.ld + start,
                      bytes, bar);
}

template <class Dispatch, typename T>
__global__ void __launch_bounds__(128, BatchShape<T>::min_blocks)
batch_kernel_prefetch(const __grid_constant__ BatchArgs<T> a)
{
    constexpr uint32_t R = Dispatch::max_rows;
    extern __shared__ __align__(128) double s_rows[];  // [2][R][tn]
    __shared__ __align__(8) uint64_t s_bar[2];
    const uint32_t tn = a.nodes_per_tile;
    if (threadIdx.x == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t tile = blockIdx.x;
    if (threadIdx.x == 0 && tile < a.total_tiles)
        batch_stage(a, tile, s_rows, tn, &s_bar[0]);
    uint32_t parity[2] = {0u, 0u};
    bool in_flight[2] = {tile < a.total_tiles, false};
    int timed_out = 0;
    for (uint32_t k = 0; tile < a.total_tiles; tile += gridDim.x, ++k) {
        const uint32_t b = k & 1u;
        const uint32_t next = tile + gridDim.x;
        __syncthreads();  // every thread has read buffer b^1 (the previous tile)
        if (next < a.total_tiles) {
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                batch_stage(a, next, s_rows + (uint64_t)(b ^ 1u) * R * tn, tn, &s_bar[b ^ 1u]);
            }
            in_flight[b ^ 1u] = true;
        }
        const bool ok = mbar_wait_bounded(&s_bar[b], parity[b]);
        if (__syncthreads_or(!ok)) {  // one decision for the whole CTA
            timed_out = 1;
            break;
        }
        parity[b] ^= 1u;
        in_flight[b] = false;
        const BatchPop& pop = a.pops[batch_pop_of(a, tile)];
        const uint32_t node = (tile - pop.tile_begin) * tn + threadIdx.x;
        if (node < pop.num_nodes)
            Dispatch::template run_from<T>(pop.kind, pop.io, node, a.params(pop.poff), a.PD + pop.poff,
                                           s_rows + (uint64_t)b * R * tn + threadIdx.x, tn);
    }
    if (timed_out) {
        if (threadIdx.x == 0)
            atomicOr(a.pops[0].io.flags, GOSS_FLAG_ITERATION_CAP);
        // let the copies still in flight land before the CTA's shared memory goes away
        for (int q = 0; q < 2; ++q)
            if (in_flight[q])
                mbar_wait_bounded(&s_bar[q], parity[q]);
    }
}

// Host side: fill a BatchArgs from a goss_batch_launch; ParamBlock(kind, params, out)
// writes the FP64 parameter block (parameters + derived constants) of a kind.
template <class Dispatch, typename T>
inline int launch_batch_t(const goss_batch_launch* L)
{
    if (L->num_pops == 0)
        return 0;
    if (L->num_pops > (uint32_t)kBatchMaxPops)
        return GOSS_ERR_ARGUMENT;
    BatchArgs<T> a;
    a.num_pops = L->num_pops;
    a.nodes_per_tile = L->block ? L->block : 128;
    a.schedule = L->schedule;
    a.counters = L->counters;
    uint32_t off = 0, tiles = 0;
    for (uint32_t i = 0; i < L->num_pops; ++i) {
        const goss_batch_pop& q = L->pops[L->order ? L->order[i] : i];
        BatchPop& p = a.pops[i];
        const int np = Dispatch::param_block_size(q.kind);
        if (np < 0 || off + (uint32_t)np > (uint32_t)kBatchMaxParams)
            return GOSS_ERR_ARGUMENT;
        Dispatch::param_block(q.kind, q.params, a.PD + off);
        if constexpr (sizeof(T) == 4)
            for (int k = 0; k < np; ++k)
                a.P[off + k] = T(a.PD[off + k]);
        const unsigned long nsteps = explicit_num_steps(q.solver_params->ldt, L->interval);
        p.io = NodeIO{q.states, q.field_params, q.node_status, q.flags, q.ld, nsteps, L->t, L->interval / nsteps,
                      q.solver_params->delta, L->forwards ? L->forwards : 1u, L->first_forward, L->interval};
        p.kind = q.kind;
        p.num_nodes = q.num_nodes;
        Dispatch::row_counts(q.kind, &p.state_rows, &p.field_rows);
        p.tile_begin = tiles;
        p.poff = off;
        off += (uint32_t)np;
        tiles += (q.num_nodes + a.nodes_per_tile - 1) / a.nodes_per_tile;
    }
    a.total_tiles = tiles;
    if (tiles == 0)
        return 0;
    const unsigned block = a.nodes_per_tile;
    if (L->schedule == 2) {
        // persistent grid of prefetching CTAs: as many as are resident
        const size_t shm = 2ull * Dispatch::max_rows * block * sizeof(double);
        auto kern = batch_kernel_prefetch<Dispatch, T>;
        if (shm > 48 * 1024 &&
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) != cudaSuccess)
            return GOSS_ERR_CUDA;
        unsigned grid = L->grid;
        if (!grid) {
            int dev = 0, sms = 0, active = 0;
            if (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&active, kern, (int)block, shm) != cudaSuccess)
                return GOSS_ERR_CUDA;
            grid = (unsigned)(sms * (active > 0 ? active : 1));
        }
        if (grid > tiles)
            grid = tiles;
        kern<<<grid, block, shm, (cudaStream_t)L->stream>>>(a);
        return cudaPeekAtLastError() == cudaSuccess ? 0 : GOSS_ERR_CUDA;
    }
    unsigned grid = L->grid ? L->grid : tiles;
    if (grid > tiles)
        grid = tiles;
    batch_kernel<Dispatch, T><<<grid, block, 0, (cudaStream_t)L->stream>>>(a);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : GOSS_ERR_CUDA;
}

template <class Dispatch>
inline int launch_batch(const goss_batch_launch* L)
{
    return L->precision == GOSS_FP32 ? launch_batch_t<Dispatch, float>(L) : launch_batch_t<Dispatch, double>(L);
}

}  // namespace goss_b200
#endif
