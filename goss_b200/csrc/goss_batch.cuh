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

// Resident 128-thread blocks per SM the batch kernel is compiled for: a launch
// streams every population's states through HBM for a step or a few, so
// warps in flight matter -- FP32 fits 4 blocks (128 registers), FP64 stays at
// the compiler's choice (its models spill heavily below ~240 registers).
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
                      q.solver_params->delta};
        p.kind = q.kind;
        p.num_nodes = q.num_nodes;
        p.tile_begin = tiles;
        p.poff = off;
        off += (uint32_t)np;
        tiles += (q.num_nodes + a.nodes_per_tile - 1) / a.nodes_per_tile;
    }
    a.total_tiles = tiles;
    if (tiles == 0)
        return 0;
    const unsigned block = a.nodes_per_tile;
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
