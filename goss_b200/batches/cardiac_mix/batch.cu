// Generated by goss_b200.codegen.batchgen (batch cardiac_mix); do not edit.
// One persistent kernel for the kinds: fitzhughnagumo__5dc98ee0/RK4, oscilator__5dc98ee0/RK4, tentusscher_2004_mcell__dc47354d/GRL1, tentusscher_panfilov_2006_M_cell__dc47354d/GRL1
#include "goss_batch.cuh"
#include "models/fitzhughnagumo__5dc98ee0/device.cuh"
#include "models/oscilator__5dc98ee0/device.cuh"
#include "models/tentusscher_2004_mcell__dc47354d/device.cuh"
#include "models/tentusscher_panfilov_2006_M_cell__dc47354d/device.cuh"

namespace {
struct Dispatch {
    template <typename T>
    __device__ static __forceinline__ void run(int kind, const goss_b200::NodeIO& io, uint32_t node,
                                               const T* __restrict__ P, const double* __restrict__ PD)
    {
        switch (kind) {
        case 0: goss_b200::explicit_node<goss_b200::models::M_fitzhughnagumo__5dc98ee0, T, goss_b200::Explicit::RK4>(io, node, P, PD); break;
        case 1: goss_b200::explicit_node<goss_b200::models::M_oscilator__5dc98ee0, T, goss_b200::Explicit::RK4>(io, node, P, PD); break;
        case 2: goss_b200::explicit_node<goss_b200::models::M_tentusscher_2004_mcell__dc47354d, T, goss_b200::Explicit::GRL1>(io, node, P, PD); break;
        case 3: goss_b200::explicit_node<goss_b200::models::M_tentusscher_panfilov_2006_M_cell__dc47354d, T, goss_b200::Explicit::GRL1>(io, node, P, PD); break;
        default: break;
        }
    }
    // the same with the node's state rows, then its field-parameter rows, at
    // rows[r * stride] (a tile staged in shared memory)
    static constexpr int max_rows = 23;
    template <typename T>
    __device__ static __forceinline__ void run_from(int kind, const goss_b200::NodeIO& io, uint32_t node,
                                                    const T* __restrict__ P, const double* __restrict__ PD,
                                                    const double* rows, uint32_t stride)
    {
        switch (kind) {
        case 0: goss_b200::explicit_node_from<goss_b200::models::M_fitzhughnagumo__5dc98ee0, T, goss_b200::Explicit::RK4>(io, node, P, PD, rows, stride); break;
        case 1: goss_b200::explicit_node_from<goss_b200::models::M_oscilator__5dc98ee0, T, goss_b200::Explicit::RK4>(io, node, P, PD, rows, stride); break;
        case 2: goss_b200::explicit_node_from<goss_b200::models::M_tentusscher_2004_mcell__dc47354d, T, goss_b200::Explicit::GRL1>(io, node, P, PD, rows, stride); break;
        case 3: goss_b200::explicit_node_from<goss_b200::models::M_tentusscher_panfilov_2006_M_cell__dc47354d, T, goss_b200::Explicit::GRL1>(io, node, P, PD, rows, stride); break;
        default: break;
        }
    }
    static int param_block_size(int kind)
    {
        switch (kind) {
        case 0: return goss_b200::Dims<goss_b200::models::M_fitzhughnagumo__5dc98ee0>::np;
        case 1: return goss_b200::Dims<goss_b200::models::M_oscilator__5dc98ee0>::np;
        case 2: return goss_b200::Dims<goss_b200::models::M_tentusscher_2004_mcell__dc47354d>::np;
        case 3: return goss_b200::Dims<goss_b200::models::M_tentusscher_panfilov_2006_M_cell__dc47354d>::np;
        default: return -1;
        }
    }
    static void row_counts(int kind, uint32_t* ns, uint32_t* nf)
    {
        switch (kind) {
        case 0: *ns = 2; *nf = 2; return;
        case 1: *ns = 2; *nf = 2; return;
        case 2: *ns = 17; *nf = 4; return;
        case 3: *ns = 19; *nf = 4; return;
        default: *ns = *nf = 0; return;
        }
    }
    static void param_block(int kind, const double* params, double* out)
    {
        switch (kind) {
        case 0: { double tmp[goss_b200::Dims<goss_b200::models::M_fitzhughnagumo__5dc98ee0>::np]; goss_b200::parameter_block<goss_b200::models::M_fitzhughnagumo__5dc98ee0>(params, tmp); for (int i = 0; i < goss_b200::Dims<goss_b200::models::M_fitzhughnagumo__5dc98ee0>::np; ++i) out[i] = tmp[i]; return; }
        case 1: { double tmp[goss_b200::Dims<goss_b200::models::M_oscilator__5dc98ee0>::np]; goss_b200::parameter_block<goss_b200::models::M_oscilator__5dc98ee0>(params, tmp); for (int i = 0; i < goss_b200::Dims<goss_b200::models::M_oscilator__5dc98ee0>::np; ++i) out[i] = tmp[i]; return; }
        case 2: { double tmp[goss_b200::Dims<goss_b200::models::M_tentusscher_2004_mcell__dc47354d>::np]; goss_b200::parameter_block<goss_b200::models::M_tentusscher_2004_mcell__dc47354d>(params, tmp); for (int i = 0; i < goss_b200::Dims<goss_b200::models::M_tentusscher_2004_mcell__dc47354d>::np; ++i) out[i] = tmp[i]; return; }
        case 3: { double tmp[goss_b200::Dims<goss_b200::models::M_tentusscher_panfilov_2006_M_cell__dc47354d>::np]; goss_b200::parameter_block<goss_b200::models::M_tentusscher_panfilov_2006_M_cell__dc47354d>(params, tmp); for (int i = 0; i < goss_b200::Dims<goss_b200::models::M_tentusscher_panfilov_2006_M_cell__dc47354d>::np; ++i) out[i] = tmp[i]; return; }
        default: return;
        }
    }
};
static const char* const kind_variants[] = {"fitzhughnagumo__5dc98ee0", "oscilator__5dc98ee0", "tentusscher_2004_mcell__dc47354d", "tentusscher_panfilov_2006_M_cell__dc47354d"};
static const int32_t kind_solvers[] = {1, 1, 2, 2};
static const uint32_t kind_num_states[] = {2, 2, 17, 19};
int launch(const goss_batch_launch* L) { return goss_b200::launch_batch<Dispatch>(L); }
}  // namespace

extern "C" GOSS_API const goss_batch_desc* goss_b200_batch_cardiac_mix(void)
{
    static const goss_batch_desc d = {GOSS_B200_ABI_VERSION, "cardiac_mix", 4u, kind_variants,
                                      kind_solvers, kind_num_states, launch};
    return &d;
}
