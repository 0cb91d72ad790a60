// Generated by goss_b200.codegen for model 'tentusscher_2004_mcell' (variant tentusscher_2004_mcell__b16bd706); do not edit.
// sm_100a solver kernels instantiated for this model and its goss_model_desc factory.
#include "goss_adjoint.cuh"
#include "goss_kernels.cuh"
#include "device.cuh"

namespace {
using Model = goss_b200::models::M_tentusscher_2004_mcell__b16bd706;
static const char* const state_names[17] = {"Xr1", "Xr2", "Xs", "m", "h", "j", "d", "f", "fCa", "s", "r", "g", "Ca_i", "Ca_SR", "Na_i", "V", "K_i"};
static const char* const parameter_names[45] = {"P_kna", "g_K1", "g_Kr", "g_Ks", "g_Na", "g_bna", "g_CaL", "g_bca", "g_to", "K_mNa", "K_mk", "P_NaK", "K_NaCa", "K_sat", "Km_Ca", "Km_Nai", "alpha", "gamma", "K_pCa", "g_pCa", "g_pK", "Buf_c", "Buf_sr", "Ca_o", "K_buf_c", "K_buf_sr", "K_up", "V_leak", "V_sr", "Vmax_up", "a_rel", "b_rel", "c_rel", "tau_g", "Na_o", "Cm", "F", "R", "T", "V_c", "stim_amplitude", "stim_duration", "stim_period", "stim_start", "K_o"};
static const char* const field_parameter_names[2] = {"g_Kr", "g_CaL"};
static const uint32_t field_parameter_indices[2] = {2, 6};
static const double initial_conditions[17] = {0.0, 1.0, 0.0, 0.0, 0.75, 0.75, 0.0, 1.0, 1.0, 1.0, 0.0, 1.0, 0.0002, 0.2, 11.6, -86.2, 138.3};
static const double default_parameters[45] = {0.03, 5.405, 0.096, 0.062, 14.838, 0.00029, 0.000175, 0.000592, 0.294, 40.0, 1.0, 1.362, 1000.0, 0.1, 1.38, 87.5, 2.5, 0.35, 0.0005, 0.825, 0.0146, 0.15, 10.0, 2.0, 0.001, 0.3, 0.00025, 8e-05, 0.001094, 0.000425, 0.016464, 0.25, 0.008232, 2.0, 140.0, 0.185, 96485.3415, 8314.472, 310.0, 0.016404, 0.0, 1.0, 1000.0, 10.0, 5.4};
static const uint8_t linear_terms[17] = {1, 1, 1, 1, 1, 1, 1, 1, 0, 1, 1, 0, 0, 0, 0, 0, 0};
static const uint32_t op_lin[9] = {300, 777, 184, 102, 4, 9, 0, 34, 26};
static const uint32_t op_rhs[9] = {157, 270, 83, 52, 4, 3, 0, 26, 22};
int launch(const goss_launch* L) { return goss_b200::launch_solver<Model>(L); }
int eval(const goss_eval_launch* L) { return goss_b200::launch_eval<Model>(L); }
uint32_t rows(int32_t s) { return goss_b200::solver_state_rows<Model>(s); }
int adjoint(const goss_adjoint_launch* L) { return goss_b200::launch_adjoint<Model>(L); }
}  // namespace

extern "C" GOSS_API const goss_model_desc* goss_b200_model_tentusscher_2004_mcell__b16bd706(void)
{
    static const goss_model_desc d = {
        GOSS_B200_ABI_VERSION,
        "tentusscher_2004_mcell",
        17u, 45u, 2u, 0u,
        state_names, parameter_names, field_parameter_names, field_parameter_indices,
        initial_conditions, default_parameters, linear_terms,
        (1u << GOSS_NUM_SOLVERS) - 1u,
        launch, eval, rows, op_lin, op_rhs, adjoint,
        1u, 71u,
    };
    return &d;
}
