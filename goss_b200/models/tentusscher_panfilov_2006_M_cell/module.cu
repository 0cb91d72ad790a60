// Generated by goss_b200.codegen for model 'tentusscher_panfilov_2006_M_cell' (variant tentusscher_panfilov_2006_M_cell); do not edit.
// sm_100a solver kernels instantiated for this model and its goss_model_desc factory.
#include "goss_adjoint.cuh"
#include "goss_kernels.cuh"
#include "device.cuh"

namespace {
using Model = goss_b200::models::M_tentusscher_panfilov_2006_M_cell;
static const char* const state_names[19] = {"Xr1", "Xr2", "Xs", "m", "h", "j", "d", "f", "f2", "fCass", "s", "r", "Ca_i", "R_prime", "Ca_SR", "Ca_ss", "Na_i", "V", "K_i"};
static const char* const parameter_names[53] = {"P_kna", "g_K1", "g_Kr", "g_Ks", "g_Na", "g_bna", "g_CaL", "g_bca", "g_to", "K_mNa", "K_mk", "P_NaK", "K_NaCa", "K_sat", "Km_Ca", "Km_Nai", "alpha", "gamma", "K_pCa", "g_pCa", "g_pK", "Buf_c", "Buf_sr", "Buf_ss", "Ca_o", "EC", "K_buf_c", "K_buf_sr", "K_buf_ss", "K_up", "V_leak", "V_rel", "V_sr", "V_ss", "V_xfer", "Vmax_up", "k1_prime", "k2_prime", "k3", "k4", "max_sr", "min_sr", "Na_o", "Cm", "F", "R", "T", "V_c", "stim_amplitude", "stim_duration", "stim_period", "stim_start", "K_o"};
static const char* const field_parameter_names[1] = {nullptr};
static const uint32_t field_parameter_indices[1] = {0};
static const double initial_conditions[19] = {0.0165, 0.473, 0.0174, 0.00165, 0.749, 0.6788, 3.288e-05, 0.7026, 0.9526, 0.9942, 0.999998, 2.347e-08, 0.000153, 0.8978, 4.272, 0.00042, 10.132, -85.423, 138.52};
static const double default_parameters[53] = {0.03, 5.405, 0.153, 0.098, 14.838, 0.00029, 3.98e-05, 0.000592, 0.294, 40.0, 1.0, 2.724, 1000.0, 0.1, 1.38, 87.5, 2.5, 0.35, 0.0005, 0.1238, 0.0146, 0.2, 10.0, 0.4, 2.0, 1.5, 0.001, 0.3, 0.00025, 0.00025, 0.00036, 0.102, 0.001094, 5.468e-05, 0.0038, 0.006375, 0.15, 0.045, 0.06, 0.005, 2.5, 1.0, 140.0, 0.185, 96485.3415, 8314.472, 310.0, 0.016404, 52.0, 1.0, 1000.0, 10.0, 5.4};
static const uint8_t linear_terms[19] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 1, 0, 0, 0, 0, 0};
static const uint32_t op_lin[9] = {337, 860, 205, 105, 4, 9, 0, 16, 18};
static const uint32_t op_rhs[9] = {176, 288, 92, 55, 4, 3, 0, 14, 15};
int launch(const goss_launch* L) { return goss_b200::launch_solver<Model>(L); }
int eval(const goss_eval_launch* L) { return goss_b200::launch_eval<Model>(L); }
uint32_t rows(int32_t s) { return goss_b200::solver_state_rows<Model>(s); }
int adjoint(const goss_adjoint_launch* L) { return goss_b200::launch_adjoint<Model>(L); }
}  // namespace

extern "C" GOSS_API const goss_model_desc* goss_b200_model_tentusscher_panfilov_2006_M_cell(void)
{
    static const goss_model_desc d = {
        GOSS_B200_ABI_VERSION,
        "tentusscher_panfilov_2006_M_cell",
        19u, 53u, 0u, 0u,
        state_names, parameter_names, field_parameter_names, field_parameter_indices,
        initial_conditions, default_parameters, linear_terms,
        (1u << GOSS_NUM_SOLVERS) - 1u,
        launch, eval, rows, op_lin, op_rhs, adjoint,
        0u, 82u,
    };
    return &d;
}
