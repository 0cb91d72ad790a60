// Generated by goss_b200.codegen for model 'fhn' (variant fhn); do not edit.
// sm_100a solver kernels instantiated for this model and its goss_model_desc factory.
#include "goss_adjoint.cuh"
#include "goss_kernels.cuh"
#include "device.cuh"

namespace {
using Model = goss_b200::models::M_fhn;
static const char* const state_names[2] = {"v", "s"};
static const char* const parameter_names[11] = {"a", "b", "c_1", "c_2", "c_3", "stim_amplitude", "stim_duration", "stim_period", "stim_start", "v_peak", "v_rest"};
static const char* const field_parameter_names[1] = {nullptr};
static const uint32_t field_parameter_indices[1] = {0};
static const double initial_conditions[2] = {-85.0, 0.0};
static const double default_parameters[11] = {0.13, 0.013, 0.26, 0.1, 1.0, 50.0, 1.0, 1000.0, 1.0, 40.0, -85.0};
static const uint8_t linear_terms[2] = {0, 1};
static const uint32_t op_lin[9] = {23, 41, 8, 2, 0, 0, 0, 0, 0};
static const uint32_t op_rhs[9] = {14, 21, 4, 2, 0, 0, 0, 0, 0};
int launch(const goss_launch* L) { return goss_b200::launch_solver<Model>(L); }
int eval(const goss_eval_launch* L) { return goss_b200::launch_eval<Model>(L); }
uint32_t rows(int32_t s) { return goss_b200::solver_state_rows<Model>(s); }
int adjoint(const goss_adjoint_launch* L) { return goss_b200::launch_adjoint<Model>(L); }
}  // namespace

extern "C" GOSS_API const goss_model_desc* goss_b200_model_fhn(void)
{
    static const goss_model_desc d = {
        GOSS_B200_ABI_VERSION,
        "fhn",
        2u, 11u, 0u, 0u,
        state_names, parameter_names, field_parameter_names, field_parameter_indices,
        initial_conditions, default_parameters, linear_terms,
        (1u << GOSS_NUM_SOLVERS) - 1u,
        launch, eval, rows, op_lin, op_rhs, adjoint,
        0u, 4u,
    };
    return &d;
}
