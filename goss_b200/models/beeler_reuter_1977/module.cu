// Generated by goss_b200.codegen for model 'beeler_reuter_1977' (variant beeler_reuter_1977); do not edit.
// sm_100a solver kernels instantiated for this model and its goss_model_desc factory.
#include "goss_adjoint.cuh"
#include "goss_kernels.cuh"
#include "device.cuh"

namespace {
using Model = goss_b200::models::M_beeler_reuter_1977;
static const char* const state_names[8] = {"m", "h", "j", "Cai", "d", "f", "x1", "V"};
static const char* const parameter_names[10] = {"E_Na", "g_Na", "g_Nac", "g_s", "IstimAmplitude", "IstimEnd", "IstimPeriod", "IstimPulseDuration", "IstimStart", "C"};
static const char* const field_parameter_names[1] = {nullptr};
static const uint32_t field_parameter_indices[1] = {0};
static const double initial_conditions[8] = {0.011, 0.988, 0.975, 0.0001, 0.003, 0.994, 0.0001, -84.624};
static const double default_parameters[10] = {50.0, 0.04, 3e-05, 0.0005, 0.5, 50000.0, 1000.0, 1.0, 10.0, 0.01};
static const uint8_t linear_terms[8] = {1, 1, 1, 0, 1, 1, 1, 0};
static const uint32_t op_lin[9] = {77, 163, 23, 38, 1, 0, 0, 11, 12};
static const uint32_t op_rhs[9] = {53, 99, 14, 25, 1, 0, 0, 9, 9};
int launch(const goss_launch* L) { return goss_b200::launch_solver<Model>(L); }
int eval(const goss_eval_launch* L) { return goss_b200::launch_eval<Model>(L); }
uint32_t rows(int32_t s) { return goss_b200::solver_state_rows<Model>(s); }
int adjoint(const goss_adjoint_launch* L) { return goss_b200::launch_adjoint<Model>(L); }
}  // namespace

extern "C" GOSS_API const goss_model_desc* goss_b200_model_beeler_reuter_1977(void)
{
    static const goss_model_desc d = {
        GOSS_B200_ABI_VERSION,
        "beeler_reuter_1977",
        8u, 10u, 0u, 0u,
        state_names, parameter_names, field_parameter_names, field_parameter_indices,
        initial_conditions, default_parameters, linear_terms,
        (1u << GOSS_NUM_SOLVERS) - 1u,
        launch, eval, rows, op_lin, op_rhs, adjoint,
        0u, 24u,
    };
    return &d;
}
