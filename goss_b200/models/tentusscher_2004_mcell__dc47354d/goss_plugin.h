// Generated by goss_b200.codegen from the 'tentusscher_2004_mcell' model; do not edit.
// goss::ParameterizedODE plugin consumed by the oracle build of the reference solvers.
#ifndef TENTUSSCHER_2004_MCELL_GOSS_PLUGIN_H
#define TENTUSSCHER_2004_MCELL_GOSS_PLUGIN_H
#include <cmath>
#include <memory>
#include <stdexcept>
#include "goss/ParameterizedODE.h"

namespace goss {
class Tentusscher_2004_mcell : public ParameterizedODE
{
  public:
    Tentusscher_2004_mcell() : ParameterizedODE(17, 45, 0, 4, 0), P_kna(0.03), g_K1(5.405), g_Kr(0.096), g_Ks(0.062), g_Na(14.838), g_bna(0.00029), g_CaL(0.000175), g_bca(0.000592), g_to(0.294), K_mNa(40.0), K_mk(1.0), P_NaK(1.362), K_NaCa(1000.0), K_sat(0.1), Km_Ca(1.38), Km_Nai(87.5), alpha(2.5), gamma(0.35), K_pCa(0.0005), g_pCa(0.825), g_pK(0.0146), Buf_c(0.15), Buf_sr(10.0), Ca_o(2.0), K_buf_c(0.001), K_buf_sr(0.3), K_up(0.00025), V_leak(8e-05), V_sr(0.001094), Vmax_up(0.000425), a_rel(0.016464), b_rel(0.25), c_rel(0.008232), tau_g(2.0), Na_o(140.0), Cm(0.185), F(96485.3415), R(8314.472), T(310.0), V_c(0.016404), stim_amplitude(0.0), stim_duration(1.0), stim_period(1000.0), stim_start(10.0), K_o(5.4)
    {
        _state_names[0] = "Xr1";
        _state_names[1] = "Xr2";
        _state_names[2] = "Xs";
        _state_names[3] = "m";
        _state_names[4] = "h";
        _state_names[5] = "j";
        _state_names[6] = "d";
        _state_names[7] = "f";
        _state_names[8] = "fCa";
        _state_names[9] = "s";
        _state_names[10] = "r";
        _state_names[11] = "g";
        _state_names[12] = "Ca_i";
        _state_names[13] = "Ca_SR";
        _state_names[14] = "Na_i";
        _state_names[15] = "V";
        _state_names[16] = "K_i";
        _parameter_names[0] = "P_kna";
        _parameter_names[1] = "g_K1";
        _parameter_names[2] = "g_Kr";
        _parameter_names[3] = "g_Ks";
        _parameter_names[4] = "g_Na";
        _parameter_names[5] = "g_bna";
        _parameter_names[6] = "g_CaL";
        _parameter_names[7] = "g_bca";
        _parameter_names[8] = "g_to";
        _parameter_names[9] = "K_mNa";
        _parameter_names[10] = "K_mk";
        _parameter_names[11] = "P_NaK";
        _parameter_names[12] = "K_NaCa";
        _parameter_names[13] = "K_sat";
        _parameter_names[14] = "Km_Ca";
        _parameter_names[15] = "Km_Nai";
        _parameter_names[16] = "alpha";
        _parameter_names[17] = "gamma";
        _parameter_names[18] = "K_pCa";
        _parameter_names[19] = "g_pCa";
        _parameter_names[20] = "g_pK";
        _parameter_names[21] = "Buf_c";
        _parameter_names[22] = "Buf_sr";
        _parameter_names[23] = "Ca_o";
        _parameter_names[24] = "K_buf_c";
        _parameter_names[25] = "K_buf_sr";
        _parameter_names[26] = "K_up";
        _parameter_names[27] = "V_leak";
        _parameter_names[28] = "V_sr";
        _parameter_names[29] = "Vmax_up";
        _parameter_names[30] = "a_rel";
        _parameter_names[31] = "b_rel";
        _parameter_names[32] = "c_rel";
        _parameter_names[33] = "tau_g";
        _parameter_names[34] = "Na_o";
        _parameter_names[35] = "Cm";
        _parameter_names[36] = "F";
        _parameter_names[37] = "R";
        _parameter_names[38] = "T";
        _parameter_names[39] = "V_c";
        _parameter_names[40] = "stim_amplitude";
        _parameter_names[41] = "stim_duration";
        _parameter_names[42] = "stim_period";
        _parameter_names[43] = "stim_start";
        _parameter_names[44] = "K_o";
        _field_parameter_names[0] = "g_Kr";
        _field_parameter_names[1] = "g_Ks";
        _field_parameter_names[2] = "g_CaL";
        _field_parameter_names[3] = "g_to";
        _param_to_value["P_kna"] = &P_kna;
        _param_to_value["g_K1"] = &g_K1;
        _param_to_value["g_Kr"] = &g_Kr;
        _param_to_value["g_Ks"] = &g_Ks;
        _param_to_value["g_Na"] = &g_Na;
        _param_to_value["g_bna"] = &g_bna;
        _param_to_value["g_CaL"] = &g_CaL;
        _param_to_value["g_bca"] = &g_bca;
        _param_to_value["g_to"] = &g_to;
        _param_to_value["K_mNa"] = &K_mNa;
        _param_to_value["K_mk"] = &K_mk;
        _param_to_value["P_NaK"] = &P_NaK;
        _param_to_value["K_NaCa"] = &K_NaCa;
        _param_to_value["K_sat"] = &K_sat;
        _param_to_value["Km_Ca"] = &Km_Ca;
        _param_to_value["Km_Nai"] = &Km_Nai;
        _param_to_value["alpha"] = &alpha;
        _param_to_value["gamma"] = &gamma;
        _param_to_value["K_pCa"] = &K_pCa;
        _param_to_value["g_pCa"] = &g_pCa;
        _param_to_value["g_pK"] = &g_pK;
        _param_to_value["Buf_c"] = &Buf_c;
        _param_to_value["Buf_sr"] = &Buf_sr;
        _param_to_value["Ca_o"] = &Ca_o;
        _param_to_value["K_buf_c"] = &K_buf_c;
        _param_to_value["K_buf_sr"] = &K_buf_sr;
        _param_to_value["K_up"] = &K_up;
        _param_to_value["V_leak"] = &V_leak;
        _param_to_value["V_sr"] = &V_sr;
        _param_to_value["Vmax_up"] = &Vmax_up;
        _param_to_value["a_rel"] = &a_rel;
        _param_to_value["b_rel"] = &b_rel;
        _param_to_value["c_rel"] = &c_rel;
        _param_to_value["tau_g"] = &tau_g;
        _param_to_value["Na_o"] = &Na_o;
        _param_to_value["Cm"] = &Cm;
        _param_to_value["F"] = &F;
        _param_to_value["R"] = &R;
        _param_to_value["T"] = &T;
        _param_to_value["V_c"] = &V_c;
        _param_to_value["stim_amplitude"] = &stim_amplitude;
        _param_to_value["stim_duration"] = &stim_duration;
        _param_to_value["stim_period"] = &stim_period;
        _param_to_value["stim_start"] = &stim_start;
        _param_to_value["K_o"] = &K_o;
        _linear_terms[0] = 1;
        _linear_terms[1] = 1;
        _linear_terms[2] = 1;
        _linear_terms[3] = 1;
        _linear_terms[4] = 1;
        _linear_terms[5] = 1;
        _linear_terms[6] = 1;
        _linear_terms[7] = 1;
        _linear_terms[9] = 1;
        _linear_terms[10] = 1;
    }
    Tentusscher_2004_mcell(const Tentusscher_2004_mcell& ode) : ParameterizedODE(ode), P_kna(ode.P_kna), g_K1(ode.g_K1), g_Kr(ode.g_Kr), g_Ks(ode.g_Ks), g_Na(ode.g_Na), g_bna(ode.g_bna), g_CaL(ode.g_CaL), g_bca(ode.g_bca), g_to(ode.g_to), K_mNa(ode.K_mNa), K_mk(ode.K_mk), P_NaK(ode.P_NaK), K_NaCa(ode.K_NaCa), K_sat(ode.K_sat), Km_Ca(ode.Km_Ca), Km_Nai(ode.Km_Nai), alpha(ode.alpha), gamma(ode.gamma), K_pCa(ode.K_pCa), g_pCa(ode.g_pCa), g_pK(ode.g_pK), Buf_c(ode.Buf_c), Buf_sr(ode.Buf_sr), Ca_o(ode.Ca_o), K_buf_c(ode.K_buf_c), K_buf_sr(ode.K_buf_sr), K_up(ode.K_up), V_leak(ode.V_leak), V_sr(ode.V_sr), Vmax_up(ode.Vmax_up), a_rel(ode.a_rel), b_rel(ode.b_rel), c_rel(ode.c_rel), tau_g(ode.tau_g), Na_o(ode.Na_o), Cm(ode.Cm), F(ode.F), R(ode.R), T(ode.T), V_c(ode.V_c), stim_amplitude(ode.stim_amplitude), stim_duration(ode.stim_duration), stim_period(ode.stim_period), stim_start(ode.stim_start), K_o(ode.K_o) {}

    void eval(const double* states, double time, double* values)
    {
        const double Xr1 = states[0];
        const double Xr2 = states[1];
        const double Xs = states[2];
        const double m = states[3];
        const double h = states[4];
        const double j = states[5];
        const double d = states[6];
        const double f = states[7];
        const double fCa = states[8];
        const double s = states[9];
        const double r = states[10];
        const double g = states[11];
        const double Ca_i = states[12];
        const double Ca_SR = states[13];
        const double Na_i = states[14];
        const double V = states[15];
        const double K_i = states[16];
        const double E_Na = (R*T*std::log((Na_o/Na_i))/F);
        const double E_K = (R*T*std::log((K_o/K_i))/F);
        const double E_Ks = (R*T*std::log(((K_o + (Na_o*P_kna))/(K_i + (Na_i*P_kna))))/F);
        const double E_Ca = (0.5*R*T*std::log((Ca_o/Ca_i))/F);
        const double alpha_K1 = (0.1/(1.0 + (6.14421235332821e-06*std::exp(((0.06*V) - ((0.06*E_K)))))));
        const double beta_K1 = (((0.36787944117144233*std::exp(((0.1*V) - ((0.1*E_K))))) + (3.0606040200802673*std::exp(((0.0002*V) - ((0.0002*E_K))))))/(1.0 + std::exp(((0.5*E_K) - ((0.5*V))))));
        const double xK1_inf = (alpha_K1/(alpha_K1 + beta_K1));
        const double i_K1 = (0.4303314829119352*g_K1*xK1_inf*std::sqrt(K_o)*(V - ((E_K))));
        const double i_Kr = (0.4303314829119352*Xr1*Xr2*g_Kr*std::sqrt(K_o)*(V - ((E_K))));
        const double xr1_inf = (1.0/(1.0 + std::exp(((-3.7142857142857144) - ((0.14285714285714285*V))))));
        const double alpha_xr1 = (450.0/(1.0 + std::exp(((-4.5) - ((0.1*V))))));
        const double beta_xr1 = (6.0/(1.0 + (13.581324522578193*std::exp((0.08695652173913043*V)))));
        const double tau_xr1 = (alpha_xr1*beta_xr1);
        const double xr2_inf = (1.0/(1.0 + std::exp((3.6666666666666665 + (0.041666666666666664*V)))));
        const double alpha_xr2 = (3.0/(1.0 + std::exp(((-3.0) - ((0.05*V))))));
        const double beta_xr2 = (1.12/(1.0 + std::exp(((-3.0) + (0.05*V)))));
        const double tau_xr2 = (alpha_xr2*beta_xr2);
        const double i_Ks = (g_Ks*(Xs*Xs)*(V - ((E_Ks))));
        const double xs_inf = (1.0/(1.0 + std::exp(((-0.35714285714285715) - ((0.07142857142857142*V))))));
        const double alpha_xs = (1100.0/std::sqrt((1.0 + std::exp(((-1.6666666666666667) - ((0.16666666666666666*V)))))));
        const double beta_xs = (1.0/(1.0 + std::exp(((-3.0) + (0.05*V)))));
        const double tau_xs = (alpha_xs*beta_xs);
        const double i_Na = (g_Na*h*j*(m*m*m)*(V - ((E_Na))));
        const double m_inf = (1.0/((1.0 + (0.0018422115811651339*std::exp((-(0.1107419712070875*V)))))*(1.0 + (0.0018422115811651339*std::exp((-(0.1107419712070875*V)))))));
        const double alpha_m = (1.0/(1.0 + std::exp(((-12.0) - ((0.2*V))))));
        const double beta_m = ((0.1/(1.0 + std::exp((7.0 + (0.2*V))))) + (0.1/(1.0 + std::exp(((-0.25) + (0.005*V))))));
        const double tau_m = (alpha_m*beta_m);
        const double h_inf = (1.0/((1.0 + (15212.593285654404*std::exp((0.13458950201884254*V))))*(1.0 + (15212.593285654404*std::exp((0.13458950201884254*V))))));
        const double alpha_h = ((V < (-40.0)) ? (4.4312679295805147e-07*std::exp((-(0.14705882352941177*V)))) : 0.0);
        const double beta_h = ((V < (-40.0)) ? ((310000.0*std::exp((0.3485*V))) + (2.7*std::exp((0.079*V)))) : (0.77/(0.13 + (0.049758141083938695*std::exp((-(0.0900900900900901*V)))))));
        const double tau_h = (1.0/(alpha_h + beta_h));
        const double j_inf = (1.0/((1.0 + (15212.593285654404*std::exp((0.13458950201884254*V))))*(1.0 + (15212.593285654404*std::exp((0.13458950201884254*V))))));
        const double alpha_j = ((V < (-40.0)) ? ((37.78 + V)*((-(25428.0*std::exp((0.2444*V)))) - ((6.948e-06*std::exp((-(0.04391*V))))))/(1.0 + (50262745825.95399*std::exp((0.311*V))))) : 0.0);
        const double beta_j = ((V < (-40.0)) ? (0.02424*std::exp((-(0.01052*V)))/(1.0 + (0.003960868339904256*std::exp((-(0.1378*V)))))) : (0.6*std::exp((0.057*V))/(1.0 + (0.040762203978366204*std::exp((-(0.1*V)))))));
        const double tau_j = (1.0/(alpha_j + beta_j));
        const double i_b_Na = (g_bna*(V - ((E_Na))));
        const double i_CaL = (4.0*V*d*f*fCa*g_CaL*(F*F)*((-(0.341*Ca_o)) + (Ca_i*std::exp((2.0*F*V/(R*T)))))/(R*T*((-1.0) + std::exp((2.0*F*V/(R*T))))));
        const double d_inf = (1.0/(1.0 + (0.513417119032592*std::exp((-(0.13333333333333333*V))))));
        const double alpha_d = (0.25 + (1.4/(1.0 + std::exp(((-2.6923076923076925) - ((0.07692307692307693*V)))))));
        const double beta_d = (1.4/(1.0 + std::exp((1.0 + (0.2*V)))));
        const double gamma_d = (1.0/(1.0 + std::exp((2.5 - ((0.05*V))))));
        const double tau_d = (gamma_d + (alpha_d*beta_d));
        const double f_inf = (1.0/(1.0 + std::exp((2.857142857142857 + (0.14285714285714285*V)))));
        const double tau_f = (80.0 + (165.0/(1.0 + std::exp((2.5 - ((0.1*V)))))) + (1125.0*std::exp((-(0.004166666666666667*((27.0 + V)*(27.0 + V)))))));
        const double alpha_fCa = (1.0/(1.0 + (8.03402376701711e+27*(((Ca_i*Ca_i)*(Ca_i*Ca_i))*((Ca_i*Ca_i)*(Ca_i*Ca_i))))));
        const double exp_arg_0 = ((-5.0) + (10000.0*Ca_i));
        const double exp_arg_00 = ((exp_arg_0 < 500.0) ? exp_arg_0 : 500.0);
        const double beta_fCa = (0.1/(1.0 + std::exp(exp_arg_00)));
        const double exp_arg_1 = ((-0.9375) + (1250.0*Ca_i));
        const double exp_arg_11 = ((exp_arg_1 < 500.0) ? exp_arg_1 : 500.0);
        const double gama_fCa = (0.2/(1.0 + std::exp(exp_arg_11)));
        const double fCa_inf = (0.15753424657534246 + (0.684931506849315*alpha_fCa) + (0.684931506849315*beta_fCa) + (0.684931506849315*gama_fCa));
        const double tau_fCa = 2.0;
        const double d_fCa = ((fCa_inf - ((fCa)))/tau_fCa);
        const double i_b_Ca = (g_bca*(V - ((E_Ca))));
        const double i_to = (g_to*r*s*(V - ((E_K))));
        const double s_inf = (1.0/(1.0 + std::exp((4.0 + (0.2*V)))));
        const double tau_s = (3.0 + (5.0/(1.0 + std::exp(((-4.0) + (0.2*V))))) + (85.0*std::exp((-(0.003125*((45.0 + V)*(45.0 + V)))))));
        const double r_inf = (1.0/(1.0 + std::exp((3.3333333333333335 - ((0.16666666666666666*V))))));
        const double tau_r = (0.8 + (9.5*std::exp((-(0.0005555555555555556*((40.0 + V)*(40.0 + V)))))));
        const double i_NaK = (K_o*Na_i*P_NaK/((K_mNa + Na_i)*(K_mk + K_o)*(1.0 + (0.0353*std::exp((-(F*V/(R*T))))) + (0.1245*std::exp((-(0.1*F*V/(R*T))))))));
        const double i_NaCa = (K_NaCa*((Ca_o*(Na_i*Na_i*Na_i)*std::exp((F*V*gamma/(R*T)))) - ((Ca_i*alpha*(Na_o*Na_o*Na_o)*std::exp((F*V*((-1.0) + gamma)/(R*T))))))/((1.0 + (K_sat*std::exp((F*V*((-1.0) + gamma)/(R*T)))))*(Ca_o + Km_Ca)*((Km_Nai*Km_Nai*Km_Nai) + (Na_o*Na_o*Na_o))));
        const double i_p_Ca = (Ca_i*g_pCa/(Ca_i + K_pCa));
        const double i_p_K = (g_pK*(V - ((E_K)))/(1.0 + (65.40521574193832*std::exp((-(0.16722408026755853*V))))));
        const double i_rel = (d*g*(c_rel + (a_rel*(Ca_SR*Ca_SR)/((Ca_SR*Ca_SR) + (b_rel*b_rel)))));
        const double i_up = (Vmax_up/(1.0 + ((K_up*K_up)/(Ca_i*Ca_i))));
        const double i_leak = (V_leak*(Ca_SR - ((Ca_i))));
        const double g_inf = ((Ca_i < 0.00035) ? (1.0/(1.0 + (5.439910241481018e+20*((Ca_i*Ca_i*Ca_i)*(Ca_i*Ca_i*Ca_i))))) : (1.0/(1.0 + (1.9720198874049195e+55*((((Ca_i*Ca_i)*(Ca_i*Ca_i))*((Ca_i*Ca_i)*(Ca_i*Ca_i)))*(((Ca_i*Ca_i)*(Ca_i*Ca_i))*((Ca_i*Ca_i)*(Ca_i*Ca_i))))))));
        const double d_g = ((g_inf - ((g)))/tau_g);
        const double Ca_i_bufc = (1.0/(1.0 + (Buf_c*K_buf_c/((Ca_i + K_buf_c)*(Ca_i + K_buf_c)))));
        const double Ca_sr_bufsr = (1.0/(1.0 + (Buf_sr*K_buf_sr/((Ca_SR + K_buf_sr)*(Ca_SR + K_buf_sr)))));
        const double i_Stim = ((((time - ((stim_period*std::floor((time/stim_period))))) >= stim_start) && ((time - ((stim_period*std::floor((time/stim_period))))) <= (stim_duration + stim_start))) ? (-(stim_amplitude)) : 0.0);
        values[0] = ((xr1_inf - ((Xr1)))/tau_xr1);
        values[1] = ((xr2_inf - ((Xr2)))/tau_xr2);
        values[2] = ((xs_inf - ((Xs)))/tau_xs);
        values[3] = ((m_inf - ((m)))/tau_m);
        values[4] = ((h_inf - ((h)))/tau_h);
        values[5] = ((j_inf - ((j)))/tau_j);
        values[6] = ((d_inf - ((d)))/tau_d);
        values[7] = ((f_inf - ((f)))/tau_f);
        values[8] = (((V > (-60.0)) && (fCa_inf > fCa)) ? 0.0 : d_fCa);
        values[9] = ((s_inf - ((s)))/tau_s);
        values[10] = ((r_inf - ((r)))/tau_r);
        values[11] = (((V > (-60.0)) && (g_inf > g)) ? 0.0 : d_g);
        values[12] = (Ca_i_bufc*(i_leak + i_rel - ((i_up)) - ((0.5*Cm*(i_CaL + i_b_Ca + i_p_Ca - ((2.0*i_NaCa)))/(F*V_c)))));
        values[13] = (Ca_sr_bufsr*V_c*(i_up - ((i_leak)) - ((i_rel)))/V_sr);
        values[14] = (Cm*((-(i_Na)) - ((i_b_Na)) - ((3.0*i_NaCa)) - ((3.0*i_NaK)))/(F*V_c));
        values[15] = ((-(i_CaL)) - ((i_K1)) - ((i_Kr)) - ((i_Ks)) - ((i_Na)) - ((i_NaCa)) - ((i_NaK)) - ((i_Stim)) - ((i_b_Ca)) - ((i_b_Na)) - ((i_p_Ca)) - ((i_p_K)) - ((i_to)));
        values[16] = (Cm*((-(i_K1)) - ((i_Kr)) - ((i_Ks)) - ((i_Stim)) - ((i_p_K)) - ((i_to)) + (2.0*i_NaK))/(F*V_c));
    }

    void linearized_eval(const double* states, double time, double* linear, double* rhs,
                         bool only_linear) const
    {
        const double Xr1 = states[0];
        const double Xr2 = states[1];
        const double Xs = states[2];
        const double m = states[3];
        const double h = states[4];
        const double j = states[5];
        const double d = states[6];
        const double f = states[7];
        const double fCa = states[8];
        const double s = states[9];
        const double r = states[10];
        const double g = states[11];
        const double Ca_i = states[12];
        const double Ca_SR = states[13];
        const double Na_i = states[14];
        const double V = states[15];
        const double K_i = states[16];
        const double E_Na = (R*T*std::log((Na_o/Na_i))/F);
        const double E_K = (R*T*std::log((K_o/K_i))/F);
        const double E_Ks = (R*T*std::log(((K_o + (Na_o*P_kna))/(K_i + (Na_i*P_kna))))/F);
        const double E_Ca = (0.5*R*T*std::log((Ca_o/Ca_i))/F);
        const double alpha_K1 = (0.1/(1.0 + (6.14421235332821e-06*std::exp(((0.06*V) - ((0.06*E_K)))))));
        const double beta_K1 = (((0.36787944117144233*std::exp(((0.1*V) - ((0.1*E_K))))) + (3.0606040200802673*std::exp(((0.0002*V) - ((0.0002*E_K))))))/(1.0 + std::exp(((0.5*E_K) - ((0.5*V))))));
        const double xK1_inf = (alpha_K1/(alpha_K1 + beta_K1));
        const double i_K1 = (0.4303314829119352*g_K1*xK1_inf*std::sqrt(K_o)*(V - ((E_K))));
        const double i_Kr = (0.4303314829119352*Xr1*Xr2*g_Kr*std::sqrt(K_o)*(V - ((E_K))));
        const double xr1_inf = (1.0/(1.0 + std::exp(((-3.7142857142857144) - ((0.14285714285714285*V))))));
        const double alpha_xr1 = (450.0/(1.0 + std::exp(((-4.5) - ((0.1*V))))));
        const double beta_xr1 = (6.0/(1.0 + (13.581324522578193*std::exp((0.08695652173913043*V)))));
        const double tau_xr1 = (alpha_xr1*beta_xr1);
        const double xr2_inf = (1.0/(1.0 + std::exp((3.6666666666666665 + (0.041666666666666664*V)))));
        const double alpha_xr2 = (3.0/(1.0 + std::exp(((-3.0) - ((0.05*V))))));
        const double beta_xr2 = (1.12/(1.0 + std::exp(((-3.0) + (0.05*V)))));
        const double tau_xr2 = (alpha_xr2*beta_xr2);
        const double i_Ks = (g_Ks*(Xs*Xs)*(V - ((E_Ks))));
        const double xs_inf = (1.0/(1.0 + std::exp(((-0.35714285714285715) - ((0.07142857142857142*V))))));
        const double alpha_xs = (1100.0/std::sqrt((1.0 + std::exp(((-1.6666666666666667) - ((0.16666666666666666*V)))))));
        const double beta_xs = (1.0/(1.0 + std::exp(((-3.0) + (0.05*V)))));
        const double tau_xs = (alpha_xs*beta_xs);
        const double i_Na = (g_Na*h*j*(m*m*m)*(V - ((E_Na))));
        const double m_inf = (1.0/((1.0 + (0.0018422115811651339*std::exp((-(0.1107419712070875*V)))))*(1.0 + (0.0018422115811651339*std::exp((-(0.1107419712070875*V)))))));
        const double alpha_m = (1.0/(1.0 + std::exp(((-12.0) - ((0.2*V))))));
        const double beta_m = ((0.1/(1.0 + std::exp((7.0 + (0.2*V))))) + (0.1/(1.0 + std::exp(((-0.25) + (0.005*V))))));
        const double tau_m = (alpha_m*beta_m);
        const double h_inf = (1.0/((1.0 + (15212.593285654404*std::exp((0.13458950201884254*V))))*(1.0 + (15212.593285654404*std::exp((0.13458950201884254*V))))));
        const double alpha_h = ((V < (-40.0)) ? (4.4312679295805147e-07*std::exp((-(0.14705882352941177*V)))) : 0.0);
        const double beta_h = ((V < (-40.0)) ? ((310000.0*std::exp((0.3485*V))) + (2.7*std::exp((0.079*V)))) : (0.77/(0.13 + (0.049758141083938695*std::exp((-(0.0900900900900901*V)))))));
        const double tau_h = (1.0/(alpha_h + beta_h));
        const double j_inf = (1.0/((1.0 + (15212.593285654404*std::exp((0.13458950201884254*V))))*(1.0 + (15212.593285654404*std::exp((0.13458950201884254*V))))));
        const double alpha_j = ((V < (-40.0)) ? ((37.78 + V)*((-(25428.0*std::exp((0.2444*V)))) - ((6.948e-06*std::exp((-(0.04391*V))))))/(1.0 + (50262745825.95399*std::exp((0.311*V))))) : 0.0);
        const double beta_j = ((V < (-40.0)) ? (0.02424*std::exp((-(0.01052*V)))/(1.0 + (0.003960868339904256*std::exp((-(0.1378*V)))))) : (0.6*std::exp((0.057*V))/(1.0 + (0.040762203978366204*std::exp((-(0.1*V)))))));
        const double tau_j = (1.0/(alpha_j + beta_j));
        const double i_b_Na = (g_bna*(V - ((E_Na))));
        const double i_CaL = (4.0*V*d*f*fCa*g_CaL*(F*F)*((-(0.341*Ca_o)) + (Ca_i*std::exp((2.0*F*V/(R*T)))))/(R*T*((-1.0) + std::exp((2.0*F*V/(R*T))))));
        const double d_inf = (1.0/(1.0 + (0.513417119032592*std::exp((-(0.13333333333333333*V))))));
        const double alpha_d = (0.25 + (1.4/(1.0 + std::exp(((-2.6923076923076925) - ((0.07692307692307693*V)))))));
        const double beta_d = (1.4/(1.0 + std::exp((1.0 + (0.2*V)))));
        const double gamma_d = (1.0/(1.0 + std::exp((2.5 - ((0.05*V))))));
        const double tau_d = (gamma_d + (alpha_d*beta_d));
        const double f_inf = (1.0/(1.0 + std::exp((2.857142857142857 + (0.14285714285714285*V)))));
        const double tau_f = (80.0 + (165.0/(1.0 + std::exp((2.5 - ((0.1*V)))))) + (1125.0*std::exp((-(0.004166666666666667*((27.0 + V)*(27.0 + V)))))));
        const double alpha_fCa = (1.0/(1.0 + (8.03402376701711e+27*(((Ca_i*Ca_i)*(Ca_i*Ca_i))*((Ca_i*Ca_i)*(Ca_i*Ca_i))))));
        const double exp_arg_0 = ((-5.0) + (10000.0*Ca_i));
        const double exp_arg_00 = ((exp_arg_0 < 500.0) ? exp_arg_0 : 500.0);
        const double beta_fCa = (0.1/(1.0 + std::exp(exp_arg_00)));
        const double exp_arg_1 = ((-0.9375) + (1250.0*Ca_i));
        const double exp_arg_11 = ((exp_arg_1 < 500.0) ? exp_arg_1 : 500.0);
        const double gama_fCa = (0.2/(1.0 + std::exp(exp_arg_11)));
        const double fCa_inf = (0.15753424657534246 + (0.684931506849315*alpha_fCa) + (0.684931506849315*beta_fCa) + (0.684931506849315*gama_fCa));
        const double tau_fCa = 2.0;
        const double d_fCa = ((fCa_inf - ((fCa)))/tau_fCa);
        const double i_b_Ca = (g_bca*(V - ((E_Ca))));
        const double i_to = (g_to*r*s*(V - ((E_K))));
        const double s_inf = (1.0/(1.0 + std::exp((4.0 + (0.2*V)))));
        const double tau_s = (3.0 + (5.0/(1.0 + std::exp(((-4.0) + (0.2*V))))) + (85.0*std::exp((-(0.003125*((45.0 + V)*(45.0 + V)))))));
        const double r_inf = (1.0/(1.0 + std::exp((3.3333333333333335 - ((0.16666666666666666*V))))));
        const double tau_r = (0.8 + (9.5*std::exp((-(0.0005555555555555556*((40.0 + V)*(40.0 + V)))))));
        const double i_NaK = (K_o*Na_i*P_NaK/((K_mNa + Na_i)*(K_mk + K_o)*(1.0 + (0.0353*std::exp((-(F*V/(R*T))))) + (0.1245*std::exp((-(0.1*F*V/(R*T))))))));
        const double i_NaCa = (K_NaCa*((Ca_o*(Na_i*Na_i*Na_i)*std::exp((F*V*gamma/(R*T)))) - ((Ca_i*alpha*(Na_o*Na_o*Na_o)*std::exp((F*V*((-1.0) + gamma)/(R*T))))))/((1.0 + (K_sat*std::exp((F*V*((-1.0) + gamma)/(R*T)))))*(Ca_o + Km_Ca)*((Km_Nai*Km_Nai*Km_Nai) + (Na_o*Na_o*Na_o))));
        const double i_p_Ca = (Ca_i*g_pCa/(Ca_i + K_pCa));
        const double i_p_K = (g_pK*(V - ((E_K)))/(1.0 + (65.40521574193832*std::exp((-(0.16722408026755853*V))))));
        const double i_rel = (d*g*(c_rel + (a_rel*(Ca_SR*Ca_SR)/((Ca_SR*Ca_SR) + (b_rel*b_rel)))));
        const double i_up = (Vmax_up/(1.0 + ((K_up*K_up)/(Ca_i*Ca_i))));
        const double i_leak = (V_leak*(Ca_SR - ((Ca_i))));
        const double g_inf = ((Ca_i < 0.00035) ? (1.0/(1.0 + (5.439910241481018e+20*((Ca_i*Ca_i*Ca_i)*(Ca_i*Ca_i*Ca_i))))) : (1.0/(1.0 + (1.9720198874049195e+55*((((Ca_i*Ca_i)*(Ca_i*Ca_i))*((Ca_i*Ca_i)*(Ca_i*Ca_i)))*(((Ca_i*Ca_i)*(Ca_i*Ca_i))*((Ca_i*Ca_i)*(Ca_i*Ca_i))))))));
        const double d_g = ((g_inf - ((g)))/tau_g);
        const double Ca_i_bufc = (1.0/(1.0 + (Buf_c*K_buf_c/((Ca_i + K_buf_c)*(Ca_i + K_buf_c)))));
        const double Ca_sr_bufsr = (1.0/(1.0 + (Buf_sr*K_buf_sr/((Ca_SR + K_buf_sr)*(Ca_SR + K_buf_sr)))));
        const double i_Stim = ((((time - ((stim_period*std::floor((time/stim_period))))) >= stim_start) && ((time - ((stim_period*std::floor((time/stim_period))))) <= (stim_duration + stim_start))) ? (-(stim_amplitude)) : 0.0);
        rhs[0] = ((xr1_inf - ((Xr1)))/tau_xr1);
        rhs[1] = ((xr2_inf - ((Xr2)))/tau_xr2);
        rhs[2] = ((xs_inf - ((Xs)))/tau_xs);
        rhs[3] = ((m_inf - ((m)))/tau_m);
        rhs[4] = ((h_inf - ((h)))/tau_h);
        rhs[5] = ((j_inf - ((j)))/tau_j);
        rhs[6] = ((d_inf - ((d)))/tau_d);
        rhs[7] = ((f_inf - ((f)))/tau_f);
        rhs[8] = (((V > (-60.0)) && (fCa_inf > fCa)) ? 0.0 : d_fCa);
        rhs[9] = ((s_inf - ((s)))/tau_s);
        rhs[10] = ((r_inf - ((r)))/tau_r);
        rhs[11] = (((V > (-60.0)) && (g_inf > g)) ? 0.0 : d_g);
        rhs[12] = (Ca_i_bufc*(i_leak + i_rel - ((i_up)) - ((0.5*Cm*(i_CaL + i_b_Ca + i_p_Ca - ((2.0*i_NaCa)))/(F*V_c)))));
        rhs[13] = (Ca_sr_bufsr*V_c*(i_up - ((i_leak)) - ((i_rel)))/V_sr);
        rhs[14] = (Cm*((-(i_Na)) - ((i_b_Na)) - ((3.0*i_NaCa)) - ((3.0*i_NaK)))/(F*V_c));
        rhs[15] = ((-(i_CaL)) - ((i_K1)) - ((i_Kr)) - ((i_Ks)) - ((i_Na)) - ((i_NaCa)) - ((i_NaK)) - ((i_Stim)) - ((i_b_Ca)) - ((i_b_Na)) - ((i_p_Ca)) - ((i_p_K)) - ((i_to)));
        rhs[16] = (Cm*((-(i_K1)) - ((i_Kr)) - ((i_Ks)) - ((i_Stim)) - ((i_p_K)) - ((i_to)) + (2.0*i_NaK))/(F*V_c));
        linear[0] = (-(1.0/tau_xr1));
        linear[1] = (-(1.0/tau_xr2));
        linear[2] = (-(1.0/tau_xs));
        linear[3] = (-(1.0/tau_m));
        linear[4] = (-(1.0/tau_h));
        linear[5] = (-(1.0/tau_j));
        linear[6] = (-(1.0/tau_d));
        linear[7] = (-(1.0/tau_f));
        linear[9] = (-(1.0/tau_s));
        linear[10] = (-(1.0/tau_r));
        if (only_linear) return;
        const double dd_fCa_dfCa = (-(1.0/tau_fCa));
        const double dd_g_dg = (-(1.0/tau_g));
        const double dCa_i_bufc_dCa_i = (2.0*Buf_c*K_buf_c/(((1.0 + (Buf_c*K_buf_c/((Ca_i + K_buf_c)*(Ca_i + K_buf_c))))*(1.0 + (Buf_c*K_buf_c/((Ca_i + K_buf_c)*(Ca_i + K_buf_c)))))*((Ca_i + K_buf_c)*(Ca_i + K_buf_c)*(Ca_i + K_buf_c))));
        const double di_CaL_dCa_i = (4.0*V*d*f*fCa*g_CaL*(F*F)*std::exp((2.0*F*V/(R*T)))/(R*T*((-1.0) + std::exp((2.0*F*V/(R*T))))));
        const double di_NaCa_dCa_i = (-(K_NaCa*alpha*(Na_o*Na_o*Na_o)*std::exp((F*V*((-1.0) + gamma)/(R*T)))/((1.0 + (K_sat*std::exp((F*V*((-1.0) + gamma)/(R*T)))))*(Ca_o + Km_Ca)*((Km_Nai*Km_Nai*Km_Nai) + (Na_o*Na_o*Na_o)))));
        const double dE_Ca_dCa_i = (-(0.5*R*T/(Ca_i*F)));
        const double di_b_Ca_dCa_i = (-(dE_Ca_dCa_i*g_bca));
        const double di_leak_dCa_i = (-(V_leak));
        const double di_p_Ca_dCa_i = ((g_pCa/(Ca_i + K_pCa)) - ((Ca_i*g_pCa/((Ca_i + K_pCa)*(Ca_i + K_pCa)))));
        const double di_up_dCa_i = (2.0*Vmax_up*(K_up*K_up)/((Ca_i*Ca_i*Ca_i)*((1.0 + ((K_up*K_up)/(Ca_i*Ca_i)))*(1.0 + ((K_up*K_up)/(Ca_i*Ca_i))))));
        const double dCa_sr_bufsr_dCa_SR = (2.0*Buf_sr*K_buf_sr/(((1.0 + (Buf_sr*K_buf_sr/((Ca_SR + K_buf_sr)*(Ca_SR + K_buf_sr))))*(1.0 + (Buf_sr*K_buf_sr/((Ca_SR + K_buf_sr)*(Ca_SR + K_buf_sr)))))*((Ca_SR + K_buf_sr)*(Ca_SR + K_buf_sr)*(Ca_SR + K_buf_sr))));
        const double di_rel_dCa_SR = (d*g*((-(2.0*a_rel*(Ca_SR*Ca_SR*Ca_SR)/(((Ca_SR*Ca_SR) + (b_rel*b_rel))*((Ca_SR*Ca_SR) + (b_rel*b_rel))))) + (2.0*Ca_SR*a_rel/((Ca_SR*Ca_SR) + (b_rel*b_rel)))));
        const double di_NaCa_dNa_i = (3.0*Ca_o*K_NaCa*(Na_i*Na_i)*std::exp((F*V*gamma/(R*T)))/((1.0 + (K_sat*std::exp((F*V*((-1.0) + gamma)/(R*T)))))*(Ca_o + Km_Ca)*((Km_Nai*Km_Nai*Km_Nai) + (Na_o*Na_o*Na_o))));
        const double di_NaK_dNa_i = ((K_o*P_NaK/((K_mNa + Na_i)*(K_mk + K_o)*(1.0 + (0.0353*std::exp((-(F*V/(R*T))))) + (0.1245*std::exp((-(0.1*F*V/(R*T)))))))) - ((K_o*Na_i*P_NaK/(((K_mNa + Na_i)*(K_mNa + Na_i))*(K_mk + K_o)*(1.0 + (0.0353*std::exp((-(F*V/(R*T))))) + (0.1245*std::exp((-(0.1*F*V/(R*T))))))))));
        const double dE_Na_dNa_i = (-(R*T/(F*Na_i)));
        const double di_Na_dNa_i = (-(dE_Na_dNa_i*g_Na*h*j*(m*m*m)));
        const double di_b_Na_dNa_i = (-(dE_Na_dNa_i*g_bna));
        const double di_CaL_dV = ((4.0*d*f*fCa*g_CaL*(F*F)*((-(0.341*Ca_o)) + (Ca_i*std::exp((2.0*F*V/(R*T)))))/(R*T*((-1.0) + std::exp((2.0*F*V/(R*T)))))) - ((8.0*V*d*f*fCa*g_CaL*(F*F*F)*((-(0.341*Ca_o)) + (Ca_i*std::exp((2.0*F*V/(R*T)))))*std::exp((2.0*F*V/(R*T)))/((R*R)*(T*T)*(((-1.0) + std::exp((2.0*F*V/(R*T))))*((-1.0) + std::exp((2.0*F*V/(R*T)))))))) + (8.0*Ca_i*V*d*f*fCa*g_CaL*(F*F*F)*std::exp((2.0*F*V/(R*T)))/((R*R)*(T*T)*((-1.0) + std::exp((2.0*F*V/(R*T)))))));
        const double dalpha_K1_dV = (-(3.686527411996926e-08*std::exp(((0.06*V) - ((0.06*E_K))))/((1.0 + (6.14421235332821e-06*std::exp(((0.06*V) - ((0.06*E_K))))))*(1.0 + (6.14421235332821e-06*std::exp(((0.06*V) - ((0.06*E_K)))))))));
        const double dbeta_K1_dV = ((((0.0006121208040160535*std::exp(((0.0002*V) - ((0.0002*E_K))))) + (0.036787944117144235*std::exp(((0.1*V) - ((0.1*E_K))))))/(1.0 + std::exp(((0.5*E_K) - ((0.5*V)))))) + (0.5*((0.36787944117144233*std::exp(((0.1*V) - ((0.1*E_K))))) + (3.0606040200802673*std::exp(((0.0002*V) - ((0.0002*E_K))))))*std::exp(((0.5*E_K) - ((0.5*V))))/((1.0 + std::exp(((0.5*E_K) - ((0.5*V)))))*(1.0 + std::exp(((0.5*E_K) - ((0.5*V))))))));
        const double dxK1_inf_dV = ((dalpha_K1_dV*((1.0/(alpha_K1 + beta_K1)) - ((alpha_K1/((alpha_K1 + beta_K1)*(alpha_K1 + beta_K1)))))) - ((alpha_K1*dbeta_K1_dV/((alpha_K1 + beta_K1)*(alpha_K1 + beta_K1)))));
        const double di_K1_dV = ((0.4303314829119352*g_K1*xK1_inf*std::sqrt(K_o)) + (0.4303314829119352*dxK1_inf_dV*g_K1*std::sqrt(K_o)*(V - ((E_K)))));
        const double di_Kr_dV = (0.4303314829119352*Xr1*Xr2*g_Kr*std::sqrt(K_o));
        const double di_Ks_dV = (g_Ks*(Xs*Xs));
        const double di_NaCa_dV = ((K_NaCa*((Ca_o*F*gamma*(Na_i*Na_i*Na_i)*std::exp((F*V*gamma/(R*T)))/(R*T)) - ((Ca_i*F*alpha*(Na_o*Na_o*Na_o)*((-1.0) + gamma)*std::exp((F*V*((-1.0) + gamma)/(R*T)))/(R*T))))/((1.0 + (K_sat*std::exp((F*V*((-1.0) + gamma)/(R*T)))))*(Ca_o + Km_Ca)*((Km_Nai*Km_Nai*Km_Nai) + (Na_o*Na_o*Na_o)))) - ((F*K_NaCa*K_sat*((-1.0) + gamma)*((Ca_o*(Na_i*Na_i*Na_i)*std::exp((F*V*gamma/(R*T)))) - ((Ca_i*alpha*(Na_o*Na_o*Na_o)*std::exp((F*V*((-1.0) + gamma)/(R*T))))))*std::exp((F*V*((-1.0) + gamma)/(R*T)))/(R*T*((1.0 + (K_sat*std::exp((F*V*((-1.0) + gamma)/(R*T)))))*(1.0 + (K_sat*std::exp((F*V*((-1.0) + gamma)/(R*T))))))*(Ca_o + Km_Ca)*((Km_Nai*Km_Nai*Km_Nai) + (Na_o*Na_o*Na_o))))));
        const double di_NaK_dV = (K_o*Na_i*P_NaK*((0.0353*F*std::exp((-(F*V/(R*T))))/(R*T)) + (0.012450000000000001*F*std::exp((-(0.1*F*V/(R*T))))/(R*T)))/((K_mNa + Na_i)*(K_mk + K_o)*((1.0 + (0.0353*std::exp((-(F*V/(R*T))))) + (0.1245*std::exp((-(0.1*F*V/(R*T))))))*(1.0 + (0.0353*std::exp((-(F*V/(R*T))))) + (0.1245*std::exp((-(0.1*F*V/(R*T)))))))));
        const double di_Na_dV = (g_Na*h*j*(m*m*m));
        const double di_p_K_dV = ((g_pK/(1.0 + (65.40521574193832*std::exp((-(0.16722408026755853*V)))))) + (10.937327047146876*g_pK*(V - ((E_K)))*std::exp((-(0.16722408026755853*V)))/((1.0 + (65.40521574193832*std::exp((-(0.16722408026755853*V)))))*(1.0 + (65.40521574193832*std::exp((-(0.16722408026755853*V))))))));
        const double di_to_dV = (g_to*r*s);
        const double dE_K_dK_i = (-(R*T/(F*K_i)));
        const double dalpha_K1_dK_i = (3.686527411996926e-08*dE_K_dK_i*std::exp(((0.06*V) - ((0.06*E_K))))/((1.0 + (6.14421235332821e-06*std::exp(((0.06*V) - ((0.06*E_K))))))*(1.0 + (6.14421235332821e-06*std::exp(((0.06*V) - ((0.06*E_K))))))));
        const double dbeta_K1_dK_i = (dE_K_dK_i*((((-(0.0006121208040160535*std::exp(((0.0002*V) - ((0.0002*E_K)))))) - ((0.036787944117144235*std::exp(((0.1*V) - ((0.1*E_K)))))))/(1.0 + std::exp(((0.5*E_K) - ((0.5*V)))))) - ((0.5*((0.36787944117144233*std::exp(((0.1*V) - ((0.1*E_K))))) + (3.0606040200802673*std::exp(((0.0002*V) - ((0.0002*E_K))))))*std::exp(((0.5*E_K) - ((0.5*V))))/((1.0 + std::exp(((0.5*E_K) - ((0.5*V)))))*(1.0 + std::exp(((0.5*E_K) - ((0.5*V))))))))));
        const double dxK1_inf_dK_i = ((dalpha_K1_dK_i*((1.0/(alpha_K1 + beta_K1)) - ((alpha_K1/((alpha_K1 + beta_K1)*(alpha_K1 + beta_K1)))))) - ((alpha_K1*dbeta_K1_dK_i/((alpha_K1 + beta_K1)*(alpha_K1 + beta_K1)))));
        const double di_K1_dK_i = ((0.4303314829119352*dxK1_inf_dK_i*g_K1*std::sqrt(K_o)*(V - ((E_K)))) - ((0.4303314829119352*dE_K_dK_i*g_K1*xK1_inf*std::sqrt(K_o))));
        const double di_Kr_dK_i = (-(0.4303314829119352*Xr1*Xr2*dE_K_dK_i*g_Kr*std::sqrt(K_o)));
        const double dE_Ks_dK_i = (-(R*T/(F*(K_i + (Na_i*P_kna)))));
        const double di_Ks_dK_i = (-(dE_Ks_dK_i*g_Ks*(Xs*Xs)));
        const double di_p_K_dK_i = (-(dE_K_dK_i*g_pK/(1.0 + (65.40521574193832*std::exp((-(0.16722408026755853*V)))))));
        const double di_to_dK_i = (-(dE_K_dK_i*g_to*r*s));
        linear[8] = (2.0*dd_fCa_dfCa*(((V > (-60.0)) && (fCa < fCa_inf)) ? 0.0 : 1.0));
        linear[11] = (2.0*dd_g_dg*(((V > (-60.0)) && (g < g_inf)) ? 0.0 : 1.0));
        linear[12] = ((Ca_i_bufc*di_leak_dCa_i) + (dCa_i_bufc_dCa_i*(i_leak + i_rel - ((i_up)) - ((0.5*Cm*(i_CaL + i_b_Ca + i_p_Ca - ((2.0*i_NaCa)))/(F*V_c))))) - ((Ca_i_bufc*di_up_dCa_i)) + (Ca_i_bufc*Cm*di_NaCa_dCa_i/(F*V_c)) - ((0.5*Ca_i_bufc*Cm*di_CaL_dCa_i/(F*V_c))) - ((0.5*Ca_i_bufc*Cm*di_b_Ca_dCa_i/(F*V_c))) - ((0.5*Ca_i_bufc*Cm*di_p_Ca_dCa_i/(F*V_c))));
        linear[13] = ((V_c*dCa_sr_bufsr_dCa_SR*(i_up - ((i_leak)) - ((i_rel)))/V_sr) - ((Ca_sr_bufsr*V_c*V_leak/V_sr)) - ((Ca_sr_bufsr*V_c*di_rel_dCa_SR/V_sr)));
        linear[14] = ((-(Cm*di_Na_dNa_i/(F*V_c))) - ((Cm*di_b_Na_dNa_i/(F*V_c))) - ((3.0*Cm*di_NaCa_dNa_i/(F*V_c))) - ((3.0*Cm*di_NaK_dNa_i/(F*V_c))));
        linear[15] = ((-(di_CaL_dV)) - ((di_K1_dV)) - ((di_Kr_dV)) - ((di_Ks_dV)) - ((di_NaCa_dV)) - ((di_NaK_dV)) - ((di_Na_dV)) - ((di_p_K_dV)) - ((di_to_dV)) - ((g_bca)) - ((g_bna)));
        linear[16] = ((-(Cm*di_K1_dK_i/(F*V_c))) - ((Cm*di_Kr_dK_i/(F*V_c))) - ((Cm*di_Ks_dK_i/(F*V_c))) - ((Cm*di_p_K_dK_i/(F*V_c))) - ((Cm*di_to_dK_i/(F*V_c))));
    }

    void get_ic(goss::DoubleVector* values) const
    {
        values->n = _num_states;
        values->data.reset(new double[_num_states]);
        values->data[0] = 0.0;
        values->data[1] = 1.0;
        values->data[2] = 0.0;
        values->data[3] = 0.0;
        values->data[4] = 0.75;
        values->data[5] = 0.75;
        values->data[6] = 0.0;
        values->data[7] = 1.0;
        values->data[8] = 1.0;
        values->data[9] = 1.0;
        values->data[10] = 0.0;
        values->data[11] = 1.0;
        values->data[12] = 0.0002;
        values->data[13] = 0.2;
        values->data[14] = 11.6;
        values->data[15] = -86.2;
        values->data[16] = 138.3;
    }

    std::shared_ptr<ODE> copy() const { return std::make_shared<Tentusscher_2004_mcell>(*this); }

    void eval_monitored(const double* states, double time, double* monitored) const
    {
        throw std::runtime_error("No monitored in the \'Tentusscher_2004_mcell\' model.");
    }

    void set_field_parameters(const double* field_params)
    {
        g_Kr = field_params[0];
        g_Ks = field_params[1];
        g_CaL = field_params[2];
        g_to = field_params[3];
    }

  private:
    double P_kna, g_K1, g_Kr, g_Ks, g_Na, g_bna, g_CaL, g_bca, g_to, K_mNa, K_mk, P_NaK, K_NaCa, K_sat, Km_Ca, Km_Nai, alpha, gamma, K_pCa, g_pCa, g_pK, Buf_c, Buf_sr, Ca_o, K_buf_c, K_buf_sr, K_up, V_leak, V_sr, Vmax_up, a_rel, b_rel, c_rel, tau_g, Na_o, Cm, F, R, T, V_c, stim_amplitude, stim_duration, stim_period, stim_start, K_o;
};
}  // namespace goss

extern "C" __attribute__((visibility("default"))) goss::ParameterizedODE* create_Tentusscher_2004_mcell()
{
    return new goss::Tentusscher_2004_mcell;
}
#endif
