// receptor.cuh -- the ionotropic receptor model shared by the synapse kernel and the
// adjoint's replay: constants of AMPA, NMDA, GABA-A and glycine, the device table of
// their permeabilities, and the current (modifier_helpers.h:1213-1279).  Each
// translation unit that includes it holds its own table and initialises it with
// k_init_receptors once per device.
#pragma once
#include "physics.cuh"

namespace bnc {

namespace {

// Ionotropic receptor constants (receptors_biological.cpp:42-82 through
// modifier_helpers.h:1213-1279): AMPA, NMDA, GABA-A, glycine.  The permeabilities at
// the default conductance are computed once on the device with the same helpers the
// models use, so they equal the constants a per-type specialisation folds.
struct RecKind {
    float gamma_ps, EC50, tau_rise, tau_decay, P_Na_ratio, P_K_ratio, P_Ca_ratio, tau_desens, K_desens;
    int is_anion, nmda;
    double P_Na, P_K, P_Ca, P_Cl;
};

__device__ RecKind gRec[4];

__global__ void k_init_receptors() {
    const float c[4][9] = {{8.0f, 0.5f, 0.5f, 3.0f, 0.5f, 0.5f, 0.0f, 3.0f, 0.0f},
                           {50.0f, 1.0f, 5.0f, 50.0f, 0.08f, 0.08f, 0.84f, 0.0f, 0.0f},
                           {28.0f, 1.0f, 1.0f, 5.0f, 0.0f, 0.0f, 0.0f, 2000.0f, 0.0f},
                           {60.0f, 0.5f, 0.3f, 5.0f, 0.0f, 0.0f, 0.0f, 2000.0f, 0.0f}};
    for (int k = 0; k < 4; k++) {
        RecKind& r = gRec[k];
        r.gamma_ps = c[k][0]; r.EC50 = c[k][1]; r.tau_rise = c[k][2]; r.tau_decay = c[k][3];
        r.P_Na_ratio = c[k][4]; r.P_K_ratio = c[k][5]; r.P_Ca_ratio = c[k][6];
        r.tau_desens = c[k][7]; r.K_desens = c[k][8];
        r.is_anion = k >= 2;
        r.nmda = k == 1;
        dp_partial_P(r.gamma_ps, r.P_Na_ratio, r.P_K_ratio, r.P_Ca_ratio, &r.P_Na, &r.P_K, &r.P_Ca);
        r.P_Cl = dp_ghk_P(r.gamma_ps, 1.0f, GHK_CBAR_CL_MM);
    }
}

__device__ __forceinline__ int receptor_kind(uint8_t type) {
    return type == 8 ? 0 : (type == 9 ? 1 : (type == 11 ? 2 : 3));
}

// modifier_helpers.h:1213-1279 (ionotropic_ghk_current) with the receptor's constants
// as data; NMDA adds the Mg2+ block and CDI/co-agonist factor (receptors_biological.cpp:48-70).
__device__ __forceinline__ double receptor_current(const RecKind& K, DMod& m, DSeg& s, float dt, float nt,
                                                  float mod_scale) {
    float area = m.area;
    double V = ((double)s.V);
    double vol = s.vol;
    double cpm = FARADAY_CONST * vol / 1000.0;
    const bool custom = m.av != 0;   // conductance override through active_vars
    float p_gamma_ps = K.gamma_ps;
    if (custom) {
        float stav = (m.av == 7) ? m.area : (m.av == 1 ? m.st[1] : (m.av == 2 ? m.st[2] : 0.0f));
        p_gamma_ps = (m.av > 0 && m.av < 8 && ((double)stav) > 0.0f) ? (float)((double)stav) : K.gamma_ps;
    }
    float r_inf = nt / (nt + K.EC50);
    float r = m.st[0];
    float tau = (r_inf > r) ? K.tau_rise : K.tau_decay;
    m.st[0] = (float)(((double)m.st[0]) + (r_inf - r) * dt / tau);
    if (((double)m.st[0]) < 0.0f) m.st[0] = 0.0f;
    if (((double)m.st[0]) > 1.0f) m.st[0] = 1.0f;
    float open_prob = m.st[0];
    if (K.tau_desens > 0.0f) {
        float kd = (K.K_desens > 0.0f) ? K.K_desens : K.EC50;
        float dd = m.st[1];
        float d_inf = nt / (nt + kd);
        dd += (d_inf - dd) * dt / K.tau_desens;
        if (dd < 0.0f) dd = 0.0f;
        if (dd > 1.0f) dd = 1.0f;
        m.st[1] = dd;
        open_prob *= (1.0f - dd);
    }
    double N = ((double)m.den) * area;
    double I;
    if (K.is_anion) {
        double P_Cl = custom ? dp_ghk_P(p_gamma_ps, 1.0f, GHK_CBAR_CL_MM) : K.P_Cl;
        double flux_Cl = dp_ghk_anion_c(s.gc, V, ((double)s.in[3]), ((double)s.out[3]));
        double I_Cl = P_Cl * flux_Cl * N * open_prob * mod_scale * A_TO_PA;
        s.in[3] = (float)(((double)s.in[3]) + (I_Cl * dt) / cpm);
        dp_clamp_ions(s.in);
        I = -I_Cl;
    } else {
        double P_Na = K.P_Na, P_K = K.P_K, P_Ca = K.P_Ca;
        if (custom) dp_partial_P(p_gamma_ps, K.P_Na_ratio, K.P_K_ratio, K.P_Ca_ratio, &P_Na, &P_K, &P_Ca);
        double I_Na = P_Na * dp_ghk_mono_c(s.gc, V, ((double)s.in[0]), ((double)s.out[0])) * N * open_prob * mod_scale * A_TO_PA;
        double I_K = P_K * dp_ghk_mono_c(s.gc, V, ((double)s.in[1]), ((double)s.out[1])) * N * open_prob * mod_scale * A_TO_PA;
        double I_total = I_Na + I_K;
        s.in[0] = (float)(((double)s.in[0]) - (I_Na * dt) / cpm);
        s.in[1] = (float)(((double)s.in[1]) - (I_K * dt) / cpm);
        if (K.P_Ca_ratio > 0.0f) {
            double I_Ca = P_Ca * dp_ghk_div_c(s.gc, V, ((double)s.in[2]), ((double)s.out[2])) * N * open_prob * mod_scale * A_TO_PA;
            I_total += I_Ca;
            s.in[2] = (float)(((double)s.in[2]) - (I_Ca * dt) / (2.0f * cpm));
        }
        dp_clamp_ions(s.in);
        I = -I_total;
    }
    if (K.nmda) {
        float mg_block = (float)(1.0f / (1.0f + (1.0f / 3.57f) * dm_exp(-0.062f * ((double)s.V))));
        double c = dp_nmda_cdi_coagonist(m, s, dt);
        I = I * mg_block * c;
    }
    return I;
}

}  // namespace

}  // namespace bnc
