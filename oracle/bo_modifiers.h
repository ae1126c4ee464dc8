/*
 * bo_modifiers.h -- CPU oracle (test infrastructure only): per-modifier
 * current functions of the reference restated with FP32 state (see the rule in
 * bo_physics.h).  One function per supported modifier type; each cites the
 * reference function it follows.
 */
#ifndef BO_MODIFIERS_H
#define BO_MODIFIERS_H
#include "bo_physics.h"

/* hh_biological.cpp:193-232 (Nav1.6) and :238-277 (Nav1.2) */
static double bo_nav_current(OMod* m, OSeg* s, float dt, int is12) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    if (SV < -200.0f) s->V = -200.0f;
    if (SV > 200.0f) s->V = 200.0f;
    V = (float)SV;
    float minf = is12 ? nav12_m_inf(V) : nav16_m_inf(V);
    float mtau = is12 ? nav12_m_tau(V) : nav16_m_tau(V);
    float hinf = is12 ? nav12_h_inf(V) : nav16_h_inf(V);
    float htau = is12 ? nav12_h_tau(V) : nav16_h_tau(V);
    double m_val = minf + (MST(0) - minf) * bo_exp(-dt / mtau);
    double h_val = hinf + (MST(1) - hinf) * bo_exp(-dt / htau);
    if (m_val < 0.0f) m_val = 0.0f;
    if (m_val > 1.0f) m_val = 1.0f;
    if (h_val < 0.0f) h_val = 0.0f;
    if (h_val > 1.0f) h_val = 1.0f;
    m->st[0] = BO_ST(m_val);
    m->st[1] = BO_ST(h_val);
    float open_prob = (float)(m_val * m_val * m_val * h_val);
    double ttx = (MST(5) > 0.0f) ? MST(5) : 0.0f;
    open_prob = (float)(open_prob / (1.0f + ttx / (is12 ? 10.0f : 5.0f)));
    float pkc = 0.0f, pka = 0.0f;   /* no PKC/PKA modifiers in supported networks */
    open_prob *= (1.0f - (is12 ? 0.7f : 0.2f) * (pkc + pka) * 0.5f);
    if (open_prob < 0.0f) open_prob = 0.0f;
    double P_single = bo_ghk_P(is12 ? 20.8f : 20.7f, 1.0f, GHK_CBAR_NA_MM);
    double flux = bo_ghk_mono(V, SIN(0), SOUT(0));
    double I_A = P_single * flux * (MDEN * area) * open_prob;
    double I_Na = I_A * A_TO_PA;
    double vol = bo_seg_volume(s);
    double cpv = FARADAY_CONST * vol / 1000.0;
    s->in[0] = BO_ST(SIN(0) - (I_Na * dt) / cpv);
    s->out[0] = BO_ST(SOUT(0) + (I_Na * dt) / (cpv * EXTRA_VOLUME_RATIO));
    bo_clamp_ions(s->in);
    bo_clamp_ions(s->out);
    return -I_Na;
}

/* hh_biological.cpp:142-187 (Cav1.3) */
static double bo_cav13_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double Vhalf = (MST(3) != 0.0f) ? -fabs(MST(3)) : -35.0f;
    double k = (MST(4) > 0.0f) ? MST(4) : 7.0f;
    double gamma_ps = (MST(2) > 0.0f) ? MST(2) : 25.0f;
    float m_inf = (float)(1.0f / (1.0f + bo_exp(-(V - Vhalf) / (k + 1e-6f))));
    float tau_m = 2.0f;
    m->st[0] = BO_ST(MST(0) + (m_inf - MST(0)) * dt / tau_m);
    float Ca = (float)(SIN(2) * MM_TO_UM);
    float h_inf = 1.0f / (1.0f + bo_exp((V + 52.0f) / 8.0f));
    h_inf *= 1.0f / (1.0f + Ca / 3.0f);
    float tau_h = 100.0f;
    m->st[1] = BO_ST(MST(1) + (h_inf - MST(1)) * dt / tau_h);
    if (MST(0) < 0.0f) m->st[0] = 0.0f;
    if (MST(1) < 0.0f) m->st[1] = 0.0f;
    if (MST(0) > 1.0f) m->st[0] = 1.0f;
    if (MST(1) > 1.0f) m->st[1] = 1.0f;
    float ca_in = s->in[2];
    float ca_out = s->out[2];
    double P_single = bo_ghk_P((float)gamma_ps, 2.0f, GHK_CBAR_CA_MM);
    double open_prob = MST(0) * MST(0) * MST(1);
    double flux = bo_ghk_div(V, ca_in, ca_out);
    double I_A = P_single * flux * (MDEN * area) * open_prob;
    double I_Ca = I_A * A_TO_PA;
    double vol = bo_seg_volume(s);
    double cpm = FARADAY_CONST * vol / 1000.0;
    s->in[2] = BO_ST(SIN(2) - (I_Ca * dt) / (2.0f * cpm));
    s->out[2] = BO_ST(SOUT(2) - (I_Ca * dt) / (2.0f * cpm * EXTRA_VOLUME_RATIO));
    bo_clamp_ions(s->in);
    bo_clamp_ions(s->out);
    return -I_Ca;
}

/* hh_biological.cpp:364-388 (Cav2.1: gates only, current goes to the bouton) */
static double bo_cav21_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float m_inf = cav21_m_inf(V);
    m->st[0] = BO_ST(MST(0) + (m_inf - MST(0)) * dt / 1.0f);
    float Ca = (float)(SIN(2) * MM_TO_UM);
    float h_inf = cav21_h_inf(V, Ca);
    m->st[1] = BO_ST(MST(1) + (h_inf - MST(1)) * dt / 300.0f);
    if (MST(0) < 0.0f) m->st[0] = 0.0f;
    if (MST(1) < 0.0f) m->st[1] = 0.0f;
    if (MST(0) > 1.0f) m->st[0] = 1.0f;
    if (MST(1) > 1.0f) m->st[1] = 1.0f;
    return 0.0f;
}

/* hh_biological.cpp:57-97 (Na/K-ATPase) */
static double bo_nak_pump_current(OMod* m, OSeg* s, float dt) {
    float area = bo_eff_area(m, s);
    float v_norm = nak_pump_vnorm((float)SV, (float)SIN(0), (float)SOUT(1), s->atp, 10.0f, 1.5f);
    double N = MDEN * area;
    float I_pump = (float)(N * v_norm * 75.0f * ELEMENTARY_CHARGE_C * A_TO_PA);
    float volume = (float)bo_seg_volume(s);
    double cpm = FARADAY_CONST * volume / 1000.0;
    float transport = (float)(I_pump * dt / cpm);
    float na_avail = (float)((SIN(0) - 1e-9f) / 3.0f);
    float k_avail = (float)((SOUT(1) - 1e-9f) * EXTRA_VOLUME_RATIO / 2.0f);
    if (na_avail < 0.0f) na_avail = 0.0f;
    if (k_avail < 0.0f) k_avail = 0.0f;
    float max_t = (na_avail < k_avail) ? na_avail : k_avail;
    if (transport > max_t) transport = max_t;
    s->in[0] = BO_ST(SIN(0) - 3.0f * transport);
    s->out[0] = BO_ST(SOUT(0) + 3.0f * transport / EXTRA_VOLUME_RATIO);
    s->in[1] = BO_ST(SIN(1) + 2.0f * transport);
    s->out[1] = BO_ST(SOUT(1) - 2.0f * transport / EXTRA_VOLUME_RATIO);
    bo_clamp_ions(s->in);
    bo_clamp_ions(s->out);
    s->atp -= I_pump * dt * 1e-8f;
    if (s->atp < 0.0f) s->atp = 0.0f;
    return -I_pump;
}

/* shared K-channel ion bookkeeping: intra K -= I*dt/cpv, extra K += .../EVR, clamp extra */
static inline void bo_k_flux(OSeg* s, double I_K, float dt, double cpv) {
    s->in[1] = BO_ST(SIN(1) - (I_K * dt) / cpv);
    s->out[1] = BO_ST(SOUT(1) + (I_K * dt) / (cpv * EXTRA_VOLUME_RATIO));
    bo_clamp_ions(s->out);
}

/* hh_biological.cpp:789-841 (Kv4.2) */
static double bo_kv42_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double Vhalf = (MST(4) != 0.0f) ? -fabs(MST(4)) : -10.0f;
    double k = (MST(5) > 0.0f) ? MST(5) : 13.5f;
    double gamma_ps = (MST(2) > 0.0f) ? MST(2) : 5.0f;
    float m_inf = (float)(1.0f / (1.0f + bo_exp(-(V - Vhalf) / (k + 1e-6f))));
    float tau_m = 1.5f;
    m->st[0] = BO_ST(MST(0) + (m_inf - MST(0)) * dt / tau_m);
    float h_inf = 1.0f / (1.0f + bo_exp((V + 65.0f) / 8.0f));
    float tau_h = kv42_h_tau(V);
    m->st[1] = BO_ST(MST(1) + (h_inf - MST(1)) * dt / tau_h);
    if (MST(0) < 0.0f) m->st[0] = 0.0f;
    if (MST(1) < 0.0f) m->st[1] = 0.0f;
    if (MST(0) > 1.0f) m->st[0] = 1.0f;
    if (MST(1) > 1.0f) m->st[1] = 1.0f;
    float camkii = 0.0f;   /* no CaMKII modifiers in supported networks */
    m->st[3] = BO_ST(MST(3) + (camkii * 0.5f - MST(3)) * dt / 5000.0f);
    if (MST(3) < 0.0f) m->st[3] = 0.0f;
    if (MST(3) > 1.0f) m->st[3] = 1.0f;
    double gamma_eff = gamma_ps * (1.0f - MST(3) * 0.7f);
    float K_i = s->in[1];
    float K_o = s->out[1];
    double P_single = bo_ghk_P((float)gamma_eff, 1.0f, GHK_CBAR_K_MM);
    double open_prob = MST(0) * MST(0) * MST(0) * MST(1);
    double flux = bo_ghk_mono(V, K_i, K_o);
    double I_A = P_single * flux * (MDEN * area) * open_prob;
    double I_K = I_A * A_TO_PA;
    double vol = bo_seg_volume(s);
    double cpv = FARADAY_CONST * vol / 1000.0;
    bo_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:1043-1100 (Kv3.1) */
static double bo_kv31_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    float Vhalf = 10.0f, k = 10.0f, gamma_ps = 27.0f;
    float m_inf = 1.0f / (1.0f + bo_exp(-(V - Vhalf) / (k + 1e-6f)));
    float tau_m = 1.0f;
    m->st[0] = BO_ST(MST(0) + (m_inf - MST(0)) * dt / tau_m);
    if (MST(0) < 0.0f) m->st[0] = 0.0f;
    if (MST(0) > 1.0f) m->st[0] = 1.0f;
    float h_inf = 1.0f / (1.0f + bo_exp((V + 30.0f) / 6.0f));
    float tau_h = 2000.0f;
    m->st[1] = BO_ST(MST(1) + (h_inf - MST(1)) * dt / tau_h);
    if (MST(1) < 0.0f) m->st[1] = 0.0f;
    if (MST(1) > 1.0f) m->st[1] = 1.0f;
    float K_i = s->in[1];
    float K_o = s->out[1];
    double P_single = bo_ghk_P(gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double open_prob = MST(0) * MST(0) * MST(0) * MST(1);
    double tea = (MST(5) > 0.0f) ? MST(5) : 0.0f;
    open_prob /= (1.0f + tea / 0.2f);
    float pkc = 0.0f;
    float k_phos = 5.6e-6f;
    float k_dephos = 1e-4f;
    m->st[2] = BO_ST(MST(2) + (k_phos * pkc * (1.0f - MST(2)) - k_dephos * MST(2)) * dt);
    if (MST(2) < 0.0f) m->st[2] = 0.0f;
    if (MST(2) > 1.0f) m->st[2] = 1.0f;
    open_prob *= (1.0f - 0.27f * MST(2));
    double flux = bo_ghk_mono(V, K_i, K_o);
    double I_A = P_single * flux * (MDEN * area) * open_prob;
    double I_K = I_A * A_TO_PA;
    double vol = bo_seg_volume(s);
    double cpv = FARADAY_CONST * vol / 1000.0;
    bo_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:2070-2105 (Cav3.1) */
static double bo_cav31_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double gamma_ps = (MST(2) > 0.0f) ? MST(2) : 7.5f;
    double m_val = MST(0), h_val = MST(1);
    float m_inf = bo_bz_act(V, -45.0f, 5.5f);
    float h_inf = bo_bz_inact(V, -77.0f, 6.0f);
    float tau_m = cav31_m_tau(V);
    float tau_h = cav31_h_tau(V);
    float sub_dt = dt / 10.0f;
    for (int step = 0; step < 10; step++) {
        m_val += (m_inf - m_val) * sub_dt / tau_m;
        h_val += (h_inf - h_val) * sub_dt / tau_h;
    }
    if (m_val < 0.0f) m_val = 0.0f;
    if (m_val > 1.0f) m_val = 1.0f;
    if (h_val < 0.0f) h_val = 0.0f;
    if (h_val > 1.0f) h_val = 1.0f;
    m->st[0] = BO_ST(m_val);
    m->st[1] = BO_ST(h_val);
    float open_prob = (float)(m_val * m_val * m_val * h_val);
    double ni = (MST(3) > 0.0f) ? MST(3) : 0.0f;
    double mib = (MST(4) > 0.0f) ? MST(4) : 0.0f;
    double tta = (MST(5) > 0.0f) ? MST(5) : 0.0f;
    double z944 = (MST(6) > 0.0f) ? MST(6) : 0.0f;
    open_prob = (float)(open_prob / ((1.0f + ni / 250.0f) * (1.0f + mib / 1.6f)
                                     * (1.0f + tta / 82.0f) * (1.0f + z944 / 100.0f)));
    double P_single = bo_ghk_P((float)gamma_ps, 2.0f, GHK_CBAR_CA_MM);
    double flux = bo_ghk_div(V, SIN(2), SOUT(2));
    double I_A = P_single * flux * (MDEN * area) * open_prob;
    double I_CaT = I_A * A_TO_PA;
    float volume = (float)bo_seg_volume(s);
    float charge_per_mole = (float)(FARADAY_CONST * volume / 1000.0);
    s->in[2] = BO_ST(SIN(2) - (I_CaT * dt) / (2.0f * charge_per_mole));
    return -I_CaT;
}

/* hh_biological.cpp:2574-2613 (PMCA) */
static double bo_pmca_current(OMod* m, OSeg* s, float dt) {
    float area = bo_eff_area(m, s);
    double K_m_Ca = (MST(1) > 0.0f) ? MST(1) : 0.0003f;
    double hill_n = (MST(2) > 0.0f) ? MST(2) : 2.0f;
    float atp = s->atp;
    if (atp < 0.0f) atp = 0.0f;
    float f_ATP = atp / (atp + 0.2f);
    float ca = s->in[2];
    if (ca < 1e-9f) ca = 1e-9f;
    float ca_pow = (float)bo_pow(ca, hill_n);
    float f_Ca = (float)(ca_pow / (ca_pow + bo_pow(K_m_Ca, hill_n)));
    double N = MDEN * area;
    float I_pump = (float)(N * 100.0f * f_Ca * f_ATP * ELEMENTARY_CHARGE_C * 2.0f * A_TO_PA);
    float volume = (float)bo_seg_volume(s);
    double cpv = FARADAY_CONST * volume / 1000.0;
    float transport = (float)(I_pump * dt / (2.0f * cpv));
    float ca_avail = (float)(SIN(2) - 1e-9f);
    if (ca_avail < 0.0f) ca_avail = 0.0f;
    if (transport > ca_avail) transport = ca_avail;
    s->in[2] = BO_ST(SIN(2) - transport);
    s->out[2] = BO_ST(SOUT(2) + transport / EXTRA_VOLUME_RATIO);
    bo_clamp_ions(s->in);
    s->atp -= I_pump * dt * 1e-8f;
    if (s->atp < 0.0f) s->atp = 0.0f;
    return -I_pump;
}

/* hh_biological.cpp:2616-2646 (NCX) */
static double bo_ncx_current(OMod* m, OSeg* s, float dt) {
    float area = bo_eff_area(m, s);
    float Na_i = s->in[0]; if (Na_i < 1e-9f) Na_i = 1e-9f;
    float Na_o = s->out[0]; if (Na_o < 1e-9f) Na_o = 1e-9f;
    float Ca_i = s->in[2]; if (Ca_i < 1e-9f) Ca_i = 1e-9f;
    float Ca_o = s->out[2]; if (Ca_o < 1e-9f) Ca_o = 1e-9f;
    float flux_norm = ncx_flux_norm((float)SV, Na_i, Na_o, Ca_i, Ca_o);
    double N = MDEN * area;
    float I_ncx = (float)(N * 500.0f * flux_norm * ELEMENTARY_CHARGE_C * A_TO_PA);
    float volume = (float)bo_seg_volume(s);
    double cpv = FARADAY_CONST * volume / 1000.0;
    float transport = (float)(I_ncx * dt / cpv);
    if (transport > Ca_i) transport = Ca_i;
    if (transport < -Na_i / 3.0f) transport = -Na_i / 3.0f;
    s->in[2] = BO_ST(SIN(2) - transport);
    s->out[2] = BO_ST(SOUT(2) + transport / EXTRA_VOLUME_RATIO);
    s->in[0] = BO_ST(SIN(0) + 3.0f * transport);
    s->out[0] = BO_ST(SOUT(0) - 3.0f * transport / EXTRA_VOLUME_RATIO);
    bo_clamp_ions(s->in);
    return I_ncx;
}

/* hh_biological.cpp:2648-2702 (KCC2) */
static double bo_kcc2_current(OMod* m, OSeg* s, float dt) {
    float area = bo_eff_area(m, s);
    double Km_K_i = (MST(1) > 0.0f) ? MST(1) : 6.5f;
    double Km_Cl_i = (MST(2) > 0.0f) ? MST(2) : 6.5f;
    float K_i = s->in[1]; if (K_i < 1e-9f) K_i = 1e-9f;
    float Cl_i = s->in[3]; if (Cl_i < 1e-9f) Cl_i = 1e-9f;
    float K_o = s->out[1]; if (K_o < 1e-9f) K_o = 1e-9f;
    float Cl_o = s->out[3]; if (Cl_o < 1e-9f) Cl_o = 1e-9f;
    float f_K = (float)(K_i / (K_i + Km_K_i));
    float f_Cl = (float)(Cl_i / (Cl_i + Km_Cl_i));
    float driving = 1.0f - (K_o * Cl_o) / (K_i * Cl_i);
    if (driving > 1.0f) driving = 1.0f;
    if (driving < -1.0f) driving = -1.0f;
    float flux_mol = (float)(5.0f * NMOL_CM2_S_TO_MOL_UM2_MS * MDEN * area * f_K * f_Cl * driving * dt);
    float dconc = (float)(flux_mol / (bo_seg_volume(s) * UM3_TO_M3));
    if (dconc > 0.0f) {
        float k_avail = K_i - 1e-9f;
        float cl_avail = Cl_i - 1e-9f;
        float min_avail = (k_avail < cl_avail) ? k_avail : cl_avail;
        if (min_avail < 0.0f) min_avail = 0.0f;
        if (dconc > min_avail) dconc = min_avail;
    } else {
        float k_avail = (K_o - 1e-9f) * EXTRA_VOLUME_RATIO;
        float cl_avail = (Cl_o - 1e-9f) * EXTRA_VOLUME_RATIO;
        float min_avail = (k_avail < cl_avail) ? k_avail : cl_avail;
        if (min_avail < 0.0f) min_avail = 0.0f;
        float mag = -dconc;
        if (mag > min_avail) mag = min_avail;
        dconc = -mag;
    }
    s->in[1] = BO_ST(SIN(1) - dconc);
    s->in[3] = BO_ST(SIN(3) - dconc);
    s->out[1] = BO_ST(SOUT(1) + dconc / EXTRA_VOLUME_RATIO);
    s->out[3] = BO_ST(SOUT(3) + dconc / EXTRA_VOLUME_RATIO);
    bo_clamp_ions(s->in);
    return 0.0f;
}

/* hh_biological.cpp:2825-2857 (Ca2+ buffer) */
static double bo_ca_buffer_current(OMod* m, OSeg* s, float dt) {
    double B_total_ref = (MST(0) > 0.0f) ? MST(0) : 0.15f;
    double B_total = B_total_ref * MDEN;
    double K_d = (MST(2) > 0.0f) ? MST(2) : 0.0005f;
    double k_on = (MST(3) > 0.0f) ? MST(3) : 0.1f;
    double k_off = (MST(4) > 0.0f) ? MST(4) : (K_d * k_on);
    double Ca_bound = MST(1);
    if (Ca_bound <= 0.0f && B_total > 0.0f) {
        float Ca_free0 = s->in[2];
        Ca_bound = B_total * Ca_free0 / (Ca_free0 + K_d);
        m->st[1] = BO_ST(Ca_bound);
    }
    float Ca_free = s->in[2];
    if (Ca_free < 1e-9f) Ca_free = 1e-9f;
    float B_free = (float)(B_total - Ca_bound);
    if (B_free < 0.0f) B_free = 0.0f;
    float dCa_bound = (float)((k_on * Ca_free * B_free - k_off * Ca_bound) * dt);
    Ca_bound += dCa_bound;
    if (Ca_bound < 0.0f) Ca_bound = 0.0f;
    if (Ca_bound > B_total) Ca_bound = B_total;
    s->in[2] = BO_ST(SIN(2) - dCa_bound);
    if (SIN(2) < 1e-9f) {
        float deficit = (float)(1e-9f - SIN(2));
        s->in[2] = 1e-9f;
        Ca_bound -= deficit;
        if (Ca_bound < 0.0f) Ca_bound = 0.0f;
    }
    m->st[1] = BO_ST(Ca_bound);
    return 0.0f;
}

/* hh_biological.cpp:2859-2888 (SK) */
static double bo_sk_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double open_prob = MST(0);
    double gamma_ps = (MST(3) > 0.0f) ? MST(3) : 10.0f;
    double tau_open = (MST(4) > 0.0f) ? MST(4) : 5.0f;
    double tau_close = (MST(5) > 0.0f) ? MST(5) : 50.0f;
    float ca = s->in[2];
    float p_inf = sk_p_inf(ca);
    float tau = (float)((p_inf > open_prob) ? tau_open : tau_close);
    open_prob += (p_inf - open_prob) * dt / tau;
    if (open_prob < 0.0f) open_prob = 0.0f;
    if (open_prob > 1.0f) open_prob = 1.0f;
    m->st[0] = BO_ST(open_prob);
    float K_i = s->in[1], K_o = s->out[1];
    double P_single = bo_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double flux = bo_ghk_mono(V, K_i, K_o);
    double I_A = P_single * flux * (MDEN * area) * open_prob;
    float I_K = (float)(I_A * A_TO_PA);
    double vol = bo_seg_volume(s);
    double cpv = FARADAY_CONST * vol / 1000.0f;
    s->in[1] = BO_ST(SIN(1) - (I_K * dt) / cpv);
    s->out[1] = BO_ST(SOUT(1) + (I_K * dt) / (cpv * EXTRA_VOLUME_RATIO));
    bo_clamp_ions(s->out);
    return -I_K;
}

/* hh_biological.cpp:2922-2949 (BK) */
static double bo_bk_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double open_prob = MST(0);
    double gamma_ps = (MST(1) > 0.0f) ? MST(1) : 250.0f;
    double tau_ch = (MST(2) > 0.0f) ? MST(2) : 1.0f;
    float Ca = s->in[2];
    float po_inf = bk_ha_po(V, Ca);
    open_prob += (po_inf - open_prob) * dt / tau_ch;
    if (open_prob < 0.0f) open_prob = 0.0f;
    if (open_prob > 1.0f) open_prob = 1.0f;
    m->st[0] = BO_ST(open_prob);
    float K_i = s->in[1], K_o = s->out[1];
    double P_single = bo_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double flux = bo_ghk_mono(V, K_i, K_o);
    double I_A = P_single * flux * (MDEN * area) * open_prob;
    float I_K = (float)(I_A * A_TO_PA);
    double vol = bo_seg_volume(s);
    double cpv = FARADAY_CONST * vol / 1000.0f;
    s->in[1] = BO_ST(SIN(1) - (I_K * dt) / cpv);
    s->out[1] = BO_ST(SOUT(1) + (I_K * dt) / (cpv * EXTRA_VOLUME_RATIO));
    bo_clamp_ions(s->out);
    return -I_K;
}

/* hh_biological.cpp:2951-2978 (NaP) */
static double bo_nap_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double m_val = MST(0);
    double V_half = (MST(1) != 0.0f) ? MST(1) : -58.7f;
    double k_m = (MST(2) > 0.0f) ? MST(2) : 6.0f;
    double gamma_ps = (MST(3) > 0.0f) ? MST(3) : 20.7f;
    double tau_m = (MST(4) > 0.0f) ? MST(4) : 5.0f;
    double Po = (MST(5) > 0.0f) ? MST(5) : 0.016f;
    float m_inf = bo_bz_act(V, (float)V_half, (float)k_m);
    m_val += (m_inf - m_val) * dt / tau_m;
    if (m_val < 0.0f) m_val = 0.0f;
    if (m_val > 1.0f) m_val = 1.0f;
    m->st[0] = BO_ST(m_val);
    float Na_i = s->in[0], Na_o = s->out[0];
    double P_single = bo_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_NA_MM);
    double flux = bo_ghk_mono(V, Na_i, Na_o);
    double I_A = P_single * flux * (MDEN * area) * (m_val * Po);
    float I_Na = (float)(I_A * A_TO_PA);
    double vol = bo_seg_volume(s);
    double cpv = FARADAY_CONST * vol / 1000.0f;
    s->in[0] = BO_ST(SIN(0) - (I_Na * dt) / cpv);
    bo_clamp_ions(s->in);
    return -I_Na;
}

/* hh_biological.cpp:3018-3038 (Kir2.1) */
static double bo_kir_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double gamma_ps = (MST(3) > 0.0f) ? MST(3) : 30.0f;
    float K_i = s->in[1], K_o = s->out[1];
    float f_open = kir_f_open(V);
    double P_single = bo_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double flux = bo_ghk_mono(V, K_i, K_o);
    double I_A = P_single * flux * (MDEN * area) * f_open;
    double I_K = I_A * A_TO_PA;
    double vol = bo_seg_volume(s);
    double cpv = FARADAY_CONST * vol / 1000.0f;
    bo_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:3063-3084 (K2P leak) */
static double bo_k2p_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double gamma_ps = (MST(0) > 0.0f) ? MST(0) : 100.0f;
    double Po = (MST(1) > 0.0f) ? MST(1) : 0.012f;
    float K_i = s->in[1];
    float K_o = s->out[1];
    double P_single = bo_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double flux = bo_ghk_mono(V, K_i, K_o);
    double I_A = P_single * flux * (MDEN * area) * Po;
    double I_K = I_A * A_TO_PA;
    double vol = bo_seg_volume(s);
    double cpv = FARADAY_CONST * vol / 1000.0;
    bo_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:3158-3202 (Kv7 M-current) */
static double bo_kv7_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double m_val = MST(0);
    double V_half = (MST(1) != 0.0f) ? MST(1) : -38.0f;
    double k_slope = (MST(2) > 0.0f) ? MST(2) : 10.0f;
    double tau_act = (MST(4) > 0.0f) ? MST(4) : 100.0f;
    double tau_deact = (MST(5) > 0.0f) ? MST(5) : 60.0f;
    double pip2 = (MST(6) >= 0.0f) ? MST(6) : 1.0f;
    float m_inf = (float)(1.0f / (1.0f + bo_exp(-(V - V_half) / k_slope)));
    float tau_m = (float)(tau_deact + (tau_act - tau_deact) * m_inf);
    if (tau_m < 1.0f) tau_m = 1.0f;
    m_val += (m_inf - m_val) * dt / tau_m;
    if (m_val < 0.0f) m_val = 0.0f;
    if (m_val > 1.0f) m_val = 1.0f;
    m->st[0] = BO_ST(m_val);
    if (pip2 < 0.01f) return 0.0f;
    float K_i = s->in[1];
    float K_o = s->out[1];
    double P_single = bo_ghk_P(7.0f, 1.0f, GHK_CBAR_K_MM);
    float pkc = 0.0f;
    float pkc_suppress = 1.0f - 0.8f * pkc;
    if (pkc_suppress < 0.0f) pkc_suppress = 0.0f;
    double flux = bo_ghk_mono(V, K_i, K_o);
    double I_A = P_single * flux * (MDEN * area) * (m_val * pip2 * pkc_suppress);
    double I_K = I_A * A_TO_PA;
    double vol = bo_seg_volume(s);
    double cpv = FARADAY_CONST * vol / 1000.0;
    bo_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:2763-2797 (Kv1.1 delayed rectifier) */
static double bo_kvdr_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double m_val = MST(0);
    double V_half = (MST(1) != 0.0f) ? MST(1) : -30.0f;
    double k = (MST(2) > 0.0f) ? MST(2) : 6.0f;
    double tau = (MST(4) > 0.0f) ? MST(4) : kv_dr_m_tau(V, (float)V_half);
    float m_inf = (float)(1.0f / (1.0f + bo_exp(-(V - V_half) / (k + 1e-6f))));
    m_val += (m_inf - m_val) * dt / (tau + 1e-6f);
    if (m_val < 0.0f) m_val = 0.0f;
    if (m_val > 1.0f) m_val = 1.0f;
    m->st[0] = BO_ST(m_val);
    float K_i = s->in[1];
    float K_o = s->out[1];
    double P_single = bo_ghk_P(12.0f, 1.0f, GHK_CBAR_K_MM);
    double flux = bo_ghk_mono(V, K_i, K_o);
    double I_A = P_single * flux * (MDEN * area) * m_val;
    double I_K = I_A * A_TO_PA;
    double vol = bo_seg_volume(s);
    float charge_per_mole_vol = (float)(FARADAY_CONST * vol / 1000.0);
    s->in[1] = BO_ST(SIN(1) - (I_K * dt) / charge_per_mole_vol);
    s->out[1] = BO_ST(SOUT(1) + (I_K * dt) / (charge_per_mole_vol * EXTRA_VOLUME_RATIO));
    bo_clamp_ions(s->in);
    bo_clamp_ions(s->out);
    return -I_K;
}

/* modifier_helpers.h:1442-1484 (hcn_generic_current) via hh_biological.cpp:3598 (HCN1) */
static double bo_hcn1_current(OMod* m, OSeg* s, float dt) {
    double V = SV;
    float area = bo_eff_area(m, s);
    float V_half = (MST(1) != 0) ? (float)MST(1) : -69.0f;
    float k = (MST(2) > 0) ? (float)MST(2) : 6.0f;
    float gamma_ps = (MST(3) > 0) ? (float)MST(3) : 0.84f;
    float tau_open = (MST(4) > 0) ? (float)MST(4) : 84.0f;
    float tau_close = (MST(5) > 0) ? (float)MST(5) : 300.0f;
    float camp = 0.1f;  /* segment_camp_um: no cAMP/PKA modifier -> basal 0.1 uM (units.h:324) */
    float Ve = V_half + 15.0f * camp / (camp + 0.5f);
    float mv = m->st[0];
    float mi = 1.0f / (1.0f + bo_exp(((float)V - Ve) / k));
    float tau_eff = (V < Ve) ? (float)(tau_open * bo_exp((V - Ve) / 15.0f)) : tau_close;
    mv += (mi - mv) * dt / tau_eff;
    if (mv < 0.0f) mv = 0.0f;
    if (mv > 1.0f) mv = 1.0f;
    m->st[0] = mv;
    double P_Na, P_K, P_Ca;
    bo_partial_P(gamma_ps, 0.2f, 0.8f, 0.0f, &P_Na, &P_K, &P_Ca);
    double N = MDEN * area;
    double flux_Na = bo_ghk_mono(V, SIN(0), SOUT(0));
    double flux_K = bo_ghk_mono(V, SIN(1), SOUT(1));
    double In = P_Na * flux_Na * N * mv * A_TO_PA;
    double Ik = P_K * flux_K * N * mv * A_TO_PA;
    double vol = bo_seg_volume(s);
    double cpm = FARADAY_CONST * vol / 1000.0;
    s->in[0] = BO_ST(SIN(0) - (In * dt) / cpm);
    s->in[1] = BO_ST(SIN(1) - (Ik * dt) / cpm);
    s->out[0] = BO_ST(SOUT(0) + (In * dt) / (cpm * EXTRA_VOLUME_RATIO));
    s->out[1] = BO_ST(SOUT(1) + (Ik * dt) / (cpm * EXTRA_VOLUME_RATIO));
    bo_clamp_ions(s->in);
    bo_clamp_ions(s->out);
    return -(In + Ik);
}

/* hh_biological.cpp:3609-3641 (NALCN; the returned sign follows the reference) */
static double bo_nalcn_current(OMod* m, OSeg* s, float dt) {
    float V = s->V;
    float area = bo_eff_area(m, s);
    double gamma_ps = (MST(0) > 0.0f) ? MST(0) : 27.0f;
    double P_Na, P_K, P_Ca;
    bo_nalcn_partial_P((float)gamma_ps, &P_Na, &P_K, &P_Ca);
    double N = MDEN * area;
    float Ina = (float)(P_Na * bo_ghk_mono(V, SIN(0), SOUT(0)) * N * A_TO_PA);
    float Ik = (float)(P_K * bo_ghk_mono(V, SIN(1), SOUT(1)) * N * A_TO_PA);
    float Ica = (float)(P_Ca * bo_ghk_div(V, SIN(2), SOUT(2)) * N * A_TO_PA);
    double vol = bo_seg_volume(s);
    double cpm = FARADAY_CONST * vol / 1000.0;
    s->in[0] = BO_ST(SIN(0) - (Ina * dt) / cpm);
    s->in[1] = BO_ST(SIN(1) - (Ik * dt) / cpm);
    s->in[2] = BO_ST(SIN(2) - (Ica * dt) / (2.0f * cpm));
    s->out[0] = BO_ST(SOUT(0) + (Ina * dt) / (cpm * EXTRA_VOLUME_RATIO));
    s->out[1] = BO_ST(SOUT(1) + (Ik * dt) / (cpm * EXTRA_VOLUME_RATIO));
    s->out[2] = BO_ST(SOUT(2) + (Ica * dt) / (2.0f * cpm * EXTRA_VOLUME_RATIO));
    bo_clamp_ions(s->in);
    bo_clamp_ions(s->out);
    return -(Ina - Ik + Ica);
}

/* modifier_helpers.h:1213-1278 (ionotropic_ghk_current) */
static double bo_ionotropic(OMod* m, OSeg* s, float dt, float gamma_ps, float EC50, float tau_rise,
                            float tau_decay, int nt_index, float P_Na_ratio, float P_K_ratio,
                            float P_Ca_ratio, int is_anion, float tau_desens, float K_desens,
                            float mod_scale) {
    float area = bo_eff_area(m, s);
    double V = SV;
    double vol = bo_seg_volume(s);
    double cpm = FARADAY_CONST * vol / 1000.0;
    float p_gamma_ps = (m->active_vars > 0 && m->active_vars < 8 && MST(m->active_vars) > 0.0f)
                       ? (float)MST(m->active_vars) : gamma_ps;
    float nt = s->nt[nt_index];
    float r_inf = nt / (nt + EC50);
    float r = m->st[0];
    float tau = (r_inf > r) ? tau_rise : tau_decay;
    m->st[0] = BO_ST(MST(0) + (r_inf - r) * dt / tau);
    if (MST(0) < 0.0f) m->st[0] = 0.0f;
    if (MST(0) > 1.0f) m->st[0] = 1.0f;
    float open_prob = m->st[0];
    if (tau_desens > 0.0f) {
        float kd = (K_desens > 0.0f) ? K_desens : EC50;
        float d = m->st[1];
        float d_inf = nt / (nt + kd);
        d += (d_inf - d) * dt / tau_desens;
        if (d < 0.0f) d = 0.0f;
        if (d > 1.0f) d = 1.0f;
        m->st[1] = d;
        open_prob *= (1.0f - d);
    }
    double N = MDEN * area;
    double I_total = 0.0;
    if (is_anion) {
        double P_Cl = bo_ghk_P(p_gamma_ps, 1.0f, GHK_CBAR_CL_MM);
        double flux_Cl = bo_ghk_anion(V, SIN(3), SOUT(3));
        double I_Cl = P_Cl * flux_Cl * N * open_prob * mod_scale * A_TO_PA;
        s->in[3] = BO_ST(SIN(3) + (I_Cl * dt) / cpm);
        bo_clamp_ions(s->in);
        return -I_Cl;
    }
    double P_Na, P_K, P_Ca;
    bo_partial_P(p_gamma_ps, P_Na_ratio, P_K_ratio, P_Ca_ratio, &P_Na, &P_K, &P_Ca);
    double I_Na = P_Na * bo_ghk_mono(V, SIN(0), SOUT(0)) * N * open_prob * mod_scale * A_TO_PA;
    double I_K = P_K * bo_ghk_mono(V, SIN(1), SOUT(1)) * N * open_prob * mod_scale * A_TO_PA;
    I_total = I_Na + I_K;
    s->in[0] = BO_ST(SIN(0) - (I_Na * dt) / cpm);
    s->in[1] = BO_ST(SIN(1) - (I_K * dt) / cpm);
    if (P_Ca_ratio > 0.0f) {
        double I_Ca = P_Ca * bo_ghk_div(V, SIN(2), SOUT(2)) * N * open_prob * mod_scale * A_TO_PA;
        I_total += I_Ca;
        s->in[2] = BO_ST(SIN(2) - (I_Ca * dt) / (2.0f * cpm));
    }
    bo_clamp_ions(s->in);
    return -I_total;
}

/* modifier_helpers.h:1281-1290 */
static double bo_nmda_cdi_coagonist(OMod* m, OSeg* s, float dt) {
    double Ca_uM = SIN(2) * MM_TO_UM;
    double cdi_inf = 1.0 - 0.8f * Ca_uM / (Ca_uM + 1.0f);
    float tau = (cdi_inf < MST(2)) ? 500.0f : 9000.0f;
    m->st[2] = BO_ST(MST(2) + (cdi_inf - MST(2)) * dt / tau);
    if (MST(2) < 0.0f) m->st[2] = 0.0f;
    if (MST(2) > 1.0f) m->st[2] = 1.0f;
    float coagonist = 10.0f / (10.0f + 1.0f);
    return MST(2) * coagonist;
}

/* receptors_biological.cpp:42-82 (AMPA, NMDA, GABA-A, glycine) */
static double bo_ampa_current(OMod* m, OSeg* s, float dt, float scale) {
    return bo_ionotropic(m, s, dt, 8.0f, 0.5f, 0.5f, 3.0f, 0, 0.5f, 0.5f, 0.0f, 0, 3.0f, 0.0f, scale);
}
static double bo_nmda_current(OMod* m, OSeg* s, float dt, float scale) {
    double I = bo_ionotropic(m, s, dt, 50.0f, 1.0f, 5.0f, 50.0f, 0, 0.08f, 0.08f, 0.84f, 0, 0.0f, 0.0f, scale);
    float mg_block = (float)(1.0f / (1.0f + (1.0f / 3.57f) * bo_exp(-0.062f * SV)));
    double c = bo_nmda_cdi_coagonist(m, s, dt);
    return I * mg_block * c;
}
static double bo_gabaa_current(OMod* m, OSeg* s, float dt, float scale) {
    return bo_ionotropic(m, s, dt, 28.0f, 1.0f, 1.0f, 5.0f, 1, 0.0f, 0.0f, 0.0f, 1, 2000.0f, 0.0f, scale);
}
static double bo_glycine_current(OMod* m, OSeg* s, float dt, float scale) {
    return bo_ionotropic(m, s, dt, 60.0f, 0.5f, 0.3f, 5.0f, 7, 0.0f, 0.0f, 0.0f, 1, 2000.0f, 0.0f, scale);
}

/* kernel_dispatch.h:337-570 restricted to the supported types; 0 for unknown types
 * (the oracle's loader rejects them, so this branch is never taken). */
/* hh_biological.cpp:1746-1767 (eCB synthesis, 2-AG from Ca2+ and DAG).  segment_dag
 * (modifier_helpers.h:1496-1500) reads a PLC/IP3/DAG modifier, which no supported
 * network carries, so DAG is 0 here. */
static double bo_ecb_synthesis_current(OMod* m, OSeg* s, float dt) {
    float Ca = (float)((double)s->in[2] * (double)MM_TO_UM);
    double synth_rate = (m->st[1] > 0.0f) ? (double)m->st[1] : (double)0.01f;
    double degrad_rate = (m->st[2] > 0.0f) ? (double)m->st[2] : (double)0.005f;
    float dag = 0.0f;
    dt = (float)((double)dt * (double)m->density);
    float Ca_n = Ca * Ca;
    float synth = (float)(synth_rate * (double)Ca_n / (double)(Ca_n + 0.25f + 1e-9f) * (double)(1.0f + dag));
    m->st[0] = BO_ST((double)m->st[0] + ((double)synth - (double)m->st[0] * degrad_rate) * (double)dt);
    if (m->st[0] < 0.0f) m->st[0] = 0.0f;
    if (m->st[0] > 10.0f) m->st[0] = 10.0f;
    return 0.0;
}

/* hh_biological.cpp:725-733 (GLAST, glial glutamate transporter) through
 * glial_nt_uptake_current (modifier_helpers.h:418-454): 3 Na+ in, 1 K+ out, net +2,
 * glutamate taken from the segment's own neurotransmitter pool. */
static double bo_glast_current(OMod* m, OSeg* s, float dt) {
    const float k_m_rel = 10.0f, imax = 2.0f, rel_per_mm = 667.0f;
    const int na_in = 3, k_out = 1, net_charge = 2;
    float area = (m->st[7] > 0.0f) ? (float)m->st[7] : bo_seg_area(s);
    float NT = s->nt[0];
    if (NT < 0.0f) NT = 0.0f;
    float frac = NT / (NT + k_m_rel);
    float I = (float)((double)imax * (double)m->density * (double)area * (double)(1e-8f * 1e6f) * (double)frac);
    float volume = (float)bo_seg_volume(s);
    double cpm = FARADAY_CONST * (double)volume / 1000.0;
    float transport = (float)((double)(I * dt) / ((double)(float)net_charge * cpm));
    float nt_avail = NT / rel_per_mm;
    float na_avail = (float)((double)s->out[0] * (double)EXTRA_VOLUME_RATIO / (double)(float)na_in);
    if (transport > nt_avail) transport = nt_avail;
    if (transport > na_avail) transport = na_avail;
    if (k_out && (double)transport > (double)s->in[1]) transport = (float)s->in[1];
    if (transport < 0.0f) transport = 0.0f;
    s->in[0] = BO_ST((double)s->in[0] + (double)((float)na_in * transport));
    s->out[0] = BO_ST((double)s->out[0] - (double)((float)na_in * transport / EXTRA_VOLUME_RATIO));
    s->in[1] = BO_ST((double)s->in[1] - (double)((float)k_out * transport));
    s->out[1] = BO_ST((double)s->out[1] + (double)((float)k_out * transport / EXTRA_VOLUME_RATIO));
    s->nt[0] -= transport * rel_per_mm;
    if (s->nt[0] < 0.0f) s->nt[0] = 0.0f;
    bo_clamp_ions(s->in);
    bo_clamp_ions(s->out);
    return I;
}

/* hh_biological.cpp:3266-3308 (connexin-36) and 3310-3350 (connexin-43), the same
 * steps: connexon turnover, phosphorylation toward CaMKII and cAMP drives, P_open from
 * phosphorylation and pH.  No current; gap junctions read state[0] and state[4]. */
static double bo_connexin_current(OMod* m, OSeg* s, float dt) {
    double synth_rate = (m->st[2] > 0.0f) ? (double)m->st[2] : (double)0.001f;
    double degrad_rate = (m->st[3] > 0.0f) ? (double)m->st[3] : (double)0.0005f;
    double pH = (m->st[5] > 4.0f) ? (double)m->st[5] : (double)7.2f;
    m->st[0] = BO_ST((double)m->st[0] + (synth_rate - degrad_rate * (double)m->st[0]) * (double)dt / (double)3600000.0f);
    if (m->st[0] < 0.0f) m->st[0] = 0.0f;
    if (m->st[0] > 1.0f) m->st[0] = 1.0f;
    float camkii_act = 0.0f;
    for (uint8_t j = 0; j < s->nmod; j++)
        if (s->mods[j].type == 82) camkii_act = (float)s->mods[j].st[0];
    double pka_drive = (double)m->st[6];
    float p_target = (float)((double)(camkii_act * 0.6f) + pka_drive * (double)0.3f);
    m->st[1] = BO_ST((double)m->st[1] + ((double)p_target - (double)m->st[1]) * (double)dt / (double)5000.0f);
    if (m->st[1] < 0.0f) m->st[1] = 0.0f;
    if (m->st[1] > 1.0f) m->st[1] = 1.0f;
    float pH_factor = (pH < 6.8f) ? (float)((pH - (double)6.0f) / (double)0.8f) : 1.0f;
    if (pH_factor < 0.0f) pH_factor = 0.0f;
    double camkii_P_open = 1.0f - (double)m->st[1] * (double)0.5f;
    double pka_P_open = 1.0f + (double)m->st[1] * (double)0.3f;
    m->st[4] = BO_ST((camkii_P_open * (double)0.5f + pka_P_open * (double)0.5f) * (double)pH_factor);
    if (m->st[4] < 0.05f) m->st[4] = 0.05f;
    if (m->st[4] > 2.0f) m->st[4] = 2.0f;
    return 0.0;
}

static double bo_dispatch(uint8_t type, OMod* m, OSeg* s, float dt) {
    switch (type) {
        case 1: return bo_cav13_current(m, s, dt);
        case 4: return 0.0f;
        case 7: return bo_nak_pump_current(m, s, dt);
        case 8: return bo_ampa_current(m, s, dt, 1.0f);
        case 9: return bo_nmda_current(m, s, dt, 1.0f);
        case 11: return bo_gabaa_current(m, s, dt, 1.0f);
        case 12: return bo_glycine_current(m, s, dt, 1.0f);
        case 85: return bo_kv42_current(m, s, dt);
        case 98: return bo_pmca_current(m, s, dt);
        case 99: return bo_ncx_current(m, s, dt);
        case 100: return bo_kcc2_current(m, s, dt);
        case 102: return bo_ca_buffer_current(m, s, dt);
        case 103: return bo_sk_current(m, s, dt);
        case 104: return bo_bk_current(m, s, dt);
        case 105: return bo_nap_current(m, s, dt);
        case 106: return bo_kir_current(m, s, dt);
        case 107: return bo_k2p_current(m, s, dt);
        case 112: return bo_kv7_current(m, s, dt);
        case 123: return bo_kvdr_current(m, s, dt);
        case 129: return bo_hcn1_current(m, s, dt);
        case 133: return bo_nalcn_current(m, s, dt);
        case 140: return bo_cav21_current(m, s, dt);
        case 141: return bo_nav_current(m, s, dt, 0);
        case 142: return bo_nav_current(m, s, dt, 1);
        case 150: return bo_kv31_current(m, s, dt);
        case 200: return bo_cav31_current(m, s, dt);
        case 86: return bo_ecb_synthesis_current(m, s, dt);
        case 147: return bo_glast_current(m, s, dt);
        case 114: case 198: return bo_connexin_current(m, s, dt);
        default: return 0.0f;
    }
}

static int bo_type_supported(uint8_t t) {
    switch (t) {
        case 1: case 4: case 7: case 8: case 9: case 11: case 12: case 85: case 98: case 99:
        case 100: case 102: case 103: case 104: case 105: case 106: case 107: case 112:
        case 123: case 129: case 133: case 140: case 141: case 142: case 150: case 200: case 86: case 147: case 114: case 198:
            return 1;
        default: return 0;
    }
}

/* kernel_dispatch.h:283-309 */
static int bo_is_ionotropic(uint8_t type) {
    return (type <= 2) || (type >= 8 && type <= 16) || type == 97 || type == 134 || type == 194;
}
static int bo_is_myelin_blocked(uint8_t type) {
    return bo_is_ionotropic(type) || type == 107 || type == 151 || type == 152 || type == 153 ||
           type == 133 || type == 85 || type == 202 || type == 203 || type == 204 || type == 150 ||
           type == 205 || type == 206 || type == 207 || type == 154 || type == 156 || type == 157 ||
           type == 159 || type == 112 || type == 123 || type == 121 || type == 105 || type == 195 ||
           type == 84 || type == 96 || type == 191 || type == 200 || type == 201 || type == 140 ||
           type == 158 || type == 168 || type == 129 || type == 130 || type == 131 || type == 132 ||
           type == 103 || type == 209 || type == 104;
}

#endif
