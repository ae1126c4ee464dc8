// physics.cuh -- device physics of the reference's per-tick loop: channel, pump,
// receptor currents and their ion bookkeeping, GHK/Nernst helpers, gating
// functions.  Each function restates the reference function cited beside it.
//
// Precision rule: state the reference keeps in double (V_m, ion concentrations,
// modifier density/state) is stored as float and promoted to double exactly where
// the reference reads a double, so every expression keeps the reference's operand
// types; each store rounds to float.  Locals keep the reference's types.  exp/log/
// pow come from device_math.cuh; the translation units are built with
// --fmad=false so no multiply-add is fused behind the source's back.
#pragma once
#include <cstdint>
#include "device_math.cuh"

namespace bnc {

// GHK factors that depend on V_m only.  V_m is constant while a segment's modifiers
// (step 1) or a postsynaptic segment's receptors (step 3) run, so exp(-V_norm) and the
// prefactor of run_tick_common.h:274-312 are evaluated once per segment and tick.  The
// cached values are the same doubles the full functions compute, so every GHK result is
// unchanged; a call with another V (the bouton voltage divider, a clamped V) falls back
// to the full evaluation.
struct GhkCache {
    float Vc;          // V the factors belong to
    uint8_t m1, m2;    // branch: 0 general, 1 |V_norm| < 1e-6, 2 V_norm > 20, 3 V_norm < -20
    double A1, e1, D1; // monovalent/anion: k*F*V*0.001, exp(-V_norm), 1 - exp(-V_norm)
    double A2, e2, D2; // divalent
};

// Segment state visible to a modifier while it runs (registers).
struct DSeg {
    float V;
    float in[7];
    float out[7];
    float atp;
    float area;    // geometric membrane area, um^2 (run_tick_common.h:209-214)
    double vol;    // segment volume, um^3 (run_tick_common.h:262-266)
    GhkCache gc;
};

// One modifier (or receptor) instance.  st[0..6] are the reference's state[0..6];
// state[7] is the effective area, held in `area` (set_modifier_effective_area,
// run_tick_common.h:234-238, or pre/post_area for synaptic receptors).
struct DMod {
    float den;
    float st[7];
    float area;
    uint8_t av;    // active_vars (receptor conductance override index)
};

/* ---- constants (reference include/types.h:417-420, include/units.h) ---- */
#define FARADAY_CONST 96485.0
#define GAS_CONST 8.314f
#define CELSIUS_37 310.15f
#define PI_F 3.14159265f
#define MM_TO_UM 1e3f
#define MV_TO_V 1e-3f
#define UM3_TO_M3 1e-18f
#define A_TO_PA 1e12f
#define PS_TO_S 1e-12f
#define ELEMENTARY_CHARGE_C 1.602176634e-19f
#define EXTRA_VOLUME_RATIO (0.2f / (1.0f - 0.2f))
#define NMOL_CM2_S_TO_MOL_UM2_MS 1e-20f
#define GHK_CBAR_NA_MM 55.964f
#define GHK_CBAR_K_MM 40.514f
#define GHK_CBAR_CA_MM 0.12775f
#define GHK_CBAR_CL_MM 36.20f




/* ---- helpers: reference include/run_tick_common.h, include/modifier_helpers.h ---- */

/* modifier_helpers.h:1117-1121: arrays are double in the reference */
__device__ __forceinline__ void dp_clamp_ions(float* arr) {
    for (int i = 0; i < 7; i++)
        if ((double)arr[i] < 1e-9) arr[i] = (float)1e-9;
}
/* run_tick_common.h:274-312 */
static __device__ __forceinline__ double dp_ghk_mono(double V, double c_in, double c_out) {
    double V_norm = FARADAY_CONST * V * 0.001 / (GAS_CONST * CELSIUS_37);
    if (fabs(V_norm) < 1e-6) return FARADAY_CONST * (c_in - c_out);
    double k = FARADAY_CONST / (GAS_CONST * CELSIUS_37);
    if (V_norm > 20.0) return k * FARADAY_CONST * V * 0.001 * c_in;
    if (V_norm < -20.0) return k * FARADAY_CONST * V * 0.001 * c_out;
    return k * FARADAY_CONST * V * 0.001 * (c_in - c_out * dm_exp(-V_norm)) / (1.0 - dm_exp(-V_norm));
}
static __device__ __forceinline__ double dp_ghk_div(double V, double c_in, double c_out) {
    double V_norm = 2.0 * FARADAY_CONST * V * 0.001 / (GAS_CONST * CELSIUS_37);
    if (fabs(V_norm) < 1e-6) return 2.0 * FARADAY_CONST * (c_in - c_out);
    double k = 4.0 * FARADAY_CONST / (GAS_CONST * CELSIUS_37);
    if (V_norm > 20.0) return k * FARADAY_CONST * V * 0.001 * c_in;
    if (V_norm < -20.0) return k * FARADAY_CONST * V * 0.001 * c_out;
    return k * FARADAY_CONST * V * 0.001 * (c_in - c_out * dm_exp(-V_norm)) / (1.0 - dm_exp(-V_norm));
}
static __device__ __forceinline__ double dp_ghk_anion(double V, double c_in, double c_out) {
    double V_norm = FARADAY_CONST * V * 0.001 / (GAS_CONST * CELSIUS_37);
    if (fabs(V_norm) < 1e-6) return FARADAY_CONST * (c_out - c_in);
    double k = FARADAY_CONST / (GAS_CONST * CELSIUS_37);
    if (V_norm > 20.0) return k * FARADAY_CONST * V * 0.001 * c_out;
    if (V_norm < -20.0) return k * FARADAY_CONST * V * 0.001 * c_in;
    return k * FARADAY_CONST * V * 0.001 * (c_out - c_in * dm_exp(-V_norm)) / (1.0 - dm_exp(-V_norm));
}

/* GHK with the per-segment factors (see GhkCache); identical results to
 * dp_ghk_mono/div/anion above. */
static __device__ __forceinline__ void ghk_cache_fill(GhkCache& c, float Vf) {
    double V = Vf;
    c.Vc = Vf;
    double Vn1 = FARADAY_CONST * V * 0.001 / (GAS_CONST * CELSIUS_37);
    c.m1 = (fabs(Vn1) < 1e-6) ? 1 : (Vn1 > 20.0) ? 2 : (Vn1 < -20.0) ? 3 : 0;
    double k1 = FARADAY_CONST / (GAS_CONST * CELSIUS_37);
    c.A1 = k1 * FARADAY_CONST * V * 0.001;
    c.e1 = (c.m1 == 0) ? dm_exp(-Vn1) : 0.0;
    c.D1 = 1.0 - c.e1;
    double Vn2 = 2.0 * FARADAY_CONST * V * 0.001 / (GAS_CONST * CELSIUS_37);
    c.m2 = (fabs(Vn2) < 1e-6) ? 1 : (Vn2 > 20.0) ? 2 : (Vn2 < -20.0) ? 3 : 0;
    double k2 = 4.0 * FARADAY_CONST / (GAS_CONST * CELSIUS_37);
    c.A2 = k2 * FARADAY_CONST * V * 0.001;
    c.e2 = (c.m2 == 0) ? dm_exp(-Vn2) : 0.0;
    c.D2 = 1.0 - c.e2;
}
static __device__ __forceinline__ double dp_ghk_mono_c(const GhkCache& c, double V, double c_in, double c_out) {
    if ((float)V != c.Vc) return dp_ghk_mono(V, c_in, c_out);
    switch (c.m1) {
        case 1: return FARADAY_CONST * (c_in - c_out);
        case 2: return c.A1 * c_in;
        case 3: return c.A1 * c_out;
        default: return c.A1 * (c_in - c_out * c.e1) / c.D1;
    }
}
static __device__ __forceinline__ double dp_ghk_div_c(const GhkCache& c, double V, double c_in, double c_out) {
    if ((float)V != c.Vc) return dp_ghk_div(V, c_in, c_out);
    switch (c.m2) {
        case 1: return 2.0 * FARADAY_CONST * (c_in - c_out);
        case 2: return c.A2 * c_in;
        case 3: return c.A2 * c_out;
        default: return c.A2 * (c_in - c_out * c.e2) / c.D2;
    }
}
static __device__ __forceinline__ double dp_ghk_anion_c(const GhkCache& c, double V, double c_in, double c_out) {
    if ((float)V != c.Vc) return dp_ghk_anion(V, c_in, c_out);
    switch (c.m1) {
        case 1: return FARADAY_CONST * (c_out - c_in);
        case 2: return c.A1 * c_out;
        case 3: return c.A1 * c_in;
        default: return c.A1 * (c_out - c_in * c.e1) / c.D1;
    }
}

/* modifier_helpers.h:48-54 */
__device__ __forceinline__ double dp_ghk_P(float gamma_pS, float z, float cbar_mM) {
    double gamma_S = gamma_pS * PS_TO_S;
    double z2F2 = z * z * FARADAY_CONST * FARADAY_CONST;
    double RT = GAS_CONST * CELSIUS_37;
    return gamma_S * RT / (z2F2 * cbar_mM);
}
/* modifier_helpers.h:58-66 */
__device__ __forceinline__ void dp_nalcn_partial_P(float gamma_pS, double* P_Na, double* P_K, double* P_Ca) {
    const double fNa = 1.3, fK = 1.2, fCa = 0.5;
    double w = fNa * GHK_CBAR_NA_MM + fK * GHK_CBAR_K_MM + fCa * 4.0 * GHK_CBAR_CA_MM;
    *P_Na = dp_ghk_P((float)(gamma_pS * fNa * GHK_CBAR_NA_MM / w), 1.0f, GHK_CBAR_NA_MM);
    *P_K = dp_ghk_P((float)(gamma_pS * fK * GHK_CBAR_K_MM / w), 1.0f, GHK_CBAR_K_MM);
    *P_Ca = dp_ghk_P((float)(gamma_pS * fCa * 4.0 * GHK_CBAR_CA_MM / w), 2.0f, GHK_CBAR_CA_MM);
}
/* modifier_helpers.h:69-76 */
__device__ __forceinline__ void dp_partial_P(float gamma_pS, float fNa, float fK, float fCa,
                                double* P_Na, double* P_K, double* P_Ca) {
    double w = fNa * GHK_CBAR_NA_MM + fK * GHK_CBAR_K_MM + fCa * 4.0 * GHK_CBAR_CA_MM;
    *P_Na = dp_ghk_P((float)(gamma_pS * fNa * GHK_CBAR_NA_MM / w), 1.0f, GHK_CBAR_NA_MM);
    *P_K = dp_ghk_P((float)(gamma_pS * fK * GHK_CBAR_K_MM / w), 1.0f, GHK_CBAR_K_MM);
    *P_Ca = dp_ghk_P((float)(gamma_pS * fCa * 4.0 * GHK_CBAR_CA_MM / w), 2.0f, GHK_CBAR_CA_MM);
}
/* modifier_helpers.h:30-34 */
__device__ __forceinline__ float dp_nernst(float intra, float extra, float valence) {
    if (intra < 1e-9f) intra = 1e-9f;
    if (extra < 1e-9f) extra = 1e-9f;
    return (float)((GAS_CONST * CELSIUS_37) / (valence * FARADAY_CONST) * dm_log(extra / intra) * 1000.0f);
}
/* modifier_helpers.h:132-135 */
__device__ __forceinline__ float dp_vtrap(float x, float y) {
    if (fabsf(x / y) < 1e-6f) return y * (1.0f - x / (2.0f * y));
    return x / (1.0f - dm_exp(-x / y));
}
/* modifier_helpers.h:1090-1095 */
__device__ __forceinline__ float dp_bz_act(float V, float vh, float k) { return 1.0f / (1.0f + dm_exp(-(V - vh) / k)); }
__device__ __forceinline__ float dp_bz_inact(float V, float vh, float k) { return 1.0f / (1.0f + dm_exp((V - vh) / k)); }

/* ---- gating helpers (modifier_helpers.h:145-215, 264-271, 468-472, 689-702, 1008-1018, 882-892, 909-913, 954-967, 1137-1170, 1188-1210) ---- */
__device__ __forceinline__ float nav16_am(float V) { return 0.182f * dp_vtrap(V + 43.0f, 6.0f); }
__device__ __forceinline__ float nav16_bm(float V) { return 0.124f * dp_vtrap(-(V + 43.0f), 6.0f); }
__device__ __forceinline__ float nav16_ah(float V) { return 0.024f * dp_vtrap(V + 50.0f, 5.0f); }
__device__ __forceinline__ float nav16_bh(float V) { return 0.0091f * dp_vtrap(-(V + 75.0f), 5.0f); }
__device__ __forceinline__ float nav16_m_inf(float V) { float a = nav16_am(V), b = nav16_bm(V); return a / (a + b); }
__device__ __forceinline__ float nav16_m_tau(float V) { return 1.0f / (nav16_am(V) + nav16_bm(V)); }
__device__ __forceinline__ float nav16_h_inf(float V) { return 1.0f / (1.0f + dm_exp((V + 72.0f) / 6.2f)); }
__device__ __forceinline__ float nav16_h_tau(float V) { return 1.0f / (nav16_ah(V) + nav16_bh(V)); }
__device__ __forceinline__ float nav12_am(float V) { return 0.182f * dp_vtrap(V + 23.0f, 6.0f); }
__device__ __forceinline__ float nav12_bm(float V) { return 0.124f * dp_vtrap(-(V + 23.0f), 6.0f); }
__device__ __forceinline__ float nav12_ah(float V) { return 0.024f * dp_vtrap(V + 41.5f, 5.0f); }
__device__ __forceinline__ float nav12_bh(float V) { return 0.0091f * dp_vtrap(-(V + 66.5f), 5.0f); }
__device__ __forceinline__ float nav12_m_inf(float V) { float a = nav12_am(V), b = nav12_bm(V); return a / (a + b); }
__device__ __forceinline__ float nav12_m_tau(float V) { return 1.0f / (nav12_am(V) + nav12_bm(V)); }
__device__ __forceinline__ float nav12_h_inf(float V) { return 1.0f / (1.0f + dm_exp((V + 63.5f) / 6.2f)); }
__device__ __forceinline__ float nav12_h_tau(float V) { return 1.0f / (nav12_ah(V) + nav12_bh(V)); }
__device__ __forceinline__ float cav21_m_inf(float V) { return 1.0f / (1.0f + dm_exp(-(V - -15.0f) / (6.0f + 1e-6f))); }
__device__ __forceinline__ float cav21_h_inf(float V, float Ca_uM) {
    float h = 1.0f / (1.0f + dm_exp((V - -50.0f) / 8.0f));
    h *= 1.0f / (1.0f + Ca_uM / 3.0f);
    return h;
}
__device__ __forceinline__ float kv42_h_tau(float V) {
    return 15.0f + (170.0f - 15.0f) / (1.0f + dm_exp((V - -60.0f) / 8.0f));
}
__device__ __forceinline__ float cav31_h_tau(float V) {
    return 25.0f + (250.0f - 25.0f) / (1.0f + dm_exp((V - -65.0f) / 8.0f));
}
__device__ __forceinline__ float cav31_m_tau(float V) {
    float dv = V - -20.0f;
    float g = dm_exp(-(dv * dv) / (2.0f * 22.0f * 22.0f));
    return 1.25f + (15.0f - 1.25f) * g;
}
__device__ __forceinline__ float kv_dr_m_tau(float V, float V_half) {
    float tau = 14.6f * dm_exp(-(V - V_half) / 30.1f);
    if (tau < 0.3f) tau = 0.3f;
    if (tau > 200.0f) tau = 200.0f;
    return tau;
}
__device__ __forceinline__ float kir_f_open(float V) {
    float Vn = (float)(FARADAY_CONST * V * 0.001f / (GAS_CONST * CELSIUS_37));
    float Kd_Mg = 0.3f * dm_exp(-0.6f * 2.0f * Vn);
    float mg_block = 0.5f / Kd_Mg;
    float Kd_spm = 0.0775f * dm_exp(-0.5f * 4.0f * Vn);
    float r = 0.001f / Kd_spm;
    float spm_block = 0.0f, rk = r;
    for (int k = 0; k < 3; k++) { spm_block += rk; rk *= r; }
    return 1.0f / (1.0f + mg_block + spm_block);
}
__device__ __forceinline__ float sk_p_inf(float Ca) {
    if (Ca < 1e-9f) Ca = 1e-9f;
    float r = 0.0004f / Ca;
    return 1.0f / (1.0f + dm_pow(r, 4.0f));
}
__device__ __forceinline__ float bk_ha_po(float V_mV, float Ca) {
    float Vn = (float)(FARADAY_CONST * V_mV * MV_TO_V / (GAS_CONST * CELSIUS_37));
    float J = 0.104f * dm_exp(0.55f * Vn);
    float L = 3.7e-8f * dm_exp(0.30f * Vn);
    if (Ca < 0.0f) Ca = 0.0f;
    float K = Ca / 0.044f;
    float o = 1.0f + K * 23.0f + J * 32.0f + J * K * 23.0f * 32.0f * 3.7f;
    float c = 1.0f + K + J + J * K * 3.7f;
    o *= o; o *= o;
    c *= c; c *= c;
    float num = L * o;
    return num / (num + c);
}
__device__ __forceinline__ float nak_pump_vnorm(float V_mV, float Na_i, float K_o, float ATP_level, float K_m_Na, float K_m_K) {
    float Na3 = Na_i * Na_i * Na_i;
    float K2 = K_o * K_o;
    float K_Na3 = K_m_Na * K_m_Na * K_m_Na;
    float K_K2 = K_m_K * K_m_K;
    float f_Na = Na3 / (Na3 + K_Na3);
    float f_K = K2 / (K2 + K_K2);
    float atp = ATP_level;
    if (atp < 0.0f) atp = 0.0f;
    float f_ATP = atp / (atp + 0.5f);
    float eta = (float)(0.8f * FARADAY_CONST * (V_mV * MV_TO_V) / (GAS_CONST * CELSIUS_37));
    float a2 = 60.0f * dm_exp(0.5f * eta);
    float b2 = 6.0f * dm_exp(-(1.0f - 0.5f) * eta);
    float a1 = 200.0f * f_Na * f_ATP;
    float a3 = 200.0f * f_K;
    float a4 = 60.0f;
    float denom = a3 / a1 + (b2 + a3) / a2 + 1.0f + a3 / a4;
    float turnover = a3 / denom;
    float k3 = 200.0f;
    float v_max = k3 / (k3 / 200.0f + 1.0f + k3 / 60.0f);
    return turnover / v_max;
}
__device__ __forceinline__ float ncx_flux_norm(float V_mV, float Na_i, float Na_o, float Ca_i, float Ca_o) {
    float V_v = V_mV * MV_TO_V;
    float FRT = (float)(FARADAY_CONST / (GAS_CONST * CELSIUS_37));
    float e_eta = dm_exp(0.35f * FRT * V_v);
    float e_eta1 = dm_exp((0.35f - 1.0f) * FRT * V_v);
    float Na_i3 = Na_i * Na_i * Na_i;
    float Na_o3 = Na_o * Na_o * Na_o;
    float fwd = e_eta1 * Na_o3 * Ca_i;
    float rev = e_eta * Na_i3 * Ca_o;
    float denom = 1.0f + 0.27f * e_eta1;
    float ca_ratio = 0.000125f / Ca_i;
    float Allo = 1.0f / (1.0f + ca_ratio * ca_ratio);
    return Allo * (fwd - rev) / (denom * 530.2f);
}


/*
 * dp_modifiers.h -- CPU oracle (test infrastructure only): per-modifier
 * current functions of the reference restated with FP32 state (see the rule in
 * dp_physics.h).  One function per supported modifier type; each cites the
 * reference function it follows.
 */

/* hh_biological.cpp:193-232 (Nav1.6) and :238-277 (Nav1.2) */
template <bool kDef>
__device__ __forceinline__ double dp_nav_current(DMod& m, DSeg& s, float dt, int is12) {
    float V = s.V;
    float area = m.area;
    if (((double)s.V) < -200.0f) s.V = -200.0f;
    if (((double)s.V) > 200.0f) s.V = 200.0f;
    V = (float)((double)s.V);
    float minf = is12 ? nav12_m_inf(V) : nav16_m_inf(V);
    float mtau = is12 ? nav12_m_tau(V) : nav16_m_tau(V);
    float hinf = is12 ? nav12_h_inf(V) : nav16_h_inf(V);
    float htau = is12 ? nav12_h_tau(V) : nav16_h_tau(V);
    double m_val = minf + (((double)m.st[0]) - minf) * dm_exp(-dt / mtau);
    double h_val = hinf + (((double)m.st[1]) - hinf) * dm_exp(-dt / htau);
    if (m_val < 0.0f) m_val = 0.0f;
    if (m_val > 1.0f) m_val = 1.0f;
    if (h_val < 0.0f) h_val = 0.0f;
    if (h_val > 1.0f) h_val = 1.0f;
    m.st[0] = (float)m_val;
    m.st[1] = (float)h_val;
    float open_prob = (float)(m_val * m_val * m_val * h_val);
    double ttx = ((kDef ? 0.0 : ((double)m.st[5])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[5])) : 0.0f;
    open_prob = (float)(open_prob / (1.0f + ttx / (is12 ? 10.0f : 5.0f)));
    float pkc = 0.0f, pka = 0.0f;   /* no PKC/PKA modifiers in supported networks */
    open_prob *= (1.0f - (is12 ? 0.7f : 0.2f) * (pkc + pka) * 0.5f);
    if (open_prob < 0.0f) open_prob = 0.0f;
    double P_single = dp_ghk_P(is12 ? 20.8f : 20.7f, 1.0f, GHK_CBAR_NA_MM);
    double flux = dp_ghk_mono_c(s.gc, V, ((double)s.in[0]), ((double)s.out[0]));
    double I_A = P_single * flux * (((double)m.den) * area) * open_prob;
    double I_Na = I_A * A_TO_PA;
    double vol = s.vol;
    double cpv = FARADAY_CONST * vol / 1000.0;
    s.in[0] = (float)(((double)s.in[0]) - (I_Na * dt) / cpv);
    s.out[0] = (float)(((double)s.out[0]) + (I_Na * dt) / (cpv * EXTRA_VOLUME_RATIO));
    dp_clamp_ions(s.in);
    dp_clamp_ions(s.out);
    return -I_Na;
}

/* hh_biological.cpp:142-187 (Cav1.3) */
template <bool kDef>
__device__ __forceinline__ double dp_cav13_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double Vhalf = ((kDef ? 0.0 : ((double)m.st[3])) != 0.0f) ? -fabs((kDef ? 0.0 : ((double)m.st[3]))) : -35.0f;
    double k = ((kDef ? 0.0 : ((double)m.st[4])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[4])) : 7.0f;
    double gamma_ps = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 25.0f;
    float m_inf = (float)(1.0f / (1.0f + dm_exp(-(V - Vhalf) / (k + 1e-6f))));
    float tau_m = 2.0f;
    m.st[0] = (float)(((double)m.st[0]) + (m_inf - ((double)m.st[0])) * dt / tau_m);
    float Ca = (float)(((double)s.in[2]) * MM_TO_UM);
    float h_inf = 1.0f / (1.0f + dm_exp((V + 52.0f) / 8.0f));
    h_inf *= 1.0f / (1.0f + Ca / 3.0f);
    float tau_h = 100.0f;
    m.st[1] = (float)(((double)m.st[1]) + (h_inf - ((double)m.st[1])) * dt / tau_h);
    if (((double)m.st[0]) < 0.0f) m.st[0] = 0.0f;
    if (((double)m.st[1]) < 0.0f) m.st[1] = 0.0f;
    if (((double)m.st[0]) > 1.0f) m.st[0] = 1.0f;
    if (((double)m.st[1]) > 1.0f) m.st[1] = 1.0f;
    float ca_in = s.in[2];
    float ca_out = s.out[2];
    double P_single = dp_ghk_P((float)gamma_ps, 2.0f, GHK_CBAR_CA_MM);
    double open_prob = ((double)m.st[0]) * ((double)m.st[0]) * ((double)m.st[1]);
    double flux = dp_ghk_div_c(s.gc, V, ca_in, ca_out);
    double I_A = P_single * flux * (((double)m.den) * area) * open_prob;
    double I_Ca = I_A * A_TO_PA;
    double vol = s.vol;
    double cpm = FARADAY_CONST * vol / 1000.0;
    s.in[2] = (float)(((double)s.in[2]) - (I_Ca * dt) / (2.0f * cpm));
    s.out[2] = (float)(((double)s.out[2]) - (I_Ca * dt) / (2.0f * cpm * EXTRA_VOLUME_RATIO));
    dp_clamp_ions(s.in);
    dp_clamp_ions(s.out);
    return -I_Ca;
}

/* hh_biological.cpp:364-388 (Cav2.1: gates only, current goes to the bouton) */
__device__ __forceinline__ double dp_cav21_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float m_inf = cav21_m_inf(V);
    m.st[0] = (float)(((double)m.st[0]) + (m_inf - ((double)m.st[0])) * dt / 1.0f);
    float Ca = (float)(((double)s.in[2]) * MM_TO_UM);
    float h_inf = cav21_h_inf(V, Ca);
    m.st[1] = (float)(((double)m.st[1]) + (h_inf - ((double)m.st[1])) * dt / 300.0f);
    if (((double)m.st[0]) < 0.0f) m.st[0] = 0.0f;
    if (((double)m.st[1]) < 0.0f) m.st[1] = 0.0f;
    if (((double)m.st[0]) > 1.0f) m.st[0] = 1.0f;
    if (((double)m.st[1]) > 1.0f) m.st[1] = 1.0f;
    return 0.0f;
}

/* hh_biological.cpp:57-97 (Na/K-ATPase) */
__device__ __forceinline__ double dp_nak_pump_current(DMod& m, DSeg& s, float dt) {
    float area = m.area;
    float v_norm = nak_pump_vnorm((float)((double)s.V), (float)((double)s.in[0]), (float)((double)s.out[1]), s.atp, 10.0f, 1.5f);
    double N = ((double)m.den) * area;
    float I_pump = (float)(N * v_norm * 75.0f * ELEMENTARY_CHARGE_C * A_TO_PA);
    float volume = (float)s.vol;
    double cpm = FARADAY_CONST * volume / 1000.0;
    float transport = (float)(I_pump * dt / cpm);
    float na_avail = (float)((((double)s.in[0]) - 1e-9f) / 3.0f);
    float k_avail = (float)((((double)s.out[1]) - 1e-9f) * EXTRA_VOLUME_RATIO / 2.0f);
    if (na_avail < 0.0f) na_avail = 0.0f;
    if (k_avail < 0.0f) k_avail = 0.0f;
    float max_t = (na_avail < k_avail) ? na_avail : k_avail;
    if (transport > max_t) transport = max_t;
    s.in[0] = (float)(((double)s.in[0]) - 3.0f * transport);
    s.out[0] = (float)(((double)s.out[0]) + 3.0f * transport / EXTRA_VOLUME_RATIO);
    s.in[1] = (float)(((double)s.in[1]) + 2.0f * transport);
    s.out[1] = (float)(((double)s.out[1]) - 2.0f * transport / EXTRA_VOLUME_RATIO);
    dp_clamp_ions(s.in);
    dp_clamp_ions(s.out);
    s.atp -= I_pump * dt * 1e-8f;
    if (s.atp < 0.0f) s.atp = 0.0f;
    return -I_pump;
}

/* shared K-channel ion bookkeeping: intra K -= I*dt/cpv, extra K += .../EVR, clamp extra */
__device__ __forceinline__ void dp_k_flux(DSeg& s, double I_K, float dt, double cpv) {
    s.in[1] = (float)(((double)s.in[1]) - (I_K * dt) / cpv);
    s.out[1] = (float)(((double)s.out[1]) + (I_K * dt) / (cpv * EXTRA_VOLUME_RATIO));
    dp_clamp_ions(s.out);
}

/* hh_biological.cpp:789-841 (Kv4.2) */
template <bool kDef>
__device__ __forceinline__ double dp_kv42_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double Vhalf = ((kDef ? 0.0 : ((double)m.st[4])) != 0.0f) ? -fabs((kDef ? 0.0 : ((double)m.st[4]))) : -10.0f;
    double k = ((kDef ? 0.0 : ((double)m.st[5])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[5])) : 13.5f;
    double gamma_ps = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 5.0f;
    float m_inf = (float)(1.0f / (1.0f + dm_exp(-(V - Vhalf) / (k + 1e-6f))));
    float tau_m = 1.5f;
    m.st[0] = (float)(((double)m.st[0]) + (m_inf - ((double)m.st[0])) * dt / tau_m);
    float h_inf = 1.0f / (1.0f + dm_exp((V + 65.0f) / 8.0f));
    float tau_h = kv42_h_tau(V);
    m.st[1] = (float)(((double)m.st[1]) + (h_inf - ((double)m.st[1])) * dt / tau_h);
    if (((double)m.st[0]) < 0.0f) m.st[0] = 0.0f;
    if (((double)m.st[1]) < 0.0f) m.st[1] = 0.0f;
    if (((double)m.st[0]) > 1.0f) m.st[0] = 1.0f;
    if (((double)m.st[1]) > 1.0f) m.st[1] = 1.0f;
    float camkii = 0.0f;   /* no CaMKII modifiers in supported networks */
    m.st[3] = (float)(((double)m.st[3]) + (camkii * 0.5f - ((double)m.st[3])) * dt / 5000.0f);
    if (((double)m.st[3]) < 0.0f) m.st[3] = 0.0f;
    if (((double)m.st[3]) > 1.0f) m.st[3] = 1.0f;
    double gamma_eff = gamma_ps * (1.0f - ((double)m.st[3]) * 0.7f);
    float K_i = s.in[1];
    float K_o = s.out[1];
    double P_single = dp_ghk_P((float)gamma_eff, 1.0f, GHK_CBAR_K_MM);
    double open_prob = ((double)m.st[0]) * ((double)m.st[0]) * ((double)m.st[0]) * ((double)m.st[1]);
    double flux = dp_ghk_mono_c(s.gc, V, K_i, K_o);
    double I_A = P_single * flux * (((double)m.den) * area) * open_prob;
    double I_K = I_A * A_TO_PA;
    double vol = s.vol;
    double cpv = FARADAY_CONST * vol / 1000.0;
    dp_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:1043-1100 (Kv3.1) */
template <bool kDef>
__device__ __forceinline__ double dp_kv31_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    float Vhalf = 10.0f, k = 10.0f, gamma_ps = 27.0f;
    float m_inf = 1.0f / (1.0f + dm_exp(-(V - Vhalf) / (k + 1e-6f)));
    float tau_m = 1.0f;
    m.st[0] = (float)(((double)m.st[0]) + (m_inf - ((double)m.st[0])) * dt / tau_m);
    if (((double)m.st[0]) < 0.0f) m.st[0] = 0.0f;
    if (((double)m.st[0]) > 1.0f) m.st[0] = 1.0f;
    float h_inf = 1.0f / (1.0f + dm_exp((V + 30.0f) / 6.0f));
    float tau_h = 2000.0f;
    m.st[1] = (float)(((double)m.st[1]) + (h_inf - ((double)m.st[1])) * dt / tau_h);
    if (((double)m.st[1]) < 0.0f) m.st[1] = 0.0f;
    if (((double)m.st[1]) > 1.0f) m.st[1] = 1.0f;
    float K_i = s.in[1];
    float K_o = s.out[1];
    double P_single = dp_ghk_P(gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double open_prob = ((double)m.st[0]) * ((double)m.st[0]) * ((double)m.st[0]) * ((double)m.st[1]);
    double tea = ((kDef ? 0.0 : ((double)m.st[5])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[5])) : 0.0f;
    open_prob /= (1.0f + tea / 0.2f);
    float pkc = 0.0f;
    float k_phos = 5.6e-6f;
    float k_dephos = 1e-4f;
    m.st[2] = (float)(((double)m.st[2]) + (k_phos * pkc * (1.0f - ((double)m.st[2])) - k_dephos * ((double)m.st[2])) * dt);
    if (((double)m.st[2]) < 0.0f) m.st[2] = 0.0f;
    if (((double)m.st[2]) > 1.0f) m.st[2] = 1.0f;
    open_prob *= (1.0f - 0.27f * ((double)m.st[2]));
    double flux = dp_ghk_mono_c(s.gc, V, K_i, K_o);
    double I_A = P_single * flux * (((double)m.den) * area) * open_prob;
    double I_K = I_A * A_TO_PA;
    double vol = s.vol;
    double cpv = FARADAY_CONST * vol / 1000.0;
    dp_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:2070-2105 (Cav3.1) */
template <bool kDef>
__device__ __forceinline__ double dp_cav31_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double gamma_ps = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 7.5f;
    double m_val = ((double)m.st[0]), h_val = ((double)m.st[1]);
    float m_inf = dp_bz_act(V, -45.0f, 5.5f);
    float h_inf = dp_bz_inact(V, -77.0f, 6.0f);
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
    m.st[0] = (float)m_val;
    m.st[1] = (float)h_val;
    float open_prob = (float)(m_val * m_val * m_val * h_val);
    double ni = ((kDef ? 0.0 : ((double)m.st[3])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[3])) : 0.0f;
    double mib = ((kDef ? 0.0 : ((double)m.st[4])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[4])) : 0.0f;
    double tta = ((kDef ? 0.0 : ((double)m.st[5])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[5])) : 0.0f;
    double z944 = ((kDef ? 0.0 : ((double)m.st[6])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[6])) : 0.0f;
    open_prob = (float)(open_prob / ((1.0f + ni / 250.0f) * (1.0f + mib / 1.6f)
                                     * (1.0f + tta / 82.0f) * (1.0f + z944 / 100.0f)));
    double P_single = dp_ghk_P((float)gamma_ps, 2.0f, GHK_CBAR_CA_MM);
    double flux = dp_ghk_div_c(s.gc, V, ((double)s.in[2]), ((double)s.out[2]));
    double I_A = P_single * flux * (((double)m.den) * area) * open_prob;
    double I_CaT = I_A * A_TO_PA;
    float volume = (float)s.vol;
    float charge_per_mole = (float)(FARADAY_CONST * volume / 1000.0);
    s.in[2] = (float)(((double)s.in[2]) - (I_CaT * dt) / (2.0f * charge_per_mole));
    return -I_CaT;
}

/* hh_biological.cpp:2574-2613 (PMCA) */
template <bool kDef>
__device__ __forceinline__ double dp_pmca_current(DMod& m, DSeg& s, float dt) {
    float area = m.area;
    double K_m_Ca = ((kDef ? 0.0 : ((double)m.st[1])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[1])) : 0.0003f;
    double hill_n = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 2.0f;
    float atp = s.atp;
    if (atp < 0.0f) atp = 0.0f;
    float f_ATP = atp / (atp + 0.2f);
    float ca = s.in[2];
    if (ca < 1e-9f) ca = 1e-9f;
    float ca_pow = (float)dm_pow(ca, hill_n);
    float f_Ca = (float)(ca_pow / (ca_pow + dm_pow(K_m_Ca, hill_n)));
    double N = ((double)m.den) * area;
    float I_pump = (float)(N * 100.0f * f_Ca * f_ATP * ELEMENTARY_CHARGE_C * 2.0f * A_TO_PA);
    float volume = (float)s.vol;
    double cpv = FARADAY_CONST * volume / 1000.0;
    float transport = (float)(I_pump * dt / (2.0f * cpv));
    float ca_avail = (float)(((double)s.in[2]) - 1e-9f);
    if (ca_avail < 0.0f) ca_avail = 0.0f;
    if (transport > ca_avail) transport = ca_avail;
    s.in[2] = (float)(((double)s.in[2]) - transport);
    s.out[2] = (float)(((double)s.out[2]) + transport / EXTRA_VOLUME_RATIO);
    dp_clamp_ions(s.in);
    s.atp -= I_pump * dt * 1e-8f;
    if (s.atp < 0.0f) s.atp = 0.0f;
    return -I_pump;
}

/* hh_biological.cpp:2616-2646 (NCX) */
__device__ __forceinline__ double dp_ncx_current(DMod& m, DSeg& s, float dt) {
    float area = m.area;
    float Na_i = s.in[0]; if (Na_i < 1e-9f) Na_i = 1e-9f;
    float Na_o = s.out[0]; if (Na_o < 1e-9f) Na_o = 1e-9f;
    float Ca_i = s.in[2]; if (Ca_i < 1e-9f) Ca_i = 1e-9f;
    float Ca_o = s.out[2]; if (Ca_o < 1e-9f) Ca_o = 1e-9f;
    float flux_norm = ncx_flux_norm((float)((double)s.V), Na_i, Na_o, Ca_i, Ca_o);
    double N = ((double)m.den) * area;
    float I_ncx = (float)(N * 500.0f * flux_norm * ELEMENTARY_CHARGE_C * A_TO_PA);
    float volume = (float)s.vol;
    double cpv = FARADAY_CONST * volume / 1000.0;
    float transport = (float)(I_ncx * dt / cpv);
    if (transport > Ca_i) transport = Ca_i;
    if (transport < -Na_i / 3.0f) transport = -Na_i / 3.0f;
    s.in[2] = (float)(((double)s.in[2]) - transport);
    s.out[2] = (float)(((double)s.out[2]) + transport / EXTRA_VOLUME_RATIO);
    s.in[0] = (float)(((double)s.in[0]) + 3.0f * transport);
    s.out[0] = (float)(((double)s.out[0]) - 3.0f * transport / EXTRA_VOLUME_RATIO);
    dp_clamp_ions(s.in);
    return I_ncx;
}

/* hh_biological.cpp:2648-2702 (KCC2) */
template <bool kDef>
__device__ __forceinline__ double dp_kcc2_current(DMod& m, DSeg& s, float dt) {
    float area = m.area;
    double Km_K_i = ((kDef ? 0.0 : ((double)m.st[1])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[1])) : 6.5f;
    double Km_Cl_i = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 6.5f;
    float K_i = s.in[1]; if (K_i < 1e-9f) K_i = 1e-9f;
    float Cl_i = s.in[3]; if (Cl_i < 1e-9f) Cl_i = 1e-9f;
    float K_o = s.out[1]; if (K_o < 1e-9f) K_o = 1e-9f;
    float Cl_o = s.out[3]; if (Cl_o < 1e-9f) Cl_o = 1e-9f;
    float f_K = (float)(K_i / (K_i + Km_K_i));
    float f_Cl = (float)(Cl_i / (Cl_i + Km_Cl_i));
    float driving = 1.0f - (K_o * Cl_o) / (K_i * Cl_i);
    if (driving > 1.0f) driving = 1.0f;
    if (driving < -1.0f) driving = -1.0f;
    float flux_mol = (float)(5.0f * NMOL_CM2_S_TO_MOL_UM2_MS * ((double)m.den) * area * f_K * f_Cl * driving * dt);
    float dconc = (float)(flux_mol / (s.vol * UM3_TO_M3));
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
    s.in[1] = (float)(((double)s.in[1]) - dconc);
    s.in[3] = (float)(((double)s.in[3]) - dconc);
    s.out[1] = (float)(((double)s.out[1]) + dconc / EXTRA_VOLUME_RATIO);
    s.out[3] = (float)(((double)s.out[3]) + dconc / EXTRA_VOLUME_RATIO);
    dp_clamp_ions(s.in);
    return 0.0f;
}

/* hh_biological.cpp:2825-2857 (Ca2+ buffer) */
template <bool kDef>
__device__ __forceinline__ double dp_ca_buffer_current(DMod& m, DSeg& s, float dt) {
    double B_total_ref = ((kDef ? 0.0 : ((double)m.st[0])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[0])) : 0.15f;
    double B_total = B_total_ref * ((double)m.den);
    double K_d = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 0.0005f;
    double k_on = ((kDef ? 0.0 : ((double)m.st[3])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[3])) : 0.1f;
    double k_off = ((kDef ? 0.0 : ((double)m.st[4])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[4])) : (K_d * k_on);
    double Ca_bound = ((double)m.st[1]);
    if (Ca_bound <= 0.0f && B_total > 0.0f) {
        float Ca_free0 = s.in[2];
        Ca_bound = B_total * Ca_free0 / (Ca_free0 + K_d);
        m.st[1] = (float)Ca_bound;
    }
    float Ca_free = s.in[2];
    if (Ca_free < 1e-9f) Ca_free = 1e-9f;
    float B_free = (float)(B_total - Ca_bound);
    if (B_free < 0.0f) B_free = 0.0f;
    float dCa_bound = (float)((k_on * Ca_free * B_free - k_off * Ca_bound) * dt);
    Ca_bound += dCa_bound;
    if (Ca_bound < 0.0f) Ca_bound = 0.0f;
    if (Ca_bound > B_total) Ca_bound = B_total;
    s.in[2] = (float)(((double)s.in[2]) - dCa_bound);
    if (((double)s.in[2]) < 1e-9f) {
        float deficit = (float)(1e-9f - ((double)s.in[2]));
        s.in[2] = 1e-9f;
        Ca_bound -= deficit;
        if (Ca_bound < 0.0f) Ca_bound = 0.0f;
    }
    m.st[1] = (float)Ca_bound;
    return 0.0f;
}

/* hh_biological.cpp:2859-2888 (SK) */
template <bool kDef>
__device__ __forceinline__ double dp_sk_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double open_prob = ((double)m.st[0]);
    double gamma_ps = ((kDef ? 0.0 : ((double)m.st[3])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[3])) : 10.0f;
    double tau_open = ((kDef ? 0.0 : ((double)m.st[4])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[4])) : 5.0f;
    double tau_close = ((kDef ? 0.0 : ((double)m.st[5])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[5])) : 50.0f;
    float ca = s.in[2];
    float p_inf = sk_p_inf(ca);
    float tau = (float)((p_inf > open_prob) ? tau_open : tau_close);
    open_prob += (p_inf - open_prob) * dt / tau;
    if (open_prob < 0.0f) open_prob = 0.0f;
    if (open_prob > 1.0f) open_prob = 1.0f;
    m.st[0] = (float)open_prob;
    float K_i = s.in[1], K_o = s.out[1];
    double P_single = dp_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double flux = dp_ghk_mono_c(s.gc, V, K_i, K_o);
    double I_A = P_single * flux * (((double)m.den) * area) * open_prob;
    float I_K = (float)(I_A * A_TO_PA);
    double vol = s.vol;
    double cpv = FARADAY_CONST * vol / 1000.0f;
    s.in[1] = (float)(((double)s.in[1]) - (I_K * dt) / cpv);
    s.out[1] = (float)(((double)s.out[1]) + (I_K * dt) / (cpv * EXTRA_VOLUME_RATIO));
    dp_clamp_ions(s.out);
    return -I_K;
}

/* hh_biological.cpp:2922-2949 (BK) */
template <bool kDef>
__device__ __forceinline__ double dp_bk_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double open_prob = ((double)m.st[0]);
    double gamma_ps = ((kDef ? 0.0 : ((double)m.st[1])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[1])) : 250.0f;
    double tau_ch = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 1.0f;
    float Ca = s.in[2];
    float po_inf = bk_ha_po(V, Ca);
    open_prob += (po_inf - open_prob) * dt / tau_ch;
    if (open_prob < 0.0f) open_prob = 0.0f;
    if (open_prob > 1.0f) open_prob = 1.0f;
    m.st[0] = (float)open_prob;
    float K_i = s.in[1], K_o = s.out[1];
    double P_single = dp_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double flux = dp_ghk_mono_c(s.gc, V, K_i, K_o);
    double I_A = P_single * flux * (((double)m.den) * area) * open_prob;
    float I_K = (float)(I_A * A_TO_PA);
    double vol = s.vol;
    double cpv = FARADAY_CONST * vol / 1000.0f;
    s.in[1] = (float)(((double)s.in[1]) - (I_K * dt) / cpv);
    s.out[1] = (float)(((double)s.out[1]) + (I_K * dt) / (cpv * EXTRA_VOLUME_RATIO));
    dp_clamp_ions(s.out);
    return -I_K;
}

/* hh_biological.cpp:2951-2978 (NaP) */
template <bool kDef>
__device__ __forceinline__ double dp_nap_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double m_val = ((double)m.st[0]);
    double V_half = ((kDef ? 0.0 : ((double)m.st[1])) != 0.0f) ? (kDef ? 0.0 : ((double)m.st[1])) : -58.7f;
    double k_m = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 6.0f;
    double gamma_ps = ((kDef ? 0.0 : ((double)m.st[3])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[3])) : 20.7f;
    double tau_m = ((kDef ? 0.0 : ((double)m.st[4])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[4])) : 5.0f;
    double Po = ((kDef ? 0.0 : ((double)m.st[5])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[5])) : 0.016f;
    float m_inf = dp_bz_act(V, (float)V_half, (float)k_m);
    m_val += (m_inf - m_val) * dt / tau_m;
    if (m_val < 0.0f) m_val = 0.0f;
    if (m_val > 1.0f) m_val = 1.0f;
    m.st[0] = (float)m_val;
    float Na_i = s.in[0], Na_o = s.out[0];
    double P_single = dp_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_NA_MM);
    double flux = dp_ghk_mono_c(s.gc, V, Na_i, Na_o);
    double I_A = P_single * flux * (((double)m.den) * area) * (m_val * Po);
    float I_Na = (float)(I_A * A_TO_PA);
    double vol = s.vol;
    double cpv = FARADAY_CONST * vol / 1000.0f;
    s.in[0] = (float)(((double)s.in[0]) - (I_Na * dt) / cpv);
    dp_clamp_ions(s.in);
    return -I_Na;
}

/* hh_biological.cpp:3018-3038 (Kir2.1) */
template <bool kDef>
__device__ __forceinline__ double dp_kir_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double gamma_ps = ((kDef ? 0.0 : ((double)m.st[3])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[3])) : 30.0f;
    float K_i = s.in[1], K_o = s.out[1];
    float f_open = kir_f_open(V);
    double P_single = dp_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double flux = dp_ghk_mono_c(s.gc, V, K_i, K_o);
    double I_A = P_single * flux * (((double)m.den) * area) * f_open;
    double I_K = I_A * A_TO_PA;
    double vol = s.vol;
    double cpv = FARADAY_CONST * vol / 1000.0f;
    dp_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:3063-3084 (K2P leak) */
template <bool kDef>
__device__ __forceinline__ double dp_k2p_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double gamma_ps = ((kDef ? 0.0 : ((double)m.st[0])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[0])) : 100.0f;
    double Po = ((kDef ? 0.0 : ((double)m.st[1])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[1])) : 0.012f;
    float K_i = s.in[1];
    float K_o = s.out[1];
    double P_single = dp_ghk_P((float)gamma_ps, 1.0f, GHK_CBAR_K_MM);
    double flux = dp_ghk_mono_c(s.gc, V, K_i, K_o);
    double I_A = P_single * flux * (((double)m.den) * area) * Po;
    double I_K = I_A * A_TO_PA;
    double vol = s.vol;
    double cpv = FARADAY_CONST * vol / 1000.0;
    dp_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:3158-3202 (Kv7 M-current) */
template <bool kDef>
__device__ __forceinline__ double dp_kv7_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double m_val = ((double)m.st[0]);
    double V_half = ((kDef ? 0.0 : ((double)m.st[1])) != 0.0f) ? (kDef ? 0.0 : ((double)m.st[1])) : -38.0f;
    double k_slope = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 10.0f;
    double tau_act = ((kDef ? 0.0 : ((double)m.st[4])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[4])) : 100.0f;
    double tau_deact = ((kDef ? 0.0 : ((double)m.st[5])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[5])) : 60.0f;
    double pip2 = ((kDef ? 1.0 : ((double)m.st[6])) >= 0.0f) ? (kDef ? 1.0 : ((double)m.st[6])) : 1.0f;
    float m_inf = (float)(1.0f / (1.0f + dm_exp(-(V - V_half) / k_slope)));
    float tau_m = (float)(tau_deact + (tau_act - tau_deact) * m_inf);
    if (tau_m < 1.0f) tau_m = 1.0f;
    m_val += (m_inf - m_val) * dt / tau_m;
    if (m_val < 0.0f) m_val = 0.0f;
    if (m_val > 1.0f) m_val = 1.0f;
    m.st[0] = (float)m_val;
    if (pip2 < 0.01f) return 0.0f;
    float K_i = s.in[1];
    float K_o = s.out[1];
    double P_single = dp_ghk_P(7.0f, 1.0f, GHK_CBAR_K_MM);
    float pkc = 0.0f;
    float pkc_suppress = 1.0f - 0.8f * pkc;
    if (pkc_suppress < 0.0f) pkc_suppress = 0.0f;
    double flux = dp_ghk_mono_c(s.gc, V, K_i, K_o);
    double I_A = P_single * flux * (((double)m.den) * area) * (m_val * pip2 * pkc_suppress);
    double I_K = I_A * A_TO_PA;
    double vol = s.vol;
    double cpv = FARADAY_CONST * vol / 1000.0;
    dp_k_flux(s, I_K, dt, cpv);
    return -I_K;
}

/* hh_biological.cpp:2763-2797 (Kv1.1 delayed rectifier) */
template <bool kDef>
__device__ __forceinline__ double dp_kvdr_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double m_val = ((double)m.st[0]);
    double V_half = ((kDef ? 0.0 : ((double)m.st[1])) != 0.0f) ? (kDef ? 0.0 : ((double)m.st[1])) : -30.0f;
    double k = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : 6.0f;
    double tau = ((kDef ? 0.0 : ((double)m.st[4])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[4])) : kv_dr_m_tau(V, (float)V_half);
    float m_inf = (float)(1.0f / (1.0f + dm_exp(-(V - V_half) / (k + 1e-6f))));
    m_val += (m_inf - m_val) * dt / (tau + 1e-6f);
    if (m_val < 0.0f) m_val = 0.0f;
    if (m_val > 1.0f) m_val = 1.0f;
    m.st[0] = (float)m_val;
    float K_i = s.in[1];
    float K_o = s.out[1];
    double P_single = dp_ghk_P(12.0f, 1.0f, GHK_CBAR_K_MM);
    double flux = dp_ghk_mono_c(s.gc, V, K_i, K_o);
    double I_A = P_single * flux * (((double)m.den) * area) * m_val;
    double I_K = I_A * A_TO_PA;
    double vol = s.vol;
    float charge_per_mole_vol = (float)(FARADAY_CONST * vol / 1000.0);
    s.in[1] = (float)(((double)s.in[1]) - (I_K * dt) / charge_per_mole_vol);
    s.out[1] = (float)(((double)s.out[1]) + (I_K * dt) / (charge_per_mole_vol * EXTRA_VOLUME_RATIO));
    dp_clamp_ions(s.in);
    dp_clamp_ions(s.out);
    return -I_K;
}

/* modifier_helpers.h:1442-1484 (hcn_generic_current) via hh_biological.cpp:3598 (HCN1) */
template <bool kDef>
__device__ __forceinline__ double dp_hcn1_current(DMod& m, DSeg& s, float dt) {
    double V = ((double)s.V);
    float area = m.area;
    float V_half = ((kDef ? 0.0 : ((double)m.st[1])) != 0) ? (float)(kDef ? 0.0 : ((double)m.st[1])) : -69.0f;
    float k = ((kDef ? 0.0 : ((double)m.st[2])) > 0) ? (float)(kDef ? 0.0 : ((double)m.st[2])) : 6.0f;
    float gamma_ps = ((kDef ? 0.0 : ((double)m.st[3])) > 0) ? (float)(kDef ? 0.0 : ((double)m.st[3])) : 0.84f;
    float tau_open = ((kDef ? 0.0 : ((double)m.st[4])) > 0) ? (float)(kDef ? 0.0 : ((double)m.st[4])) : 84.0f;
    float tau_close = ((kDef ? 0.0 : ((double)m.st[5])) > 0) ? (float)(kDef ? 0.0 : ((double)m.st[5])) : 300.0f;
    float camp = 0.1f;  /* segment_camp_um: no cAMP/PKA modifier -> basal 0.1 uM (units.h:324) */
    float Ve = V_half + 15.0f * camp / (camp + 0.5f);
    float mv = m.st[0];
    float mi = 1.0f / (1.0f + dm_exp(((float)V - Ve) / k));
    float tau_eff = (V < Ve) ? (float)(tau_open * dm_exp((V - Ve) / 15.0f)) : tau_close;
    mv += (mi - mv) * dt / tau_eff;
    if (mv < 0.0f) mv = 0.0f;
    if (mv > 1.0f) mv = 1.0f;
    m.st[0] = mv;
    double P_Na, P_K, P_Ca;
    dp_partial_P(gamma_ps, 0.2f, 0.8f, 0.0f, &P_Na, &P_K, &P_Ca);
    double N = ((double)m.den) * area;
    double flux_Na = dp_ghk_mono_c(s.gc, V, ((double)s.in[0]), ((double)s.out[0]));
    double flux_K = dp_ghk_mono_c(s.gc, V, ((double)s.in[1]), ((double)s.out[1]));
    double In = P_Na * flux_Na * N * mv * A_TO_PA;
    double Ik = P_K * flux_K * N * mv * A_TO_PA;
    double vol = s.vol;
    double cpm = FARADAY_CONST * vol / 1000.0;
    s.in[0] = (float)(((double)s.in[0]) - (In * dt) / cpm);
    s.in[1] = (float)(((double)s.in[1]) - (Ik * dt) / cpm);
    s.out[0] = (float)(((double)s.out[0]) + (In * dt) / (cpm * EXTRA_VOLUME_RATIO));
    s.out[1] = (float)(((double)s.out[1]) + (Ik * dt) / (cpm * EXTRA_VOLUME_RATIO));
    dp_clamp_ions(s.in);
    dp_clamp_ions(s.out);
    return -(In + Ik);
}

/* hh_biological.cpp:3609-3641 (NALCN; the returned sign follows the reference) */
template <bool kDef>
__device__ __forceinline__ double dp_nalcn_current(DMod& m, DSeg& s, float dt) {
    float V = s.V;
    float area = m.area;
    double gamma_ps = ((kDef ? 0.0 : ((double)m.st[0])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[0])) : 27.0f;
    double P_Na, P_K, P_Ca;
    dp_nalcn_partial_P((float)gamma_ps, &P_Na, &P_K, &P_Ca);
    double N = ((double)m.den) * area;
    float Ina = (float)(P_Na * dp_ghk_mono_c(s.gc, V, ((double)s.in[0]), ((double)s.out[0])) * N * A_TO_PA);
    float Ik = (float)(P_K * dp_ghk_mono_c(s.gc, V, ((double)s.in[1]), ((double)s.out[1])) * N * A_TO_PA);
    float Ica = (float)(P_Ca * dp_ghk_div_c(s.gc, V, ((double)s.in[2]), ((double)s.out[2])) * N * A_TO_PA);
    double vol = s.vol;
    double cpm = FARADAY_CONST * vol / 1000.0;
    s.in[0] = (float)(((double)s.in[0]) - (Ina * dt) / cpm);
    s.in[1] = (float)(((double)s.in[1]) - (Ik * dt) / cpm);
    s.in[2] = (float)(((double)s.in[2]) - (Ica * dt) / (2.0f * cpm));
    s.out[0] = (float)(((double)s.out[0]) + (Ina * dt) / (cpm * EXTRA_VOLUME_RATIO));
    s.out[1] = (float)(((double)s.out[1]) + (Ik * dt) / (cpm * EXTRA_VOLUME_RATIO));
    s.out[2] = (float)(((double)s.out[2]) + (Ica * dt) / (2.0f * cpm * EXTRA_VOLUME_RATIO));
    dp_clamp_ions(s.in);
    dp_clamp_ions(s.out);
    return -(Ina - Ik + Ica);
}

/* modifier_helpers.h:1213-1278 (ionotropic_ghk_current) */
template <bool kDef>
__device__ __forceinline__ double dp_ionotropic(DMod& m, DSeg& s, float dt, float nt, float gamma_ps, float EC50, float tau_rise,
                            float tau_decay, float P_Na_ratio, float P_K_ratio,
                            float P_Ca_ratio, int is_anion, float tau_desens, float K_desens,
                            float mod_scale) {
    float area = m.area;
    double V = ((double)s.V);
    double vol = s.vol;
    double cpm = FARADAY_CONST * vol / 1000.0;
    float p_gamma_ps = gamma_ps;
    if (!kDef) {
        float stav = (m.av == 7) ? m.area : ((m.av > 0 && m.av < 7) ? m.st[m.av] : 0.0f);
        p_gamma_ps = (m.av > 0 && m.av < 8 && ((double)stav) > 0.0f) ? (float)((double)stav) : gamma_ps;
    }
    float r_inf = nt / (nt + EC50);
    float r = m.st[0];
    float tau = (r_inf > r) ? tau_rise : tau_decay;
    m.st[0] = (float)(((double)m.st[0]) + (r_inf - r) * dt / tau);
    if (((double)m.st[0]) < 0.0f) m.st[0] = 0.0f;
    if (((double)m.st[0]) > 1.0f) m.st[0] = 1.0f;
    float open_prob = m.st[0];
    if (tau_desens > 0.0f) {
        float kd = (K_desens > 0.0f) ? K_desens : EC50;
        float d = m.st[1];
        float d_inf = nt / (nt + kd);
        d += (d_inf - d) * dt / tau_desens;
        if (d < 0.0f) d = 0.0f;
        if (d > 1.0f) d = 1.0f;
        m.st[1] = d;
        open_prob *= (1.0f - d);
    }
    double N = ((double)m.den) * area;
    double I_total = 0.0;
    if (is_anion) {
        double P_Cl = dp_ghk_P(p_gamma_ps, 1.0f, GHK_CBAR_CL_MM);
        double flux_Cl = dp_ghk_anion_c(s.gc, V, ((double)s.in[3]), ((double)s.out[3]));
        double I_Cl = P_Cl * flux_Cl * N * open_prob * mod_scale * A_TO_PA;
        s.in[3] = (float)(((double)s.in[3]) + (I_Cl * dt) / cpm);
        dp_clamp_ions(s.in);
        return -I_Cl;
    }
    double P_Na, P_K, P_Ca;
    dp_partial_P(p_gamma_ps, P_Na_ratio, P_K_ratio, P_Ca_ratio, &P_Na, &P_K, &P_Ca);
    double I_Na = P_Na * dp_ghk_mono_c(s.gc, V, ((double)s.in[0]), ((double)s.out[0])) * N * open_prob * mod_scale * A_TO_PA;
    double I_K = P_K * dp_ghk_mono_c(s.gc, V, ((double)s.in[1]), ((double)s.out[1])) * N * open_prob * mod_scale * A_TO_PA;
    I_total = I_Na + I_K;
    s.in[0] = (float)(((double)s.in[0]) - (I_Na * dt) / cpm);
    s.in[1] = (float)(((double)s.in[1]) - (I_K * dt) / cpm);
    if (P_Ca_ratio > 0.0f) {
        double I_Ca = P_Ca * dp_ghk_div_c(s.gc, V, ((double)s.in[2]), ((double)s.out[2])) * N * open_prob * mod_scale * A_TO_PA;
        I_total += I_Ca;
        s.in[2] = (float)(((double)s.in[2]) - (I_Ca * dt) / (2.0f * cpm));
    }
    dp_clamp_ions(s.in);
    return -I_total;
}

/* modifier_helpers.h:1281-1290 */
__device__ __forceinline__ double dp_nmda_cdi_coagonist(DMod& m, DSeg& s, float dt) {
    double Ca_uM = ((double)s.in[2]) * MM_TO_UM;
    double cdi_inf = 1.0 - 0.8f * Ca_uM / (Ca_uM + 1.0f);
    float tau = (cdi_inf < ((double)m.st[2])) ? 500.0f : 9000.0f;
    m.st[2] = (float)(((double)m.st[2]) + (cdi_inf - ((double)m.st[2])) * dt / tau);
    if (((double)m.st[2]) < 0.0f) m.st[2] = 0.0f;
    if (((double)m.st[2]) > 1.0f) m.st[2] = 1.0f;
    float coagonist = 10.0f / (10.0f + 1.0f);
    return ((double)m.st[2]) * coagonist;
}

/* receptors_biological.cpp:42-82 (AMPA, NMDA, GABA-A, glycine) */
template <bool kDef>
__device__ __forceinline__ double dp_ampa_current(DMod& m, DSeg& s, float dt, float nt, float scale) {
    return dp_ionotropic<kDef>(m, s, dt, nt, 8.0f, 0.5f, 0.5f, 3.0f, 0.5f, 0.5f, 0.0f, 0, 3.0f, 0.0f, scale);
}
template <bool kDef>
__device__ __forceinline__ double dp_nmda_current(DMod& m, DSeg& s, float dt, float nt, float scale) {
    double I = dp_ionotropic<kDef>(m, s, dt, nt, 50.0f, 1.0f, 5.0f, 50.0f, 0.08f, 0.08f, 0.84f, 0, 0.0f, 0.0f, scale);
    float mg_block = (float)(1.0f / (1.0f + (1.0f / 3.57f) * dm_exp(-0.062f * ((double)s.V))));
    double c = dp_nmda_cdi_coagonist(m, s, dt);
    return I * mg_block * c;
}
template <bool kDef>
__device__ __forceinline__ double dp_gabaa_current(DMod& m, DSeg& s, float dt, float nt, float scale) {
    return dp_ionotropic<kDef>(m, s, dt, nt, 28.0f, 1.0f, 1.0f, 5.0f, 0.0f, 0.0f, 0.0f, 1, 2000.0f, 0.0f, scale);
}
template <bool kDef>
__device__ __forceinline__ double dp_glycine_current(DMod& m, DSeg& s, float dt, float nt, float scale) {
    return dp_ionotropic<kDef>(m, s, dt, nt, 60.0f, 0.5f, 0.3f, 5.0f, 0.0f, 0.0f, 0.0f, 1, 2000.0f, 0.0f, scale);
}

/* hh_biological.cpp:1746-1767 (eCB synthesis: 2-AG from Ca2+; segment_dag is 0, as no
 * supported network carries the PLC/IP3/DAG modifier).  No current; the retrograde
 * release into the clefts runs in the synapse kernel. */
template <bool kDef>
__device__ __forceinline__ double dp_ecb_synthesis_current(DMod& m, DSeg& s, float dt) {
    float Ca = (float)((double)s.in[2] * (double)MM_TO_UM);
    double synth_rate = ((kDef ? 0.0 : ((double)m.st[1])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[1])) : (double)0.01f;
    double degrad_rate = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : (double)0.005f;
    float dag = 0.0f;
    dt = (float)((double)dt * (double)m.den);
    float Ca_n = Ca * Ca;
    float synth = (float)(synth_rate * (double)Ca_n / (double)(Ca_n + 0.25f + 1e-9f) * (double)(1.0f + dag));
    m.st[0] = (float)((double)m.st[0] + ((double)synth - (double)m.st[0] * degrad_rate) * (double)dt);
    if (m.st[0] < 0.0f) m.st[0] = 0.0f;
    if (m.st[0] > 10.0f) m.st[0] = 10.0f;
    return 0.0;
}

/* hh_biological.cpp:3266-3308 (connexin-36) and 3310-3350 (connexin-43), the same
 * steps: connexon turnover, phosphorylation toward the CaMKII drive (0: CaMKII is not
 * a supported modifier) and the cAMP drive in state[6], P_open from phosphorylation
 * and pH.  No current; gap junctions read state[0] and state[4]. */
template <bool kDef>
__device__ __forceinline__ double dp_connexin_current(DMod& m, DSeg& s, float dt) {
    (void)s;
    double synth_rate = ((kDef ? 0.0 : ((double)m.st[2])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[2])) : (double)0.001f;
    double degrad_rate = ((kDef ? 0.0 : ((double)m.st[3])) > 0.0f) ? (kDef ? 0.0 : ((double)m.st[3])) : (double)0.0005f;
    double pH = ((kDef ? 0.0 : ((double)m.st[5])) > 4.0f) ? (kDef ? 0.0 : ((double)m.st[5])) : (double)7.2f;
    m.st[0] = (float)((double)m.st[0] + (synth_rate - degrad_rate * (double)m.st[0]) * (double)dt / (double)3600000.0f);
    if (m.st[0] < 0.0f) m.st[0] = 0.0f;
    if (m.st[0] > 1.0f) m.st[0] = 1.0f;
    float camkii_act = 0.0f;
    double pka_drive = kDef ? 0.0 : (double)m.st[6];
    float p_target = (float)((double)(camkii_act * 0.6f) + pka_drive * (double)0.3f);
    m.st[1] = (float)((double)m.st[1] + ((double)p_target - (double)m.st[1]) * (double)dt / (double)5000.0f);
    if (m.st[1] < 0.0f) m.st[1] = 0.0f;
    if (m.st[1] > 1.0f) m.st[1] = 1.0f;
    float pH_factor = (pH < 6.8f) ? (float)((pH - (double)6.0f) / (double)0.8f) : 1.0f;
    if (pH_factor < 0.0f) pH_factor = 0.0f;
    double camkii_P_open = 1.0f - (double)m.st[1] * (double)0.5f;
    double pka_P_open = 1.0f + (double)m.st[1] * (double)0.3f;
    m.st[4] = (float)((camkii_P_open * (double)0.5f + pka_P_open * (double)0.5f) * (double)pH_factor);
    if (m.st[4] < 0.05f) m.st[4] = 0.05f;
    if (m.st[4] > 2.0f) m.st[4] = 2.0f;
    return 0.0;
}

/* hh_biological.cpp:725-733 (GLAST, glial glutamate transporter) through
 * glial_nt_uptake_current (modifier_helpers.h:418-454): 3 Na+ in, 1 K+ out, net +2,
 * glutamate taken from the segment's own neurotransmitter pool `glu`, which the
 * caller stores back. */
__device__ __forceinline__ double dp_glast_current(DMod& m, DSeg& s, float dt, float& glu) {
    const float k_m_rel = 10.0f, imax = 2.0f, rel_per_mm = 667.0f;
    const int na_in = 3, k_out = 1, net_charge = 2;
    float area = m.area;
    float NT = glu;
    if (NT < 0.0f) NT = 0.0f;
    float frac = NT / (NT + k_m_rel);
    float I = (float)((double)imax * (double)m.den * (double)area * (double)(1e-8f * 1e6f) * (double)frac);
    float volume = (float)s.vol;
    double cpm = FARADAY_CONST * (double)volume / 1000.0;
    float transport = (float)((double)(I * dt) / ((double)(float)net_charge * cpm));
    float nt_avail = NT / rel_per_mm;
    float na_avail = (float)((double)s.out[0] * (double)EXTRA_VOLUME_RATIO / (double)(float)na_in);
    if (transport > nt_avail) transport = nt_avail;
    if (transport > na_avail) transport = na_avail;
    if (k_out && (double)transport > (double)s.in[1]) transport = s.in[1];
    if (transport < 0.0f) transport = 0.0f;
    s.in[0] = (float)((double)s.in[0] + (double)((float)na_in * transport));
    s.out[0] = (float)((double)s.out[0] - (double)((float)na_in * transport / EXTRA_VOLUME_RATIO));
    s.in[1] = (float)((double)s.in[1] - (double)((float)k_out * transport));
    s.out[1] = (float)((double)s.out[1] + (double)((float)k_out * transport / EXTRA_VOLUME_RATIO));
    glu -= transport * rel_per_mm;
    if (glu < 0.0f) glu = 0.0f;
    dp_clamp_ions(s.in);
    dp_clamp_ions(s.out);
    return I;
}

/* kernel_dispatch.h:337-570 restricted to the supported types; 0 for unknown types
 * (the oracle's loader rejects them, so this branch is never taken). */
template <bool kDef>
__device__ __forceinline__ double dp_dispatch_t(uint8_t type, DMod& m, DSeg& s, float dt,
                                                float nt_glu, float nt_gaba, float nt_gly) {
    switch (type) {
        case 1: return dp_cav13_current<kDef>(m, s, dt);
        case 4: return 0.0f;
        case 7: return dp_nak_pump_current(m, s, dt);
        case 8: return dp_ampa_current<kDef>(m, s, dt, nt_glu, 1.0f);
        case 9: return dp_nmda_current<kDef>(m, s, dt, nt_glu, 1.0f);
        case 11: return dp_gabaa_current<kDef>(m, s, dt, nt_gaba, 1.0f);
        case 12: return dp_glycine_current<kDef>(m, s, dt, nt_gly, 1.0f);
        case 85: return dp_kv42_current<kDef>(m, s, dt);
        case 98: return dp_pmca_current<kDef>(m, s, dt);
        case 99: return dp_ncx_current(m, s, dt);
        case 100: return dp_kcc2_current<kDef>(m, s, dt);
        case 102: return dp_ca_buffer_current<kDef>(m, s, dt);
        case 103: return dp_sk_current<kDef>(m, s, dt);
        case 104: return dp_bk_current<kDef>(m, s, dt);
        case 105: return dp_nap_current<kDef>(m, s, dt);
        case 106: return dp_kir_current<kDef>(m, s, dt);
        case 107: return dp_k2p_current<kDef>(m, s, dt);
        case 112: return dp_kv7_current<kDef>(m, s, dt);
        case 123: return dp_kvdr_current<kDef>(m, s, dt);
        case 129: return dp_hcn1_current<kDef>(m, s, dt);
        case 133: return dp_nalcn_current<kDef>(m, s, dt);
        case 140: return dp_cav21_current(m, s, dt);
        case 141: return dp_nav_current<kDef>(m, s, dt, 0);
        case 142: return dp_nav_current<kDef>(m, s, dt, 1);
        case 150: return dp_kv31_current<kDef>(m, s, dt);
        case 200: return dp_cav31_current<kDef>(m, s, dt);
        case 86: return dp_ecb_synthesis_current<kDef>(m, s, dt);
        default: return 0.0f;
    }
}

// kernel_dispatch.h:337-570 restricted to the device-implemented types.  `defaults`:
// every parameter state of this modifier holds its default, so the specialisation
// with constant parameters runs.
__device__ __forceinline__ double dp_dispatch(uint8_t type, DMod& m, DSeg& s, float dt,
                                              float nt_glu, float nt_gaba, float nt_gly, bool defaults) {
    return defaults ? dp_dispatch_t<true>(type, m, s, dt, nt_glu, nt_gaba, nt_gly)
                    : dp_dispatch_t<false>(type, m, s, dt, nt_glu, nt_gaba, nt_gly);
}

__device__ __forceinline__ int dp_type_supported(uint8_t t) {
    switch (t) {
        case 1: case 4: case 7: case 8: case 9: case 11: case 12: case 85: case 98: case 99:
        case 100: case 102: case 103: case 104: case 105: case 106: case 107: case 112:
        case 123: case 129: case 133: case 140: case 141: case 142: case 150: case 200:
            return 1;
        default: return 0;
    }
}

/* kernel_dispatch.h:283-309 */
__device__ __forceinline__ int dp_is_ionotropic(uint8_t type) {
    return (type <= 2) || (type >= 8 && type <= 16) || type == 97 || type == 134 || type == 194;
}
__device__ __forceinline__ int dp_is_myelin_blocked(uint8_t type) {
    return dp_is_ionotropic(type) || type == 107 || type == 151 || type == 152 || type == 153 ||
           type == 133 || type == 85 || type == 202 || type == 203 || type == 204 || type == 150 ||
           type == 205 || type == 206 || type == 207 || type == 154 || type == 156 || type == 157 ||
           type == 159 || type == 112 || type == 123 || type == 121 || type == 105 || type == 195 ||
           type == 84 || type == 96 || type == 191 || type == 200 || type == 201 || type == 140 ||
           type == 158 || type == 168 || type == 129 || type == 130 || type == 131 || type == 132 ||
           type == 103 || type == 209 || type == 104;
}

}  // namespace bnc
