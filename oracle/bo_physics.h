/*
 * bo_physics.h -- CPU oracle (test infrastructure only): channel, pump,
 * receptor and synapse physics of the reference, restated in C with FP32 state.
 *
 * Rule used throughout: every value the reference keeps in state (V_m, ion
 * concentrations, modifier density/state, which are double there) is stored
 * here as float and read back promoted to double exactly where the reference
 * reads a double, so each expression has the reference's operand types; every
 * store rounds to float.  Locals keep the reference's types.  exp/log/pow come
 * from bo_math.h.  Citations are reference file:line.
 */
#ifndef BO_PHYSICS_H
#define BO_PHYSICS_H
#include <stdint.h>
#include "bo_math.h"

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

/* State storage type.  The oracle proper stores FP32 state (bo_real = float).
 * Built with -DBO_FP64 the same source stores double, as the reference's Segment
 * and Modifier do (types.h:451-500), and with -DBO_LIBM it calls the C library's
 * elementary functions as the reference does: that build (oracle/liboracle64.so)
 * must then reproduce the reference's own core_run_tick, which pins this
 * restatement's operation order independently of FP32 rounding. */
#ifdef BO_FP64
typedef double bo_real;
#else
typedef float bo_real;
#endif
#define BO_ST(x) ((bo_real)(x))

typedef struct {
    uint8_t type;
    uint8_t active_vars;
    bo_real density;
    bo_real st[8];
} OMod;

typedef struct {
    uint32_t id;
    uint8_t type;
    float length, radius;
    float px, py, pz;
    bo_real V;
    bo_real in[8], out[8];
    float intra_nt[15], nt[15];
    float atp, temp, txn;
    double ibuf;
    uint8_t nmod;
    OMod mods[32];
} OSeg;

#define SV ((double)s->V)
#define SIN(i) ((double)s->in[i])
#define SOUT(i) ((double)s->out[i])
#define MST(k) ((double)m->st[k])
#define MDEN ((double)m->density)

/* ---- helpers: reference include/run_tick_common.h, include/modifier_helpers.h ---- */

/* run_tick_common.h:209-214 */
static inline float bo_seg_area(const OSeg* s) {
    return (s->type == 1 || s->type == 3 || s->type == 4)
        ? 4.0f * PI_F * s->radius * s->radius
        : 2.0f * PI_F * s->radius * s->length;
}
/* run_tick_common.h:262-266 */
static inline double bo_seg_volume(const OSeg* s) {
    if (s->type == 1 || s->type == 3 || s->type == 4)
        return (4.0 / 3.0) * PI_F * (double)s->radius * (double)s->radius * (double)s->radius;
    return PI_F * (double)s->radius * (double)s->radius * (double)s->length;
}
/* modifier_helpers.h:109-112 */
static inline float bo_eff_area(const OMod* m, const OSeg* s) {
    if (MST(7) > 0.0f) return (float)MST(7);
    return bo_seg_area(s);
}
/* modifier_helpers.h:1117-1121: arrays are double in the reference */
static inline void bo_clamp_ions(bo_real* arr) {
    for (int i = 0; i < 7; i++)
        if ((double)arr[i] < 1e-9) arr[i] = BO_ST(1e-9);
}
/* run_tick_common.h:274-312 */
static inline double bo_ghk_mono(double V, double c_in, double c_out) {
    double V_norm = FARADAY_CONST * V * 0.001 / (GAS_CONST * CELSIUS_37);
    if (fabs(V_norm) < 1e-6) return FARADAY_CONST * (c_in - c_out);
    double k = FARADAY_CONST / (GAS_CONST * CELSIUS_37);
    if (V_norm > 20.0) return k * FARADAY_CONST * V * 0.001 * c_in;
    if (V_norm < -20.0) return k * FARADAY_CONST * V * 0.001 * c_out;
    return k * FARADAY_CONST * V * 0.001 * (c_in - c_out * bo_exp(-V_norm)) / (1.0 - bo_exp(-V_norm));
}
static inline double bo_ghk_div(double V, double c_in, double c_out) {
    double V_norm = 2.0 * FARADAY_CONST * V * 0.001 / (GAS_CONST * CELSIUS_37);
    if (fabs(V_norm) < 1e-6) return 2.0 * FARADAY_CONST * (c_in - c_out);
    double k = 4.0 * FARADAY_CONST / (GAS_CONST * CELSIUS_37);
    if (V_norm > 20.0) return k * FARADAY_CONST * V * 0.001 * c_in;
    if (V_norm < -20.0) return k * FARADAY_CONST * V * 0.001 * c_out;
    return k * FARADAY_CONST * V * 0.001 * (c_in - c_out * bo_exp(-V_norm)) / (1.0 - bo_exp(-V_norm));
}
static inline double bo_ghk_anion(double V, double c_in, double c_out) {
    double V_norm = FARADAY_CONST * V * 0.001 / (GAS_CONST * CELSIUS_37);
    if (fabs(V_norm) < 1e-6) return FARADAY_CONST * (c_out - c_in);
    double k = FARADAY_CONST / (GAS_CONST * CELSIUS_37);
    if (V_norm > 20.0) return k * FARADAY_CONST * V * 0.001 * c_out;
    if (V_norm < -20.0) return k * FARADAY_CONST * V * 0.001 * c_in;
    return k * FARADAY_CONST * V * 0.001 * (c_out - c_in * bo_exp(-V_norm)) / (1.0 - bo_exp(-V_norm));
}
/* modifier_helpers.h:48-54 */
static inline double bo_ghk_P(float gamma_pS, float z, float cbar_mM) {
    double gamma_S = gamma_pS * PS_TO_S;
    double z2F2 = z * z * FARADAY_CONST * FARADAY_CONST;
    double RT = GAS_CONST * CELSIUS_37;
    return gamma_S * RT / (z2F2 * cbar_mM);
}
/* modifier_helpers.h:58-66 */
static inline void bo_nalcn_partial_P(float gamma_pS, double* P_Na, double* P_K, double* P_Ca) {
    const double fNa = 1.3, fK = 1.2, fCa = 0.5;
    double w = fNa * GHK_CBAR_NA_MM + fK * GHK_CBAR_K_MM + fCa * 4.0 * GHK_CBAR_CA_MM;
    *P_Na = bo_ghk_P((float)(gamma_pS * fNa * GHK_CBAR_NA_MM / w), 1.0f, GHK_CBAR_NA_MM);
    *P_K = bo_ghk_P((float)(gamma_pS * fK * GHK_CBAR_K_MM / w), 1.0f, GHK_CBAR_K_MM);
    *P_Ca = bo_ghk_P((float)(gamma_pS * fCa * 4.0 * GHK_CBAR_CA_MM / w), 2.0f, GHK_CBAR_CA_MM);
}
/* modifier_helpers.h:69-76 */
static inline void bo_partial_P(float gamma_pS, float fNa, float fK, float fCa,
                                double* P_Na, double* P_K, double* P_Ca) {
    double w = fNa * GHK_CBAR_NA_MM + fK * GHK_CBAR_K_MM + fCa * 4.0 * GHK_CBAR_CA_MM;
    *P_Na = bo_ghk_P((float)(gamma_pS * fNa * GHK_CBAR_NA_MM / w), 1.0f, GHK_CBAR_NA_MM);
    *P_K = bo_ghk_P((float)(gamma_pS * fK * GHK_CBAR_K_MM / w), 1.0f, GHK_CBAR_K_MM);
    *P_Ca = bo_ghk_P((float)(gamma_pS * fCa * 4.0 * GHK_CBAR_CA_MM / w), 2.0f, GHK_CBAR_CA_MM);
}
/* modifier_helpers.h:30-34 */
static inline float bo_nernst(float intra, float extra, float valence) {
    if (intra < 1e-9f) intra = 1e-9f;
    if (extra < 1e-9f) extra = 1e-9f;
    return (float)((GAS_CONST * CELSIUS_37) / (valence * FARADAY_CONST) * bo_log(extra / intra) * 1000.0f);
}
/* modifier_helpers.h:132-135 */
static inline float bo_vtrap(float x, float y) {
    if (fabsf(x / y) < 1e-6f) return y * (1.0f - x / (2.0f * y));
    return x / (1.0f - bo_exp(-x / y));
}
/* modifier_helpers.h:1090-1095 */
static inline float bo_bz_act(float V, float vh, float k) { return 1.0f / (1.0f + bo_exp(-(V - vh) / k)); }
static inline float bo_bz_inact(float V, float vh, float k) { return 1.0f / (1.0f + bo_exp((V - vh) / k)); }

/* ---- gating helpers (modifier_helpers.h:145-215, 264-271, 468-472, 689-702, 1008-1018, 882-892, 909-913, 954-967, 1137-1170, 1188-1210) ---- */
static inline float nav16_am(float V) { return 0.182f * bo_vtrap(V + 43.0f, 6.0f); }
static inline float nav16_bm(float V) { return 0.124f * bo_vtrap(-(V + 43.0f), 6.0f); }
static inline float nav16_ah(float V) { return 0.024f * bo_vtrap(V + 50.0f, 5.0f); }
static inline float nav16_bh(float V) { return 0.0091f * bo_vtrap(-(V + 75.0f), 5.0f); }
static inline float nav16_m_inf(float V) { float a = nav16_am(V), b = nav16_bm(V); return a / (a + b); }
static inline float nav16_m_tau(float V) { return 1.0f / (nav16_am(V) + nav16_bm(V)); }
static inline float nav16_h_inf(float V) { return 1.0f / (1.0f + bo_exp((V + 72.0f) / 6.2f)); }
static inline float nav16_h_tau(float V) { return 1.0f / (nav16_ah(V) + nav16_bh(V)); }
static inline float nav12_am(float V) { return 0.182f * bo_vtrap(V + 23.0f, 6.0f); }
static inline float nav12_bm(float V) { return 0.124f * bo_vtrap(-(V + 23.0f), 6.0f); }
static inline float nav12_ah(float V) { return 0.024f * bo_vtrap(V + 41.5f, 5.0f); }
static inline float nav12_bh(float V) { return 0.0091f * bo_vtrap(-(V + 66.5f), 5.0f); }
static inline float nav12_m_inf(float V) { float a = nav12_am(V), b = nav12_bm(V); return a / (a + b); }
static inline float nav12_m_tau(float V) { return 1.0f / (nav12_am(V) + nav12_bm(V)); }
static inline float nav12_h_inf(float V) { return 1.0f / (1.0f + bo_exp((V + 63.5f) / 6.2f)); }
static inline float nav12_h_tau(float V) { return 1.0f / (nav12_ah(V) + nav12_bh(V)); }
static inline float cav21_m_inf(float V) { return 1.0f / (1.0f + bo_exp(-(V - -15.0f) / (6.0f + 1e-6f))); }
static inline float cav21_h_inf(float V, float Ca_uM) {
    float h = 1.0f / (1.0f + bo_exp((V - -50.0f) / 8.0f));
    h *= 1.0f / (1.0f + Ca_uM / 3.0f);
    return h;
}
static inline float kv42_h_tau(float V) {
    return 15.0f + (170.0f - 15.0f) / (1.0f + bo_exp((V - -60.0f) / 8.0f));
}
static inline float cav31_h_tau(float V) {
    return 25.0f + (250.0f - 25.0f) / (1.0f + bo_exp((V - -65.0f) / 8.0f));
}
static inline float cav31_m_tau(float V) {
    float dv = V - -20.0f;
    float g = bo_exp(-(dv * dv) / (2.0f * 22.0f * 22.0f));
    return 1.25f + (15.0f - 1.25f) * g;
}
static inline float kv_dr_m_tau(float V, float V_half) {
    float tau = 14.6f * bo_exp(-(V - V_half) / 30.1f);
    if (tau < 0.3f) tau = 0.3f;
    if (tau > 200.0f) tau = 200.0f;
    return tau;
}
static inline float kir_f_open(float V) {
    float Vn = (float)(FARADAY_CONST * V * 0.001f / (GAS_CONST * CELSIUS_37));
    float Kd_Mg = 0.3f * bo_exp(-0.6f * 2.0f * Vn);
    float mg_block = 0.5f / Kd_Mg;
    float Kd_spm = 0.0775f * bo_exp(-0.5f * 4.0f * Vn);
    float r = 0.001f / Kd_spm;
    float spm_block = 0.0f, rk = r;
    for (int k = 0; k < 3; k++) { spm_block += rk; rk *= r; }
    return 1.0f / (1.0f + mg_block + spm_block);
}
static inline float sk_p_inf(float Ca) {
    if (Ca < 1e-9f) Ca = 1e-9f;
    float r = 0.0004f / Ca;
    return 1.0f / (1.0f + bo_pow(r, 4.0f));
}
static inline float bk_ha_po(float V_mV, float Ca) {
    float Vn = (float)(FARADAY_CONST * V_mV * MV_TO_V / (GAS_CONST * CELSIUS_37));
    float J = 0.104f * bo_exp(0.55f * Vn);
    float L = 3.7e-8f * bo_exp(0.30f * Vn);
    if (Ca < 0.0f) Ca = 0.0f;
    float K = Ca / 0.044f;
    float o = 1.0f + K * 23.0f + J * 32.0f + J * K * 23.0f * 32.0f * 3.7f;
    float c = 1.0f + K + J + J * K * 3.7f;
    o *= o; o *= o;
    c *= c; c *= c;
    float num = L * o;
    return num / (num + c);
}
static inline float nak_pump_vnorm(float V_mV, float Na_i, float K_o, float ATP_level, float K_m_Na, float K_m_K) {
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
    float a2 = 60.0f * bo_exp(0.5f * eta);
    float b2 = 6.0f * bo_exp(-(1.0f - 0.5f) * eta);
    float a1 = 200.0f * f_Na * f_ATP;
    float a3 = 200.0f * f_K;
    float a4 = 60.0f;
    float denom = a3 / a1 + (b2 + a3) / a2 + 1.0f + a3 / a4;
    float turnover = a3 / denom;
    float k3 = 200.0f;
    float v_max = k3 / (k3 / 200.0f + 1.0f + k3 / 60.0f);
    return turnover / v_max;
}
static inline float ncx_flux_norm(float V_mV, float Na_i, float Na_o, float Ca_i, float Ca_o) {
    float V_v = V_mV * MV_TO_V;
    float FRT = (float)(FARADAY_CONST / (GAS_CONST * CELSIUS_37));
    float e_eta = bo_exp(0.35f * FRT * V_v);
    float e_eta1 = bo_exp((0.35f - 1.0f) * FRT * V_v);
    float Na_i3 = Na_i * Na_i * Na_i;
    float Na_o3 = Na_o * Na_o * Na_o;
    float fwd = e_eta1 * Na_o3 * Ca_i;
    float rev = e_eta * Na_i3 * Ca_o;
    float denom = 1.0f + 0.27f * e_eta1;
    float ca_ratio = 0.000125f / Ca_i;
    float Allo = 1.0f / (1.0f + ca_ratio * ca_ratio);
    return Allo * (fwd - rev) / (denom * 530.2f);
}

#endif
