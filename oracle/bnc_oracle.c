/*
 * bnc_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; never part of the
 * product path): the reference's per-tick loop restated in C with FP32 state.
 *
 * Follows reference src/simulation_host.cpp:174-657 (core_run_tick_impl) step by
 * step, include/diffusion_kernel.h:41-364 (step 2.5), include/modifier_helpers.h
 * and include/kernel_dispatch.h for the helpers, with the same loop orders.  The
 * only intended difference from the reference is storage precision: V_m, ions,
 * modifier densities/states are float here (double in the reference); I_buffer
 * stays double.  Parity of this file against the reference itself is pinned by
 * tests/test_oracle_vs_reference.py (reference built by oracle/Makefile) and the
 * golden fixtures in tests/golden/.
 *
 * Supported subset (the loader rejects the rest with an error): modifier types
 * listed in bo_type_supported(), chemical synapses, pre-autoreceptors that are
 * bouton K/Na channels or release modulators, every stimulus kind of GpuStimulusData (current steps,
 * clamps, ramps, ion and ligand injections; bo_upload_stimuli), mechano stimuli
 * (bo_upload_mechano), no consolidation.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include "../include/bnc_abi.h"
#include "bo_modifiers.h"

typedef struct {
    uint32_t id, pre, post;
    uint8_t type;
    float weight, delay, pre_area, post_area;
    OMod pre_ar[8];
    uint8_t n_pre_ar;
    OMod post_r[8];
    uint8_t n_post_r;
    float p_rel, amt, cleft[15], facil, depr, tau_clear;
    uint8_t refractory;
    float RRP, RRP_max, RRP_rec, bouton_Ca, spine_Ca, spine_camkii, spine_calcineurin;
    float w_scale;   /* receptor density scale (1 in plain runs) */
} OSyn;

typedef struct {
    uint64_t arrival;
    float amount;
    uint8_t nt;
} ODelay;

typedef struct BoSim {
    uint32_t n, m, k;
    OSeg* seg;
    BncIntraConnection* conn;
    OSyn* syn;
    ODelay* delay;          /* k * 4 slots */
    uint64_t tick;
    BncCurrentStimulus* stim;
    uint32_t n_stim;
    /* the other stimulus kinds of GpuStimulusData (types.h:608-674), set by
       bo_upload_stimuli; injections are one-shot (simulation_host.cpp:304-306) */
    BncVoltageClamp vc[BNC_GPU_MAX_STIMULI];
    uint32_t n_vc;
    BncRampStimulus ramp[BNC_GPU_MAX_STIMULI];
    uint32_t n_ramp;
    BncIonInjection ion_inj[BNC_GPU_MAX_STIMULI];
    uint32_t n_ion_inj;
    BncLigandInjection lig_inj[BNC_GPU_MAX_STIMULI];
    uint32_t n_lig_inj;
    /* mechano stimuli for the next tick (simulation_host.cpp:211-230), one-shot */
    BncMechanoStimulus* mech;
    uint32_t n_mech;
    uint32_t* spike_count;  /* per segment, threshold -40 mV upward crossings */
    float nt_D[15];
    char err[256];
    /* release log (bo_set_release_log): every amount that enters a cleft */
    uint32_t *log_syn;
    uint64_t *log_tick;
    float *log_amt;
    uint8_t *log_slot;
    uint32_t log_cap, log_n;
    /* electrodiffusion options (bo_set_diffusion_mode): bit 0 residual-controlled FP64
     * Jacobi per convergence group (connected component), bit 1 the per-ion ledger */
    uint32_t dmode, jmax;
    double jtol;
    uint32_t *grp, n_grp;   /* group of each segment */
    uint8_t *gdone, *gmore; /* per group */
    double *vd, *vnd, *offdd, *rhsd, *dend, *phin;
    uint32_t jstats[4];     /* max V sweeps, max phi sweeps, V and phi group solves at the cap */
    double ledger[14];      /* per ion: rounding of the FP32 NP updates, bath exchange */
} BoSim;

static void bo_log_release(BoSim* S, uint32_t syn, uint64_t tick, float amt, uint8_t slot) {
    if (!S->log_syn) return;
    if (S->log_n < S->log_cap) {
        S->log_syn[S->log_n] = syn;
        S->log_tick[S->log_n] = tick;
        S->log_amt[S->log_n] = amt;
        S->log_slot[S->log_n] = slot;
    }
    S->log_n++;
}

/* ---- diffusion scratch (reference keeps these as function statics) ---- */
typedef struct {
    double *phi, *phi_new, *sigma, *diag, *goff_d;
    float *goff, *gdiag, *inp, *Vold, *Vnew, *offd;
    double *intra_acc, *extra_acc;
    float *ntd_in, *ntd_out, *atpd, *tempd, *txnd;
} BoScratch;

static BoScratch g_scr;
static uint32_t g_scr_n = 0, g_scr_m = 0;

static void scratch_reserve(uint32_t n, uint32_t m) {
    if (n <= g_scr_n && m <= g_scr_m) return;
    BoScratch* s = &g_scr;
    free(s->phi); free(s->phi_new); free(s->sigma); free(s->diag); free(s->goff_d);
    free(s->goff); free(s->gdiag); free(s->inp); free(s->Vold); free(s->Vnew); free(s->offd);
    free(s->intra_acc); free(s->extra_acc); free(s->ntd_in); free(s->ntd_out);
    free(s->atpd); free(s->tempd); free(s->txnd);
    size_t N = n + 1, M = m + 1;
    s->phi = calloc(N, 8); s->phi_new = calloc(N, 8); s->sigma = calloc(N, 8); s->diag = calloc(N, 8);
    s->goff_d = calloc(M, 8); s->goff = calloc(M, 4); s->gdiag = calloc(N, 4); s->inp = calloc(N, 4);
    s->Vold = calloc(N, 4); s->Vnew = calloc(N, 4); s->offd = calloc(N, 4);
    s->intra_acc = calloc(N * 7, 8); s->extra_acc = calloc(N * 7, 8);
    s->ntd_in = calloc(N * 15, 4); s->ntd_out = calloc(N * 15, 4);
    s->atpd = calloc(N, 4); s->tempd = calloc(N, 4); s->txnd = calloc(N, 4);
    g_scr_n = n; g_scr_m = m;
}

/* run_tick_common.h:216-231 */
static float bo_capacitance(const OSeg* s) {
    float area = bo_seg_area(s);
    float C_m = area * 0.01f;
    if (C_m < 1e-4f) C_m = 1e-4f;
    for (uint8_t j = 0; j < s->nmod && j < 16; j++) {
        if (s->mods[j].type == 4) {
            float gr = s->mods[j].st[0];
            if (gr <= 0.0f || gr >= 1.0f) gr = 0.6f;
            float factor = 100.0f * (1.0f / gr - 1.0f) / (1.0f / 0.6f - 1.0f);
            C_m /= factor;
            break;
        }
    }
    return C_m;
}

/* diffusion_kernel.h:108-113 */
static inline float bo_sg_bernoulli(float x) {
    if (fabsf(x) < 1e-3f) return 1.0f - 0.5f * x;
    if (x > 50.0f) return 0.0f;
    if (x < -50.0f) return -x;
    return x / (bo_exp(x) - 1.0f);
}

static const float NP_Z[7] = {1.0f, 1.0f, 2.0f, -1.0f, 2.0f, -1.0f, 1.0f};
static const float DIFF_C[7] = {1.33f, 1.96f, 0.22f, 2.03f, 0.10f, 0.0f, 9.31f};
static const float BATH_ION[7] = {140.0f, 3.0f, 1.2f, 130.0f, 1.0f, 0.0f, 4.0e-5f};

/* diffusion_kernel.h:41-104 */
static void bo_solve_phi_e(BoSim* S) {
    OSeg* sg = S->seg;
    uint32_t n = S->n, m = S->m;
    BoScratch* c = &g_scr;
    for (uint32_t i = 0; i < n; i++) c->phi[i] = 0.0;
    for (uint32_t i = 0; i < n; i++) {
        double s = 0.0;
        for (int ion = 0; ion < 7; ion++)
            s += NP_Z[ion] * NP_Z[ion] * DIFF_C[ion] * (double)sg[i].out[ion];
        c->sigma[i] = 3.612f * s;
        double g_bath = c->sigma[i] * bo_seg_area(&sg[i]) / 1.0f;
        c->diag[i] = g_bath;
    }
    for (uint32_t i = 0; i < m; i++) {
        uint32_t a = S->conn[i].segment_a, b = S->conn[i].segment_b;
        c->goff_d[i] = 0.0;
        if (a >= n || b >= n) continue;
        float r_min = sg[a].radius < sg[b].radius ? sg[a].radius : sg[b].radius;
        float area_conn = PI_F * r_min * r_min;
        if (area_conn < 1e-6f) area_conn = 1e-6f;
        float dist = (sg[a].length + sg[b].length) * 0.5f;
        if (dist < 0.1f) dist = 0.1f;
        double g = 0.5 * (c->sigma[a] + c->sigma[b]) * area_conn / dist;
        c->goff_d[i] = g;
        c->diag[a] += g;
        c->diag[b] += g;
    }
    if (S->dmode & 1u) {   /* residual-controlled: sweeps until every group converged */
        memset(S->gdone, 0, S->n_grp);
        uint32_t it = 0;
        while (it < S->jmax) {
            for (uint32_t i = 0; i < n; i++) c->phi_new[i] = 0.0;
            for (uint32_t i = 0; i < m; i++) {
                uint32_t a = S->conn[i].segment_a, b = S->conn[i].segment_b;
                if (a >= n || b >= n) continue;
                double g = c->goff_d[i];
                if (g <= 0.0) continue;
                c->phi_new[a] += g * c->phi[b];
                c->phi_new[b] += g * c->phi[a];
            }
            memset(S->gmore, 0, S->n_grp);
            for (uint32_t i = 0; i < n; i++) {
                if (S->gdone[S->grp[i]]) { S->phin[i] = c->phi[i]; continue; }
                double v = (c->diag[i] > 1e-9) ? (c->phi_new[i] - sg[i].ibuf) / c->diag[i] : 0.0;
                if (v > 10.0) v = 10.0;
                if (v < -10.0) v = -10.0;
                if (fabs(v - c->phi[i]) > S->jtol) S->gmore[S->grp[i]] = 1;
                S->phin[i] = v;
            }
            memcpy(c->phi, S->phin, (size_t)n * sizeof(double));
            it++;
            int any = 0;
            for (uint32_t g = 0; g < S->n_grp; g++)
                if (!S->gdone[g]) { if (S->gmore[g]) any = 1; else S->gdone[g] = 1; }
            if (!any) break;
        }
        if (it > S->jstats[1]) S->jstats[1] = it;
        for (uint32_t g = 0; g < S->n_grp; g++) S->jstats[3] += S->gdone[g] ? 0u : 1u;
        return;
    }
    for (int iter = 0; iter < 50; iter++) {
        for (uint32_t i = 0; i < n; i++) c->phi_new[i] = 0.0;
        for (uint32_t i = 0; i < m; i++) {
            uint32_t a = S->conn[i].segment_a, b = S->conn[i].segment_b;
            if (a >= n || b >= n) continue;
            double g = c->goff_d[i];
            if (g <= 0.0) continue;
            c->phi_new[a] += g * c->phi[b];
            c->phi_new[b] += g * c->phi[a];
        }
        for (uint32_t i = 0; i < n; i++) {
            c->phi[i] = (c->diag[i] > 1e-9) ? (c->phi_new[i] - sg[i].ibuf) / c->diag[i] : 0.0;
            if (c->phi[i] > 10.0) c->phi[i] = 10.0;
            if (c->phi[i] < -10.0) c->phi[i] = -10.0;
        }
    }
}

/* the volume the Nernst-Planck updates divide by: float, at least 1e-6 um^3 */
static float bo_vol_f(const OSeg* s) {
    float v = (float)bo_seg_volume(s);
    return v < 1e-6f ? 1e-6f : v;
}

/* diffusion_kernel.h:115-364 */
static void bo_diffusion(BoSim* S, float dt) {
    uint32_t n = S->n, m = S->m;
    if (m == 0) return;
    OSeg* sg = S->seg;
    BoScratch* c = &g_scr;
    for (size_t i = 0; i < (size_t)n * 7; i++) { c->extra_acc[i] = 0.0; c->intra_acc[i] = 0.0; }
    for (size_t i = 0; i < (size_t)n * 15; i++) { c->ntd_in[i] = 0.0f; c->ntd_out[i] = 0.0f; }
    for (uint32_t i = 0; i < n; i++) { c->atpd[i] = 0.0f; c->tempd[i] = 0.0f; c->txnd[i] = 0.0f; }
    bo_solve_phi_e(S);

    /* intracellular Nernst-Planck, 5 substeps (diffusion_kernel.h:152-238) */
    const float dt_sub = dt / 5;
    for (int sub = 0; sub < 5; sub++) {
        for (size_t i = 0; i < (size_t)n * 7; i++) c->intra_acc[i] = 0.0;
        for (uint32_t i = 0; i < n; i++) { c->gdiag[i] = 0.0f; c->inp[i] = 0.0f; }
        for (uint32_t i = 0; i < m; i++) {
            BncIntraConnection* cn = &S->conn[i];
            uint32_t a = cn->segment_a, b = cn->segment_b;
            if (a >= n || b >= n) continue;
            if (cn->is_intracellular == 0) continue;
            float r_min = sg[a].radius < sg[b].radius ? sg[a].radius : sg[b].radius;
            float area_conn = PI_F * r_min * r_min;
            if (area_conn < 1e-6f) area_conn = 1e-6f;
            float dist = (sg[a].length + sg[b].length) * 0.5f;
            if (dist < 0.1f) dist = 0.1f;
            float vol_a = (float)bo_seg_volume(&sg[a]);
            float vol_b = (float)bo_seg_volume(&sg[b]);
            if (vol_a < 1e-6f) vol_a = 1e-6f;
            if (vol_b < 1e-6f) vol_b = 1e-6f;
            float sigma_i = 0.0f;
            for (int ion = 0; ion < 7; ion++) {
                float C_bar = (float)(0.5f * ((double)sg[a].in[ion] + (double)sg[b].in[ion]));
                sigma_i += NP_Z[ion] * NP_Z[ion] * DIFF_C[ion] * C_bar;
            }
            float g_ax = 3.612f * sigma_i * area_conn / dist;
            c->goff[i] = g_ax;
            c->gdiag[a] += g_ax;
            c->gdiag[b] += g_ax;
            float dV = (float)(((double)sg[a].V + c->phi[a]) - ((double)sg[b].V + c->phi[b]));
            float I_np = 0.0f;
            for (int ion = 0; ion < 7; ion++) {
                float C_a = sg[a].in[ion];
                float C_b = sg[b].in[ion];
                float x = NP_Z[ion] * 0.03742f * dV;
                float flux = DIFF_C[ion] * area_conn * dt_sub / dist *
                             (C_a * bo_sg_bernoulli(-x) - C_b * bo_sg_bernoulli(x));
                c->intra_acc[a * 7 + ion] -= (double)flux / vol_a;
                c->intra_acc[b * 7 + ion] += (double)flux / vol_b;
                I_np += NP_Z[ion] * 96.485f * flux / dt_sub;
            }
            c->inp[a] += I_np - g_ax * dV;
            c->inp[b] -= I_np - g_ax * dV;
        }
        for (uint32_t i = 0; i < n; i++) { c->Vold[i] = sg[i].V; c->Vnew[i] = sg[i].V; }
        if (S->dmode & 1u) {   /* residual-controlled, FP64 iterates */
            for (uint32_t i = 0; i < n; i++) {
                float C_dt = bo_capacitance(&sg[i]) / dt_sub;
                if (C_dt < 1e-9f) C_dt = 1e-9f;
                S->vd[i] = (double)c->Vold[i];
                S->rhsd[i] = (double)C_dt * (double)c->Vold[i] + (double)c->inp[i];
                S->dend[i] = (double)C_dt + (double)c->gdiag[i];
            }
            memset(S->gdone, 0, S->n_grp);
            uint32_t it = 0;
            while (it < S->jmax) {
                for (uint32_t i = 0; i < n; i++) S->offdd[i] = 0.0;
                for (uint32_t i = 0; i < m; i++) {
                    BncIntraConnection* cn = &S->conn[i];
                    uint32_t a = cn->segment_a, b = cn->segment_b;
                    if (a >= n || b >= n) continue;
                    if (cn->is_intracellular == 0) continue;
                    S->offdd[a] += (double)c->goff[i] * S->vd[b];
                    S->offdd[b] += (double)c->goff[i] * S->vd[a];
                }
                memset(S->gmore, 0, S->n_grp);
                for (uint32_t i = 0; i < n; i++) {
                    if (S->gdone[S->grp[i]]) { S->vnd[i] = S->vd[i]; continue; }
                    const double nv = (S->rhsd[i] + S->offdd[i]) / S->dend[i];
                    if (fabs(nv - S->vd[i]) > S->jtol) S->gmore[S->grp[i]] = 1;
                    S->vnd[i] = nv;
                }
                double* tmp = S->vd; S->vd = S->vnd; S->vnd = tmp;
                it++;
                int any = 0;
                for (uint32_t g = 0; g < S->n_grp; g++)
                    if (!S->gdone[g]) { if (S->gmore[g]) any = 1; else S->gdone[g] = 1; }
                if (!any) break;
            }
            if (it > S->jstats[0]) S->jstats[0] = it;
            for (uint32_t g = 0; g < S->n_grp; g++) S->jstats[2] += S->gdone[g] ? 0u : 1u;
            for (uint32_t i = 0; i < n; i++) c->Vnew[i] = (float)S->vd[i];
        } else
        for (int iter = 0; iter < 50; iter++) {
            for (uint32_t i = 0; i < n; i++) c->offd[i] = 0.0f;
            for (uint32_t i = 0; i < m; i++) {
                BncIntraConnection* cn = &S->conn[i];
                uint32_t a = cn->segment_a, b = cn->segment_b;
                if (a >= n || b >= n) continue;
                if (cn->is_intracellular == 0) continue;
                c->offd[a] += c->goff[i] * c->Vnew[b];
                c->offd[b] += c->goff[i] * c->Vnew[a];
            }
            for (uint32_t i = 0; i < n; i++) {
                float C_dt = bo_capacitance(&sg[i]) / dt_sub;
                if (C_dt < 1e-9f) C_dt = 1e-9f;
                c->Vnew[i] = (C_dt * c->Vold[i] + c->inp[i] + c->offd[i]) / (C_dt + c->gdiag[i]);
            }
        }
        for (uint32_t i = 0; i < n; i++) sg[i].V = c->Vnew[i];
        for (uint32_t i = 0; i < n; i++)
            for (int ion = 0; ion < 7; ion++) {
                const bo_real old = sg[i].in[ion];
                const double acc = c->intra_acc[i * 7 + ion];
                sg[i].in[ion] = BO_ST((double)old + (double)(float)acc);
                if (S->dmode & 2u) S->ledger[ion] += ((double)sg[i].in[ion] - (double)old - acc) * (double)bo_vol_f(&sg[i]);
            }
    }

    /* extracellular Nernst-Planck, 5 substeps (diffusion_kernel.h:244-281) */
    for (int sub = 0; sub < 5; sub++) {
        for (size_t i = 0; i < (size_t)n * 7; i++) c->extra_acc[i] = 0.0;
        for (uint32_t i = 0; i < m; i++) {
            BncIntraConnection* cn = &S->conn[i];
            uint32_t a = cn->segment_a, b = cn->segment_b;
            if (a >= n || b >= n) continue;
            float r_min = sg[a].radius < sg[b].radius ? sg[a].radius : sg[b].radius;
            float area_conn = PI_F * r_min * r_min;
            if (area_conn < 1e-6f) area_conn = 1e-6f;
            float dist = (sg[a].length + sg[b].length) * 0.5f;
            if (dist < 0.1f) dist = 0.1f;
            float vol_a = (float)bo_seg_volume(&sg[a]);
            float vol_b = (float)bo_seg_volume(&sg[b]);
            if (vol_a < 1e-6f) vol_a = 1e-6f;
            if (vol_b < 1e-6f) vol_b = 1e-6f;
            for (int ion = 0; ion < 7; ion++) {
                double Ca = sg[a].out[ion];
                double Cb = sg[b].out[ion];
                double dphi = c->phi[a] - c->phi[b];
                float x = (float)(NP_Z[ion] * 0.03742f * dphi);
                double flux = DIFF_C[ion] * area_conn * dt_sub / dist *
                              (Ca * bo_sg_bernoulli(-x) - Cb * bo_sg_bernoulli(x));
                c->extra_acc[a * 7 + ion] -= flux / (vol_a * EXTRA_VOLUME_RATIO);
                c->extra_acc[b * 7 + ion] += flux / (vol_b * EXTRA_VOLUME_RATIO);
            }
        }
        for (uint32_t i = 0; i < n; i++)
            for (int ion = 0; ion < 7; ion++) {
                const bo_real old = sg[i].out[ion];
                const double acc = c->extra_acc[i * 7 + ion];
                sg[i].out[ion] = BO_ST((double)old + acc);
                if (S->dmode & 2u)
                    S->ledger[ion] += ((double)sg[i].out[ion] - (double)old - acc) *
                                      (double)(bo_vol_f(&sg[i]) * EXTRA_VOLUME_RATIO);
            }
    }

    /* NT / ATP / heat / transcription (diffusion_kernel.h:284-345) */
    for (uint32_t i = 0; i < m; i++) {
        BncIntraConnection* cn = &S->conn[i];
        uint32_t a = cn->segment_a, b = cn->segment_b;
        if (a >= n || b >= n) continue;
        float r_min = sg[a].radius < sg[b].radius ? sg[a].radius : sg[b].radius;
        float area_conn = PI_F * r_min * r_min;
        if (area_conn < 1e-6f) area_conn = 1e-6f;
        float dist = (sg[a].length + sg[b].length) * 0.5f;
        if (dist < 0.1f) dist = 0.1f;
        float vol_a = (float)bo_seg_volume(&sg[a]);
        float vol_b = (float)bo_seg_volume(&sg[b]);
        if (vol_a < 1e-6f) vol_a = 1e-6f;
        if (vol_b < 1e-6f) vol_b = 1e-6f;
        int extra_only = (cn->is_intracellular == 0);
        if (!extra_only) {
            for (int nt = 0; nt < 15; nt++) {
                float dC = sg[a].intra_nt[nt] - sg[b].intra_nt[nt];
                if (dC < 1e-12f && dC > -1e-12f) continue;
                float D = S->nt_D[nt];
                float flux = D * area_conn * dC * dt / dist;
                c->ntd_in[a * 15 + nt] -= flux / vol_a;
                c->ntd_in[b * 15 + nt] += flux / vol_b;
            }
        }
        for (int nt = 0; nt < 15; nt++) {
            float dC = sg[a].nt[nt] - sg[b].nt[nt];
            if (dC < 1e-12f && dC > -1e-12f) continue;
            float D = S->nt_D[nt];
            float flux = D * area_conn * dC * dt / dist;
            c->ntd_out[a * 15 + nt] -= flux / vol_a;
            c->ntd_out[b * 15 + nt] += flux / vol_b;
        }
        if (!extra_only) {
            float dATP = sg[a].atp - sg[b].atp;
            if (dATP > 1e-12f || dATP < -1e-12f) {
                float f = 0.14f * area_conn * dATP * dt / dist;
                c->atpd[a] -= f / vol_a;
                c->atpd[b] += f / vol_b;
            }
            float dT = sg[a].temp - sg[b].temp;
            if (dT > 0.001f || dT < -0.001f) {
                float f = 0.0014f * area_conn * dT * dt / dist;
                c->tempd[a] -= f / vol_a;
                c->tempd[b] += f / vol_b;
            }
            float dTx = sg[a].txn - sg[b].txn;
            if (dTx > 1e-9f || dTx < -1e-9f) {
                float f = 0.01f * area_conn * dTx * dt / dist;
                c->txnd[a] -= f / vol_a;
                c->txnd[b] += f / vol_b;
            }
        }
    }
    for (uint32_t i = 0; i < n; i++) {
        for (int ion = 0; ion < 7; ion++) {
            const bo_real old = sg[i].out[ion];
            double e = (double)sg[i].out[ion];
            e += (BATH_ION[ion] - e) * dt / 1.0f;
            if (e < 1e-9) e = 1e-9;
            if (e > 1000.0) e = 1000.0;
            sg[i].out[ion] = BO_ST(e);
            if (S->dmode & 2u)
                S->ledger[7 + ion] += ((double)sg[i].out[ion] - (double)old) *
                                      (double)(bo_vol_f(&sg[i]) * EXTRA_VOLUME_RATIO);
        }
        for (int nt = 0; nt < 15; nt++) {
            sg[i].intra_nt[nt] += c->ntd_in[i * 15 + nt];
            sg[i].nt[nt] += c->ntd_out[i * 15 + nt];
        }
        sg[i].atp += c->atpd[i];
        sg[i].temp += c->tempd[i];
        sg[i].txn += c->txnd[i];
    }
}

static int bo_has_myelin(const OSeg* s) {
    for (uint8_t j = 0; j < s->nmod; j++) if (s->mods[j].type == 4) return 1;
    return 0;
}

/* xorshift32 release draw, simulation_host.cpp:150-156 */
static inline float bo_xorshift32_rnd(uint32_t seed) {
    uint32_t x = seed;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    return (float)(x & 0x7FFFFFFFu) / (float)0x7FFFFFFFu;
}

/* Plugin modifiers (modifier_interface.h:38 register_modifier_current; a registered
 * function overrides the built-in model of its ID on the reference's CPU path,
 * kernel_dispatch.h:336-343).  The oracle's plugins see the FP32 state through this
 * view -- the same fields the device modifiers of the tested library see. */
typedef struct {
    float* V;
    float* in;        /* 7 intracellular ions */
    float* out;       /* 7 extracellular ions */
    float* atp;
    float area;       /* effective area, the reference's state[7] */
    double vol;
    float density;
    float* state;     /* 8 state words; state[7] holds the area */
    uint8_t type;
} BoPluginView;
typedef double (*BoPluginFn)(BoPluginView* v, float dt);
static BoPluginFn g_bo_plugins[128];

int bo_register_modifier(uint8_t type, BoPluginFn fn) {
#ifdef BO_FP64
    (void)fn;
    return -1;
#endif
    if (type >= 128) return -1;
    g_bo_plugins[type] = fn;
    return 0;
}

static double bo_call_modifier(uint8_t type, OMod* m, OSeg* s, float dt) {
#ifndef BO_FP64   /* the plugin view is the FP32 state; the FP64 build takes no plugins */
    if (type < 128 && g_bo_plugins[type]) {
        BoPluginView v;
        v.V = &s->V; v.in = s->in; v.out = s->out; v.atp = &s->atp;
        v.area = m->st[7]; v.vol = bo_seg_volume(s);
        v.density = m->density; v.state = m->st; v.type = type;
        return g_bo_plugins[type](&v, dt);
    }
#endif
    return bo_dispatch(type, m, s, dt);
}

/* (uint32_t)(V_m * 1000.0f) with V_m double, as x86-64 g++ evaluates it:
 * truncation to a 64-bit integer, then modulo 2^32 (simulation_host.cpp:438-440). */
static inline uint32_t bo_vm_seed_bits(bo_real V) {
    double x = (double)V * 1000.0f;
    return (uint32_t)(int64_t)x;
}

/* modifier_helpers.h:747-806 */
static float bo_bouton_gamma(uint8_t t) {
    switch (t) {
        case 156: return 10.0f;
        case 157: return 16.0f;
        case 123: return 11.0f;
        case 150: return 27.0f;
        case 112: return 7.0f;
        case 107: return 100.0f;
        case 141: return 20.7f;
        case 142: return 20.8f;
        default: return 0.0f;
    }
}

/* Release modulators of presynaptic autoreceptors (receptors_biological.cpp:428-509,
 * dispatched by kernel_dispatch.h:575-604): kind 1 Gi/o (state[0] relaxes to the
 * activation with tau 50 ms, factor 1 - 0.7 s0 scale), kind 2 Gs (tau 30 ms, factor
 * 1 + 0.5 s0 scale), kind 3 ionotropic (factor 1 + 0.3 activation scale), with
 * activation = nt / (nt + 0.5) of the cleft transmitter the type reads and scale =
 * density x effective_area_mod (state[7] if > 0, else 1).  Other types (the bouton
 * channels) take the dispatch's default, 1. */
static int bo_modulator_kind(uint8_t t, int* nt) {
    switch (t) {
        case 18: case 19: *nt = 3; return 1;   /* 5-HT1A, 5-HT1B: serotonin */
        case 22: *nt = 2; return 1;            /* D2: dopamine */
        case 27: *nt = 5; return 1;            /* A1: adenosine */
        case 29: case 30: *nt = 0; return 1;   /* mGluR2, mGluR3: glutamate */
        case 35: *nt = 6; return 1;            /* alpha2: noradrenaline */
        case 36: *nt = 9; return 1;            /* CB1: endocannabinoid */
        case 38: *nt = 8; return 1;            /* H3: histamine */
        case 44: *nt = 2; return 2;            /* D1: dopamine */
        case 46: *nt = 5; return 2;            /* A2A: adenosine */
        case 13: *nt = 4; return 3;            /* nicotinic: acetylcholine */
        default: *nt = 0; return 0;
    }
}

static float bo_release_modulator(OMod* m, const float* cleft, float dt) {
    int nt;
    const int kind = bo_modulator_kind(m->type, &nt);
    if (!kind) return 1.0f;
    const float c = cleft[nt];
    const float activation = c / (c + 0.5f);
    const float area = (m->st[7] > 0.0f) ? (float)m->st[7] : 1.0f;
    const double scale = (double)m->density * (double)area;
    if (kind == 3) return (float)(1.0f + (double)(0.3f * activation) * scale);
    const float tau = (kind == 1) ? 50.0f : 30.0f;
    m->st[0] = BO_ST((double)m->st[0] + ((double)activation - (double)m->st[0]) * (double)dt / (double)tau);
    if (kind == 1) return (float)(1.0f - (double)0.7f * (double)m->st[0] * scale);
    return (float)(1.0f + (double)0.5f * (double)m->st[0] * scale);
}

/* run_tick_common.h:114-122: the slow Ca2+/calmodulin gate of a gap junction */
static float bo_gj_cam_update(float m_slow, float ca_pre, float ca_post, float dt) {
    float ca_avg = 0.5f * (ca_pre + ca_post);
    float cam_act = (ca_avg * ca_avg) / (ca_avg * ca_avg + 0.0003f * 0.0003f);
    m_slow += (cam_act - m_slow) * dt / 100.0f;
    if (m_slow < 0.0f) m_slow = 0.0f;
    if (m_slow > 1.0f) m_slow = 1.0f;
    return m_slow;
}

/* run_tick_common.h:79-110: the junction's conductance (nS) from the connexins of both
 * segments (the density is the presynaptic segment's), Cx43's Vj gate and the slow gate */
static float bo_gj_g_eff(const OSeg* pre, const OSeg* post, float m_slow, float Vj) {
    float g_gap_ps = 0.0f;
    for (int cx = 0; cx < 2; cx++) {
        uint8_t cx_type = (cx == 0) ? 114 : 198;
        float gamma = (cx == 0) ? 14.0f : 100.0f;
        float density = 0.0f;
        float f = 1.0f;
        for (uint8_t j = 0; j < pre->nmod; j++)
            if (pre->mods[j].type == cx_type) {
                density = (float)pre->mods[j].density;
                f = (float)((double)f * ((double)pre->mods[j].st[0] * (double)pre->mods[j].st[4]));
            }
        for (uint8_t j = 0; j < post->nmod; j++)
            if (post->mods[j].type == cx_type)
                f = (float)((double)f * ((double)post->mods[j].st[0] * (double)post->mods[j].st[4]));
        if (cx == 1) {
            float vj_abs = Vj < 0.0f ? -Vj : Vj;
            float f_vj = (float)(1.0f / (1.0f + bo_exp((double)((vj_abs - 40.0f) / 5.0f))));
            f *= f_vj;
        }
        if (f < 0.01f) f = 0.01f;
        g_gap_ps += density * f * gamma;
    }
    return g_gap_ps * 1e-3f * (1.0f - m_slow);
}

static void bo_bouton_ca_step(const OSeg* pre, OSyn* syn, float dt) {
    float g_K = 0.0f, g_Na = 0.0f;
    for (uint8_t j = 0; j < syn->n_pre_ar; j++) {
        uint8_t t = syn->pre_ar[j].type;
        float g = (float)((double)syn->pre_ar[j].density * bo_bouton_gamma(t));
        if (t == 141 || t == 142) g_Na += g;
        else g_K += g;
    }
    float V_bouton = pre->V;
    if (g_K > 0.0f || g_Na > 0.0f) {
        float E_K = bo_nernst(pre->in[1], pre->out[1], 1.0f);
        float E_Na = bo_nernst(pre->in[0], pre->out[0], 1.0f);
        V_bouton = (float)((300.0f * (double)pre->V + g_K * E_K + g_Na * E_Na) / (300.0f + g_K + g_Na));
    }
    float cav21_dens = 0.0f, mm = 0.0f, h = 0.0f;
    for (uint8_t j = 0; j < pre->nmod; j++) {
        if (pre->mods[j].type == 140) {
            cav21_dens = pre->mods[j].density;
            float m_inf = cav21_m_inf(V_bouton);
            float h_inf = cav21_h_inf(V_bouton, syn->bouton_Ca * MM_TO_UM);
            mm = m_inf;
            h = (float)(h_inf + ((double)pre->mods[j].st[1] - h_inf) * bo_exp(-dt / 300.0f));
        }
    }
    float cav21_open = mm * mm * h;
    double P_single = bo_ghk_P(15.0f, 2.0f, GHK_CBAR_CA_MM);
    double flux = bo_ghk_div(V_bouton, syn->bouton_Ca, (double)pre->out[2]);
    double I_A = P_single * flux * (cav21_dens * syn->pre_area) * cav21_open;
    float I_Ca = (float)(I_A * A_TO_PA);
    syn->bouton_Ca = (float)(syn->bouton_Ca - I_Ca * dt * 1000.0f / (2.0f * FARADAY_CONST * 0.1f));
    syn->bouton_Ca += (0.0001f - syn->bouton_Ca) * dt / 5.0f;
    if (syn->bouton_Ca < 0.0f) syn->bouton_Ca = 0.0f;
}

/* modifier_helpers.h:808-817 */
static void bo_spine_ca_step(OSyn* syn, float I_syn, float dt) {
    float I_abs = I_syn < 0.0f ? -I_syn : I_syn;
    float I_Ca = I_abs * 0.1f;
    float influx = (float)(I_Ca * dt * 1000.0f / (2.0f * FARADAY_CONST * 0.05f * 100.0f));
    syn->spine_Ca += influx;
    syn->spine_Ca += (0.0001f - syn->spine_Ca) * dt / 50.0f;
    if (syn->spine_Ca < 0.0f) syn->spine_Ca = 0.0f;
}

/* modifier_helpers.h:819-833 */
static void bo_spine_plasticity_step(OSyn* syn, float dt) {
    float Ca_uM = syn->spine_Ca * MM_TO_UM;
    float Ca4 = Ca_uM * Ca_uM * Ca_uM * Ca_uM;
    float camkii_inf = Ca4 / (Ca4 + 1.0f + 1e-9f);
    syn->spine_camkii += (camkii_inf - syn->spine_camkii) * dt / 2000.0f;
    if (syn->spine_camkii < 0.0f) syn->spine_camkii = 0.0f;
    if (syn->spine_camkii > 1.0f) syn->spine_camkii = 1.0f;
    float Ca2 = Ca_uM * Ca_uM;
    float calcineurin_inf = Ca2 / (Ca2 + 0.05f * 0.05f + 1e-9f);
    syn->spine_calcineurin += (calcineurin_inf - syn->spine_calcineurin) * dt / 300.0f;
    if (syn->spine_calcineurin < 0.0f) syn->spine_calcineurin = 0.0f;
    if (syn->spine_calcineurin > 1.0f) syn->spine_calcineurin = 1.0f;
}

/* run_tick_common.h:199-206 */
static uint8_t bo_nt_from_receptor(uint8_t rt) {
    if (rt == 11 || rt == 17) return 1;
    if (rt == 12) return 7;
    if (rt == 14) return 3;
    if (rt == 13) return 4;
    if (rt == 44 || rt == 22) return 2;
    return 0;
}

static double bo_receptor(uint8_t rtype, OMod* m, OSeg* post, float dt, float scale) {
    switch (rtype) {
        case 8: return bo_ampa_current(m, post, dt, scale);
        case 9: return bo_nmda_current(m, post, dt, scale);
        case 11: return bo_gabaa_current(m, post, dt, scale);
        case 12: return bo_glycine_current(m, post, dt, scale);
        default: return bo_dispatch(rtype, m, post, dt);
    }
}

/* simulation_host.cpp:174-657 (mechano stimuli, steps 1, 2.5, 3, 4; no consolidation) */
static void bo_tick(BoSim* S, float dt) {
    uint64_t tick = S->tick++;
    OSeg* sg = S->seg;
    uint32_t n = S->n;
    /* expiry of current stimuli (:189-209) */
    {
        uint32_t w = 0;
        for (uint32_t r = 0; r < S->n_stim; r++) {
            BncCurrentStimulus st = S->stim[r];
            if (!(tick >= st.start_tick + (uint64_t)(st.duration_ms / dt))) S->stim[w++] = st;
        }
        S->n_stim = w;
        w = 0;
        for (uint32_t r = 0; r < S->n_vc; r++)
            if (!(tick >= S->vc[r].end_tick)) S->vc[w++] = S->vc[r];
        S->n_vc = w;
        w = 0;
        for (uint32_t r = 0; r < S->n_ramp; r++)
            if (!(tick >= S->ramp[r].end_tick)) S->ramp[w++] = S->ramp[r];
        S->n_ramp = w;
    }
    /* mechano stimuli (:211-230): the value into state[state_idx] of the first modifier
       of the type on the first segment with the id, in order, then cleared */
    for (uint32_t m = 0; m < S->n_mech; m++) {
        const BncMechanoStimulus* ms = &S->mech[m];
        for (uint32_t i = 0; i < n; i++) {
            if (sg[i].id != ms->segment_id) continue;
            for (uint8_t j = 0; j < sg[i].nmod; j++)
                if (sg[i].mods[j].type == ms->mod_type) {
                    if (ms->state_idx >= 0 && ms->state_idx < 8) sg[i].mods[j].st[ms->state_idx] = BO_ST(ms->value);
                    break;
                }
            break;
        }
    }
    S->n_mech = 0;
    /* step 1 (:234-303) */
    for (uint32_t i = 0; i < n; i++) {
        OSeg* s = &sg[i];
        double I_total = 0.0;
        int myel = bo_has_myelin(s);
        for (uint8_t j = 0; j < s->nmod; j++) {
            uint8_t type = s->mods[j].type;
            if (myel && type != 4 && bo_is_myelin_blocked(type)) continue;
            s->mods[j].st[7] = bo_seg_area(s);
            I_total += bo_call_modifier(type, &s->mods[j], s, dt);
        }
        for (uint32_t k = 0; k < S->n_stim; k++) {
            const BncCurrentStimulus* st = &S->stim[k];
            if (st->segment_id == s->id) {
                uint64_t dur_ticks = (uint64_t)(st->duration_ms / dt);
                if (tick >= st->start_tick && tick < st->start_tick + dur_ticks)
                    I_total += st->amplitude_pA;
            }
        }
        /* ramps (:261-276): amplitude interpolated in FP32 */
        for (uint32_t r = 0; r < S->n_ramp; r++) {
            const BncRampStimulus* rs = &S->ramp[r];
            if (rs->segment_id != s->id) continue;
            if (tick >= rs->start_tick && tick < rs->end_tick) {
                float frac = (rs->end_tick > rs->start_tick)
                    ? (float)(tick - rs->start_tick) / (float)(rs->end_tick - rs->start_tick)
                    : 1.0f;
                float amp = rs->start_pA + (rs->end_pA - rs->start_pA) * frac;
                I_total += amp;
            }
        }
        /* ion injections (:279-287), in upload order */
        for (uint32_t r = 0; r < S->n_ion_inj; r++) {
            const BncIonInjection* ij = &S->ion_inj[r];
            if (ij->segment_id != s->id || ij->ion_idx < 0 || ij->ion_idx >= 7) continue;
            bo_real* ions = ij->extracellular ? s->out : s->in;
            ions[ij->ion_idx] = BO_ST((double)ions[ij->ion_idx] + (double)ij->amount_mM);
        }
        /* ligand injections (:289-300) */
        for (uint32_t r = 0; r < S->n_lig_inj; r++) {
            const BncLigandInjection* lj = &S->lig_inj[r];
            if (lj->segment_id != s->id || lj->nt_idx < 0 || lj->nt_idx >= 15) continue;
            if (lj->intracellular) s->intra_nt[lj->nt_idx] += lj->amount;
            else s->nt[lj->nt_idx] += lj->amount;
        }
        s->ibuf = I_total;
    }
    S->n_ion_inj = 0;   /* one-shot (:304-306) */
    S->n_lig_inj = 0;
    /* step 2.5 */
    bo_diffusion(S, dt);
    /* step 3 (:322-593) */
    if (S->k > 0)
        for (uint32_t i = 0; i < n; i++)
            for (int q = 0; q < 15; q++) sg[i].nt[q] = 0.0f;
    for (uint32_t i = 0; i < n; i++)
        for (uint8_t j = 0; j < sg[i].nmod; j++)
            if (sg[i].mods[j].type == 9) sg[i].nt[0] = 1.0f;
    for (uint32_t i = 0; i < n; i++)
        for (uint8_t j = 0; j < sg[i].nmod; j++)
            if (sg[i].mods[j].type == 43) sg[i].nt[3] = 0.0f;
    /* glial segments (:351-355): the first 256 with a GLAST modifier */
    uint32_t glia[256];
    uint32_t n_glia = 0;
    for (uint32_t g = 0; g < n && n_glia < 256; g++)
        for (uint8_t j = 0; j < sg[g].nmod; j++)
            if (sg[g].mods[j].type == 147) { glia[n_glia++] = g; break; }
    for (uint32_t i = 0; i < S->k; i++) {
        OSyn* syn = &S->syn[i];
        if (syn->pre >= n || syn->post >= n) continue;
        OSeg* pre = &sg[syn->pre];
        OSeg* post = &sg[syn->post];
        if (syn->delay > 0.0f) {
            ODelay* slots = &S->delay[(size_t)i * 4];
            for (int q = 0; q < 4; q++) {
                if (slots[q].arrival == 0) continue;
                if (slots[q].arrival <= tick) {
                    syn->cleft[slots[q].nt] += slots[q].amount;
                    bo_log_release(S, i, tick, slots[q].amount, (uint8_t)q);
                    slots[q].arrival = 0;
                }
            }
        }
        /* electrical synapse or dendritic bridge (:373-402, run_tick_common.h:79-122) */
        if (syn->type == 1 || syn->type == 2) {
            float Vj = (float)((double)pre->V - (double)post->V);
            float m_slow = bo_gj_cam_update(syn->depr, (float)pre->in[2], (float)post->in[2], dt);
            syn->depr = m_slow;
            float g_eff = bo_gj_g_eff(pre, post, m_slow, Vj);
            float I_gap_raw = g_eff * Vj;
            if (syn->delay > 0.001f) {
                float I_filtered = syn->cleft[0];
                I_filtered += (I_gap_raw - I_filtered) * dt / syn->delay;
                syn->cleft[0] = I_filtered;
                pre->ibuf -= I_filtered;
                post->ibuf += I_filtered;
            } else {
                pre->ibuf -= I_gap_raw;
                post->ibuf += I_gap_raw;
            }
            continue;
        }
        /* rrp_do_recovery (kernel_dispatch.h:612-630); no CaMKII/calcineurin modifiers */
        if (!(syn->RRP_max <= 0.0f || syn->RRP >= syn->RRP_max)) {
            float ca_pre = pre->in[2];
            float ca_f = ca_pre / (0.0005f + ca_pre);
            float camkii = 0, calcn = 0;
            float priming = syn->RRP_rec + camkii * 0.02f + calcn * 0.01f;
            priming *= ca_f;
            float rec = (syn->RRP_max - syn->RRP) * priming * dt;
            syn->RRP += rec;
            if (syn->RRP > syn->RRP_max) syn->RRP = syn->RRP_max;
        }
        bo_bouton_ca_step(pre, syn, dt);
        if (syn->refractory == 0) {
            float Ca_uM = syn->bouton_Ca * MM_TO_UM;
            float ca_act = bo_pow(Ca_uM, 4.0f) / (bo_pow(Ca_uM, 4.0f) + bo_pow(10.0f, 4.0f));
            float p = syn->p_rel * ca_act;
            for (int j = 0; j < syn->n_pre_ar; j++) {
                syn->pre_ar[j].st[7] = syn->pre_area;
                p *= bo_release_modulator(&syn->pre_ar[j], syn->cleft, dt);
            }
            uint32_t seed = syn->id ^ ((uint32_t)tick) ^ bo_vm_seed_bits(pre->V);
            if (bo_xorshift32_rnd(seed) < p) {
                uint8_t nt_type = (syn->n_post_r > 0) ? bo_nt_from_receptor(syn->post_r[0].type) : 0;
                float release_amt;
                if (syn->RRP_max <= 0.0f) release_amt = syn->amt * p;
                else {
                    float avail = syn->amt;
                    if (avail > syn->RRP) avail = syn->RRP;
                    release_amt = avail * p;
                    syn->RRP -= release_amt;
                    if (syn->RRP < 0) syn->RRP = 0;
                }
                uint64_t delay_ticks = (syn->delay <= 0.0f || dt <= 0.0f) ? 0
                                       : (uint64_t)((syn->delay / dt) + 0.5f);
                if (delay_ticks > 0) {
                    ODelay* slots = &S->delay[(size_t)i * 4];
                    for (int q = 0; q < 4; q++) {
                        if (slots[q].arrival == 0) {
                            slots[q].arrival = tick + delay_ticks;
                            slots[q].amount = release_amt;
                            slots[q].nt = nt_type;
                            break;
                        }
                    }
                } else {
                    syn->cleft[nt_type] += release_amt;
                    bo_log_release(S, i, tick, release_amt, 4);
                }
                syn->refractory = (uint8_t)(uint32_t)(20.0f / dt + 0.5f);
            }
        }
        for (int q = 0; q < 15; q++) post->nt[q] += syn->cleft[q];
        /* glial capture (:467-487): a share of glutamate, glycine and GABA goes to the
           glial segment nearest in z, rate-limited by the clearance time constant */
        if (n_glia > 0) {
            for (int kk = 0; kk < 3; kk++) {
                int q = (kk == 0) ? 0 : (kk == 1) ? 7 : 1;
                if (syn->cleft[q] <= 0.0f) continue;
                float best_dz = 1e30f;
                uint32_t best_g = glia[0];
                for (uint32_t gi = 0; gi < n_glia; gi++) {
                    float dz = fabsf(sg[glia[gi]].pz - post->pz);
                    if (dz < best_dz) { best_dz = dz; best_g = glia[gi]; }
                }
                float tau = (syn->tau_clear > 0.0f) ? syn->tau_clear : 5.0f;
                float capture = (float)((double)syn->cleft[q] * (1.0 - bo_exp(-dt / tau)));
                sg[best_g].nt[q] += capture;
                syn->cleft[q] -= capture;
            }
        }
        int myel_post = bo_has_myelin(post);
        float I_syn = 0.0f;
        for (int j = 0; j < syn->n_post_r; j++) {
            uint8_t rtype = syn->post_r[j].type;
            if (myel_post && bo_is_ionotropic(rtype)) continue;
            syn->post_r[j].st[7] = syn->post_area;
            I_syn = (float)(I_syn + bo_receptor(rtype, &syn->post_r[j], post, dt, syn->w_scale));
        }
        post->ibuf += I_syn;
        bo_spine_ca_step(syn, I_syn, dt);
        for (int q = 0; q < 15; q++) {
            if ((q == 0 || q == 7 || q == 1) && n_glia > 0) continue;   /* the glia took their share */
            syn->cleft[q] *= bo_exp(-dt / syn->tau_clear);
            if (syn->cleft[q] < 0.0f) syn->cleft[q] = 0.0f;
        }
        float Ca_uM = syn->spine_Ca * 1000.0f;
        float Ca_sq = Ca_uM * Ca_uM;
        float tau_theta = 300000.0f;
        syn->facil += (Ca_sq - syn->facil) * dt / tau_theta;
        if (syn->facil < 0.0f) syn->facil = 0.0f;
        syn->depr = syn->facil + 0.01f;
        bo_spine_plasticity_step(syn, dt);
        float camkii_act = syn->spine_camkii;
        float calcineurin_act = syn->spine_calcineurin;
        int inhib = 0;
        for (int j = 0; j < syn->n_post_r; j++) {
            uint8_t rt = syn->post_r[j].type;
            if (rt == 11 || rt == 17 || rt == 12) { inhib = 1; break; }
        }
        float dw = 0.0f;
        if (camkii_act > 0.0f) dw += 0.0003f * camkii_act * dt;
        float pp1_active = 0.5f;
        if (calcineurin_act > 0.0f) dw -= 0.0001f * calcineurin_act * pp1_active * dt;
        if (inhib) dw = -dw;
        syn->weight += dw;
        if (syn->weight != syn->weight) syn->weight = 0.5f;
        if (syn->facil != syn->facil) syn->facil = 0.0f;
        if (syn->depr != syn->depr) syn->depr = 0.01f;
        if (syn->weight < 0.01f) syn->weight = 0.01f;
        if (syn->weight > 10.0f) syn->weight = 10.0f;
        /* eCB retrograde signalling (:578-589): the post segment's first eCB-synthesis
           modifier puts 2-AG into this cleft and loses a tenth of it */
        for (uint8_t j = 0; j < post->nmod; j++) {
            if (post->mods[j].type != 86) continue;
            float ecb = (float)post->mods[j].st[0];
            if (ecb > 0.0f) {
                syn->cleft[9] += ecb * 0.1f * dt;
                post->mods[j].st[0] = BO_ST((double)post->mods[j].st[0] * (double)0.9f);
            }
            break;
        }
        if (syn->refractory > 0) syn->refractory--;
    }
    /* step 4 (:596-649) */
    for (uint32_t i = 0; i < n; i++) {
        OSeg* s = &sg[i];
        if (s->ibuf != s->ibuf) s->ibuf = 0.0f;
        if (s->ibuf > 10000.0f) s->ibuf = 10000.0f;
        if (s->ibuf < -10000.0f) s->ibuf = -10000.0f;
        float C_m = bo_capacitance(s);
        float prev_V = s->V;
        float dV = (float)(s->ibuf / C_m * dt);
        if (dV > 50.0f) dV = 50.0f;
        if (dV < -50.0f) dV = -50.0f;
        s->V = BO_ST((double)s->V + dV);
        if (S->spike_count && prev_V <= -40.0f && s->V > -40.0f) S->spike_count[i]++;
        s->ibuf = 0.0f;
        /* voltage clamps (:633-643): the last active clamp of the segment wins */
        for (uint32_t v = 0; v < S->n_vc; v++) {
            const BncVoltageClamp* vc = &S->vc[v];
            if (vc->segment_id == s->id && tick >= vc->start_tick && tick < vc->end_tick) s->V = vc->target_mV;
        }
        if (s->V != s->V) { s->V = -65.0f; }
        else {
            if (s->V < -120.0f) s->V = -120.0f;
            if (s->V > 150.0f) s->V = 150.0f;
        }
    }
}

/* ------------------------------------------------------------------ */
/* C API used by the tests (through ctypes)                            */
/* ------------------------------------------------------------------ */

static void load_mod(OMod* o, const BncModifier* m) {
    o->type = m->type;
    o->active_vars = m->active_vars;
    o->density = BO_ST(m->density);
    for (int k = 0; k < 8; k++) o->st[k] = BO_ST(m->state[k]);
}

/* rrp_apply_protein_mapping (kernel_dispatch.h:651-663): protein levels of genes
   UNC13A (42), SYT1 (40) and CPLX1 (44) (types.h:357-361) set RRP_max, the release
   probability and RRP recovery. */
void bo_protein_mapping(const float* protein_level, float* rrp_max, float* p_rel, float* rrp_rec) {
    float munc13 = protein_level[42];
    *rrp_max = 10.0f + munc13 * 40.0f;
    float syt1 = protein_level[40];
    *p_rel = 0.3f + syt1 * 0.7f;
    float cplx1 = protein_level[44];
    *rrp_rec = 0.02f + munc13 * 0.08f - cplx1 * 0.01f;
    if (*rrp_rec < 0.005f) *rrp_rec = 0.005f;
    if (*rrp_rec > 0.2f) *rrp_rec = 0.2f;
}

BoSim* bo_create(const BncBionData* d, const BncCurrentStimulus* stim, uint32_t n_stim,
                 char* err, int errlen) {
    BoSim* S = calloc(1, sizeof(BoSim));
    S->n = d->num_segments;
    S->m = d->num_connections;
    S->k = d->num_synapses;
    S->seg = calloc(S->n ? S->n : 1, sizeof(OSeg));
    S->conn = calloc(S->m ? S->m : 1, sizeof(BncIntraConnection));
    S->syn = calloc(S->k ? S->k : 1, sizeof(OSyn));
    S->delay = calloc((size_t)(S->k ? S->k : 1) * 4, sizeof(ODelay));
    S->stim = calloc(n_stim ? n_stim : 1, sizeof(BncCurrentStimulus));
    S->spike_count = calloc(S->n ? S->n : 1, sizeof(uint32_t));
    if (n_stim) memcpy(S->stim, stim, n_stim * sizeof(BncCurrentStimulus));
    S->n_stim = n_stim;
    const float mass[15] = {147.0f, 103.0f, 153.0f, 176.0f, 146.0f, 267.0f, 169.0f, 75.0f, 111.0f,
                            348.0f, 507.0f, 232.0f, 24.0f, 162.0f, 0.0f};
    for (int q = 0; q < 15; q++) {
        float ms = mass[q];
        if (ms < 1.0f) ms = 1.0f;
        S->nt_D[q] = 1.33f * bo_powf(23.0f / ms, 1.0f / 3.0f);   /* powf: types.h:442 */
    }
    for (uint32_t i = 0; i < S->n; i++) {
        const BncSegment* a = &d->segments[i];
        OSeg* s = &S->seg[i];
        s->id = a->id;
        s->type = a->segment_type;
        s->length = a->length;
        s->radius = a->radius;
        s->px = a->position.x; s->py = a->position.y; s->pz = a->position.z;
        s->V = BO_ST(a->V_m);
        for (int q = 0; q < 8; q++) { s->in[q] = BO_ST(a->intra_ions[q]); s->out[q] = BO_ST(a->extra_ions[q]); }
        for (int q = 0; q < 15; q++) { s->intra_nt[q] = a->intra_nt[q]; s->nt[q] = a->neurotransmitter[q]; }
        s->atp = a->ATP_level;
        s->temp = a->temperature;
        s->txn = a->transcription_signal;
        s->ibuf = a->I_buffer;
        s->nmod = a->modifier_count > 32 ? 32 : a->modifier_count;
        for (uint8_t j = 0; j < s->nmod; j++) {
            const uint8_t mt = a->modifiers[j].type;
            if (!bo_type_supported(mt) && !(mt < 128 && g_bo_plugins[mt])) {
                snprintf(err, errlen, "segment %u: modifier type %u not supported", i, a->modifiers[j].type);
                return S;
            }
            load_mod(&s->mods[j], &a->modifiers[j]);
        }
    }
    if (S->m) memcpy(S->conn, d->connections, S->m * sizeof(BncIntraConnection));
    for (uint32_t i = 0; i < S->k; i++) {
        const BncSynapse* a = &d->synapses[i];
        OSyn* y = &S->syn[i];
        if (a->type > 2) {
            snprintf(err, errlen, "synapse %u: type %u", i, (unsigned)a->type);
            return S;
        }
        y->id = a->id; y->pre = a->pre_segment; y->post = a->post_segment; y->type = a->type;
        y->weight = a->weight; y->delay = a->delay; y->pre_area = a->pre_area; y->post_area = a->post_area;
        y->n_pre_ar = a->pre_autoreceptor_count > 8 ? 8 : a->pre_autoreceptor_count;
        for (int j = 0; j < y->n_pre_ar; j++) load_mod(&y->pre_ar[j], &a->pre_autoreceptors[j]);
        y->n_post_r = a->post_receptor_count > 8 ? 8 : a->post_receptor_count;
        for (int j = 0; j < y->n_post_r; j++) load_mod(&y->post_r[j], &a->post_receptors[j]);
        y->p_rel = a->release_probability; y->amt = a->release_amount;
        for (int q = 0; q < 15; q++) y->cleft[q] = a->cleft_neurotransmitter[q];
        y->facil = a->facilitation; y->depr = a->depression; y->tau_clear = a->tau_clearance;
        y->refractory = a->refractory;
        y->RRP = a->RRP; y->RRP_max = a->RRP_max; y->RRP_rec = a->RRP_recovery;
        y->bouton_Ca = a->bouton_Ca; y->spine_Ca = a->spine_Ca;
        y->spine_camkii = a->spine_camkii; y->spine_calcineurin = a->spine_calcineurin;
        y->w_scale = 1.0f;
        /* nucleus protein levels of the presynaptic neuron (gpu_backend_cuda.cu:275-289:
           synapses with id 0 skipped, nucleus at the position of the pre segment's
           neuron_id); with fixed protein levels the per-tick mapping is the same every
           tick, so it is applied here once */
        if (d->nuclei && d->num_nuclei && a->id != 0 && a->pre_segment < d->num_segments) {
            uint32_t nid = d->segments[a->pre_segment].neuron_id;
            if (nid < d->num_nuclei)
                bo_protein_mapping((const float*)((const uint8_t*)d->nuclei + (size_t)nid * 500 + 244),
                                   &y->RRP_max, &y->p_rel, &y->RRP_rec);
        }
    }
    scratch_reserve(S->n, S->m);
    return S;
}

/* gpu_backend_upload_stimuli (gpu_backend_cuda.cu:242-248): every list is replaced by
   the uploaded one; the injections apply at the next tick, once. */
/* The mechano argument of core_run_tick for the next tick (replaces any pending). */
void bo_upload_mechano(BoSim* S, const BncMechanoStimulus* ms, uint32_t n) {
    free(S->mech);
    S->mech = n ? malloc((size_t)n * sizeof(BncMechanoStimulus)) : NULL;
    if (n) memcpy(S->mech, ms, (size_t)n * sizeof(BncMechanoStimulus));
    S->n_mech = n;
}

void bo_upload_stimuli(BoSim* S, const BncGpuStimulusData* src) {
    uint32_t nc = src->current_stim_count < BNC_GPU_MAX_STIMULI ? src->current_stim_count : BNC_GPU_MAX_STIMULI;
    free(S->stim);
    S->stim = calloc(nc ? nc : 1, sizeof(BncCurrentStimulus));
    if (nc) memcpy(S->stim, src->current_stim, nc * sizeof(BncCurrentStimulus));
    S->n_stim = nc;
#define BO_TAKE(dst, n, srcarr, cnt) do { \
        n = (cnt) < BNC_GPU_MAX_STIMULI ? (cnt) : BNC_GPU_MAX_STIMULI; \
        memcpy(dst, srcarr, (size_t)(n) * sizeof(dst[0])); } while (0)
    BO_TAKE(S->vc, S->n_vc, src->vclamps, src->vclamp_count);
    BO_TAKE(S->ramp, S->n_ramp, src->ramps, src->ramp_count);
    BO_TAKE(S->ion_inj, S->n_ion_inj, src->ion_inj, src->ion_inj_count);
    BO_TAKE(S->lig_inj, S->n_lig_inj, src->lig_inj, src->lig_inj_count);
#undef BO_TAKE
}

void bo_destroy(BoSim* S) {
    if (!S) return;
    free(S->seg); free(S->conn); free(S->syn); free(S->delay); free(S->stim); free(S->spike_count); free(S->mech);
    free(S->grp); free(S->gdone); free(S->gmore);
    free(S->vd); free(S->vnd); free(S->offdd); free(S->rhsd); free(S->dend); free(S->phin);
    free(S);
}

static uint32_t bo_find(uint32_t* p, uint32_t x) {
    while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
    return x;
}

/* Options of step 2.5 beside the reference's fixed 50 sweeps: flags bit 0 makes the
 * phi_e and V_m solves iterate in FP64 until no value of a convergence group (a
 * connected component over all valid connections) changes by more than tol in a
 * sweep, at most max_sweeps sweeps; bit 1 keeps the per-ion FP64 ledger. */
void bo_set_diffusion_mode(BoSim* S, uint32_t flags, double tol, uint32_t max_sweeps) {
    const uint32_t n = S->n;
    S->dmode = flags;
    S->jtol = tol;
    S->jmax = max_sweeps;
    if (!S->grp) {
        uint32_t* p = malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
        for (uint32_t i = 0; i < n; i++) p[i] = i;
        for (uint32_t c = 0; c < S->m; c++) {
            uint32_t a = S->conn[c].segment_a, b = S->conn[c].segment_b;
            if (a >= n || b >= n) continue;
            a = bo_find(p, a); b = bo_find(p, b);
            if (a != b) { if (a < b) p[b] = a; else p[a] = b; }
        }
        S->grp = malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
        uint32_t* id = malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
        for (uint32_t i = 0; i < n; i++) id[i] = UINT32_MAX;
        S->n_grp = 0;
        for (uint32_t i = 0; i < n; i++) {
            uint32_t r = bo_find(p, i);
            if (id[r] == UINT32_MAX) id[r] = S->n_grp++;
            S->grp[i] = id[r];
        }
        free(p); free(id);
        size_t G = S->n_grp ? S->n_grp : 1, N = n ? n : 1;
        S->gdone = calloc(G, 1); S->gmore = calloc(G, 1);
        S->vd = calloc(N, 8); S->vnd = calloc(N, 8); S->offdd = calloc(N, 8);
        S->rhsd = calloc(N, 8); S->dend = calloc(N, 8); S->phin = calloc(N, 8);
    }
}

void bo_diffusion_stats(BoSim* S, uint32_t* stats4, double* ledger14, int reset) {
    memcpy(stats4, S->jstats, sizeof(S->jstats));
    memcpy(ledger14, S->ledger, sizeof(S->ledger));
    if (reset) { memset(S->jstats, 0, sizeof(S->jstats)); memset(S->ledger, 0, sizeof(S->ledger)); }
}

void bo_run(BoSim* S, uint32_t ticks, float dt) {
    for (uint32_t t = 0; t < ticks; t++) bo_tick(S, dt);
}

/* The reference's batch loop (daemon_main.cpp:250-258): after each tick the loop
 * increments the tick counter once more, so tick k runs with counter stride * k. */
void bo_run_stride(BoSim* S, uint32_t ticks, float dt, uint32_t stride) {
    for (uint32_t t = 0; t < ticks; t++) {
        bo_tick(S, dt);
        S->tick += stride - 1;
    }
}

/* Runs `ticks` ticks and records V of the listed segments after every tick
 * into out[t * n_rec + r]. */
void bo_run_trace(BoSim* S, uint32_t ticks, float dt, const uint32_t* rec, uint32_t n_rec, float* out) {
    for (uint32_t t = 0; t < ticks; t++) {
        bo_tick(S, dt);
        for (uint32_t r = 0; r < n_rec; r++) out[(size_t)t * n_rec + r] = S->seg[rec[r]].V;
    }
}

uint64_t bo_tick_count(const BoSim* S) { return S->tick; }

/* Starts a release log into caller-owned arrays of `cap` entries (NULL stops it);
 * returns nothing.  bo_release_log_count gives the entries seen (may exceed cap). */
void bo_set_release_log(BoSim* S, uint32_t* syn, uint64_t* tick, float* amt, uint8_t* slot, uint32_t cap) {
    S->log_syn = syn; S->log_tick = tick; S->log_amt = amt; S->log_slot = slot;
    S->log_cap = cap; S->log_n = 0;
}
uint32_t bo_release_log_count(const BoSim* S) { return S->log_n; }

/* Field export.  field: 0 V, 1 in[ion], 2 out[ion], 3 atp, 4 temp, 5 txn,
 * 6 intra_nt[idx], 7 nt[idx], 8 modifier state (idx = slot*8+k), 9 spike count. */
static double bo_seg_value(const BoSim* S, uint32_t i, int field, int idx) {
    const OSeg* s = &S->seg[i];
    switch (field) {
        case 0: return s->V;
        case 1: return s->in[idx];
        case 2: return s->out[idx];
        case 3: return s->atp;
        case 4: return s->temp;
        case 5: return s->txn;
        case 6: return s->intra_nt[idx];
        case 7: return s->nt[idx];
        case 8: return ((idx >> 3) < s->nmod) ? s->mods[idx >> 3].st[idx & 7] : 0.0;
        case 9: return (double)S->spike_count[i];
        case 10: return bo_vol_f(s);   /* the volume the Nernst-Planck updates divide by */
    }
    return 0.0;
}
void bo_get_seg_field(const BoSim* S, int field, int idx, float* out) {
    for (uint32_t i = 0; i < S->n; i++) out[i] = (float)bo_seg_value(S, i, field, idx);
}
/* the same at the storage precision of the build (exact for the FP64 build) */
void bo_get_seg_field64(const BoSim* S, int field, int idx, double* out) {
    for (uint32_t i = 0; i < S->n; i++) out[i] = bo_seg_value(S, i, field, idx);
}

/* Synapse export.  field: 0 bouton_Ca, 1 spine_Ca, 2 weight, 3 refractory,
 * 4 cleft[idx], 5 receptor state (idx = j*8+k), 6 facilitation, 7 spine_camkii,
 * 8 spine_calcineurin, 9 RRP, 10 depression. */
static double bo_syn_value(const BoSim* S, uint32_t i, int field, int idx) {
    const OSyn* y = &S->syn[i];
    switch (field) {
        case 0: return y->bouton_Ca;
        case 1: return y->spine_Ca;
        case 2: return y->weight;
        case 3: return (double)y->refractory;
        case 4: return y->cleft[idx];
        case 5: return ((idx >> 3) < y->n_post_r) ? y->post_r[idx >> 3].st[idx & 7] : 0.0;
        case 6: return y->facil;
        case 7: return y->spine_camkii;
        case 8: return y->spine_calcineurin;
        case 9: return y->RRP;
        case 10: return y->depr;
        case 11: return ((idx >> 3) < y->n_pre_ar) ? y->pre_ar[idx >> 3].st[idx & 7] : 0.0;
    }
    return 0.0;
}
void bo_get_syn_field(const BoSim* S, int field, int idx, float* out) {
    for (uint32_t i = 0; i < S->k; i++) out[i] = (float)bo_syn_value(S, i, field, idx);
}
void bo_get_syn_field64(const BoSim* S, int field, int idx, double* out) {
    for (uint32_t i = 0; i < S->k; i++) out[i] = bo_syn_value(S, i, field, idx);
}

/* Receptor density scale per synapse (the differentiable synaptic weight;
 * 1.0 reproduces the reference). */
void bo_set_syn_scale(BoSim* S, const float* scale) {
    for (uint32_t i = 0; i < S->k; i++) S->syn[i].w_scale = scale[i];
}

/* Elementary functions, exported for the accuracy tests. */
double bo_exp_d(double x) { return bo_exp(x); }
float bo_expf_f(float x) { return bo_expf(x); }
double bo_log_d(double x) { return bo_log(x); }
double bo_pow_d(double x, double y) { return bo_pow(x, y); }
float bo_xorshift_f(uint32_t seed) { return bo_xorshift32_rnd(seed); }
uint32_t bo_seed_bits(double V) { return bo_vm_seed_bits((bo_real)V); }

/* Known-answer hooks for the tests (reference tests/test_ghk_reference.cpp,
 * tests/test_reference_ionics.cpp): the oracle's GHK flux terms and Nernst
 * potential, and the physical constants they use (types.h:400-402). */
double bo_ghk_mono_d(double V, double c_in, double c_out) { return bo_ghk_mono(V, c_in, c_out); }
double bo_ghk_div_d(double V, double c_in, double c_out) { return bo_ghk_div(V, c_in, c_out); }
double bo_ghk_anion_d(double V, double c_in, double c_out) { return bo_ghk_anion(V, c_in, c_out); }
float bo_nernst_f(float intra, float extra, float valence) { return bo_nernst(intra, extra, valence); }
double bo_const(int which) {
    switch (which) {
        case 0: return FARADAY_CONST;
        case 1: return GAS_CONST;
        case 2: return CELSIUS_37;
        default: return 0.0;
    }
}
