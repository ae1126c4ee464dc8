// tile.cu -- the tile kernel of a tick and the tick launcher.
//
// One tick of the reference (simulation_host.cpp:174-657) is two launches:
//
//  k_tile (one CTA per tile of whole neurons, state resident in shared memory)
//    step 1   modifier currents: items grouped into phases (each phase holds at most
//             one modifier per segment, phases follow every segment's slot order) and
//             by type within a phase, so warps run one channel model at a time;
//             stimuli; I_buffer.
//    step 2.5 electrodiffusion (diffusion_kernel.h:115-364): phi_e Jacobi, 5 intra
//             Scharfetter-Gummel substeps with a 50-sweep Jacobi V_m solve, 5 extra
//             substeps, NT/ATP/heat/transcription Fick, bath relaxation.  Each warp
//             owns whole components, so sweeps need only __syncwarp.  Every sum is a
//             gather over the segment's incident connections in connection order,
//             which is the order of the reference's scatter loops.
//    output   state, I_buffer and the presynaptic record (V, Ca_out, Cav2.1 gate).
//
//  k_synapse (one thread per postsynaptic segment)
//    step 3   its incoming synapses in original order (post-segment CSR, no
//             atomics): delays, RRP, bouton Ca2+, the xorshift32 release draw,
//             NT transfer, receptor currents, spine Ca2+, clearance, plasticity.
//    step 4   membrane update fused in: I clamp, C_m, dV clamp, spike count, clamps.
#define BNC_MATH_OUTLINE 1   // 26 channel models in one kernel: keep exp/log out of line
#include <cuda_runtime.h>
#include "net.h"
#include "physics.cuh"

namespace bnc {

// state indices each modifier type updates every tick (read + write)
__constant__ uint8_t c_dyn_mask[256];
// state indices each type reads as parameters (default when 0)
__constant__ uint8_t c_par_mask[256];

__device__ __constant__ float kNpZ[7] = {1.0f, 1.0f, 2.0f, -1.0f, 2.0f, -1.0f, 1.0f};
__device__ __constant__ float kDiffC[7] = {1.33f, 1.96f, 0.22f, 2.03f, 0.10f, 0.0f, 9.31f};
__device__ __constant__ float kBathIon[7] = {140.0f, 3.0f, 1.2f, 130.0f, 1.0f, 0.0f, 4.0e-5f};
__device__ float gNtD[15];   // Stokes-Einstein NT diffusion coefficients, set by k_init_tables

// diffusion_kernel.h:108-113
__device__ __forceinline__ float sg_bernoulli(float x) {
    if (fabsf(x) < 1e-3f) return 1.0f - 0.5f * x;
    if (x > 50.0f) return 0.0f;
    if (x < -50.0f) return -x;
    return x / (dm_expf(x) - 1.0f);
}

struct TileSmem {
    // whole kernel
    double *itot, *vol;
    float *V, *in, *out, *atp, *c21d, *c21h, *area, *cm;
    uint16_t *incoff;
    // step 1 only: per-segment GHK factors
    double *gA1, *ge1, *gD1, *gA2, *ge2, *gD2;
    float *gV;
    uint8_t *gm1, *gm2;
    // step 2.5 only (aliases the step-1 region)
    double *phiA, *phiB, *sig;
    float *nb, *gd, *rhs, *den, *vnA, *vnB;
    // per edge
    double *ed;
    float *gax, *dve, *fl, *ie;
    uint16_t *ea, *eb, *inc;
    uint8_t *ei, *es;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline size_t tile_layout(uint32_t S, uint32_t E, unsigned char* base, TileSmem* t) {
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align16(off + bytes); return base ? base + o : nullptr; };
    const size_t Ee = E ? E : 1;
    unsigned char* p;
    p = take(8 * (size_t)S); if (t) t->itot = (double*)p;
    p = take(8 * (size_t)S); if (t) t->vol = (double*)p;
    p = take(4 * (size_t)S); if (t) t->V = (float*)p;
    p = take(4 * 7 * (size_t)S); if (t) t->in = (float*)p;
    p = take(4 * 7 * (size_t)S); if (t) t->out = (float*)p;
    p = take(4 * (size_t)S); if (t) t->atp = (float*)p;
    p = take(4 * (size_t)S); if (t) t->c21d = (float*)p;
    p = take(4 * (size_t)S); if (t) t->c21h = (float*)p;
    p = take(4 * (size_t)S); if (t) t->area = (float*)p;
    p = take(4 * (size_t)S); if (t) t->cm = (float*)p;
    p = take(2 * ((size_t)S + 1)); if (t) t->incoff = (uint16_t*)p;
    // union region: step 1 (GHK factors) and step 2.5 (solver temporaries) never overlap in time
    const size_t u0 = off;
    p = take(8 * (size_t)S); if (t) t->gA1 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->ge1 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->gD1 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->gA2 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->ge2 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->gD2 = (double*)p;
    p = take(4 * (size_t)S); if (t) t->gV = (float*)p;
    p = take((size_t)S); if (t) t->gm1 = (uint8_t*)p;
    p = take((size_t)S); if (t) t->gm2 = (uint8_t*)p;
    const size_t u1 = off;
    off = u0;
    p = take(8 * (size_t)S); if (t) t->phiA = (double*)p;
    p = take(8 * (size_t)S); if (t) t->phiB = (double*)p;
    p = take(8 * (size_t)S); if (t) t->sig = (double*)p;
    p = take(4 * (size_t)S); if (t) t->nb = (float*)p;
    p = take(4 * (size_t)S); if (t) t->gd = (float*)p;
    p = take(4 * (size_t)S); if (t) t->rhs = (float*)p;
    p = take(4 * (size_t)S); if (t) t->den = (float*)p;
    p = take(4 * (size_t)S); if (t) t->vnA = (float*)p;
    p = take(4 * (size_t)S); if (t) t->vnB = (float*)p;
    if (off < u1) off = u1;
    p = take(8 * Ee); if (t) t->ed = (double*)p;
    p = take(4 * Ee); if (t) t->gax = (float*)p;
    p = take(4 * Ee); if (t) t->dve = (float*)p;
    p = take(4 * Ee); if (t) t->fl = (float*)p;
    p = take(4 * Ee); if (t) t->ie = (float*)p;
    p = take(2 * Ee); if (t) t->ea = (uint16_t*)p;
    p = take(2 * Ee); if (t) t->eb = (uint16_t*)p;
    p = take(2 * 2 * Ee); if (t) t->inc = (uint16_t*)p;
    p = take(Ee); if (t) t->ei = (uint8_t*)p;
    p = take(Ee); if (t) t->es = (uint8_t*)p;
    return off;
}

size_t tile_smem_bytes(uint32_t max_segs, uint32_t max_edges) {
    return tile_layout(max_segs, max_edges, nullptr, nullptr);
}

// One Fick pass over a warp's components for a float field held in t.nb
// (diffusion_kernel.h:284-345): per-edge flux, then per-segment gather.  Returns the
// per-segment delta through `out_delta` (written in place into t.nb as value + delta).
// kGradStrict: the reference's ATP/heat/transcription test "d > thr || d < -thr"
// (diffusion_kernel.h:323-341); otherwise the NT test "skip if -thr < d < thr" (:301,312).
template <bool kIntraOnly, bool kGradStrict>
__device__ __forceinline__ void fick_pass(const TileSmem& t, const NetDev& d, uint32_t e0, int ws, int we, int es,
                                          int ee, int lane, float D, float thresh, float dt) {
    for (int e = es + lane; e < ee; e += 32) {
        t.es[e] = 1;
        if (kIntraOnly && !t.ei[e]) continue;
        float dC = t.nb[t.ea[e]] - t.nb[t.eb[e]];
        if (kGradStrict) { if (!(dC > thresh || dC < -thresh)) continue; }
        else if (dC < thresh && dC > -thresh) continue;
        t.fl[e] = D * d.e_area[e0 + e] * dC * dt / d.e_dist[e0 + e];
        t.es[e] = 0;
    }
    __syncwarp();
    // the gather reads only edge fluxes and the segment's own value: update in place
    for (int i = ws + lane; i < we; i += 32) {
        float vf = (float)t.vol[i];
        if (vf < 1e-6f) vf = 1e-6f;
        float acc = 0.0f;
        for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
            uint16_t ent = t.inc[k];
            int e = ent & 0x7FFF;
            if (t.es[e]) continue;
            if (ent & 0x8000) acc += t.fl[e] / vf; else acc -= t.fl[e] / vf;
        }
        t.nb[i] = t.nb[i] + acc;
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kTileThreads)
k_tile(NetDev d, float dt, unsigned long long tick, uint32_t S, uint32_t E) {
    extern __shared__ __align__(16) unsigned char smem[];
    TileSmem t;
    tile_layout(S, E, smem, &t);
    const int tid = threadIdx.x;
    const int nth = blockDim.x;
    const uint32_t tile = blockIdx.x;
    const uint32_t N = d.n_seg;
    if (d.clock) tick = d.clock[0];
    const uint32_t s0 = d.tile_seg_beg[tile];
    const int ns = (int)(d.tile_seg_beg[tile + 1] - s0);
    const uint32_t e0 = d.tile_edge_beg[tile];
    const int ne = (int)(d.tile_edge_beg[tile + 1] - e0);
    const uint32_t inc0 = d.inc_off[s0];

    // ---- load tile state ----
    for (int i = tid; i < ns; i += nth) {
        uint32_t g = s0 + i;
        t.V[i] = d.V[g];
#pragma unroll
        for (int q = 0; q < 7; q++) {
            t.in[q * S + i] = d.ion_in[(size_t)q * N + g];
            t.out[q * S + i] = d.ion_out[(size_t)q * N + g];
        }
        t.atp[i] = d.atp[g];
        t.area[i] = d.area[g];
        t.vol[i] = d.vol[g];
        t.cm[i] = d.cm[g];
        t.itot[i] = 0.0;
        float2 c = d.cav21_static[g];
        t.c21d[i] = c.x;
        t.c21h[i] = c.y;
        t.incoff[i] = (uint16_t)(d.inc_off[g] - inc0);
    }
    if (tid == 0) t.incoff[ns] = (uint16_t)(d.inc_off[s0 + ns] - inc0);
    for (int e = tid; e < ne; e += nth) {
        t.ea[e] = d.e_a[e0 + e];
        t.eb[e] = d.e_b[e0 + e];
        t.ei[e] = d.e_intra[e0 + e];
    }
    const int ninc = (int)(d.inc_off[s0 + ns] - inc0);
    for (int k = tid; k < ninc; k += nth) t.inc[k] = d.inc[inc0 + k];
    for (int i = tid; i < ns; i += nth) {   // per-segment GHK factors for step 1
        GhkCache c;
        ghk_cache_fill(c, t.V[i]);
        t.gV[i] = c.Vc; t.gm1[i] = c.m1; t.gm2[i] = c.m2;
        t.gA1[i] = c.A1; t.ge1[i] = c.e1; t.gD1[i] = c.D1;
        t.gA2[i] = c.A2; t.ge2[i] = c.e2; t.gD2[i] = c.D2;
    }
    __syncthreads();

    // ---- step 1: modifier currents (simulation_host.cpp:234-303) ----
    const uint32_t P = d.n_phases;
    const uint32_t NI = d.n_items;
    for (uint32_t p = 0; p < P; p++) {
        const uint32_t b = d.phase_off[(size_t)tile * (P + 1) + p];
        const uint32_t e = d.phase_off[(size_t)tile * (P + 1) + p + 1];
        for (uint32_t q = b + tid; q < e; q += nth) {
            const uint32_t meta = d.it_meta[q];
            const int ls = (int)(meta & 0xFFFFu);
            const uint8_t type = (uint8_t)((meta >> 16) & 0xFFu);
            const uint8_t fl = (uint8_t)(meta >> 24);
            DSeg s;
            s.V = t.V[ls];
#pragma unroll
            for (int k = 0; k < 7; k++) { s.in[k] = t.in[k * S + ls]; s.out[k] = t.out[k * S + ls]; }
            s.atp = t.atp[ls];
            s.area = t.area[ls];
            s.vol = t.vol[ls];
            s.gc.Vc = t.gV[ls]; s.gc.m1 = t.gm1[ls]; s.gc.m2 = t.gm2[ls];
            s.gc.A1 = t.gA1[ls]; s.gc.e1 = t.ge1[ls]; s.gc.D1 = t.gD1[ls];
            s.gc.A2 = t.gA2[ls]; s.gc.e2 = t.ge2[ls]; s.gc.D2 = t.gD2[ls];
            DMod m;
            m.den = d.it_den[q];
            m.area = s.area;
            m.av = (fl & 2) ? (uint8_t)((fl >> 2) & 7) : (uint8_t)0;
            uint32_t rm = c_dyn_mask[type] | ((fl & 1) ? c_par_mask[type] : 0u);
            if (fl & 2) rm |= (1u << m.av) & 0x7Fu;
#pragma unroll
            for (int k = 0; k < 7; k++) m.st[k] = ((rm >> k) & 1u) ? d.it_st[(size_t)k * NI + q] : 0.0f;
            float glu = 0.0f, gaba = 0.0f, gly = 0.0f;
            if (type == 8 || type == 9) glu = d.nt[s0 + ls];
            else if (type == 11) gaba = d.nt[(size_t)1 * N + s0 + ls];
            else if (type == 12) gly = d.nt[(size_t)7 * N + s0 + ls];
            double I = dp_dispatch(type, m, s, dt, glu, gaba, gly, (fl & 3) == 0);
            if (s.V != t.V[ls]) {   // a sodium channel clamped V to +-200 mV
                GhkCache c;
                ghk_cache_fill(c, s.V);
                t.gV[ls] = c.Vc; t.gm1[ls] = c.m1; t.gm2[ls] = c.m2;
                t.gA1[ls] = c.A1; t.ge1[ls] = c.e1; t.gD1[ls] = c.D1;
                t.gA2[ls] = c.A2; t.ge2[ls] = c.e2; t.gD2[ls] = c.D2;
            }
            t.V[ls] = s.V;
#pragma unroll
            for (int k = 0; k < 7; k++) { t.in[k * S + ls] = s.in[k]; t.out[k * S + ls] = s.out[k]; }
            t.atp[ls] = s.atp;
            t.itot[ls] += I;
            const uint32_t wm = c_dyn_mask[type];
#pragma unroll
            for (int k = 0; k < 7; k++) if ((wm >> k) & 1u) d.it_st[(size_t)k * NI + q] = m.st[k];
            if (type == 140) { t.c21d[ls] = m.den; t.c21h[ls] = m.st[1]; }
        }
        __syncthreads();
    }
    // current stimuli (simulation_host.cpp:189-209, 247-258): expiry, then add in order
    if (d.cs_off) {
        for (int i = tid; i < ns; i += nth) {
            uint32_t g = s0 + i;
            double I = t.itot[i];
            for (uint32_t k = d.cs_off[g]; k < d.cs_off[g + 1]; k++) {
                if (!d.cs_alive[k]) continue;
                unsigned long long dur = (unsigned long long)(d.cs_dur[k] / dt);
                unsigned long long st = d.cs_start[k];
                if (tick >= st + dur) { d.cs_alive[k] = 0; continue; }
                if (tick >= st && tick < st + dur) I += d.cs_amp[k];
            }
            t.itot[i] = I;
        }
        __syncthreads();
    }

    // ---- step 2.5: electrodiffusion, one warp per component group ----
    if (d.flags & NF_DIFFUSION) {
        const int w = tid >> 5, lane = tid & 31;
        const int ws = d.warp_seg[(size_t)tile * (kTileWarps + 1) + w];
        const int we = d.warp_seg[(size_t)tile * (kTileWarps + 1) + w + 1];
        const int es = d.warp_edge[(size_t)tile * (kTileWarps + 1) + w];
        const int ee = d.warp_edge[(size_t)tile * (kTileWarps + 1) + w + 1];
        // phi_e (diffusion_kernel.h:41-104)
        for (int i = ws + lane; i < we; i += 32) {
            double sacc = 0.0;
#pragma unroll
            for (int q = 0; q < 7; q++) sacc += kNpZ[q] * kNpZ[q] * kDiffC[q] * (double)t.out[q * S + i];
            t.sig[i] = 3.612f * sacc;
            t.phiA[i] = 0.0;
        }
        __syncwarp();
        for (int e = es + lane; e < ee; e += 32) {
            double g = 0.5 * (t.sig[t.ea[e]] + t.sig[t.eb[e]]) * d.e_area[e0 + e] / d.e_dist[e0 + e];
            t.ed[e] = g;
        }
        __syncwarp();
        for (int i = ws + lane; i < we; i += 32) {   // reads only its own sigma: in place
            double diag = t.sig[i] * t.area[i] / 1.0f;
            for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) diag += t.ed[t.inc[k] & 0x7FFF];
            t.sig[i] = diag;
        }
        __syncwarp();
        double* phi = t.phiA;
        double* phn = t.phiB;
        for (int it = 0; it < 50; it++) {
            for (int i = ws + lane; i < we; i += 32) {
                double pn = 0.0;
                for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                    uint16_t ent = t.inc[k];
                    int e = ent & 0x7FFF;
                    double g = t.ed[e];
                    if (g <= 0.0) continue;
                    int o = (ent & 0x8000) ? t.ea[e] : t.eb[e];
                    pn += g * phi[o];
                }
                double diag = t.sig[i];
                double v = (diag > 1e-9) ? (pn - t.itot[i]) / diag : 0.0;
                if (v > 10.0) v = 10.0;
                if (v < -10.0) v = -10.0;
                phn[i] = v;
            }
            __syncwarp();
            double* tmp = phi; phi = phn; phn = tmp;
        }
        // intracellular Nernst-Planck, 5 substeps (diffusion_kernel.h:152-238)
        const float dt_sub = dt / 5;
        for (int sub = 0; sub < 5; sub++) {
            for (int e = es + lane; e < ee; e += 32) {
                if (!t.ei[e]) continue;
                int a = t.ea[e], b = t.eb[e];
                float sigma_i = 0.0f;
#pragma unroll
                for (int q = 0; q < 7; q++) {
                    float C_bar = (float)(0.5f * ((double)t.in[q * S + a] + (double)t.in[q * S + b]));
                    sigma_i += kNpZ[q] * kNpZ[q] * kDiffC[q] * C_bar;
                }
                t.gax[e] = 3.612f * sigma_i * d.e_area[e0 + e] / d.e_dist[e0 + e];
                t.dve[e] = (float)(((double)t.V[a] + phi[a]) - ((double)t.V[b] + phi[b]));
                t.ie[e] = 0.0f;
            }
            __syncwarp();
            for (int i = ws + lane; i < we; i += 32) {
                float gd = 0.0f;
                for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                    int e = t.inc[k] & 0x7FFF;
                    if (t.ei[e]) gd += t.gax[e];
                }
                t.gd[i] = gd;
            }
#pragma unroll 1
            for (int q = 0; q < 7; q++) {
                for (int e = es + lane; e < ee; e += 32) {
                    if (!t.ei[e]) continue;
                    int a = t.ea[e], b = t.eb[e];
                    float C_a = t.in[q * S + a];
                    float C_b = t.in[q * S + b];
                    float x = kNpZ[q] * 0.03742f * t.dve[e];
                    float flux = kDiffC[q] * d.e_area[e0 + e] * dt_sub / d.e_dist[e0 + e] *
                                 (C_a * sg_bernoulli(-x) - C_b * sg_bernoulli(x));
                    t.fl[e] = flux;
                    t.ie[e] += kNpZ[q] * 96.485f * flux / dt_sub;
                }
                __syncwarp();
                for (int i = ws + lane; i < we; i += 32) {
                    float vf = (float)t.vol[i];
                    if (vf < 1e-6f) vf = 1e-6f;
                    double acc = 0.0;
                    for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                        uint16_t ent = t.inc[k];
                        int e = ent & 0x7FFF;
                        if (!t.ei[e]) continue;
                        if (ent & 0x8000) acc += (double)t.fl[e] / vf; else acc -= (double)t.fl[e] / vf;
                    }
                    t.in[q * S + i] = (float)((double)t.in[q * S + i] + (double)(float)acc);
                }
                __syncwarp();
            }
            for (int e = es + lane; e < ee; e += 32) {
                if (!t.ei[e]) continue;
                t.ie[e] = t.ie[e] - t.gax[e] * t.dve[e];
            }
            __syncwarp();
            for (int i = ws + lane; i < we; i += 32) {
                float inp = 0.0f;
                for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                    uint16_t ent = t.inc[k];
                    int e = ent & 0x7FFF;
                    if (!t.ei[e]) continue;
                    if (ent & 0x8000) inp -= t.ie[e]; else inp += t.ie[e];
                }
                float C_dt = t.cm[i] / dt_sub;
                if (C_dt < 1e-9f) C_dt = 1e-9f;
                t.rhs[i] = C_dt * t.V[i] + inp;
                t.den[i] = C_dt + t.gd[i];
                t.vnA[i] = t.V[i];
            }
            __syncwarp();
            float* vc = t.vnA;
            float* vn = t.vnB;
            for (int it = 0; it < 50; it++) {
                for (int i = ws + lane; i < we; i += 32) {
                    float off = 0.0f;
                    for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                        uint16_t ent = t.inc[k];
                        int e = ent & 0x7FFF;
                        if (!t.ei[e]) continue;
                        int o = (ent & 0x8000) ? t.ea[e] : t.eb[e];
                        off += t.gax[e] * vc[o];
                    }
                    vn[i] = (t.rhs[i] + off) / t.den[i];
                }
                __syncwarp();
                float* tmp = vc; vc = vn; vn = tmp;
            }
            for (int i = ws + lane; i < we; i += 32) t.V[i] = vc[i];
            __syncwarp();
        }
        // extracellular Nernst-Planck, 5 substeps (diffusion_kernel.h:244-281)
        for (int sub = 0; sub < 5; sub++) {
#pragma unroll 1
            for (int q = 0; q < 7; q++) {
                for (int e = es + lane; e < ee; e += 32) {
                    int a = t.ea[e], b = t.eb[e];
                    double Ca = t.out[q * S + a];
                    double Cb = t.out[q * S + b];
                    double dphi = phi[a] - phi[b];
                    float x = (float)(kNpZ[q] * 0.03742f * dphi);
                    double flux = kDiffC[q] * d.e_area[e0 + e] * dt_sub / d.e_dist[e0 + e] *
                                  (Ca * sg_bernoulli(-x) - Cb * sg_bernoulli(x));
                    t.ed[e] = flux;
                }
                __syncwarp();
                for (int i = ws + lane; i < we; i += 32) {
                    float vf = (float)t.vol[i];
                    if (vf < 1e-6f) vf = 1e-6f;
                    double acc = 0.0;
                    for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                        uint16_t ent = t.inc[k];
                        int e = ent & 0x7FFF;
                        if (ent & 0x8000) acc += t.ed[e] / (vf * EXTRA_VOLUME_RATIO);
                        else acc -= t.ed[e] / (vf * EXTRA_VOLUME_RATIO);
                    }
                    t.out[q * S + i] = (float)((double)t.out[q * S + i] + acc);
                }
                __syncwarp();
            }
        }
        // NT / ATP / heat / transcription (diffusion_kernel.h:284-363)
        if (d.flags & NF_INTRA_NT) {
            for (int nt = 0; nt < 15; nt++) {
                for (int i = ws + lane; i < we; i += 32) t.nb[i] = d.intra_nt[(size_t)nt * N + s0 + i];
                __syncwarp();
                fick_pass<true, false>(t, d, e0, ws, we, es, ee, lane, gNtD[nt], 1e-12f, dt);
                for (int i = ws + lane; i < we; i += 32) d.intra_nt[(size_t)nt * N + s0 + i] = t.nb[i];
            }
        }
        if (d.flags & NF_NT_DIFFUSE_OUT) {
            for (int nt = 0; nt < 15; nt++) {
                for (int i = ws + lane; i < we; i += 32) t.nb[i] = d.nt[(size_t)nt * N + s0 + i];
                __syncwarp();
                fick_pass<false, false>(t, d, e0, ws, we, es, ee, lane, gNtD[nt], 1e-12f, dt);
                for (int i = ws + lane; i < we; i += 32) d.nt[(size_t)nt * N + s0 + i] = t.nb[i];
            }
        }
        {
            for (int i = ws + lane; i < we; i += 32) t.nb[i] = t.atp[i];
            __syncwarp();
            fick_pass<true, true>(t, d, e0, ws, we, es, ee, lane, 0.14f, 1e-12f, dt);
            for (int i = ws + lane; i < we; i += 32) t.atp[i] = t.nb[i];
        }
        if (d.flags & NF_TEMP) {
            for (int i = ws + lane; i < we; i += 32) t.nb[i] = d.temp[s0 + i];
            __syncwarp();
            fick_pass<true, true>(t, d, e0, ws, we, es, ee, lane, 0.0014f, 0.001f, dt);
            for (int i = ws + lane; i < we; i += 32) d.temp[s0 + i] = t.nb[i];
        }
        if (d.flags & NF_TXN) {
            for (int i = ws + lane; i < we; i += 32) t.nb[i] = d.txn[s0 + i];
            __syncwarp();
            fick_pass<true, true>(t, d, e0, ws, we, es, ee, lane, 0.01f, 1e-9f, dt);
            for (int i = ws + lane; i < we; i += 32) d.txn[s0 + i] = t.nb[i];
        }
        for (int i = ws + lane; i < we; i += 32) {
#pragma unroll
            for (int q = 0; q < 7; q++) {
                double e = (double)t.out[q * S + i];
                e += (kBathIon[q] - e) * dt / 1.0f;
                if (e < 1e-9) e = 1e-9;
                if (e > 1000.0) e = 1000.0;
                t.out[q * S + i] = (float)e;
            }
        }
    }
    __syncthreads();

    // ---- write back ----
    const bool ext = (d.flags & NF_PRE_EXT) != 0;
    for (int i = tid; i < ns; i += nth) {
        uint32_t g = s0 + i;
        d.V[g] = t.V[i];
#pragma unroll
        for (int q = 0; q < 7; q++) {
            d.ion_in[(size_t)q * N + g] = t.in[q * S + i];
            d.ion_out[(size_t)q * N + g] = t.out[q * S + i];
        }
        d.atp[g] = t.atp[i];
        d.ibuf[g] = t.itot[i];
        d.pre_rec[g] = make_float4(t.V[i], t.out[2 * S + i], t.c21d[i], t.c21h[i]);
        if (ext) {
            d.pre_ext[g] = make_float4(t.in[i], t.in[S + i], t.in[2 * S + i], t.out[i]);
            d.pre_ext2[g] = t.out[S + i];
        }
    }
}

// D = 1.33 * (23/M)^(1/3); the 15th entry has no mass in the reference's table (0 -> 1)
__global__ void k_init_tables() {
    const float mass[15] = {147.0f, 103.0f, 153.0f, 176.0f, 146.0f, 267.0f, 169.0f, 75.0f, 111.0f,
                            348.0f, 507.0f, 232.0f, 24.0f, 162.0f, 0.0f};
    for (int q = 0; q < 15; q++) {
        float ms = mass[q];
        if (ms < 1.0f) ms = 1.0f;
        gNtD[q] = 1.33f * dm_powf(23.0f / ms, 1.0f / 3.0f);
    }
}

static bool g_tables_ready[64] = {false};   // per device: constant memory is per context

static cudaError_t init_tables(cudaStream_t stream) {
    int dev = 0;
    cudaError_t ge = cudaGetDevice(&dev);
    if (ge != cudaSuccess) return ge;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (g_tables_ready[dev]) return cudaSuccess;
    uint8_t dyn[256] = {0}, par[256] = {0};
    dyn[1] = 0x03; par[1] = 0x1C;
    dyn[8] = 0x03; dyn[9] = 0x05; dyn[11] = 0x03; dyn[12] = 0x03;
    dyn[85] = 0x0B; par[85] = 0x34;
    par[98] = 0x06; par[100] = 0x06;
    dyn[102] = 0x02; par[102] = 0x1D;
    dyn[103] = 0x01; par[103] = 0x38;
    dyn[104] = 0x01; par[104] = 0x06;
    dyn[105] = 0x01; par[105] = 0x3E;
    par[106] = 0x08; par[107] = 0x03;
    dyn[112] = 0x01; par[112] = 0x76;
    dyn[123] = 0x01; par[123] = 0x16;
    dyn[129] = 0x01; par[129] = 0x3E;
    par[133] = 0x01;
    dyn[140] = 0x03;
    dyn[141] = 0x03; par[141] = 0x20;
    dyn[142] = 0x03; par[142] = 0x20;
    dyn[150] = 0x07; par[150] = 0x20;
    dyn[200] = 0x03; par[200] = 0x7C;
    cudaError_t e = cudaMemcpyToSymbol(c_dyn_mask, dyn, sizeof(dyn));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_par_mask, par, sizeof(par));
    // Stokes-Einstein NT diffusion coefficients (types.h:428-445, nt_diffusion_coeff)
    if (e == cudaSuccess) {
        k_init_tables<<<1, 1, 0, stream>>>();
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    }
    if (e == cudaSuccess) g_tables_ready[dev] = true;
    return e;
}

cudaError_t prepare_tick(const NetDev& dev, const NetHost& host, cudaStream_t stream) {
    (void)dev;
    cudaError_t e = init_tables(stream);
    if (e != cudaSuccess) return e;
    const size_t smem = tile_smem_bytes(host.max_tile_segs, host.max_tile_edges);
    if (smem > 48 * 1024)
        e = cudaFuncSetAttribute(k_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return e;
}

static void enqueue_tile(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                         cudaStream_t stream) {
    const uint32_t S = host.max_tile_segs, E = host.max_tile_edges;
    k_tile<<<dev.n_tiles, kTileThreads, tile_smem_bytes(S, E), stream>>>(dev, dt, tick, S, E);
}

cudaError_t launch_tile(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                        cudaStream_t stream) {
    cudaError_t e = prepare_tick(dev, host, stream);
    if (e != cudaSuccess) return e;
    enqueue_tile(dev, host, dt, tick, stream);
    return cudaGetLastError();
}

cudaError_t enqueue_tick(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick, int first_tick,
                         cudaStream_t stream) {
    enqueue_tile(dev, host, dt, tick, stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_synapse(dev, dt, tick, first_tick, stream);
}

cudaError_t launch_tick(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick, int first_tick,
                        cudaStream_t stream) {
    cudaError_t e = launch_tile(dev, host, dt, tick, stream);
    if (e != cudaSuccess) return e;
    return launch_synapse(dev, dt, tick, first_tick, stream);
}

}  // namespace bnc
