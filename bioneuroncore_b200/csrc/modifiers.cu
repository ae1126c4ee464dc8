// modifiers.cu -- step 1 of a tick (modifier currents) and the tick launcher.
//
// One tick of the reference (simulation_host.cpp:174-657) is these launches:
//
//  k_gather      per segment: the step-1 working record (V, ions, ATP, area, volume,
//                I_total = 0), the Cav2.1 gate from its static copy.
//  k_phase x P   one launch per modifier phase over the whole network.  Every segment's
//                active modifiers sit in successive phases in slot order, at most one
//                per phase, so a phase's items touch distinct segments and need no
//                barrier; inside a phase items are ordered by type, so warps -- and the
//                SMs at any moment -- run few channel models at a time, which keeps the
//                many models' code within the instruction caches.  Each dispatch case
//                loads and stores only the record fields its model uses.
//  k_phase_group the same phases four to a launch by default (slot-order schedules):
//                one thread per segment runs its items of those phases on the record
//                held in registers, so the record crosses HBM once per group.
//  k_diffusion   (diffuse.cu) stimuli, step 2.5 electrodiffusion, the presynaptic record.
//  k_synapse     (synapse.cu) steps 3 and 4.
#define BNC_MATH_OUTLINE 1   // 26 channel models in one kernel: keep exp/log out of line
#include <algorithm>
#include <cuda_runtime.h>
#include "net.h"
#include "physics.cuh"

#ifndef BNC_GROUP_MIN_CTAS
#define BNC_GROUP_MIN_CTAS 4
#endif

namespace bnc {

// state indices each modifier type updates every tick (read + write)
__constant__ uint8_t c_dyn_mask[256];
// state indices each type reads as parameters (default when 0)
__constant__ uint8_t c_par_mask[256];

__global__ void __launch_bounds__(256)
k_gather(NetDev d, uint32_t s_begin, uint32_t s_end) {
    const uint32_t g = s_begin + blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t N = d.n_seg;
    if (g >= s_end) return;
    SegRec r;
    r.V = d.V[g];
#pragma unroll
    for (int q = 0; q < 7; q++) {
        r.in[q] = d.ion_in[(size_t)q * N + g];
        r.out[q] = d.ion_out[(size_t)q * N + g];
    }
    r.atp = d.atp[g];
    r.area = d.area[g];
    r.vol = d.vol[g];
    r.itot = 0.0;
    r.pad = 0;
    r.pad2 = 0.0;
    d.rec[g] = r;
    d.c21_cur[g] = d.cav21_static[g];
}

// The segment fields an item sees, loaded from the record and stored back inside the
// model's own dispatch case: after inlining, the loads a model does not read are
// dead, and stores of fields it leaves unchanged write back what was read.  The GHK
// factors of V are computed here, per item, from the record's V.
__device__ __forceinline__ void rec_load(DSeg& s, const SegRec* r) {
    s.V = r->V;
#pragma unroll
    for (int k = 0; k < 7; k++) { s.in[k] = r->in[k]; s.out[k] = r->out[k]; }
    s.atp = r->atp;
    s.area = r->area;
    s.vol = r->vol;
    ghk_cache_fill(s.gc, s.V);   // dead code for models without GHK currents
}

__device__ __forceinline__ void rec_store(const DSeg& s, float v0, SegRec* r) {
    (void)v0;
    r->V = s.V;
#pragma unroll
    for (int k = 0; k < 7; k++) { r->in[k] = s.in[k]; r->out[k] = s.out[k]; }
    r->atp = s.atp;
}

// kernel_dispatch.h:337-570 restricted to the device-implemented types (the builder
// rejects every other type; myelin, type 4, is never an item: it returns 0 and
// touches nothing).
template <bool kDef, bool kX>
__device__ __forceinline__ double run_item(uint8_t type, DMod& m, SegRec* r, float dt, float& glu, float gaba,
                                           float gly) {
    double I = 0.0;
    switch (type) {
#define BNC_ITEM(T, CALL)          \
    case T: {                      \
        DSeg s;                    \
        rec_load(s, r);            \
        const float v0 = s.V;      \
        m.area = s.area;           \
        I = (CALL);                \
        rec_store(s, v0, r);       \
        break;                     \
    }
        BNC_ITEM(1, dp_cav13_current<kDef>(m, s, dt))
        BNC_ITEM(7, dp_nak_pump_current(m, s, dt))
        BNC_ITEM(8, dp_ampa_current<kDef>(m, s, dt, glu, 1.0f))
        BNC_ITEM(9, dp_nmda_current<kDef>(m, s, dt, glu, 1.0f))
        BNC_ITEM(11, dp_gabaa_current<kDef>(m, s, dt, gaba, 1.0f))
        BNC_ITEM(12, dp_glycine_current<kDef>(m, s, dt, gly, 1.0f))
        BNC_ITEM(85, dp_kv42_current<kDef>(m, s, dt))
        BNC_ITEM(98, dp_pmca_current<kDef>(m, s, dt))
        BNC_ITEM(99, dp_ncx_current(m, s, dt))
        BNC_ITEM(100, dp_kcc2_current<kDef>(m, s, dt))
        BNC_ITEM(102, dp_ca_buffer_current<kDef>(m, s, dt))
        BNC_ITEM(103, dp_sk_current<kDef>(m, s, dt))
        BNC_ITEM(104, dp_bk_current<kDef>(m, s, dt))
        BNC_ITEM(105, dp_nap_current<kDef>(m, s, dt))
        BNC_ITEM(106, dp_kir_current<kDef>(m, s, dt))
        BNC_ITEM(107, dp_k2p_current<kDef>(m, s, dt))
        BNC_ITEM(112, dp_kv7_current<kDef>(m, s, dt))
        BNC_ITEM(123, dp_kvdr_current<kDef>(m, s, dt))
        BNC_ITEM(129, dp_hcn1_current<kDef>(m, s, dt))
        BNC_ITEM(133, dp_nalcn_current<kDef>(m, s, dt))
        BNC_ITEM(140, dp_cav21_current(m, s, dt))
        BNC_ITEM(141, dp_nav_current<kDef>(m, s, dt, 0))
        BNC_ITEM(142, dp_nav_current<kDef>(m, s, dt, 1))
        BNC_ITEM(150, dp_kv31_current<kDef>(m, s, dt))
        BNC_ITEM(200, dp_cav31_current<kDef>(m, s, dt))
        // models only some networks carry: their code is in the kX instantiation alone
        BNC_ITEM(86, kX ? dp_ecb_synthesis_current<kDef>(m, s, dt) : 0.0)
        BNC_ITEM(147, kX ? dp_glast_current(m, s, dt, glu) : 0.0)
        BNC_ITEM(114, kX ? dp_connexin_current<kDef>(m, s, dt) : 0.0)
        BNC_ITEM(198, kX ? dp_connexin_current<kDef>(m, s, dt) : 0.0)
#undef BNC_ITEM
        default: break;
    }
    return I;
}

// One modifier phase: items [b, e), one thread each (simulation_host.cpp:234-303 for
// the item's segment and slot).  Capped at 64 registers for 4 CTAs per SM: with the
// 96-byte record the cap costs 16 bytes of spills and the extra warps hide more of the
// record loads' latency (6.4M segments: 8.04 -> 7.80 ms per tick).
template <bool kX>
__global__ void __launch_bounds__(256, 4)
k_phase(NetDev d, float dt, uint32_t b, uint32_t e) {
    const uint32_t q = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= e) return;
    const uint32_t N = d.n_seg;
    const uint32_t NI = d.n_items;
    const uint32_t g = d.it_seg[q];
    const uint32_t tf = d.it_tf[q];
    const uint8_t type = (uint8_t)(tf & 0xFFu);
    const uint8_t fl = (uint8_t)(tf >> 8);
    if (type < 128 && ((d.user_mask[type >> 5] >> (type & 31)) & 1u)) return;   // a registered device modifier
    DMod m;
    m.den = d.it_den[q];
    m.av = (fl & 2) ? (uint8_t)((fl >> 2) & 7) : (uint8_t)0;
    uint32_t rm = c_dyn_mask[type] | ((fl & 1) ? c_par_mask[type] : 0u);
    if (fl & 2) rm |= (1u << m.av) & 0x7Fu;
#pragma unroll
    for (int k = 0; k < 7; k++) m.st[k] = ((rm >> k) & 1u) ? d.it_st[(size_t)k * NI + q] : 0.0f;
    float glu = 0.0f, gaba = 0.0f, gly = 0.0f;
    if (type == 8 || type == 9 || (kX && type == 147)) glu = d.nt[g];
    else if (type == 11) gaba = d.nt[(size_t)1 * N + g];
    else if (type == 12) gly = d.nt[(size_t)7 * N + g];
    SegRec* r = d.rec + g;
    const double I = ((fl & 3) == 0) ? run_item<true, kX>(type, m, r, dt, glu, gaba, gly)
                                     : run_item<false, kX>(type, m, r, dt, glu, gaba, gly);
    r->itot = r->itot + I;
    if (kX && type == 147) d.nt[g] = glu;   // the transporter's uptake
    const uint32_t wm = c_dyn_mask[type];
#pragma unroll
    for (int k = 0; k < 7; k++) if ((wm >> k) & 1u) d.it_st[(size_t)k * NI + q] = m.st[k];
    if (type == 140) d.c21_cur[g] = make_float2(m.den, m.st[1]);
}

// run_item on a segment held in registers: the same models in the same order, the GHK
// factors computed from the V the item starts with, as rec_load computes them.
template <bool kDef, bool kX>
__device__ __forceinline__ double run_item_s(uint8_t type, DMod& m, DSeg& s, float dt, float& glu, float gaba,
                                             float gly) {
    double I = 0.0;
    switch (type) {
#define BNC_ITEM(T, CALL)            \
    case T: {                        \
        ghk_cache_fill(s.gc, s.V);   \
        m.area = s.area;             \
        I = (CALL);                  \
        break;                       \
    }
        BNC_ITEM(1, dp_cav13_current<kDef>(m, s, dt))
        BNC_ITEM(7, dp_nak_pump_current(m, s, dt))
        BNC_ITEM(8, dp_ampa_current<kDef>(m, s, dt, glu, 1.0f))
        BNC_ITEM(9, dp_nmda_current<kDef>(m, s, dt, glu, 1.0f))
        BNC_ITEM(11, dp_gabaa_current<kDef>(m, s, dt, gaba, 1.0f))
        BNC_ITEM(12, dp_glycine_current<kDef>(m, s, dt, gly, 1.0f))
        BNC_ITEM(85, dp_kv42_current<kDef>(m, s, dt))
        BNC_ITEM(98, dp_pmca_current<kDef>(m, s, dt))
        BNC_ITEM(99, dp_ncx_current(m, s, dt))
        BNC_ITEM(100, dp_kcc2_current<kDef>(m, s, dt))
        BNC_ITEM(102, dp_ca_buffer_current<kDef>(m, s, dt))
        BNC_ITEM(103, dp_sk_current<kDef>(m, s, dt))
        BNC_ITEM(104, dp_bk_current<kDef>(m, s, dt))
        BNC_ITEM(105, dp_nap_current<kDef>(m, s, dt))
        BNC_ITEM(106, dp_kir_current<kDef>(m, s, dt))
        BNC_ITEM(107, dp_k2p_current<kDef>(m, s, dt))
        BNC_ITEM(112, dp_kv7_current<kDef>(m, s, dt))
        BNC_ITEM(123, dp_kvdr_current<kDef>(m, s, dt))
        BNC_ITEM(129, dp_hcn1_current<kDef>(m, s, dt))
        BNC_ITEM(133, dp_nalcn_current<kDef>(m, s, dt))
        BNC_ITEM(140, dp_cav21_current(m, s, dt))
        BNC_ITEM(141, dp_nav_current<kDef>(m, s, dt, 0))
        BNC_ITEM(142, dp_nav_current<kDef>(m, s, dt, 1))
        BNC_ITEM(150, dp_kv31_current<kDef>(m, s, dt))
        BNC_ITEM(200, dp_cav31_current<kDef>(m, s, dt))
        // models only some networks carry: their code is in the kX instantiation alone
        BNC_ITEM(86, kX ? dp_ecb_synthesis_current<kDef>(m, s, dt) : 0.0)
        BNC_ITEM(147, kX ? dp_glast_current(m, s, dt, glu) : 0.0)
        BNC_ITEM(114, kX ? dp_connexin_current<kDef>(m, s, dt) : 0.0)
        BNC_ITEM(198, kX ? dp_connexin_current<kDef>(m, s, dt) : 0.0)
#undef BNC_ITEM
        default: break;
    }
    return I;
}

// Item offsets of a group of consecutive phases: phase j of the group holds items
// [off[j], off[j + 1]); row q of the group owns item off[j] + q of every phase j with
// q < off[j + 1] - off[j].
struct PhaseGroup {
    uint32_t off[kMaxFuse + 1];
    uint32_t n;   // phases in the group
};

// `grp.n` consecutive modifier phases in one launch, one thread per row (a segment):
// the record is loaded once, the row's items run in phase order on it in registers,
// and it is stored once.  Items of one segment run in the order and with the
// arithmetic of the one-launch-per-phase path, so the results are the same bits.
// The builder orders rows by (item count, item types), so a warp runs one sequence of
// models; it forms groups only when no registered device modifier is present.
template <bool kX>
__global__ void __launch_bounds__(256, BNC_GROUP_MIN_CTAS)
k_phase_group(NetDev d, float dt, PhaseGroup grp) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= grp.off[1] - grp.off[0]) return;
    const uint32_t N = d.n_seg;
    const uint32_t NI = d.n_items;
    const uint32_t g = d.it_seg[grp.off[0] + q];
    SegRec* r = d.rec + g;
    DSeg s;
    s.V = r->V;
#pragma unroll
    for (int k = 0; k < 7; k++) { s.in[k] = r->in[k]; s.out[k] = r->out[k]; }
    s.atp = r->atp;
    s.area = r->area;
    s.vol = r->vol;
    double itot = r->itot;
#pragma unroll 1
    for (uint32_t j = 0; j < grp.n; j++) {
        if (q >= grp.off[j + 1] - grp.off[j]) break;
        const uint32_t qi = grp.off[j] + q;
        const uint32_t tf = d.it_tf[qi];
        const uint8_t type = (uint8_t)(tf & 0xFFu);
        const uint8_t fl = (uint8_t)(tf >> 8);
        DMod m;
        m.den = d.it_den[qi];
        m.av = (fl & 2) ? (uint8_t)((fl >> 2) & 7) : (uint8_t)0;
        uint32_t rm = c_dyn_mask[type] | ((fl & 1) ? c_par_mask[type] : 0u);
        if (fl & 2) rm |= (1u << m.av) & 0x7Fu;
#pragma unroll
        for (int k = 0; k < 7; k++) m.st[k] = ((rm >> k) & 1u) ? d.it_st[(size_t)k * NI + qi] : 0.0f;
        float glu = 0.0f, gaba = 0.0f, gly = 0.0f;
        if (type == 8 || type == 9 || (kX && type == 147)) glu = d.nt[g];
        else if (type == 11) gaba = d.nt[(size_t)1 * N + g];
        else if (type == 12) gly = d.nt[(size_t)7 * N + g];
        const double I = ((fl & 3) == 0) ? run_item_s<true, kX>(type, m, s, dt, glu, gaba, gly)
                                         : run_item_s<false, kX>(type, m, s, dt, glu, gaba, gly);
        itot = itot + I;
        if (kX && type == 147) d.nt[g] = glu;   // the transporter's uptake
        const uint32_t wm = c_dyn_mask[type];
#pragma unroll
        for (int k = 0; k < 7; k++) if ((wm >> k) & 1u) d.it_st[(size_t)k * NI + qi] = m.st[k];
        if (type == 140) d.c21_cur[g] = make_float2(m.den, m.st[1]);
    }
    r->V = s.V;
#pragma unroll
    for (int k = 0; k < 7; k++) { r->in[k] = s.in[k]; r->out[k] = s.out[k]; }
    r->atp = s.atp;
    r->itot = itot;
}

static bool g_tables_ready[64] = {false};   // per device: constant memory is per context

// The state words each built-in type updates every tick (dyn) and reads as parameters
// when non-zero (par), by state index bit.
static void fill_mask_tables(uint8_t* dyn, uint8_t* par) {
    std::fill(dyn, dyn + 256, (uint8_t)0);
    std::fill(par, par + 256, (uint8_t)0);
    dyn[1] = 0x03; par[1] = 0x1C;
    dyn[8] = 0x03; dyn[9] = 0x05; dyn[11] = 0x03; dyn[12] = 0x03;
    dyn[86] = 0x01; par[86] = 0x06;
    dyn[114] = dyn[198] = 0x13; par[114] = par[198] = 0x6C;
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
}

uint8_t host_dyn_mask(uint8_t type) {
    static uint8_t dyn[256], par[256];
    static bool ready = false;
    if (!ready) { fill_mask_tables(dyn, par); ready = true; }
    return dyn[type];
}

static cudaError_t init_tables(cudaStream_t stream) {
    int dev = 0;
    cudaError_t ge = cudaGetDevice(&dev);
    if (ge != cudaSuccess) return ge;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (g_tables_ready[dev]) return cudaSuccess;
    uint8_t dyn[256], par[256];
    fill_mask_tables(dyn, par);
    cudaError_t e = cudaMemcpyToSymbol(c_dyn_mask, dyn, sizeof(dyn));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_par_mask, par, sizeof(par));
    if (e == cudaSuccess) g_tables_ready[dev] = true;
    return e;
}

cudaError_t prepare_tick(const NetDev& dev, const NetHost& host, cudaStream_t stream) {
    (void)dev;
    cudaError_t e = init_tables(stream);
    if (e != cudaSuccess) return e;
    e = prepare_synapse(stream);
    if (e != cudaSuccess) return e;
    return prepare_diffusion(host, stream);
}

static cudaError_t enqueue_modifiers(const NetDev& dev, const NetHost& host, float dt, cudaStream_t stream) {
    const uint32_t P = dev.n_phases;
    const uint32_t C = host.n_chunks ? host.n_chunks : 1;
    const uint32_t cs = host.chunk_segs ? host.chunk_segs : dev.n_seg;
    size_t u = 0;
    for (uint32_t c = 0; c < C; c++) {
        const uint32_t s0 = c * cs, s1 = std::min(dev.n_seg, s0 + cs);
        k_gather<<<(s1 - s0 + 255) / 256, 256, 0, stream>>>(dev, s0, s1);
        if (host.fuse > 1) {   // one chunk, no registered device modifiers (the builder's rule)
            for (uint32_t p0 = 0; p0 < P; p0 += host.fuse) {
                PhaseGroup grp;
                grp.n = std::min(host.fuse, P - p0);
                for (uint32_t j = 0; j <= kMaxFuse; j++) grp.off[j] = host.phase_off[std::min(p0 + j, p0 + grp.n)];
                const uint32_t rows = grp.off[1] - grp.off[0];
                if (rows == 0) continue;
                const dim3 gs((rows + 255) / 256);
                if (grp.n == 1) {
                    if (dev.model_extras) k_phase<true><<<gs, 256, 0, stream>>>(dev, dt, grp.off[0], grp.off[1]);
                    else k_phase<false><<<gs, 256, 0, stream>>>(dev, dt, grp.off[0], grp.off[1]);
                } else if (dev.model_extras) {
                    k_phase_group<true><<<gs, 256, 0, stream>>>(dev, dt, grp);
                } else {
                    k_phase_group<false><<<gs, 256, 0, stream>>>(dev, dt, grp);
                }
            }
            continue;
        }
        for (uint32_t p = 0; p < P; p++) {
            const uint32_t bk = c * P + p;
            const uint32_t b = host.phase_off[bk], e = host.phase_off[bk + 1];
            if (e > b && dev.model_extras) k_phase<true><<<(e - b + 255) / 256, 256, 0, stream>>>(dev, dt, b, e);
            else if (e > b) k_phase<false><<<(e - b + 255) / 256, 256, 0, stream>>>(dev, dt, b, e);
            // items of registered device modifiers in this bucket (k_phase skips them)
            for (; u < host.user_ranges.size() && host.user_ranges[u].bucket == bk; u++) {
                const auto& ur = host.user_ranges[u];
                cudaError_t le = launch_device_modifier(ur.kernel, dev, (uint8_t)ur.type, ur.begin, ur.end, dt, stream);
                if (le != cudaSuccess) return le;
            }
        }
    }
    return cudaGetLastError();
}

uint32_t modifier_launches(const NetDev& dev, const NetHost& host) {
    const uint32_t P = dev.n_phases;
    const uint32_t C = host.n_chunks ? host.n_chunks : 1;
    if (host.phase_off.size() < (size_t)C * P + 1) return 0;
    uint32_t n = C;   // k_gather
    if (host.fuse > 1) {
        for (uint32_t p0 = 0; p0 < P; p0 += host.fuse) n += host.phase_off[p0 + 1] > host.phase_off[p0] ? 1u : 0u;
        return n;
    }
    for (uint32_t bk = 0; bk < C * P; bk++) n += host.phase_off[bk + 1] > host.phase_off[bk] ? 1u : 0u;
    return n + (uint32_t)host.user_ranges.size();
}

cudaError_t launch_modifiers(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                             cudaStream_t stream) {
    (void)tick;
    cudaError_t e = prepare_tick(dev, host, stream);
    if (e != cudaSuccess) return e;
    return enqueue_modifiers(dev, host, dt, stream);
}

cudaError_t launch_diffusion(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                             cudaStream_t stream) {
    cudaError_t e = prepare_tick(dev, host, stream);
    if (e != cudaSuccess) return e;
    return enqueue_diffusion(dev, host, dt, tick, stream);
}

cudaError_t enqueue_tick(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick, int first_tick,
                         cudaStream_t stream) {
    cudaError_t e = enqueue_modifiers(dev, host, dt, stream);
    if (e != cudaSuccess) return e;
    e = enqueue_diffusion(dev, host, dt, tick, stream);
    if (e != cudaSuccess) return e;
    return launch_synapse(dev, dt, tick, first_tick, stream);
}

cudaError_t launch_tick(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick, int first_tick,
                        cudaStream_t stream) {
    cudaError_t e = prepare_tick(dev, host, stream);
    if (e != cudaSuccess) return e;
    return enqueue_tick(dev, host, dt, tick, first_tick, stream);
}

}  // namespace bnc
