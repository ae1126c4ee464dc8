// adjoint.cu -- gradients of a somatic voltage-trace loss with respect to per-segment
// maximal conductances (gNa, gK, gleak: the densities of the Nav1.x, Kv delayed
// rectifier and K2P leak modifiers) and per-synapse weights (the receptor density
// scale), by a hand-written discrete adjoint of the reference tick
// (simulation_host.cpp:174-657).  The network may hold the whole small set: Cav1.3 and
// the Na/K pump run with their own densities and are differentiated too, with the ATP
// the pump consumes (a state word, diffusing by Fick in step 2.5).  Networks without
// them run kernel instantiations that leave that code out (kFull = false).
//
// Pathwise replay.  The transmitter a release puts into a cleft is taken from a log
// recorded once by the plain tick (bnc_adjoint_record), so the sampled release
// events are fixed.  With them fixed, a neuron's tick reads nothing outside the
// neuron: step 1 and the electrodiffusion of step 2.5 only couple segments joined by
// connections (which stay inside a neuron), the transmitter seen by a receptor is
// the logged clefts (the per-segment transmitter is reset before the synapse pass,
// simulation_host.cpp:330-336), and the Cav2.1 and bouton Ca2+ that decide releases
// act on nothing else.  So one CTA runs one (neuron, parameter set) through all
// ticks with its state in shared memory -- the forward pass with the device
// functions of the plain tick and the reference's operation order, so it reproduces
// the plain trajectory -- and the reverse pass runs the same CTA backwards.
//
// Reverse pass.  Checkpoints of the state every K ticks bound memory: for each
// window, the CTA re-runs the window from its checkpoint and keeps each tick's
// starting state (HBM), then walks the ticks backwards; a tick is re-run once more
// with its intermediates recorded (the phi_e and V_m Jacobi iterates, the sub-step
// states) and reversed step by step:
//   step 4 (membrane, clamps as masks) -> step 3 (receptors; local Jacobians of the
//   ionotropic current by dual numbers) -> bath relaxation -> extracellular and
//   intracellular Nernst-Planck sub-steps (hand-derived: Bernoulli fluxes, chord
//   conductances, the transposed Jacobi sweeps) -> the phi_e solve -> step 1 (local
//   Jacobians of the channel models by dual numbers, slot order reversed).
#define BNC_MATH_OUTLINE 1   // one copy of exp/log for the forward, the re-runs and the reverse
#ifndef BNC_ADJ_MIN_BLOCKS
#define BNC_ADJ_MIN_BLOCKS 4   // CTAs per SM the 64-thread backward is bounded for (5 spills: slower)
#endif
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include <cuda_pipeline.h>
#include "net.h"
#include "hostnet.h"
#include "physics.cuh"
#include "receptor.cuh"
#include "adjoint_models.cuh"

namespace bnc {

namespace {

constexpr int kMaxSeg = 128;     // segments (and connections) per neuron: threads per CTA
constexpr int kItems = 5;        // differentiable items per segment (Nav, Kv_DR, K2P, Cav1.3, Na/K pump)
// item arrays' stride per segment on the device: kItems with Cav1.3 or the pump, else 3
template <bool kFull> struct ItemStride { static constexpr uint32_t v = kFull ? kItems : 3; };
constexpr int kGates = 5;        // dynamic gate words per segment (Nav m, h; Kv_DR n; Cav1.3 m, h)
constexpr int kMaxInc = 4;       // connections per segment (the generated families have at most 3)
constexpr int kRecPerSyn = 2;    // receptors per synapse
// A segment's state words: V, 7 intra, 7 extra, then the gate words the network's
// segments need (at most kGates) and ATP when some segment carries the pump
// (AdjDev::W words; ATP at row AdjDev::atp_w).  Shared memory holds W rows twice in
// the reverse pass, so W follows the network.  The fitting family's kernels (no
// Cav1.3, no pump) use the fixed width kW3: three gate words.
constexpr uint32_t kW3 = 18;
constexpr int kSynWords = 5;     // receptor 0 (r, d), receptor 1 (r, d), cleft; an NMDA receptor's d word holds
                                 // its Ca2+-dependent inactivation gate (state[2]; it does not desensitise)
constexpr int kSynScr = 11;      // per synapse in the scratch: in[7] before it, open probabilities, NMDA gates before

__constant__ float c_z2d[7];     // z^2 * D per ion, as the reference's float product
__constant__ float c_z[7];
__constant__ float c_D[7];
__constant__ float c_bath[7];

// Device descriptor (by value).  Segments, connections and synapse slots are in
// neuron order; `seg`-indexed arrays are global over the network.
struct AdjDev {
    uint32_t nn, n_seg, n_edge, n_slot, n_syn, n_sets;
    uint32_t T, K, n_ckpt, stride, n_samples;
    uint32_t Smax, Emax, Ymax;
    uint32_t L;                    // state floats of one parameter set
    uint32_t W, atp_w;             // state words per segment, the ATP word
    float dt;
    int has_conn;
    int has_atp;                   // some segment carries the Na/K pump: ATP changes and diffuses
    int full;                      // some item is Cav1.3 or the pump: the kernels with their code
    unsigned long long tick0;
    // per neuron
    const uint32_t *nr_seg, *nr_edge, *nr_slot, *nr_st;   // [nn + 1] offsets
    const uint16_t* nr_soma;                              // local soma index
    // per segment
    const float *area, *cm;
    const double* vol;
    const uint8_t* n_it;           // differentiable items
    const uint8_t* it_type;        // [seg][kItems]
    const uint8_t* it_gate;        // first gate word of the item
    const float* it_st;            // [seg][kItems][7] parameter words
    const float* it_den;           // [seg][kItems] densities of the items without a fitted conductance
    const uint8_t* inc_n;
    const uint16_t* inc_e;         // [seg][kMaxInc] local connection ids, ascending
    const uint32_t* stim_off;      // [seg + 1]
    const unsigned long long *stim_b, *stim_e;
    const float* stim_amp;
    const uint32_t* sp_off;        // [seg + 1] synapse slots with this post segment
    // per connection (local endpoints)
    const uint16_t *ed_a, *ed_b;
    const uint8_t* ed_intra;
    const float *ed_area, *ed_dist, *ed_vola, *ed_volb;
    // per synapse slot (post order, original synapse order within a post segment)
    const uint32_t* sl_syn;        // original synapse index
    const uint8_t* sl_nrec;
    const uint8_t* sl_kind;        // [slot][kRecPerSyn] receptor table index
    const float* sl_rden;          // [slot][kRecPerSyn]
    const uint8_t* sl_rav;         // [slot][kRecPerSyn]
    const float *sl_parea, *sl_tauc;
    const uint8_t* sl_nt;          // 0 glutamate, 1 GABA, 2 glycine
    const uint32_t* ev_off;        // [slot + 1] logged cleft entries, by tick
    const unsigned long long* ev_tick;
    const float* ev_amt;
    // per parameter set
    const float* par;              // [set][3][seg]
    const float* w;                // [set][n_syn]
    const float* target;           // [n_samples][nn]
    const float* init;             // [L] initial state (shared by all sets)
    float* state;                  // [set][L]
    float* lam;                    // [set][L] adjoint state between launches
    float* ckpt;                   // [n_ckpt][set][L]
    float* win;                    // [K][set][L]
    double* loss_part;             // [set][nn]
    float* trace;                  // [set][n_samples][nn] or null
    double* g_par;                 // [set][3][seg]
    double* g_w;                   // [set][n_syn]
    float* scr;                    // per CTA: scr_floats
    size_t scr_floats;
};

// Shared-memory layout of one CTA.
struct Lay {
    double *ibuf, *phiA, *phiB, *sig, *diag, *god, *ib3, *fa, *fb;
    unsigned long long* pmask;   // reverse pass: per segment, the phi_e sweeps that did not clamp
    float *st, *gax, *term, *vnA, *vnB;
    // reverse pass only
    float *s2, *lam, *lphi, *lI, *mu, *lvB, *linp, *lgdg, *eca, *ecb, *edv, *ldiag, *jsm;
};

__host__ __device__ inline size_t lay_bytes(uint32_t S, uint32_t E, uint32_t Y, bool bwd, uint32_t W) {
    size_t dbl = (size_t)6 * S + 15 * (size_t)E;
    size_t flt = (size_t)W * S + kSynWords * Y + 2 * (size_t)E + 2 * (size_t)S;
    if (bwd) {
        dbl += S;   // pmask
        flt += 15 * (size_t)S + W * (size_t)S + kSynWords * (size_t)Y + 7 * (size_t)S + (size_t)E + 51 * (size_t)S + 4;
    }
    return dbl * 8 + flt * 4;
}

__device__ inline Lay make_lay(unsigned char* base, uint32_t S, uint32_t E, uint32_t Y, bool bwd, uint32_t W) {
    Lay l;
    double* d = reinterpret_cast<double*>(base);
    l.ibuf = d; d += S; l.phiA = d; d += S; l.phiB = d; d += S; l.sig = d; d += S; l.diag = d; d += S;
    l.god = d; d += E; l.ib3 = d; d += S; l.fa = d; d += 7 * E; l.fb = d; d += 7 * E;
    l.pmask = nullptr;
    if (bwd) { l.pmask = reinterpret_cast<unsigned long long*>(d); d += S; }
    float* f = reinterpret_cast<float*>(d);
    l.st = f; f += W * S + kSynWords * Y;
    l.gax = f; f += E; l.term = f; f += E;
    l.vnA = f; f += S; l.vnB = f; f += S;
    if (bwd) {
        l.s2 = f; f += 15 * S;
        l.lam = f; f += W * S + kSynWords * Y;   // the state's layout: segment words, then synapse words
        l.lphi = f; f += S; l.lI = f; f += S; l.mu = f; f += S; l.lvB = f; f += S;
        l.linp = f; f += S; l.lgdg = f; f += S; l.ldiag = f; f += S; l.edv = f; f += E;
        // the reverse tick's per-connection adjoints reuse the forward's flux buffers
        l.eca = reinterpret_cast<float*>(l.fa);
        l.ecb = reinterpret_cast<float*>(l.fb);
        // 16-byte aligned for the asynchronous copies
        f = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(f) + 15u) & ~(uintptr_t)15u);
        l.jsm = f; f += 51 * S;
    } else {
        l.s2 = l.lam = l.lphi = l.lI = l.mu = l.lvB = l.linp = l.lgdg = l.eca = l.ecb = l.edv = l.ldiag =
            l.jsm = nullptr;
    }
    return l;
}

// Per-CTA context, with this thread's segment and connection held in registers.
struct Ctx {
    uint32_t n, p;         // neuron, parameter set
    uint32_t s0, S, e0, E, y0, Y, soma;
    size_t st_off;         // this neuron's block within a set's state
    uint32_t L_n;          // block length
    // segment threadIdx.x (when < S): incident connections in original order, packed
    // as local id | other endpoint << 8 | (this is endpoint a) << 16 | intracellular << 17
    uint32_t g, ninc;
    uint32_t inc[kMaxInc];
    float cm, area;
    double vol;
    // connection threadIdx.x (when < E)
    uint32_t ea, eb;
    bool eintra;
    float earea, edist, eva, evb;
};

__device__ inline Ctx make_ctx(const AdjDev& d) {
    Ctx c;
    c.n = blockIdx.x;
    c.p = blockIdx.y;
    c.s0 = d.nr_seg[c.n]; c.S = d.nr_seg[c.n + 1] - c.s0;
    c.e0 = d.nr_edge[c.n]; c.E = d.nr_edge[c.n + 1] - c.e0;
    c.y0 = d.nr_slot[c.n]; c.Y = d.nr_slot[c.n + 1] - c.y0;
    c.soma = d.nr_soma[c.n];
    c.st_off = d.nr_st[c.n];
    c.L_n = d.nr_st[c.n + 1] - d.nr_st[c.n];
    const uint32_t tid = threadIdx.x;
    c.g = c.s0 + (tid < c.S ? tid : 0);
    c.ninc = 0;
#pragma unroll
    for (int k = 0; k < kMaxInc; k++) c.inc[k] = 0;
    c.cm = c.area = 0.0f;
    c.vol = 0.0;
    if (tid < c.S) {
        c.ninc = d.inc_n[c.g];
        c.cm = d.cm[c.g];
        c.area = d.area[c.g];
        c.vol = d.vol[c.g];
#pragma unroll
        for (int k = 0; k < kMaxInc; k++) {
            if ((uint32_t)k >= c.ninc) break;
            const uint32_t le = d.inc_e[c.g * kMaxInc + k];
            const uint32_t e = c.e0 + le;
            const bool isa = d.ed_a[e] == tid;
            const uint32_t o = isa ? d.ed_b[e] : d.ed_a[e];
            c.inc[k] = le | (o << 8) | ((uint32_t)isa << 16) | ((uint32_t)d.ed_intra[e] << 17);
        }
    }
    c.ea = c.eb = 0;
    c.eintra = false;
    c.earea = c.edist = c.eva = c.evb = 1.0f;
    if (tid < c.E) {
        const uint32_t e = c.e0 + tid;
        c.ea = d.ed_a[e]; c.eb = d.ed_b[e];
        c.eintra = d.ed_intra[e] != 0;
        c.earea = d.ed_area[e]; c.edist = d.ed_dist[e];
        c.eva = d.ed_vola[e]; c.evb = d.ed_volb[e];
    }
    return c;
}
__device__ inline uint32_t inc_le(uint32_t w) { return w & 0xFFu; }
__device__ inline uint32_t inc_o(uint32_t w) { return (w >> 8) & 0xFFu; }
__device__ inline bool inc_isa(uint32_t w) { return (w >> 16) & 1u; }
__device__ inline bool inc_intra(uint32_t w) { return (w >> 17) & 1u; }

// The block of a neuron: V[S], in[7][S], out[7][S], gate[4][S], then per synapse slot
// the receptor states and the cleft.  Shared memory keeps the stride Smax.
__device__ inline void block_load(float* dst, const float* src, const Ctx& c, uint32_t Smax, uint32_t W) {
    const uint32_t seg_words = W * c.S;
    for (uint32_t q = threadIdx.x; q < c.L_n; q += blockDim.x) {
        const uint32_t o = (q < seg_words) ? (q / c.S) * Smax + (q % c.S) : W * Smax + (q - seg_words);
        dst[o] = src[q];
    }
}
__device__ inline void block_store(float* dst, const float* src, const Ctx& c, uint32_t Smax, uint32_t W) {
    const uint32_t seg_words = W * c.S;
    for (uint32_t q = threadIdx.x; q < c.L_n; q += blockDim.x) {
        const uint32_t o = (q < seg_words) ? (q / c.S) * Smax + (q % c.S) : W * Smax + (q - seg_words);
        dst[q] = src[o];
    }
}

__device__ inline float bern_f(float x) {
    if (fabsf(x) < 1e-3f) return 1.0f - 0.5f * x;
    if (x > 50.0f) return 0.0f;
    if (x < -50.0f) return -x;
    return x / (dm_exp(x) - 1.0f);
}

__device__ inline float par_of(const AdjDev& d, uint32_t p, int cls, uint32_t g) {
    return d.par[((size_t)p * 3 + cls) * d.n_seg + g];
}
// the fitted conductance class of an item type (-1: Cav1.3 and the pump run with their
// network densities)
__device__ inline int cls_of(uint8_t type) {
    return type == 123 ? 1 : (type == 107 ? 2 : ((type == 141 || type == 142) ? 0 : -1));
}
__device__ inline int gates_of(uint8_t type) {
    return type == 123 ? 1 : ((type == 107 || type == 7) ? 0 : 2);
}
// the same for the fitting family's kernels (Nav, Kv_DR, K2P only)
template <bool kFull> __device__ inline int cls_k(uint8_t type) {
    return kFull ? cls_of(type) : (type == 123 ? 1 : (type == 107 ? 2 : 0));
}
template <bool kFull> __device__ inline int gates_k(uint8_t type) {
    return kFull ? gates_of(type) : (type == 123 ? 1 : (type == 107 ? 0 : 2));
}
__device__ inline float den_of(const AdjDev& d, uint32_t p, uint8_t type, uint32_t g, uint32_t j) {
    const int cls = cls_of(type);
    return cls >= 0 ? par_of(d, p, cls, g) : d.it_den[g * kItems + j];
}

// the logged cleft entries of `slot` at `tick` (sorted by tick, then the order the
// tick added them)
__device__ inline float cleft_events(const AdjDev& d, uint32_t slot, unsigned long long tick, float cleft) {
    uint32_t lo = d.ev_off[slot], hi = d.ev_off[slot + 1];
    const uint32_t end = hi;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (d.ev_tick[mid] < tick) lo = mid + 1; else hi = mid;
    }
    for (uint32_t q = lo; q < end && d.ev_tick[q] == tick; q++) cleft += d.ev_amt[q];
    return cleft;
}

// One differentiable item (kernel_dispatch.h:337-570 for its type), out of line so the
// forward tick and the reverse tick's re-run share one copy of each model.
__device__ __noinline__ double run_slot(uint8_t type, DMod& m, DSeg& s, float dt) {
    if (type == 123) return dp_kvdr_current<false>(m, s, dt);
    if (type == 107) return dp_k2p_current<false>(m, s, dt);
    if (type == 1) return dp_cav13_current<false>(m, s, dt);
    if (type == 7) return dp_nak_pump_current(m, s, dt);
    return dp_nav_current<false>(m, s, dt, type == 142 ? 1 : 0);
}

// Step 1 for this thread's segment: the differentiable items in slot order, then the
// current stimuli (simulation_host.cpp:234-303).
// kFull: the Cav1.3 / Na/K pump / ATP code is compiled in (networks with those items);
// without it the kernels hold only the fitting family's code paths.
template <bool kFull>
__device__ inline double step1_seg(const AdjDev& d, const Ctx& c, const Lay& L, unsigned long long tick, float dt,
                                   float* pre) {
    const uint32_t Sm = d.Smax;
    const uint32_t i = threadIdx.x;
    const uint32_t g = c.g;
    float* st = L.st;
    DSeg s;
    s.V = st[i];
#pragma unroll
    for (int q = 0; q < 7; q++) { s.in[q] = st[(1 + q) * Sm + i]; s.out[q] = st[(8 + q) * Sm + i]; }
    s.atp = (kFull && d.has_atp) ? st[d.atp_w * Sm + i] : 0.0f;
    s.area = c.area;
    s.vol = c.vol;
    ghk_cache_fill(s.gc, s.V);
    double I_total = 0.0;
    const uint32_t ni = d.n_it[g];
    for (uint32_t j = 0; j < ni; j++) {
        constexpr uint32_t IS = ItemStride<kFull>::v;
        const uint8_t type = d.it_type[g * IS + j];
        const uint32_t go = d.it_gate[g * IS + j];
        DMod m;
        m.den = kFull ? den_of(d, c.p, type, g, j) : par_of(d, c.p, cls_k<kFull>(type), g);
#pragma unroll
        for (int k = 0; k < 7; k++) m.st[k] = d.it_st[((size_t)g * IS + j) * 7 + k];
        m.area = s.area;
        m.av = 0;
        const int ng = gates_k<kFull>(type);
        if (ng > 0) m.st[0] = st[(15 + go) * Sm + i];
        if (ng > 1) m.st[1] = st[(16 + go) * Sm + i];
        if (pre) {   // the item's inputs, for the reverse tick
            pre[(j * 5 + 0) * Sm + i] = s.V;
            if (kFull && type == 7) {   // the pump: Na_in, K_out, ATP
                pre[(j * 5 + 1) * Sm + i] = s.in[0];
                pre[(j * 5 + 2) * Sm + i] = s.out[1];
                pre[(j * 5 + 3) * Sm + i] = s.atp;
                pre[(j * 5 + 4) * Sm + i] = 0.0f;
            } else {   // the item's ion by selects (an index would move s.in / s.out to local memory)
                const bool ca = kFull && type == 1, na = ng == 2 && !ca;
                pre[(j * 5 + 1) * Sm + i] = m.st[0];
                pre[(j * 5 + 2) * Sm + i] = m.st[1];
                pre[(j * 5 + 3) * Sm + i] = ca ? s.in[2] : (na ? s.in[0] : s.in[1]);
                pre[(j * 5 + 4) * Sm + i] = ca ? s.out[2] : (na ? s.out[0] : s.out[1]);
            }
        }
        I_total += run_slot(type, m, s, dt);
        if (ng > 0) st[(15 + go) * Sm + i] = m.st[0];
        if (ng > 1) st[(16 + go) * Sm + i] = m.st[1];
    }
    for (uint32_t q = d.stim_off[g]; q < d.stim_off[g + 1]; q++)
        if (tick >= d.stim_b[q] && tick < d.stim_e[q]) I_total += d.stim_amp[q];
    st[i] = s.V;
#pragma unroll
    for (int q = 0; q < 7; q++) { st[(1 + q) * Sm + i] = s.in[q]; st[(8 + q) * Sm + i] = s.out[q]; }
    if (kFull && d.has_atp) st[d.atp_w * Sm + i] = s.atp;
    return I_total;
}

// Scratch of one CTA: intracellular sub-step starts, Jacobi
// iterates, extracellular sub-step starts, synapse pre-states.
struct Scr {
    float* pre;       // [kItems][5][Sm]  V, gate 0, gate 1, c_in, c_out before each item
    float* istart;    // [5][8][Sm]  V, in[7]
    float* jac;       // [5][51][Sm]
    float* phs;       // [51][Sm]    phi_e before each of its sweeps
    float* estart;    // [6][7][Sm]  out before each extra sub-step and before the bath
    float* syn;       // [Ymax][kSynScr] in[7] before the synapse, receptor open probabilities, NMDA gates
    float* atpf;      // [Sm]        ATP before the Fick pass
};
// items: the item stride of the kernels; atp: whether the ATP row is recorded
__host__ __device__ inline size_t scr_floats(uint32_t S, uint32_t Y, uint32_t items, bool atp) {
    return ((size_t)40 * S + (size_t)255 * S + (size_t)51 * S + (size_t)42 * S + (size_t)kSynScr * Y + (size_t)items * 5 * S +
            (atp ? S : 0u) + 4 + 3) & ~(size_t)3;
}
template <bool kFull>
__device__ inline Scr make_scr(const AdjDev& d) {
    Scr s;
    float* base = d.scr + (size_t)(blockIdx.y * gridDim.x + blockIdx.x) * d.scr_floats;
    const uint32_t S = d.Smax;
    float* f = base;
    s.istart = f; f += 40 * S;
    s.jac = f; f += 255 * S;
    s.phs = f; f += 51 * S;
    s.estart = f; f += 42 * S;
    s.syn = f; f += kSynScr * d.Ymax;
    s.pre = f; f += (size_t)ItemStride<kFull>::v * 5 * S;
    s.atpf = f;
    return s;
}

// One tick of the neuron in shared memory; each kernel has one call site, so one copy.
// kRec records the intermediates the reverse
// tick reads (into L.s2, L.ib3, L.pmask and the CTA's scratch).
template <bool kFull>
__device__ __forceinline__ void tick_fwd(const AdjDev& d, const Ctx& c, const Lay& L, const Scr& sc, uint32_t t,
                                         bool kRec) {
    const uint32_t tid = threadIdx.x;
    const uint32_t S = c.S, E = c.E, Sm = d.Smax, Em = d.Emax;
    const bool seg = tid < S, edge = tid < E;
    const float dt = d.dt;
    const float dt_sub = dt / 5;
    const unsigned long long tick = d.tick0 + t;
    float* st = L.st;

    // ---- step 1 ----
    if (seg) L.ibuf[tid] = step1_seg<kFull>(d, c, L, tick, dt, kRec ? sc.pre : nullptr);
    __syncthreads();

    // ---- step 2.5 (diffusion_kernel.h:115-364) ----
    if (d.has_conn) {
        // phi_e (diffusion_kernel.h:41-104)
        if (seg) {
            double sacc = 0.0;
            for (int q = 0; q < 7; q++) sacc += c_z2d[q] * (double)st[(8 + q) * Sm + tid];
            L.sig[tid] = 3.612f * sacc;
            L.diag[tid] = L.sig[tid] * c.area / 1.0f;
            L.phiA[tid] = 0.0;
        }
        __syncthreads();
        if (edge) L.god[tid] = 0.5 * (L.sig[c.ea] + L.sig[c.eb]) * c.earea / c.edist;
        __syncthreads();
        double diag = 0.0, ib = 0.0;
        if (seg) {
            diag = L.diag[tid];
#pragma unroll
            for (int k = 0; k < kMaxInc; k++) {
                if ((uint32_t)k >= c.ninc) break;
                diag += L.god[inc_le(c.inc[k])];
            }
            L.diag[tid] = diag;
            ib = L.ibuf[tid];
        }
        double* ph = L.phiA;
        double* pn = L.phiB;
        unsigned long long unclamped = 0ull;
        for (int it = 0; it < 50; it++) {
            if (seg) {
                if (kRec) sc.phs[it * Sm + tid] = (float)ph[tid];
                double acc = 0.0;
#pragma unroll
                for (int k = 0; k < kMaxInc; k++) {
                    if ((uint32_t)k >= c.ninc) break;
                    const double gg = L.god[inc_le(c.inc[k])];
                    if (gg <= 0.0) continue;
                    acc += gg * ph[inc_o(c.inc[k])];
                }
                double v = (diag > 1e-9) ? (acc - ib) / diag : 0.0;
                if (kRec && diag > 1e-9 && v >= -10.0 && v <= 10.0) unclamped |= 1ull << it;
                if (v > 10.0) v = 10.0;
                if (v < -10.0) v = -10.0;
                pn[tid] = v;
            }
            __syncthreads();
            double* tmp = ph; ph = pn; pn = tmp;
        }
        // 50 sweeps: the final phi is in phiA
        const double* phi = ph;
        if (kRec && seg) L.pmask[tid] = unclamped;

        // intracellular Nernst-Planck, 5 sub-steps (diffusion_kernel.h:152-238)
        float C_dt = 1.0f;
        if (seg) {
            C_dt = c.cm / dt_sub;
            if (C_dt < 1e-9f) C_dt = 1e-9f;
        }
        for (int sub = 0; sub < 5; sub++) {
            if (kRec && seg) {
                sc.istart[(sub * 8) * Sm + tid] = st[tid];
                for (int q = 0; q < 7; q++) sc.istart[(sub * 8 + 1 + q) * Sm + tid] = st[(1 + q) * Sm + tid];
            }
            if (edge && c.eintra) {
                const uint32_t a = c.ea, b = c.eb;
                float sigma_i = 0.0f;
                for (int q = 0; q < 7; q++) {
                    float C_bar = (float)(0.5f * ((double)st[(1 + q) * Sm + a] + (double)st[(1 + q) * Sm + b]));
                    sigma_i += c_z2d[q] * C_bar;
                }
                const float g_ax = 3.612f * sigma_i * c.earea / c.edist;
                const float dV = (float)(((double)st[a] + phi[a]) - ((double)st[b] + phi[b]));
                float I_np = 0.0f;
                for (int q = 0; q < 7; q++) {
                    const float C_a = st[(1 + q) * Sm + a], C_b = st[(1 + q) * Sm + b];
                    const float x = c_z[q] * 0.03742f * dV;
                    const float flux = c_D[q] * c.earea * dt_sub / c.edist * (C_a * bern_f(-x) - C_b * bern_f(x));
                    L.fa[q * Em + tid] = (double)flux / c.eva;
                    L.fb[q * Em + tid] = (double)flux / c.evb;
                    I_np += c_z[q] * 96.485f * flux / dt_sub;
                }
                L.gax[tid] = g_ax;
                L.term[tid] = I_np - g_ax * dV;
            }
            __syncthreads();
            float gd = 0.0f, ip = 0.0f, vold = 0.0f;
            double ac[7];
            for (int q = 0; q < 7; q++) ac[q] = 0.0;
            if (seg) {
#pragma unroll
                for (int k = 0; k < kMaxInc; k++) {
                    if ((uint32_t)k >= c.ninc) break;
                    const uint32_t w = c.inc[k];
                    if (!inc_intra(w)) continue;
                    const uint32_t le = inc_le(w);
                    gd += L.gax[le];
                    if (inc_isa(w)) {
                        ip += L.term[le];
                        for (int q = 0; q < 7; q++) ac[q] -= L.fa[q * Em + le];
                    } else {
                        ip -= L.term[le];
                        for (int q = 0; q < 7; q++) ac[q] += L.fb[q * Em + le];
                    }
                }
                vold = st[tid];
                L.vnA[tid] = vold;
            }
            __syncthreads();
            float* vn = L.vnA;
            float* vx = L.vnB;
            const float den = C_dt + gd;
            for (int it = 0; it < 50; it++) {
                if (seg) {
                    if (kRec) sc.jac[(sub * 51 + it) * Sm + tid] = vn[tid];
                    float offd = 0.0f;
#pragma unroll
                    for (int k = 0; k < kMaxInc; k++) {
                        if ((uint32_t)k >= c.ninc) break;
                        const uint32_t w = c.inc[k];
                        if (!inc_intra(w)) continue;
                        offd += L.gax[inc_le(w)] * vn[inc_o(w)];
                    }
                    vx[tid] = (C_dt * vold + ip + offd) / den;
                }
                __syncthreads();
                float* tmp = vn; vn = vx; vx = tmp;
            }
            if (seg) {
                if (kRec) sc.jac[(sub * 51 + 50) * Sm + tid] = vn[tid];
                st[tid] = vn[tid];
                for (int q = 0; q < 7; q++)
                    st[(1 + q) * Sm + tid] = (float)((double)st[(1 + q) * Sm + tid] + (double)(float)ac[q]);
            }
            __syncthreads();
        }

        // extracellular Nernst-Planck, 5 sub-steps (diffusion_kernel.h:244-281); the
        // Bernoulli factors depend on phi_e only
        float bm[7], bp[7];
        if (edge) {
            const double dphi = phi[c.ea] - phi[c.eb];
            for (int q = 0; q < 7; q++) {
                const float x = (float)(c_z[q] * 0.03742f * dphi);
                bm[q] = bern_f(-x);
                bp[q] = bern_f(x);
            }
        }
        const float vea = c.eva * EXTRA_VOLUME_RATIO, veb = c.evb * EXTRA_VOLUME_RATIO;
        for (int sub = 0; sub < 5; sub++) {
            if (kRec && seg)
                for (int q = 0; q < 7; q++) sc.estart[(sub * 7 + q) * Sm + tid] = st[(8 + q) * Sm + tid];
            if (edge) {
                for (int q = 0; q < 7; q++) {
                    const double Ca = st[(8 + q) * Sm + c.ea], Cb = st[(8 + q) * Sm + c.eb];
                    const double flux = c_D[q] * c.earea * dt_sub / c.edist * (Ca * bm[q] - Cb * bp[q]);
                    L.fa[q * Em + tid] = flux / vea;
                    L.fb[q * Em + tid] = flux / veb;
                }
            }
            __syncthreads();
            if (seg) {
                double ac[7];
                for (int q = 0; q < 7; q++) ac[q] = 0.0;
#pragma unroll
                for (int k = 0; k < kMaxInc; k++) {
                    if ((uint32_t)k >= c.ninc) break;
                    const uint32_t w = c.inc[k];
                    const uint32_t le = inc_le(w);
                    if (inc_isa(w)) for (int q = 0; q < 7; q++) ac[q] -= L.fa[q * Em + le];
                    else for (int q = 0; q < 7; q++) ac[q] += L.fb[q * Em + le];
                }
                for (int q = 0; q < 7; q++) st[(8 + q) * Sm + tid] = (float)((double)st[(8 + q) * Sm + tid] + ac[q]);
            }
            __syncthreads();
        }
        // ATP (diffusion_kernel.h:284-345): on each intracellular connection whose ATP
        // difference exceeds 1e-12, flux = 0.14 area dC dt / dist in float, left to right;
        // each segment adds -+flux / its volume in connection order
        if (kFull && d.has_atp) {   // without a pump ATP is uniform in time, and the pass moves nothing
        if (kRec && seg) sc.atpf[tid] = st[d.atp_w * Sm + tid];
        if (edge) {
            float fl = 0.0f, on = 0.0f;
            if (c.eintra) {
                const float dC = st[d.atp_w * Sm + c.ea] - st[d.atp_w * Sm + c.eb];
                if (dC > 1e-12f || dC < -1e-12f) {
                    fl = 0.14f * c.earea * dC * dt / c.edist;
                    on = 1.0f;
                }
            }
            L.gax[tid] = fl;
            L.term[tid] = on;
        }
        __syncthreads();
        if (seg) {
            float vf = (float)c.vol;
            if (vf < 1e-6f) vf = 1e-6f;
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < kMaxInc; k++) {
                if ((uint32_t)k >= c.ninc) break;
                const uint32_t w = c.inc[k];
                const uint32_t le = inc_le(w);
                if (L.term[le] == 0.0f) continue;
                if (inc_isa(w)) acc -= L.gax[le] / vf;
                else acc += L.gax[le] / vf;
            }
            st[d.atp_w * Sm + tid] = st[d.atp_w * Sm + tid] + acc;
        }
        __syncthreads();
        }
        // bath relaxation and clamp of the extracellular ions (diffusion_kernel.h:348-360)
        if (seg) {
            if (kRec)
                for (int q = 0; q < 7; q++) sc.estart[(5 * 7 + q) * Sm + tid] = st[(8 + q) * Sm + tid];
            for (int q = 0; q < 7; q++) {
                double e = (double)st[(8 + q) * Sm + tid];
                e += (c_bath[q] - e) * dt / 1.0f;
                if (e < 1e-9) e = 1e-9;
                if (e > 1000.0) e = 1000.0;
                st[(8 + q) * Sm + tid] = (float)e;
            }
        }
        __syncthreads();
    }

    // ---- step 3 (simulation_host.cpp:322-593) and step 4 (:596-649), thread = post segment ----
    if (seg) {
        if (kRec)
            for (int q = 0; q < 15; q++) L.s2[q * Sm + tid] = st[q * Sm + tid];
        const uint32_t g = c.g;
        double ib = L.ibuf[tid];
        float nt_glu = 0.0f, nt_gaba = 0.0f, nt_gly = 0.0f;
        DSeg s;
        s.V = st[tid];
        for (int q = 0; q < 7; q++) { s.in[q] = st[(1 + q) * Sm + tid]; s.out[q] = st[(8 + q) * Sm + tid]; }
        s.atp = 0.0f;
        s.area = c.area;
        s.vol = c.vol;
        ghk_cache_fill(s.gc, s.V);
        float* rs = st + (kFull ? d.W : kW3) * Sm;
        for (uint32_t y = d.sp_off[g]; y < d.sp_off[g + 1]; y++) {
            const uint32_t ly = y - c.y0;
            float cleft = cleft_events(d, y, tick, rs[ly * kSynWords + 4]);
            if (d.sl_nt[y] == 0) nt_glu += cleft;
            else if (d.sl_nt[y] == 1) nt_gaba += cleft;
            else nt_gly += cleft;
            if (kRec) for (int q = 0; q < 7; q++) sc.syn[ly * kSynScr + q] = s.in[q];
            float I_syn = 0.0f;
            const float scale = d.w[(size_t)c.p * d.n_syn + d.sl_syn[y]];
            const float parea = d.sl_parea[y];
            for (uint32_t j = 0; j < d.sl_nrec[y]; j++) {
                const int kind = d.sl_kind[y * kRecPerSyn + j];
                DMod m;
                m.den = d.sl_rden[y * kRecPerSyn + j];
                const bool nmda = kind == 1;
                m.st[0] = rs[ly * kSynWords + 2 * j];
                m.st[1] = nmda ? 0.0f : rs[ly * kSynWords + 2 * j + 1];
                m.st[2] = nmda ? rs[ly * kSynWords + 2 * j + 1] : 0.0f;
                m.st[3] = m.st[4] = m.st[5] = m.st[6] = 0.0f;
                if (kRec && nmda) sc.syn[ly * kSynScr + 9 + j] = m.st[2];
                m.area = (parea > 0.0f) ? parea : s.area;
                m.av = d.sl_rav[y * kRecPerSyn + j];
                const float ntr = kind <= 1 ? nt_glu : (kind == 2 ? nt_gaba : nt_gly);
                I_syn = (float)(I_syn + receptor_current(gRec[kind], m, s, dt, ntr, scale));
                rs[ly * kSynWords + 2 * j] = m.st[0];
                rs[ly * kSynWords + 2 * j + 1] = nmda ? m.st[2] : m.st[1];
                if (kRec) sc.syn[ly * kSynScr + 7 + j] = m.st[0] * (1.0f - m.st[1]);
            }
            ib += I_syn;
            cleft *= dm_exp(-dt / d.sl_tauc[y]);
            if (cleft < 0.0f) cleft = 0.0f;
            rs[ly * kSynWords + 4] = cleft;
        }
        if (kRec) L.ib3[tid] = ib;
        float V = s.V;
        if (ib != ib) ib = 0.0f;
        if (ib > 10000.0f) ib = 10000.0f;
        if (ib < -10000.0f) ib = -10000.0f;
        float dV = (float)(ib / c.cm * dt);
        if (dV > 50.0f) dV = 50.0f;
        if (dV < -50.0f) dV = -50.0f;
        V = (float)((double)V + dV);
        if (V != V) V = -65.0f;
        else {
            if (V < -120.0f) V = -120.0f;
            if (V > 150.0f) V = 150.0f;
        }
        st[tid] = V;
        for (int q = 0; q < 7; q++) st[(1 + q) * Sm + tid] = s.in[q];
    }
    __syncthreads();
}

// Reverse of tick t.  On entry L.st holds the state
// after the recorded re-run, L.s2 / L.ib3 / L.ibuf / L.pmask and the scratch the
// intermediates, and L.lam the adjoint of the state after the tick (V, ions, gates).
// On exit L.lam holds the adjoint of the starting state; gp accumulates
// d loss / d (gNa, gK, gleak) of this thread's segment.
template <bool kFull>
__device__ void tick_rev(const AdjDev& d, const Ctx& c, const Lay& L, const Scr& sc, uint32_t t, double* gp) {
    const uint32_t tid = threadIdx.x;
    const uint32_t S = c.S, E = c.E, Sm = d.Smax, Em = d.Emax;
    const bool seg = tid < S, edge = tid < E;
    const float dt = d.dt;
    const float dt_sub = dt / 5;
    float* lam = L.lam;

    // loss: (1 / (samples * neurons)) * sum (V_soma - target)^2 after each sampled tick
    if ((t + 1) % d.stride == 0 && tid == c.soma) {
        const uint32_t smp = (t + 1) / d.stride - 1;
        const double diff = (double)L.st[c.soma] - (double)d.target[(size_t)smp * d.nn + c.n];
        lam[c.soma] += (float)(2.0 * diff / ((double)d.n_samples * (double)d.nn));
    }

    // ---- step 4 and step 3 reversed (thread = post segment) ----
    if (seg) {
        const uint32_t g = c.g;
        const double ib = L.ib3[tid];
        const float V2 = L.s2[tid];
        const float lV = lam[tid];
        // step 4: V' = clamp(V2 + clamp((float)(clamp(ib) / C_m * dt)))
        double ibc = ib;
        bool m_ib = true;
        if (ibc != ibc) { ibc = 0.0; m_ib = false; }
        if (ibc > 10000.0f) { ibc = 10000.0f; m_ib = false; }
        if (ibc < -10000.0f) { ibc = -10000.0f; m_ib = false; }
        float dV = (float)(ibc / c.cm * dt);
        bool m_dv = true;
        if (dV > 50.0f) { dV = 50.0f; m_dv = false; }
        if (dV < -50.0f) { dV = -50.0f; m_dv = false; }
        const float Vn = (float)((double)V2 + dV);
        const bool m_v = (Vn == Vn) && Vn >= -120.0f && Vn <= 150.0f;
        const float lVn = m_v ? lV : 0.0f;
        float lV2 = lVn;
        const float lib = (m_dv && m_ib) ? (float)((double)lVn * dt / c.cm) : 0.0f;
        // step 3: receptors of the segment's synapses, last first
        float lin[7], lout[7], out2[7];
        for (int q = 0; q < 7; q++) {
            lin[q] = lam[(1 + q) * Sm + tid];
            lout[q] = lam[(8 + q) * Sm + tid];
            out2[q] = L.s2[(8 + q) * Sm + tid];
        }
        for (int y = (int)d.sp_off[g + 1] - 1; y >= (int)d.sp_off[g]; y--) {
            const uint32_t ly = (uint32_t)y - c.y0;
            const uint32_t nrec = d.sl_nrec[y];
            const uint32_t syn = d.sl_syn[y];
            const float wv = d.w[(size_t)c.p * d.n_syn + syn];
            const float parea = d.sl_parea[y];
            const float area = (parea > 0.0f) ? parea : c.area;
            // the ions before each receptor of the synapse (receptor 0: recorded)
            float pre[kRecPerSyn][7];
            for (int q = 0; q < 7; q++) pre[0][q] = sc.syn[ly * kSynScr + q];
            for (uint32_t j = 0; j + 1 < nrec; j++) {
                const int kind = d.sl_kind[y * kRecPerSyn + j];
                const RecKind& K = gRec[kind];
                const float open = sc.syn[ly * kSynScr + 7 + j];
                for (int q = 0; q < 7; q++) pre[j + 1][q] = pre[j][q];
                if (kind == 1) {
                    const double z5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                    double zx[9];
                    float nv[3];
                    adj::vjp_nmda(z5, zx, K.P_Na, K.P_K, K.P_Ca, V2, pre[j], out2, wv, d.sl_rden[y * kRecPerSyn + j],
                                  area, open, sc.syn[ly * kSynScr + 9 + j], c.vol, dt, nv);
                    pre[j + 1][0] = nv[0]; pre[j + 1][1] = nv[1]; pre[j + 1][2] = nv[2];
                } else {
                    double z4[4] = {0.0, 0.0, 0.0, 0.0}, zx[8];
                    float nv[3];
                    adj::vjp_receptor(z4, zx, K.is_anion, K.is_anion ? K.P_Cl : K.P_Na, K.P_K, V2, pre[j], out2, wv,
                                      d.sl_rden[y * kRecPerSyn + j], area, open, c.vol, dt, nv);
                    pre[j + 1][0] = nv[0]; pre[j + 1][1] = nv[1]; pre[j + 1][3] = nv[2];
                }
            }
            // the adjoints of the synapse's state words (an NMDA receptor's inactivation gate)
            float* lsy = lam + (kFull ? d.W : kW3) * Sm + ly * kSynWords;
            double gw = 0.0;
            for (int j = (int)nrec - 1; j >= 0; j--) {
                const int kind = d.sl_kind[y * kRecPerSyn + j];
                const RecKind& K = gRec[kind];
                const float open = sc.syn[ly * kSynScr + 7 + j];
                float nv[3];
                if (kind == 1) {
                    const double l5[5] = {(double)lin[0], (double)lin[1], (double)lin[2], (double)lib,
                                          (double)lsy[2 * j + 1]};
                    double lx[9];
                    adj::vjp_nmda(l5, lx, K.P_Na, K.P_K, K.P_Ca, V2, pre[j], out2, wv, d.sl_rden[y * kRecPerSyn + j],
                                  area, open, sc.syn[ly * kSynScr + 9 + j], c.vol, dt, nv);
                    lV2 += (float)lx[0];
                    lin[0] = (float)lx[1]; lin[1] = (float)lx[2]; lin[2] = (float)lx[3];
                    lout[0] += (float)lx[4]; lout[1] += (float)lx[5]; lout[2] += (float)lx[6];
                    gw += lx[7];
                    lsy[2 * j + 1] = (float)lx[8];
                } else {
                    const double l4[4] = {(double)lin[0], (double)lin[1], (double)lin[3], (double)lib};
                    double lx[8];
                    adj::vjp_receptor(l4, lx, K.is_anion, K.is_anion ? K.P_Cl : K.P_Na, K.P_K, V2, pre[j], out2, wv,
                                      d.sl_rden[y * kRecPerSyn + j], area, open, c.vol, dt, nv);
                    lV2 += (float)lx[0];
                    lin[0] = (float)lx[1]; lin[1] = (float)lx[2]; lin[3] = (float)lx[3];
                    lout[0] += (float)lx[4]; lout[1] += (float)lx[5]; lout[3] += (float)lx[6];
                    gw += lx[7];
                }
            }
            d.g_w[(size_t)c.p * d.n_syn + syn] += gw;
        }
        lam[tid] = lV2;
        for (int q = 0; q < 7; q++) { lam[(1 + q) * Sm + tid] = lin[q]; lam[(8 + q) * Sm + tid] = lout[q]; }
        L.lI[tid] = lib;
        L.lphi[tid] = 0.0f;
    }
    __syncthreads();

    if (d.has_conn) {
        const double* phiF = L.phiA;   // phi_e after the solve (the re-run leaves it here)
        // ---- bath relaxation ----
        if (seg) {
            for (int q = 0; q < 7; q++) {
                const double e = (double)sc.estart[(5 * 7 + q) * Sm + tid];
                const double e2 = e + (c_bath[q] - e) * dt / 1.0f;
                const bool m = e2 >= 1e-9 && e2 <= 1000.0;
                lam[(8 + q) * Sm + tid] = m ? (float)((double)lam[(8 + q) * Sm + tid] * (1.0 - (double)dt)) : 0.0f;
            }
        }
        __syncthreads();
        // ---- the ATP Fick pass reversed: atp_a -= f / v_a, atp_b += f / v_b with
        // f = c (atp_a - atp_b) on the connections that passed the threshold ----
        if (kFull && d.has_atp) {
        if (edge) {
            float v = 0.0f;
            if (c.eintra) {
                const float dC = sc.atpf[c.ea] - sc.atpf[c.eb];
                if (dC > 1e-12f || dC < -1e-12f) {
                    const float lfl = -lam[d.atp_w * Sm + c.ea] / c.eva + lam[d.atp_w * Sm + c.eb] / c.evb;
                    v = lfl * (0.14f * c.earea * dt / c.edist);
                }
            }
            L.edv[tid] = v;
        }
        __syncthreads();
        if (seg) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < kMaxInc; k++) {
                if ((uint32_t)k >= c.ninc) break;
                const uint32_t w = c.inc[k];
                acc += inc_isa(w) ? L.edv[inc_le(w)] : -L.edv[inc_le(w)];
            }
            lam[d.atp_w * Sm + tid] += acc;
        }
        __syncthreads();
        }
        // ---- extracellular sub-steps, last first ----
        float elphi = 0.0f;
        float bm[7], bp[7], dbm[7], dbp[7], kq[7];
        if (edge) {
            const double dphi = phiF[c.ea] - phiF[c.eb];
            for (int q = 0; q < 7; q++) {
                const float x = (float)(c_z[q] * 0.03742f * dphi);
                adj::bern_pair(x, dm_expf(x), &bp[q], &dbp[q]);
                bm[q] = bp[q] + x;
                dbm[q] = -(dbp[q] + 1.0f);
                kq[q] = c_D[q] * c.earea * dt_sub / c.edist;
            }
        }
        const float rvea = 1.0f / (c.eva * EXTRA_VOLUME_RATIO), rveb = 1.0f / (c.evb * EXTRA_VOLUME_RATIO);
        for (int sub = 4; sub >= 0; sub--) {
            if (edge) {
                for (int q = 0; q < 7; q++) {
                    const float Ca = sc.estart[(sub * 7 + q) * Sm + c.ea], Cb = sc.estart[(sub * 7 + q) * Sm + c.eb];
                    const float lf = -lam[(8 + q) * Sm + c.ea] * rvea + lam[(8 + q) * Sm + c.eb] * rveb;
                    L.eca[q * Em + tid] = lf * kq[q] * bm[q];
                    L.ecb[q * Em + tid] = -lf * kq[q] * bp[q];
                    elphi += lf * kq[q] * (-Ca * dbm[q] - Cb * dbp[q]) * (c_z[q] * 0.03742f);
                }
            }
            __syncthreads();
            if (seg) {
#pragma unroll
                for (int k = 0; k < kMaxInc; k++) {
                    if ((uint32_t)k >= c.ninc) break;
                    const uint32_t w = c.inc[k];
                    const uint32_t le = inc_le(w);
                    const float* src = inc_isa(w) ? L.eca : L.ecb;
                    for (int q = 0; q < 7; q++) lam[(8 + q) * Sm + tid] += src[q * Em + le];
                }
            }
            __syncthreads();
        }
        if (edge) L.edv[tid] = elphi;
        __syncthreads();
        if (seg) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < kMaxInc; k++) {
                if ((uint32_t)k >= c.ninc) break;
                const uint32_t w = c.inc[k];
                acc += inc_isa(w) ? L.edv[inc_le(w)] : -L.edv[inc_le(w)];
            }
            L.lphi[tid] += acc;
        }
        __syncthreads();

        // ---- intracellular sub-steps, last first ----
        float C_dt = 1.0f;
        if (seg) {
            C_dt = c.cm / dt_sub;
            if (C_dt < 1e-9f) C_dt = 1e-9f;
        }
        for (int sub = 4; sub >= 0; sub--) {
            const float* Vs = sc.istart + (size_t)(sub * 8) * Sm;
            const float* Is = sc.istart + (size_t)(sub * 8 + 1) * Sm;   // [7][Sm]
            const float* jac = sc.jac + (size_t)(sub * 51) * Sm;
            float gax = 0.0f, dVe = 0.0f;
            if (edge && c.eintra) {
                float sigma_i = 0.0f;
                for (int q = 0; q < 7; q++) {
                    float C_bar = (float)(0.5f * ((double)Is[q * Sm + c.ea] + (double)Is[q * Sm + c.eb]));
                    sigma_i += c_z2d[q] * C_bar;
                }
                gax = 3.612f * sigma_i * c.earea / c.edist;
                dVe = (float)(((double)Vs[c.ea] + phiF[c.ea]) - ((double)Vs[c.eb] + phiF[c.eb]));
            }
            if (edge) L.gax[tid] = gax;
            __syncthreads();
            float gdiag = 0.0f, lVold = 0.0f, linp = 0.0f, lgdg = 0.0f;
            if (seg) {
#pragma unroll
                for (int k = 0; k < kMaxInc; k++) {
                    if ((uint32_t)k >= c.ninc) break;
                    const uint32_t w = c.inc[k];
                    if (inc_intra(w)) gdiag += L.gax[inc_le(w)];
                }
            }
            const float rden = 1.0f / (C_dt + gdiag);
            // the sub-step's 51 iterates into shared memory: asynchronous 16-byte copies, all
            // in flight at once (the stride Sm is a multiple of 4, the scratch 16-byte aligned)
            {
                const float4* src4 = reinterpret_cast<const float4*>(jac);
                float4* dst4 = reinterpret_cast<float4*>(L.jsm);
                for (uint32_t q = tid; q < 51u * Sm / 4u; q += blockDim.x) __pipeline_memcpy_async(dst4 + q, src4 + q, 16);
                __pipeline_commit();
                __pipeline_wait_prior(0);
            }
            __syncthreads();
            // one barrier per sweep: this thread's adjoint stays in a register, the mu of
            // consecutive sweeps alternate between two buffers
            float lgo = 0.0f;
            float lv = seg ? lam[tid] : 0.0f;
            const float* js = L.jsm;
            for (int k = 49; k >= 0; k--) {
                float* mu = (k & 1) ? L.lvB : L.mu;
                if (seg) {
                    const float m = lv * rden;
                    lVold += C_dt * m;
                    linp += m;
                    lgdg -= m * js[(k + 1) * Sm + tid];
                    mu[tid] = m;
                }
                __syncthreads();
                if (edge && c.eintra) lgo += mu[c.ea] * js[k * Sm + c.eb] + mu[c.eb] * js[k * Sm + c.ea];
                if (seg) {
                    float acc = 0.0f;
#pragma unroll
                    for (int q = 0; q < kMaxInc; q++) {
                        if ((uint32_t)q >= c.ninc) break;
                        const uint32_t w = c.inc[q];
                        if (!inc_intra(w)) continue;
                        acc += L.gax[inc_le(w)] * mu[inc_o(w)];
                    }
                    lv = acc;
                }
            }
            float lVs = 0.0f;
            if (seg) {
                lVs = lv + lVold;
                L.linp[tid] = linp;
                L.lgdg[tid] = lgdg;
            }
            __syncthreads();
            if (edge) {
                if (c.eintra) {
                    const uint32_t a = c.ea, b = c.eb;
                    const float dl = L.linp[a] - L.linp[b];
                    const float lgax = lgo + L.lgdg[a] + L.lgdg[b] - dl * dVe;
                    float ldV = -dl * gax;
                    const float gfac = lgax * (3.612f * c.earea / c.edist) * 0.5f;
                    const float rva = 1.0f / c.eva, rvb = 1.0f / c.evb, kk = c.earea * dt_sub / c.edist;
                    const float inp_f = dl * 96.485f / dt_sub;
                    for (int q = 0; q < 7; q++) {
                        const float Ca = Is[q * Sm + a], Cb = Is[q * Sm + b];
                        const float x = c_z[q] * 0.03742f * dVe;
                        const float k = c_D[q] * kk;
                        const float lf = inp_f * c_z[q] - lam[(1 + q) * Sm + a] * rva + lam[(1 + q) * Sm + b] * rvb;
                        float Bp, dBp;
                        adj::bern_pair(x, dm_expf(x), &Bp, &dBp);
                        const float Bm = Bp + x, dBm = -(dBp + 1.0f);
                        L.eca[q * Em + tid] = lf * k * Bm + gfac * c_z2d[q];
                        L.ecb[q * Em + tid] = -lf * k * Bp + gfac * c_z2d[q];
                        ldV += lf * k * (-Ca * dBm - Cb * dBp) * (c_z[q] * 0.03742f);
                    }
                    L.edv[tid] = ldV;
                } else {
                    L.edv[tid] = 0.0f;
                }
            }
            __syncthreads();
            if (seg) {
                float acc = 0.0f;
#pragma unroll
                for (int k = 0; k < kMaxInc; k++) {
                    if ((uint32_t)k >= c.ninc) break;
                    const uint32_t w = c.inc[k];
                    if (!inc_intra(w)) continue;
                    const uint32_t le = inc_le(w);
                    const bool isa = inc_isa(w);
                    acc += isa ? L.edv[le] : -L.edv[le];
                    const float* src = isa ? L.eca : L.ecb;
                    for (int q = 0; q < 7; q++) lam[(1 + q) * Sm + tid] += src[q * Em + le];
                }
                lam[tid] = lVs + acc;
                L.lphi[tid] += acc;
            }
            __syncthreads();
        }

        // ---- phi_e solve (one barrier per sweep, as above); which sweeps clamped was
        // recorded, and an unclamped sweep's value is the stored next iterate ----
        float ldg = 0.0f;
        float rdiag = 0.0f;
        unsigned long long pm = 0ull;
        float lp = 0.0f;
        if (seg) {
            lp = L.lphi[tid];
            rdiag = (float)(1.0 / L.diag[tid]);
            pm = L.pmask[tid];
        }
        float lI = seg ? L.lI[tid] : 0.0f;
        float lg = 0.0f;
        const double god = edge ? L.god[tid] : 0.0;
        const float godf = (float)god;
        // the recorded iterates into shared memory (the Jacobi staging area is free here)
        {
            const float4* src4 = reinterpret_cast<const float4*>(sc.phs);
            float4* dst4 = reinterpret_cast<float4*>(L.jsm);
            for (uint32_t q = tid; q < 50u * Sm / 4u; q += blockDim.x) __pipeline_memcpy_async(dst4 + q, src4 + q, 16);
            __pipeline_commit();
            __pipeline_wait_prior(0);
        }
        __syncthreads();
        const float* phs = L.jsm;
        for (int k = 49; k >= 0; k--) {
            const float* ph = phs + (size_t)k * Sm;
            float* mu = (k & 1) ? L.lvB : L.mu;
            if (seg) {
                float m = 0.0f;
                if ((pm >> k) & 1ull) {
                    m = lp * rdiag;
                    const float unc = (k == 49) ? (float)L.phiA[tid] : phs[(k + 1) * Sm + tid];
                    ldg -= m * unc;
                }
                lI -= m;
                mu[tid] = m;
            }
            __syncthreads();
            if (edge && god > 0.0) lg += mu[c.ea] * ph[c.eb] + mu[c.eb] * ph[c.ea];
            if (seg) {
                float acc = 0.0f;
#pragma unroll
                for (int q = 0; q < kMaxInc; q++) {
                    if ((uint32_t)q >= c.ninc) break;
                    const uint32_t w = c.inc[q];
                    const float gg = (float)L.god[inc_le(w)];
                    if (gg <= 0.0f) continue;
                    acc += gg * mu[inc_o(w)];
                }
                lp = acc;
            }
        }
        (void)godf;
        __syncthreads();
        if (seg) { L.ldiag[tid] = ldg; L.lI[tid] = lI; }
        __syncthreads();
        if (edge) {
            lg += L.ldiag[c.ea] + L.ldiag[c.eb];
            L.edv[tid] = (float)((double)lg * 0.5 * (double)c.earea / (double)c.edist);
        }
        __syncthreads();
        if (seg) {
            double lsig = (double)ldg * (double)c.area;
#pragma unroll
            for (int k = 0; k < kMaxInc; k++) {
                if ((uint32_t)k >= c.ninc) break;
                lsig += L.edv[inc_le(c.inc[k])];
            }
            for (int q = 0; q < 7; q++) lam[(8 + q) * Sm + tid] += (float)(lsig * 3.612 * (double)c_z2d[q]);
        }
        __syncthreads();
    }

    // ---- step 1 reversed (thread = segment): items last first, from the inputs the
    // recorded re-run kept ----
    if (seg) {
        const uint32_t g = c.g;
        const float lIt = L.lI[tid];
        const uint32_t ni = d.n_it[g];
        float lV = lam[tid];
        for (int j = (int)ni - 1; j >= 0; j--) {
            constexpr uint32_t IS = ItemStride<kFull>::v;
            const uint8_t type = d.it_type[g * IS + j];
            const uint32_t go = d.it_gate[g * IS + j];
            const float den = kFull ? den_of(d, c.p, type, g, j) : par_of(d, c.p, cls_k<kFull>(type), g);
            const float pV = sc.pre[(j * 5 + 0) * Sm + tid], pG0 = sc.pre[(j * 5 + 1) * Sm + tid],
                        pG1 = sc.pre[(j * 5 + 2) * Sm + tid], pCi = sc.pre[(j * 5 + 3) * Sm + tid],
                        pCo = sc.pre[(j * 5 + 4) * Sm + tid];
            if (kFull && type == 7) {   // the pump: inputs V, Na_in, K_out, ATP (recorded in that order)
                float lp[7] = {lV, lam[1 * Sm + tid], lam[8 * Sm + tid], lam[2 * Sm + tid], lam[9 * Sm + tid],
                               lam[d.atp_w * Sm + tid], lIt};
                adj::vjp_pump(lp, pV, pG0, pG1, pCi, den, c.area, c.vol, dt);
                lV = lp[0];
                lam[1 * Sm + tid] = lp[1];
                lam[9 * Sm + tid] = lp[4];
                lam[d.atp_w * Sm + tid] = lp[5];
                continue;
            }
            const int ion = (type == 141 || type == 142) ? 0 : ((kFull && type == 1) ? 2 : 1);
            const int cls = cls_k<kFull>(type);
            const float* pst = d.it_st + ((size_t)g * IS + j) * 7;
            const int ng = gates_k<kFull>(type);
            const float lo[6] = {lV,
                                 ng > 0 ? lam[(15 + go) * Sm + tid] : 0.0f,
                                 ng > 1 ? lam[(16 + go) * Sm + tid] : 0.0f,
                                 lam[(1 + ion) * Sm + tid],
                                 lam[(8 + ion) * Sm + tid],
                                 lIt};
            float lx[6];
            if (type == 123) adj::vjp_kvdr_f(lo, lx, pV, pG0, pCi, pCo, den, c.area, c.vol, dt, pst);
            else if (type == 107) adj::vjp_k2p_f(lo, lx, pV, pCi, pCo, den, c.area, c.vol, dt, pst);
            else if (kFull && type == 1) {   // out of line, through arrays of its own (lo / lx stay in registers)
                float lo1[6], lx1[6];
                for (int k = 0; k < 6; k++) lo1[k] = lo[k];
                adj::vjp_cav13(lo1, lx1, pV, pG0, pG1, pCi, pCo, den, c.area, c.vol, dt, pst);
                for (int k = 0; k < 6; k++) lx[k] = lx1[k];
            }
            else adj::vjp_nav_f(lo, lx, pV, pG0, pG1, pCi, pCo, den, c.area, c.vol, dt, type == 142 ? 1 : 0, pst[5]);
            lV = lx[0];
            if (ng > 0) lam[(15 + go) * Sm + tid] = lx[1];
            if (ng > 1) lam[(16 + go) * Sm + tid] = lx[2];
            lam[(1 + ion) * Sm + tid] = lx[3];
            lam[(8 + ion) * Sm + tid] = lx[4];
            if (!kFull || cls >= 0) gp[cls] += (double)lx[5];
        }
        lam[tid] = lV;
    }
    __syncthreads();
}

__global__ void k_adj_init(AdjDev d) {
    const size_t n = (size_t)d.n_sets * d.L;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        d.state[q] = d.init[q % d.L];
}

// Forward pass over ticks [t0, t1): checkpoints every K ticks, the loss and the traces.
template <bool kFull>
__global__ void __launch_bounds__(kMaxSeg) k_adj_forward(AdjDev d, uint32_t t0, uint32_t t1) {
    extern __shared__ __align__(16) unsigned char smem[];
    const Ctx c = make_ctx(d);
    const Lay L = make_lay(smem, d.Smax, d.Emax, d.Ymax, false, d.W);
    const Scr sc{};
    float* gstate = d.state + (size_t)c.p * d.L + c.st_off;
    block_load(L.st, gstate, c, d.Smax, d.W);
    __syncthreads();
    double loss = 0.0;
    for (uint32_t t = t0; t < t1; t++) {
        if (t % d.K == 0) {
            block_store(d.ckpt + ((size_t)(t / d.K) * d.n_sets + c.p) * d.L + c.st_off, L.st, c, d.Smax, d.W);
            __syncthreads();
        }
        tick_fwd<kFull>(d, c, L, sc, t, false);
        if ((t + 1) % d.stride == 0 && threadIdx.x == c.soma) {
            const uint32_t smp = (t + 1) / d.stride - 1;
            const float V = L.st[c.soma];
            if (d.target) {
                const double diff = (double)V - (double)d.target[(size_t)smp * d.nn + c.n];
                loss += diff * diff;
            }
            if (d.trace) d.trace[((size_t)c.p * d.n_samples + smp) * d.nn + c.n] = V;
        }
    }
    block_store(gstate, L.st, c, d.Smax, d.W);
    if (threadIdx.x == c.soma) d.loss_part[(size_t)c.p * d.nn + c.n] += loss;
}

// The re-run of window w from its checkpoint that the reverse pass needs: each tick's
// starting state into the window buffer.  A launch of its own, before the window's
// reverse launch: every CTA then runs the forward tick's code at the forward kernel's
// occupancy, where in the reverse kernel CTAs re-running and CTAs reversing would share
// an SM's instruction caches between the two ticks' code.
template <bool kFull>
__global__ void __launch_bounds__(kMaxSeg) k_adj_rerun(AdjDev d, uint32_t w) {
    extern __shared__ __align__(16) unsigned char smem[];
    const Ctx c = make_ctx(d);
    const uint32_t W = kFull ? d.W : kW3;
    const Lay L = make_lay(smem, d.Smax, d.Emax, d.Ymax, false, W);
    const Scr sc{};
    const uint32_t tb = w * d.K;
    const uint32_t te = min(d.T, tb + d.K);
    block_load(L.st, d.ckpt + ((size_t)w * d.n_sets + c.p) * d.L + c.st_off, c, d.Smax, W);
    __syncthreads();
    for (uint32_t t = tb; t < te; t++) {
        block_store(d.win + ((size_t)(t - tb) * d.n_sets + c.p) * d.L + c.st_off, L.st, c, d.Smax, W);
        if (t + 1 == te) break;   // the last tick is re-run by the reverse launch
        __syncthreads();
        tick_fwd<kFull>(d, c, L, sc, t, false);
    }
}

// Reverse pass over window w (ticks [w K, min((w + 1) K, T))), after k_adj_rerun has
// left each tick's starting state in the window buffer.
// kThreads / kMinBlocks: the launch bounds (neurons of at most 64 segments run a
// 64-thread instantiation bounded for 5 CTAs per SM).
template <bool kFull, int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_adj_backward(AdjDev d, uint32_t w) {
    extern __shared__ __align__(16) unsigned char smem[];
    const Ctx c = make_ctx(d);
    const uint32_t W = kFull ? d.W : kW3;
    const Lay L = make_lay(smem, d.Smax, d.Emax, d.Ymax, true, W);
    const Scr sc = make_scr<kFull>(d);
    const uint32_t tb = w * d.K;
    const uint32_t te = min(d.T, tb + d.K);
    const uint32_t Sm = d.Smax;
    {   // adjoint of the state at the window's end
        const float* src = d.lam + (size_t)c.p * d.L + c.st_off;
        block_load(L.lam, src, c, Sm, W);
    }
    // Walk the ticks backwards: each is re-run from its starting state with its
    // intermediates recorded, then reversed.
    const uint32_t n = te - tb;
    double gp[3] = {0.0, 0.0, 0.0};
    for (uint32_t step = 0; step < n; step++) {
        const uint32_t t = te - 1 - step;
        __syncthreads();
        block_load(L.st, d.win + ((size_t)(t - tb) * d.n_sets + c.p) * d.L + c.st_off, c, d.Smax, W);
        __syncthreads();
        tick_fwd<kFull>(d, c, L, sc, t, true);
        tick_rev<kFull>(d, c, L, sc, t, gp);
    }
    {
        float* dst = d.lam + (size_t)c.p * d.L + c.st_off;
        block_store(dst, L.lam, c, Sm, W);
    }
    if (threadIdx.x < c.S)
        for (int k = 0; k < 3; k++) d.g_par[((size_t)c.p * 3 + k) * d.n_seg + c.g] += gp[k];
}

}  // namespace
}  // namespace bnc

namespace bnc {
namespace {

static bool g_adj_ready[64] = {false};   // per device: constant tables and receptor table

cudaError_t adj_prepare(cudaStream_t stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (g_adj_ready[dev]) return cudaSuccess;
    const float z[7] = {1.0f, 1.0f, 2.0f, -1.0f, 2.0f, -1.0f, 1.0f};
    const float D[7] = {1.33f, 1.96f, 0.22f, 2.03f, 0.10f, 0.0f, 9.31f};
    const float bath[7] = {140.0f, 3.0f, 1.2f, 130.0f, 1.0f, 0.0f, 4.0e-5f};
    float z2d[7];
    for (int q = 0; q < 7; q++) z2d[q] = z[q] * z[q] * D[q];   // the reference's float product
    e = cudaMemcpyToSymbol(c_z2d, z2d, sizeof(z2d));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_z, z, sizeof(z));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_D, D, sizeof(D));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_bath, bath, sizeof(bath));
    if (e != cudaSuccess) return e;
    k_init_receptors<<<1, 1, 0, stream>>>();
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) g_adj_ready[dev] = true;
    return e;
}

struct Adjoint {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DeviceAllocs allocs;
    AdjDev d{};
    uint32_t threads = 32;
    size_t smem_fwd = 0, smem_bwd = 0;
    // host copies
    std::vector<uint32_t> slot_of_syn;    // original synapse -> slot (UINT32_MAX: not modelled)
    std::vector<uint32_t> soma;           // per neuron: global soma segment
    std::vector<float> par0, w0;          // defaults (from the network)
    std::vector<uint32_t> slot_syn;       // slot -> original synapse
    bool recorded = false, forward_done = false;
    float fwd_ms = 0.0f, bwd_ms = 0.0f;
    // device buffers whose pointers AdjDev holds as const
    float *par = nullptr, *w = nullptr, *target = nullptr;
    uint32_t* ev_off = nullptr;
    unsigned long long* ev_tick = nullptr;
    float* ev_amt = nullptr;
    DeviceAllocs ev_allocs, trace_allocs;

    ~Adjoint() {
        cudaSetDevice(device);
        allocs.release();
        ev_allocs.release();
        trace_allocs.release();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

template <typename T>
T* upload(DeviceAllocs& a, const std::vector<T>& v, int* rc) {
    T* p = static_cast<T*>(a.alloc(v.size() * sizeof(T)));
    if (!p) { *rc = BNC_ERR_ALLOC; return nullptr; }
    if (!v.empty() && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        *rc = BNC_ERR_CUDA;
    return p;
}

int adj_fail(int rc, const char* what) {
    if (rc == BNC_ERR_ALLOC) set_error("adjoint: device allocation failed (%s)", what);
    else if (rc == BNC_ERR_CUDA) set_error("adjoint: %s: %s", what, cudaGetErrorString(cudaGetLastError()));
    return rc;
}

// Builds the adjoint's structure from a loaded backend.  Returns BNC_OK or an error
// (bnc_last_error explains what the network uses that the adjoint does not model).
int adj_build(Adjoint* A, void* sim, const BncAdjointConfig& cfg) {
    HostNet hn;
    std::vector<BncCurrentStimulus> stim;
    uint64_t tick0 = 0;
    uint32_t n_vclamp = 0;
    int rc = backend_export_host(sim, &hn, &stim, &tick0, &A->device, &n_vclamp);
    if (rc != BNC_OK) return rc;
    if (n_vclamp) { set_error("adjoint: voltage clamps are not modelled"); return BNC_ERR_UNSUPPORTED; }
    if (cfg.n_sets == 0 || cfg.n_sets > 65535) { set_error("adjoint: n_sets must be 1..65535"); return BNC_ERR_ARG; }
    if (cfg.ticks == 0 || !(cfg.dt > 0.0f)) { set_error("adjoint: ticks and dt must be positive"); return BNC_ERR_ARG; }
    const uint32_t N = hn.num_segments;
    const uint32_t M = hn.num_connections;
    const uint32_t K = cfg.checkpoint_every ? cfg.checkpoint_every : 256u;
    const uint32_t stride = cfg.sample_every ? cfg.sample_every : 1u;
    if (N == 0) { set_error("adjoint: empty network"); return BNC_ERR_ARG; }

    // neurons: connected components of the connection graph, each a contiguous range
    std::vector<uint32_t> parent(N);
    for (uint32_t i = 0; i < N; i++) parent[i] = i;
    auto find = [&](uint32_t x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
    for (uint32_t e = 0; e < M; e++) {
        const uint32_t a = hn.conn[e].segment_a, b = hn.conn[e].segment_b;
        if (a >= N || b >= N) { set_error("adjoint: connection %u has an endpoint outside the network", e); return BNC_ERR_UNSUPPORTED; }
        uint32_t ra = find(a), rb = find(b);
        if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
    }
    std::vector<uint32_t> nr_seg;   // starts
    for (uint32_t i = 0; i < N; i++) {
        const uint32_t r = find(i);
        if (r == i) nr_seg.push_back(i);
        else if (r != find(nr_seg.back())) {
            set_error("adjoint: segment %u belongs to a neuron that is not a contiguous segment range", i);
            return BNC_ERR_UNSUPPORTED;
        }
    }
    const uint32_t nn = (uint32_t)nr_seg.size();
    nr_seg.push_back(N);
    uint32_t Smax = 0;
    for (uint32_t n = 0; n < nn; n++) Smax = std::max(Smax, nr_seg[n + 1] - nr_seg[n]);
    if (Smax > (uint32_t)kMaxSeg) { set_error("adjoint: a neuron has %u segments (at most %d)", Smax, kMaxSeg); return BNC_ERR_UNSUPPORTED; }
    std::vector<uint32_t> nrn_of(N);
    for (uint32_t n = 0; n < nn; n++) for (uint32_t i = nr_seg[n]; i < nr_seg[n + 1]; i++) nrn_of[i] = n;

    // connections per neuron, in original order; per-segment incidence (ascending)
    std::vector<uint32_t> nr_edge(nn + 1, 0);
    for (uint32_t e = 0; e < M; e++) nr_edge[nrn_of[hn.conn[e].segment_a] + 1]++;
    for (uint32_t n = 0; n < nn; n++) nr_edge[n + 1] += nr_edge[n];
    std::vector<uint32_t> fill(nr_edge.begin(), nr_edge.end() - 1);
    std::vector<uint16_t> ed_a(M), ed_b(M), inc_e((size_t)N * kMaxInc, 0);
    std::vector<uint8_t> ed_intra(M), inc_n(N, 0);
    std::vector<float> ed_area(M), ed_dist(M), ed_vola(M), ed_volb(M);
    uint32_t Emax = 0;
    for (uint32_t n = 0; n < nn; n++) Emax = std::max(Emax, nr_edge[n + 1] - nr_edge[n]);
    if (Emax > (uint32_t)kMaxSeg) { set_error("adjoint: a neuron has %u connections (at most %d)", Emax, kMaxSeg); return BNC_ERR_UNSUPPORTED; }
    for (uint32_t e = 0; e < M; e++) {
        const BncIntraConnection& cn = hn.conn[e];
        const uint32_t n = nrn_of[cn.segment_a];
        const uint32_t k = fill[n]++;
        const uint32_t le = k - nr_edge[n];
        const uint32_t a = cn.segment_a, b = cn.segment_b;
        ed_a[k] = (uint16_t)(a - nr_seg[n]);
        ed_b[k] = (uint16_t)(b - nr_seg[n]);
        ed_intra[k] = cn.is_intracellular ? 1 : 0;
        const SegLite &sa = hn.seg[a], &sb = hn.seg[b];
        float r_min = sa.radius < sb.radius ? sa.radius : sb.radius;
        float area_conn = 3.14159265f * r_min * r_min;
        if (area_conn < 1e-6f) area_conn = 1e-6f;
        float dist = (sa.length + sb.length) * 0.5f;
        if (dist < 0.1f) dist = 0.1f;
        float vol_a = (float)host_seg_volume(sa), vol_b = (float)host_seg_volume(sb);
        if (vol_a < 1e-6f) vol_a = 1e-6f;
        if (vol_b < 1e-6f) vol_b = 1e-6f;
        ed_area[k] = area_conn; ed_dist[k] = dist; ed_vola[k] = vol_a; ed_volb[k] = vol_b;
        for (uint32_t x : {a, b}) {
            if (inc_n[x] >= kMaxInc) { set_error("adjoint: segment %u has more than %d connections", x, kMaxInc); return BNC_ERR_UNSUPPORTED; }
            if (x == b && a == b) break;
            inc_e[(size_t)x * kMaxInc + inc_n[x]++] = (uint16_t)le;
        }
    }

    // per-segment statics, items, gates; the initial state blocks
    std::vector<float> area(N), cm(N);
    std::vector<double> vol(N);
    std::vector<uint8_t> n_it(N, 0), it_type((size_t)N * kItems, 0), it_gate((size_t)N * kItems, 0);
    std::vector<float> it_st((size_t)N * kItems * 7, 0.0f), it_den((size_t)N * kItems, 0.0f);
    A->par0.assign((size_t)3 * N, 0.0f);
    for (uint32_t i = 0; i < N; i++) {
        const SegLite& s = hn.seg[i];
        area[i] = host_seg_area(s);
        vol[i] = host_seg_volume(s);
        cm[i] = host_seg_capacitance(hn, i);
        bool myel = false;
        for (uint32_t j = 0; j < s.modifier_count; j++) if (hn.mod(i, j).type == BNC_MOD_MYELIN) myel = true;
        uint32_t gates = 0;
        bool cls_used[3] = {false, false, false};
        for (uint32_t j = 0; j < s.modifier_count; j++) {
            const ModLite& m = hn.mod(i, j);
            const uint8_t t = m.type;
            if (myel && t != BNC_MOD_MYELIN && host_is_myelin_blocked(t)) continue;   // simulation_host.cpp:241
            if (t == BNC_MOD_MYELIN || t == BNC_MOD_CAV21) continue;   // no current, nothing the replay reads
            if (t != BNC_MOD_NAV16 && t != BNC_MOD_NAV12 && t != BNC_MOD_KV_DR && t != BNC_MOD_K2P &&
                t != BNC_MOD_CAV13 && t != BNC_MOD_PUMP_NAK) {
                set_error("adjoint: modifier type %u (segment %u) is not differentiated (Nav1.6/1.2, Kv_DR, K2P, "
                          "Cav1.3, the Na/K pump, myelin and Cav2.1 are)", (unsigned)t, i);
                return BNC_ERR_UNSUPPORTED;
            }
            const int ng = (t == BNC_MOD_KV_DR) ? 1 : ((t == BNC_MOD_K2P || t == BNC_MOD_PUMP_NAK) ? 0 : 2);
            if (n_it[i] >= kItems || gates + ng > (uint32_t)kGates) {
                set_error("adjoint: segment %u holds more differentiable modifiers than %d items and %d gate words",
                          i, kItems, kGates);
                return BNC_ERR_UNSUPPORTED;
            }
            const int cls = (t == BNC_MOD_KV_DR) ? 1 : (t == BNC_MOD_K2P ? 2 : ((t == BNC_MOD_NAV16 || t == BNC_MOD_NAV12) ? 0 : -1));
            if (cls >= 0) {
                if (cls_used[cls]) { set_error("adjoint: segment %u holds two modifiers of one conductance class", i); return BNC_ERR_UNSUPPORTED; }
                cls_used[cls] = true;
            }
            const uint32_t k = n_it[i]++;
            it_type[(size_t)i * kItems + k] = t;
            it_gate[(size_t)i * kItems + k] = (uint8_t)gates;
            it_den[(size_t)i * kItems + k] = m.density;
            for (int q = 0; q < 7; q++) it_st[((size_t)i * kItems + k) * 7 + q] = m.state[q];
            gates += ng;
            if (cls >= 0) A->par0[(size_t)cls * N + i] = m.density;
        }
    }

    // state words per segment: the gate words the segments need, and ATP with a pump
    uint32_t gmax = 0;
    for (uint32_t i = 0; i < N; i++)
        for (uint32_t j = 0; j < n_it[i]; j++) {
            const uint8_t t = it_type[(size_t)i * kItems + j];
            const uint32_t ng = (t == BNC_MOD_KV_DR) ? 1u : ((t == BNC_MOD_K2P || t == BNC_MOD_PUMP_NAK) ? 0u : 2u);
            gmax = std::max<uint32_t>(gmax, it_gate[(size_t)i * kItems + j] + ng);
        }
    const bool has_atp = std::find(it_type.begin(), it_type.end(), (uint8_t)BNC_MOD_PUMP_NAK) != it_type.end();
    const bool full_items = has_atp || std::find(it_type.begin(), it_type.end(), (uint8_t)BNC_MOD_CAV13) != it_type.end();
    const uint32_t atp_w = 15 + gmax;
    // the fitting family's kernels take kW3 words (gmax <= 3 without Cav1.3)
    const uint32_t Wseg = full_items ? atp_w + (has_atp ? 1u : 0u) : kW3;

    // synapse slots by post segment (original order within a segment)
    const uint32_t KS = hn.num_synapses;
    A->slot_of_syn.assign(KS, UINT32_MAX);
    std::vector<uint32_t> sp_cnt(N + 1, 0);
    for (uint32_t k = 0; k < KS; k++) {
        const SynLite& y = hn.syn[k];
        if (y.type != BNC_SYN_CHEMICAL) { set_error("adjoint: synapse %u is not chemical", k); return BNC_ERR_UNSUPPORTED; }
        if (y.post_segment >= N) { set_error("adjoint: synapse %u has its post segment outside the network", k); return BNC_ERR_UNSUPPORTED; }
        sp_cnt[y.post_segment + 1]++;
    }
    for (uint32_t i = 0; i < N; i++) sp_cnt[i + 1] += sp_cnt[i];
    const uint32_t n_slot = KS;
    std::vector<uint32_t> sl_syn(n_slot), sfill(sp_cnt.begin(), sp_cnt.end() - 1);
    for (uint32_t k = 0; k < KS; k++) sl_syn[sfill[hn.syn[k].post_segment]++] = k;
    std::vector<uint8_t> sl_nrec(n_slot, 0), sl_kind((size_t)n_slot * kRecPerSyn, 0), sl_rav((size_t)n_slot * kRecPerSyn, 0),
        sl_nt(n_slot, 0);
    std::vector<float> sl_rden((size_t)n_slot * kRecPerSyn, 0.0f), sl_parea(n_slot), sl_tauc(n_slot);
    std::vector<float> rinit((size_t)n_slot * kSynWords, 0.0f);
    for (uint32_t y = 0; y < n_slot; y++) {
        const uint32_t k = sl_syn[y];
        A->slot_of_syn[k] = y;
        const SynLite& s = hn.syn[k];
        bool myel_post = false;
        const SegLite& ps = hn.seg[s.post_segment];
        for (uint32_t j = 0; j < ps.modifier_count; j++) if (hn.mod(s.post_segment, j).type == BNC_MOD_MYELIN) myel_post = true;
        const uint8_t nt = s.post_receptor_count > 0 ? host_nt_from_receptor(hn.post_rec(k, 0).type) : 0;
        if (nt > 1 && nt != BNC_NT_GLYCINE) {
            set_error("adjoint: synapse %u releases a transmitter other than glutamate, GABA or glycine", k);
            return BNC_ERR_UNSUPPORTED;
        }
        for (int q = 0; q < 15; q++)
            if (q != nt && s.cleft_neurotransmitter[q] != 0.0f) {
                set_error("adjoint: synapse %u holds a cleft transmitter it does not release", k);
                return BNC_ERR_UNSUPPORTED;
            }
        sl_nt[y] = (nt == BNC_NT_GLYCINE) ? 2 : nt;
        sl_parea[y] = s.post_area;
        sl_tauc[y] = s.tau_clearance;
        rinit[(size_t)y * kSynWords + 4] = s.cleft_neurotransmitter[nt];
        uint32_t r = 0;
        for (uint32_t j = 0; j < s.post_receptor_count; j++) {
            const ModLite& m = hn.post_rec(k, j);
            if (myel_post && host_is_ionotropic(m.type)) continue;   // simulation_host.cpp:495
            if (m.type != BNC_MOD_AMPA && m.type != BNC_MOD_NMDA && m.type != BNC_MOD_GABAA && m.type != BNC_MOD_GLYCINE) {
                set_error("adjoint: receptor type %u on synapse %u is not differentiated (AMPA, NMDA, GABA-A and glycine are)",
                          (unsigned)m.type, k);
                return BNC_ERR_UNSUPPORTED;
            }
            if (m.active_vars != 0) { set_error("adjoint: receptor conductance overrides are not modelled"); return BNC_ERR_UNSUPPORTED; }
            if (r >= (uint32_t)kRecPerSyn) { set_error("adjoint: synapse %u has more than %d receptors", k, kRecPerSyn); return BNC_ERR_UNSUPPORTED; }
            sl_kind[(size_t)y * kRecPerSyn + r] =
                (m.type == BNC_MOD_AMPA) ? 0 : (m.type == BNC_MOD_NMDA ? 1 : (m.type == BNC_MOD_GABAA ? 2 : 3));
            sl_rden[(size_t)y * kRecPerSyn + r] = m.density;
            rinit[(size_t)y * kSynWords + 2 * r] = m.state[0];
            // NMDA does not desensitise: its second word carries the inactivation gate
            rinit[(size_t)y * kSynWords + 2 * r + 1] = m.type == BNC_MOD_NMDA ? m.state[2] : m.state[1];
            r++;
        }
        sl_nrec[y] = (uint8_t)r;
    }
    A->slot_syn = sl_syn;
    A->w0.assign(KS, 1.0f);

    // per-neuron slot ranges and state offsets; the initial state
    std::vector<uint32_t> nr_slot(nn + 1), nr_st(nn + 1);
    std::vector<uint16_t> nr_soma(nn);
    A->soma.resize(nn);
    uint32_t Ymax = 1;
    nr_st[0] = 0;
    for (uint32_t n = 0; n < nn; n++) {
        nr_slot[n] = sp_cnt[nr_seg[n]];
        nr_slot[n + 1] = sp_cnt[nr_seg[n + 1]];
        const uint32_t S = nr_seg[n + 1] - nr_seg[n], Y = nr_slot[n + 1] - nr_slot[n];
        Ymax = std::max(Ymax, Y);
        nr_st[n + 1] = nr_st[n] + Wseg * S + kSynWords * Y;
        uint32_t so = 0;
        for (uint32_t i = nr_seg[n]; i < nr_seg[n + 1]; i++)
            if (hn.seg[i].segment_type == BNC_SEG_SOMA) { so = i - nr_seg[n]; break; }
        nr_soma[n] = (uint16_t)so;
        A->soma[n] = nr_seg[n] + so;
    }
    const uint32_t L = nr_st[nn];
    std::vector<float> init(L, 0.0f);
    for (uint32_t n = 0; n < nn; n++) {
        const uint32_t s0 = nr_seg[n], S = nr_seg[n + 1] - s0;
        float* b = init.data() + nr_st[n];
        for (uint32_t i = 0; i < S; i++) {
            const SegLite& s = hn.seg[s0 + i];
            b[i] = s.V_m;
            for (int q = 0; q < 7; q++) { b[(1 + q) * S + i] = s.intra_ions[q]; b[(8 + q) * S + i] = s.extra_ions[q]; }
            if (has_atp) b[atp_w * S + i] = s.ATP_level;
            for (uint32_t j = 0; j < n_it[s0 + i]; j++) {
                const uint8_t t = it_type[(size_t)(s0 + i) * kItems + j];
                const uint32_t go = it_gate[(size_t)(s0 + i) * kItems + j];
                // the item's slot: find it again in the modifier list
                for (uint32_t jj = 0; jj < s.modifier_count; jj++) {
                    const ModLite& m = hn.mod(s0 + i, jj);
                    if (m.type != t) continue;
                    if (t != BNC_MOD_K2P && t != BNC_MOD_PUMP_NAK) b[(15 + go) * S + i] = m.state[0];
                    if (t == BNC_MOD_NAV16 || t == BNC_MOD_NAV12 || t == BNC_MOD_CAV13) b[(16 + go) * S + i] = m.state[1];
                    break;
                }
            }
        }
        const uint32_t y0 = nr_slot[n], Y = nr_slot[n + 1] - y0;
        for (uint32_t y = 0; y < Y; y++)
            for (int q = 0; q < kSynWords; q++) b[Wseg * S + y * kSynWords + q] = rinit[(size_t)(y0 + y) * kSynWords + q];
    }

    // current stimuli per segment, in list order (matched by segment id, simulation_host.cpp:285-297)
    std::vector<uint32_t> stim_off(N + 1, 0);
    std::vector<std::vector<uint32_t>> per(N);
    {
        std::vector<std::pair<uint32_t, uint32_t>> ids(N);   // (id, segment)
        for (uint32_t i = 0; i < N; i++) ids[i] = {hn.seg[i].id, i};
        std::sort(ids.begin(), ids.end());
        for (uint32_t q = 0; q < stim.size(); q++) {
            auto it = std::lower_bound(ids.begin(), ids.end(), std::make_pair(stim[q].segment_id, 0u));
            for (; it != ids.end() && it->first == stim[q].segment_id; ++it) per[it->second].push_back(q);
        }
    }
    std::vector<unsigned long long> stim_b, stim_e;
    std::vector<float> stim_amp;
    for (uint32_t i = 0; i < N; i++) {
        for (uint32_t q : per[i]) {
            const BncCurrentStimulus& st = stim[q];
            const unsigned long long dur = (unsigned long long)(st.duration_ms / cfg.dt);
            stim_b.push_back(st.start_tick);
            stim_e.push_back(st.start_tick + dur);
            stim_amp.push_back(st.amplitude_pA);
        }
        stim_off[i + 1] = (uint32_t)stim_b.size();
    }

    // device
    cudaSetDevice(A->device);
    if (cudaStreamCreateWithFlags(&A->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&A->ev0) != cudaSuccess || cudaEventCreate(&A->ev1) != cudaSuccess)
        return adj_fail(BNC_ERR_CUDA, "stream");
    cudaError_t ce = adj_prepare(A->stream);
    if (ce != cudaSuccess) { set_error("adjoint: set-up: %s", cudaGetErrorString(ce)); return BNC_ERR_CUDA; }
    DeviceAllocs& al = A->allocs;
    AdjDev& d = A->d;
    rc = BNC_OK;
    d.nn = nn; d.n_seg = N; d.n_edge = M; d.n_slot = n_slot; d.n_syn = KS; d.n_sets = cfg.n_sets;
    d.T = cfg.ticks; d.K = K; d.n_ckpt = (cfg.ticks + K - 1) / K; d.stride = stride; d.n_samples = cfg.ticks / stride;
    d.Smax = (Smax + 3u) & ~3u;   // stride of the per-segment arrays: a multiple of 4 (16-byte rows)
    d.Emax = std::max(Emax, 1u); d.Ymax = Ymax; d.L = L; d.dt = cfg.dt; d.has_conn = M > 0;
    d.has_atp = has_atp ? 1 : 0;
    d.full = full_items ? 1 : 0;
    d.W = Wseg;
    d.atp_w = atp_w;
    d.tick0 = tick0;
    std::vector<uint32_t> nr_seg_v(nr_seg.begin(), nr_seg.end());
    d.nr_seg = upload(al, nr_seg_v, &rc); d.nr_edge = upload(al, nr_edge, &rc); d.nr_slot = upload(al, nr_slot, &rc);
    d.nr_st = upload(al, nr_st, &rc); d.nr_soma = upload(al, nr_soma, &rc);
    d.area = upload(al, area, &rc); d.cm = upload(al, cm, &rc); d.vol = upload(al, vol, &rc);
    if (!full_items) {   // the fitting family's kernels index items with stride 3
        std::vector<uint8_t> t3((size_t)N * 3), g3((size_t)N * 3);
        std::vector<float> s3((size_t)N * 3 * 7), d3((size_t)N * 3);
        for (uint32_t i = 0; i < N; i++)
            for (uint32_t j = 0; j < 3; j++) {
                const size_t a = (size_t)i * kItems + j, b3 = (size_t)i * 3 + j;
                t3[b3] = it_type[a]; g3[b3] = it_gate[a]; d3[b3] = it_den[a];
                for (int q = 0; q < 7; q++) s3[b3 * 7 + q] = it_st[a * 7 + q];
            }
        it_type.swap(t3); it_gate.swap(g3); it_st.swap(s3); it_den.swap(d3);
    }
    d.n_it = upload(al, n_it, &rc); d.it_type = upload(al, it_type, &rc); d.it_gate = upload(al, it_gate, &rc);
    d.it_st = upload(al, it_st, &rc); d.it_den = upload(al, it_den, &rc); d.inc_n = upload(al, inc_n, &rc); d.inc_e = upload(al, inc_e, &rc);
    d.stim_off = upload(al, stim_off, &rc); d.stim_b = upload(al, stim_b, &rc); d.stim_e = upload(al, stim_e, &rc);
    d.stim_amp = upload(al, stim_amp, &rc); d.sp_off = upload(al, sp_cnt, &rc);
    d.ed_a = upload(al, ed_a, &rc); d.ed_b = upload(al, ed_b, &rc); d.ed_intra = upload(al, ed_intra, &rc);
    d.ed_area = upload(al, ed_area, &rc); d.ed_dist = upload(al, ed_dist, &rc); d.ed_vola = upload(al, ed_vola, &rc);
    d.ed_volb = upload(al, ed_volb, &rc);
    d.sl_syn = upload(al, sl_syn, &rc); d.sl_nrec = upload(al, sl_nrec, &rc); d.sl_kind = upload(al, sl_kind, &rc);
    d.sl_rden = upload(al, sl_rden, &rc); d.sl_rav = upload(al, sl_rav, &rc); d.sl_parea = upload(al, sl_parea, &rc);
    d.sl_tauc = upload(al, sl_tauc, &rc); d.sl_nt = upload(al, sl_nt, &rc);
    d.init = upload(al, init, &rc);
    std::vector<float> par_all((size_t)cfg.n_sets * 3 * N), w_all((size_t)cfg.n_sets * KS);
    for (uint32_t p = 0; p < cfg.n_sets; p++) {
        std::copy(A->par0.begin(), A->par0.end(), par_all.begin() + (size_t)p * 3 * N);
        std::copy(A->w0.begin(), A->w0.end(), w_all.begin() + (size_t)p * KS);
    }
    A->par = upload(al, par_all, &rc); d.par = A->par;
    A->w = upload(al, w_all, &rc); d.w = A->w;
    if (rc != BNC_OK) return adj_fail(rc, "network upload");
    const size_t setL = (size_t)cfg.n_sets * L;
    d.state = static_cast<float*>(al.alloc(setL * sizeof(float)));
    d.lam = static_cast<float*>(al.alloc(setL * sizeof(float)));
    d.ckpt = static_cast<float*>(al.alloc((size_t)d.n_ckpt * setL * sizeof(float)));
    d.win = static_cast<float*>(al.alloc((size_t)K * setL * sizeof(float)));
    d.loss_part = static_cast<double*>(al.alloc((size_t)cfg.n_sets * nn * sizeof(double)));
    d.g_par = static_cast<double*>(al.alloc((size_t)cfg.n_sets * 3 * N * sizeof(double)));
    d.g_w = static_cast<double*>(al.alloc((size_t)cfg.n_sets * std::max(KS, 1u) * sizeof(double)));
    d.scr_floats = scr_floats(d.Smax, Ymax, full_items ? (uint32_t)kItems : 3u, has_atp);
    d.scr = static_cast<float*>(al.alloc((size_t)nn * cfg.n_sets * d.scr_floats * sizeof(float)));
    if (!d.state || !d.lam || !d.ckpt || !d.win || !d.loss_part || !d.g_par || !d.g_w || !d.scr)
        return adj_fail(BNC_ERR_ALLOC, "state, checkpoints and scratch");
    // an empty release log until bnc_adjoint_record
    std::vector<uint32_t> ev_off(n_slot + 1, 0);
    A->ev_off = upload(A->ev_allocs, ev_off, &rc);
    std::vector<unsigned long long> one_tick(1, 0);
    std::vector<float> one_amt(1, 0.0f);
    A->ev_tick = upload(A->ev_allocs, one_tick, &rc);
    A->ev_amt = upload(A->ev_allocs, one_amt, &rc);
    if (rc != BNC_OK) return adj_fail(rc, "release log");
    d.ev_off = A->ev_off; d.ev_tick = A->ev_tick; d.ev_amt = A->ev_amt;
    d.target = nullptr;
    d.trace = nullptr;
    A->threads = ((std::max(d.Smax, d.Emax) + 31u) / 32u) * 32u;
    A->smem_fwd = lay_bytes(d.Smax, d.Emax, Ymax, false, Wseg);
    A->smem_bwd = lay_bytes(d.Smax, d.Emax, Ymax, true, Wseg);
    if (A->smem_bwd > 227u * 1024u) { set_error("adjoint: a neuron needs %zu bytes of shared memory", A->smem_bwd); return BNC_ERR_UNSUPPORTED; }
    if (cudaFuncSetAttribute(k_adj_forward<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A->smem_fwd) != cudaSuccess ||
        cudaFuncSetAttribute(k_adj_forward<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A->smem_fwd) != cudaSuccess ||
        cudaFuncSetAttribute(k_adj_rerun<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A->smem_fwd) != cudaSuccess ||
        cudaFuncSetAttribute(k_adj_rerun<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A->smem_fwd) != cudaSuccess ||
        cudaFuncSetAttribute(k_adj_backward<false, kMaxSeg, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A->smem_bwd) != cudaSuccess ||
        cudaFuncSetAttribute(k_adj_backward<true, kMaxSeg, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A->smem_bwd) != cudaSuccess ||
        cudaFuncSetAttribute(k_adj_backward<false, 64, BNC_ADJ_MIN_BLOCKS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A->smem_bwd) != cudaSuccess ||
        cudaFuncSetAttribute(k_adj_backward<true, 64, BNC_ADJ_MIN_BLOCKS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A->smem_bwd) != cudaSuccess)
        return adj_fail(BNC_ERR_CUDA, "shared-memory limit");
    return BNC_OK;
}

}  // namespace
}  // namespace bnc

using namespace bnc;

extern "C" {

void* bnc_adjoint_create(void* sim, const BncAdjointConfig* cfg) {
    if (!sim || !cfg) { set_error("null argument"); return nullptr; }
    Adjoint* A = new (std::nothrow) Adjoint();
    if (!A) { set_error("out of host memory"); return nullptr; }
    int rc = adj_build(A, sim, *cfg);
    if (rc != BNC_OK) { delete A; return nullptr; }
    return A;
}

void bnc_adjoint_destroy(void* adj) { delete static_cast<Adjoint*>(adj); }

int bnc_adjoint_info(void* adj, BncAdjointInfo* info) {
    if (!adj || !info) { set_error("null argument"); return BNC_ERR_ARG; }
    const Adjoint* A = static_cast<const Adjoint*>(adj);
    std::memset(info, 0, sizeof(*info));
    info->n_neurons = A->d.nn;
    info->n_segments = A->d.n_seg;
    info->n_synapses = A->d.n_syn;
    info->n_samples = A->d.n_samples;
    info->n_sets = A->d.n_sets;
    info->ticks = A->d.T;
    info->checkpoint_every = A->d.K;
    info->threads = A->threads;
    info->smem_forward = (uint32_t)A->smem_fwd;
    info->smem_backward = (uint32_t)A->smem_bwd;
    const size_t setL = (size_t)A->d.n_sets * A->d.L;
    info->checkpoint_bytes = (uint64_t)A->d.n_ckpt * setL * 4u;
    info->window_bytes = (uint64_t)A->d.K * setL * 4u;
    info->scratch_bytes = (uint64_t)A->d.nn * A->d.n_sets * A->d.scr_floats * 4u;
    return BNC_OK;
}

int bnc_adjoint_soma(void* adj, uint32_t* soma, uint32_t n) {
    if (!adj || !soma) { set_error("null argument"); return BNC_ERR_ARG; }
    const Adjoint* A = static_cast<const Adjoint*>(adj);
    if (n < A->d.nn) { set_error("buffer holds %u values, %u needed", n, A->d.nn); return BNC_ERR_ARG; }
    for (uint32_t q = 0; q < A->d.nn; q++) soma[q] = A->soma[q];
    return BNC_OK;
}

int bnc_adjoint_record(void* adj, void* sim) {
    if (!adj || !sim) { set_error("null argument"); return BNC_ERR_ARG; }
    Adjoint* A = static_cast<Adjoint*>(adj);
    std::vector<uint32_t> syn;
    std::vector<uint64_t> tick;
    std::vector<float> amt;
    std::vector<uint8_t> slot;
    int rc = backend_record_releases(sim, A->d.T, A->d.dt, &syn, &tick, &amt, &slot);
    if (rc != BNC_OK) return rc;
    // group by synapse slot, then tick, then the order the tick added them (delay slots
    // 0-3, then the release)
    const size_t n = syn.size();
    std::vector<uint32_t> order(n);
    for (size_t q = 0; q < n; q++) order[q] = (uint32_t)q;
    std::vector<uint32_t> sl(n);
    for (size_t q = 0; q < n; q++) {
        if (syn[q] >= A->slot_of_syn.size() || A->slot_of_syn[syn[q]] == UINT32_MAX) {
            set_error("adjoint: a logged release names synapse %u, which the adjoint does not hold", syn[q]);
            return BNC_ERR_STATE;
        }
        sl[q] = A->slot_of_syn[syn[q]];
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        if (sl[a] != sl[b]) return sl[a] < sl[b];
        if (tick[a] != tick[b]) return tick[a] < tick[b];
        return slot[a] < slot[b];
    });
    std::vector<uint32_t> ev_off(A->d.n_slot + 1, 0);
    std::vector<unsigned long long> ev_tick(std::max<size_t>(n, 1), 0);
    std::vector<float> ev_amt(std::max<size_t>(n, 1), 0.0f);
    for (size_t q = 0; q < n; q++) {
        ev_off[sl[order[q]] + 1]++;
        ev_tick[q] = tick[order[q]];
        ev_amt[q] = amt[order[q]];
    }
    for (uint32_t y = 0; y < A->d.n_slot; y++) ev_off[y + 1] += ev_off[y];
    cudaSetDevice(A->device);
    A->ev_allocs.release();
    rc = BNC_OK;
    A->ev_off = upload(A->ev_allocs, ev_off, &rc);
    A->ev_tick = upload(A->ev_allocs, ev_tick, &rc);
    A->ev_amt = upload(A->ev_allocs, ev_amt, &rc);
    if (rc != BNC_OK) return adj_fail(rc, "release log upload");
    A->d.ev_off = A->ev_off; A->d.ev_tick = A->ev_tick; A->d.ev_amt = A->ev_amt;
    A->recorded = true;
    A->forward_done = false;
    return BNC_OK;
}

int bnc_adjoint_release_count(void* adj, uint64_t* n) {
    if (!adj || !n) { set_error("null argument"); return BNC_ERR_ARG; }
    Adjoint* A = static_cast<Adjoint*>(adj);
    uint32_t last = 0;
    cudaSetDevice(A->device);
    if (cudaMemcpy(&last, A->ev_off + A->d.n_slot, sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        return adj_fail(BNC_ERR_CUDA, "read");
    *n = last;
    return BNC_OK;
}

int bnc_adjoint_set_params(void* adj, uint32_t set, const float* gNa, const float* gK, const float* gleak,
                           const float* w) {
    if (!adj) { set_error("null handle"); return BNC_ERR_ARG; }
    Adjoint* A = static_cast<Adjoint*>(adj);
    if (set >= A->d.n_sets) { set_error("parameter set %u out of range", set); return BNC_ERR_ARG; }
    cudaSetDevice(A->device);
    const uint32_t N = A->d.n_seg;
    const float* src[3] = {gNa, gK, gleak};
    for (int k = 0; k < 3; k++)
        if (src[k] && cudaMemcpy(A->par + ((size_t)set * 3 + k) * N, src[k], (size_t)N * sizeof(float),
                                 cudaMemcpyHostToDevice) != cudaSuccess)
            return adj_fail(BNC_ERR_CUDA, "parameter upload");
    if (w && A->d.n_syn &&
        cudaMemcpy(A->w + (size_t)set * A->d.n_syn, w, (size_t)A->d.n_syn * sizeof(float), cudaMemcpyHostToDevice) !=
            cudaSuccess)
        return adj_fail(BNC_ERR_CUDA, "weight upload");
    A->forward_done = false;
    return BNC_OK;
}

int bnc_adjoint_get_params(void* adj, uint32_t set, float* gNa, float* gK, float* gleak, float* w) {
    if (!adj) { set_error("null handle"); return BNC_ERR_ARG; }
    Adjoint* A = static_cast<Adjoint*>(adj);
    if (set >= A->d.n_sets) { set_error("parameter set %u out of range", set); return BNC_ERR_ARG; }
    cudaSetDevice(A->device);
    const uint32_t N = A->d.n_seg;
    float* dst[3] = {gNa, gK, gleak};
    for (int k = 0; k < 3; k++)
        if (dst[k] && cudaMemcpy(dst[k], A->par + ((size_t)set * 3 + k) * N, (size_t)N * sizeof(float),
                                 cudaMemcpyDeviceToHost) != cudaSuccess)
            return adj_fail(BNC_ERR_CUDA, "parameter read");
    if (w && A->d.n_syn &&
        cudaMemcpy(w, A->w + (size_t)set * A->d.n_syn, (size_t)A->d.n_syn * sizeof(float), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
        return adj_fail(BNC_ERR_CUDA, "weight read");
    return BNC_OK;
}

int bnc_adjoint_set_target(void* adj, const float* target) {
    if (!adj || !target) { set_error("null argument"); return BNC_ERR_ARG; }
    Adjoint* A = static_cast<Adjoint*>(adj);
    cudaSetDevice(A->device);
    const size_t n = (size_t)A->d.n_samples * A->d.nn;
    if (!A->target) {
        A->target = static_cast<float*>(A->allocs.alloc(std::max<size_t>(n, 1) * sizeof(float)));
        if (!A->target) return adj_fail(BNC_ERR_ALLOC, "target");
    }
    if (n && cudaMemcpy(A->target, target, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return adj_fail(BNC_ERR_CUDA, "target upload");
    A->d.target = A->target;
    A->forward_done = false;
    return BNC_OK;
}

int bnc_adjoint_forward(void* adj, double* loss, float* trace) {
    if (!adj) { set_error("null handle"); return BNC_ERR_ARG; }
    Adjoint* A = static_cast<Adjoint*>(adj);
    if (!A->recorded) { set_error("adjoint: record the releases first (bnc_adjoint_record)"); return BNC_ERR_STATE; }
    cudaSetDevice(A->device);
    AdjDev d = A->d;
    const size_t ntr = (size_t)d.n_sets * d.n_samples * d.nn;
    float* tr = nullptr;
    if (trace) {
        A->trace_allocs.release();
        tr = static_cast<float*>(A->trace_allocs.alloc(std::max<size_t>(ntr, 1) * sizeof(float)));
        if (!tr) return adj_fail(BNC_ERR_ALLOC, "trace");
    }
    d.trace = tr;
    cudaMemsetAsync(d.loss_part, 0, (size_t)d.n_sets * d.nn * sizeof(double), A->stream);
    cudaEventRecord(A->ev0, A->stream);
    k_adj_init<<<1024, 256, 0, A->stream>>>(d);
    const dim3 grid(d.nn, d.n_sets);
    for (uint32_t t0 = 0; t0 < d.T; t0 += d.K) {
        const uint32_t t1 = std::min(d.T, t0 + d.K);
        if (d.full) k_adj_forward<true><<<grid, A->threads, A->smem_fwd, A->stream>>>(d, t0, t1);
        else k_adj_forward<false><<<grid, A->threads, A->smem_fwd, A->stream>>>(d, t0, t1);
    }
    cudaEventRecord(A->ev1, A->stream);
    cudaError_t e = cudaStreamSynchronize(A->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) { set_error("adjoint forward: %s", cudaGetErrorString(e)); return BNC_ERR_CUDA; }
    cudaEventElapsedTime(&A->fwd_ms, A->ev0, A->ev1);
    if (loss) {
        std::vector<double> part((size_t)d.n_sets * d.nn);
        if (cudaMemcpy(part.data(), d.loss_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return adj_fail(BNC_ERR_CUDA, "loss read");
        for (uint32_t p = 0; p < d.n_sets; p++) {
            double s = 0.0;
            for (uint32_t n = 0; n < d.nn; n++) s += part[(size_t)p * d.nn + n];
            loss[p] = (d.n_samples && d.nn) ? s / ((double)d.n_samples * (double)d.nn) : 0.0;
        }
    }
    if (trace && ntr && cudaMemcpy(trace, tr, ntr * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return adj_fail(BNC_ERR_CUDA, "trace read");
    A->forward_done = true;
    return BNC_OK;
}

int bnc_adjoint_backward(void* adj, float* g_gNa, float* g_gK, float* g_gleak, float* g_w) {
    if (!adj) { set_error("null handle"); return BNC_ERR_ARG; }
    Adjoint* A = static_cast<Adjoint*>(adj);
    if (!A->forward_done) { set_error("adjoint: run bnc_adjoint_forward with the current parameters first"); return BNC_ERR_STATE; }
    if (!A->d.target) { set_error("adjoint: no target traces set"); return BNC_ERR_STATE; }
    cudaSetDevice(A->device);
    const AdjDev& d = A->d;
    const size_t setL = (size_t)d.n_sets * d.L;
    cudaMemsetAsync(d.lam, 0, setL * sizeof(float), A->stream);
    cudaMemsetAsync(d.g_par, 0, (size_t)d.n_sets * 3 * d.n_seg * sizeof(double), A->stream);
    cudaMemsetAsync(d.g_w, 0, (size_t)d.n_sets * std::max(d.n_syn, 1u) * sizeof(double), A->stream);
    cudaEventRecord(A->ev0, A->stream);
    const dim3 grid(d.nn, d.n_sets);
    for (int w = (int)d.n_ckpt - 1; w >= 0; w--) {
        if (d.full) k_adj_rerun<true><<<grid, A->threads, A->smem_fwd, A->stream>>>(d, (uint32_t)w);
        else k_adj_rerun<false><<<grid, A->threads, A->smem_fwd, A->stream>>>(d, (uint32_t)w);
        if (A->threads <= 64) {
            if (d.full) k_adj_backward<true, 64, BNC_ADJ_MIN_BLOCKS><<<grid, A->threads, A->smem_bwd, A->stream>>>(d, (uint32_t)w);
            else k_adj_backward<false, 64, BNC_ADJ_MIN_BLOCKS><<<grid, A->threads, A->smem_bwd, A->stream>>>(d, (uint32_t)w);
        } else {
            if (d.full) k_adj_backward<true, kMaxSeg, 1><<<grid, A->threads, A->smem_bwd, A->stream>>>(d, (uint32_t)w);
            else k_adj_backward<false, kMaxSeg, 1><<<grid, A->threads, A->smem_bwd, A->stream>>>(d, (uint32_t)w);
        }
    }
    cudaEventRecord(A->ev1, A->stream);
    cudaError_t e = cudaStreamSynchronize(A->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) { set_error("adjoint backward: %s", cudaGetErrorString(e)); return BNC_ERR_CUDA; }
    cudaEventElapsedTime(&A->bwd_ms, A->ev0, A->ev1);
    std::vector<double> gp((size_t)d.n_sets * 3 * d.n_seg), gw((size_t)d.n_sets * d.n_syn);
    if (cudaMemcpy(gp.data(), d.g_par, gp.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
        (d.n_syn && cudaMemcpy(gw.data(), d.g_w, gw.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess))
        return adj_fail(BNC_ERR_CUDA, "gradient read");
    float* out[3] = {g_gNa, g_gK, g_gleak};
    for (uint32_t p = 0; p < d.n_sets; p++) {
        for (int k = 0; k < 3; k++)
            if (out[k])
                for (uint32_t i = 0; i < d.n_seg; i++)
                    out[k][(size_t)p * d.n_seg + i] = (float)gp[((size_t)p * 3 + k) * d.n_seg + i];
        if (g_w)
            for (uint32_t k = 0; k < d.n_syn; k++) g_w[(size_t)p * d.n_syn + k] = (float)gw[(size_t)p * d.n_syn + k];
    }
    return BNC_OK;
}

int bnc_adjoint_timings(void* adj, float* forward_ms, float* backward_ms) {
    if (!adj) { set_error("null handle"); return BNC_ERR_ARG; }
    const Adjoint* A = static_cast<const Adjoint*>(adj);
    if (forward_ms) *forward_ms = A->fwd_ms;
    if (backward_ms) *backward_ms = A->bwd_ms;
    return BNC_OK;
}

}  // extern "C"
