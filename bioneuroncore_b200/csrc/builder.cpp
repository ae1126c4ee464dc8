// builder.cpp -- AoS (reference layout) -> device structure-of-arrays.
//
// What the builder decides, once per load:
//  * tiles: connected components of the intra-connection graph (whole neurons),
//    packed into tiles of <= kMaxTileSegs segments with each component owned by one
//    warp; the device segment order is the concatenation of tiles;
//  * the modifier phase schedule: a global sequence of phases such that every
//    segment's active modifiers appear in increasing slot order, each phase holding
//    at most one modifier per segment.  A greedy shortest-common-supersequence
//    pass picks, at each step, the type that is next for the most segments, so a
//    phase is a single modifier type when slot orders allow it (warp-uniform
//    dispatch); otherwise phases fall back to slot order with items sorted by type;
//  * incidence lists per segment in original connection order, so every gather in
//    the kernels sums in the reference's scatter order (diffusion_kernel.h loops
//    over connections in index order);
//  * the post-segment CSR of synapses in original synapse order, so per-post
//    accumulation follows simulation_host.cpp:357-592.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <atomic>
#include <mutex>
#include <thread>
#include "net.h"
#include "hostnet.h"
#include "par.h"

namespace bnc {

DeviceAllocs::~DeviceAllocs() { release(); }

void* DeviceAllocs::alloc(size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return p;
}

void DeviceAllocs::release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
}

namespace {

// ---- host restatements of the static per-segment helpers ----
// run_tick_common.h:209-214
float seg_area(const SegLite& s) {
    return (s.segment_type == 1 || s.segment_type == 3 || s.segment_type == 4)
        ? 4.0f * 3.14159265f * s.radius * s.radius
        : 2.0f * 3.14159265f * s.radius * s.length;
}
// run_tick_common.h:262-266
double seg_volume(const SegLite& s) {
    if (s.segment_type == 1 || s.segment_type == 3 || s.segment_type == 4)
        return (4.0 / 3.0) * 3.14159265f * (double)s.radius * (double)s.radius * (double)s.radius;
    return 3.14159265f * (double)s.radius * (double)s.radius * (double)s.length;
}
// run_tick_common.h:216-231 (C_m in pF; myelin state[0] = g-ratio is static)
float seg_capacitance(const HostNet& hn, uint32_t i) {
    const SegLite& s = hn.seg[i];
    float area = seg_area(s);
    float C_m = area * 0.01f;
    if (C_m < 1e-4f) C_m = 1e-4f;
    for (uint8_t j = 0; j < s.modifier_count && j < 16; j++) {
        if (hn.mod(i, j).type == BNC_MOD_MYELIN) {
            float gr = hn.mod(i, j).state[0];
            if (gr <= 0.0f || gr >= 1.0f) gr = 0.6f;
            float factor = 100.0f * (1.0f / gr - 1.0f) / (1.0f / 0.6f - 1.0f);
            C_m /= factor;
            break;
        }
    }
    return C_m;
}

bool type_supported(uint8_t t) {
    switch (t) {
        case 1: case 4: case 7: case 8: case 9: case 11: case 12: case 85: case 98: case 99:
        case 100: case 102: case 103: case 104: case 105: case 106: case 107: case 112:
        case 123: case 129: case 133: case 140: case 141: case 142: case 150: case 200: case 86: case 147: case 114: case 198:
            return true;
        default: return false;
    }
}
bool receptor_supported(uint8_t t) { return t == 8 || t == 9 || t == 11 || t == 12; }
// kernel_dispatch.h:283-309
bool is_ionotropic(uint8_t t) { return t <= 2 || (t >= 8 && t <= 16) || t == 97 || t == 134 || t == 194; }
bool is_myelin_blocked(uint8_t t) {
    static const uint8_t list[] = {107, 151, 152, 153, 133, 85, 202, 203, 204, 150, 205, 206, 207, 154, 156,
                                   157, 159, 112, 123, 121, 105, 195, 84, 96, 191, 200, 201, 140, 158, 168,
                                   129, 130, 131, 132, 103, 209, 104};
    if (is_ionotropic(t)) return true;
    for (uint8_t x : list) if (x == t) return true;
    return false;
}
// modifier_helpers.h:747-758
float bouton_gamma(uint8_t t) {
    switch (t) {
        case 156: return 10.0f; case 157: return 16.0f; case 123: return 11.0f; case 150: return 27.0f;
        case 112: return 7.0f; case 107: return 100.0f; case 141: return 20.7f; case 142: return 20.8f;
        default: return 0.0f;
    }
}
// Presynaptic release modulators (receptors_biological.cpp:428-509, dispatched by
// kernel_dispatch.h:575-604): kind << 4 | the cleft transmitter the type reads; kind 1
// Gi/o, 2 Gs, 3 ionotropic; 0 for every other type (the dispatch's default factor 1).
uint8_t modulator_code(uint8_t t) {
    switch (t) {
        case 18: case 19: return 0x13;   // 5-HT1A, 5-HT1B: serotonin
        case 22: return 0x12;            // D2: dopamine
        case 27: return 0x15;            // A1: adenosine
        case 29: case 30: return 0x10;   // mGluR2, mGluR3: glutamate
        case 35: return 0x16;            // alpha2: noradrenaline
        case 36: return 0x19;            // CB1: endocannabinoid
        case 38: return 0x18;            // H3: histamine
        case 44: return 0x22;            // D1: dopamine
        case 46: return 0x25;            // A2A: adenosine
        case 13: return 0x34;            // nicotinic: acetylcholine
        default: return 0;
    }
}
// run_tick_common.h:199-206
uint8_t nt_from_receptor(uint8_t rt) {
    if (rt == 11 || rt == 17) return 1;
    if (rt == 12) return 7;
    if (rt == 14) return 3;
    if (rt == 13) return 4;
    if (rt == 44 || rt == 22) return 2;
    return 0;
}
// state indices that are parameters (read-only, default when 0) per type
uint8_t param_words(uint8_t t) {
    switch (t) {
        case 1: return 0x1C;      // 2,3,4
        case 85: return 0x34;     // 2,4,5
        case 98: return 0x06;     // 1,2
        case 100: return 0x06;
        case 102: return 0x1D;    // 0,2,3,4
        case 103: return 0x38;    // 3,4,5
        case 104: return 0x06;    // 1,2
        case 105: return 0x3E;    // 1..5
        case 106: return 0x08;    // 3
        case 107: return 0x03;    // 0,1
        case 112: return 0x76;    // 1,2,4,5,6
        case 123: return 0x16;    // 1,2,4
        case 129: return 0x3E;    // 1..5
        case 133: return 0x01;    // 0
        case 141: case 142: return 0x20;  // 5
        case 150: return 0x20;    // 5
        case 200: return 0x7C;    // 2..6
        case 86: return 0x06;     // 1,2
        case 114: case 198: return 0x6C;   // 2,3,5,6
        default: return 0;
    }
}

template <typename T>
T* up(DeviceAllocs* a, const std::vector<T>& v, int* rc) {
    T* p = (T*)a->alloc(v.size() * sizeof(T));
    if (!p) { *rc = BNC_ERR_ALLOC; return nullptr; }
    if (!v.empty() && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        *rc = BNC_ERR_CUDA;
    return p;
}
template <typename T>
T* zeros(DeviceAllocs* a, size_t n, int* rc) {
    T* p = (T*)a->alloc(n * sizeof(T));
    if (!p) { *rc = BNC_ERR_ALLOC; return nullptr; }
    if (cudaMemset(p, 0, n * sizeof(T)) != cudaSuccess) *rc = BNC_ERR_CUDA;
    return p;
}

struct UF {
    std::vector<uint32_t> p;
    explicit UF(uint32_t n) : p(n) { std::iota(p.begin(), p.end(), 0u); }
    uint32_t f(uint32_t x) { while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; } return x; }
    void u(uint32_t a, uint32_t b) { a = f(a); b = f(b); if (a != b) { if (a < b) p[b] = a; else p[a] = b; } }
};

}  // namespace

float host_bouton_gamma(uint8_t type) { return bouton_gamma(type); }
uint8_t param_mask(uint8_t type) { return param_words(type); }
bool host_receptor_supported(uint8_t type) { return receptor_supported(type); }

int upload_stimuli(const Stimuli& stim, NetHost& host, NetDev* dev, DeviceAllocs* allocs) {
    int rc = BNC_OK;
    uint32_t n = host.n_seg;
    // current stimuli: the reference matches segments[i].id (simulation_host.cpp:250-258);
    // ids equal original indices for generated and well-formed networks, others are mapped
    // through the id list at load time by the caller.
    {
        std::vector<uint32_t> cnt(n + 1, 0);
        for (const auto& s : stim.current) if (s.segment_id < n) cnt[host.inv[s.segment_id] + 1]++;
        for (uint32_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
        std::vector<float> amp(cnt[n]), dur(cnt[n]);
        std::vector<unsigned long long> start(cnt[n]);
        std::vector<uint8_t> alive(cnt[n], 1);
        std::vector<uint32_t> pos(cnt.begin(), cnt.end() - 1);
        host.stim_identity = true;
        uint32_t j = 0;
        for (const auto& s : stim.current) {
            if (s.segment_id >= n) { host.stim_identity = false; continue; }
            uint32_t k = pos[host.inv[s.segment_id]]++;
            if (k != j++) host.stim_identity = false;
            amp[k] = s.amplitude_pA; dur[k] = s.duration_ms; start[k] = s.start_tick;
        }
        if (cnt[n]) {
            dev->cs_off = up(allocs, cnt, &rc);
            dev->cs_amp = up(allocs, amp, &rc);
            dev->cs_dur = up(allocs, dur, &rc);
            dev->cs_start = up(allocs, start, &rc);
            dev->cs_alive = up(allocs, alive, &rc);
        } else {
            dev->cs_off = nullptr;
        }
    }
    {
        std::vector<uint32_t> cnt(n + 1, 0);
        for (const auto& s : stim.vclamp) if (s.segment_id < n) cnt[host.inv[s.segment_id] + 1]++;
        for (uint32_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
        std::vector<float> tgt(cnt[n]);
        std::vector<unsigned long long> st(cnt[n]), en(cnt[n]);
        std::vector<uint32_t> pos(cnt.begin(), cnt.end() - 1);
        for (const auto& s : stim.vclamp) {
            if (s.segment_id >= n) continue;
            uint32_t k = pos[host.inv[s.segment_id]]++;
            tgt[k] = s.target_mV; st[k] = s.start_tick; en[k] = s.end_tick;
        }
        if (cnt[n]) {
            dev->vc_off = up(allocs, cnt, &rc);
            dev->vc_target = up(allocs, tgt, &rc);
            dev->vc_start = up(allocs, st, &rc);
            dev->vc_end = up(allocs, en, &rc);
        } else {
            dev->vc_off = nullptr;
        }
    }
    {
        std::vector<uint32_t> cnt(n + 1, 0);
        for (const auto& s : stim.ramp) if (s.segment_id < n) cnt[host.inv[s.segment_id] + 1]++;
        for (uint32_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
        std::vector<float> from(cnt[n]), to(cnt[n]);
        std::vector<unsigned long long> st(cnt[n]), en(cnt[n]);
        std::vector<uint32_t> pos(cnt.begin(), cnt.end() - 1);
        for (const auto& s : stim.ramp) {
            if (s.segment_id >= n) continue;
            uint32_t k = pos[host.inv[s.segment_id]]++;
            from[k] = s.start_pA; to[k] = s.end_pA; st[k] = s.start_tick; en[k] = s.end_tick;
        }
        if (cnt[n]) {
            dev->rp_off = up(allocs, cnt, &rc);
            dev->rp_from = up(allocs, from, &rc);
            dev->rp_to = up(allocs, to, &rc);
            dev->rp_start = up(allocs, st, &rc);
            dev->rp_end = up(allocs, en, &rc);
        } else {
            dev->rp_off = nullptr;
        }
    }
    {
        // Injections (simulation_host.cpp:279-300) land after the segment's step-1
        // currents and before step 2.5, per segment in upload order: ions first, then
        // ligands, which touch other arrays.  With synapses, step 3 zeroes every
        // extracellular neurotransmitter entry before it accumulates (:326-330) and
        // nothing reads the entry in between but step 2.5's own diffusion of it, so an
        // extracellular ligand injection leaves no trace and is dropped here.
        std::vector<uint4> ops;
        bool intra_nt = false;
        for (const auto& j : stim.ion_inj) {
            if (j.segment_id >= n || j.ion_idx < 0 || j.ion_idx >= 7) continue;
            uint32_t a;
            std::memcpy(&a, &j.amount_mM, 4);
            ops.push_back(make_uint4(host.inv[j.segment_id], (uint32_t)j.ion_idx + (j.extracellular ? 8u : 0u), a, 0u));
        }
        for (const auto& j : stim.lig_inj) {
            if (j.segment_id >= n || j.nt_idx < 0 || j.nt_idx >= 15) continue;
            if (!j.intracellular && (dev->flags & NF_SYNAPSES)) continue;
            uint32_t a;
            std::memcpy(&a, &j.amount, 4);
            ops.push_back(make_uint4(host.inv[j.segment_id], (uint32_t)j.nt_idx + (j.intracellular ? 16u : 32u), a, 0u));
            if (j.intracellular) intra_nt = true;
        }
        // An injected intracellular transmitter is a gradient that step 2.5 diffuses.
        if (intra_nt && (dev->flags & NF_DIFFUSION)) dev->flags |= NF_INTRA_NT;
        if (!ops.empty()) {
            std::vector<uint32_t> count(1, (uint32_t)ops.size());
            dev->inj = up(allocs, ops, &rc);
            dev->inj_n = up(allocs, count, &rc);
        } else {
            dev->inj = nullptr;
            dev->inj_n = nullptr;
        }
    }
    return rc;
}

void hostnet_add_segment(HostNet& hn, const BncSegment& s) {
    SegLite L;
    std::memset(&L, 0, sizeof(L));
    L.id = s.id;
    L.segment_type = s.segment_type;
    L.modifier_count = s.modifier_count > BNC_MAX_MODIFIERS ? (uint8_t)BNC_MAX_MODIFIERS : s.modifier_count;
    if (s.modifier_count > BNC_MAX_MODIFIERS && hn.bad_modifier_count_seg == UINT32_MAX)
        hn.bad_modifier_count_seg = (uint32_t)hn.seg.size();
    L.radius = s.radius; L.length = s.length;
    L.pos_z = s.position.z;
    L.V_m = (float)s.V_m;
    for (int q = 0; q < 7; q++) { L.intra_ions[q] = (float)s.intra_ions[q]; L.extra_ions[q] = (float)s.extra_ions[q]; }
    for (int q = 0; q < 15; q++) { L.intra_nt[q] = s.intra_nt[q]; L.neurotransmitter[q] = s.neurotransmitter[q]; }
    L.ATP_level = s.ATP_level; L.temperature = s.temperature; L.transcription_signal = s.transcription_signal;
    L.I_buffer = s.I_buffer;
    L.mod_off = hn.mods.size();
    for (uint8_t j = 0; j < L.modifier_count; j++) {
        const BncModifier& m = s.modifiers[j];
        ModLite M;
        M.type = m.type; M.active_vars = m.active_vars; M.density = (float)m.density;
        for (int k = 0; k < 8; k++) M.state[k] = (float)m.state[k];
        hn.mods.push_back(M);
    }
    hn.seg.push_back(L);
    hn.num_segments = (uint32_t)hn.seg.size();
}

void hostnet_add_synapse(HostNet& hn, const BncSynapse& y) {
    SynLite L;
    std::memset(&L, 0, sizeof(L));
    L.id = y.id; L.pre_segment = y.pre_segment; L.post_segment = y.post_segment; L.type = y.type;
    L.pre_autoreceptor_count = y.pre_autoreceptor_count; L.post_receptor_count = y.post_receptor_count;
    L.refractory = y.refractory;
    L.weight = y.weight; L.delay = y.delay; L.pre_area = y.pre_area; L.post_area = y.post_area;
    L.release_probability = y.release_probability; L.release_amount = y.release_amount;
    L.tau_clearance = y.tau_clearance; L.facilitation = y.facilitation; L.depression = y.depression;
    L.RRP = y.RRP; L.RRP_max = y.RRP_max; L.RRP_recovery = y.RRP_recovery;
    L.bouton_Ca = y.bouton_Ca; L.spine_Ca = y.spine_Ca; L.spine_camkii = y.spine_camkii;
    L.spine_calcineurin = y.spine_calcineurin;
    for (int q = 0; q < 15; q++) L.cleft_neurotransmitter[q] = y.cleft_neurotransmitter[q];
    L.rec_off = hn.recs.size();
    uint8_t npr = y.post_receptor_count > 8 ? 8 : y.post_receptor_count;
    uint8_t npa = y.pre_autoreceptor_count > 8 ? 8 : y.pre_autoreceptor_count;
    for (uint8_t j = 0; j < npr + npa; j++) {
        const BncModifier& m = j < npr ? y.post_receptors[j] : y.pre_autoreceptors[j - npr];
        ModLite M;
        M.type = m.type; M.active_vars = m.active_vars; M.density = (float)m.density;
        for (int k = 0; k < 8; k++) M.state[k] = (float)m.state[k];
        hn.recs.push_back(M);
    }
    hn.syn.push_back(L);
    hn.num_synapses = (uint32_t)hn.syn.size();
}

float host_seg_area(const SegLite& s) { return seg_area(s); }
double host_seg_volume(const SegLite& s) { return seg_volume(s); }
float host_seg_capacitance(const HostNet& hn, uint32_t i) { return seg_capacitance(hn, i); }
bool host_is_myelin_blocked(uint8_t type) { return is_myelin_blocked(type); }
bool host_is_ionotropic(uint8_t type) { return is_ionotropic(type); }
uint8_t host_nt_from_receptor(uint8_t type) { return nt_from_receptor(type); }

void hostnet_from_aos(const BncBionData& aos, HostNet* hn) {
    *hn = HostNet();
    size_t n_mods = 0, n_recs = 0;
    for (uint32_t i = 0; i < aos.num_segments; i++)
        n_mods += aos.segments[i].modifier_count > BNC_MAX_MODIFIERS ? BNC_MAX_MODIFIERS : aos.segments[i].modifier_count;
    for (uint32_t k = 0; k < aos.num_synapses; k++)
        n_recs += (size_t)std::min<uint32_t>(aos.synapses[k].post_receptor_count, 8u) +
                  std::min<uint32_t>(aos.synapses[k].pre_autoreceptor_count, 8u);
    hn->seg.reserve(aos.num_segments);
    hn->mods.reserve(n_mods);
    hn->syn.reserve(aos.num_synapses);
    hn->recs.reserve(n_recs);
    for (uint32_t i = 0; i < aos.num_segments; i++) hostnet_add_segment(*hn, aos.segments[i]);
    hn->conn.assign(aos.connections, aos.connections + aos.num_connections);
    hn->num_connections = aos.num_connections;
    for (uint32_t k = 0; k < aos.num_synapses; k++) hostnet_add_synapse(*hn, aos.synapses[k]);
}

int build_network(const HostNet& hn, const Stimuli& stim, NetDev* dev, NetHost* host,
                  DeviceAllocs* allocs, const BuildOptions& opt) {
    const bool verbose = std::getenv("BNC_VERBOSE") != nullptr;
    auto t_last = std::chrono::steady_clock::now();
    auto lap = [&](const char* what) {
        if (!verbose) return;
        auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "[bnc build] %-28s %8.3f s\n", what, std::chrono::duration<double>(now - t_last).count());
        t_last = now;
    };
    std::memset(dev, 0, sizeof(*dev));
    const uint32_t n = hn.num_segments;
    const HostVec<SegLite>& S = hn.seg;
    const HostNet& aos = hn;
    if (n == 0 || S.empty()) { set_error("network has no segments"); return BNC_ERR_ARG; }
    if (n >= (1u << 31)) { set_error("too many segments"); return BNC_ERR_ARG; }
    // modifier IDs run by registered device modifiers (they override built-in models of
    // the same ID, as the reference's plugin table does on its CPU path)
    bool user_type[256] = {false};
    for (int t = 0; t < 128; t++) user_type[t] = device_modifier_registered((uint8_t)t);
    host->n_seg = n;
    host->n_conn = aos.num_connections;
    host->n_syn_total = aos.num_synapses;
    if (hn.bad_modifier_count_seg != UINT32_MAX) {
        set_error("segment %u: modifier_count > %d", hn.bad_modifier_count_seg, BNC_MAX_MODIFIERS);
        return BNC_ERR_FORMAT;
    }
    // segment ids must be the positions (stimuli and the reference match on id)
    for (uint32_t i = 0; i < n; i++) {
        if (S[i].modifier_count > BNC_MAX_MODIFIERS) { set_error("segment %u: modifier_count %u > 32", i, S[i].modifier_count); return BNC_ERR_FORMAT; }
        for (uint8_t j = 0; j < S[i].modifier_count; j++) {
            const uint8_t t = hn.mod(i, j).type;
            if (!user_type[t] && host_plugin_registered(t)) {
                // the reference would run the plugin's CPU function for this ID
                // (kernel_dispatch.h:336-343); there is no CPU path here
                set_error("segment %u slot %u: modifier type %u is registered by a host plugin (a CPU function); "
                          "register device code for it (biocore_gpu_register_device_modifier)", i, j, t);
                return BNC_ERR_UNSUPPORTED;
            }
            if (!type_supported(t) && !user_type[t]) {
                set_error("segment %u slot %u: modifier type %u has no device implementation in this backend",
                          i, j, t);
                return BNC_ERR_UNSUPPORTED;
            }
        }
    }
    // ---- valid connections and components ----
    std::vector<uint32_t> conn_ok;
    conn_ok.reserve(aos.num_connections);
    UF uf(n);
    for (uint32_t c = 0; c < aos.num_connections; c++) {
        const auto& cn = hn.conn[c];
        if (cn.segment_a >= n || cn.segment_b >= n) continue;  // skipped by every reference loop
        conn_ok.push_back(c);
        uf.u(cn.segment_a, cn.segment_b);
    }
    std::vector<uint32_t> comp_of(n);
    std::vector<uint32_t> comp_size(n, 0);
    for (uint32_t i = 0; i < n; i++) { comp_of[i] = uf.f(i); comp_size[comp_of[i]]++; }
    // components ordered by their smallest segment (root of the union-find is the minimum)
    std::vector<uint32_t> roots;
    for (uint32_t i = 0; i < n; i++) if (comp_of[i] == i) roots.push_back(i);
    std::vector<uint32_t> comp_members_off(n + 1, 0);
    {
        std::vector<uint32_t> rank(n, 0);
        for (uint32_t r = 0; r < roots.size(); r++) rank[roots[r]] = r;
        std::vector<uint32_t> cnt(roots.size() + 1, 0);
        for (uint32_t i = 0; i < n; i++) cnt[rank[comp_of[i]] + 1]++;
        for (size_t r = 0; r < roots.size(); r++) cnt[r + 1] += cnt[r];
        host->perm.assign(n, 0);
        std::vector<uint32_t> pos(cnt.begin(), cnt.end() - 1);
        for (uint32_t i = 0; i < n; i++) host->perm[pos[rank[comp_of[i]]]++] = i;
        comp_members_off.assign(cnt.begin(), cnt.end());
    }
    if (opt.warp_cap < 1 || opt.tile_segs < 32 || opt.tile_segs > (uint32_t)kMaxTileSegs || opt.phase_cap > 4096) {
        set_error("build options out of range (warp_cap %u, tile_segs %u, phase_cap %u)", opt.warp_cap,
                  opt.tile_segs, opt.phase_cap);
        return BNC_ERR_ARG;
    }
    host->opt = opt;
    const uint32_t warp_cap = opt.warp_cap;
    const uint32_t tile_cap = opt.tile_segs;
    // A component larger than a tile spans a pair of tiles run by one 2-CTA cluster.
    // Its segments are laid out depth first from its root (neighbours in ascending
    // order), so cutting the list in half separates subtrees and few connections
    // cross between the two tiles.  The order changes no arithmetic: every gather
    // follows original connection order.
    bool any_big = false;
    for (size_t r = 0; r < roots.size(); r++)
        if (comp_members_off[r + 1] - comp_members_off[r] > tile_cap) any_big = true;
    if (any_big) {
        std::vector<uint32_t> adj_off(n + 1, 0);
        for (uint32_t c : conn_ok) {
            const auto& cn = hn.conn[c];
            if (comp_size[comp_of[cn.segment_a]] <= tile_cap) continue;
            adj_off[cn.segment_a + 1]++;
            adj_off[cn.segment_b + 1]++;
        }
        for (uint32_t i = 0; i < n; i++) adj_off[i + 1] += adj_off[i];
        std::vector<uint32_t> adj(adj_off[n]);
        {
            std::vector<uint32_t> pos(adj_off.begin(), adj_off.end() - 1);
            for (uint32_t c : conn_ok) {
                const auto& cn = hn.conn[c];
                if (comp_size[comp_of[cn.segment_a]] <= tile_cap) continue;
                adj[pos[cn.segment_a]++] = cn.segment_b;
                adj[pos[cn.segment_b]++] = cn.segment_a;
            }
        }
        for (uint32_t i = 0; i < n; i++) std::sort(adj.begin() + adj_off[i], adj.begin() + adj_off[i + 1]);
        std::vector<uint8_t> seen(n, 0);
        std::vector<uint32_t> stack;
        for (size_t r = 0; r < roots.size(); r++) {
            const uint32_t b = comp_members_off[r], e = comp_members_off[r + 1];
            if (e - b <= tile_cap) continue;
            uint32_t k = b;
            stack.assign(1, roots[r]);
            while (!stack.empty()) {
                const uint32_t x = stack.back();
                stack.pop_back();
                if (seen[x]) continue;
                seen[x] = 1;
                host->perm[k++] = x;
                for (uint32_t j = adj_off[x + 1]; j > adj_off[x]; j--)   // smallest neighbour on top
                    if (!seen[adj[j - 1]]) stack.push_back(adj[j - 1]);
            }
            if (k != e) { set_error("internal: depth-first layout of component %zu incomplete", r); return BNC_ERR_ARG; }
        }
    }
    host->inv.assign(n, 0);
    host->perm_identity = true;
    for (uint32_t d = 0; d < n; d++) {
        host->inv[host->perm[d]] = d;
        if (host->perm[d] != d) host->perm_identity = false;
    }
    lap("components");
    // ---- tile packing: whole components, one component per warp slot ----
    std::vector<uint32_t> tile_seg_beg{0};
    std::vector<uint16_t> warp_seg;   // per tile kTileWarps+1 entries
    {
        uint32_t cur_tile_segs = 0, cur_warp = 0, cur_warp_segs = 0;
        std::vector<uint16_t> wb(kTileWarps + 1, 0);
        auto close_tile = [&]() {
            for (int w = (int)cur_warp + 1; w <= kTileWarps; w++) wb[w] = (uint16_t)cur_tile_segs;
            warp_seg.insert(warp_seg.end(), wb.begin(), wb.end());
            tile_seg_beg.push_back(tile_seg_beg.back() + cur_tile_segs);
            cur_tile_segs = 0; cur_warp = 0; cur_warp_segs = 0;
            std::fill(wb.begin(), wb.end(), 0);
        };
        // a tile of `segs` segments of one large component (one warp group)
        auto push_tile = [&](uint32_t segs) {
            std::vector<uint16_t> w(kTileWarps + 1, (uint16_t)segs);
            w[0] = 0;
            warp_seg.insert(warp_seg.end(), w.begin(), w.end());
            tile_seg_beg.push_back(tile_seg_beg.back() + segs);
        };
        for (size_t r = 0; r < roots.size(); r++) {
            uint32_t sz = comp_members_off[r + 1] - comp_members_off[r];
            if (sz > tile_cap) {
                if (sz > 2 * tile_cap) {
                    set_error("connected component of %u segments exceeds two %u-segment tiles", sz, tile_cap);
                    return BNC_ERR_UNSUPPORTED;
                }
                if (cur_tile_segs > 0) close_tile();
                if ((tile_seg_beg.size() - 1) % 2 == 1) push_tile(0);   // the pair starts a cluster
                const uint32_t h = (sz + 1) / 2;
                push_tile(h);
                push_tile(sz - h);
                continue;
            }
            bool fits_warp = cur_warp_segs > 0 && cur_warp_segs + sz <= warp_cap;
            if (!fits_warp && cur_warp_segs > 0) {  // move to the next warp
                cur_warp++;
                wb[cur_warp] = (uint16_t)cur_tile_segs;
                cur_warp_segs = 0;
            }
            if (cur_warp >= (uint32_t)kTileWarps || cur_tile_segs + sz > tile_cap) {
                // the open warp index is past the end or the tile is full: close it
                if (cur_warp >= (uint32_t)kTileWarps) cur_warp = kTileWarps - 1;
                close_tile();
            }
            cur_tile_segs += sz;
            cur_warp_segs += sz;
            wb[cur_warp + 1] = (uint16_t)cur_tile_segs;
        }
        if (cur_tile_segs > 0) close_tile();
        if (any_big && (tile_seg_beg.size() - 1) % 2 == 1) push_tile(0);   // whole clusters only
    }
    const uint32_t T = (uint32_t)tile_seg_beg.size() - 1;
    host->cluster = any_big ? 2 : 1;
    std::vector<uint32_t> tile_of(n);
    for (uint32_t t = 0; t < T; t++)
        for (uint32_t d = tile_seg_beg[t]; d < tile_seg_beg[t + 1]; d++) tile_of[d] = t;
    lap("tiles");
    // ---- connections per tile, in original order ----
    // A connection whose endpoints sit in the two tiles of a pair is in both tiles:
    // each CTA computes it from identical values and gathers it for its own segment.
    // A tile refers to the other tile's endpoint through a ghost slot after its own
    // segments; the diffusion kernel refreshes ghosts from the owner after updates.
    std::vector<uint32_t> tile_edge_beg(T + 1, 0);
    std::vector<uint16_t> warp_edge(T * (kTileWarps + 1), 0);
    std::vector<uint32_t> edge_conn;   // device edge -> original connection index
    std::vector<uint32_t> gh_off(T + 1, 0), gh_seg, gh_src;
    std::vector<uint16_t> e_a, e_b;
    {
        std::vector<std::vector<uint32_t>> tile_conns(T);
        for (uint32_t c : conn_ok) {
            const uint32_t da = host->inv[hn.conn[c].segment_a], db = host->inv[hn.conn[c].segment_b];
            const uint32_t ta = tile_of[da], tb = tile_of[db];
            tile_conns[ta].push_back(c);
            if (tb != ta) {
                if ((ta ^ 1u) != tb) { set_error("internal: connection %u crosses unpaired tiles", c); return BNC_ERR_ARG; }
                tile_conns[tb].push_back(c);
            }
        }
        std::vector<uint32_t> ghosts;
        for (uint32_t t = 0; t < T; t++) {
            const uint32_t e0 = (uint32_t)edge_conn.size();
            const uint32_t ns_t = tile_seg_beg[t + 1] - tile_seg_beg[t];
            ghosts.clear();
            auto local = [&](uint32_t x) -> uint16_t {
                if (tile_of[x] == t) return (uint16_t)(x - tile_seg_beg[t]);
                for (size_t g = 0; g < ghosts.size(); g++) if (ghosts[g] == x) return (uint16_t)(ns_t + g);
                ghosts.push_back(x);
                return (uint16_t)(ns_t + ghosts.size() - 1);
            };
            for (uint32_t c : tile_conns[t]) {
                edge_conn.push_back(c);
                e_a.push_back(local(host->inv[hn.conn[c].segment_a]));
                e_b.push_back(local(host->inv[hn.conn[c].segment_b]));
            }
            for (uint32_t x : ghosts) {
                gh_seg.push_back(x);
                gh_src.push_back(x - tile_seg_beg[tile_of[x]]);   // owner tile is t ^ 1 (the pair)
            }
            gh_off[t + 1] = (uint32_t)gh_seg.size();
            const uint32_t ne_t = (uint32_t)edge_conn.size() - e0;
            for (int w = 0; w <= kTileWarps; w++) warp_edge[t * (kTileWarps + 1) + w] = (uint16_t)(w == 0 ? 0 : ne_t);
            tile_edge_beg[t + 1] = (uint32_t)edge_conn.size();
            if (ne_t > 32767) { set_error("tile %u has more than 32767 connections", t); return BNC_ERR_UNSUPPORTED; }
            if (ns_t + ghosts.size() > 65535) { set_error("tile %u has too many ghost segments", t); return BNC_ERR_UNSUPPORTED; }
        }
    }
    const uint32_t E = (uint32_t)edge_conn.size();
    // ---- barrier groups of the diffusion kernel ----
    // Every pass of step 2.5 couples only the two ends of a connection.  Where no
    // connection of a tile joins segments in different aligned groups of G threads
    // (G = 32, else 64), a group synchronises only itself (a warp, or a 64-thread named
    // barrier) instead of the CTA.  Each connection of such a tile is then handled by
    // the thread of one of its segments: breadth first from each component's first
    // segment, a segment owns the connection it was reached by, so a thread handles at
    // most one.  A tile whose connections cannot all be owned so (a cycle, a repeated
    // connection) keeps CTA-wide barriers.
    std::vector<uint8_t> tile_gmode(T, 0);
    std::vector<uint16_t> seg_edge(n, 0xFFFF);
    host->group_tiles_32 = host->group_tiles_64 = 0;
    if (host->cluster == 1 && opt.group_barriers) {
        std::vector<uint32_t> adj_off, adj, queue;
        std::vector<uint8_t> seen;
        for (uint32_t t = 0; t < T; t++) {
            const uint32_t s0 = tile_seg_beg[t], ns_t = tile_seg_beg[t + 1] - s0;
            const uint32_t e0 = tile_edge_beg[t], ne_t = tile_edge_beg[t + 1] - e0;
            uint32_t G = 0;
            for (uint32_t g : {32u, 64u}) {
                bool ok = true;
                for (uint32_t e = e0; e < e0 + ne_t && ok; e++) ok = e_a[e] < ns_t && e_b[e] < ns_t && e_a[e] / g == e_b[e] / g;
                if (ok) { G = g; break; }
            }
            if (ne_t == 0) { tile_gmode[t] = 32; continue; }   // nothing couples its segments
            if (!G) continue;
            adj_off.assign(ns_t + 1, 0);
            for (uint32_t e = e0; e < e0 + ne_t; e++) { adj_off[e_a[e] + 1]++; adj_off[e_b[e] + 1]++; }
            for (uint32_t x = 0; x < ns_t; x++) adj_off[x + 1] += adj_off[x];
            adj.assign(2 * (size_t)ne_t, 0);
            {
                std::vector<uint32_t> pos(adj_off.begin(), adj_off.end() - 1);
                for (uint32_t e = e0; e < e0 + ne_t; e++) {
                    adj[pos[e_a[e]]++] = (e - e0) << 16 | e_b[e];
                    adj[pos[e_b[e]]++] = (e - e0) << 16 | e_a[e];
                }
            }
            seen.assign(ns_t, 0);
            uint32_t owned = 0;
            for (uint32_t r = 0; r < ns_t; r++) {
                if (seen[r]) continue;
                seen[r] = 1;
                queue.assign(1, r);
                for (size_t h = 0; h < queue.size(); h++) {
                    const uint32_t x = queue[h];
                    for (uint32_t k = adj_off[x]; k < adj_off[x + 1]; k++) {
                        const uint32_t y = adj[k] & 0xFFFFu;
                        if (seen[y]) continue;
                        seen[y] = 1;
                        seg_edge[s0 + y] = (uint16_t)(adj[k] >> 16);
                        owned++;
                        queue.push_back(y);
                    }
                }
            }
            if (owned != ne_t) {
                for (uint32_t x = 0; x < ns_t; x++) seg_edge[s0 + x] = 0xFFFF;
                continue;
            }
            tile_gmode[t] = (uint8_t)G;
        }
    }
    {
        // The kernel is compiled per barrier mode, so the mode is the network's: warps
        // (32) when every tile's connections stay inside aligned warps, else 64-thread
        // groups when every tile's stay inside those (a warp-grouped tile is also
        // 64-grouped), else the CTA.  A 64-thread group is two whole warps: the CTA is
        // a multiple of 64 threads, and its groups take named barriers 1..15.
        uint32_t mts0 = 0;
        for (uint32_t t = 0; t < T; t++) mts0 = std::max(mts0, tile_seg_beg[t + 1] - tile_seg_beg[t]);
        bool all32 = T > 0, all_grouped = T > 0;
        for (uint32_t t = 0; t < T; t++) {
            all32 &= tile_gmode[t] == 32;
            all_grouped &= tile_gmode[t] != 0;
        }
        uint32_t gm = all32 ? 32u : (all_grouped ? 64u : 0u);
        uint32_t th = (mts0 + (gm == 64 ? 63 : 31)) / (gm == 64 ? 64 : 32) * (gm == 64 ? 64 : 32);
        if (gm == 64 && th > 960) {
            gm = 0;
            th = (mts0 + 31) / 32 * 32;
        }
        if (gm == 0) std::fill(seg_edge.begin(), seg_edge.end(), (uint16_t)0xFFFF);
        host->diff_gm = gm;
        host->diff_threads = th < 32 ? 32 : th;
        host->group_tiles_32 = gm == 32 ? T : 0;
        host->group_tiles_64 = gm == 64 ? T : 0;
    }
    std::vector<uint8_t> e_intra(E);
    std::vector<float> e_area(E), e_dist(E);
    for (uint32_t e = 0; e < E; e++) {
        const auto& cn = hn.conn[edge_conn[e]];
        e_intra[e] = cn.is_intracellular;
        const SegLite& A = S[cn.segment_a];
        const SegLite& B = S[cn.segment_b];
        float r_min = A.radius < B.radius ? A.radius : B.radius;
        float area_conn = 3.14159265f * r_min * r_min;
        if (area_conn < 1e-6f) area_conn = 1e-6f;
        float dist = (A.length + B.length) * 0.5f;
        if (dist < 0.1f) dist = 0.1f;
        e_area[e] = area_conn;
        e_dist[e] = dist;
    }
    lap("edges");
    // incidence lists per device segment: the connections of its own tile that touch
    // it, in original connection order, a-role before b-role
    std::vector<uint32_t> inc_off(n + 1, 0);
    for (uint32_t t = 0; t < T; t++)
        for (uint32_t e = tile_edge_beg[t]; e < tile_edge_beg[t + 1]; e++) {
            const auto& cn = hn.conn[edge_conn[e]];
            const uint32_t da = host->inv[cn.segment_a], db = host->inv[cn.segment_b];
            if (tile_of[da] == t) inc_off[da + 1]++;
            if (tile_of[db] == t) inc_off[db + 1]++;
        }
    for (uint32_t i = 0; i < n; i++) inc_off[i + 1] += inc_off[i];
    std::vector<uint16_t> inc(inc_off[n]);
    {
        std::vector<uint32_t> pos(inc_off.begin(), inc_off.end() - 1);
        std::vector<uint64_t> key(inc_off[n]);
        for (uint32_t t = 0; t < T; t++)
            for (uint32_t e = tile_edge_beg[t]; e < tile_edge_beg[t + 1]; e++) {
                const auto& cn = hn.conn[edge_conn[e]];
                const uint16_t le = (uint16_t)(e - tile_edge_beg[t]);
                const uint32_t da = host->inv[cn.segment_a], db = host->inv[cn.segment_b];
                if (tile_of[da] == t) {
                    const uint32_t ka = pos[da]++;
                    inc[ka] = le;
                    key[ka] = ((uint64_t)edge_conn[e] << 1) | 0u;
                }
                if (tile_of[db] == t) {
                    const uint32_t kb = pos[db]++;
                    inc[kb] = (uint16_t)(le | 0x8000u);
                    key[kb] = ((uint64_t)edge_conn[e] << 1) | 1u;
                }
            }
        std::vector<uint32_t> idx;
        for (uint32_t d = 0; d < n; d++) {
            uint32_t b = inc_off[d], e = inc_off[d + 1];
            if (e - b < 2) continue;
            idx.resize(e - b);
            std::iota(idx.begin(), idx.end(), b);
            std::sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return key[x] < key[y]; });
            std::vector<uint16_t> tmpi(e - b);
            for (uint32_t k = 0; k < e - b; k++) tmpi[k] = inc[idx[k]];
            std::copy(tmpi.begin(), tmpi.end(), inc.begin() + b);
        }
    }
    lap("incidence");
    // ---- phase schedule (greedy shortest common supersequence over active types) ----
    std::vector<uint32_t> act_off(n + 1, 0);   // per original segment active slot list
    std::vector<uint8_t> sflags(n, 0);
    // a modifier is active unless it is myelin or a channel myelin blocks
    // (simulation_host.cpp:241; myelin_modulator returns 0 and touches nothing)
    auto seg_flags = [&](uint32_t i) -> uint8_t {
        bool myel = false, nmda = false;
        for (uint8_t j = 0; j < S[i].modifier_count; j++) {
            if (hn.mod(i, j).type == BNC_MOD_MYELIN) myel = true;
            if (hn.mod(i, j).type == BNC_MOD_NMDA) nmda = true;
        }
        return (uint8_t)((myel ? SF_MYELIN : 0) | (nmda ? SF_NMDA : 0));
    };
    auto active = [&](uint8_t t, uint8_t fl) {
        return t != BNC_MOD_MYELIN && !((fl & SF_MYELIN) && is_myelin_blocked(t));
    };
    parallel_for(n, [&](size_t i0, size_t i1) {
        for (uint32_t i = (uint32_t)i0; i < (uint32_t)i1; i++) {
            const uint8_t fl = seg_flags(i);
            uint32_t c = 0;
            for (uint8_t j = 0; j < S[i].modifier_count; j++) c += active(hn.mod(i, j).type, fl) ? 1u : 0u;
            act_off[i + 1] = c;
            sflags[i] = fl;
        }
    });
    uint32_t max_active = 0;
    for (uint32_t i = 0; i < n; i++) {
        max_active = std::max(max_active, act_off[i + 1]);
        act_off[i + 1] += act_off[i];
    }
    HostVec<uint8_t> act_slot(act_off[n]);
    HostVec<uint16_t> item_phase(act_slot.size(), 0);
    HostVec<uint8_t> act_type(act_slot.size());
    parallel_for(n, [&](size_t i0, size_t i1) {
        for (uint32_t i = (uint32_t)i0; i < (uint32_t)i1; i++) {
            uint32_t k = act_off[i];
            for (uint8_t j = 0; j < S[i].modifier_count; j++) {
                const uint8_t t = hn.mod(i, j).type;
                if (!active(t, sflags[i])) continue;
                act_slot[k] = j;
                act_type[k] = t;
                k++;
            }
        }
    });
    lap("active lists");
    uint32_t n_phases = 0;
    {
        std::vector<uint32_t> ptr(n, 0);
        uint64_t remaining = act_slot.size();
        std::vector<uint64_t> count(256);
        const uint32_t cap = opt.phase_cap ? opt.phase_cap : std::max<uint32_t>(2 * max_active + 4, 8);
        bool greedy_ok = true;
        std::mutex mu;
        while (remaining > 0) {
            std::fill(count.begin(), count.end(), 0);
            parallel_for(n, [&](size_t i0, size_t i1) {
                uint64_t local[256] = {0};
                for (size_t i = i0; i < i1; i++) {
                    uint32_t k = act_off[i] + ptr[i];
                    if (k < act_off[i + 1]) local[act_type[k]]++;
                }
                std::lock_guard<std::mutex> lock(mu);
                for (int t = 0; t < 256; t++) count[t] += local[t];
            });
            int best = (int)(std::max_element(count.begin(), count.end()) - count.begin());
            std::atomic<uint64_t> taken{0};
            parallel_for(n, [&](size_t i0, size_t i1) {
                uint64_t c = 0;
                for (size_t i = i0; i < i1; i++) {
                    uint32_t k = act_off[i] + ptr[i];
                    if (k < act_off[i + 1] && act_type[k] == best) {
                        item_phase[k] = (uint16_t)n_phases;
                        ptr[i]++;
                        c++;
                    }
                }
                taken += c;
            });
            remaining -= taken.load();
            n_phases++;
            if (n_phases > cap) { greedy_ok = false; break; }
        }
        if (!greedy_ok) {  // slot-order phases: phase = rank among the segment's active modifiers
            for (uint32_t i = 0; i < n; i++)
                for (uint32_t k = act_off[i]; k < act_off[i + 1]; k++) item_phase[k] = (uint16_t)(k - act_off[i]);
            n_phases = max_active;
        }
    }
    if (n_phases == 0) n_phases = 1;
    lap("phase schedule");
    // ---- items ordered by (phase, type, device segment): two counting passes ----
    // A phase is one launch of the modifier kernel over the whole network; sorting
    // by type inside it keeps warps, and the SMs at any moment, on few channel models.
    struct ItemKey { uint16_t phase; uint8_t type; uint32_t dseg; uint32_t k; };
    // Items are bucketed by (chunk, phase): a chunk is a run of chunk_segs segments whose
    // step-1 records stay resident in L2 while all phases of the chunk run.
    const uint32_t chunk_segs = opt.chunk_segs ? std::min(opt.chunk_segs, n) : n;
    const uint32_t n_chunks = (n + chunk_segs - 1) / chunk_segs;
    host->chunk_segs = chunk_segs;
    host->n_chunks = n_chunks;
    const size_t NB = (size_t)n_chunks * n_phases;
    std::vector<uint32_t> bucket_off(NB + 1, 0);
    for (uint32_t d = 0; d < n; d++) {
        uint32_t i = host->perm[d];
        for (uint32_t k = act_off[i]; k < act_off[i + 1]; k++)
            bucket_off[(size_t)(d / chunk_segs) * n_phases + item_phase[k] + 1]++;
    }
    for (size_t b = 0; b < NB; b++) bucket_off[b + 1] += bucket_off[b];
    // Fused phase groups: F consecutive phases run in one launch, one thread per segment
    // running its items of those phases in order with the step-1 record in registers.
    // That needs every segment's items in phases 0..c-1 (the slot-order schedule), so
    // that the segments with an item in phase p0 + j are the first rows of the group
    // once rows are sorted by their item count, and item (row r, phase p0 + j) sits at
    // bucket_off[p0 + j] + r.  Rows are sorted by (count descending, the types of their
    // items) so that warps run one sequence of models.
    uint32_t fuse = std::min<uint32_t>(std::max<uint32_t>(opt.fuse_phases, 1u), kMaxFuse);
    if (n_chunks != 1 || n_phases < 2) fuse = 1;
    for (uint32_t i = 0; i < n && fuse > 1; i++)
        for (uint32_t k = act_off[i]; k < act_off[i + 1]; k++)
            if (item_phase[k] != k - act_off[i] || user_type[act_type[k]]) { fuse = 1; break; }
    HostVec<ItemKey> keys(act_slot.size());
    if (fuse > 1) {
        uint32_t rank[256];
        uint32_t R = 0;
        {
            bool seen[256] = {false};
            for (uint8_t t : act_type) seen[t] = true;
            for (int t = 0; t < 256; t++) rank[t] = seen[t] ? ++R : 0u;   // 1..R; 0: no item
        }
        // A warp of the group kernel runs, for each item, every model its 32 rows hold
        // there in turn.  Rows sorted by their items' types share a model while enough
        // rows share the types before it; when slots are in no particular order (drawn
        // types listed as drawn), deep groups leave warps on several models per item and
        // the SMs on most of the 26 models' code at once.  The grouping is redone with
        // one phase fewer per group while the mean distinct models per warp and item
        // exceeds kMaxWarpTypes.
        for (;;) {
            // groups are independent (their items go to disjoint phase ranges): one thread each
            const uint32_t n_groups = (n_phases + fuse - 1) / fuse;
            std::vector<int> group_err(n_groups, 0);
            std::vector<uint64_t> g_models(n_groups, 0), g_warp_items(n_groups, 0);
            parallel_for(n_groups, [&](size_t g0, size_t g1) {
                std::vector<uint32_t> rows, tmp, cnt;
                std::vector<uint8_t> kb;
                for (size_t gi = g0; gi < g1; gi++) {
                    const uint32_t p0 = (uint32_t)gi * fuse;
                    const uint32_t F = std::min(fuse, n_phases - p0);
                    const uint32_t W = F + 1;   // per row: the item types of the group, then the count key
                    rows.clear();
                    kb.clear();
                    for (uint32_t d = 0; d < n; d++) {   // device order: the order inside a class
                        const uint32_t i = host->perm[d];
                        const uint32_t c = act_off[i + 1] - act_off[i];
                        if (c <= p0) continue;
                        const uint32_t m = std::min(F, c - p0);
                        rows.push_back(d);
                        for (uint32_t j = 0; j < F; j++) kb.push_back(j < m ? (uint8_t)rank[act_type[act_off[i] + p0 + j]] : 0);
                        kb.push_back((uint8_t)(F - m));
                    }
                    if (rows.size() != bucket_off[p0 + 1] - bucket_off[p0]) { group_err[gi] = 1; continue; }
                    // stable counting sorts, least significant first: the type of each item from
                    // the last phase of the group to the first, then the item count (descending)
                    std::vector<uint32_t> idx(rows.size());
                    std::iota(idx.begin(), idx.end(), 0u);
                    tmp.resize(rows.size());
                    for (int pass = (int)F - 1; pass >= -1; pass--) {
                        const uint32_t j = pass < 0 ? F : (uint32_t)pass;
                        const uint32_t nb = (j == F ? F : R) + 2;
                        cnt.assign(nb, 0u);
                        for (uint32_t x : idx) cnt[kb[(size_t)x * W + j] + 1]++;
                        for (uint32_t c = 0; c + 1 < nb; c++) cnt[c + 1] += cnt[c];
                        for (uint32_t x : idx) tmp[cnt[kb[(size_t)x * W + j]]++] = x;
                        idx.swap(tmp);
                    }
                    for (uint32_t r = 0; r < (uint32_t)idx.size(); r++) {
                        const uint32_t d = rows[idx[r]];
                        const uint32_t i = host->perm[d];
                        const uint32_t m = F - kb[(size_t)idx[r] * W + F];
                        for (uint32_t j = 0; j < m; j++) {
                            const uint32_t k = act_off[i] + p0 + j;
                            const uint32_t pos = bucket_off[p0 + j] + r;
                            if (pos >= bucket_off[p0 + j + 1]) { group_err[gi] = 2; break; }
                            keys[pos] = {(uint16_t)(p0 + j), act_type[k], d, k};
                        }
                        if (group_err[gi]) break;
                    }
                    // distinct models per warp (32 consecutive rows) and item
                    for (size_t w0 = 0; w0 < idx.size(); w0 += 32) {
                        const size_t w1 = std::min(idx.size(), w0 + 32);
                        for (uint32_t j = 0; j < F; j++) {
                            uint64_t bits[4] = {0, 0, 0, 0};
                            for (size_t r = w0; r < w1; r++) {
                                const uint32_t t = kb[(size_t)idx[r] * W + j];
                                if (t) bits[t >> 6] |= 1ull << (t & 63);
                            }
                            const uint32_t c = __builtin_popcountll(bits[0]) + __builtin_popcountll(bits[1]) +
                                               __builtin_popcountll(bits[2]) + __builtin_popcountll(bits[3]);
                            if (c) { g_models[gi] += c; g_warp_items[gi]++; }
                        }
                    }
                }
            }, 1);
            for (uint32_t gi = 0; gi < n_groups; gi++)
                if (group_err[gi]) {
                    set_error("fused phase schedule: phase group %u does not nest (%d)", gi, group_err[gi]);
                    return BNC_ERR_FORMAT;
                }
            uint64_t models = 0, warp_items = 0;
            for (uint32_t gi = 0; gi < n_groups; gi++) { models += g_models[gi]; warp_items += g_warp_items[gi]; }
            host->warp_models = warp_items ? (double)models / (double)warp_items : 1.0;
            if (!opt.fuse_adaptive || fuse <= 2 || n < kAdaptiveFuseMinSegs || host->warp_models <= kMaxWarpTypes)
                break;
            fuse--;
        }
    } else {
        std::vector<uint32_t> pos(bucket_off.begin(), bucket_off.end() - 1);
        for (uint32_t d = 0; d < n; d++) {   // device order: each bucket fills in segment order
            uint32_t i = host->perm[d];
            for (uint32_t k = act_off[i]; k < act_off[i + 1]; k++)
                keys[pos[(size_t)(d / chunk_segs) * n_phases + item_phase[k]]++] = {item_phase[k], act_type[k], d, k};
        }
        std::vector<ItemKey> tmp;
        uint32_t tc[257];
        for (size_t b = 0; b < NB; b++) {   // stable counting sort by type inside each bucket
            uint32_t lo = bucket_off[b], hi = bucket_off[b + 1];
            if (hi - lo < 2) continue;
            std::fill(tc, tc + 257, 0u);
            for (uint32_t q = lo; q < hi; q++) tc[keys[q].type + 1]++;
            for (int t = 0; t < 256; t++) tc[t + 1] += tc[t];
            tmp.assign(keys.begin() + lo, keys.begin() + hi);
            for (const ItemKey& kk : tmp) keys[lo + tc[kk.type]++] = kk;
        }
    }
    host->fuse = fuse;
    lap("item sort");
    const uint32_t NI = (uint32_t)keys.size();
    std::vector<uint32_t> phase_off(bucket_off.begin(), bucket_off.end());
    // The items' values (density, state, flags) are gathered on the device from the
    // modifier records (device_convert_state); the host keeps each item's segment and slot.
    host->item_seg.resize(NI);
    host->item_slot.resize(NI);
    host->phase_off = phase_off;
    parallel_for(NI, [&](size_t q0, size_t q1) {
        for (size_t q = q0; q < q1; q++) {
            host->item_seg[q] = host->perm[keys[q].dseg];
            host->item_slot[q] = act_slot[keys[q].k];
        }
    });
    auto item_type = [&](uint32_t q) { return keys[q].type; };
    bool type_present[256] = {false};   // item types of the network (the scans below skip absent ones)
    for (uint8_t t : act_type) type_present[t] = true;
    if (!allocs) {   // a host-only plan checks what the device conversion would
        FirstError bad;
        parallel_for(NI, [&](size_t q0, size_t q1) {
            for (size_t q = q0; q < q1; q++) {
                const ModLite& m = hn.mod(host->item_seg[q], host->item_slot[q]);
                if (receptor_supported(m.type) && m.active_vars >= 8) bad.note(q);
            }
        });
        if (bad.any()) {
            const uint32_t q = (uint32_t)bad.at.load();
            set_error("segment %u slot %u: active_vars %u out of range", host->item_seg[q], host->item_slot[q],
                      hn.mod(host->item_seg[q], host->item_slot[q]).active_vars);
            return BNC_ERR_FORMAT;
        }
    }
    lap("item fill");
    {   // the state words some item updates on the device (registered types: all 7)
        uint8_t seen[256] = {0};
        for (uint8_t t : act_type) seen[t] = 1;
        uint8_t rows = 0;
        for (int t = 0; t < 256; t++)
            if (seen[t]) rows |= (t < 128 && user_type[t]) ? (uint8_t)0x7F : host_dyn_mask((uint8_t)t);
        host->item_dyn_rows = rows;
    }
    // registered device modifiers: their items form one contiguous run per phase and type
    host->user_ranges.clear();
    std::memset(dev->user_mask, 0, sizeof(dev->user_mask));
    for (uint32_t p = 0; p < (uint32_t)NB; p++) {   // bucket: chunk * n_phases + phase
        uint32_t q = phase_off[p];
        while (q < phase_off[p + 1]) {
            const uint8_t t = item_type(q);
            uint32_t r = q;
            while (r < phase_off[p + 1] && item_type(r) == t) r++;
            if (user_type[t]) {
                host->user_ranges.push_back({p, t, q, r, nullptr});
                dev->user_mask[t >> 5] |= 1u << (t & 31);
            }
            q = r;
        }
    }
    lap("items");
    // ---- per-segment statics in device order (the state is gathered on the device) ----
    std::vector<float> area(n), cm(n);
    std::vector<double> vol(n);
    std::vector<uint8_t> dflags(n);
    bool intra_nt_grad = false, temp_grad = false, txn_grad = false;
    parallel_for(n, [&](size_t d0, size_t d1) {
    for (uint32_t d = (uint32_t)d0; d < (uint32_t)d1; d++) {
        const SegLite& s = S[host->perm[d]];
        area[d] = seg_area(s); vol[d] = seg_volume(s); cm[d] = seg_capacitance(hn, host->perm[d]);
        dflags[d] = sflags[host->perm[d]];
    }
    });
    for (uint32_t c : conn_ok) {
        const auto& cn = hn.conn[c];
        const SegLite& A = S[cn.segment_a];
        const SegLite& B = S[cn.segment_b];
        if (cn.is_intracellular) {
            for (int q = 0; q < 15; q++) if (A.intra_nt[q] != B.intra_nt[q]) intra_nt_grad = true;
            if (A.temperature != B.temperature) temp_grad = true;
            if (A.transcription_signal != B.transcription_signal) txn_grad = true;
        }
    }
    lap("segment state");
    // ---- synapses: valid chemical ones in post-segment CSR order ----
    std::vector<uint32_t> syn_valid;
    bool need_pre_ext = false, any_delay = false;
    uint32_t nt_mask = 0;
    // status of synapse k: 0 kept, 1 skipped (indices out of range), 2 and up an error,
    // whose message is written when `report` is set
    auto check_syn = [&](uint32_t k, bool report) -> int {
        const SynLite& y = hn.syn[k];
        if (y.pre_segment >= n || y.post_segment >= n) return 1;   // simulation_host.cpp:362
        if (y.type > 2) {
            if (report) set_error("synapse %u: type %u", k, (unsigned)y.type);
            return BNC_ERR_UNSUPPORTED;
        }
        if (y.post_receptor_count > BNC_MAX_POST_RECEPTORS || y.pre_autoreceptor_count > BNC_MAX_PRE_AUTORECEPTORS) {
            if (report) set_error("synapse %u: receptor count out of range", k);
            return BNC_ERR_FORMAT;
        }
        // an electrical synapse or dendritic bridge runs only the gap-junction step
        // (simulation_host.cpp:373-402): its receptors and transmitter are never read
        if (y.type != BNC_SYN_CHEMICAL) return 0;
        for (uint8_t j = 0; j < y.post_receptor_count; j++)
            if (host_plugin_registered(hn.post_rec(k, j).type)) {
                if (report)
                    set_error("synapse %u receptor %u: type %u is registered by a host plugin (a CPU function), "
                              "which this backend cannot run", k, j, hn.post_rec(k, j).type);
                return BNC_ERR_UNSUPPORTED;
            } else if (!receptor_supported(hn.post_rec(k, j).type)) {
                if (report)
                    set_error("synapse %u receptor %u: type %u has no device implementation as a receptor", k, j,
                              hn.post_rec(k, j).type);
                return BNC_ERR_UNSUPPORTED;
            }
        for (uint8_t j = 0; j < y.pre_autoreceptor_count; j++)
            if (host_plugin_registered(hn.pre_ar(k, j).type)) {
                if (report)
                    set_error("synapse %u autoreceptor %u: type %u is registered by a host plugin (a CPU function), "
                              "which this backend cannot run", k, j, hn.pre_ar(k, j).type);
                return BNC_ERR_UNSUPPORTED;
            } else if (bouton_gamma(hn.pre_ar(k, j).type) == 0.0f && modulator_code(hn.pre_ar(k, j).type) == 0) {
                if (report)
                    set_error("synapse %u autoreceptor %u: type %u is neither a bouton channel nor a release modulator",
                              k, j, hn.pre_ar(k, j).type);
                return BNC_ERR_UNSUPPORTED;
            }
        uint8_t ntt = y.post_receptor_count > 0 ? nt_from_receptor(hn.post_rec(k, 0).type) : 0;
        for (int q = 0; q < 15; q++)
            if (q != ntt && q != 9 && y.cleft_neurotransmitter[q] != 0.0f) {   // 9: endocannabinoid
                if (report) set_error("synapse %u: cleft holds neurotransmitter %d other than the one it releases", k, q);
                return BNC_ERR_UNSUPPORTED;
            }
        return 0;
    };
    {
        std::vector<int8_t> status(aos.num_synapses);
        parallel_for(aos.num_synapses, [&](size_t k0, size_t k1) {
            for (size_t k = k0; k < k1; k++) status[k] = (int8_t)check_syn((uint32_t)k, false);
        });
        for (uint32_t k = 0; k < aos.num_synapses; k++) {
            if (status[k] == 1) continue;
            if (status[k] != 0) return check_syn(k, true);
            const SynLite& y = hn.syn[k];
            if (y.type != BNC_SYN_CHEMICAL) {   // a gap junction reads both segments' Ca2+
                need_pre_ext = true;
                syn_valid.push_back(k);
                continue;
            }
            if (y.pre_autoreceptor_count > 0 || y.RRP_max > 0.0f) need_pre_ext = true;
            if (y.delay > 0.0f) any_delay = true;
            nt_mask |= 1u << (y.post_receptor_count > 0 ? nt_from_receptor(hn.post_rec(k, 0).type) : 0);
            syn_valid.push_back(k);
        }
    }
    lap("syn check");
    // The synapse kernel's entries: each chemical synapse once, for its post segment;
    // each gap junction twice, for its pre segment (side 2) and then its post segment
    // (side 1), since the reference's loop changes both segments' I_buffer
    // (simulation_host.cpp:373-402).  Entries are kept in original synapse order per
    // owning segment.
    std::vector<uint8_t> ent_side;
    {
        bool any_gap = false;
        for (uint32_t k : syn_valid) if (hn.syn[k].type != BNC_SYN_CHEMICAL) { any_gap = true; break; }
        if (any_gap) {
            std::vector<uint32_t> ent;
            ent.reserve(syn_valid.size() + 64);
            for (uint32_t k : syn_valid) {
                if (hn.syn[k].type != BNC_SYN_CHEMICAL) { ent.push_back(k); ent_side.push_back(2); }
                ent.push_back(k);
                ent_side.push_back(hn.syn[k].type != BNC_SYN_CHEMICAL ? 1 : 0);
            }
            syn_valid.swap(ent);
        }
    }
    auto owner = [&](uint32_t q) {   // device segment of entry q
        const SynLite& y = hn.syn[syn_valid[q]];
        return host->inv[(!ent_side.empty() && ent_side[q] == 2) ? y.pre_segment : y.post_segment];
    };
    const uint32_t K = (uint32_t)syn_valid.size();
    std::vector<uint32_t> post_off(n + 1, 0);
    for (uint32_t q = 0; q < K; q++) post_off[owner(q) + 1]++;
    for (uint32_t i = 0; i < n; i++) post_off[i + 1] += post_off[i];
    {   // stable counting sort by owning device segment (original order within a segment)
        std::vector<uint32_t> pos(post_off.begin(), post_off.end() - 1);
        std::vector<uint32_t> sorted(K);
        std::vector<uint8_t> sorted_side(ent_side.size());
        for (uint32_t q = 0; q < K; q++) {
            const uint32_t at = pos[owner(q)]++;
            sorted[at] = syn_valid[q];
            if (!ent_side.empty()) sorted_side[at] = ent_side[q];
        }
        syn_valid.swap(sorted);
        ent_side.swap(sorted_side);
    }
    lap("syn sort");
    // ---- synapse-kernel threads and the sliced synapse order ----
    // Thread t of the synapse kernel handles segment th_seg[t]: first every segment
    // with synapses, by synapse count descending (stable in device order), then the
    // rest.  Within a warp the lanes that still have a k-th synapse therefore form a
    // prefix, and the k-th synapses of a warp's lanes sit next to each other: synapse
    // (warp w, k, lane l) is at w_off[w] + sum over k' < k of the active lanes + l.
    // Receptors of the synapses of slice (w, k): receptor j of each lane that has
    // one, lanes in order, j ascending.  Each lane still walks its own synapses and
    // receptors in original order.
    std::vector<uint32_t> th_seg;
    std::vector<uint16_t> th_cnt;
    th_seg.reserve(n);
    th_cnt.reserve(n);
    {
        std::vector<uint32_t> post_list, rest_list;
        for (uint32_t d = 0; d < n; d++) (post_off[d + 1] > post_off[d] ? post_list : rest_list).push_back(d);
        // Segments of equal count are ordered by the class sequence of their synapses
        // (bit k: the k-th synapse, in original order, carries an inhibitory receptor),
        // so the lanes of a warp take the same receptor path at each k.  Only which
        // thread runs a segment changes; each thread still walks its segment's synapses
        // in original order.
        std::vector<uint32_t> sig(n, 0);
        parallel_for(post_list.size(), [&](size_t a0, size_t a1) {
            for (size_t a = a0; a < a1; a++) {
                const uint32_t d = post_list[a];
                uint32_t m = 0;
                for (uint32_t q = post_off[d], k = 0; q < post_off[d + 1] && k < 32; q++, k++) {
                    const uint32_t sk = syn_valid[q];
                    const SynLite& y = hn.syn[sk];
                    bool inh = false;
                    for (uint8_t j = 0; j < y.post_receptor_count; j++) {
                        const uint8_t rt = hn.post_rec(sk, j).type;
                        if (rt == 11 || rt == 17 || rt == 12) { inh = true; break; }
                    }
                    if (inh) m |= 1u << k;
                }
                sig[d] = m;
            }
        });
        std::stable_sort(post_list.begin(), post_list.end(), [&](uint32_t a, uint32_t b) {
            const uint32_t ca = post_off[a + 1] - post_off[a], cb = post_off[b + 1] - post_off[b];
            if (ca != cb) return ca > cb;
            return sig[a] < sig[b];
        });
        for (uint32_t d : post_list) {
            const uint32_t c = post_off[d + 1] - post_off[d];
            if (c > 65535) { set_error("segment %u receives %u synapses (at most 65535)", host->perm[d], c); return BNC_ERR_UNSUPPORTED; }
            th_seg.push_back(d);
            th_cnt.push_back((uint16_t)c);
        }
        for (uint32_t d : rest_list) { th_seg.push_back(d); th_cnt.push_back(0); }
    }
    lap("syn threads");
    const uint32_t NW = (n + 31) / 32;
    std::vector<uint32_t> w_off(NW + 1, 0), rw_off(NW + 1, 0);
    std::vector<uint32_t> slot_syn;   // sliced position -> index into syn_valid (post-sorted)
    slot_syn.reserve(K);
    for (uint32_t w = 0; w < NW; w++) {
        w_off[w] = (uint32_t)slot_syn.size();
        uint32_t maxc = 0;
        for (uint32_t l = 0; l < 32 && 32 * w + l < n; l++) maxc = std::max<uint32_t>(maxc, th_cnt[32 * w + l]);
        for (uint32_t k = 0; k < maxc; k++)
            for (uint32_t l = 0; l < 32 && 32 * w + l < n; l++) {
                const uint32_t t = 32 * w + l;
                if (th_cnt[t] > k) slot_syn.push_back(post_off[th_seg[t]] + k);
            }
    }
    w_off[NW] = (uint32_t)slot_syn.size();
    {
        std::vector<uint32_t> sliced(K);
        for (uint32_t q = 0; q < K; q++) sliced[q] = syn_valid[slot_syn[q]];
        syn_valid.swap(sliced);
        if (!ent_side.empty()) {
            std::vector<uint8_t> sliced_side(K);
            for (uint32_t q = 0; q < K; q++) sliced_side[q] = ent_side[slot_syn[q]];
            ent_side.swap(sliced_side);
        }
    }
    lap("syn slices");
    // The synapses' and receptors' values are gathered on the device from their records
    // (device_convert_synapses); the host decides which receptors each synapse keeps.
    std::vector<uint8_t> rc_cnt(K, 0), kept((size_t)K * 8, 0);
    host->syn_orig = syn_valid;
    host->rec_syn.clear(); host->rec_slot.clear();
    host->syn_nt.assign(K, 0);
    // per synapse: 0 or the error its receptors raise (the lowest such synapse is reported)
    auto fill_syn = [&](uint32_t q, bool report) -> int {
        const SynLite& y = hn.syn[syn_valid[q]];
        host->syn_nt[q] = y.post_receptor_count > 0 ? nt_from_receptor(hn.post_rec(syn_valid[q], 0).type) : 0;
        bool myel_post = (sflags[y.post_segment] & SF_MYELIN) != 0;
        uint32_t nr = 0;
        for (uint8_t j = 0; j < y.post_receptor_count; j++) {
            const ModLite& r = hn.post_rec(syn_valid[q], j);
            if (myel_post && is_ionotropic(r.type)) continue;   // simulation_host.cpp:495
            if (r.active_vars >= 8) {
                if (report) set_error("synapse %u receptor %u: active_vars out of range", syn_valid[q], j);
                return BNC_ERR_FORMAT;
            }
            if (r.active_vars >= 3 && r.active_vars <= 6) {
                if (report) set_error("synapse %u receptor %u: active_vars %u not supported", syn_valid[q], j, r.active_vars);
                return BNC_ERR_UNSUPPORTED;
            }
            kept[(size_t)q * 8 + nr] = j;
            nr++;
        }
        rc_cnt[q] = (uint8_t)nr;
        return 0;
    };
    {
        FirstError bad;
        parallel_for(K, [&](size_t q0, size_t q1) {
            for (size_t q = q0; q < q1; q++)
                if (fill_syn((uint32_t)q, false) != 0) bad.note(q);
        });
        if (bad.any()) return fill_syn((uint32_t)bad.at.load(), true);
    }
    lap("syn fill");
    // endocannabinoid retrograde signalling (simulation_host.cpp:578-589): each post
    // segment's first eCB-synthesis modifier (its item) and each synapse's eCB cleft entry
    std::vector<uint32_t> seg_ecb_item;
    std::vector<float> sy_cleft_ecb;
    {
        bool any_ecb = false;
        std::vector<uint8_t> best_slot;
        for (uint32_t q = 0; q < NI && type_present[86]; q++) {
            if (item_type(q) != 86) continue;
            if (!any_ecb) { any_ecb = true; seg_ecb_item.assign(n, UINT32_MAX); best_slot.assign(n, 0xFF); }
            const uint32_t dseg = host->inv[host->item_seg[q]];
            if (host->item_slot[q] < best_slot[dseg]) { best_slot[dseg] = host->item_slot[q]; seg_ecb_item[dseg] = q; }
        }
        for (uint32_t q = 0; q < K && !any_ecb; q++)
            if (hn.syn[syn_valid[q]].cleft_neurotransmitter[9] != 0.0f) any_ecb = true;
        if (any_ecb) {
            sy_cleft_ecb.resize(K);
            for (uint32_t q = 0; q < K; q++) sy_cleft_ecb[q] = hn.syn[syn_valid[q]].cleft_neurotransmitter[9];
        }
    }
    // gap junctions (simulation_host.cpp:373-402, run_tick_common.h:79-122)
    std::vector<uint32_t> sy_gj, gj_pre, gj_post, seg_cx;
    std::vector<float> gj_delay, gj_dep, gj_flt;
    host->gj_syn.clear();
    if (!ent_side.empty()) {
        std::vector<uint32_t>& gap_list = host->gj_syn;   // original indices, ascending
        for (uint32_t q = 0; q < K; q++) if (ent_side[q] == 1) gap_list.push_back(syn_valid[q]);
        std::sort(gap_list.begin(), gap_list.end());
        std::vector<uint32_t> gidx(hn.syn.size(), UINT32_MAX);
        for (uint32_t g = 0; g < gap_list.size(); g++) gidx[gap_list[g]] = g;
        sy_gj.assign(K, UINT32_MAX);
        for (uint32_t q = 0; q < K; q++)
            if (ent_side[q]) sy_gj[q] = gidx[syn_valid[q]] | (ent_side[q] == 2 ? 0x80000000u : 0u);
        // The junction reads both segments' Ca2+ as the loop has left it at its
        // position; the kernel reads it as step 3 began, which is the same while no
        // earlier synapse onto either segment carries an NMDA receptor (the only
        // Ca2+-permeable receptor; a myelinated post segment skips it).
        std::vector<uint32_t> first_nmda(n, UINT32_MAX);
        for (uint32_t k = 0; k < hn.syn.size(); k++) {
            const SynLite& y = hn.syn[k];
            if (y.type != BNC_SYN_CHEMICAL || y.pre_segment >= n || y.post_segment >= n) continue;
            if (sflags[y.post_segment] & SF_MYELIN) continue;
            for (uint8_t j = 0; j < y.post_receptor_count; j++)
                if (hn.post_rec(k, j).type == 9) { first_nmda[y.post_segment] = std::min(first_nmda[y.post_segment], k); break; }
        }
        for (uint32_t k : gap_list) {
            const SynLite& y = hn.syn[k];
            if (first_nmda[y.pre_segment] < k || first_nmda[y.post_segment] < k) {
                set_error("gap junction %u: an earlier synapse onto one of its segments has an NMDA receptor, whose "
                          "Ca2+ the junction would read mid-step", k);
                return BNC_ERR_UNSUPPORTED;
            }
            gj_pre.push_back(host->inv[y.pre_segment]);
            gj_post.push_back(host->inv[y.post_segment]);
            gj_delay.push_back(y.delay);
            gj_dep.push_back(y.depression);
            gj_flt.push_back(y.cleft_neurotransmitter[0]);
        }
        // each segment's connexin-36 and connexin-43 items (at most one of each)
        seg_cx.assign((size_t)2 * n, UINT32_MAX);
        for (uint32_t q = 0; q < NI && (type_present[114] || type_present[198]); q++) {
            const uint8_t t = item_type(q);
            if (t != 114 && t != 198) continue;
            const size_t at = (size_t)(t == 198 ? 1 : 0) * n + host->inv[host->item_seg[q]];
            if (seg_cx[at] != UINT32_MAX) {
                set_error("segment %u holds two connexin-%d modifiers", host->item_seg[q], t == 198 ? 43 : 36);
                return BNC_ERR_UNSUPPORTED;
            }
            seg_cx[at] = q;
        }
    }
    // glia (simulation_host.cpp:351-355, 467-487): the first 256 segments with a GLAST
    // transporter; each synapse gives its capture to the one nearest its post segment in z
    std::vector<uint32_t> gl_seg, gl_off, gl_syn;
    if (K) {
        std::vector<uint32_t> glia;
        for (uint32_t i = 0; i < n && glia.size() < 256 && type_present[147]; i++)
            for (uint8_t j = 0; j < hn.seg[i].modifier_count; j++)
                if (hn.mod(i, j).type == 147) { glia.push_back(i); break; }
        if (!glia.empty()) {
            std::vector<int32_t> near(n, -1);
            for (uint32_t g : glia) near[g] = -2;
            for (uint32_t q = 0; q < K; q++)
                if ((ent_side.empty() || ent_side[q] == 0) && near[hn.syn[syn_valid[q]].post_segment] == -2) {
                    // its own synapses' transmitter and the captures would interleave
                    set_error("synapse %u targets glial segment %u (a segment with a GLAST transporter)",
                              syn_valid[q], hn.syn[syn_valid[q]].post_segment);
                    return BNC_ERR_UNSUPPORTED;
                }
            std::vector<uint32_t> order(K);
            std::iota(order.begin(), order.end(), 0u);
            std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return syn_valid[a] < syn_valid[b]; });
            std::vector<uint32_t> of(K);
            gl_off.assign(glia.size() + 1, 0);
            for (uint32_t q = 0; q < K; q++) {
                if (!ent_side.empty() && ent_side[q] != 0) { of[q] = UINT32_MAX; continue; }   // a gap junction
                const uint32_t post = hn.syn[syn_valid[q]].post_segment;
                if (near[post] < 0) {
                    float best_dz = 1e30f;
                    int32_t best = 0;
                    for (uint32_t gi = 0; gi < glia.size(); gi++) {
                        const float dz = std::fabs(hn.seg[glia[gi]].pos_z - hn.seg[post].pos_z);
                        if (dz < best_dz) { best_dz = dz; best = (int32_t)gi; }
                    }
                    near[post] = best;
                }
                of[q] = (uint32_t)near[post];
                gl_off[of[q] + 1]++;
            }
            for (size_t gi = 0; gi < glia.size(); gi++) gl_off[gi + 1] += gl_off[gi];
            gl_syn.resize(gl_off.back());
            std::vector<uint32_t> pos(gl_off.begin(), gl_off.end() - 1);
            for (uint32_t q : order)   // original synapse order per glial segment
                if (of[q] != UINT32_MAX) gl_syn[pos[of[q]]++] = q;
            for (uint32_t g : glia) gl_seg.push_back(host->inv[g]);
        }
    }
    lap("syn ecb gap glia");
    // release modulators of the autoreceptors, per sliced synapse in autoreceptor order
    std::vector<uint32_t> md_off;
    std::vector<uint8_t> md_code;
    std::vector<double> md_scale;
    std::vector<float> md_st;
    host->md_syn.clear(); host->md_slot.clear();
    {
        uint32_t total = 0;
        std::vector<uint32_t> cnt(K, 0);
        for (uint32_t q = 0; q < K; q++) {
            const SynLite& y = hn.syn[syn_valid[q]];
            for (uint8_t j = 0; j < y.pre_autoreceptor_count; j++)
                if (modulator_code(hn.pre_ar(syn_valid[q], j).type)) cnt[q]++;
            total += cnt[q];
        }
        if (total) {
            md_off.assign(K + 1, 0);
            for (uint32_t q = 0; q < K; q++) md_off[q + 1] = md_off[q] + cnt[q];
            md_code.resize(total); md_scale.resize(total); md_st.resize(total);
            host->md_syn.resize(total); host->md_slot.resize(total);
            for (uint32_t q = 0; q < K; q++) {
                const SynLite& y = hn.syn[syn_valid[q]];
                uint32_t o = md_off[q];
                // effective_area_mod: state[7], which the release step sets to pre_area, if > 0
                const float area = y.pre_area > 0.0f ? y.pre_area : 1.0f;
                for (uint8_t j = 0; j < y.pre_autoreceptor_count; j++) {
                    const ModLite& m = hn.pre_ar(syn_valid[q], j);
                    const uint8_t code = modulator_code(m.type);
                    if (!code) continue;
                    md_code[o] = code;
                    md_scale[o] = (double)m.density * (double)area;
                    md_st[o] = m.state[0];
                    host->md_syn[o] = syn_valid[q];
                    host->md_slot[o] = j;
                    o++;
                }
            }
        }
    }
    lap("syn modulators");
    // receptor order: slice by slice, receptor j of each lane that has one.  A warp's
    // receptors are those of its synapses, so a prefix sum of per-warp counts places
    // each warp's run and the warps fill in parallel.
    for (uint32_t w = 0; w < NW; w++) {
        uint32_t c = 0;
        for (uint32_t q = w_off[w]; q < w_off[w + 1]; q++) c += rc_cnt[q];
        rw_off[w + 1] = rw_off[w] + c;
    }
    const size_t NRC = rw_off[NW];
    host->rec_syn.resize(NRC); host->rec_slot.resize(NRC);
    parallel_for(NW, [&](size_t w0, size_t w1) {
        for (uint32_t w = (uint32_t)w0; w < (uint32_t)w1; w++) {
            size_t o = rw_off[w];
            uint32_t maxc = 0;
            for (uint32_t l = 0; l < 32 && 32 * w + l < n; l++) maxc = std::max<uint32_t>(maxc, th_cnt[32 * w + l]);
            uint32_t q = w_off[w];
            for (uint32_t k = 0; k < maxc; k++) {
                uint32_t a = 0;   // lanes with a k-th synapse: a prefix of the warp
                while (a < 32 && 32 * w + a < n && th_cnt[32 * w + a] > k) a++;
                uint32_t maxr = 0;
                for (uint32_t l = 0; l < a; l++) maxr = std::max<uint32_t>(maxr, rc_cnt[q + l]);
                for (uint32_t j = 0; j < maxr; j++)
                    for (uint32_t l = 0; l < a; l++) {
                        const uint32_t qq = q + l;
                        if (rc_cnt[qq] <= j) continue;
                        const uint8_t slot = kept[(size_t)qq * 8 + j];
                        host->rec_syn[o] = qq;
                        host->rec_slot[o] = slot;
                        o++;
                    }
                q += a;
            }
        }
    }, 1024);
    rw_off[NW] = (uint32_t)NRC;

    lap("synapses");
    const uint32_t NR = (uint32_t)NRC;
    lap("receptors");
    // tile sizes for the shared-memory plan: own segments (threads), own + ghost
    // segments (the per-segment array stride), connections
    uint32_t mts = 0, mte = 0, mst = 0;
    for (uint32_t t = 0; t < T; t++) {
        const uint32_t ns_t = tile_seg_beg[t + 1] - tile_seg_beg[t];
        mts = std::max(mts, ns_t);
        mst = std::max(mst, ns_t + gh_off[t + 1] - gh_off[t]);
        mte = std::max(mte, tile_edge_beg[t + 1] - tile_edge_beg[t]);
    }
    host->max_tile_segs = mts;
    host->max_tile_stride = mst;
    host->max_tile_edges = mte;
    host->smem_bytes = diffusion_smem_bytes(mst, mte);
    if (host->smem_bytes > 227 * 1024) {
        set_error("tile of %u segments (%u with ghosts) and %u connections needs %zu bytes of shared memory "
                  "(227 KB per CTA)", mts, mst, mte, host->smem_bytes);
        return BNC_ERR_UNSUPPORTED;
    }
    // ---- convergence groups of the residual-controlled Jacobi mode: the connected
    // components, numbered in device order within each tile (within each tile pair for
    // 2-CTA clusters, whose halves share one component); bit 15 marks a group's first
    // segment ----
    std::vector<uint16_t> seg_grp(n, 0);
    {
        const uint32_t span = host->cluster == 2 ? 2u : 1u;
        std::vector<uint32_t> local(n, UINT32_MAX);   // component root -> group index of the current tile
        for (uint32_t t0 = 0; t0 < T; t0 += span) {
            const uint32_t d0 = tile_seg_beg[t0], d1 = tile_seg_beg[std::min(T, t0 + span)];
            uint32_t next = 0;
            for (uint32_t d = d0; d < d1; d++) {
                const uint32_t root = comp_of[host->perm[d]];
                bool first = false;
                if (local[root] == UINT32_MAX) { local[root] = next++; first = true; }
                if (local[root] >= 0x800u) {
                    set_error("tile %u holds more than 2048 components", t0);
                    return BNC_ERR_UNSUPPORTED;
                }
                seg_grp[d] = (uint16_t)(local[root] | (first ? 0x8000u : 0u));
            }
            for (uint32_t d = d0; d < d1; d++) local[comp_of[host->perm[d]]] = UINT32_MAX;
        }
    }
    // ---- upload (skipped for a host-only plan) ----
    int rc = BNC_OK;
    dev->n_seg = n; dev->n_tiles = T; dev->n_items = NI; dev->n_phases = n_phases;
    dev->n_syn = K; dev->n_rec = NR; dev->n_edges = E;
    uint32_t flags = 0;
    if (!conn_ok.empty()) flags |= NF_DIFFUSION;
    if (aos.num_synapses > 0) flags |= NF_SYNAPSES;     // the reset keys on num_synapses, valid or not
    if (intra_nt_grad) flags |= NF_INTRA_NT;
    if (temp_grad) flags |= NF_TEMP;
    if (txn_grad) flags |= NF_TXN;
    if (need_pre_ext) flags |= NF_PRE_EXT;
    if (any_delay) flags |= NF_DELAY;
    if (!(flags & NF_SYNAPSES)) flags |= NF_NT_DIFFUSE_OUT;
    dev->flags = flags;
    bool any_nmda = false;
    for (uint32_t i = 0; i < n; i++) if (sflags[i] & SF_NMDA) any_nmda = true;
    dev->nt_used_mask = nt_mask | (any_nmda ? 1u : 0u) | (sy_cleft_ecb.empty() ? 0u : 1u << 9);
    dev->syn_extras = (!md_off.empty() || !sy_cleft_ecb.empty() || !gl_seg.empty() || !sy_gj.empty()) ? 1u : 0u;
    dev->n_gj = (uint32_t)gj_pre.size();
    dev->n_glia = (uint32_t)gl_seg.size();
    if (allocs) {
        {
            uint32_t bad = UINT32_MAX;
            rc = device_convert_state(hn, host->perm, host->inv, host->item_seg, host->item_slot, dev, allocs, &bad);
            if (rc != BNC_OK) return rc;
            if (bad != UINT32_MAX) {
                set_error("segment %u slot %u: active_vars %u out of range", host->item_seg[bad], host->item_slot[bad],
                          hn.mod(host->item_seg[bad], host->item_slot[bad]).active_vars);
                return BNC_ERR_FORMAT;
            }
        }
        dev->area = up(allocs, area, &rc);
        dev->vol = up(allocs, vol, &rc);
        dev->cm = up(allocs, cm, &rc);
        dev->sflags = up(allocs, dflags, &rc);
        dev->c21_cur = zeros<float2>(allocs, n, &rc);
        dev->rec = zeros<SegRec>(allocs, n, &rc);
        dev->pre_rec = zeros<float4>(allocs, n, &rc);
        if (need_pre_ext) {
            dev->pre_ext = zeros<float4>(allocs, n, &rc);
            dev->pre_ext2 = zeros<float>(allocs, n, &rc);
        }
        dev->tile_seg_beg = up(allocs, tile_seg_beg, &rc);
        dev->tile_edge_beg = up(allocs, tile_edge_beg, &rc);
        dev->phase_off = up(allocs, phase_off, &rc);
        dev->warp_seg = up(allocs, warp_seg, &rc);
        dev->warp_edge = up(allocs, warp_edge, &rc);
        dev->seg_edge = host->diff_gm ? up(allocs, seg_edge, &rc) : nullptr;
        dev->e_a = up(allocs, e_a, &rc);
        dev->e_b = up(allocs, e_b, &rc);
        dev->e_intra = up(allocs, e_intra, &rc);
        dev->e_area = up(allocs, e_area, &rc);
        dev->e_dist = up(allocs, e_dist, &rc);
        dev->inc_off = up(allocs, inc_off, &rc);
        dev->inc = up(allocs, inc, &rc);
        dev->gh_off = up(allocs, gh_off, &rc);
        dev->gh_seg = up(allocs, gh_seg, &rc);
        dev->gh_src = up(allocs, gh_src, &rc);
        for (auto& ur : host->user_ranges) {
            int krc = device_modifier_kernel((uint8_t)ur.type, &ur.kernel);
            if (krc != BNC_OK) return krc;
        }
        dev->th_seg = up(allocs, th_seg, &rc);
        dev->th_cnt = up(allocs, th_cnt, &rc);
        dev->w_off = up(allocs, w_off, &rc);
        dev->rw_off = up(allocs, rw_off, &rc);
        if (rc == BNC_OK) rc = device_convert_synapses(hn, host->syn_orig, host->inv, host->rec_syn, host->rec_slot, dev, allocs);
        dev->rc_cnt = up(allocs, rc_cnt, &rc);
        if (!sy_gj.empty()) {
            dev->sy_gj = up(allocs, sy_gj, &rc);
            dev->gj_pre = up(allocs, gj_pre, &rc);
            dev->gj_post = up(allocs, gj_post, &rc);
            dev->gj_delay = up(allocs, gj_delay, &rc);
            dev->gj_dep = up(allocs, gj_dep, &rc);
            dev->gj_dep_new = up(allocs, gj_dep, &rc);
            dev->gj_flt = up(allocs, gj_flt, &rc);
            dev->gj_flt_new = up(allocs, gj_flt, &rc);
            dev->seg_cx = up(allocs, seg_cx, &rc);
            dev->n_gj = (uint32_t)gj_pre.size();
        }
        dev->model_extras = (type_present[86] || type_present[114] || type_present[147] || type_present[198]) ? 1u : 0u;
        if (!gl_seg.empty()) {
            dev->gl_cap = zeros<float>(allocs, K, &rc);
            dev->gl_seg = up(allocs, gl_seg, &rc);
            dev->gl_off = up(allocs, gl_off, &rc);
            dev->gl_syn = up(allocs, gl_syn, &rc);
            dev->n_glia = (uint32_t)gl_seg.size();
        }
        if (!sy_cleft_ecb.empty()) {
            dev->sy_cleft_ecb = up(allocs, sy_cleft_ecb, &rc);
            if (!seg_ecb_item.empty()) dev->seg_ecb_item = up(allocs, seg_ecb_item, &rc);
        }
        if (!md_off.empty()) {
            dev->md_off = up(allocs, md_off, &rc);
            dev->md_code = up(allocs, md_code, &rc);
            dev->md_scale = up(allocs, md_scale, &rc);
            dev->md_st = up(allocs, md_st, &rc);
            dev->n_md = (uint32_t)md_st.size();
        }
        if (any_delay) {
            dev->dl_arr = zeros<unsigned long long>(allocs, (size_t)4 * K, &rc);
            dev->dl_amt = zeros<float>(allocs, (size_t)4 * K, &rc);
            dev->dl_nt = zeros<uint8_t>(allocs, (size_t)4 * K, &rc);
        }
        dev->spike_count = zeros<uint32_t>(allocs, n, &rc);
        dev->err_flag = zeros<int>(allocs, 1, &rc);
        dev->seg_grp = up(allocs, seg_grp, &rc);
        dev->jac_stats = zeros<uint32_t>(allocs, 4, &rc);
        dev->ledger = zeros<double>(allocs, 14, &rc);
        dev->diff_mode = 0;
        dev->jac_max = 0;
        dev->jac_tol = 0.0;
        if (rc == BNC_OK) rc = upload_stimuli(stim, *host, dev, allocs);
        if (rc != BNC_OK) { set_error("device allocation/upload failed (%d)", rc); return rc; }
    }
    lap("upload");
    // ---- algorithmic bytes per tick of this schema (what one tick must move at minimum) ----
    {
        // kernel A per segment: read V, 14 ions, ATP, geometry+C_m (radius, length, area,
        // vol, cm, type, flags), write V, 14 ions, ATP, I_buffer, pre-record.
        double seg_a = 4 * 2 + 56 * 2 + 4 * 2 + (4 + 4 + 4 + 8 + 4 + 1 + 1) + 8 + 16;
        if (flags & NF_INTRA_NT) seg_a += 120;
        if (flags & NF_TEMP) seg_a += 8;
        if (flags & NF_TXN) seg_a += 8;
        if (flags & NF_DIFFUSION) seg_a += 4 * 2.0 * E / n + 8 * 2.0 * E / n;   // incidence + edge statics
        // modifier items: meta + density read, dynamic state read+write
        double items = 0;
        for (uint32_t q = 0; q < NI; q++) {
            const uint8_t t = item_type(q);
            int dyn = 0;
            switch (t) {
                case 1: case 8: case 11: case 12: case 85: case 140: case 141: case 142: case 200: dyn = 2; break;
                case 9: dyn = 2; break;
                case 150: dyn = 3; break;
                case 102: case 103: case 104: case 105: case 112: case 123: case 129: dyn = 1; break;
                default: dyn = 0;
            }
            if (t == 85) dyn = 3;
            items += 4 + 4 + 8.0 * dyn;
        }
        // kernel B per segment: I_buffer, V rw, 7 intra ions rw, 4 extra ions, C_m, flags,
        // used neurotransmitters written, CSR offset
        int nt_used = __builtin_popcount(dev->nt_used_mask);
        double seg_b = 8 + 4 * 2 + 28 * 2 + 16 + 4 + 1 + 4.0 * nt_used + 4;
        // per synapse: pre index, id, pre-record, scalar params, dynamic state rw, receptors
        double syn = 4 + 4 + 16 + 4 * 5 + 1 + 1 + (4 * 6 + 1) * 2 + 4;
        double rec = 0;
        rec += (1 + 4 + 8.0 * 2) * NR;
        host->seg_bytes = (seg_a + seg_b) * n + items;
        host->syn_bytes = syn * K + rec + 4.0 * (K + 1);
        host->tile_bytes = seg_a * n + items;
        host->synk_bytes = seg_b * n + host->syn_bytes;
        host->algo_bytes_per_tick = host->seg_bytes + host->syn_bytes;
        // Per kernel of the three-kernel tick (the state between steps 1 and 2.5 makes
        // one round trip through HBM, which the tick-level figure above does not count):
        // k_modifiers reads V, 14 ions, ATP, area, vol, the static Cav2.1 gate and writes
        // V, 14 ions, ATP, I_buffer, the Cav2.1 gate; k_diffusion reads them back with
        // C_m and the connection statics and writes the state and the presynaptic record.
        host->mod_bytes = (4 * 2 + 56 * 2 + 4 * 2 + 4 + 8 + 8 + 8 + 8) * (double)n + items;
        double seg_d = 4 * 2 + 56 * 2 + 4 * 2 + 4 + 4 + 8 + 8 + 8 + 16;
        if (flags & NF_INTRA_NT) seg_d += 120;
        if (flags & NF_TEMP) seg_d += 8;
        if (flags & NF_TXN) seg_d += 8;
        if (flags & NF_DIFFUSION) seg_d += 4 * 2.0 * E / n + 8 * 2.0 * E / n;
        host->diff_bytes = seg_d * n;
    }
    return BNC_OK;
}

}  // namespace bnc
