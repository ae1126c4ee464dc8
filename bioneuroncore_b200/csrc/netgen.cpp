// netgen.cpp -- seeded synthetic networks in the reference's data model.
//
// Generator choices (documented, since the workload descriptions leave them open):
//  * Morphology: segment 0 of a neuron is the soma (segment_type 1, sphere); the
//    remaining segments are an even split into a dendrite chain and an axon chain
//    (segment_type 2, cylinders), both attached to the soma.  Trees: a complete
//    binary tree rooted at the soma.  Length U[10,50] um, radius log-U[0.3,5] um.
//  * Every axon segment carries Cav2.1 (type 140): release is gated by bouton Ca2+,
//    which only a Cav2.1 modifier on the presynaptic segment can raise (reference
//    include/modifier_helpers.h:764-806).
//  * Small set per segment: Nav1.6 (141; Nav1.2 142 on dendrites), Kv delayed
//    rectifier (123), K2P leak (107), Cav1.3 (1), Na/K pump (7), myelin (4) on odd
//    axon segments.  Large set: 16 draws with replacement from 24 types with the
//    weights in kLargeTypes, listed by type ID (BNC_NETGEN_DRAW_ORDER keeps draw order);
//    the tick processes a segment's modifiers in slot order either way.
//  * Synapses: presynaptic segment uniform over axon segments, postsynaptic
//    uniform over soma+dendrite segments; 80 % AMPA / 20 % GABA-A receptor class;
//    release probability 0.3, tau_clearance 1 ms, release_amount 1, areas 0.1 um2.
//    Large network: 8 receptors per synapse of the same class (AMPA/NMDA or
//    GABA-A/glycine), weight log-normal(mu=-1, sigma=0.5).
//  * Stimuli: 10 % of somata (seeded choice) get a current step for the whole run.
#include "netgen.h"
#include <cmath>
#include <cstring>
#include <algorithm>

namespace bnc {

namespace {

struct Rng {  // SplitMix64-seeded xorshift64*
    uint64_t s;
    explicit Rng(uint64_t seed) {
        uint64_t z = seed + 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        s = (z ^ (z >> 31)) | 1ull;
    }
    uint64_t next() {
        s ^= s >> 12; s ^= s << 25; s ^= s >> 27;
        return s * 0x2545F4914F6CDD1Dull;
    }
    double u01() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return n ? next() % n : 0; }
    double normal() {
        double u1 = u01(), u2 = u01();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct TypeSpec { uint8_t type; float weight; float density; int cls; };
// cls: 0 Na, 1 K, 2 leak, 3 Ca, 4 other (scaled by conductance_scale[cls] for 0..3)
const TypeSpec kLargeTypes[24] = {
    {BNC_MOD_NAV16, 2.0f, 15.0f, 0},   {BNC_MOD_NAV12, 2.0f, 15.0f, 0},
    {BNC_MOD_KV_DR, 3.0f, 8.3f, 1},    {BNC_MOD_K2P, 3.0f, 4.17f, 2},
    {BNC_MOD_PUMP_NAK, 2.0f, 1500.0f, 4}, {BNC_MOD_KV42, 1.0f, 0.4f, 1},
    {BNC_MOD_KV7, 1.0f, 1.0f, 1},      {BNC_MOD_KV31, 1.0f, 1.0f, 1},
    {BNC_MOD_SK, 1.0f, 0.12f, 1},      {BNC_MOD_BK, 1.0f, 0.03f, 1},
    {BNC_MOD_KIR, 1.0f, 0.033f, 1},    {BNC_MOD_NAP, 1.0f, 1.0f, 0},
    {BNC_MOD_HCN1, 1.0f, 120.0f, 4},   {BNC_MOD_NALCN, 1.0f, 0.11f, 2},
    {BNC_MOD_CAV13, 1.0f, 0.04f, 3},   {BNC_MOD_CAV31, 1.0f, 0.28f, 3},
    {BNC_MOD_PMCA, 1.0f, 300.0f, 4},   {BNC_MOD_NCX, 1.0f, 30.0f, 4},
    {BNC_MOD_KCC2, 1.0f, 0.093f, 4},   {BNC_MOD_CA_BUFFER, 1.0f, 0.5f, 4},
    {BNC_MOD_AMPA, 0.5f, 0.05f, 4},    {BNC_MOD_NMDA, 0.25f, 0.05f, 4},
    {BNC_MOD_GABAA, 0.5f, 0.05f, 4},   {BNC_MOD_GLYCINE, 0.25f, 0.05f, 4},
};

const float kIonIn[BNC_ION_COUNT] = {12.0f, 140.0f, 1e-4f, 7.0f, 0.5f, 0.0f, 6e-5f};
const float kIonOut[BNC_ION_COUNT] = {145.0f, 4.0f, 2.0f, 120.0f, 1.0f, 0.0f, 4e-5f};

struct Family {
    uint32_t n_neurons, segs, depth;
    uint64_t n_syn;
    bool tree;
    bool large_set;
    int receptors_per_syn;
    float stim_pA;
};

Family family_defaults(uint32_t fam) {
    switch (fam) {
        case BNC_NET_SMALL: return {64, 32, 0, 400, false, false, 1, 200.0f};
        case BNC_NET_LARGE: return {100000, 64, 0, 10000000, false, true, 8, 200.0f};
        case BNC_NET_TREES: return {16384, 0, 10, 0, true, false, 1, 200.0f};
        case BNC_NET_ENSEMBLE_MEMBER: return {64, 32, 0, 400, false, false, 1, 200.0f};
        case BNC_NET_ADJOINT: return {256, 64, 0, 2000, false, false, 1, 1000.0f};
        default: return {0, 0, 0, 0, false, false, 0, 0.0f};
    }
}

void set_mod(BncModifier& m, uint8_t type, double density) {
    std::memset(&m, 0, sizeof(m));
    m.type = type;
    m.density = (double)(float)density;            // float-representable: FP32 state holds it exactly
    if (type == BNC_MOD_MYELIN) m.state[0] = (double)0.7f;  // g-ratio
    if (type == BNC_MOD_KV7) m.state[6] = 1.0;     // PIP2 present (0 closes the channel)
    if (type == BNC_MOD_CAV21) m.state[1] = (double)0.8f;   // inactivation gate near rest steady state
    if (type == BNC_MOD_NMDA) m.state[2] = 1.0;    // CDI gate starts uninactivated
}

float scale_of(const BncNetgenParams& p, int cls) {
    if (cls < 0 || cls > 3) return 1.0f;
    float s = p.conductance_scale[cls];
    return s > 0.0f ? s : 1.0f;
}

}  // namespace

int generate_network(const BncNetgenParams& p, NetSink& sink, NetShape* shape_out) {
    Family f = family_defaults(p.family);
    if (f.n_neurons == 0 && f.segs == 0 && !f.tree) return BNC_ERR_ARG;
    uint32_t n_neurons = p.n_neurons ? p.n_neurons : f.n_neurons;
    uint32_t depth = p.tree_depth ? p.tree_depth : f.depth;
    if (f.tree && (depth < 1 || depth > 14)) return BNC_ERR_ARG;
    uint32_t segs = f.tree ? ((1u << (depth + 1)) - 1u) : (p.segs_per_neuron ? p.segs_per_neuron : f.segs);
    if (n_neurons == 0 || segs < 2 || segs > 4096) return BNC_ERR_ARG;
    uint64_t n_seg64 = (uint64_t)n_neurons * segs;
    if (n_seg64 >= 0xFFFFFFF0ull) return BNC_ERR_ARG;
    uint32_t n_seg = (uint32_t)n_seg64;
    uint32_t n_dend = f.tree ? 0 : (segs - 1) / 2;      // dendrite chain length
    uint32_t n_axon = f.tree ? 0 : segs - 1 - n_dend;   // axon chain length
    uint64_t n_syn = p.n_synapses;
    if (n_syn == 0) n_syn = (uint64_t)((double)f.n_syn * ((double)n_neurons / (double)f.n_neurons) + 0.5);
    if ((p.flags & BNC_NETGEN_NO_SYNAPSES) || f.tree) n_syn = 0;
    uint32_t n_conn = (p.flags & BNC_NETGEN_NO_CONNECTIONS) ? 0 : n_neurons * (segs - 1);
    uint32_t n_stim = (p.flags & BNC_NETGEN_NO_STIMULI) ? 0 : (uint32_t)(0.1 * n_neurons + 0.5);
    if (n_stim == 0 && !(p.flags & BNC_NETGEN_NO_STIMULI) && n_neurons >= 1) n_stim = 1;

    // electrical synapses between the somata of consecutive neurons, spread through
    // the chemical ones in the synapse order
    const uint64_t n_gj = ((p.flags & BNC_NETGEN_GAP_JUNCTIONS) && n_syn && n_neurons > 1 && !f.tree) ? n_neurons - 1 : 0;

    NetShape shape;
    shape.n_neurons = n_neurons; shape.n_segments = n_seg; shape.n_connections = n_conn;
    shape.n_synapses = n_syn + n_gj; shape.n_stimuli = n_stim;
    if (shape_out) *shape_out = shape;

    Rng rng_geo(p.seed * 4 + 1), rng_mod(p.seed * 4 + 2), rng_syn(p.seed * 4 + 3), rng_stim(p.seed * 4 + 4);
    Rng rng_extra(p.seed * 4 + 0x9E37);   // BNC_NETGEN_SYNAPSE_EXTRAS only
    Rng rng_modul(p.seed * 4 + 0x5BD1);   // BNC_NETGEN_RELEASE_MODULATORS only
    float wsum = 0.0f;
    for (const auto& t : kLargeTypes) wsum += t.weight;

    sink.begin(n_neurons, n_seg, n_conn, n_syn + n_gj, n_stim);

    BncSegment seg;
    for (uint32_t nrn = 0; nrn < n_neurons; nrn++) {
        BncNeuron nr;
        std::memset(&nr, 0, sizeof(nr));
        nr.id = nrn; nr.segment_start = nrn * segs; nr.segment_count = segs;
        nr.soma_index = nrn * segs; nr.threshold = -40.0f; nr.type = 0;
        sink.neuron(nr);
        for (uint32_t k = 0; k < segs; k++) {
            std::memset(&seg, 0, sizeof(seg));
            uint32_t gi = nrn * segs + k;
            seg.id = gi;
            seg.neuron_id = nrn;
            bool soma = (k == 0);
            bool axon = !f.tree && k > n_dend;
            uint32_t axon_idx = axon ? (k - n_dend - 1) : 0;
            seg.segment_type = soma ? BNC_SEG_SOMA : BNC_SEG_NEURITE;
            seg.length = (float)(10.0 + 40.0 * rng_geo.u01());
            seg.radius = (float)std::exp(std::log(0.3) + rng_geo.u01() * (std::log(5.0) - std::log(0.3)));
            if (soma && seg.radius < 3.0f) seg.radius = 3.0f + seg.radius;  // somata are the fat compartments
            seg.position.x = (float)nrn * 100.0f;
            seg.position.y = (float)k * 10.0f;
            seg.direction.y = 1.0f;
            seg.V_m = -65.0;
            for (int i = 0; i < BNC_ION_COUNT; i++) {
                double pin = 1.0, pout = 1.0;
                if (p.flags & BNC_NETGEN_PERTURB_IONS) {
                    pin = 0.95 + 0.1 * rng_geo.u01();
                    pout = 0.95 + 0.1 * rng_geo.u01();
                }
                seg.intra_ions[i] = (double)kIonIn[i] * pin;
                seg.extra_ions[i] = (double)kIonOut[i] * pout;
            }
            seg.ATP_level = 2.0f;
            seg.temperature = 37.0f;
            seg.ER_Ca2 = 0.4f;
            int mc = 0;
            if (f.large_set) {
                int picks[16];
                for (int d = 0; d < 16; d++) {
                    float r = (float)rng_mod.u01() * wsum;
                    int pick = 23;
                    for (int t = 0; t < 24; t++) {
                        if (r < kLargeTypes[t].weight) { pick = t; break; }
                        r -= kLargeTypes[t].weight;
                    }
                    picks[d] = pick;
                }
                if (!(p.flags & BNC_NETGEN_DRAW_ORDER))   // list the drawn modifiers by type ID
                    std::sort(picks, picks + 16, [](int a, int b) { return kLargeTypes[a].type < kLargeTypes[b].type; });
                for (int d = 0; d < 16; d++) {
                    const TypeSpec& ts = kLargeTypes[picks[d]];
                    set_mod(seg.modifiers[mc++], ts.type, ts.density * scale_of(p, ts.cls));
                }
            } else {
                uint8_t nav = (!soma && !axon && !f.tree) ? BNC_MOD_NAV12 : BNC_MOD_NAV16;
                set_mod(seg.modifiers[mc++], nav, 15.0 * scale_of(p, 0));
                set_mod(seg.modifiers[mc++], BNC_MOD_KV_DR, 8.3 * scale_of(p, 1));
                set_mod(seg.modifiers[mc++], BNC_MOD_K2P, 4.17 * scale_of(p, 2));
                // the fitting family keeps the three fitted conductances unless asked for
                // the whole small set
                if (p.family != BNC_NET_ADJOINT || (p.flags & BNC_NETGEN_FULL_SMALL_SET)) {
                    set_mod(seg.modifiers[mc++], BNC_MOD_CAV13, 0.04 * scale_of(p, 3));
                    set_mod(seg.modifiers[mc++], BNC_MOD_PUMP_NAK, 1500.0);
                }
                if (axon && (axon_idx & 1u)) set_mod(seg.modifiers[mc++], BNC_MOD_MYELIN, 1.0);
            }
            if (axon) set_mod(seg.modifiers[mc++], BNC_MOD_CAV21, 100.0 * scale_of(p, 3));
            if ((p.flags & BNC_NETGEN_GAP_JUNCTIONS) && soma && mc + 2 <= BNC_MAX_MODIFIERS) {
                set_mod(seg.modifiers[mc], 114, 1.0);   // connexin-36
                seg.modifiers[mc].state[0] = (double)0.8f;
                seg.modifiers[mc].state[4] = 1.0;
                mc++;
                if (nrn & 1u) {                         // connexin-43 on every other soma
                    set_mod(seg.modifiers[mc], 198, 0.5);
                    seg.modifiers[mc].state[0] = (double)0.6f;
                    seg.modifiers[mc].state[4] = 1.0;
                    mc++;
                }
            }
            if ((p.flags & BNC_NETGEN_GLIA) && axon && (axon_idx % 4u) == 0 && mc < BNC_MAX_MODIFIERS)
                set_mod(seg.modifiers[mc++], 147, 1.0);   // GLAST: a glial segment
            if (p.flags & BNC_NETGEN_GLIA) seg.position.z = (float)((nrn * 7u) % 13u) * 10.0f + (float)k;
            if ((p.flags & BNC_NETGEN_ECB) && !axon && mc < BNC_MAX_MODIFIERS) {
                set_mod(seg.modifiers[mc], 86, 1.0);   // eCB synthesis
                seg.modifiers[mc].state[0] = (double)0.5f;
                mc++;
            }
            seg.modifier_count = (uint8_t)mc;
            // intra_connection_ids: the connections touching this segment (the reference
            // loader fills the same list, bion_loader_host.cpp:410-425)
            if (n_conn) {
                uint32_t cnt = 0;
                uint32_t base = nrn * (segs - 1);
                // connection j (0-based within the neuron) joins child j+1 to its parent
                if (k > 0) seg.intra_connection_ids[cnt++] = base + (k - 1);
                if (f.tree) {
                    uint32_t c1 = 2 * k + 1, c2 = 2 * k + 2;
                    if (c1 < segs) seg.intra_connection_ids[cnt++] = base + (c1 - 1);
                    if (c2 < segs) seg.intra_connection_ids[cnt++] = base + (c2 - 1);
                } else {
                    if (k == 0) {
                        if (n_dend > 0) seg.intra_connection_ids[cnt++] = base + 0;
                        if (n_axon > 0) seg.intra_connection_ids[cnt++] = base + n_dend;
                    } else if (k < n_dend || (axon && k + 1 < segs)) {
                        seg.intra_connection_ids[cnt++] = base + k;
                    }
                }
                seg.intra_connection_count = (uint8_t)cnt;
            }
            sink.segment(seg);
        }
    }

    if (n_conn) {
        for (uint32_t nrn = 0; nrn < n_neurons; nrn++) {
            uint32_t s0 = nrn * segs;
            for (uint32_t k = 1; k < segs; k++) {
                BncIntraConnection c;
                std::memset(&c, 0, sizeof(c));
                uint32_t parent;
                if (f.tree) parent = (k - 1) / 2;
                else if (k == 1 || k == n_dend + 1) parent = 0;
                else parent = k - 1;
                c.segment_a = s0 + parent;
                c.segment_b = s0 + k;
                c.is_intracellular = 1;
                sink.connection(c);
            }
        }
    }

    if (n_syn) {
        uint64_t n_axon_total = (uint64_t)n_neurons * n_axon;
        uint64_t n_post_total = (uint64_t)n_neurons * (1 + n_dend);
        BncSynapse sy;
        uint64_t gj_done = 0;
        for (uint64_t i = 0; i < n_syn; i++) {
            std::memset(&sy, 0, sizeof(sy));
            uint64_t a = rng_syn.below(n_axon_total);
            uint64_t b = rng_syn.below(n_post_total);
            uint32_t pre = (uint32_t)((a / n_axon) * segs + 1 + n_dend + (a % n_axon));
            uint32_t post = (uint32_t)((b / (1 + n_dend)) * segs + (b % (1 + n_dend)));
            bool inhib = rng_syn.u01() < 0.2;
            sy.id = (uint32_t)i;
            sy.pre_segment = pre;
            sy.post_segment = post;
            sy.type = BNC_SYN_CHEMICAL;
            sy.weight = f.large_set ? (float)std::exp(-1.0 + 0.5 * rng_syn.normal()) : 1.0f;
            sy.delay = 0.0f;
            sy.pre_area = 0.1f;
            sy.post_area = 0.1f;
            int nr = f.receptors_per_syn;
            for (int j = 0; j < nr; j++) {
                uint8_t rt;
                if (j == 0) rt = ((p.flags & BNC_NETGEN_GLYCINE) && (i & 1)) ? BNC_MOD_GLYCINE
                                                                             : (inhib ? BNC_MOD_GABAA : BNC_MOD_AMPA);
                else if (inhib) rt = (rng_syn.u01() < 0.5) ? BNC_MOD_GABAA : BNC_MOD_GLYCINE;
                else rt = (rng_syn.u01() < 0.5) ? BNC_MOD_AMPA : BNC_MOD_NMDA;
                set_mod(sy.post_receptors[j], rt, 200.0);
            }
            if ((p.flags & BNC_NETGEN_NMDA) && sy.post_receptors[0].type == BNC_MOD_AMPA && nr < BNC_MAX_POST_RECEPTORS)
                set_mod(sy.post_receptors[nr++], BNC_MOD_NMDA, 200.0);
            sy.post_receptor_count = (uint8_t)nr;
            if (p.flags & BNC_NETGEN_SYNAPSE_EXTRAS) {
                if (rng_extra.u01() < 0.3) {
                    sy.RRP_max = 25.0f;
                    sy.RRP = (float)(10.0 + 15.0 * rng_extra.u01());
                    sy.RRP_recovery = 0.01f;
                }
                if (rng_extra.u01() < 0.3) {
                    const bool nav = rng_extra.u01() < 0.5;
                    set_mod(sy.pre_autoreceptors[0], nav ? BNC_MOD_NAV16 : BNC_MOD_KV_DR, nav ? 0.5 : 1.0);
                    sy.pre_autoreceptor_count = 1;
                }
                if (rng_extra.u01() < 0.3) sy.delay = (float)(0.5 + 1.5 * rng_extra.u01());
            }
            if ((p.flags & BNC_NETGEN_ECB) && rng_modul.u01() < 0.5 &&
                sy.pre_autoreceptor_count < BNC_MAX_PRE_AUTORECEPTORS) {
                BncModifier& m = sy.pre_autoreceptors[sy.pre_autoreceptor_count++];
                set_mod(m, 36, (double)(float)(0.5 + 0.5 * rng_modul.u01()));   // CB1
            }
            if (p.flags & BNC_NETGEN_RELEASE_MODULATORS) {
                static const uint8_t kModulators[12] = {18, 19, 22, 27, 29, 30, 35, 36, 38, 44, 46, 13};
                if (rng_modul.u01() < 0.5) {
                    const int nm = rng_modul.u01() < 0.5 ? 1 : 2;
                    for (int q = 0; q < nm && sy.pre_autoreceptor_count < BNC_MAX_PRE_AUTORECEPTORS; q++) {
                        BncModifier& m = sy.pre_autoreceptors[sy.pre_autoreceptor_count++];
                        set_mod(m, kModulators[rng_modul.below(12)], (double)(float)(0.2 + 0.8 * rng_modul.u01()));
                        m.state[0] = (double)(float)(0.5 * rng_modul.u01());
                    }
                }
            }
            sy.release_probability = 0.3f;
            sy.release_amount = 1.0f;
            sy.tau_clearance = 1.0f;
            sy.facilitation = 0.0f;
            sy.depression = 0.01f;
            sy.bouton_Ca = 1e-4f;
            sy.spine_Ca = 1e-4f;
            sink.synapse(sy);
            while (gj_done < n_gj && (i + 1) * (n_gj + 1) >= (gj_done + 1) * n_syn) {
                std::memset(&sy, 0, sizeof(sy));
                sy.id = (uint32_t)(n_syn + gj_done);
                sy.pre_segment = (uint32_t)gj_done * segs;
                sy.post_segment = (uint32_t)(gj_done + 1) * segs;
                sy.type = (gj_done & 1u) ? 2 : BNC_SYN_ELECTRICAL;   // dendritic bridge, electrical
                sy.delay = (gj_done % 3u == 0) ? 0.5f : 0.0f;        // 0.5 ms: the filtered current
                sy.weight = 1.0f;
                sy.tau_clearance = 1.0f;
                sink.synapse(sy);
                gj_done++;
            }
        }
    }

    if (n_stim) {
        // seeded choice of distinct somata (partial Fisher-Yates over neuron ids)
        std::vector<uint32_t> ids(n_neurons);
        for (uint32_t i = 0; i < n_neurons; i++) ids[i] = i;
        for (uint32_t i = 0; i < n_stim; i++) {
            uint32_t j = i + (uint32_t)rng_stim.below(n_neurons - i);
            std::swap(ids[i], ids[j]);
        }
        std::sort(ids.begin(), ids.begin() + n_stim);
        for (uint32_t i = 0; i < n_stim; i++) {
            BncCurrentStimulus st;
            std::memset(&st, 0, sizeof(st));
            st.segment_id = ids[i] * segs;
            st.amplitude_pA = p.stim_pA > 0.0f ? p.stim_pA : f.stim_pA;
            st.duration_ms = p.stim_duration_ms > 0.0f ? p.stim_duration_ms : 1e9f;
            st.start_tick = 0;
            sink.stimulus(st);
        }
    }
    sink.end();
    return BNC_OK;
}

}  // namespace bnc
