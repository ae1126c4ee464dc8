// backend.cu -- the backend object behind the C ABI of include/bnc_b200.h.
//
// One Backend per handle, bound to one device and one stream.  The drop-in
// gpu_backend_* calls keep the reference's semantics (gpu_backend_cuda.cu:316-390):
// the host AoS view returned by gpu_backend_bion_data is refreshed after every
// gpu_backend_run_tick.  bnc_run_ticks runs many ticks without that refresh.
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "net.h"
#include "par.h"
#include "netgen.h"
#include "hostnet.h"
#include "bion_file.h"

namespace bnc {

struct Backend {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool loaded = false;
    bool failed = false;
    bool owns_aos = false;
    BncBionData aos{};        // host AoS view (drop-in)
    NetDev dev{};
    NetHost host;
    DeviceAllocs allocs;
    DeviceAllocs stim_allocs;
    Stimuli stim;
    // injections uploaded but not yet applied by a tick (the device list is consumed by
    // the next tick; these copies let a checkpoint carry them)
    std::vector<BncIonInjection> pend_ion;
    std::vector<BncLigandInjection> pend_lig;
    uint64_t tick = 0;
    uint64_t ticks_run = 0;
    // Drop-in records (aos.segments, aos.synapses) in managed memory, written on the
    // device after each tick; the index maps the export kernels need (owned by allocs)
    bool aos_managed = false;
    struct {
        uint32_t* perm;       // device segment -> record
        uint32_t* item_seg;   // item -> record
        uint16_t* item_sm;    // item -> modifier slot | state words it updates << 8
        uint32_t* syn_orig;   // device synapse -> record
        uint8_t* syn_nt;      // device synapse -> the cleft entry it carries
        uint32_t* rec_syn;    // device receptor -> device synapse
        uint8_t* rec_slot;    // device receptor -> receptor slot
        uint32_t* md_syn;     // release modulator -> record
        uint8_t* md_slot;     // release modulator -> autoreceptor slot
        uint32_t* gj_syn;     // gap junction -> record
    } xm{};
    uint32_t tick_stride = 1;   // the tick counter's step per tick (2: the reference's batch mode)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // ensemble members (empty for a single network): ranges in original order
    std::vector<BncEnsembleMember> members;
    // captured tick loop (bnc_run_ticks_graph)
    unsigned long long* clock = nullptr;   // device [2], owned by allocs
    cudaGraphExec_t graph_exec = nullptr;
    float graph_dt = 0.0f;

    ~Backend() {
        cudaSetDevice(device);
        drop_graph();
        allocs.release();
        stim_allocs.release();
        free_aos();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
    void free_aos() {
        if (owns_aos) {
            delete[] aos.neurons;
            delete[] aos.connections;
            delete[] static_cast<uint8_t*>(aos.nuclei);
            if (aos_managed) {
                cudaFree(aos.segments);
                cudaFree(aos.synapses);
            } else {
                delete[] aos.segments;
                delete[] aos.synapses;
            }
        }
        std::memset(&aos, 0, sizeof(aos));
        owns_aos = false;
        aos_managed = false;
        std::memset(&xm, 0, sizeof(xm));
    }
    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }
    void reset_network() {
        drop_graph();
        clock = nullptr;
        members.clear();
        allocs.release();
        stim_allocs.release();
        free_aos();
        std::memset(&dev, 0, sizeof(dev));
        host = NetHost();
        stim = Stimuli();
        pend_ion.clear();
        pend_lig.clear();
        loaded = false;
        failed = false;
        tick = 0;
        ticks_run = 0;
    }
};

static int cuda_fail(cudaError_t e, const char* what) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return BNC_ERR_CUDA;
}

// ---- AoS <- device export ----
template <typename T>
static bool d2h(std::vector<T>& v, const T* p, size_t n) {
    v.resize(n);
    if (n == 0) return true;
    return cudaMemcpy(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess;
}

// Pinned staging for exports, kept for the process and grown on demand (one exporter at
// a time); pageable memory when a pinned allocation fails.
namespace {
std::mutex g_stage_mu;
void* g_stage = nullptr;
size_t g_stage_cap = 0;
std::vector<unsigned char> g_stage_pageable;

unsigned char* stage_reserve(size_t bytes) {
    if (bytes <= g_stage_cap && g_stage) return static_cast<unsigned char*>(g_stage);
    if (g_stage) cudaFreeHost(g_stage);
    g_stage = nullptr;
    g_stage_cap = 0;
    if (cudaMallocHost(&g_stage, bytes) == cudaSuccess) {
        g_stage_cap = bytes;
        return static_cast<unsigned char*>(g_stage);
    }
    cudaGetLastError();
    g_stage = nullptr;
    g_stage_pageable.resize(bytes);
    return g_stage_pageable.data();
}
}  // namespace

// Device state -> the host AoS view.  Fields the network's flags show cannot change on
// the device (intracellular NT, temperature, transcription without gradients) and the
// modifier state words no item type updates are not copied; the scatter into the AoS
// records runs on all host cores.
int export_network(const NetDev& d, const NetHost& h, uint64_t ticks_run, BncBionData* aos) {
    if (!aos || !aos->segments) return BNC_OK;
    const uint32_t n = d.n_seg, NI = d.n_items, K = d.n_syn, NR = d.n_rec;
    const bool x_int = (d.flags & NF_INTRA_NT) != 0, x_temp = (d.flags & NF_TEMP) != 0,
               x_txn = (d.flags & NF_TXN) != 0;
    const uint8_t rows = h.item_dyn_rows;
    // staging layout (floats, then the refractory bytes)
    size_t off = 0;
    auto take = [&](size_t floats) { size_t o = off; off += floats; return o; };
    const size_t oV = take(n), oIn = take((size_t)7 * n), oOut = take((size_t)7 * n), oNt = take((size_t)15 * n),
                 oAtp = take(n), oInt = x_int ? take((size_t)15 * n) : 0, oTemp = x_temp ? take(n) : 0,
                 oTxn = x_txn ? take(n) : 0;
    size_t oSt[7];
    for (int k = 0; k < 7; k++) oSt[k] = ((rows >> k) & 1u) ? take(NI) : 0;
    size_t oSy[8] = {0}, oRc = 0, oMd = 0, oEc = 0, oGd = 0, oGf = 0;
    if (K) {
        for (int f = 0; f < 8; f++) oSy[f] = take(K);
        oRc = take((size_t)3 * NR);
        oMd = take(d.n_md);
        oEc = d.sy_cleft_ecb ? take(K) : 0;
        oGd = take(d.n_gj);
        oGf = take(d.n_gj);
    }
    const size_t bytes = off * sizeof(float) + K;
    std::vector<uint32_t> gjv;   // the gap-junction sides among the entries
    std::lock_guard<std::mutex> lock(g_stage_mu);
    unsigned char* base = stage_reserve(bytes);
    float* F = reinterpret_cast<float*>(base);
    uint8_t* refr = base + off * sizeof(float);
    bool ok = true;
    auto get = [&](size_t o, const void* src, size_t nbytes) {
        if (ok && nbytes) ok = cudaMemcpy(F + o, src, nbytes, cudaMemcpyDeviceToHost) == cudaSuccess;
    };
    get(oV, d.V, (size_t)n * 4);
    get(oIn, d.ion_in, (size_t)7 * n * 4);
    get(oOut, d.ion_out, (size_t)7 * n * 4);
    get(oNt, d.nt, (size_t)15 * n * 4);
    get(oAtp, d.atp, (size_t)n * 4);
    if (x_int) get(oInt, d.intra_nt, (size_t)15 * n * 4);
    if (x_temp) get(oTemp, d.temp, (size_t)n * 4);
    if (x_txn) get(oTxn, d.txn, (size_t)n * 4);
    for (int k = 0; k < 7; k++)
        if ((rows >> k) & 1u) get(oSt[k], d.it_st + (size_t)k * NI, (size_t)NI * 4);
    if (K) {
        const float* src[8] = {d.sy_bouton, d.sy_spine, d.sy_camkii, d.sy_calcn, d.sy_facil, d.sy_weight,
                               d.sy_cleft, d.sy_rrp};
        for (int f = 0; f < 8; f++) get(oSy[f], src[f], (size_t)K * 4);
        get(oRc, d.rc_st, (size_t)3 * NR * 4);
        get(oMd, d.md_st, (size_t)d.n_md * 4);
        if (d.sy_cleft_ecb) get(oEc, d.sy_cleft_ecb, (size_t)K * 4);
        get(oGd, d.gj_dep, (size_t)d.n_gj * 4);
        get(oGf, d.gj_flt, (size_t)d.n_gj * 4);
        if (ok && d.sy_gj) ok = d2h(gjv, d.sy_gj, K);
        if (ok) ok = cudaMemcpy(refr, d.sy_refr, K, cudaMemcpyDeviceToHost) == cudaSuccess;
    }
    if (!ok) { set_error("export: device read failed"); return BNC_ERR_CUDA; }
    parallel_for(n, [&](size_t d0, size_t d1) {
        for (size_t dd = d0; dd < d1; dd++) {
            BncSegment& s = aos->segments[h.perm[dd]];
            s.V_m = F[oV + dd];
            for (int q = 0; q < 7; q++) {
                s.intra_ions[q] = F[oIn + (size_t)q * n + dd];
                s.extra_ions[q] = F[oOut + (size_t)q * n + dd];
            }
            for (int q = 0; q < 15; q++) s.neurotransmitter[q] = F[oNt + (size_t)q * n + dd];
            if (x_int) for (int q = 0; q < 15; q++) s.intra_nt[q] = F[oInt + (size_t)q * n + dd];
            s.ATP_level = F[oAtp + dd];
            if (x_temp) s.temperature = F[oTemp + dd];
            if (x_txn) s.transcription_signal = F[oTxn + dd];
            if (ticks_run > 0) s.I_buffer = 0.0;   // step 4 clears it (simulation_host.cpp:624)
        }
    });
    parallel_for(NI, [&](size_t q0, size_t q1) {
        for (size_t q = q0; q < q1; q++) {
            BncSegment& s = aos->segments[h.item_seg[q]];
            BncModifier& m = s.modifiers[h.item_slot[q]];
            const uint8_t t = m.type;
            const bool user = t < 128 && ((d.user_mask[t >> 5] >> (t & 31)) & 1u);
            const uint8_t wm = user ? (uint8_t)0x7F : host_dyn_mask(t);
            for (int k = 0; k < 7; k++)
                if ((wm >> k) & 1u) m.state[k] = F[oSt[k] + q];
            if (ticks_run > 0)
                m.state[7] = (s.segment_type == 1 || s.segment_type == 3 || s.segment_type == 4)
                    ? 4.0f * 3.14159265f * s.radius * s.radius : 2.0f * 3.14159265f * s.radius * s.length;
        }
    });
    if (K) {
        parallel_for(K, [&](size_t q0, size_t q1) {
            for (size_t q = q0; q < q1; q++) {
                if (!gjv.empty() && gjv[q] != UINT32_MAX) continue;   // a gap junction's side
                BncSynapse& y = aos->synapses[h.syn_orig[q]];
                y.bouton_Ca = F[oSy[0] + q]; y.spine_Ca = F[oSy[1] + q]; y.spine_camkii = F[oSy[2] + q];
                y.spine_calcineurin = F[oSy[3] + q]; y.facilitation = F[oSy[4] + q]; y.weight = F[oSy[5] + q];
                y.cleft_neurotransmitter[h.syn_nt[q]] = F[oSy[6] + q];
                y.RRP = F[oSy[7] + q]; y.refractory = refr[q];
                if (d.sy_cleft_ecb) y.cleft_neurotransmitter[9] = F[oEc + q];
                if (ticks_run > 0) y.depression = F[oSy[4] + q] + 0.01f;
            }
        });
        parallel_for(NR, [&](size_t r0, size_t r1) {
            for (size_t r = r0; r < r1; r++) {
                BncSynapse& y = aos->synapses[h.syn_orig[h.rec_syn[r]]];
                BncModifier& m = y.post_receptors[h.rec_slot[r]];
                m.state[0] = F[oRc + r]; m.state[1] = F[oRc + (size_t)NR + r];
                m.state[2] = F[oRc + (size_t)2 * NR + r];
                if (ticks_run > 0) m.state[7] = y.post_area;
            }
        });
        for (uint32_t g = 0; g < d.n_gj; g++) {
            BncSynapse& y = aos->synapses[h.gj_syn[g]];
            y.depression = F[oGd + g];
            y.cleft_neurotransmitter[0] = F[oGf + g];
        }
        for (uint32_t q = 0; q < d.n_md; q++) {
            BncSynapse& y = aos->synapses[h.md_syn[q]];
            BncModifier& m = y.pre_autoreceptors[h.md_slot[q]];
            m.state[0] = F[oMd + q];
            if (ticks_run > 0) m.state[7] = y.pre_area;
        }
    }
    return BNC_OK;
}

// ---- generator -> compact host network (no AoS materialised) ----
namespace {
struct HostNetSink : NetSink {
    HostNet* hn;
    std::vector<BncCurrentStimulus>* stim;
    void begin(uint32_t, uint32_t n_segments, uint32_t n_connections, uint64_t n_synapses, uint32_t) override {
        *hn = HostNet();
        hn->seg.reserve(n_segments);
        hn->mods.reserve((size_t)n_segments * 17);
        hn->conn.reserve(n_connections);
        hn->syn.reserve(n_synapses);
        hn->recs.reserve(n_synapses * 8);
        hn->num_connections = n_connections;
    }
    void neuron(const BncNeuron&) override {}
    void segment(const BncSegment& s) override { hostnet_add_segment(*hn, s); }
    void connection(const BncIntraConnection& c) override { hn->conn.push_back(c); }
    void synapse(const BncSynapse& s) override { hostnet_add_synapse(*hn, s); }
    void stimulus(const BncCurrentStimulus& st) override { stim->push_back(st); }
};
// Appends networks one after another into one HostNet: every index a member
// holds (segment ids, connection endpoints, synapse pre/post, stimulus targets) is
// offset by the member's first segment; synapse ids are kept.
struct EnsembleSink : NetSink {
    HostNet* hn;
    std::vector<BncCurrentStimulus>* stim;
    uint32_t base = 0;
    uint64_t n_conn = 0, n_syn = 0;
    void begin(uint32_t, uint32_t, uint32_t n_connections, uint64_t n_synapses, uint32_t) override {
        base = (uint32_t)hn->seg.size();
        hn->num_connections += n_connections;
        n_conn = n_connections;
        n_syn = n_synapses;
    }
    void neuron(const BncNeuron&) override {}
    void segment(const BncSegment& s) override {
        BncSegment t = s;
        t.id += base;
        hostnet_add_segment(*hn, t);
    }
    void connection(const BncIntraConnection& c) override {
        BncIntraConnection t = c;
        t.segment_a += base;
        t.segment_b += base;
        hn->conn.push_back(t);
    }
    void synapse(const BncSynapse& y) override {
        BncSynapse t = y;
        t.pre_segment += base;
        t.post_segment += base;
        hostnet_add_synapse(*hn, t);
    }
    void stimulus(const BncCurrentStimulus& st) override {
        BncCurrentStimulus t = st;
        t.segment_id += base;
        stim->push_back(t);
    }
};

// Whether a member has intra-connections and synapses: network-wide switches of the
// reference tick (step 2.5 runs only with connections, diffusion_kernel.h:118; step 3
// resets neurotransmitter only with synapses, simulation_host.cpp:328).
struct MemberSwitches { bool conn, syn; };

// Records the member that was just appended (its ranges start at the given offsets)
// and checks that it agrees with member 0 on the switches.
static int add_member(std::vector<BncEnsembleMember>& members, std::vector<MemberSwitches>& sw, const HostNet& hn,
                      size_t n_stim_total, uint32_t seg_begin, uint32_t syn_begin, uint32_t stim_begin,
                      uint64_t n_valid_conn) {
    BncEnsembleMember m;
    m.seg_begin = seg_begin;
    m.n_segments = (uint32_t)hn.seg.size() - seg_begin;
    m.syn_begin = syn_begin;
    m.n_synapses = (uint32_t)hn.syn.size() - syn_begin;
    m.stim_begin = stim_begin;
    m.n_stimuli = (uint32_t)(n_stim_total - stim_begin);
    if (m.n_segments == 0) { set_error("ensemble member %zu has no segments", members.size()); return BNC_ERR_ARG; }
    MemberSwitches w{n_valid_conn > 0, m.n_synapses > 0};
    if (!sw.empty() && (w.conn != sw[0].conn || w.syn != sw[0].syn)) {
        set_error("ensemble member %zu %s intra-connections and %s synapses, member 0 %s and %s: members must "
                  "agree on both", members.size(), w.conn ? "has" : "has no", w.syn ? "has" : "has no",
                  sw[0].conn ? "has" : "has not", sw[0].syn ? "has" : "has not");
        return BNC_ERR_UNSUPPORTED;
    }
    members.push_back(m);
    sw.push_back(w);
    return BNC_OK;
}

// Streams generated members into one HostNet.
static int gather_generated(const BncNetgenParams* params, uint32_t n, HostNet* hn, std::vector<BncCurrentStimulus>* stim,
                            std::vector<BncEnsembleMember>* members) {
    if (!params || n == 0) { set_error("ensemble: no members"); return BNC_ERR_ARG; }
    std::vector<MemberSwitches> sw;
    EnsembleSink sink;
    sink.hn = hn;
    sink.stim = stim;
    for (uint32_t m = 0; m < n; m++) {
        const uint32_t seg0 = (uint32_t)hn->seg.size(), syn0 = (uint32_t)hn->syn.size(), st0 = (uint32_t)stim->size();
        NetShape shape;
        int rc = generate_network(params[m], sink, &shape);
        if (rc != BNC_OK) { set_error("ensemble member %u: invalid generator parameters", m); return rc; }
        if ((uint64_t)hn->seg.size() >= (1ull << 31)) { set_error("ensemble too large"); return BNC_ERR_ARG; }
        rc = add_member(*members, sw, *hn, stim->size(), seg0, syn0, st0, sink.n_conn);
        if (rc != BNC_OK) return rc;
    }
    hn->num_segments = (uint32_t)hn->seg.size();
    hn->num_synapses = (uint32_t)hn->syn.size();
    return BNC_OK;
}

}  // namespace

// Nucleus records (types.h:508-524, 500 bytes with 57 genes): protein_level at 244; the
// 46-gene records of older v7-v14 files (412 bytes) hold it at 200
// (bion_format.h:492-535).  Gene indices of the protein -> parameter mapping
// (types.h:357-361).
constexpr size_t kNucleusBytes = 500, kNucleus46Bytes = 412;
constexpr size_t kProteinOff = 244, kProtein46Off = 200, kGeneActOff = 16, kTail46Off = 384, kTailOff = 472;
constexpr int kGeneSYT1 = 40, kGeneUNC13A = 42, kGeneCPLX1 = 44;

static int sync_stream(Backend* b);

// ---- Drop-in records in managed memory ----
// The reference's backend keeps the Segment and Synapse records in managed memory and
// its kernels update them in place (bion_loader.cpp:634, gpu_backend_cuda.cu:250-308):
// after a tick the records are coherent, and a host read migrates only the pages it
// touches.  The same here: the records of a network loaded for the drop-in calls move
// to managed memory, and after each tick these kernels write the changing words of
// the device state into them (the words export_network writes on the host path).
// Records are packed structs; every word written sits at its natural alignment
// (BncSegment V_m at 40, ions at 48 and 112, modifier states at 296 + 88 j + 16, ...).
namespace {
template <typename T>
__device__ __forceinline__ void put(unsigned char* rec, size_t off, T v) { *reinterpret_cast<T*>(rec + off) = v; }

constexpr size_t kSegBytes = sizeof(BncSegment), kSynBytes = sizeof(BncSynapse), kModBytes = sizeof(BncModifier);
constexpr size_t kOffMods = offsetof(BncSegment, modifiers), kOffModState = offsetof(BncModifier, state);
static_assert(offsetof(BncSegment, V_m) % 8 == 0 && offsetof(BncSegment, intra_ions) % 8 == 0 &&
              offsetof(BncSegment, extra_ions) % 8 == 0 && offsetof(BncSegment, I_buffer) % 8 == 0 &&
              kOffMods % 8 == 0 && kModBytes % 8 == 0 && kOffModState % 8 == 0 && kSegBytes % 8 == 0 &&
              offsetof(BncSynapse, post_receptors) % 8 == 0 && kSynBytes % 8 == 0 &&
              offsetof(BncSegment, neurotransmitter) % 4 == 0 && offsetof(BncSegment, intra_nt) % 4 == 0 &&
              offsetof(BncSegment, ATP_level) % 4 == 0 && offsetof(BncSegment, temperature) % 4 == 0 &&
              offsetof(BncSegment, transcription_signal) % 4 == 0 && offsetof(BncSynapse, bouton_Ca) % 4 == 0 &&
              offsetof(BncSynapse, cleft_neurotransmitter) % 4 == 0,
              "record words are naturally aligned");

__global__ void k_export_segments(NetDev d, const uint32_t* perm, unsigned char* seg, int x_int, int x_temp,
                                  int x_txn, int clear_ibuf) {
    const uint32_t n = d.n_seg;
    for (uint32_t dd = blockIdx.x * blockDim.x + threadIdx.x; dd < n; dd += gridDim.x * blockDim.x) {
        unsigned char* r = seg + (size_t)perm[dd] * kSegBytes;
        put<double>(r, offsetof(BncSegment, V_m), (double)d.V[dd]);
        for (int q = 0; q < 7; q++) {
            put<double>(r, offsetof(BncSegment, intra_ions) + 8 * q, (double)d.ion_in[(size_t)q * n + dd]);
            put<double>(r, offsetof(BncSegment, extra_ions) + 8 * q, (double)d.ion_out[(size_t)q * n + dd]);
        }
        for (int q = 0; q < 15; q++) put<float>(r, offsetof(BncSegment, neurotransmitter) + 4 * q, d.nt[(size_t)q * n + dd]);
        if (x_int)
            for (int q = 0; q < 15; q++) put<float>(r, offsetof(BncSegment, intra_nt) + 4 * q, d.intra_nt[(size_t)q * n + dd]);
        put<float>(r, offsetof(BncSegment, ATP_level), d.atp[dd]);
        if (x_temp) put<float>(r, offsetof(BncSegment, temperature), d.temp[dd]);
        if (x_txn) put<float>(r, offsetof(BncSegment, transcription_signal), d.txn[dd]);
        if (clear_ibuf) put<double>(r, offsetof(BncSegment, I_buffer), 0.0);   // step 4 clears it
    }
}

// One thread per modifier item: the state words its type updates, and (after a tick)
// state[7], the effective area the tick wrote (run_tick_common.h:234-238), computed
// from the record's geometry as the host export does.
__global__ void k_export_items(NetDev d, const uint32_t* item_seg, const uint16_t* item_sm, unsigned char* seg,
                               int set_area) {
    const uint32_t NI = d.n_items;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < NI; q += gridDim.x * blockDim.x) {
        unsigned char* r = seg + (size_t)item_seg[q] * kSegBytes;
        const uint32_t sm = item_sm[q];
        unsigned char* m = r + kOffMods + (size_t)(sm & 0xFFu) * kModBytes;
        const uint32_t wm = sm >> 8;
        for (int k = 0; k < 7; k++)
            if ((wm >> k) & 1u) put<double>(m, kOffModState + 8 * k, (double)d.it_st[(size_t)k * NI + q]);
        if (set_area) {
            const uint8_t st = r[offsetof(BncSegment, segment_type)];
            const float rad = *reinterpret_cast<const float*>(r + offsetof(BncSegment, radius));
            const float len = *reinterpret_cast<const float*>(r + offsetof(BncSegment, length));
            const float area = (st == 1 || st == 3 || st == 4) ? 4.0f * 3.14159265f * rad * rad
                                                                : 2.0f * 3.14159265f * rad * len;
            put<double>(m, kOffModState + 8 * 7, (double)area);
        }
    }
}

__global__ void k_export_synapses(NetDev d, const uint32_t* syn_orig, const uint8_t* syn_nt, unsigned char* syn,
                                  int after_tick) {
    const uint32_t K = d.n_syn;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < K; q += gridDim.x * blockDim.x) {
        if (d.sy_gj && d.sy_gj[q] != UINT32_MAX) continue;   // a gap junction's side: k_export_gaps
        unsigned char* y = syn + (size_t)syn_orig[q] * kSynBytes;
        put<float>(y, offsetof(BncSynapse, bouton_Ca), d.sy_bouton[q]);
        put<float>(y, offsetof(BncSynapse, spine_Ca), d.sy_spine[q]);
        put<float>(y, offsetof(BncSynapse, spine_camkii), d.sy_camkii[q]);
        put<float>(y, offsetof(BncSynapse, spine_calcineurin), d.sy_calcn[q]);
        put<float>(y, offsetof(BncSynapse, facilitation), d.sy_facil[q]);
        put<float>(y, offsetof(BncSynapse, weight), d.sy_weight[q]);
        put<float>(y, offsetof(BncSynapse, cleft_neurotransmitter) + 4 * (size_t)syn_nt[q], d.sy_cleft[q]);
        put<float>(y, offsetof(BncSynapse, RRP), d.sy_rrp[q]);
        if (d.sy_cleft_ecb) put<float>(y, offsetof(BncSynapse, cleft_neurotransmitter) + 4 * 9, d.sy_cleft_ecb[q]);
        y[offsetof(BncSynapse, refractory)] = d.sy_refr[q];
        if (after_tick) put<float>(y, offsetof(BncSynapse, depression), d.sy_facil[q] + 0.01f);
    }
}

__global__ void k_export_receptors(NetDev d, const uint32_t* rec_syn, const uint8_t* rec_slot, const uint32_t* syn_orig,
                                   unsigned char* syn, int after_tick) {
    const uint32_t NR = d.n_rec;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < NR; r += gridDim.x * blockDim.x) {
        unsigned char* y = syn + (size_t)syn_orig[rec_syn[r]] * kSynBytes;
        unsigned char* m = y + offsetof(BncSynapse, post_receptors) + (size_t)rec_slot[r] * kModBytes;
        for (int k = 0; k < 3; k++) put<double>(m, kOffModState + 8 * k, (double)d.rc_st[(size_t)k * NR + r]);
        if (after_tick)
            put<double>(m, kOffModState + 8 * 7, (double)*reinterpret_cast<const float*>(y + offsetof(BncSynapse, post_area)));
    }
}

// gap junctions: the slow gate in depression, the filtered current in cleft entry 0
__global__ void k_export_gaps(NetDev d, const uint32_t* gj_syn, unsigned char* syn) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < d.n_gj; g += gridDim.x * blockDim.x) {
        unsigned char* y = syn + (size_t)gj_syn[g] * kSynBytes;
        put<float>(y, offsetof(BncSynapse, depression), d.gj_dep[g]);
        put<float>(y, offsetof(BncSynapse, cleft_neurotransmitter), d.gj_flt[g]);
    }
}

__global__ void k_export_modulators(NetDev d, const uint32_t* md_syn, const uint8_t* md_slot, unsigned char* syn,
                                    int after_tick) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < d.n_md; q += gridDim.x * blockDim.x) {
        unsigned char* y = syn + (size_t)md_syn[q] * kSynBytes;
        unsigned char* m = y + offsetof(BncSynapse, pre_autoreceptors) + (size_t)md_slot[q] * kModBytes;
        put<double>(m, kOffModState, (double)d.md_st[q]);
        if (after_tick)
            put<double>(m, kOffModState + 8 * 7, (double)*reinterpret_cast<const float*>(y + offsetof(BncSynapse, pre_area)));
    }
}

template <typename T>
T* upload_map(Backend* b, const std::vector<T>& v, bool* ok) {
    if (!*ok || v.empty()) return nullptr;
    T* p = static_cast<T*>(b->allocs.alloc(v.size() * sizeof(T)));
    if (!p || cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) *ok = false;
    return p;
}
}  // namespace

// Moves the records of a loaded single network into managed memory and uploads the
// export maps.  Where the device cannot share managed memory with the host
// concurrently the records stay in host memory and export_network updates them.
static int make_records_managed(Backend* b) {
    if (!b->owns_aos || !b->members.empty() || b->aos_managed) return BNC_OK;
    int cma = 0;
    if (cudaDeviceGetAttribute(&cma, cudaDevAttrConcurrentManagedAccess, b->device) != cudaSuccess || !cma) {
        cudaGetLastError();
        return BNC_OK;
    }
    const size_t n = b->aos.num_segments, k = b->aos.num_synapses;
    void *ms = nullptr, *my = nullptr;
    if (cudaMallocManaged(&ms, (n ? n : 1) * kSegBytes) != cudaSuccess ||
        cudaMallocManaged(&my, (k ? k : 1) * kSynBytes) != cudaSuccess) {
        cudaGetLastError();
        if (ms) cudaFree(ms);
        return BNC_OK;   // host records, host export
    }
    auto& x = b->xm;
    if (!x.perm) {   // the export maps, once per network
        const NetHost& h = b->host;
        std::vector<uint16_t> sm(h.item_seg.size());
        for (size_t q = 0; q < sm.size(); q++) {
            const uint8_t t = b->aos.segments[h.item_seg[q]].modifiers[h.item_slot[q]].type;
            const bool user = t < 128 && ((b->dev.user_mask[t >> 5] >> (t & 31)) & 1u);
            sm[q] = (uint16_t)(h.item_slot[q] | ((user ? 0x7Fu : host_dyn_mask(t)) << 8));
        }
        bool ok = true;
        x.perm = upload_map(b, h.perm, &ok);
        x.item_seg = upload_map(b, h.item_seg, &ok);
        x.item_sm = upload_map(b, sm, &ok);
        x.syn_orig = upload_map(b, h.syn_orig, &ok);
        x.syn_nt = upload_map(b, h.syn_nt, &ok);
        x.rec_syn = upload_map(b, h.rec_syn, &ok);
        x.rec_slot = upload_map(b, h.rec_slot, &ok);
        x.md_syn = upload_map(b, h.md_syn, &ok);
        x.md_slot = upload_map(b, h.md_slot, &ok);
        x.gj_syn = upload_map(b, h.gj_syn, &ok);
        if (!ok) {
            cudaFree(ms);
            cudaFree(my);
            std::memset(&x, 0, sizeof(x));
            return cuda_fail(cudaGetLastError(), "upload of the record export maps");
        }
    }
    if (n) std::memcpy(ms, b->aos.segments, n * kSegBytes);
    if (k) std::memcpy(my, b->aos.synapses, k * kSynBytes);
    delete[] b->aos.segments;
    delete[] b->aos.synapses;
    b->aos.segments = static_cast<BncSegment*>(ms);
    b->aos.synapses = static_cast<BncSynapse*>(my);
    b->aos_managed = true;
    // the device writes the records every tick: start them resident there
    cudaMemPrefetchAsync(ms, (n ? n : 1) * kSegBytes, b->device, b->stream);
    cudaMemPrefetchAsync(my, (k ? k : 1) * kSynBytes, b->device, b->stream);
    cudaGetLastError();
    return BNC_OK;
}

// The records coherent with the device state: on the device into managed records,
// else by the host export.  The stream is synchronised on return.
static int export_records(Backend* b) {
    if (!b->aos_managed) {
        int rc = sync_stream(b);
        if (rc != BNC_OK) return rc;
        return export_network(b->dev, b->host, b->ticks_run, &b->aos);
    }
    const NetDev& d = b->dev;
    const int after = b->ticks_run > 0 ? 1 : 0;
    unsigned char* seg = reinterpret_cast<unsigned char*>(b->aos.segments);
    unsigned char* syn = reinterpret_cast<unsigned char*>(b->aos.synapses);
    auto grid = [](uint32_t m) { return (unsigned)std::min<uint32_t>((m + 255) / 256, 148u * 16u); };
    if (d.n_seg)
        k_export_segments<<<grid(d.n_seg), 256, 0, b->stream>>>(d, b->xm.perm, seg, (d.flags & NF_INTRA_NT) != 0,
                                                                (d.flags & NF_TEMP) != 0, (d.flags & NF_TXN) != 0, after);
    if (d.n_items) k_export_items<<<grid(d.n_items), 256, 0, b->stream>>>(d, b->xm.item_seg, b->xm.item_sm, seg, after);
    if (d.n_syn) k_export_synapses<<<grid(d.n_syn), 256, 0, b->stream>>>(d, b->xm.syn_orig, b->xm.syn_nt, syn, after);
    if (d.n_rec)
        k_export_receptors<<<grid(d.n_rec), 256, 0, b->stream>>>(d, b->xm.rec_syn, b->xm.rec_slot, b->xm.syn_orig, syn,
                                                                 after);
    if (d.n_md) k_export_modulators<<<grid(d.n_md), 256, 0, b->stream>>>(d, b->xm.md_syn, b->xm.md_slot, syn, after);
    if (d.n_gj) k_export_gaps<<<grid(d.n_gj), 256, 0, b->stream>>>(d, b->xm.gj_syn, syn);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { b->failed = true; return cuda_fail(e, "record export launch"); }
    return sync_stream(b);
}

// The reference's GPU backend maps the nucleus protein levels of each synapse's
// presynaptic neuron onto its release parameters before every synaptic step
// (gpu_backend_cuda.cu:275-289, rrp_apply_protein_mapping, kernel_dispatch.h:651-663):
// synapses with id 0 are skipped, the nucleus is the one at the position of the
// presynaptic segment's neuron_id.  Nothing on that path changes protein levels, so the
// mapping gives the same values every tick: it is applied once, to the records, when a
// network with nuclei is loaded.
static void apply_protein_mapping(BncBionData& d) {
    if (!d.nuclei || d.num_nuclei == 0) return;
    const uint8_t* nu = static_cast<const uint8_t*>(d.nuclei);
    for (uint32_t i = 0; i < d.num_synapses; i++) {
        BncSynapse& y = d.synapses[i];
        if (y.id == 0) continue;
        if (y.pre_segment >= d.num_segments) continue;
        const uint32_t nid = d.segments[y.pre_segment].neuron_id;
        if (nid >= d.num_nuclei) continue;
        const float* pl = reinterpret_cast<const float*>(nu + (size_t)nid * kNucleusBytes + kProteinOff);
        const float munc13 = pl[kGeneUNC13A];
        y.RRP_max = 10.0f + munc13 * 40.0f;
        const float syt1 = pl[kGeneSYT1];
        y.release_probability = 0.3f + syt1 * 0.7f;
        const float cplx1 = pl[kGeneCPLX1];
        y.RRP_recovery = 0.02f + munc13 * 0.08f - cplx1 * 0.01f;
        if (y.RRP_recovery < 0.005f) y.RRP_recovery = 0.005f;
        if (y.RRP_recovery > 0.2f) y.RRP_recovery = 0.2f;
    }
}

static int load_common(Backend* b, BncBionData& aos, bool keep_aos) {
    cudaSetDevice(b->device);
    apply_protein_mapping(aos);
    HostNet hn;
    hostnet_from_aos(aos, &hn);
    int rc = build_network(hn, b->stim, &b->dev, &b->host, &b->allocs);
    if (rc != BNC_OK) { b->reset_network(); return rc; }
    if (keep_aos) { b->aos = aos; b->owns_aos = true; }
    b->loaded = true;
    if (keep_aos) return make_records_managed(b);
    return BNC_OK;
}

static void free_aos_arrays(BncBionData& a) { bion_free(a); }

static int copy_aos(const BncBionData* src, BncBionData* dst) {
    std::memset(dst, 0, sizeof(*dst));
    dst->header = src->header;
    dst->num_neurons = src->num_neurons; dst->num_segments = src->num_segments;
    dst->num_connections = src->num_connections; dst->num_synapses = src->num_synapses;
    dst->neurons = new (std::nothrow) BncNeuron[src->num_neurons ? src->num_neurons : 1];
    dst->segments = new (std::nothrow) BncSegment[src->num_segments ? src->num_segments : 1];
    dst->connections = new (std::nothrow) BncIntraConnection[src->num_connections ? src->num_connections : 1];
    dst->synapses = new (std::nothrow) BncSynapse[src->num_synapses ? src->num_synapses : 1];
    if (!dst->neurons || !dst->segments || !dst->connections || !dst->synapses) { free_aos_arrays(*dst); return BNC_ERR_ALLOC; }
    if (src->num_neurons && src->neurons) std::memcpy(dst->neurons, src->neurons, sizeof(BncNeuron) * src->num_neurons);
    if (src->num_segments) std::memcpy(dst->segments, src->segments, sizeof(BncSegment) * src->num_segments);
    if (src->num_connections) std::memcpy(dst->connections, src->connections, sizeof(BncIntraConnection) * src->num_connections);
    if (src->num_synapses) std::memcpy(dst->synapses, src->synapses, sizeof(BncSynapse) * src->num_synapses);
    dst->nuclei = nullptr;
    dst->num_nuclei = 0;
    if (src->num_nuclei && src->nuclei) {
        uint8_t* nu = new (std::nothrow) uint8_t[(size_t)src->num_nuclei * kNucleusBytes];
        if (!nu) { free_aos_arrays(*dst); return BNC_ERR_ALLOC; }
        std::memcpy(nu, src->nuclei, (size_t)src->num_nuclei * kNucleusBytes);
        dst->nuclei = nu;
        dst->num_nuclei = src->num_nuclei;
    }
    return BNC_OK;
}

// Pending injections are consumed by the first tick enqueued after their upload (the
// kernel zeroes the device count); later ticks need not launch k_inject.
static void injections_enqueued(Backend* b) {
    b->dev.inj = nullptr;
    b->dev.inj_n = nullptr;
    b->pend_ion.clear();
    b->pend_lig.clear();
}

// Counter bookkeeping after one tick is enqueued; every tick entry point uses it.
static void tick_enqueued(Backend* b) {
    b->tick += b->tick_stride;
    b->ticks_run++;
    injections_enqueued(b);
}

static int run_ticks(Backend* b, uint32_t n, float dt) {
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    if (b->failed) { set_error("backend is in a failed state after a device error"); return BNC_ERR_STATE; }
    cudaSetDevice(b->device);
    for (uint32_t t = 0; t < n; t++) {
        cudaError_t e = launch_tick(b->dev, b->host, dt, b->tick, b->ticks_run == 0 ? 1 : 0, b->stream);
        if (e != cudaSuccess) { b->failed = true; return cuda_fail(e, "tick launch"); }
        tick_enqueued(b);
    }
    return BNC_OK;
}

// The captured tick loop: one graph whose conditional WHILE node runs its body -- one
// tick, the device clock advance, and a countdown -- until the countdown reaches zero,
// so one graph launch runs all ticks of a call.  The countdown is set before each
// launch; it is capped at kLoopMax iterations, and any count outside 1..kLoopMax ends
// the loop, so the loop always ends.
constexpr uint32_t kGraphTicks = 32;           // minimum trial length of the tuner
constexpr unsigned long long kLoopMax = 1ull << 24;

namespace {
__global__ void k_loop_countdown(cudaGraphConditionalHandle h, unsigned long long* count) {
    const unsigned long long c = *count;
    if (c <= 1 || c > kLoopMax) {
        *count = 0;
        cudaGraphSetConditional(h, 0);
    } else {
        *count = c - 1;
    }
}
__global__ void k_loop_set(unsigned long long* count, unsigned long long n) { *count = n; }
}  // namespace

static int capture_graph(Backend* b, float dt) {
    b->drop_graph();
    if (!b->clock) {
        // clock[0] tick counter, clock[1] ticks run, clock[2] the loop's countdown
        b->clock = static_cast<unsigned long long*>(b->allocs.alloc(3 * sizeof(unsigned long long)));
        if (!b->clock) { set_error("device allocation of the tick clock failed"); return BNC_ERR_ALLOC; }
    }
    cudaError_t e = prepare_tick(b->dev, b->host, b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "tick set-up");
    NetDev d = b->dev;
    d.clock = b->clock;
    cudaGraph_t g = nullptr;
    e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphCreate");
    cudaGraphConditionalHandle h;
    e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNode_t node = nullptr;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(e, "conditional graph node"); }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(b->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(e, "capture of the loop body"); }
    cudaError_t le = enqueue_tick(d, b->host, dt, 0, 0, b->stream);
    if (le == cudaSuccess) le = launch_advance_clock(b->clock, b->stream);
    if (le == cudaSuccess) {
        k_loop_countdown<<<1, 1, 0, b->stream>>>(h, b->clock + 2);
        le = cudaGetLastError();
    }
    cudaGraph_t cap = nullptr;
    e = cudaStreamEndCapture(b->stream, &cap);
    if (le != cudaSuccess || e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(le != cudaSuccess ? le : e, "tick loop capture");
    }
    e = cudaGraphInstantiate(&b->graph_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->graph_exec = nullptr; return cuda_fail(e, "cudaGraphInstantiate"); }
    b->graph_dt = dt;
    return BNC_OK;
}

static int run_ticks_graph(Backend* b, uint32_t n, float dt) {
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    if (b->failed) { set_error("backend is in a failed state after a device error"); return BNC_ERR_STATE; }
    if (b->tick_stride != 1) return run_ticks(b, n, dt);   // the captured clock steps by one
    if (b->dev.inj && n > 0) {   // the tick that applies pending injections runs uncaptured
        int rc = run_ticks(b, 1, dt);
        if (rc != BNC_OK) return rc;
        n--;
    }
    if (n == 0) return BNC_OK;
    if ((unsigned long long)n > kLoopMax) {
        int rc = run_ticks_graph(b, (uint32_t)kLoopMax, dt);
        return rc != BNC_OK ? rc : run_ticks_graph(b, n - (uint32_t)kLoopMax, dt);
    }
    cudaSetDevice(b->device);
    if (!b->graph_exec || b->graph_dt != dt) {
        int rc = capture_graph(b, dt);
        if (rc != BNC_OK) return rc;
    }
    cudaError_t e = launch_set_clock(b->clock, b->tick, b->ticks_run, b->stream);
    if (e == cudaSuccess) {
        k_loop_set<<<1, 1, 0, b->stream>>>(b->clock + 2, (unsigned long long)n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaGraphLaunch(b->graph_exec, b->stream);
    if (e != cudaSuccess) { b->failed = true; return cuda_fail(e, "graph launch"); }
    b->tick += n;
    b->ticks_run += n;
    return BNC_OK;
}

static int sync_stream(Backend* b) {
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) { b->failed = true; return cuda_fail(e, "tick execution"); }
    return BNC_OK;
}

// .bion files: bion_file.cpp (every version the reference reads; the v14 writer).
static int save_bion(const BncBionData& d, const char* path) { return bion_write(d, path); }
static int load_bion_file(const char* path, BncBionData* d, bool default_nuclei = true) {
    return bion_read(path, d, default_nuclei);
}

int backend_export_host(void* sim, HostNet* hn, std::vector<BncCurrentStimulus>* stim, uint64_t* tick,
                        int* device, uint32_t* n_vclamp) {
    if (!sim) { set_error("null handle"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    if (!b->owns_aos || !b->aos.segments) {
        set_error("the network must be loaded from AoS arrays (bnc_load_aos)");
        return BNC_ERR_UNSUPPORTED;
    }
    if (!b->members.empty()) { set_error("an ensemble backend holds several networks"); return BNC_ERR_UNSUPPORTED; }
    cudaSetDevice(b->device);
    int rc = export_records(b);
    if (rc != BNC_OK) return rc;
    hostnet_from_aos(b->aos, hn);
    *stim = b->stim.current;
    *tick = b->tick;
    *device = b->device;
    *n_vclamp = (uint32_t)b->stim.vclamp.size();
    return BNC_OK;
}

int backend_set_tick_stride(void* sim, uint32_t stride) {
    if (!sim || stride == 0) { set_error("null handle or zero stride"); return BNC_ERR_ARG; }
    static_cast<Backend*>(sim)->tick_stride = stride;
    return BNC_OK;
}

int backend_record_releases(void* sim, uint32_t ticks, float dt, std::vector<uint32_t>* syn,
                            std::vector<uint64_t>* tick, std::vector<float>* amt, std::vector<uint8_t>* slot) {
    if (!sim) { set_error("null handle"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    cudaSetDevice(b->device);
    syn->clear(); tick->clear(); amt->clear(); slot->clear();
    const uint64_t t_begin = b->tick;
    // Cleft entries per synapse: one immediate release per refractory period (the
    // reference's uint8 refractory count, simulation_host.cpp:458) plus one delayed
    // arrival per release.
    uint32_t refr = (uint32_t)(uint8_t)(uint32_t)(20.0f / dt + 0.5f);
    if (refr == 0) refr = 1;
    const uint64_t per_syn = 2ull * ((uint64_t)ticks / refr + 1u);
    const uint64_t cap64 = (uint64_t)b->dev.n_syn * per_syn + 16u;
    if (cap64 > 0x7FFFFFFFull) { set_error("release log of %llu entries is too large", (unsigned long long)cap64); return BNC_ERR_ARG; }
    {
        const uint32_t cap = (uint32_t)cap64;
        uint4* buf = nullptr;
        uint32_t* n = nullptr;
        if (cudaMalloc(&buf, (size_t)cap * sizeof(uint4)) != cudaSuccess ||
            cudaMalloc(&n, sizeof(uint32_t)) != cudaSuccess) {
            cudaFree(buf);
            set_error("device allocation of the release log (%u entries) failed", cap);
            return BNC_ERR_ALLOC;
        }
        cudaMemsetAsync(n, 0, sizeof(uint32_t), b->stream);
        b->drop_graph();   // a captured tick holds the descriptor without the log
        b->dev.ev_buf = buf; b->dev.ev_n = n; b->dev.ev_cap = cap;
        int rc = run_ticks(b, ticks, dt);
        b->dev.ev_buf = nullptr; b->dev.ev_n = nullptr; b->dev.ev_cap = 0;
        if (rc == BNC_OK) rc = sync_stream(b);
        uint32_t count = 0;
        if (rc == BNC_OK && cudaMemcpy(&count, n, sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "release log read");
        if (rc == BNC_OK && count > cap) {
            rc = BNC_ERR_STATE;
            set_error("release log overflow (%u entries, room for %u)", count, cap);
        }
        std::vector<uint4> h(rc == BNC_OK ? count : 0);
        if (rc == BNC_OK && count &&
            cudaMemcpy(h.data(), buf, (size_t)count * sizeof(uint4), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "release log read");
        cudaFree(buf); cudaFree(n);
        if (rc != BNC_OK) return rc;
        syn->reserve(count); tick->reserve(count); amt->reserve(count); slot->reserve(count);
        for (const uint4& e : h) {
            // the low 32 bits of the tick, widened against the run's first tick
            uint64_t t = (t_begin & ~0xFFFFFFFFull) | e.y;
            if (t < t_begin) t += 0x100000000ull;
            syn->push_back(b->host.syn_orig[e.x]);
            tick->push_back(t);
            float a;
            std::memcpy(&a, &e.z, sizeof(a));
            amt->push_back(a);
            slot->push_back((uint8_t)e.w);
        }
        return BNC_OK;
    }
}

}  // namespace bnc

using namespace bnc;

extern "C" {

void* gpu_backend_create_on_device(int device_index) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("no CUDA device"); return nullptr; }
    if (device_index < 0 || device_index >= ndev) device_index = 0;
    Backend* b = new (std::nothrow) Backend();
    if (!b) return nullptr;
    b->device = device_index;
    if (cudaSetDevice(device_index) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
        set_error("CUDA context creation failed");
        delete b;
        return nullptr;
    }
    return b;
}

void* gpu_backend_create(void) { return gpu_backend_create_on_device(0); }

void gpu_backend_destroy(void* sim) { delete static_cast<Backend*>(sim); }

int gpu_backend_load_bion(void* sim, const char* filename) {
    if (!sim || !filename) return -1;
    Backend* b = static_cast<Backend*>(sim);
    b->reset_network();
    BncBionData d;
    int rc = load_bion_file(filename, &d);
    if (rc != BNC_OK) return rc;
    rc = load_common(b, d, true);
    if (rc != BNC_OK) free_aos_arrays(d);
    return rc;
}

void gpu_backend_run_tick(void* sim, float dt) {
    if (!sim) return;
    Backend* b = static_cast<Backend*>(sim);
    if (run_ticks(b, 1, dt) != BNC_OK) return;
    export_records(b);
}

void* gpu_backend_bion_data(void* sim) {
    if (!sim) return nullptr;
    Backend* b = static_cast<Backend*>(sim);
    return b->owns_aos ? &b->aos : nullptr;
}

void gpu_backend_upload_stimuli(void* sim, const BncGpuStimulusData* src) {
    if (!sim || !src) return;
    Backend* b = static_cast<Backend*>(sim);
    set_error("%s", "");   // the call returns nothing: an empty error string means success
    if (!b->loaded) { set_error("no network loaded"); return; }
    auto take = [](auto& dst, const auto* arr, uint32_t cnt) {
        dst.assign(arr, arr + std::min<uint32_t>(cnt, BNC_GPU_MAX_STIMULI));
    };
    take(b->stim.current, src->current_stim, src->current_stim_count);
    take(b->stim.vclamp, src->vclamps, src->vclamp_count);
    take(b->stim.ramp, src->ramps, src->ramp_count);
    take(b->stim.ion_inj, src->ion_inj, src->ion_inj_count);
    take(b->stim.lig_inj, src->lig_inj, src->lig_inj_count);
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    b->drop_graph();   // a captured tick holds the stimulus arrays freed below
    b->stim_allocs.release();
    if (upload_stimuli(b->stim, b->host, &b->dev, &b->stim_allocs) != BNC_OK)
        set_error("device allocation of the stimulus arrays failed");
    // injections are one-shot: a later rebuild from these lists must not repeat them;
    // the pending copies last until a tick applies them
    b->pend_ion.swap(b->stim.ion_inj);
    b->pend_lig.swap(b->stim.lig_inj);
    b->stim.ion_inj.clear();
    b->stim.lig_inj.clear();
}

int bnc_upload_mechano(void* sim, const BncMechanoStimulus* ms, uint32_t n) {
    if (!sim || (n && !ms)) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    if (!b->members.empty()) { set_error("mechano stimuli address one network, not an ensemble"); return BNC_ERR_UNSUPPORTED; }
    if (!b->owns_aos || !b->aos.segments) {
        set_error("mechano stimuli need the network's records (load it from AoS arrays or a .bion)");
        return BNC_ERR_UNSUPPORTED;
    }
    if (!n) return BNC_OK;
    cudaSetDevice(b->device);
    int rc = sync_stream(b);
    if (rc != BNC_OK) return rc;
    // each stimulus -> (record, slot), as simulation_host.cpp:213-228 searches them
    struct Hit { uint32_t seg; uint8_t slot; int idx; float value; uint32_t item; };
    std::vector<Hit> hits;
    BncBionData& a = b->aos;
    for (uint32_t m = 0; m < n; m++) {
        BncMechanoStimulus st;
        std::memcpy(&st, reinterpret_cast<const unsigned char*>(ms) + (size_t)m * sizeof(BncMechanoStimulus), sizeof(st));
        for (uint32_t i = 0; i < a.num_segments; i++) {
            if (a.segments[i].id != st.segment_id) continue;
            const uint8_t mc = a.segments[i].modifier_count;
            for (uint8_t j = 0; j < mc && j < BNC_MAX_MODIFIERS; j++)
                if (a.segments[i].modifiers[j].type == st.mod_type) {
                    if (st.state_idx >= 0 && st.state_idx < BNC_MAX_STATE) hits.push_back({i, j, st.state_idx, st.value, UINT32_MAX});
                    break;
                }
            break;
        }
    }
    if (hits.empty()) return BNC_OK;
    // the items of those slots (a slot myelin blocks has none: only its record changes)
    const NetHost& h = b->host;
    parallel_for(h.item_seg.size(), [&](size_t q0, size_t q1) {
        for (size_t q = q0; q < q1; q++)
            for (Hit& x : hits)
                if (h.item_seg[q] == x.seg && h.item_slot[q] == x.slot) x.item = (uint32_t)q;
    });
    const NetDev& d = b->dev;
    for (const Hit& x : hits) {
        a.segments[x.seg].modifiers[x.slot].state[x.idx] = (double)x.value;
        if (x.item == UINT32_MAX || x.idx >= 7) continue;
        cudaError_t e = cudaMemcpy(d.it_st + (size_t)x.idx * d.n_items + x.item, &x.value, 4, cudaMemcpyHostToDevice);
        const uint8_t type = a.segments[x.seg].modifiers[x.slot].type;
        if (e == cudaSuccess && x.value != 0.0f && ((param_mask(type) >> x.idx) & 1u)) {
            // a parameter word now set: the item reads its parameters
            uint16_t tf = 0;
            e = cudaMemcpy(&tf, d.it_tf + x.item, 2, cudaMemcpyDeviceToHost);
            tf = (uint16_t)(tf | (1u << 8));
            if (e == cudaSuccess) e = cudaMemcpy(d.it_tf + x.item, &tf, 2, cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) return cuda_fail(e, "mechano stimulus write");
    }
    return BNC_OK;
}

int gpu_backend_device_count(void) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) return 0;
    return ndev;
}

int gpu_backend_get_device_info(int index, BncGpuDeviceInfo* info) {
    if (!info) return -1;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) return -1;
    if (index < 0 || index >= ndev) return -1;
    std::memset(info, 0, sizeof(*info));
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, index) != cudaSuccess) return -1;
    std::strncpy(info->name, prop.name, 127);
    info->vendor_id = 0x10DE;
    info->is_cpu = 0;
    info->global_mem_bytes = prop.totalGlobalMem;
    info->max_compute_units = prop.multiProcessorCount;
    info->device_index = index;
    std::strncpy(info->backend_type, "cuda", 15);
    return 0;
}

int gpu_backend_ibuf_offset(void) { return (int)offsetof(BncSegment, I_buffer); }
int gpu_backend_vm_offset(void) { return (int)offsetof(BncSegment, V_m); }
int gpu_backend_seg_size(void) { return (int)sizeof(BncSegment); }

int bnc_load_aos(void* sim, const BncBionData* data, const BncCurrentStimulus* stim, uint32_t n_stim) {
    if (!sim || !data) { set_error("bnc_load_aos: null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    b->reset_network();
    if (stim && n_stim) b->stim.current.assign(stim, stim + n_stim);
    BncBionData d;
    int rc = copy_aos(data, &d);
    if (rc != BNC_OK) { set_error("bnc_load_aos: out of host memory"); return rc; }
    rc = load_common(b, d, true);
    if (rc != BNC_OK) free_aos_arrays(d);
    return rc;
}

static BuildOptions to_options(const BncBuildOptions* o) {
    BuildOptions opt;
    if (o) {
        if (o->warp_cap) opt.warp_cap = o->warp_cap;
        if (o->tile_segs) opt.tile_segs = o->tile_segs;
        opt.phase_cap = o->phase_cap;
        if (o->chunk_segs) opt.chunk_segs = o->chunk_segs;
        if (o->fuse_phases) {
            opt.fuse_phases = o->fuse_phases;
            opt.fuse_adaptive = false;
        }
        opt.group_barriers = o->cta_barriers == 0;
    }
    return opt;
}

int bnc_load_generated_opts(void* sim, const BncNetgenParams* p, const BncBuildOptions* o) {
    if (!sim || !p) { set_error("bnc_load_generated: null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    b->reset_network();
    HostNet hn;
    HostNetSink sink;
    sink.hn = &hn;
    sink.stim = &b->stim.current;
    NetShape shape;
    int rc = generate_network(*p, sink, &shape);
    if (rc != BNC_OK) { set_error("bnc_load_generated: invalid parameters"); return rc; }
    cudaSetDevice(b->device);
    rc = build_network(hn, b->stim, &b->dev, &b->host, &b->allocs, to_options(o));
    if (rc != BNC_OK) { b->reset_network(); return rc; }
    b->loaded = true;
    return BNC_OK;
}

int bnc_load_generated(void* sim, const BncNetgenParams* p) { return bnc_load_generated_opts(sim, p, nullptr); }

static int plan_info(const HostNet& hn, const Stimuli& stim, BncNetInfo* info,
                     const BuildOptions& opt = BuildOptions()) {
    NetDev dev;
    NetHost host;
    int rc = build_network(hn, stim, &dev, &host, nullptr, opt);
    if (rc != BNC_OK) return rc;
    std::memset(info, 0, sizeof(*info));
    info->n_segments = dev.n_seg; info->n_connections = host.n_conn; info->n_synapses = dev.n_syn;
    info->n_tiles = dev.n_tiles; info->n_items = dev.n_items; info->n_phases = dev.n_phases;
    info->n_receptors = dev.n_rec; info->max_tile_segs = host.max_tile_segs;
    info->max_tile_edges = host.max_tile_edges; info->smem_bytes = (uint32_t)host.smem_bytes;
    info->flags = dev.flags; info->algo_bytes_per_tick = host.algo_bytes_per_tick;
    info->seg_bytes_per_tick = host.seg_bytes; info->syn_bytes_per_tick = host.syn_bytes;
    info->tile_bytes_per_tick = host.tile_bytes; info->synapse_kernel_bytes_per_tick = host.synk_bytes;
    info->warp_cap = host.opt.warp_cap; info->tile_segs = host.opt.tile_segs;
    info->modifier_kernel_bytes = host.mod_bytes; info->diffusion_kernel_bytes = host.diff_bytes;
    info->modifier_launches = modifier_launches(dev, host); info->fuse_phases = host.fuse;
    info->group_tiles_32 = host.group_tiles_32; info->group_tiles_64 = host.group_tiles_64;
    info->diffusion_threads = host.diff_threads;
    info->synapse_launches = synapse_launches(dev);
    return BNC_OK;
}

int bnc_plan_generated(const BncNetgenParams* p, BncNetInfo* info) { return bnc_plan_generated_opts(p, nullptr, info); }

int bnc_plan_generated_opts(const BncNetgenParams* p, const BncBuildOptions* o, BncNetInfo* info) {
    if (!p || !info) { set_error("bnc_plan_generated: null argument"); return BNC_ERR_ARG; }
    HostNet hn;
    Stimuli stim;
    HostNetSink sink;
    sink.hn = &hn;
    sink.stim = &stim.current;
    NetShape shape;
    int rc = generate_network(*p, sink, &shape);
    if (rc != BNC_OK) { set_error("bnc_plan_generated: invalid parameters"); return rc; }
    return plan_info(hn, stim, info, to_options(o));
}

static int load_members(Backend* b, const BncNetgenParams* members, uint32_t n_members, const BuildOptions& opt) {
    b->reset_network();
    HostNet hn;
    std::vector<BncEnsembleMember> mem;
    int rc = gather_generated(members, n_members, &hn, &b->stim.current, &mem);
    if (rc != BNC_OK) { b->reset_network(); return rc; }
    cudaSetDevice(b->device);
    rc = build_network(hn, b->stim, &b->dev, &b->host, &b->allocs, opt);
    if (rc != BNC_OK) { b->reset_network(); return rc; }
    b->members = std::move(mem);
    b->loaded = true;
    return BNC_OK;
}

int bnc_load_ensemble_generated(void* sim, const BncNetgenParams* members, uint32_t n_members) {
    if (!sim) { set_error("null handle"); return BNC_ERR_ARG; }
    return load_members(static_cast<Backend*>(sim), members, n_members, BuildOptions());
}

static int time_graph(Backend* b, uint32_t n, float dt, float* ms) {
    cudaEventRecord(b->ev0, b->stream);
    int rc = run_ticks_graph(b, n, dt);
    if (rc != BNC_OK) return rc;
    cudaEventRecord(b->ev1, b->stream);
    rc = sync_stream(b);
    if (rc != BNC_OK) return rc;
    cudaEventElapsedTime(ms, b->ev0, b->ev1);
    return BNC_OK;
}

// Groupings the autotuner tries: (segments per warp group, segments per tile).
static const BuildOptions kTuneCandidates[] = {
    {32, 256}, {64, 256}, {64, 512}, {128, 512}, {64, 1024}, {128, 1024}, {256, 1024},
};

int bnc_load_ensemble_tuned(void* sim, const BncNetgenParams* members, uint32_t n_members, uint32_t trial_ticks,
                            float dt, BncTuning* out) {
    if (!sim || !members || n_members == 0) { set_error("bnc_load_ensemble_tuned: null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    // Tune on an evenly strided sample of at most 64 members (every member's own
    // sizes, so the sample keeps the ensemble's size mix), then build everything.
    const uint32_t stride = n_members > 64 ? (n_members + 63) / 64 : 1;
    std::vector<BncNetgenParams> sample;
    for (uint32_t m = 0; m < n_members; m += stride) sample.push_back(members[m]);
    if (trial_ticks < kGraphTicks) trial_ticks = kGraphTicks;
    BncTuning best{};
    best.ms_per_tick = -1.0f;
    uint32_t tried = 0;
    for (const BuildOptions& opt : kTuneCandidates) {
        int rc = load_members(b, sample.data(), (uint32_t)sample.size(), opt);
        if (rc == BNC_ERR_UNSUPPORTED) continue;   // a component larger than this tile
        if (rc != BNC_OK) return rc;
        float ms = 0.0f;
        rc = run_ticks_graph(b, 1, dt);                     // first tick and set-up, untimed
        if (rc == BNC_OK) rc = time_graph(b, trial_ticks, dt, &ms);
        if (rc != BNC_OK) { b->reset_network(); return rc; }
        tried++;
        const float per_tick = ms / (float)trial_ticks;
        if (best.ms_per_tick < 0.0f || per_tick < best.ms_per_tick) {
            best.warp_cap = opt.warp_cap;
            best.tile_segs = opt.tile_segs;
            best.ms_per_tick = per_tick;
        }
    }
    b->reset_network();
    if (tried == 0) { set_error("no grouping fits the ensemble's largest component"); return BNC_ERR_UNSUPPORTED; }
    best.candidates_tried = tried;
    best.sample_members = (uint32_t)sample.size();
    BuildOptions opt;
    opt.warp_cap = best.warp_cap;
    opt.tile_segs = best.tile_segs;
    int rc = load_members(b, members, n_members, opt);
    if (rc == BNC_OK && out) *out = best;
    return rc;
}

int bnc_time_ticks_graph(void* sim, uint32_t n_ticks, float dt, float* ms) {
    if (!sim || !ms) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    cudaSetDevice(b->device);
    return time_graph(b, n_ticks, dt, ms);
}

int bnc_load_ensemble_aos(void* sim, const BncBionData* members, const BncCurrentStimulus* const* stim,
                          const uint32_t* n_stim, uint32_t n_members) {
    if (!sim || !members || n_members == 0) { set_error("bnc_load_ensemble_aos: null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    b->reset_network();
    HostNet hn;
    std::vector<BncEnsembleMember> mem;
    std::vector<MemberSwitches> sw;
    EnsembleSink sink;
    sink.hn = &hn;
    sink.stim = &b->stim.current;
    for (uint32_t m = 0; m < n_members; m++) {
        const BncBionData& d = members[m];
        if (!d.segments || d.num_segments == 0) { b->reset_network(); set_error("ensemble member %u has no segments", m); return BNC_ERR_ARG; }
        const uint32_t seg0 = (uint32_t)hn.seg.size(), syn0 = (uint32_t)hn.syn.size();
        const uint32_t st0 = (uint32_t)b->stim.current.size();
        uint32_t ns = (stim && n_stim && stim[m]) ? n_stim[m] : 0;
        sink.begin(d.num_neurons, d.num_segments, d.num_connections, d.num_synapses, ns);
        uint64_t valid_conn = 0;
        for (uint32_t i = 0; i < d.num_segments; i++) sink.segment(d.segments[i]);
        for (uint32_t c = 0; c < d.num_connections; c++) {
            if (d.connections[c].segment_a < d.num_segments && d.connections[c].segment_b < d.num_segments) valid_conn++;
            sink.connection(d.connections[c]);
        }
        for (uint32_t k = 0; k < d.num_synapses; k++) sink.synapse(d.synapses[k]);
        for (uint32_t k = 0; k < ns; k++) sink.stimulus(stim[m][k]);
        int rc = add_member(mem, sw, hn, b->stim.current.size(), seg0, syn0, st0, valid_conn);
        if (rc != BNC_OK) { b->reset_network(); return rc; }
    }
    cudaSetDevice(b->device);
    int rc = build_network(hn, b->stim, &b->dev, &b->host, &b->allocs);
    if (rc != BNC_OK) { b->reset_network(); return rc; }
    b->members = std::move(mem);
    b->loaded = true;
    return BNC_OK;
}

int bnc_ensemble_member(void* sim, uint32_t member, BncEnsembleMember* out) {
    if (!sim || !out) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (member >= b->members.size()) {
        set_error("ensemble member %u out of range (%zu members loaded)", member, b->members.size());
        return BNC_ERR_ARG;
    }
    *out = b->members[member];
    return BNC_OK;
}

int bnc_plan_ensemble_generated(const BncNetgenParams* members, uint32_t n_members, BncNetInfo* info) {
    if (!members || !info) { set_error("bnc_plan_ensemble_generated: null argument"); return BNC_ERR_ARG; }
    HostNet hn;
    Stimuli st;
    std::vector<BncEnsembleMember> mem;
    int rc = gather_generated(members, n_members, &hn, &st.current, &mem);
    if (rc != BNC_OK) return rc;
    return plan_info(hn, st, info);
}

int bnc_run_ticks_graph(void* sim, uint32_t n_ticks, float dt) {
    if (!sim) { set_error("null handle"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    int rc = run_ticks_graph(b, n_ticks, dt);
    if (rc != BNC_OK) return rc;
    return sync_stream(b);
}

int bnc_plan_aos(const BncBionData* data, const BncCurrentStimulus* stim, uint32_t n_stim, BncNetInfo* info) {
    if (!data || !info || (!data->segments && data->num_segments)) { set_error("bnc_plan_aos: null argument"); return BNC_ERR_ARG; }
    HostNet hn;
    hostnet_from_aos(*data, &hn);
    Stimuli st;
    if (stim && n_stim) st.current.assign(stim, stim + n_stim);
    return plan_info(hn, st, info);
}

int bnc_bion_load(const char* filename, BncBionData* out) {
    if (!filename || !out) { set_error("bnc_bion_load: null argument"); return BNC_ERR_ARG; }
    return load_bion_file(filename, out);
}

void bnc_bion_unload(BncBionData* data) {
    if (data) free_aos_arrays(*data);
}

int bnc_bion_save(const char* filename, const BncBionData* data) {
    if (!filename || !data || !data->segments) { set_error("bnc_bion_save: null argument"); return BNC_ERR_ARG; }
    return save_bion(*data, filename);
}

int bnc_run_ticks(void* sim, uint32_t n_ticks, float dt) {
    if (!sim) { set_error("null handle"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    int rc = run_ticks(b, n_ticks, dt);
    if (rc != BNC_OK) return rc;
    return sync_stream(b);
}

int bnc_time_ticks(void* sim, uint32_t n_ticks, float dt, float* ms) {
    if (!sim || !ms) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    cudaSetDevice(b->device);
    cudaEventRecord(b->ev0, b->stream);
    int rc = run_ticks(b, n_ticks, dt);
    if (rc != BNC_OK) return rc;
    cudaEventRecord(b->ev1, b->stream);
    rc = sync_stream(b);
    if (rc != BNC_OK) return rc;
    cudaEventElapsedTime(ms, b->ev0, b->ev1);
    return BNC_OK;
}

int bnc_step_io(void* sim, float dt, const float* stim_amp, uint32_t n_amp, float* v_out, uint32_t n_v) {
    if (!sim) { set_error("null handle"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    cudaSetDevice(b->device);
    cudaError_t e;
    if (stim_amp && n_amp) {
        if (!b->dev.cs_off || n_amp != (uint32_t)b->stim.current.size()) {
            set_error("stimulus amplitude count %u does not match the %zu loaded current stimuli", n_amp,
                      b->stim.current.size());
            return BNC_ERR_ARG;
        }
        if (b->host.stim_identity) {
            e = cudaMemcpyAsync(b->dev.cs_amp, stim_amp, n_amp * sizeof(float), cudaMemcpyHostToDevice, b->stream);
            if (e != cudaSuccess) return cuda_fail(e, "stimulus upload");
        } else {
            set_error("per-step amplitudes need stimuli uploaded in per-segment order");
            return BNC_ERR_UNSUPPORTED;
        }
    }
    int rc = run_ticks(b, 1, dt);
    if (rc != BNC_OK) return rc;
    if (v_out && n_v) {
        if (n_v < b->dev.n_seg) { set_error("V buffer too short"); return BNC_ERR_ARG; }
        if (!b->host.perm_identity) { set_error("V read-back in step_io needs an identity segment order"); return BNC_ERR_UNSUPPORTED; }
        e = cudaMemcpyAsync(v_out, b->dev.V, b->dev.n_seg * sizeof(float), cudaMemcpyDeviceToHost, b->stream);
        if (e != cudaSuccess) return cuda_fail(e, "V read-back");
    }
    return sync_stream(b);
}

int bnc_profile_ticks(void* sim, uint32_t n_ticks, float dt, float* ms_modifiers, float* ms_diffusion,
                      float* ms_synapse) {
    if (!sim || !ms_modifiers || !ms_diffusion || !ms_synapse) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    cudaSetDevice(b->device);
    cudaEvent_t e[4];
    for (auto& x : e) cudaEventCreate(&x);
    float tm = 0.0f, td = 0.0f, ts = 0.0f;
    int rc = BNC_OK;
    for (uint32_t t = 0; t < n_ticks && rc == BNC_OK; t++) {
        cudaEventRecord(e[0], b->stream);
        cudaError_t er = launch_modifiers(b->dev, b->host, dt, b->tick, b->stream);
        if (er != cudaSuccess) { rc = cuda_fail(er, "modifier kernel launch"); break; }
        cudaEventRecord(e[1], b->stream);
        er = launch_diffusion(b->dev, b->host, dt, b->tick, b->stream);
        if (er != cudaSuccess) { rc = cuda_fail(er, "diffusion kernel launch"); break; }
        cudaEventRecord(e[2], b->stream);
        er = launch_synapse(b->dev, dt, b->tick, b->ticks_run == 0 ? 1 : 0, b->stream);
        if (er != cudaSuccess) { rc = cuda_fail(er, "synapse kernel launch"); break; }
        cudaEventRecord(e[3], b->stream);
        tick_enqueued(b);
        rc = sync_stream(b);
        if (rc != BNC_OK) break;
        float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
        cudaEventElapsedTime(&a0, e[0], e[1]);
        cudaEventElapsedTime(&a1, e[1], e[2]);
        cudaEventElapsedTime(&a2, e[2], e[3]);
        tm += a0;
        td += a1;
        ts += a2;
    }
    for (auto& x : e) cudaEventDestroy(x);
    *ms_modifiers = tm;
    *ms_diffusion = td;
    *ms_synapse = ts;
    return rc;
}

int bnc_sync_to_host(void* sim) {
    if (!sim) { set_error("null handle"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    cudaSetDevice(b->device);
    return export_records(b);
}

int bnc_records_managed(void* sim) {
    return (sim && static_cast<Backend*>(sim)->aos_managed) ? 1 : 0;
}

int bnc_set_records_residency(void* sim, int on_host) {
    if (!sim) { set_error("null handle"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded || !b->owns_aos) { set_error("no drop-in records"); return BNC_ERR_STATE; }
    cudaSetDevice(b->device);
    int rc = sync_stream(b);
    if (rc != BNC_OK) return rc;
    if (!on_host) return b->aos_managed ? BNC_OK : make_records_managed(b);
    if (!b->aos_managed) return BNC_OK;
    // back to host records, updated by the bulk host export after each tick
    const size_t n = b->aos.num_segments, k = b->aos.num_synapses;
    BncSegment* hs = new (std::nothrow) BncSegment[n ? n : 1];
    BncSynapse* hy = new (std::nothrow) BncSynapse[k ? k : 1];
    if (!hs || !hy) { delete[] hs; delete[] hy; set_error("host record allocation failed"); return BNC_ERR_ALLOC; }
    if (n) std::memcpy(hs, b->aos.segments, n * sizeof(BncSegment));
    if (k) std::memcpy(hy, b->aos.synapses, k * sizeof(BncSynapse));
    cudaFree(b->aos.segments);
    cudaFree(b->aos.synapses);
    b->aos.segments = hs;
    b->aos.synapses = hy;
    b->aos_managed = false;
    return BNC_OK;
}

int bnc_read_segment_field(void* sim, int field, int index, float* out, uint32_t n) {
    if (!sim || !out) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    const NetDev& d = b->dev;
    const uint32_t N = d.n_seg;
    if (n < N) { set_error("output buffer holds %u values, %u needed", n, N); return BNC_ERR_ARG; }
    cudaSetDevice(b->device);
    int rc = sync_stream(b);
    if (rc != BNC_OK) return rc;
    std::vector<float> v(N);
    const float* src = nullptr;
    switch (field) {
        case 0: src = d.V; break;
        case 1: if (index < 0 || index > 6) return BNC_ERR_ARG; src = d.ion_in + (size_t)index * N; break;
        case 2: if (index < 0 || index > 6) return BNC_ERR_ARG; src = d.ion_out + (size_t)index * N; break;
        case 3: src = d.atp; break;
        case 4: src = d.temp; break;
        case 5: src = d.txn; break;
        case 6: if (index < 0 || index > 14) return BNC_ERR_ARG; src = d.intra_nt + (size_t)index * N; break;
        case 7: if (index < 0 || index > 14) return BNC_ERR_ARG; src = d.nt + (size_t)index * N; break;
        case 8: {
            int slot = index >> 3, k = index & 7;
            if (k > 6) { set_error("state[7] is the effective area"); return BNC_ERR_ARG; }
            std::vector<float> st;
            if (!d2h(st, d.it_st + (size_t)k * d.n_items, d.n_items)) return cuda_fail(cudaGetLastError(), "read");
            for (uint32_t i = 0; i < N; i++) {
                out[i] = 0.0f;
                if (b->owns_aos && slot < b->aos.segments[i].modifier_count)
                    out[i] = (float)b->aos.segments[i].modifiers[slot].state[k];
            }
            for (uint32_t q = 0; q < d.n_items; q++)
                if (b->host.item_slot[q] == slot) out[b->host.item_seg[q]] = st[q];
            return BNC_OK;
        }
        case 9: {
            std::vector<uint32_t> c;
            if (!d2h(c, d.spike_count, N)) return cuda_fail(cudaGetLastError(), "read");
            for (uint32_t dd = 0; dd < N; dd++) out[b->host.perm[dd]] = (float)c[dd];
            return BNC_OK;
        }
        default: set_error("unknown segment field %d", field); return BNC_ERR_ARG;
    }
    if (cudaMemcpy(v.data(), src, N * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "read");
    for (uint32_t dd = 0; dd < N; dd++) out[b->host.perm[dd]] = v[dd];
    return BNC_OK;
}

int bnc_read_synapse_field(void* sim, int field, int index, float* out, uint32_t n) {
    if (!sim || !out) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    const NetDev& d = b->dev;
    const uint32_t K = d.n_syn, KT = b->host.n_syn_total;
    if (n < KT) { set_error("output buffer holds %u values, %u needed", n, KT); return BNC_ERR_ARG; }
    cudaSetDevice(b->device);
    int rc = sync_stream(b);
    if (rc != BNC_OK) return rc;
    for (uint32_t i = 0; i < KT; i++) out[i] = 0.0f;
    std::vector<float> v;
    const float* src = nullptr;
    switch (field) {
        case 0: src = d.sy_bouton; break;
        case 1: src = d.sy_spine; break;
        case 2: src = d.sy_weight; break;
        case 3: {
            std::vector<uint8_t> r;
            if (!d2h(r, d.sy_refr, K)) return cuda_fail(cudaGetLastError(), "read");
            for (uint32_t q = 0; q < K; q++) out[b->host.syn_orig[q]] = (float)r[q];
            return BNC_OK;
        }
        case 4: {
            if (index == 9 && d.sy_cleft_ecb) {   // the endocannabinoid entry
                if (!d2h(v, d.sy_cleft_ecb, K)) return cuda_fail(cudaGetLastError(), "read");
                for (uint32_t q = 0; q < K; q++) out[b->host.syn_orig[q]] = v[q];
                return BNC_OK;
            }
            if (!d2h(v, d.sy_cleft, K)) return cuda_fail(cudaGetLastError(), "read");
            for (uint32_t q = 0; q < K; q++) out[b->host.syn_orig[q]] = (b->host.syn_nt[q] == index) ? v[q] : 0.0f;
            if (index == 0 && d.n_gj) {   // a gap junction's cleft entry 0 holds its filtered current
                if (!d2h(v, d.gj_flt, d.n_gj)) return cuda_fail(cudaGetLastError(), "read");
                for (uint32_t g = 0; g < d.n_gj; g++) out[b->host.gj_syn[g]] = v[g];
            }
            return BNC_OK;
        }
        case 5: {
            int j = index >> 3, k = index & 7;
            if (k > 2) { set_error("receptor states above 2 are not tracked"); return BNC_ERR_ARG; }
            if (!d2h(v, d.rc_st + (size_t)k * d.n_rec, d.n_rec)) return cuda_fail(cudaGetLastError(), "read");
            for (uint32_t r = 0; r < d.n_rec; r++)
                if (b->host.rec_slot[r] == j) out[b->host.syn_orig[b->host.rec_syn[r]]] = v[r];
            return BNC_OK;
        }
        case 6: src = d.sy_facil; break;
        case 7: src = d.sy_camkii; break;
        case 8: src = d.sy_calcn; break;
        case 9: src = d.sy_rrp; break;
        case 10: {   // depression: BCM's threshold (facilitation + 0.01 after a tick), a gap junction's slow gate
            if (!d2h(v, d.sy_facil, K)) return cuda_fail(cudaGetLastError(), "read");
            for (uint32_t q = 0; q < K; q++) {
                const uint32_t o = b->host.syn_orig[q];
                out[o] = b->ticks_run > 0 ? v[q] + 0.01f
                                          : ((b->owns_aos && b->aos.synapses) ? b->aos.synapses[o].depression : 0.0f);
            }
            if (d.n_gj) {
                if (!d2h(v, d.gj_dep, d.n_gj)) return cuda_fail(cudaGetLastError(), "read");
                for (uint32_t g = 0; g < d.n_gj; g++) out[b->host.gj_syn[g]] = v[g];
            }
            return BNC_OK;
        }
        case 11: {   // autoreceptor state: index = slot * 8 + word; word 0 of release modulators
            const int j = index >> 3, w = index & 7;
            if (w != 0) { set_error("autoreceptor states other than word 0 of release modulators are not tracked"); return BNC_ERR_ARG; }
            if (d.n_md && !d2h(v, d.md_st, d.n_md)) return cuda_fail(cudaGetLastError(), "read");
            for (uint32_t q = 0; q < d.n_md; q++)
                if (b->host.md_slot[q] == j) out[b->host.md_syn[q]] = v[q];
            return BNC_OK;
        }
        default: set_error("unknown synapse field %d", field); return BNC_ERR_ARG;
    }
    if (!d2h(v, src, K)) return cuda_fail(cudaGetLastError(), "read");
    for (uint32_t q = 0; q < K; q++) out[b->host.syn_orig[q]] = v[q];
    return BNC_OK;
}

int bnc_set_synapse_scale(void* sim, const float* scale, uint32_t n) {
    if (!sim || !scale) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    if (n < b->host.n_syn_total) { set_error("scale array too short"); return BNC_ERR_ARG; }
    std::vector<float> v(b->dev.n_syn);
    for (uint32_t q = 0; q < b->dev.n_syn; q++) v[q] = scale[b->host.syn_orig[q]];
    cudaSetDevice(b->device);
    if (cudaMemcpy(b->dev.sy_scale, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "scale upload");
    return BNC_OK;
}

int bnc_network_info(void* sim, BncNetInfo* info) {
    if (!sim || !info) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    std::memset(info, 0, sizeof(*info));
    if (!b->loaded) return BNC_ERR_STATE;
    const NetDev& d = b->dev;
    info->n_segments = d.n_seg; info->n_connections = b->host.n_conn; info->n_synapses = d.n_syn;
    info->n_tiles = d.n_tiles; info->n_items = d.n_items; info->n_phases = d.n_phases; info->n_receptors = d.n_rec;
    info->max_tile_segs = b->host.max_tile_segs; info->max_tile_edges = b->host.max_tile_edges;
    info->smem_bytes = (uint32_t)b->host.smem_bytes; info->flags = d.flags;
    info->ticks = b->ticks_run;
    info->algo_bytes_per_tick = b->host.algo_bytes_per_tick;
    info->seg_bytes_per_tick = b->host.seg_bytes;
    info->syn_bytes_per_tick = b->host.syn_bytes;
    info->tile_bytes_per_tick = b->host.tile_bytes;
    info->synapse_kernel_bytes_per_tick = b->host.synk_bytes;
    info->modifier_launches = modifier_launches(d, b->host); info->fuse_phases = b->host.fuse;
    info->group_tiles_32 = b->host.group_tiles_32; info->group_tiles_64 = b->host.group_tiles_64;
    info->diffusion_threads = b->host.diff_threads;
    info->synapse_launches = synapse_launches(d);
    info->warp_cap = b->host.opt.warp_cap; info->tile_segs = b->host.opt.tile_segs;
    info->modifier_kernel_bytes = b->host.mod_bytes; info->diffusion_kernel_bytes = b->host.diff_bytes;
    return BNC_OK;
}

int bnc_save_bion(void* sim, const char* filename) {
    if (!sim || !filename) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->owns_aos) { set_error("no host AoS view (network was generated on the device)"); return BNC_ERR_STATE; }
    int rc = bnc_sync_to_host(sim);
    if (rc != BNC_OK) return rc;
    return save_bion(b->aos, filename);
}

// ---- Electrodiffusion options: residual-controlled Jacobi solves, the ion ledger ----
int bnc_set_diffusion_mode(void* sim, uint32_t flags, double tol, uint32_t max_sweeps) {
    if (!sim) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    if (flags & ~(uint32_t)(BNC_DIFFUSION_RESIDUAL | BNC_DIFFUSION_LEDGER)) {
        set_error("unknown diffusion flags 0x%x", flags);
        return BNC_ERR_ARG;
    }
    if ((flags & BNC_DIFFUSION_RESIDUAL) && (!(tol > 0.0) || max_sweeps == 0)) {
        set_error("the residual mode needs tol > 0 and max_sweeps >= 1 (tol %g, max_sweeps %u)", tol, max_sweeps);
        return BNC_ERR_ARG;
    }
    b->drop_graph();   // a captured tick holds the descriptor by value
    b->dev.diff_mode = flags;
    b->dev.jac_tol = (flags & BNC_DIFFUSION_RESIDUAL) ? tol : 0.0;
    b->dev.jac_max = (flags & BNC_DIFFUSION_RESIDUAL) ? max_sweeps : 0u;
    return BNC_OK;
}

int bnc_diffusion_stats(void* sim, BncDiffusionStats* out, int reset) {
    if (!sim || !out) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    cudaSetDevice(b->device);
    int rc = sync_stream(b);
    if (rc != BNC_OK) return rc;
    std::memset(out, 0, sizeof(*out));
    uint32_t st[4] = {0, 0, 0, 0};
    double led[14] = {0};
    cudaError_t e = cudaMemcpy(st, b->dev.jac_stats, sizeof(st), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(led, b->dev.ledger, sizeof(led), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && reset) {
        e = cudaMemset(b->dev.jac_stats, 0, sizeof(st));
        if (e == cudaSuccess) e = cudaMemset(b->dev.ledger, 0, sizeof(led));
    }
    if (e != cudaSuccess) return cuda_fail(e, "diffusion statistics");
    out->max_sweeps_v = st[0];
    out->max_sweeps_phi = st[1];
    out->capped_v = st[2];
    out->capped_phi = st[3];
    for (int q = 0; q < 7; q++) { out->rounding[q] = led[q]; out->bath[q] = led[7 + q]; }
    return BNC_OK;
}

// ---- The daemon's state frame (daemon_state.cpp:66-79) from the device state ----
int bnc_state_frame(void* sim, void* buf, uint64_t cap, uint64_t* len) {
    if (!sim || !len) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    if (!b->owns_aos || !b->aos.segments) { set_error("no host AoS view (network was generated on the device)"); return BNC_ERR_STATE; }
    const uint32_t N = b->aos.num_segments, K = b->aos.num_synapses;
    const uint64_t need = 16ull + (uint64_t)N * sizeof(BncSegment) + (uint64_t)K * sizeof(BncSynapse);
    *len = need;
    if (!buf || cap < need) { set_error("frame needs %llu bytes", (unsigned long long)need); return BNC_ERR_ARG; }
    uint8_t* p = static_cast<uint8_t*>(buf);
    // the records' static fields from the host copy, then the device state written over
    // them in place
    BncBionData view = b->aos;
    view.segments = reinterpret_cast<BncSegment*>(p + 16);
    view.synapses = reinterpret_cast<BncSynapse*>(p + 16 + (size_t)N * sizeof(BncSegment));
    std::memcpy(view.segments, b->aos.segments, (size_t)N * sizeof(BncSegment));
    if (K) std::memcpy(view.synapses, b->aos.synapses, (size_t)K * sizeof(BncSynapse));
    cudaSetDevice(b->device);
    int rc = sync_stream(b);
    if (rc != BNC_OK) return rc;
    rc = export_network(b->dev, b->host, b->ticks_run, &view);
    if (rc != BNC_OK) return rc;
    const uint64_t tick = b->tick;
    std::memcpy(p, &tick, 8);
    std::memcpy(p + 8, &N, 4);
    std::memcpy(p + 12, &K, 4);
    return BNC_OK;
}

// ---- Checkpoints: the .bion plus what it does not hold ----
// The .bion records the AoS state.  A run also carries the tick counter (it seeds the
// release draws and times the stimuli), whether the first tick has run, the stimuli
// (current steps, voltage clamps, ramps, and ion and ligand injections uploaded but not
// yet applied), the per-synapse receptor density scales and the pending delayed
// releases (delay_buffer.h:15-64).  The sidecar `<path>.state` holds them, so a loaded
// checkpoint continues bit for bit.  Version 1 files held no ramps and no pending
// injections; they are refused, since a run with either would not resume exactly.
namespace {
const char kStateMagic[8] = {'B', 'N', 'C', 'S', 'T', 'A', 'T', 'E'};
constexpr uint32_t kStateVersion = 2;
struct DelaySlot {
    unsigned long long arrival;
    float amount;
    uint8_t nt, pad[3];
};
}  // namespace

int bnc_save_checkpoint(void* sim, const char* path) {
    if (!sim || !path) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    if (!b->members.empty()) { set_error("checkpoints hold one network, not an ensemble"); return BNC_ERR_UNSUPPORTED; }
    int rc = bnc_save_bion(sim, path);
    if (rc != BNC_OK) return rc;
    const NetDev& d = b->dev;
    const uint32_t K = d.n_syn;
    const uint32_t KS = b->host.n_syn_total;
    std::vector<float> scale_dev, scale(KS, 1.0f);
    if (K && !d2h(scale_dev, d.sy_scale, K)) return cuda_fail(cudaGetLastError(), "checkpoint read");
    for (uint32_t k = 0; k < K; k++) scale[b->host.syn_orig[k]] = scale_dev[k];
    std::vector<DelaySlot> slots;
    uint32_t has_delay = d.dl_arr ? 1u : 0u;
    if (has_delay) {
        std::vector<unsigned long long> arr;
        std::vector<float> amt;
        std::vector<uint8_t> nt;
        if (!d2h(arr, d.dl_arr, (size_t)4 * K) || !d2h(amt, d.dl_amt, (size_t)4 * K) || !d2h(nt, d.dl_nt, (size_t)4 * K))
            return cuda_fail(cudaGetLastError(), "checkpoint read");
        slots.assign((size_t)4 * KS, DelaySlot{0, 0.0f, 0, {0, 0, 0}});
        for (uint32_t k = 0; k < K; k++)
            for (int q = 0; q < 4; q++) {
                DelaySlot& sl = slots[(size_t)b->host.syn_orig[k] * 4 + q];
                sl.arrival = arr[(size_t)q * K + k];
                sl.amount = amt[(size_t)q * K + k];
                sl.nt = nt[(size_t)q * K + k];
            }
    }
    const std::string sp = std::string(path) + ".state";
    FILE* f = fopen(sp.c_str(), "wb");
    if (!f) { set_error("cannot write %s", sp.c_str()); return BNC_BION_ERR_FILE_OPEN; }
    const uint32_t n_cur = (uint32_t)b->stim.current.size(), n_vc = (uint32_t)b->stim.vclamp.size();
    const uint32_t n_ramp = (uint32_t)b->stim.ramp.size();
    const uint32_t n_ion = (uint32_t)b->pend_ion.size(), n_lig = (uint32_t)b->pend_lig.size();
    const uint32_t head[9] = {kStateVersion, b->host.n_seg, KS, n_cur, n_vc, has_delay, n_ramp, n_ion, n_lig};
    const uint64_t ticks[2] = {b->tick, b->ticks_run};
    bool ok = fwrite(kStateMagic, 1, 8, f) == 8 && fwrite(head, sizeof(head), 1, f) == 1 && fwrite(ticks, sizeof(ticks), 1, f) == 1;
    if (ok && n_cur) ok = fwrite(b->stim.current.data(), sizeof(BncCurrentStimulus), n_cur, f) == n_cur;
    if (ok && n_vc) ok = fwrite(b->stim.vclamp.data(), sizeof(BncVoltageClamp), n_vc, f) == n_vc;
    if (ok && n_ramp) ok = fwrite(b->stim.ramp.data(), sizeof(BncRampStimulus), n_ramp, f) == n_ramp;
    if (ok && n_ion) ok = fwrite(b->pend_ion.data(), sizeof(BncIonInjection), n_ion, f) == n_ion;
    if (ok && n_lig) ok = fwrite(b->pend_lig.data(), sizeof(BncLigandInjection), n_lig, f) == n_lig;
    if (ok && KS) ok = fwrite(scale.data(), sizeof(float), KS, f) == KS;
    if (ok && has_delay && KS) ok = fwrite(slots.data(), sizeof(DelaySlot), slots.size(), f) == slots.size();
    if (fclose(f) != 0) ok = false;
    if (!ok) { set_error("write error on %s", sp.c_str()); return BNC_BION_ERR_WRITE_FAIL; }
    return BNC_OK;
}

int bnc_load_checkpoint(void* sim, const char* path) {
    if (!sim || !path) { set_error("null argument"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    const std::string sp = std::string(path) + ".state";
    FILE* f = fopen(sp.c_str(), "rb");
    if (!f) { set_error("cannot read %s", sp.c_str()); return BNC_BION_ERR_FILE_OPEN; }
    char magic[8];
    uint32_t version = 0;
    uint32_t head[9];
    uint64_t ticks[2];
    bool ok = fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kStateMagic, 8) == 0 && fread(&version, 4, 1, f) == 1;
    if (ok && version != kStateVersion) {
        fclose(f);
        set_error("%s is a version %u state file; this library reads version %u (version 1 held no ramps "
                  "and no pending injections)", sp.c_str(), version, kStateVersion);
        return BNC_ERR_FORMAT;
    }
    head[0] = version;
    ok = ok && fread(head + 1, sizeof(head) - 4, 1, f) == 1 && fread(ticks, sizeof(ticks), 1, f) == 1 &&
         head[6] <= BNC_GPU_MAX_STIMULI && head[7] <= BNC_GPU_MAX_STIMULI && head[8] <= BNC_GPU_MAX_STIMULI;
    Stimuli stim;
    std::vector<float> scale;
    std::vector<DelaySlot> slots;
    if (ok) {
        stim.current.resize(head[3]);
        stim.vclamp.resize(head[4]);
        stim.ramp.resize(head[6]);
        stim.ion_inj.resize(head[7]);
        stim.lig_inj.resize(head[8]);
        scale.resize(head[2]);
        if (head[3]) ok = fread(stim.current.data(), sizeof(BncCurrentStimulus), head[3], f) == head[3];
        if (ok && head[4]) ok = fread(stim.vclamp.data(), sizeof(BncVoltageClamp), head[4], f) == head[4];
        if (ok && head[6]) ok = fread(stim.ramp.data(), sizeof(BncRampStimulus), head[6], f) == head[6];
        if (ok && head[7]) ok = fread(stim.ion_inj.data(), sizeof(BncIonInjection), head[7], f) == head[7];
        if (ok && head[8]) ok = fread(stim.lig_inj.data(), sizeof(BncLigandInjection), head[8], f) == head[8];
        if (ok && head[2]) ok = fread(scale.data(), sizeof(float), head[2], f) == head[2];
        if (ok && head[5] && head[2]) {
            slots.resize((size_t)4 * head[2]);
            ok = fread(slots.data(), sizeof(DelaySlot), slots.size(), f) == slots.size();
        }
    }
    fclose(f);
    if (!ok) { set_error("%s is not a checkpoint state file of this version", sp.c_str()); return BNC_ERR_FORMAT; }
    b->reset_network();
    BncBionData aos;
    int rc = load_bion_file(path, &aos, false);   // the nuclei the run had, none added
    if (rc != BNC_OK) return rc;
    if (aos.num_segments != head[1] || aos.num_synapses != head[2]) {
        free_aos_arrays(aos);
        set_error("checkpoint state does not match %s", path);
        return BNC_ERR_FORMAT;
    }
    b->stim = stim;
    rc = load_common(b, aos, true);
    if (rc != BNC_OK) { free_aos_arrays(aos); return rc; }
    // the pending injections went to the device with the build; the next tick applies them
    b->pend_ion.swap(b->stim.ion_inj);
    b->pend_lig.swap(b->stim.lig_inj);
    b->stim.ion_inj.clear();
    b->stim.lig_inj.clear();
    b->tick = ticks[0];
    b->ticks_run = ticks[1];
    const NetDev& d = b->dev;
    const uint32_t K = d.n_syn;
    if (K) {
        std::vector<float> sdev(K);
        for (uint32_t k = 0; k < K; k++) sdev[k] = scale[b->host.syn_orig[k]];
        if (cudaMemcpy(d.sy_scale, sdev.data(), K * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
            return cuda_fail(cudaGetLastError(), "checkpoint upload");
    }
    if (!slots.empty()) {
        if (!d.dl_arr) {
            for (const DelaySlot& sl : slots)
                if (sl.arrival) { set_error("pending delayed releases, but the network has no delays"); return BNC_ERR_FORMAT; }
        } else {
            std::vector<unsigned long long> arr((size_t)4 * K);
            std::vector<float> amt((size_t)4 * K);
            std::vector<uint8_t> nt((size_t)4 * K);
            for (uint32_t k = 0; k < K; k++)
                for (int q = 0; q < 4; q++) {
                    const DelaySlot& sl = slots[(size_t)b->host.syn_orig[k] * 4 + q];
                    arr[(size_t)q * K + k] = sl.arrival;
                    amt[(size_t)q * K + k] = sl.amount;
                    nt[(size_t)q * K + k] = sl.nt;
                }
            if (cudaMemcpy(d.dl_arr, arr.data(), arr.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(d.dl_amt, amt.data(), amt.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(d.dl_nt, nt.data(), nt.size(), cudaMemcpyHostToDevice) != cudaSuccess)
                return cuda_fail(cudaGetLastError(), "checkpoint upload");
        }
    }
    return BNC_OK;
}

}  // extern "C"

// ---- Ticks with the presynaptic exchange records in a library-owned array ----
//
// Each tick the diffusion kernel writes, for every segment, the record the synapse
// kernel reads for that segment as a presynaptic site: V, Ca_out and the Cav2.1
// density and h gate (float4), plus Na_in, K_in, Ca_in, Na_out (float4) and K_out
// (float) when some synapse has autoreceptors or a readily releasable pool.  That
// is 36 bytes of scratch per segment, rewritten every tick.  bnc_run_ticks takes it
// from buffers allocated with the network; bnc_run_ticks_static_scratch takes it
// from the fixed array below, for callers that cannot allocate device memory while
// they run the simulation.
namespace bnc {
namespace {

constexpr uint32_t kScratchSegs = BNC_STATIC_SCRATCH_MAX_SEGMENTS;
constexpr size_t kScratchRecOff = 0;                                             // float4 [kScratchSegs]
constexpr size_t kScratchExtOff = (size_t)kScratchSegs * sizeof(float4);         // float4 [kScratchSegs]
constexpr size_t kScratchExt2Off = (size_t)kScratchSegs * 2 * sizeof(float4);    // float  [kScratchSegs]
constexpr size_t kScratchBytes = kScratchExt2Off + (size_t)kScratchSegs * sizeof(float);
static_assert(kScratchExtOff % 256 == 0 && kScratchExt2Off % 256 == 0, "scratch parts stay 256-byte aligned");

// One copy per device that loads the library, alive until the process exits.  In
// host code this name is only a stand-in for the symbol: the kernels get the device
// address that cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_tick_scratch[kScratchBytes];

constexpr int kScratchMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char* g_scratch_addr[kScratchMaxDevices] = {};

// Device address of g_tick_scratch on `device`, which must be the current device.
// Looked up on the first call per device and kept.
int scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kScratchMaxDevices) {
        set_error("bnc_run_ticks_static_scratch: device %d outside 0..%d", device, kScratchMaxDevices - 1);
        return BNC_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_tick_scratch);
        if (e != cudaSuccess || !p) return cuda_fail(e, "cudaGetSymbolAddress of the static tick scratch");
        g_scratch_addr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[device];
    return BNC_OK;
}

}  // namespace
}  // namespace bnc

extern "C" int bnc_run_ticks_static_scratch(void* sim, uint32_t n_ticks, float dt) {
    if (!sim) { set_error("null handle"); return BNC_ERR_ARG; }
    Backend* b = static_cast<Backend*>(sim);
    if (!b->loaded) { set_error("no network loaded"); return BNC_ERR_STATE; }
    if (b->failed) { set_error("backend is in a failed state after a device error"); return BNC_ERR_STATE; }
    const uint32_t n = b->dev.n_seg;
    if (n > kScratchSegs) {
        set_error("bnc_run_ticks_static_scratch: the network has %u segments, the static scratch holds at most %u "
                  "(BNC_STATIC_SCRATCH_MAX_SEGMENTS); use bnc_run_ticks", n, kScratchSegs);
        return BNC_ERR_ARG;
    }
    cudaError_t e = cudaSetDevice(b->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    unsigned char* base = nullptr;
    int rc = scratch_address(b->device, &base);
    if (rc != BNC_OK) return rc;

    // The network's own pointers, with the exchange records redirected into the array
    // (the optional part only where the network has one).
    NetDev d = b->dev;
    d.pre_rec = reinterpret_cast<float4*>(base + kScratchRecOff);
    if (b->dev.pre_ext) d.pre_ext = reinterpret_cast<float4*>(base + kScratchExtOff);
    if (b->dev.pre_ext2) d.pre_ext2 = reinterpret_cast<float*>(base + kScratchExt2Off);
    // The array keeps whatever the previous call left; start from zero as the
    // network's own buffers do.
    if (n) {
        e = cudaMemsetAsync(d.pre_rec, 0, (size_t)n * sizeof(float4), b->stream);
        if (e == cudaSuccess && b->dev.pre_ext) e = cudaMemsetAsync(d.pre_ext, 0, (size_t)n * sizeof(float4), b->stream);
        if (e == cudaSuccess && b->dev.pre_ext2) e = cudaMemsetAsync(d.pre_ext2, 0, (size_t)n * sizeof(float), b->stream);
        if (e != cudaSuccess) { b->failed = true; return cuda_fail(e, "clearing the static tick scratch"); }
    }
    for (uint32_t t = 0; t < n_ticks; t++) {
        e = launch_tick(d, b->host, dt, b->tick, b->ticks_run == 0 ? 1 : 0, b->stream);
        if (e != cudaSuccess) { b->failed = true; return cuda_fail(e, "tick launch"); }
        tick_enqueued(b);
        d.inj = nullptr;
        d.inj_n = nullptr;
    }
    return sync_stream(b);
}
