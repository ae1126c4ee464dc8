// capi_host.cpp -- host-only C ABI: the synthetic generator's AoS output and the
// per-thread error message.  No CUDA calls, so these work on a machine without a GPU.
#include <cmath>
#include <cstring>
#include <cstdio>
#include <new>
#include <string>
#include "netgen.h"
#include "common.h"

namespace bnc {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

namespace {

// Sink that materialises the reference-layout AoS arrays.
struct AosSink : NetSink {
    BncBionData* out;
    std::vector<BncCurrentStimulus> stim;
    uint32_t ni = 0, si = 0, ci = 0;
    uint64_t yi = 0;
    bool ok = true;
    explicit AosSink(BncBionData* o) : out(o) {}
    void begin(uint32_t n_neurons, uint32_t n_segments, uint32_t n_connections, uint64_t n_synapses,
               uint32_t n_stimuli) override {
        std::memset(out, 0, sizeof(*out));
        out->header.magic = 0x42494F4Eu;  // BION_MAGIC (bion_format.h:12)
        out->header.version = 14;
        out->header.num_neurons = n_neurons;
        out->header.num_segments = n_segments;
        out->header.num_intra_connections = n_connections;
        out->header.num_synapses = (uint32_t)n_synapses;
        out->header.file_sz_segment = sizeof(BncSegment);
        out->header.file_sz_synapse = sizeof(BncSynapse);
        out->header.file_sz_intraconnection = sizeof(BncIntraConnection);
        out->header.file_sz_neuron = sizeof(BncNeuron);
        out->header.file_sz_modifier = sizeof(BncModifier);
        out->num_neurons = n_neurons;
        out->num_segments = n_segments;
        out->num_connections = n_connections;
        out->num_synapses = (uint32_t)n_synapses;
        out->neurons = new (std::nothrow) BncNeuron[n_neurons ? n_neurons : 1];
        out->segments = new (std::nothrow) BncSegment[n_segments ? n_segments : 1];
        out->connections = new (std::nothrow) BncIntraConnection[n_connections ? n_connections : 1];
        out->synapses = new (std::nothrow) BncSynapse[n_synapses ? n_synapses : 1];
        ok = out->neurons && out->segments && out->connections && out->synapses;
        stim.reserve(n_stimuli);
    }
    void neuron(const BncNeuron& n) override { if (ok) out->neurons[ni++] = n; }
    void segment(const BncSegment& s) override { if (ok) out->segments[si++] = s; }
    void connection(const BncIntraConnection& c) override { if (ok) out->connections[ci++] = c; }
    void synapse(const BncSynapse& s) override { if (ok) out->synapses[yi++] = s; }
    void stimulus(const BncCurrentStimulus& st) override { stim.push_back(st); }
};

}  // namespace
}  // namespace bnc

using namespace bnc;

extern "C" {

const char* bnc_last_error(void) { return g_last_error.c_str(); }

int bnc_netgen_aos(const BncNetgenParams* p, BncBionData* out, BncCurrentStimulus** stim,
                   uint32_t* n_stim) {
    if (!p || !out) { set_error("bnc_netgen_aos: null argument"); return BNC_ERR_ARG; }
    AosSink sink(out);
    NetShape shape;
    int rc = generate_network(*p, sink, &shape);
    if (rc != BNC_OK) { set_error("bnc_netgen_aos: invalid parameters (family %u)", p->family); return rc; }
    if (!sink.ok) { bnc_netgen_free(out, nullptr); set_error("bnc_netgen_aos: out of host memory"); return BNC_ERR_ALLOC; }
    if (stim) {
        *stim = nullptr;
        if (!sink.stim.empty()) {
            *stim = new BncCurrentStimulus[sink.stim.size()];
            std::memcpy(*stim, sink.stim.data(), sink.stim.size() * sizeof(BncCurrentStimulus));
        }
    }
    if (n_stim) *n_stim = (uint32_t)sink.stim.size();
    return BNC_OK;
}

int bnc_ensemble_params(uint64_t seed, uint32_t n_members, uint32_t min_segments, uint32_t max_segments,
                        BncNetgenParams* out) {
    if (!out || n_members == 0 || min_segments < 32 || max_segments < min_segments) {
        set_error("bnc_ensemble_params: need n_members > 0 and 32 <= min_segments <= max_segments");
        return BNC_ERR_ARG;
    }
    // SplitMix64 over (seed, member): sizes, conductance factors and member seeds
    auto mix = [](uint64_t z) {
        z += 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    auto u01 = [](uint64_t z) { return (double)(z >> 11) * (1.0 / 9007199254740992.0); };
    const double lo = std::log((double)min_segments), hi = std::log((double)max_segments);
    for (uint32_t m = 0; m < n_members; m++) {
        uint64_t s = mix(seed * 0x100000001B3ull + m);
        BncNetgenParams& p = out[m];
        std::memset(&p, 0, sizeof(p));
        p.family = BNC_NET_ENSEMBLE_MEMBER;
        double segs = std::exp(lo + (hi - lo) * u01(s));
        uint32_t nn = (uint32_t)(segs / 32.0 + 0.5);
        p.n_neurons = nn < 1 ? 1 : nn;
        for (int c = 0; c < 4; c++) {
            s = mix(s);
            p.conductance_scale[c] = (float)(0.5 + 1.5 * u01(s));   // U[0.5, 2]
        }
        p.seed = mix(s ^ 0xD1B54A32D192ED03ull);
    }
    return BNC_OK;
}

void bnc_netgen_free(BncBionData* d, BncCurrentStimulus* stim) {
    if (d) {
        delete[] d->neurons;
        delete[] d->segments;
        delete[] d->connections;
        delete[] d->synapses;
        d->neurons = nullptr; d->segments = nullptr; d->connections = nullptr; d->synapses = nullptr;
    }
    delete[] stim;
}

}  // extern "C"
