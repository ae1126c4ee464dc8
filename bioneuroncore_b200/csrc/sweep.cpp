// sweep.cpp -- the parameter-sweep entry: many parameterised runs of one network as
// one ensemble launch.
//
// The reference runs a parameterised task one process (or one daemon session) at a
// time: load the .bion, apply the parameter overrides, vary the synapses' release
// probabilities by a seed, run the ticks, compute the metrics (daemon_main.cpp:79-155,
// 160-300 for the batch mode; daemon_server.cpp:1164-1310 for MSG_RUN_TASK_PARAMS;
// simulation_host.cpp:825-880 for core_compute_metrics).  Here every task becomes one
// member of an ensemble (bnc_load_ensemble_aos), so a sweep of N tasks is one build
// and one tick loop over all members, and each member's results equal a standalone
// run of its task.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "net.h"

namespace bnc {
namespace {

constexpr uint32_t kModTypeCount = 212;   // MOD_TYPE_COUNT, types.h:263

bool name_matches(const char* name, const std::string& key) {
    // the key is a case-insensitive prefix of the name (daemon_main.cpp:121-134)
    const char* n = name;
    const char* k = key.c_str();
    while (*n && *k) {
        if (std::tolower((unsigned char)*n) != std::tolower((unsigned char)*k)) break;
        n++; k++;
    }
    return *k == 0;
}

// core_compute_metrics (simulation_host.cpp:825-880) on one member's state.
void member_metrics(const float* V, uint32_t n_seg, const BncNeuron* neurons, uint32_t n_neurons, uint64_t tick,
                    BncSweepResult* r) {
    float sum_vm = 0.0f;
    uint32_t spikes = 0;
    for (uint32_t i = 0; i < n_seg; i++) {
        sum_vm = (float)((double)sum_vm + (double)V[i]);   // the AoS V_m is double
        if ((double)V[i] > -20.0f) spikes++;
    }
    const float mean_vm = n_seg > 0 ? sum_vm / (float)n_seg : 0.0f;
    uint32_t sync = 0;
    for (uint32_t i = 0; i < n_seg; i++)
        if (fabsf((float)((double)V[i] - mean_vm)) < 10.0f) sync++;
    const float synchrony = n_seg > 0 ? (float)sync / (float)n_seg : 1.0f;
    char type_vm[512] = "";
    if (neurons && n_neurons > 0) {
        float sums[256] = {0};
        uint32_t counts[256] = {0};
        for (uint32_t q = 0; q < n_neurons; q++) {
            const uint8_t t = neurons[q].type;
            if (neurons[q].segment_count > 0 && neurons[q].soma_index < n_seg) {
                sums[t] = (float)((double)sums[t] + (double)V[neurons[q].soma_index]);
                counts[t]++;
            }
        }
        int pos = snprintf(type_vm, sizeof(type_vm), "\"type_vm\":{");
        bool first = true;
        for (int t = 0; t < 256 && pos < (int)sizeof(type_vm) - 20; t++) {
            if (!counts[t]) continue;
            if (!first) pos += snprintf(type_vm + pos, sizeof(type_vm) - pos, ",");
            pos += snprintf(type_vm + pos, sizeof(type_vm) - pos, "\"%d\":%.2f", t, sums[t] / (float)counts[t]);
            first = false;
        }
        snprintf(type_vm + pos, sizeof(type_vm) - pos, "}");
    }
    r->mean_vm = mean_vm;
    r->spike_count = spikes;
    r->synchrony = synchrony;
    r->tick = tick;
    snprintf(r->metrics_json, sizeof(r->metrics_json), "{\"mean_vm\":%.2f,\"spike_count\":%u,\"synchrony\":%.4f,\"tick\":%lu%s%s}",
             mean_vm, spikes, synchrony, (unsigned long)tick, type_vm[0] ? "," : "", type_vm);
}

}  // namespace
}  // namespace bnc

using namespace bnc;

extern "C" {

int bnc_sweep_parse_params(const char* json, const char* const* names, const uint8_t* name_ids, uint32_t n_names,
                           uint8_t* type_ids, float* values, uint32_t cap, uint32_t* n_out) {
    if (!json || !n_out || (cap && (!type_ids || !values))) { set_error("null argument"); return BNC_ERR_ARG; }
    uint32_t n = 0;
    const char* p = json;
    while (*p) {
        while (*p && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '{' || *p == '}' || *p == ','))
            p++;
        if (!*p) break;
        std::string key;
        if (*p == '"') {
            p++;
            while (*p && *p != '"') key += *p++;
            if (*p == '"') p++;
        } else {
            while (*p >= '0' && *p <= '9') key += *p++;
        }
        if (key.empty()) break;
        while (*p == ' ' || *p == '\t' || *p == ':') p++;
        if (!*p) break;
        char* end = nullptr;
        const float val = strtof(p, &end);
        if (end == p) break;
        p = end;
        uint32_t id = 0;
        bool found = false;
        if (key[0] >= '0' && key[0] <= '9') {
            id = (uint32_t)atoi(key.c_str());
            found = id < kModTypeCount;
        } else {
            // names in type-ID order, as the plugin table is searched
            uint32_t best = UINT32_MAX;
            for (uint32_t q = 0; q < n_names; q++)
                if (names && name_ids && names[q] && names[q][0] && name_matches(names[q], key) && name_ids[q] < best)
                    best = name_ids[q];
            if (best != UINT32_MAX) { id = best; found = true; }
        }
        if (!found || id >= kModTypeCount) continue;
        if (n < cap) { type_ids[n] = (uint8_t)id; values[n] = val; }
        n++;
    }
    *n_out = n;
    if (n > cap) { set_error("%u overrides, room for %u", n, cap); return BNC_ERR_ARG; }
    return BNC_OK;
}

int bnc_sweep_apply(BncBionData* net, const BncSweepTask* task) {
    if (!net || !task) { set_error("null argument"); return BNC_ERR_ARG; }
    if (task->n_overrides && (!task->type_ids || !task->values)) { set_error("null override arrays"); return BNC_ERR_ARG; }
    // parameter overrides: state[0] of each segment's first modifier of the type
    for (uint32_t o = 0; o < task->n_overrides; o++) {
        const uint8_t id = task->type_ids[o];
        for (uint32_t i = 0; i < net->num_segments; i++) {
            BncSegment& s = net->segments[i];
            for (int j = 0; j < BNC_MAX_MODIFIERS; j++) {
                if (s.modifiers[j].type == id && s.modifiers[j].type != 0) {
                    s.modifiers[j].state[0] = task->values[o];
                    break;
                }
            }
        }
    }
    // the seed's deterministic release-probability variation (daemon_main.cpp:199-206)
    if (task->seed != 0) {
        for (uint32_t k = 0; k < net->num_synapses; k++) {
            const uint32_t hash = task->seed ^ (net->synapses[k].id * 2654435761u);
            const float variation = (float)(hash & 0xFFFFu) / 65536.0f * 0.02f;
            net->synapses[k].release_probability *= (1.0f + variation);
        }
    }
    return BNC_OK;
}

int bnc_sweep_run(void* sim, const BncBionData* base, const BncCurrentStimulus* stim, uint32_t n_stim,
                  const BncSweepTask* tasks, uint32_t n_tasks, uint32_t ticks, float dt, uint32_t flags,
                  BncSweepResult* results) {
    if (!sim || !base || !tasks || !results || n_tasks == 0) { set_error("null argument or no tasks"); return BNC_ERR_ARG; }
    if (!(dt > 0.0f) || ticks == 0) { set_error("ticks and dt must be positive"); return BNC_ERR_ARG; }
    const uint32_t N = base->num_segments, K = base->num_synapses;
    // one modified copy of the segments and synapses per task; the rest is shared
    std::vector<std::vector<BncSegment>> segs(n_tasks);
    std::vector<std::vector<BncSynapse>> syns(n_tasks);
    std::vector<BncBionData> members(n_tasks);
    std::vector<const BncCurrentStimulus*> stim_ptr(n_tasks, stim);
    std::vector<uint32_t> stim_n(n_tasks, stim ? n_stim : 0u);
    for (uint32_t q = 0; q < n_tasks; q++) {
        segs[q].assign(base->segments, base->segments + N);
        syns[q].assign(base->synapses, base->synapses + K);
        members[q] = *base;
        members[q].segments = segs[q].data();
        members[q].synapses = syns[q].data();
        int rc = bnc_sweep_apply(&members[q], &tasks[q]);
        if (rc != BNC_OK) return rc;
    }
    int rc = bnc_load_ensemble_aos(sim, members.data(), stim_ptr.data(), stim_n.data(), n_tasks);
    if (rc != BNC_OK) return rc;
    // the batch mode advances its tick counter twice per tick; the daemon task once
    rc = backend_set_tick_stride(sim, (flags & BNC_SWEEP_SINGLE_TICK) ? 1u : 2u);
    if (rc != BNC_OK) return rc;
    rc = bnc_run_ticks_graph(sim, ticks, dt);
    backend_set_tick_stride(sim, 1u);   // later calls on the handle step the counter once per tick
    if (rc != BNC_OK) return rc;
    BncNetInfo info;
    rc = bnc_network_info(sim, &info);
    if (rc != BNC_OK) return rc;
    std::vector<float> V(info.n_segments);
    rc = bnc_read_segment_field(sim, 0, 0, V.data(), info.n_segments);
    if (rc != BNC_OK) return rc;
    const uint64_t tick = (uint64_t)ticks * ((flags & BNC_SWEEP_SINGLE_TICK) ? 1u : 2u);
    for (uint32_t q = 0; q < n_tasks; q++) {
        BncEnsembleMember m;
        rc = bnc_ensemble_member(sim, q, &m);
        if (rc != BNC_OK) return rc;
        member_metrics(V.data() + m.seg_begin, m.n_segments, base->neurons, base->num_neurons, tick, &results[q]);
    }
    return BNC_OK;
}

}  // extern "C"
