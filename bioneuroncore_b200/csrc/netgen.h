// netgen.h -- seeded synthetic network generator for the five workload families
// (small plain network, 6.4M-segment plain network, electrodiffusion trees,
// uneven ensembles, adjoint fitting network).
//
// The generator streams segments, intra-connections and synapses into a sink, so
// the same routine can fill reference-layout AoS arrays (for the CPU reference and
// the oracle) or feed the device builder directly without materialising 36 GB of
// AoS for the 6.4M-segment network.
#pragma once
#include <cstdint>
#include <vector>
#include "bnc_abi.h"
#include "bnc_b200.h"

namespace bnc {

struct NetSink {
    virtual ~NetSink() {}
    // Called once before any element with the exact totals.
    virtual void begin(uint32_t n_neurons, uint32_t n_segments, uint32_t n_connections,
                       uint64_t n_synapses, uint32_t n_stimuli) = 0;
    virtual void neuron(const BncNeuron& n) = 0;
    virtual void segment(const BncSegment& s) = 0;
    virtual void connection(const BncIntraConnection& c) = 0;
    virtual void synapse(const BncSynapse& s) = 0;
    virtual void stimulus(const BncCurrentStimulus& st) = 0;
    virtual void end() {}
};

// Resolved sizes of a generated network (filled before streaming).
struct NetShape {
    uint32_t n_neurons = 0;
    uint32_t n_segments = 0;
    uint32_t n_connections = 0;
    uint64_t n_synapses = 0;
    uint32_t n_stimuli = 0;
};

// Fills `shape` and streams the network into `sink`.  Returns 0 or a negative
// BNC_ERR_* code for an invalid parameter set.
int generate_network(const BncNetgenParams& p, NetSink& sink, NetShape* shape);

}  // namespace bnc
