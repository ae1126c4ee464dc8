// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together
// with the reference's own src/simulation_host.cpp (included below from the
// reference checkout, not copied), so that the tests can call the reference's
// file-local release helpers directly:
//   * xorshift32_rnd (simulation_host.cpp:150-156), the release draw;
//   * the release seed exactly as core_run_tick_impl forms it from a synapse id,
//     the tick counter and the presynaptic V_m (simulation_host.cpp:438-440), with
//     the reference's operand types (uint32 id, uint64 tick, double V_m), so that
//     g++ evaluates the conversion of a negative V_m*1000 the way the reference's
//     build does.
#include "simulation_host.cpp"

extern "C" float ref_xorshift32_rnd(uint32_t seed) { return xorshift32_rnd(seed); }

extern "C" uint32_t ref_release_seed(uint32_t syn_id, uint64_t tick, double V_m) {
    Segment pre_seg;
    Segment* pre = &pre_seg;
    pre->V_m = V_m;
    return syn_id ^ ((uint32_t)tick) ^ ((uint32_t)(pre->V_m * 1000.0f));
}

// The release decision of core_run_tick_impl for one synapse given its release
// probability p (release_probability x ca_act x modulators).
extern "C" int ref_release_decision(uint32_t syn_id, uint64_t tick, double V_m, float p) {
    return xorshift32_rnd(ref_release_seed(syn_id, tick, V_m)) < p ? 1 : 0;
}

// rrp_apply_protein_mapping (kernel_dispatch.h:651-663) on a synapse whose other fields
// are zero: returns RRP_max, release_probability and RRP_recovery.
extern "C" void ref_protein_mapping(const float* protein_level, float* out3) {
    Synapse syn;
    memset(&syn, 0, sizeof(syn));
    rrp_apply_protein_mapping(&syn, protein_level);
    out3[0] = syn.RRP_max;
    out3[1] = syn.release_probability;
    out3[2] = syn.RRP_recovery;
}
