// hostnet.h -- compact host-side network, the builder's input.
//
// The reference's AoS records reserve room for 32 modifiers per segment and 8+8
// receptors per synapse (3216 B and 1568 B).  A 6.4M-segment, 10M-synapse network
// would need 36 GB of host memory in that layout; these records keep only the
// occupied modifier/receptor slots, with state in the precision the device keeps.
// Filled from AoS arrays (drop-in loads) or directly by the generator.
#pragma once
#include <sys/mman.h>

#include <cstdint>
#include <cstdlib>
#include <new>
#include <vector>

#include "common.h"
#include "par.h"

namespace bnc {

// Allocator of the compact network's arrays.  The loaders append records one at a
// time on one thread, so a plain vector takes its page faults one 4 KB page at a time
// on that thread (about 1 GB/s here, for some 10 GB at 6.4M segments).  This one asks
// for transparent huge pages and faults the pages in on all cores when the vector
// reserves them.
template <class T>
struct PrefaultAlloc {
    typedef T value_type;
    PrefaultAlloc() = default;
    template <class U>
    PrefaultAlloc(const PrefaultAlloc<U>&) {}
    T* allocate(size_t n) {
        const size_t kHuge = (size_t)2 << 20;
        const size_t bytes = n * sizeof(T);
        if (bytes < ((size_t)64 << 20)) {
            void* p = std::malloc(bytes ? bytes : 1);
            if (!p) throw std::bad_alloc();
            return static_cast<T*>(p);
        }
        const size_t len = (bytes + kHuge - 1) / kHuge * kHuge;
        void* p = std::aligned_alloc(kHuge, len);
        if (!p) throw std::bad_alloc();
        madvise(p, len, MADV_HUGEPAGE);   // a hint: without huge pages the touch below still runs on all cores
        char* c = static_cast<char*>(p);
        parallel_for(len / 4096, [c](size_t b, size_t e) {
            for (size_t i = b; i < e; i++) c[i * 4096] = 0;
        }, (size_t)1 << 14);
        return static_cast<T*>(p);
    }
    void deallocate(T* p, size_t) { std::free(p); }
    template <class U>
    bool operator==(const PrefaultAlloc<U>&) const { return true; }
    template <class U>
    bool operator!=(const PrefaultAlloc<U>&) const { return false; }
};
template <class T>
using HostVec = std::vector<T, PrefaultAlloc<T>>;

struct ModLite {
    uint8_t type;
    uint8_t active_vars;
    float density;
    float state[8];
};

struct SegLite {
    uint32_t id;
    uint8_t segment_type;
    uint8_t modifier_count;
    float radius, length;
    float pos_z;   // position.z (glial capture picks the nearest glial segment in z)
    float V_m;
    float intra_ions[7], extra_ions[7];
    float intra_nt[15], neurotransmitter[15];
    float ATP_level, temperature, transcription_signal;
    double I_buffer;
    uint64_t mod_off;
};

struct SynLite {
    uint32_t id, pre_segment, post_segment;
    uint8_t type, pre_autoreceptor_count, post_receptor_count, refractory;
    float weight, delay, pre_area, post_area, release_probability, release_amount, tau_clearance;
    float facilitation, depression, RRP, RRP_max, RRP_recovery;
    float bouton_Ca, spine_Ca, spine_camkii, spine_calcineurin;
    float cleft_neurotransmitter[15];
    uint64_t rec_off;   // post receptors, then pre autoreceptors, in HostNet::recs
};

struct HostNet {
    uint32_t num_segments = 0, num_connections = 0, num_synapses = 0;
    HostVec<SegLite> seg;
    HostVec<ModLite> mods;
    HostVec<BncIntraConnection> conn;
    HostVec<SynLite> syn;
    HostVec<ModLite> recs;
    // First segment whose modifier_count exceeded BNC_MAX_MODIFIERS (UINT32_MAX: none);
    // its modifier list is truncated here and the builder rejects the network.
    uint32_t bad_modifier_count_seg = UINT32_MAX;
    const ModLite& mod(uint32_t i, uint32_t j) const { return mods[seg[i].mod_off + j]; }
    const ModLite& post_rec(uint32_t k, uint32_t j) const { return recs[syn[k].rec_off + j]; }
    const ModLite& pre_ar(uint32_t k, uint32_t j) const {
        return recs[syn[k].rec_off + syn[k].post_receptor_count + j];
    }
};

// Static per-segment quantities and type predicates of the reference, as the builder
// computes them (run_tick_common.h:209-266, kernel_dispatch.h:283-309).
float host_seg_area(const SegLite& s);
double host_seg_volume(const SegLite& s);
float host_seg_capacitance(const HostNet& hn, uint32_t i);
bool host_is_myelin_blocked(uint8_t type);
bool host_is_ionotropic(uint8_t type);
uint8_t host_nt_from_receptor(uint8_t type);

void hostnet_add_segment(HostNet& hn, const BncSegment& s);
void hostnet_add_synapse(HostNet& hn, const BncSynapse& y);
void hostnet_from_aos(const BncBionData& aos, HostNet* hn);

}  // namespace bnc
