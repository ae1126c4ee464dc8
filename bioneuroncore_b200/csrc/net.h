// net.h -- the device-resident network: structure-of-arrays state, static
// geometry, tile/phase schedule and synapse CSR, plus the host-side maps needed
// to export back to the reference's AoS layout.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
#include "common.h"

namespace bnc {

// Launch geometry of the tile kernel (segments per tile, warps per tile).
constexpr int kTileWarps = 8;
constexpr int kTileThreads = kTileWarps * 32;
constexpr int kMaxTileSegs = 1024;

// Network-level flags.
enum : uint32_t {
    NF_DIFFUSION = 1u,      // any valid connection: step 2.5 runs (diffusion_kernel.h:118)
    NF_SYNAPSES = 2u,       // any synapse: step 3 resets neurotransmitter (simulation_host.cpp:328)
    NF_INTRA_NT = 4u,       // some intra_nt gradient exists: intracellular NT diffusion needed
    NF_TEMP = 8u,           // some temperature gradient exists
    NF_TXN = 16u,           // some transcription-signal gradient exists
    NF_PRE_EXT = 32u,       // synapses read presynaptic intracellular ions (RRP or bouton channels)
    NF_DELAY = 64u,         // some synapse has a transmission delay
    NF_NT_DIFFUSE_OUT = 128u, // neurotransmitter diffusion result is live (no synapses reset it)
};

// Per-segment flags.
enum : uint8_t { SF_MYELIN = 1u, SF_NMDA = 2u };

// The state a modifier reads and writes, gathered per segment for step 1 so that an
// item touches a few contiguous 32-byte runs instead of many scattered words:
// V and the 7 intra ions | 7 extra ions and ATP | area | volume and I_total
// (96 bytes, 16-aligned).  The GHK factors of V are recomputed per item: cheaper
// than moving them through HBM in every phase.
struct __align__(16) SegRec {
    float V;
    float in[7];
    float out[7];
    float atp;
    float area;
    uint32_t pad;
    double vol;
    double itot;
    double pad2;
};
static_assert(sizeof(SegRec) == 96, "SegRec layout");

// Plain-old-data descriptor passed by value to the kernels.
struct NetDev {
    uint32_t n_seg, n_tiles, n_items, n_phases, n_syn, n_rec, n_edges;
    uint32_t flags;
    uint32_t nt_used_mask;  // neurotransmitter indices that synapses/bath can make nonzero
    uint32_t user_mask[4];  // modifier IDs 0-127 run by registered device modifiers (plugins.cu)
    // segment state (device order, ion-major for the 7-ion arrays)
    float* V;
    float* ion_in;    // [7][n_seg]
    float* ion_out;   // [7][n_seg]
    float* intra_nt;  // [15][n_seg]
    float* nt;        // [15][n_seg]
    float* atp;
    float* temp;
    float* txn;
    double* ibuf;
    // segment statics
    float* radius;
    float* length;
    float* area;
    double* vol;
    float* cm;
    uint8_t* stype;
    uint8_t* sflags;
    float2* cav21_static;   // (density, state[1]) of the last Cav2.1 when it never updates
    float2* c21_cur;        // the same after step 1 of the current tick (k_modifiers -> k_diffusion)
    struct SegRec* rec;     // per-segment working record of step 1 (k_gather -> phases -> k_diffusion)
    float4* pre_rec;        // V, Ca_out, Cav2.1 density, Cav2.1 h  (after step 2.5)
    float4* pre_ext;        // Na_in, K_in, Ca_in, Na_out
    float* pre_ext2;        // K_out
    // tiles
    uint32_t* tile_seg_beg;   // [n_tiles+1] device segment offsets
    uint32_t* tile_edge_beg;  // [n_tiles+1]
    uint32_t* phase_off;      // [n_chunks*n_phases+1] item offsets of the (chunk, phase) buckets
    uint16_t* warp_seg;       // [n_tiles*(kTileWarps+1)] tile-local offsets
    uint16_t* warp_edge;      // [n_tiles*(kTileWarps+1)]
    // diffusion barrier groups (NetHost::diff_gm nonzero): per segment the tile-local
    // connection its thread handles (0xFFFF: none); null otherwise
    uint16_t* seg_edge;
    // edges (tile-grouped, tile-local endpoints)
    uint16_t* e_a;
    uint16_t* e_b;
    uint8_t* e_intra;
    float* e_area;
    float* e_dist;
    uint32_t* inc_off;        // [n_seg+1]
    uint16_t* inc;            // tile-local edge index | (endpoint-is-b << 15)
    // ghosts of tiles paired in a 2-CTA cluster (a component larger than one tile):
    // tile t's ghost g is device segment gh_seg[gh_off[t] + g], at tile-local index
    // n_own + g, owned by tile t ^ 1 at its local index gh_src[gh_off[t] + g]
    uint32_t* gh_off;         // [n_tiles+1]
    uint32_t* gh_seg;
    uint32_t* gh_src;
    // modifier items, by (phase, type, device segment)
    uint32_t* it_seg;         // device segment
    uint16_t* it_tf;          // type (8) | flags (8): bit0 non-default parameters, bit1 receptor override, av << 2
    float* it_den;
    float* it_st;             // [7][n_items]
    // current stimuli, per-segment CSR in stimulus order
    uint32_t* cs_off;         // [n_seg+1] (nullptr when none)
    float* cs_amp;
    float* cs_dur;
    unsigned long long* cs_start;
    uint8_t* cs_alive;
    // voltage clamps, per-segment CSR
    uint32_t* vc_off;         // (nullptr when none)
    float* vc_target;
    unsigned long long* vc_start;
    unsigned long long* vc_end;
    // ramp stimuli, per-segment CSR in upload order (simulation_host.cpp:261-276)
    uint32_t* rp_off;         // (nullptr when none)
    float* rp_from;           // start_pA
    float* rp_to;             // end_pA
    unsigned long long* rp_start;
    unsigned long long* rp_end;
    // one-shot ion and ligand injections in upload order: (device segment, what, amount
    // bits, 0); what = ion (0-6) | 8 extracellular ion, 16 + nt intra_nt, 32 + nt
    // neurotransmitter.  k_inject applies *inj_n of them and sets *inj_n to 0.
    uint4* inj;               // (nullptr when none is pending)
    uint32_t* inj_n;
    // synapse-kernel threads: segments with synapses by count descending, then the rest
    uint32_t* th_seg;         // [n_seg] device segment of thread t
    uint16_t* th_cnt;         // [n_seg] its synapse count
    uint32_t* w_off;          // [warps+1] first sliced synapse of each warp
    uint32_t* rw_off;         // [warps+1] first sliced receptor of each warp
    // synapses in sliced order (warp, k-th synapse of the lane, lane)
    uint32_t* sy_pre;         // device index of the presynaptic segment
    uint32_t* sy_id;
    float* sy_prel;
    float* sy_amt;
    float* sy_tauc;
    float* sy_delay;
    float* sy_pre_area;
    float* sy_post_area;
    float* sy_gK;
    float* sy_gNa;
    uint8_t* sy_refr;
    uint8_t* sy_flags;        // bit0 inhibitory, bits 4..7 released NT index
    float* sy_bouton;
    float* sy_spine;
    float* sy_camkii;
    float* sy_calcn;
    float* sy_facil;
    float* sy_weight;
    float* sy_cleft;          // cleft concentration of the released NT
    float* sy_rrp;
    float* sy_rrp_max;
    float* sy_rrp_rec;
    float* sy_scale;          // receptor density scale (1 reproduces the reference)
    uint8_t* rc_cnt;          // [n_syn] receptors of each synapse (receptors sliced likewise)
    uint8_t* rc_type;
    uint8_t* rc_av;
    float* rc_den;
    float* rc_st;             // [3][n_rec]
    unsigned long long* dl_arr;  // [4][n_syn]
    float* dl_amt;
    uint8_t* dl_nt;
    // Release modulators among the presynaptic autoreceptors (md_off null when the
    // network has none): those of sliced synapse k are [md_off[k], md_off[k + 1]), in
    // autoreceptor order.
    // Endocannabinoid signalling (null when the network has none): each synapse's eCB
    // cleft entry, and per device segment the item of its first eCB-synthesis modifier
    // (UINT32_MAX: none)
    float* sy_cleft_ecb;      // [n_syn]
    uint32_t* seg_ecb_item;   // [n_seg] (null when no segment has one)
    // Glia (gl_cap null when no segment has a GLAST transporter): the first 256 such
    // segments, each with the sliced synapses whose post segment is nearest to it in
    // z, in original synapse order; gl_cap holds each synapse's capture of the tick
    // Gap junctions (sy_gj null when the network has none): per entry of the synapse
    // kernel the junction it is a side of (bit 31: the pre side), UINT32_MAX for a
    // chemical synapse; per junction its segments, delay (the filter's time constant),
    // slow gate and filtered current as the tick began (gj_dep, gj_flt) and as the
    // post side leaves them (gj_dep_new, gj_flt_new, copied back after step 3); per
    // segment the items of its connexin-36 and connexin-43 ([2][n_seg], UINT32_MAX)
    uint32_t* sy_gj;
    uint32_t* gj_pre;
    uint32_t* gj_post;
    float* gj_delay;
    float* gj_dep;
    float* gj_dep_new;
    float* gj_flt;
    float* gj_flt_new;
    uint32_t* seg_cx;
    uint32_t n_gj;
    float* gl_cap;            // [n_syn]
    uint32_t* gl_seg;         // [n_glia] device segment
    uint32_t* gl_off;         // [n_glia + 1]
    uint32_t* gl_syn;         // sliced synapse indices
    uint32_t n_glia;
    uint32_t model_extras;    // 1: some item is eCB synthesis, GLAST or a connexin (86, 147, 114, 198)
    uint32_t syn_extras;      // 1: release modulators, eCB, glia or gap junctions (the fused synapse kernel)
    uint32_t* md_off;         // [n_syn + 1]
    uint8_t* md_code;         // kind << 4 | cleft NT index; kind 1 Gi/o, 2 Gs, 3 ionotropic
    double* md_scale;         // density x effective area (pre_area, or 1 when not positive)
    float* md_st;             // state[0]
    uint32_t n_md;
    uint32_t* spike_count;    // [n_seg]
    int* err_flag;            // device-side error report (0 = ok)
    // Captured tick loops: when set, the kernels take the tick from clock[0] and the
    // first-tick flag from clock[1] == 0 (ticks run so far) instead of their launch
    // parameters, and k_advance_clock moves both on after each tick.
    unsigned long long* clock;
    // Release log (null: off).  Every transmitter amount that enters a synaptic cleft
    // -- a delayed arrival (slot 0-3) or an immediate release (slot 4) -- is appended
    // as {device synapse, tick (low 32 bits), amount bits, slot}; entries past ev_cap
    // are counted but not written.
    uint4* ev_buf;
    uint32_t* ev_n;
    uint32_t ev_cap;
    // Electrodiffusion options (bnc_set_diffusion_mode).  diff_mode bit 0: the Jacobi
    // solves iterate in FP64 until no value of a convergence group changes by more than
    // jac_tol in a sweep (at most jac_max sweeps) instead of the reference's fixed 50;
    // bit 1: the per-ion FP64 ledger of step 2.5 is kept.
    uint32_t diff_mode;
    uint32_t jac_max;
    double jac_tol;
    uint16_t* seg_grp;        // [n_seg] convergence group (connected component) within the
                              // tile or tile pair, bit 15: the group's first segment
    uint32_t* jac_stats;      // [4] max V sweeps, max phi sweeps, V and phi group solves at the cap
    double* ledger;           // [14] per ion: FP32 rounding of the Nernst-Planck updates, bath exchange
};

// How components are grouped: a warp group holds components until their segments
// would exceed warp_cap (a larger component gets a warp group to itself), and a tile
// holds up to kTileWarps warp groups and at most tile_segs segments.  The grouping
// changes which CTA and warp handle a segment, never the arithmetic.
struct BuildOptions {
    uint32_t warp_cap = 64;
    uint32_t tile_segs = kMaxTileSegs;
    // Modifier phases: the greedy type-uniform schedule is kept while it needs at most
    // phase_cap phases (0: 2 x the longest active-modifier list + 4), else slot order.
    uint32_t phase_cap = 0;
    // Segments per chunk of the modifier pass (0: the whole network in one chunk).
    // All phases of a chunk run before the next chunk, so a chunk's step-1 records
    // (96 bytes per segment) can stay in L2 between phases.
    uint32_t chunk_segs = BNC_DEFAULT_CHUNK_SEGS;
    // Modifier phases per launch (1: one launch per phase).  Applies to slot-order
    // schedules in one chunk without registered device modifiers; up to kMaxFuse.
    // 6.4M-segment large set, step 1 per tick: 1 phase 7.8 ms; at 3.2M segments
    // 1: 3.94, 2: 2.89, 3: 2.40, 4: 2.15, 6: 2.43, 9: 4.97, 17: 19.5 ms (deeper groups
    // diverge: rows sorted by their items' types share fewer types further down).
    uint32_t fuse_phases = 4;
    // Lower fuse_phases while the rows sorted for its groups leave warps on more than
    // kMaxWarpTypes distinct models per item on average (an explicit fuse_phases option
    // turns this off).
    bool fuse_adaptive = true;
    // Diffusion barriers over aligned thread groups where the tile allows (false: always
    // the whole CTA).
    bool group_barriers = true;
};
constexpr uint32_t kMaxFuse = 32;
// Distinct channel models a warp may run per item of a phase group, on average over
// the group's warps and items, before a shallower group is preferred.  Large set,
// 640k segments: slots listed by type ID give 1.05 at 4 phases per group; slots in
// draw order 1.21 at 3 and 3.36 at 4, where step 1 took 3.0x longer at 6.4M segments
// (16.1 against 5.5 ms per tick: instruction-cache misses, 12 of 32 lanes active).
constexpr double kMaxWarpTypes = 1.3;
// Below this many segments a modifier launch is a few microseconds of work, its count
// matters more than divergence, and the requested depth is kept.
constexpr uint32_t kAdaptiveFuseMinSegs = 1u << 16;

// Host copy of everything the exporter needs to map device state back.
struct NetHost {
    uint32_t n_seg = 0, n_conn = 0, n_syn_total = 0;
    std::vector<uint32_t> perm;      // device index -> original segment index
    std::vector<uint32_t> inv;       // original segment index -> device index
    std::vector<uint32_t> item_seg;  // item -> original segment index
    std::vector<uint8_t> item_slot;  // item -> modifier slot
    std::vector<uint32_t> syn_orig;  // device synapse -> original synapse index
    std::vector<uint32_t> rec_syn;   // device receptor -> device synapse
    std::vector<uint8_t> rec_slot;   // device receptor -> receptor slot
    std::vector<uint8_t> syn_nt;     // released NT per device synapse
    std::vector<uint32_t> md_syn;    // release modulator -> original synapse index
    std::vector<uint8_t> md_slot;    // release modulator -> autoreceptor slot
    std::vector<uint32_t> gj_syn;    // gap junction -> original synapse index
    uint32_t max_tile_segs = 0, max_tile_edges = 0;
    uint32_t max_tile_stride = 0;            // own + ghost segments of the largest tile
    uint32_t cluster = 1;                    // CTAs per diffusion cluster (2: tiles in pairs)
    uint32_t diff_threads = 32;              // threads per diffusion CTA
    uint32_t diff_gm = 0;                    // diffusion barrier groups: 0 (CTA), 32 or 64 threads
    uint32_t group_tiles_32 = 0, group_tiles_64 = 0;   // tiles with warp / 64-thread barrier groups
    std::vector<uint32_t> phase_off;         // item range of each (chunk, phase) bucket (host copy)
    uint32_t chunk_segs = 0, n_chunks = 1;   // modifier-pass chunks of consecutive segments
    uint32_t fuse = 1;                       // modifier phases per launch (item order follows)
    double warp_models = 1.0;                // mean distinct models per warp and item of a group
    uint8_t item_dyn_rows = 0;               // state words (bits) any item updates: the rows exported
    struct UserRange { uint32_t bucket, type, begin, end; const void* kernel; };
    std::vector<UserRange> user_ranges;      // registered device modifiers' items, per bucket
    size_t smem_bytes = 0;
    BuildOptions opt;                        // grouping the network was built with
    double algo_bytes_per_tick = 0;  // algorithmic HBM bytes per tick of this state schema
    double seg_bytes = 0, syn_bytes = 0;     // split by owner: segment state vs synapse state
    double tile_bytes = 0, synk_bytes = 0;   // tick figure split by step: 1 + 2.5 vs 3 + 4
    double mod_bytes = 0, diff_bytes = 0;    // per launch of k_modifiers / k_diffusion
    bool perm_identity = true;               // device segment order equals the original order
    bool stim_identity = true;               // per-segment stimulus CSR order equals upload order
};

struct Stimuli {
    std::vector<BncCurrentStimulus> current;
    std::vector<BncVoltageClamp> vclamp;
    std::vector<BncRampStimulus> ramp;
    std::vector<BncIonInjection> ion_inj;       // one-shot: cleared once uploaded to the device
    std::vector<BncLigandInjection> lig_inj;
};

// Builds host-side SoA from AoS and uploads it.  Returns 0 or BNC_ERR_*; on error
// bnc_last_error() explains.  `dev` receives device pointers (owned by `allocs`).
struct DeviceAllocs {
    std::vector<void*> ptrs;
    ~DeviceAllocs();
    void* alloc(size_t bytes);
    void release();
};

struct HostNet;
int build_network(const HostNet& hn, const Stimuli& stim, NetDev* dev, NetHost* host,
                  DeviceAllocs* allocs, const BuildOptions& opt = BuildOptions());

// Rebuilds the per-segment stimulus CSRs after an upload of new stimuli.
int upload_stimuli(const Stimuli& stim, NetHost& host, NetDev* dev, DeviceAllocs* allocs);

// Writes device state back into the AoS arrays.
int export_network(const NetDev& dev, const NetHost& host, uint64_t ticks_run, BncBionData* aos);
// State words (bits) a built-in modifier type updates every tick; 0 for other types.
uint8_t host_dyn_mask(uint8_t type);
// State words (bits) a built-in type reads as parameters (its default when 0).
uint8_t param_mask(uint8_t type);
// Receptor types the synapse and modifier kernels implement (AMPA, NMDA, GABA-A, glycine).
bool host_receptor_supported(uint8_t type);
// The bouton channel conductance (pS) an autoreceptor of this type adds (0: none).
float host_bouton_gamma(uint8_t type);

// The segment state and the modifier items in device order, gathered on the device
// from the host records (convert.cu): perm maps device to original segments, inv the
// reverse; item q belongs to original segment item_seg[q], slot item_slot[q].  Sets
// *bad_item to the lowest item whose receptor override (active_vars) is out of range.
int device_convert_state(const HostNet& hn, const std::vector<uint32_t>& perm, const std::vector<uint32_t>& inv,
                         const std::vector<uint32_t>& item_seg, const std::vector<uint8_t>& item_slot, NetDev* dev,
                         DeviceAllocs* allocs, uint32_t* bad_item);
// The synapse and receptor arrays in device order, gathered on the device (convert.cu):
// device synapse q is original synapse syn_orig[q]; device receptor r is slot
// rec_slot[r] of device synapse rec_syn[r].
int device_convert_synapses(const HostNet& hn, const std::vector<uint32_t>& syn_orig,
                            const std::vector<uint32_t>& inv, const std::vector<uint32_t>& rec_syn,
                            const std::vector<uint8_t>& rec_slot, NetDev* dev, DeviceAllocs* allocs);

// Kernel launchers (tile.cu, synapse.cu).  prepare_tick does the per-device and
// per-network set-up that must not happen inside a stream capture (constant tables,
// the tile kernel's shared-memory limit); enqueue_tick only enqueues kernels.
cudaError_t prepare_tick(const NetDev& dev, const NetHost& host, cudaStream_t stream);
cudaError_t enqueue_tick(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick, int first_tick,
                         cudaStream_t stream);
cudaError_t launch_tick(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick, int first_tick,
                        cudaStream_t stream);
// the three kernels of a tick, one at a time (profiling)
// Launches step 1 makes per tick (k_gather per chunk, phase or phase-group launches,
// registered device modifiers), as enqueue_modifiers issues them.
uint32_t modifier_launches(const NetDev& dev, const NetHost& host);
uint32_t synapse_launches(const NetDev& dev);
cudaError_t launch_modifiers(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                             cudaStream_t stream);
cudaError_t launch_diffusion(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                             cudaStream_t stream);
cudaError_t launch_synapse(const NetDev& dev, float dt, unsigned long long tick, int first_tick,
                           cudaStream_t stream);
cudaError_t launch_set_clock(unsigned long long* clock, unsigned long long tick, unsigned long long ticks_run,
                             cudaStream_t stream);
cudaError_t launch_advance_clock(unsigned long long* clock, cudaStream_t stream);
// plugins.cu: registered device modifiers (user modifier IDs 0-127)
bool device_modifier_registered(uint8_t type);
// A host plugin registered a CPU function for the ID (plugin_host.cpp).
bool host_plugin_registered(uint8_t type);
int device_modifier_kernel(uint8_t type, const void** kernel);   // loads on first use (needs a device)
cudaError_t launch_device_modifier(const void* kernel, const NetDev& d, uint8_t type, uint32_t b, uint32_t e, float dt,
                                   cudaStream_t stream);
// synapse.cu: per-device receptor constants (outside stream capture)
cudaError_t prepare_synapse(cudaStream_t stream);
// backend.cu: what the adjoint (adjoint.cu) takes from a loaded backend
struct HostNet;
int backend_export_host(void* sim, HostNet* hn, std::vector<BncCurrentStimulus>* stim, uint64_t* tick,
                        int* device, uint32_t* n_vclamp);
// Steps the tick counter by `stride` per tick (1: the reference tick; 2: its batch mode,
// daemon_main.cpp:250-258, which increments the counter once more after each tick).
int backend_set_tick_stride(void* sim, uint32_t stride);
// Runs `ticks` plain ticks with the release log on; returns each cleft entry as
// (original synapse index, tick, amount, slot) in the order the kernel wrote them.
int backend_record_releases(void* sim, uint32_t ticks, float dt, std::vector<uint32_t>* syn,
                            std::vector<uint64_t>* tick, std::vector<float>* amt, std::vector<uint8_t>* slot);
// diffuse.cu
cudaError_t prepare_diffusion(const NetHost& host, cudaStream_t stream);
cudaError_t enqueue_diffusion(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                              cudaStream_t stream);
size_t diffusion_smem_bytes(uint32_t max_segs, uint32_t max_edges);

}  // namespace bnc
