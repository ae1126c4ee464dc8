/*
 * bnc_b200.h -- C ABI of the B200 backend for BioNeuronCore's per-tick loop.
 *
 * Two groups of entry points:
 *
 * 1. The drop-in set.  Same names, signatures and error conventions as the
 *    reference CUDA backend's `extern "C"` block (src/gpu_backend_cuda.cu:316-390;
 *    the set a loader must find is listed in tests/smoke_cuda.sh:24-29).  A caller
 *    that dlopen()s the reference's libbiocore_gpu_backend_cuda.so can dlopen
 *    this library instead.
 *
 * 2. New entry points (prefix bnc_) for what the reference has no call for:
 *    multi-tick runs without a host round trip, field reads of the device
 *    structure-of-arrays, the synthetic generator, ensembles and the adjoint.
 *
 * Handles are opaque `void*` as in the reference.  Functions returning int use
 * 0 for success and a negative BNC_ERR_* code otherwise; bnc_last_error()
 * returns a message for the most recent failure on the calling thread.
 */
#ifndef BNC_B200_H
#define BNC_B200_H

#include <stdint.h>
#include <stddef.h>
#include "bnc_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* .bion loader codes: the reference's BION_ERR_* values (src/bion_loader_host.cpp:13-24),
 * so gpu_backend_load_bion fails with the same numbers as the reference backend. */
#define BNC_OK 0
#define BNC_BION_ERR_FILE_OPEN -1
#define BNC_BION_ERR_BAD_MAGIC -2
#define BNC_BION_ERR_BAD_VERSION -3
#define BNC_BION_ERR_ZERO_SEGS -4
#define BNC_ERR_ALLOC -5
#define BNC_BION_ERR_BAD_CONN -6
#define BNC_BION_ERR_BAD_SYNAPSE -7
#define BNC_BION_ERR_BAD_NEURON -8
#define BNC_ERR_FORMAT -9
#define BNC_BION_ERR_WRITE_FAIL -10
#define BNC_BION_ERR_FILE_READ -11
/* backend codes */
#define BNC_ERR_ARG -20
#define BNC_ERR_UNSUPPORTED -21
#define BNC_ERR_CUDA -22
#define BNC_ERR_STATE -23
#define BNC_ERR_DEVICE_TIMEOUT -24

/* ------------------------------------------------------------------ */
/* 1. drop-in set (reference src/gpu_backend_cuda.cu:316-390)          */
/* ------------------------------------------------------------------ */

/* Replaces gpu_backend_create (gpu_backend_cuda.cu:325-327): backend on device 0;
 * NULL when no CUDA device exists. */
void* gpu_backend_create(void);
/* Replaces gpu_backend_create_on_device (gpu_backend_cuda.cu:316-323); an
 * out-of-range index falls back to device 0 as in the reference. */
void* gpu_backend_create_on_device(int device_index);
/* Replaces gpu_backend_destroy (gpu_backend_cuda.cu:329-331). */
void gpu_backend_destroy(void* sim);
/* Replaces gpu_backend_load_bion (gpu_backend_cuda.cu:333-336): loads a .bion
 * file of any version the reference reads (3-14, with its migrations,
 * bion_loader_host.cpp:26-428, bion_format.h:59-340).  A file without nucleus
 * records gets one default nucleus per neuron, as the reference's loader creates
 * them; the nucleus protein levels are mapped onto each synapse's RRP_max, release
 * probability and RRP recovery as the reference's backend does every tick
 * (gpu_backend_cuda.cu:275-289), so with default nuclei every synapse whose id is not
 * 0 takes 10, 0.3 and 0.02.  0 on success, the reference's BION_ERR_* codes on file
 * errors, BNC_ERR_UNSUPPORTED when the network uses something the device path does
 * not implement (message in bnc_last_error). */
int gpu_backend_load_bion(void* sim, const char* filename);
/* Replaces gpu_backend_run_tick (gpu_backend_cuda.cu:338-341): one tick of dt
 * ms; afterwards the AoS view returned by gpu_backend_bion_data is coherent
 * (the reference synchronises every tick, gpu_backend_cuda.cu:308). */
void gpu_backend_run_tick(void* sim, float dt);
/* Replaces gpu_backend_bion_data (gpu_backend_cuda.cu:343-346): host AoS view
 * (BncBionData*, layout of reference include/bion_loader.h:16-28). */
void* gpu_backend_bion_data(void* sim);
/* Replaces gpu_backend_upload_stimuli (gpu_backend_cuda.cu:348-351).  Every list of
 * `src` replaces the previous one (at most 256 entries each; `current_tick` is ignored,
 * the tick counter is internal).  Current steps, clamps and ramps follow the CPU tick
 * (simulation_host.cpp:189-276, 633-643); ion and ligand injections apply once, at the
 * next tick, after the segment's modifier currents (:279-306).  Returns nothing, as the
 * reference's does: bnc_last_error() is empty after a successful upload. */
void gpu_backend_upload_stimuli(void* sim, const BncGpuStimulusData* src);
/* Replaces gpu_backend_device_count (gpu_backend_cuda.cu:353-357). */
int gpu_backend_device_count(void);
/* Replaces gpu_backend_get_device_info (gpu_backend_cuda.cu:359-380). */
int gpu_backend_get_device_info(int index, BncGpuDeviceInfo* info);
/* Replace the ABI probes gpu_backend_ibuf_offset/vm_offset/seg_size
 * (gpu_backend_cuda.cu:384-386). */
int gpu_backend_ibuf_offset(void);
int gpu_backend_vm_offset(void);
int gpu_backend_seg_size(void);

/* ------------------------------------------------------------------ */
/* 2. new entry points                                                 */
/* ------------------------------------------------------------------ */

/* Synthetic workload families (seeded). */
#define BNC_NET_SMALL 1        /* 64 x 32-segment neurons, 6 modifiers, 400 synapses */
#define BNC_NET_LARGE 2        /* 100k x 64-segment neurons, 16 of 24 types, 10M synapses */
#define BNC_NET_TREES 3        /* depth-10 binary dendritic trees, electrodiffusion */
#define BNC_NET_ENSEMBLE_MEMBER 4 /* one network of an uneven ensemble */
#define BNC_NET_ADJOINT 5      /* 256 x 64-segment neurons, 2000 synapses; Nav, Kv_DR, K2P (+ myelin, Cav2.1; Cav1.3 and the pump with BNC_NETGEN_FULL_SMALL_SET); 1 nA steps */

typedef struct {
    uint32_t family;          /* BNC_NET_* */
    uint32_t n_neurons;       /* 0: family default */
    uint64_t n_synapses;      /* 0: family default, scaled with n_neurons */
    uint64_t seed;
    uint32_t segs_per_neuron; /* 0: family default (ignored for trees) */
    uint32_t tree_depth;      /* trees only; 0: 10 */
    float conductance_scale[4]; /* gNa, gK, gleak, gCa multipliers (0 = 1.0) */
    uint32_t flags;           /* BNC_NETGEN_* */
    float stim_pA;            /* 0: family default */
    float stim_duration_ms;   /* 0: whole run (1e9 ms) */
} BncNetgenParams;

#define BNC_NETGEN_NO_SYNAPSES 1u
#define BNC_NETGEN_NO_CONNECTIONS 2u
#define BNC_NETGEN_NO_STIMULI 4u
#define BNC_NETGEN_PERTURB_IONS 8u
#define BNC_NETGEN_DRAW_ORDER 16u   /* large set: keep modifiers in draw order (default: by type ID) */
/* Synapses also exercise the presynaptic machinery: about 30% each get a readily
 * releasable pool (RRP_max 25, recovery 0.01), a presynaptic autoreceptor channel
 * (Kv delayed rectifier 123 or Nav1.6 141 on the bouton) and a transmission delay
 * of 0.5-2 ms (drawn from a stream of their own: other draws are unchanged). */
#define BNC_NETGEN_SYNAPSE_EXTRAS 32u
/* The fitting family (BNC_NET_ADJOINT) with the whole small set: Cav1.3 and the Na/K
 * pump on every segment as well, beside the three fitted conductances. */
#define BNC_NETGEN_FULL_SMALL_SET 64u
/* Synapses with an odd index take a glycine receptor (transmitter glycine) as their
 * first receptor instead of AMPA or GABA-A; other draws are unchanged. */
#define BNC_NETGEN_GLYCINE 128u
/* About half the synapses also get one or two presynaptic release-modulator
 * autoreceptors (Gi/o, Gs and ionotropic types: 5-HT1A/1B, D1, D2, A1, A2A, mGluR2/3,
 * alpha2, CB1, H3, nicotinic), density 0.2-1, state[0] 0-0.5, after any bouton
 * channel (drawn from a stream of their own: other draws are unchanged). */
#define BNC_NETGEN_RELEASE_MODULATORS 256u
/* Endocannabinoid retrograde signalling: an eCB-synthesis modifier (86, density 1,
 * state[0] 0.5) on every soma and dendrite segment, and a CB1 release modulator on
 * about half the synapses (from the release-modulator stream). */
#define BNC_NETGEN_ECB 512u
/* Glia: a GLAST glutamate transporter (147) on every fourth axon segment, which makes
 * it a glial segment that takes up transmitter from the clefts nearest to it in z;
 * segments get spread z positions (neuron-dependent offsets). */
#define BNC_NETGEN_GLIA 1024u
/* Gap junctions: electrical synapses (alternately type 1 and 2, every third with a
 * 0.5 ms delay) from the soma of each neuron to the next one's, spread through the
 * chemical synapses in the synapse order; connexin-36 (114) on every soma and
 * connexin-43 (198) on every other one. */
#define BNC_NETGEN_GAP_JUNCTIONS 2048u
/* Synapses whose first receptor is AMPA also get an NMDA receptor (9) as their next
 * one: density 200, CDI gate (state[2]) 1; other draws are unchanged. */
#define BNC_NETGEN_NMDA 4096u

/* Generates a network into host AoS arrays in the reference layout.  The arrays
 * are owned by the library; release with bnc_netgen_free.  *stim receives the
 * current stimuli (may be NULL when none). */
int bnc_netgen_aos(const BncNetgenParams* p, BncBionData* out,
                   BncCurrentStimulus** stim, uint32_t* n_stim);
void bnc_netgen_free(BncBionData* data, BncCurrentStimulus* stim);

/* Loads a network from host AoS arrays in the reference layout (copied; the
 * backend keeps its own AoS for gpu_backend_bion_data).  `stim` may be NULL. */
int bnc_load_aos(void* sim, const BncBionData* data, const BncCurrentStimulus* stim, uint32_t n_stim);

/* Generates a network and builds it on the device without keeping a host AoS
 * copy (gpu_backend_bion_data then returns NULL); for networks too large for it. */
int bnc_load_generated(void* sim, const BncNetgenParams* p);

/* Runs n ticks of dt ms on the device without refreshing the host AoS view. */
int bnc_run_ticks(void* sim, uint32_t n_ticks, float dt);

/* No counterpart in the reference.  Same ticks and results as bnc_run_ticks, for
 * callers that cannot call cudaMalloc while they drive the simulation: a host
 * whose own pool allocator has reserved the device memory and treats any other
 * allocation as an error, or a control loop that cannot afford the device-wide
 * synchronisation a cudaFree brings.  Each tick the diffusion kernel hands the
 * synapse kernel a per-segment record of the presynaptic state (36 bytes per segment);
 * here that scratch is a fixed array inside the library instead of buffers of the
 * network, and the call allocates nothing.
 *   - Limit: networks of at most BNC_STATIC_SCRATCH_MAX_SEGMENTS segments (the
 *     array is 4.5 MiB on every GPU that loads the library, held until exit);
 *     larger networks are rejected with BNC_ERR_ARG.
 *   - The first call on a device looks up the array's device address (one
 *     runtime query, no allocation); make that first call before any stream
 *     capture.
 *   - All calls on a device share the one array.  Each call clears the part it
 *     uses before its first tick, but calls that overlap on the GPU (two handles
 *     on one device, different streams, different host threads) race on it:
 *     serialise them. */
#define BNC_STATIC_SCRATCH_MAX_SEGMENTS 131072u
int bnc_run_ticks_static_scratch(void* sim, uint32_t n_ticks, float dt);

/* Runs n ticks bracketed by CUDA events on the backend's stream; *ms receives the
 * elapsed device time. */
int bnc_time_ticks(void* sim, uint32_t n_ticks, float dt, float* ms);

/* One serving step: uploads per-stimulus amplitudes (pA, one per loaded current
 * stimulus, host memory -- pinned for an asynchronous copy), runs one tick and
 * copies V_m of every segment into v_out (host, original order).  Either buffer
 * may be NULL to skip that copy. */
int bnc_step_io(void* sim, float dt, const float* stim_amp, uint32_t n_amp, float* v_out, uint32_t n_v);

/* Runs n ticks with CUDA events around each kernel; returns the summed device
 * time of the modifier kernel (step 1), the electrodiffusion kernel (step 2.5)
 * and the synapse + membrane kernel (steps 3 and 4). */
int bnc_profile_ticks(void* sim, uint32_t n_ticks, float dt, float* ms_modifiers, float* ms_diffusion,
                      float* ms_synapse);

/* Copies device state into the host AoS view (no-op when none is held). */
int bnc_sync_to_host(void* sim);
/* 1 when the handle's Segment/Synapse records (gpu_backend_bion_data) live in managed
 * memory and are written on the device after each tick, as the reference's backend
 * keeps them (bion_loader.cpp:634); 0 when they are host memory updated by a host
 * export (devices without concurrent managed access) or there are none. */
int bnc_records_managed(void* sim);
/* Where the drop-in records live between ticks.  on_host = 0 (the default where the
 * device supports concurrent managed access, as the reference's backend keeps them):
 * managed memory resident on the device, written there after each tick; a host read
 * migrates the pages it touches, and the next tick brings them back.  on_host = 1:
 * plain host memory, updated after each tick by copying the changing state to the
 * host and scattering it into the records on all host cores; for callers that read
 * every record every tick.  A switch moves the records: the segments and synapses
 * pointers of gpu_backend_bion_data change, and pointers taken before are invalid.
 * BNC_ERR_STATE when the handle has no drop-in records. */
int bnc_set_records_residency(void* sim, int on_host);

/* Field reads in original segment / synapse order (host float arrays of n).
 * Segment fields: 0 V_m, 1 intra ion[index], 2 extra ion[index], 3 ATP,
 *   4 temperature, 5 transcription, 6 intra_nt[index], 7 neurotransmitter[index],
 *   8 modifier state (index = slot*8 + k), 9 spike count (V crossing -40 mV upward).
 * Synapse fields: 0 bouton_Ca, 1 spine_Ca, 2 weight, 3 refractory,
 *   4 cleft_neurotransmitter[index] (a gap junction's entry 0: its filtered current),
 *   5 receptor state (index = j*8 + k), 6 facilitation, 7 spine_camkii,
 *   8 spine_calcineurin, 9 RRP, 10 depression (a gap junction's slow gate),
 *   11 autoreceptor state (index = j*8, word 0 of release modulators). */
int bnc_read_segment_field(void* sim, int field, int index, float* out, uint32_t n);
int bnc_read_synapse_field(void* sim, int field, int index, float* out, uint32_t n);

/* Per-synapse multiplicative scale of the receptor density (the differentiable
 * synaptic weight; 1.0 everywhere reproduces the reference). */
int bnc_set_synapse_scale(void* sim, const float* scale, uint32_t n);

typedef struct {
    uint32_t n_segments, n_connections, n_synapses, n_tiles, n_items, n_phases, n_receptors;
    uint32_t max_tile_segs, max_tile_edges, smem_bytes, flags;
    uint64_t ticks;
    double algo_bytes_per_tick;   /* algorithmic HBM bytes one tick moves (state schema) */
    double seg_bytes_per_tick, syn_bytes_per_tick;          /* split by state owner */
    double tile_bytes_per_tick, synapse_kernel_bytes_per_tick; /* split: steps 1 + 2.5 / steps 3 + 4 */
    uint32_t warp_cap, tile_segs;  /* grouping the network was built with */
    double modifier_kernel_bytes, diffusion_kernel_bytes;  /* per launch of each (state round trip included) */
    uint32_t modifier_launches;   /* launches of step 1 per tick: k_gather, phase launches, device modifiers */
    uint32_t fuse_phases;         /* modifier phases per launch the network runs with */
    uint32_t group_tiles_32, group_tiles_64;  /* tiles whose diffusion barriers span one warp / 64 threads */
    uint32_t diffusion_threads;   /* threads per diffusion CTA */
    uint32_t synapse_launches;    /* launches of steps 3-4 per tick: k_release (networks without release
                                     modulators, eCB, glia or gap junctions), k_synapse, k_glia, k_gj_commit */
} BncNetInfo;
int bnc_network_info(void* sim, BncNetInfo* info);

/* Host-only: generates a network and runs the builder's planning (tiles, phase
 * schedule, CSRs) without a device; fills `info` (no upload, no CUDA call). */
int bnc_plan_generated(const BncNetgenParams* p, BncNetInfo* info);

/* ---- Batched ensembles: many independent networks in one device structure ----
 * Members are concatenated in the given order (segments, connections, synapses
 * and stimuli keep their order inside each member, indices offset by the member's
 * first segment) and run by the same two kernels per tick: one launch covers every
 * member.  Each member keeps its own synapse ids, so its release stream is the one
 * it has when run alone, and every member's state evolves exactly as in a separate
 * run.  The reference has no such call: it runs parameter sweeps as separate
 * processes (src/daemon_server.cpp:1164-1290).  Members must agree on whether they
 * have intra-connections and on whether they have synapses (network-wide switches
 * of the reference tick); BNC_ERR_UNSUPPORTED otherwise.  Segment and synapse
 * fields of a member are the ranges bnc_ensemble_member reports within the
 * bnc_read_*_field arrays. */
typedef struct {
    uint32_t seg_begin, n_segments;
    uint32_t syn_begin, n_synapses;
    uint32_t stim_begin, n_stimuli;
} BncEnsembleMember;
int bnc_load_ensemble_generated(void* sim, const BncNetgenParams* members, uint32_t n_members);
int bnc_load_ensemble_aos(void* sim, const BncBionData* members, const BncCurrentStimulus* const* stim,
                          const uint32_t* n_stim, uint32_t n_members);
int bnc_ensemble_member(void* sim, uint32_t member, BncEnsembleMember* out);
/* Host-only planning of a generated ensemble (no device). */
int bnc_plan_ensemble_generated(const BncNetgenParams* members, uint32_t n_members, BncNetInfo* info);
/* Host-only: parameters of a seeded uneven ensemble: member sizes log-uniform in
 * [min_segments, max_segments] (32-segment neurons of BNC_NET_ENSEMBLE_MEMBER),
 * gNa/gK/gleak/gCa scaled by independent U[0.5, 2] factors, one seed per member. */
int bnc_ensemble_params(uint64_t seed, uint32_t n_members, uint32_t min_segments, uint32_t max_segments,
                        BncNetgenParams* out);

/* Autotuned ensemble load: tries several groupings of components into warp
 * groups and tiles on a strided sample of at most 64 members (build, one untimed
 * tick, then trial_ticks timed with the captured loop), keeps the fastest and
 * builds the whole ensemble with it.  The grouping never changes results.  `out`
 * (may be NULL) receives the choice and its per-tick time on the sample. */
typedef struct {
    uint32_t warp_cap, tile_segs;   /* chosen grouping (segments per warp group / tile) */
    float ms_per_tick;              /* on the sample */
    uint32_t candidates_tried, sample_members;
} BncTuning;
int bnc_load_ensemble_tuned(void* sim, const BncNetgenParams* members, uint32_t n_members, uint32_t trial_ticks,
                            float dt, BncTuning* out);

/* bnc_run_ticks_graph bracketed by CUDA events; *ms receives the device time. */
int bnc_time_ticks_graph(void* sim, uint32_t n_ticks, float dt, float* ms);

/* Runs n ticks as one launch of a CUDA graph captured once: a conditional while node
 * around one tick, the device-side clock advance and a countdown set before each
 * launch (the tick counter lives on the device) -- same results as bnc_run_ticks,
 * one launch per call whatever n.  The tick that applies pending injections runs
 * before the graph as a plain launch.  The graph is re-captured when dt changes, a
 * network is loaded or stimuli are uploaded. */
int bnc_run_ticks_graph(void* sim, uint32_t n_ticks, float dt);

/* Build options of a network's device layout.  None of them changes results:
 *   warp_cap, tile_segs  grouping of components into warp groups and tiles
 *                        (defaults 64 and 1024);
 *   phase_cap            the modifier schedule keeps the greedy type-uniform
 *                        phases while they number at most phase_cap (0: twice the
 *                        longest modifier list + 4), else phases follow slot order;
 *   chunk_segs           the modifier pass runs all its phases on chunks of this
 *                        many consecutive segments in turn, so a chunk's working
 *                        records (96 bytes per segment) can stay in L2 between
 *                        phases (0: BNC_DEFAULT_CHUNK_SEGS, one chunk).  On B200
 *                        the extra launches cost more than L2 residency saves
 *                        (6.4M segments: 9.4 ms per tick in one chunk, 9.5 ms in
 *                        524,288-segment chunks, 11.6 ms in 262,144).
 *   fuse_phases          modifier phases per launch (default 4, at most 32; 1: one
 *                        launch per phase).  A launch runs each segment's items of
 *                        its phases with the segment's working record in registers,
 *                        so the record crosses HBM once per group instead of once per
 *                        phase.  It applies to slot-order schedules in one chunk
 *                        without registered device modifiers; others run one launch
 *                        per phase.  At 3.2M segments of the large set, step 1 takes
 *                        3.94 ms per tick with 1, 2.15 ms with 4 and 19.5 ms with 17
 *                        (one launch: warps diverge over the later items).
 * Zero fields take the defaults. */
typedef struct {
    uint32_t warp_cap, tile_segs, phase_cap, chunk_segs, fuse_phases;
    /* nonzero: the diffusion kernel synchronises whole CTAs even where every
     * connection stays inside an aligned group of 32 or 64 threads (for tests) */
    uint32_t cta_barriers;
} BncBuildOptions;
#define BNC_DEFAULT_CHUNK_SEGS 0xFFFFFFFFu
int bnc_load_generated_opts(void* sim, const BncNetgenParams* p, const BncBuildOptions* opt);
int bnc_plan_generated_opts(const BncNetgenParams* p, const BncBuildOptions* opt, BncNetInfo* info);

/* ---- Device modifiers: user modifier IDs 0-127 on the GPU ----
 * The reference registers plugin modifiers as host functions
 * (register_modifier_current, modifier_interface.h:38, called from a plugin's
 * biocore_plugin_init, plugin_manager.cpp:260-313); they override the built-in
 * model of that ID on its CPU path only (kernel_dispatch.h:336-343).  These calls
 * register device code instead: CUDA C++ source defining an extern "C" __global__
 * entry with the interface of bnc_device_modifier.h, compiled here by NVRTC for
 * sm_100a (no device needed to register).  Networks loaded afterwards run the
 * entry on that type's items, overriding a built-in model of the same ID; a
 * network that uses an ID with neither a built-in model nor a registration is
 * rejected with BNC_ERR_UNSUPPORTED (no CPU fallback).  Registering an ID again
 * replaces it for networks loaded later.
 *   biocore_gpu_register_device_modifier: source from a file (cu_path).
 *   Errors: BNC_ERR_ARG (ID >= 128, compile errors -- the NVRTC log is in
 *   bnc_last_error), BNC_ERR_UNSUPPORTED (NVRTC not available). */
int biocore_gpu_register_device_modifier(uint8_t type_id, const char* cu_path, const char* entry);
int bnc_register_device_modifier(uint8_t type_id, const char* source, const char* entry);
/* 1 when a device modifier is registered for the ID, else 0. */
int bnc_device_modifier_registered(uint8_t type_id);

/* ---- Reference modifier plugins (plugin_host.cpp) ----
 * The registration functions a reference plugin's biocore_plugin_init calls, with the
 * reference's names and linkage (modifier_interface.h:38-39 and, C++ linkage,
 * plugin_manager.h:98-99: register_user_modifier / register_user_modulator): they
 * record the CPU function per ID 0-127 (types >= 128 ignored, as the reference does).
 * ModifierFunc / ReleaseModulatorFunc are the reference's function types; this
 * backend never calls them.  A network using an ID that a host plugin registered is
 * refused with BNC_ERR_UNSUPPORTED unless device code is registered for the ID
 * (biocore_gpu_register_device_modifier): no CPU fallback. */
#ifndef BNC_PLUGIN_HOST_IMPL   /* plugin_host.cpp defines them with the reference's types */
typedef void (*BncPluginFunc)(void);   /* stands for ModifierFunc / ReleaseModulatorFunc */
void register_modifier_current(uint8_t type, BncPluginFunc func);
void register_modulator_release(uint8_t type, BncPluginFunc func);
#endif
/* plugin_load (plugin_manager.cpp:208-258): dlopen(RTLD_LAZY | RTLD_GLOBAL), this
 * library first made visible to the plugin; biocore_plugin_desc parsed when present;
 * biocore_plugin_init called.  Returns what init returned (> 0), or -1 (dlopen
 * failed), -2 (no biocore_plugin_init), -3 (init returned <= 0); the message is in
 * bnc_last_error().  The handle stays open for the process. */
int bnc_plugin_load(const char* so_path);
/* Every regular *.so file of a directory (plugin_load_directory,
 * plugin_manager.cpp:260-300); returns the sum of the positive registration counts. */
int bnc_plugin_load_directory(const char* dir_path);
/* bit 0: a current function is registered for the ID, bit 1: a release modulator. */
int bnc_plugin_registered(uint8_t type_id);
/* Plugins loaded so far. */
int bnc_plugin_count(void);
/* Forgets every registration (the libraries stay loaded). */
void bnc_plugin_unregister_all(void);

/* Mechano stimuli: the mechano argument of the reference's core_run_tick
 * (simulation_host.cpp:211-230), which the GPU backend's GpuStimulusData does not
 * carry.  Each stimulus writes its value into state[state_idx] of the first modifier
 * of type mod_type on the first segment whose id is segment_id, in the order given,
 * before the next tick's modifier currents (one-shot).  A stimulus whose segment,
 * type or index (0-7) does not exist does nothing; state[7] is the effective area,
 * which every tick rewrites, so a write there reaches only the records.  Nothing
 * reads modifier state between ticks, so the writes are made at once (device state
 * and records).  Needs the network's records (a network loaded from AoS arrays or a
 * .bion); BNC_ERR_UNSUPPORTED for generated networks and ensembles. */
int bnc_upload_mechano(void* sim, const BncMechanoStimulus* stimuli, uint32_t n);

/* Host-only: runs the builder's planning on AoS arrays in memory (validation,
 * supported-type checks, tiles, schedule) without a device.  Returns the same
 * codes a load of that network would. */
int bnc_plan_aos(const BncBionData* data, const BncCurrentStimulus* stim, uint32_t n_stim, BncNetInfo* info);

/* Host-only .bion I/O with the reference loader's semantics: bnc_bion_load
 * replaces bion_load_host (src/bion_loader_host.cpp:26-428: versions 3-14 with the
 * same migrations, default nuclei for a file without any, the same BION_ERR_* codes
 * and validation; arrays owned by the library until bnc_bion_unload, which replaces
 * bion_unload_host).  Bytes the reference's migrations leave unwritten are zero
 * here.  bnc_bion_save replaces bion_save (src/bion_loader_host.cpp:449-504, writes
 * v14). */
int bnc_bion_load(const char* filename, BncBionData* out);
void bnc_bion_unload(BncBionData* data);
int bnc_bion_save(const char* filename, const BncBionData* data);

/* Writes the host AoS view to a .bion v14 file (reference bion_save layout). */
int bnc_save_bion(void* sim, const char* filename);

/* Message for the last error on this thread ("" when none). */
const char* bnc_last_error(void);

/* Electrodiffusion options of step 2.5 for the loaded network.  They have no
 * counterpart in the reference, which always runs 50 Jacobi sweeps per solve
 * (diffusion_kernel.h:25,27); the default (flags 0) is that parity mode.
 *   BNC_DIFFUSION_RESIDUAL  the phi_e solve and each V_m solve iterate in FP64
 *                           until no value of a convergence group (a connected
 *                           component) changes by more than `tol` in a sweep,
 *                           at most `max_sweeps` sweeps.  V_m is stored as float.
 *   BNC_DIFFUSION_LEDGER    an FP64 ledger per ion over the run: `rounding`, the
 *                           amount (concentration x volume) that storing the
 *                           Nernst-Planck updates in FP32 added, and `bath`, the
 *                           amount the bath relaxation and clamps added to the
 *                           extracellular space.  Step 2.5 changes each ion's total
 *                           (intracellular + extracellular amount) by exactly their
 *                           sum, up to FP64 rounding.
 * Loading a network resets the mode to 0.  bnc_diffusion_stats reads the largest
 * sweep counts of a solve, the group solves that reached max_sweeps and the ledger
 * accumulated since the load or the last reset. */
#define BNC_DIFFUSION_RESIDUAL 1u
#define BNC_DIFFUSION_LEDGER 2u
typedef struct {
    uint32_t max_sweeps_v, max_sweeps_phi;   /* most sweeps of one V_m / phi_e solve */
    uint32_t capped_v, capped_phi;           /* group solves that stopped at max_sweeps */
    double rounding[7];                      /* per ion, amount units (mM x um^3) */
    double bath[7];
} BncDiffusionStats;
int bnc_set_diffusion_mode(void* sim, uint32_t flags, double tol, uint32_t max_sweeps);
int bnc_diffusion_stats(void* sim, BncDiffusionStats* out, int reset);

/* The daemon's MSG_STATE_FRAME payload (daemon_state.cpp:66-79): the tick counter
 * (u64), the segment and synapse counts (u32 each), then the Segment and Synapse
 * records of the current state, filled from the device state directly into `buf`.
 * *len receives the frame's size; BNC_ERR_ARG when buf is NULL or cap is smaller
 * (a size query). */
int bnc_state_frame(void* sim, void* buf, uint64_t cap, uint64_t* len);

/* Checkpoints that resume bit for bit.  The .bion (bion_loader_host.cpp:26-504)
 * records the AoS state; a running simulation also carries the tick counter (it seeds
 * the release draws, simulation_host.cpp:438-459, and times the stimuli), whether its
 * first tick has run, its stimuli, the receptor density scales
 * (bnc_set_synapse_scale) and the pending delayed releases (delay_buffer.h:15-64).
 * bnc_save_checkpoint writes `path` (.bion) and `path`.state with those;
 * bnc_load_checkpoint loads both, and the next tick continues the saved run exactly.
 * Single networks only (BNC_ERR_UNSUPPORTED for an ensemble). */
int bnc_save_checkpoint(void* sim, const char* path);
int bnc_load_checkpoint(void* sim, const char* path);

/* ------------------------------------------------------------------ */
/* 5b. parameter sweeps: many parameterised runs as one ensemble       */
/* ------------------------------------------------------------------ */
/* A task of the reference's parameterised runs (daemon_main.cpp:79-300, the batch
 * mode with --params-json and --seed; daemon_server.cpp:1164-1310, MSG_RUN_TASK_PARAMS):
 * parameter overrides -- state[0] of each segment's first modifier of the given type
 * set to the value -- and a seed that scales every synapse's release probability by
 * 1 + 0.02 * (hash(seed, id) & 0xFFFF) / 65536 (0: no variation). */
typedef struct {
    const uint8_t* type_ids;
    const float* values;
    uint32_t n_overrides;
    uint32_t seed;
} BncSweepTask;

/* core_compute_metrics (simulation_host.cpp:825-880) of one task's final state. */
typedef struct {
    float mean_vm;          /* mean V_m over the member's segments, mV */
    uint32_t spike_count;   /* segments with V_m > -20 mV */
    float synchrony;        /* fraction of segments within 10 mV of the mean */
    uint64_t tick;          /* the tick counter after the run */
    char metrics_json[2048];/* the reference's metrics string, type_vm included */
} BncSweepResult;

/* Step the tick counter once per tick, as a daemon task does.  Without it the counter
 * steps twice per tick, as the batch mode's loop does (core_run_tick increments it,
 * then the loop again, daemon_main.cpp:250-258). */
#define BNC_SWEEP_SINGLE_TICK 1u

/* The reference's parameter-JSON reader (daemon_main.cpp:79-155): numeric keys are
 * modifier type IDs (< 212); other keys resolve through the name table (a key that is
 * a case-insensitive prefix of a name, the lowest ID first), as the plugin
 * descriptors' names do.  Writes up to cap overrides; *n_out receives the count
 * (BNC_ERR_ARG if above cap). */
int bnc_sweep_parse_params(const char* json, const char* const* names, const uint8_t* name_ids, uint32_t n_names,
                           uint8_t* type_ids, float* values, uint32_t cap, uint32_t* n_out);
/* Applies one task to a network in place (host arrays). */
int bnc_sweep_apply(BncBionData* net, const BncSweepTask* task);
/* Runs every task on its own copy of `base` as one ensemble in `sim` (loaded by the
 * call; the members are readable afterwards with bnc_ensemble_member and the
 * bnc_read_*_field calls), `ticks` ticks of `dt`, and writes each task's metrics.
 * `stim` (may be NULL) applies to every member. */
int bnc_sweep_run(void* sim, const BncBionData* base, const BncCurrentStimulus* stim, uint32_t n_stim,
                  const BncSweepTask* tasks, uint32_t n_tasks, uint32_t ticks, float dt, uint32_t flags,
                  BncSweepResult* results);

/* ------------------------------------------------------------------ */
/* 6. adjoint: gradients of a somatic voltage-trace loss               */
/* ------------------------------------------------------------------ */
/* The forward/backward pair differentiates the tick of simulation_host.cpp:174-657
 * with respect to per-segment maximal conductances -- gNa, gK, gleak: the densities
 * of the segment's Nav1.6/Nav1.2 (141/142), Kv delayed rectifier (123) and K2P leak
 * (107) modifiers -- and per-synapse weights, a multiplicative scale on the density
 * of the synapse's receptors (the `mod_scale` of ionotropic_ghk_current,
 * modifier_helpers.h:421; 1 reproduces the reference).  The reference has no
 * gradient path; these entry points are new.
 *
 * Loss of parameter set p: (1 / (S * n)) * sum over the S sampled ticks and the n
 * neurons of (V_soma - target)^2, V_soma taken after every `sample_every`-th tick.
 *
 * Release events are pathwise: bnc_adjoint_record runs the plain tick on `sim` and
 * logs every transmitter amount that enters a cleft; the forward and backward passes
 * replay that log for every parameter set.  With the releases fixed each neuron
 * evolves on its own, so a forward pass runs one CTA per (neuron, parameter set).
 * The backward pass re-runs windows of `checkpoint_every` ticks from checkpoints and
 * walks each window backwards.
 *
 * Modelled networks (others are rejected with BNC_ERR_UNSUPPORTED): segment
 * modifiers Nav1.6, Nav1.2, Kv_DR, K2P (differentiated), myelin and Cav2.1 (no
 * current); chemical synapses with AMPA, NMDA, GABA-A and glycine receptors (at most 2 each);
 * neurons of at most 128 segments and 4 connections per segment, each a contiguous segment range joined by its
 * connections; no voltage clamps. */
typedef struct {
    uint32_t n_sets;           /* parameter sets run side by side, 1..65535 */
    uint32_t ticks;            /* ticks of the run */
    uint32_t checkpoint_every; /* K: ticks between checkpoints (0: 256) */
    uint32_t sample_every;     /* somatic V_m sampled after every this many ticks (0: 1) */
    float dt;                  /* ms */
} BncAdjointConfig;

typedef struct {
    uint32_t n_neurons, n_segments, n_synapses, n_samples, n_sets, ticks, checkpoint_every;
    uint32_t threads, smem_forward, smem_backward;   /* per CTA */
    uint64_t checkpoint_bytes, window_bytes, scratch_bytes;
} BncAdjointInfo;

/* Takes structure, state and parameters from the network loaded in `sim` (loaded
 * from AoS arrays, at its current tick).  NULL on error (bnc_last_error).  Every
 * parameter set starts from the network's densities and weight scale 1. */
void* bnc_adjoint_create(void* sim, const BncAdjointConfig* cfg);
void bnc_adjoint_destroy(void* adj);
int bnc_adjoint_info(void* adj, BncAdjointInfo* info);
/* The global segment index of each neuron's soma (the order of the loss's neurons). */
int bnc_adjoint_soma(void* adj, uint32_t* soma, uint32_t n);
/* Runs cfg.ticks plain ticks on `sim` (the network the adjoint was created from, at
 * the same tick) and keeps the release log they produce. */
int bnc_adjoint_record(void* adj, void* sim);
int bnc_adjoint_release_count(void* adj, uint64_t* n);
/* Parameters of one set, in original segment / synapse order; NULL leaves an array. */
int bnc_adjoint_set_params(void* adj, uint32_t set, const float* gNa, const float* gK, const float* gleak,
                           const float* w);
int bnc_adjoint_get_params(void* adj, uint32_t set, float* gNa, float* gK, float* gleak, float* w);
/* Target somatic traces [n_samples][n_neurons], shared by all sets. */
int bnc_adjoint_set_target(void* adj, const float* target);
/* Forward pass of every set from the network's state at creation: loss[n_sets]
 * (may be NULL; needs a target), trace [n_sets][n_samples][n_neurons] (may be NULL). */
int bnc_adjoint_forward(void* adj, double* loss, float* trace);
/* Backward pass after a forward pass with the same parameters: gradients of each
 * set's loss, [n_sets][n_segments] for each conductance and [n_sets][n_synapses] for
 * the weights (any may be NULL).  A segment without the modifier gets 0. */
int bnc_adjoint_backward(void* adj, float* g_gNa, float* g_gK, float* g_gleak, float* g_w);
/* Device time of the last forward and backward pass (CUDA events). */
int bnc_adjoint_timings(void* adj, float* forward_ms, float* backward_ms);

#ifdef __cplusplus
}
#endif
#endif /* BNC_B200_H */
