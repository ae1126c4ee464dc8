/*
 * bnc_abi.h -- binary layout of the BioNeuronCore data model, restated for the
 * B200 backend.
 *
 * Every struct here must be byte-compatible with the reference's `.bion` v14
 * in-memory model, because the drop-in backend hands these structs across the
 * same C ABI the reference's `gpu_backend_*` functions use:
 *
 *   Modifier        88 B   reference include/types.h:451-459
 *   Segment       3216 B   reference include/types.h:470-493
 *   Neuron          24 B   reference include/types.h:496-504
 *   IntraConnection 16 B   reference include/types.h:528-534
 *   Synapse       1568 B   reference include/types.h:537-569
 *   NetworkHeader  100 B   reference include/types.h:578-603
 *   stimulus structs        reference include/types.h:608-674
 *   GpuDeviceInfo          reference include/types.h:690-698
 *   BionData               reference include/bion_loader.h:16-28
 *
 * The offsets asserted at the bottom are the ones the reference's ABI test
 * checks (tests/test_abi_segment_layout.cpp:14-57).  The constants are the
 * reference's IDs (include/types.h:22-313); names carry a BNC_ prefix.
 */
#ifndef BNC_ABI_H
#define BNC_ABI_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- limits (reference include/types.h:400-407) ---- */
#define BNC_ION_COUNT 7
#define BNC_ION_MAX 8
#define BNC_NT_COUNT 15
#define BNC_MAX_MODIFIERS 32
#define BNC_MAX_STATE 8
#define BNC_MAX_PRE_AUTORECEPTORS 8
#define BNC_MAX_POST_RECEPTORS 8
#define BNC_MAX_INTRACONN_PER_SEG 16
#define BNC_GPU_MAX_STIMULI 256
#define BNC_MAX_DELAY_SLOTS 4

/* ions (reference include/types.h:266-274) */
#define BNC_ION_NA 0
#define BNC_ION_K 1
#define BNC_ION_CA 2
#define BNC_ION_CL 3
#define BNC_ION_MG 4
#define BNC_ION_A 5
#define BNC_ION_H 6

/* neurotransmitters (reference include/types.h:294-309) */
#define BNC_NT_GLUTAMATE 0
#define BNC_NT_GABA 1
#define BNC_NT_DOPAMINE 2
#define BNC_NT_SEROTONIN 3
#define BNC_NT_ACETYLCHOLINE 4
#define BNC_NT_GLYCINE 7
#define BNC_NT_ENDOCANNABINOID 9

/* synapse types (reference include/types.h:395-398) */
#define BNC_SYN_CHEMICAL 0
#define BNC_SYN_ELECTRICAL 1
#define BNC_SYN_DENDRITIC_BRIDGE 2

/* segment types (reference include/types.h:464-468) */
#define BNC_SEG_SOMA 1
#define BNC_SEG_NEURITE 2
#define BNC_SEG_BOUTON 3
#define BNC_SEG_SPINE 4

/* modifier type IDs used by the backend (reference include/types.h:22-263) */
#define BNC_MOD_CAV13 1
#define BNC_MOD_IONOTROPIC_CL 2
#define BNC_MOD_MYELIN 4
#define BNC_MOD_PUMP_NAK 7
#define BNC_MOD_AMPA 8
#define BNC_MOD_NMDA 9
#define BNC_MOD_GABAA 11
#define BNC_MOD_GLYCINE 12
#define BNC_MOD_TRPV1 16
#define BNC_MOD_GABAB 17
#define BNC_MOD_5HT3 14
#define BNC_MOD_NICOTINIC 13
#define BNC_MOD_D1 44
#define BNC_MOD_D2 22
#define BNC_MOD_5HT7 43
#define BNC_MOD_CAMKII 82
#define BNC_MOD_CALCINEURIN 83
#define BNC_MOD_KV42 85
#define BNC_MOD_ECB_SYNTHESIS 86
#define BNC_MOD_NICOTINIC_ALPHA7 97
#define BNC_MOD_PMCA 98
#define BNC_MOD_NCX 99
#define BNC_MOD_KCC2 100
#define BNC_MOD_CA_BUFFER 102
#define BNC_MOD_SK 103
#define BNC_MOD_BK 104
#define BNC_MOD_NAP 105
#define BNC_MOD_KIR 106
#define BNC_MOD_K2P 107
#define BNC_MOD_KV7 112
#define BNC_MOD_PP1_DARPP32 113
#define BNC_MOD_CX36 114
#define BNC_MOD_KV_DR 123
#define BNC_MOD_HCN1 129
#define BNC_MOD_NALCN 133
#define BNC_MOD_P2X2 134
#define BNC_MOD_CAMP_PKA 135
#define BNC_MOD_PKC 137
#define BNC_MOD_CAV21 140
#define BNC_MOD_NAV16 141
#define BNC_MOD_NAV12 142
#define BNC_MOD_GLAST 147
#define BNC_MOD_KV31 150
#define BNC_MOD_NMDA_2B 194
#define BNC_MOD_CX43 198
#define BNC_MOD_CAV31 200
#define BNC_MOD_TYPE_COUNT 212
#define BNC_MOD_USER_TABLE_SIZE 128

#pragma pack(push, 1)

typedef struct { float x, y, z; } BncVec3;

typedef struct {
    uint8_t type;
    uint8_t _pad[7];
    double density;
    double state[BNC_MAX_STATE];
    uint8_t active_vars;
    uint8_t flags;
    uint8_t _reserved[6];
} BncModifier;

typedef struct {
    uint32_t id;
    uint32_t neuron_id;
    BncVec3 position;
    BncVec3 direction;
    float length;
    float radius;
    double V_m;
    double intra_ions[BNC_ION_MAX];
    double extra_ions[BNC_ION_MAX];
    float intra_nt[BNC_NT_COUNT];
    float neurotransmitter[BNC_NT_COUNT];
    BncModifier modifiers[BNC_MAX_MODIFIERS];
    uint8_t modifier_count;
    uint8_t segment_type;
    uint8_t reserved1[6];
    float ATP_level;
    float temperature;
    double I_buffer;
    float transcription_signal;
    uint32_t intra_connection_ids[BNC_MAX_INTRACONN_PER_SEG];
    uint8_t intra_connection_count;
    uint8_t reserved2[7];
    float ER_Ca2;
} BncSegment;

typedef struct {
    uint32_t id;
    uint32_t segment_start;
    uint32_t segment_count;
    uint32_t soma_index;
    float threshold;
    uint8_t type;
    uint8_t reserved[3];
} BncNeuron;

typedef struct {
    uint32_t segment_a;
    uint32_t segment_b;
    uint8_t is_intracellular;
    uint8_t reserved[3];
    uint32_t _pad;
} BncIntraConnection;

typedef struct {
    uint32_t id;
    uint32_t pre_segment;
    uint32_t post_segment;
    uint8_t type;
    uint8_t reserved[3];
    float weight;
    float delay;
    float pre_area;
    float post_area;
    BncModifier pre_autoreceptors[BNC_MAX_PRE_AUTORECEPTORS];
    uint8_t pre_autoreceptor_count;
    uint8_t reserved2[7];
    BncModifier post_receptors[BNC_MAX_POST_RECEPTORS];
    uint8_t post_receptor_count;
    uint8_t reserved3[3];
    float release_probability;
    float release_amount;
    float cleft_neurotransmitter[BNC_NT_COUNT];
    float facilitation;
    float depression;
    float tau_clearance;
    uint8_t refractory;
    uint8_t reserved4[7];
    float RRP;
    float RRP_max;
    float RRP_recovery;
    float bouton_Ca;
    float spine_Ca;
    float spine_camkii;
    float spine_calcineurin;
} BncSynapse;

typedef struct {
    uint32_t magic;
    uint32_t version;
    uint8_t mode;
    uint8_t diffusion_type;
    uint16_t reserved;
    uint32_t num_neurons;
    uint32_t num_segments;
    uint32_t num_intra_connections;
    uint32_t num_synapses;
    uint32_t grid_dim_x;
    uint32_t grid_dim_y;
    uint32_t grid_dim_z;
    float voxel_size;
    uint64_t timestamp;
    char build_id[16];
    uint32_t num_nuclei;
    uint32_t nucleus_version;
    uint32_t file_sz_segment;
    uint32_t file_sz_synapse;
    uint32_t file_sz_nucleus;
    uint32_t file_sz_intraconnection;
    uint32_t file_sz_neuron;
    uint32_t file_sz_modifier;
} BncNetworkHeader;

typedef struct {
    uint32_t segment_id;
    float amplitude_pA;
    float duration_ms;
    uint64_t start_tick;
} BncCurrentStimulus;

typedef struct {
    uint32_t segment_id;
    float target_mV;
    uint64_t start_tick;
    uint64_t end_tick;
} BncVoltageClamp;

typedef struct {
    uint32_t segment_id;
    float start_pA;
    float end_pA;
    uint64_t start_tick;
    uint64_t end_tick;
} BncRampStimulus;

typedef struct {
    uint32_t segment_id;
    int32_t ion_idx;
    float amount_mM;
    uint8_t extracellular;
    uint8_t _pad[3];
} BncIonInjection;

typedef struct {
    uint32_t segment_id;
    int32_t nt_idx;
    float amount;
    uint8_t intracellular;
    uint8_t _pad2[3];
} BncLigandInjection;

typedef struct {
    uint32_t current_stim_count;
    uint32_t vclamp_count;
    uint32_t ramp_count;
    uint32_t ion_inj_count;
    uint32_t lig_inj_count;
    uint64_t current_tick;
    BncCurrentStimulus current_stim[BNC_GPU_MAX_STIMULI];
    BncVoltageClamp vclamps[BNC_GPU_MAX_STIMULI];
    BncRampStimulus ramps[BNC_GPU_MAX_STIMULI];
    BncIonInjection ion_inj[BNC_GPU_MAX_STIMULI];
    BncLigandInjection lig_inj[BNC_GPU_MAX_STIMULI];
} BncGpuStimulusData;

/* Mechano stimulus (types.h:645-655): value written into state[state_idx] of the
 * first modifier of type mod_type on the segment whose id is segment_id. */
typedef struct {
    uint32_t segment_id;
    uint8_t mod_type;
    int32_t state_idx;
    float value;
} BncMechanoStimulus;

typedef struct {
    char name[128];
    uint32_t vendor_id;
    uint8_t is_cpu;
    uint64_t global_mem_bytes;
    uint32_t max_compute_units;
    int32_t device_index;
    char backend_type[16];
} BncGpuDeviceInfo;

#pragma pack(pop)

/* Not packed: the reference's BionData is a plain struct (bion_loader.h:16-28),
 * so `segments` sits at offset 112 and `num_segments` at 148. */
typedef struct {
    BncNetworkHeader header;
    BncNeuron* neurons;
    BncSegment* segments;
    BncIntraConnection* connections;
    BncSynapse* synapses;
    void* nuclei;
    uint32_t num_neurons;
    uint32_t num_segments;
    uint32_t num_connections;
    uint32_t num_synapses;
    uint32_t num_nuclei;
} BncBionData;

#define BNC_STATIC_ASSERT(c, m) typedef char bnc_static_assert_##m[(c) ? 1 : -1]
BNC_STATIC_ASSERT(sizeof(BncModifier) == 88, modifier_size);
BNC_STATIC_ASSERT(sizeof(BncSegment) == 3216, segment_size);
BNC_STATIC_ASSERT(sizeof(BncSynapse) == 1568, synapse_size);
BNC_STATIC_ASSERT(sizeof(BncIntraConnection) == 16, conn_size);
BNC_STATIC_ASSERT(sizeof(BncNeuron) == 24, neuron_size);
BNC_STATIC_ASSERT(sizeof(BncNetworkHeader) == 100, header_size);
BNC_STATIC_ASSERT(sizeof(BncMechanoStimulus) == 13, mechano_size);
BNC_STATIC_ASSERT(offsetof(BncSegment, V_m) == 40, seg_vm);
BNC_STATIC_ASSERT(offsetof(BncSegment, intra_ions) == 48, seg_intra);
BNC_STATIC_ASSERT(offsetof(BncSegment, extra_ions) == 112, seg_extra);
BNC_STATIC_ASSERT(offsetof(BncSegment, modifier_count) == 3112, seg_mc);
BNC_STATIC_ASSERT(offsetof(BncSegment, segment_type) == 3113, seg_type);
BNC_STATIC_ASSERT(offsetof(BncSegment, I_buffer) == 3128, seg_ibuf);
BNC_STATIC_ASSERT(offsetof(BncSynapse, post_receptors) == 744, syn_post);
BNC_STATIC_ASSERT(offsetof(BncSynapse, bouton_Ca) == 1552, syn_bouton);
BNC_STATIC_ASSERT(offsetof(BncBionData, segments) == 112, bion_segments);
BNC_STATIC_ASSERT(offsetof(BncBionData, num_segments) == 148, bion_nseg);

#ifdef __cplusplus
}
#endif
#endif /* BNC_ABI_H */
