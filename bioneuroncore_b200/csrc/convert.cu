// convert.cu -- the network's state converted into the device layout on the device.
//
// The loaders (the .bion reader's records, compacted to HostNet, or the generator)
// leave one record per segment, modifier, synapse and receptor in the order of the
// file.  The builder decides the device order (segments by tile, items by phase and
// row, synapses by warp slice, receptors by slice) on the host from the structure
// alone -- types, counts, endpoints -- and these kernels gather the values: the
// records are copied to the device once, as they are, and one thread per output
// element reads its record and writes the SoA words.  The host never materialises the
// SoA state (about 8 GB at 6.4M segments and 10M synapses), whose first-touch page
// faults and strided stores were most of the set-up time.
//
// Every output is a copy of a record word or a flag computed from record words by
// integer and comparison operations, so the device result is the host fill's, bit
// for bit.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "hostnet.h"
#include "net.h"

namespace bnc {

namespace {

// per modifier type: the state words it reads as parameters (a non-zero one sets
// flag bit 0), and whether its active_vars selects a conductance override
struct TypeTable {
    uint8_t par[256];
    uint8_t rcp[256];
};

__global__ void k_conv_items(const ModLite* __restrict__ mods, const uint64_t* __restrict__ mod_off,
                             const uint32_t* __restrict__ item_seg, const uint8_t* __restrict__ item_slot,
                             const uint32_t* __restrict__ inv, uint32_t NI, TypeTable tt, uint32_t* __restrict__ it_seg,
                             uint16_t* __restrict__ it_tf, float* __restrict__ it_den, float* __restrict__ it_st,
                             unsigned* bad) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= NI) return;
    const uint32_t orig = item_seg[q];
    const ModLite m = mods[mod_off[orig] + item_slot[q]];
    uint32_t fl = 0;
    const uint32_t pm = tt.par[m.type];
#pragma unroll
    for (int b = 0; b < 7; b++)
        if (((pm >> b) & 1u) && m.state[b] != 0.0f) fl |= 1u;
    if (tt.rcp[m.type] && m.active_vars > 0) {
        if (m.active_vars >= 8) atomicMin(bad, q);
        fl |= 2u | ((uint32_t)(m.active_vars & 7u) << 2);
    }
    it_seg[q] = inv[orig];
    it_tf[q] = (uint16_t)(m.type | (fl << 8));
    it_den[q] = m.density;
#pragma unroll
    for (int b = 0; b < 7; b++) it_st[(size_t)b * NI + q] = m.state[b];
}

__global__ void k_conv_segments(const SegLite* __restrict__ segs, const ModLite* __restrict__ mods,
                                const uint32_t* __restrict__ perm, uint32_t n, float* __restrict__ V,
                                float* __restrict__ ion_in, float* __restrict__ ion_out, float* __restrict__ intra_nt,
                                float* __restrict__ nt, float* __restrict__ atp, float* __restrict__ temp,
                                float* __restrict__ txn, float* __restrict__ radius, float* __restrict__ length,
                                uint8_t* __restrict__ stype, double* __restrict__ ibuf, float2* __restrict__ c21) {
    const uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const SegLite& s = segs[perm[d]];
    V[d] = s.V_m;
#pragma unroll
    for (int q = 0; q < 7; q++) {
        ion_in[(size_t)q * n + d] = s.intra_ions[q];
        ion_out[(size_t)q * n + d] = s.extra_ions[q];
    }
#pragma unroll
    for (int q = 0; q < 15; q++) {
        intra_nt[(size_t)q * n + d] = s.intra_nt[q];
        nt[(size_t)q * n + d] = s.neurotransmitter[q];
    }
    atp[d] = s.ATP_level;
    temp[d] = s.temperature;
    txn[d] = s.transcription_signal;
    radius[d] = s.radius;
    length[d] = s.length;
    stype[d] = s.segment_type;
    ibuf[d] = s.I_buffer;
    // the last Cav2.1 of the segment (its density and state[1])
    float2 c = make_float2(0.0f, 0.0f);
    for (uint32_t j = 0; j < s.modifier_count; j++) {
        const ModLite& m = mods[s.mod_off + j];
        if (m.type == BNC_MOD_CAV21) c = make_float2(m.density, m.state[1]);
    }
    c21[d] = c;
}

// per type: the bouton channel conductance an autoreceptor adds (0: none) and the
// transmitter a first post receptor releases
struct SynTable {
    float gamma[256];
    uint8_t ntr[256];
};

struct SynOut {
    uint32_t *pre, *id;
    float *prel, *amt, *tauc, *delay, *prea, *posta, *gK, *gNa, *bouton, *spine, *camkii, *calcn, *facil, *weight,
        *cleft, *rrp, *rrpm, *rrpr, *scale;
    uint8_t *refr, *flags;
};

__global__ void k_conv_synapses(const SynLite* __restrict__ syns, const ModLite* __restrict__ recs,
                                const uint32_t* __restrict__ syn_orig, const uint32_t* __restrict__ inv, uint32_t K,
                                SynTable tb, SynOut o) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= K) return;
    const SynLite& y = syns[syn_orig[q]];
    o.pre[q] = inv[y.pre_segment];
    o.id[q] = y.id;
    o.prel[q] = y.release_probability;
    o.amt[q] = y.release_amount;
    o.tauc[q] = y.tau_clearance;
    o.delay[q] = y.delay;
    o.prea[q] = y.pre_area;
    o.posta[q] = y.post_area;
    // bouton channels of the autoreceptors, in slot order (modifier_helpers.h:767-773)
    float gK = 0.0f, gNa = 0.0f;
    for (uint32_t j = 0; j < y.pre_autoreceptor_count; j++) {
        const ModLite& m = recs[y.rec_off + y.post_receptor_count + j];
        const float g = (float)((double)m.density * (double)tb.gamma[m.type]);
        if (m.type == 141 || m.type == 142) gNa += g;
        else gK += g;
    }
    o.gK[q] = gK;
    o.gNa[q] = gNa;
    o.refr[q] = y.refractory;
    const uint8_t ntt = y.post_receptor_count > 0 ? tb.ntr[recs[y.rec_off].type] : 0;
    bool inhib = false;
    for (uint32_t j = 0; j < y.post_receptor_count; j++) {
        const uint8_t rt = recs[y.rec_off + j].type;
        if (rt == 11 || rt == 17 || rt == 12) { inhib = true; break; }
    }
    o.flags[q] = (uint8_t)((inhib ? 1u : 0u) | ((uint32_t)ntt << 4));
    o.bouton[q] = y.bouton_Ca;
    o.spine[q] = y.spine_Ca;
    o.camkii[q] = y.spine_camkii;
    o.calcn[q] = y.spine_calcineurin;
    o.facil[q] = y.facilitation;
    o.weight[q] = y.weight;
    o.cleft[q] = y.cleft_neurotransmitter[ntt];
    o.rrp[q] = y.RRP;
    o.rrpm[q] = y.RRP_max;
    o.rrpr[q] = y.RRP_recovery;
    o.scale[q] = 1.0f;
}

__global__ void k_conv_receptors(const SynLite* __restrict__ syns, const ModLite* __restrict__ recs,
                                 const uint32_t* __restrict__ syn_orig, const uint32_t* __restrict__ rec_syn,
                                 const uint8_t* __restrict__ rec_slot, uint32_t NR, uint8_t* __restrict__ type,
                                 uint8_t* __restrict__ av, float* __restrict__ den, float* __restrict__ st) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= NR) return;
    const ModLite& m = recs[syns[syn_orig[rec_syn[r]]].rec_off + rec_slot[r]];
    type[r] = m.type;
    av[r] = m.active_vars;
    den[r] = m.density;
    st[r] = m.state[0];
    st[(size_t)NR + r] = m.state[1];
    st[(size_t)2 * NR + r] = m.state[2];
}

// Device copies of host arrays that live only while the conversion runs.
struct Scratch {
    std::vector<void*> p;
    ~Scratch() {
        for (void* x : p) cudaFree(x);
    }
    template <typename T>
    const T* up(const T* h, size_t n, int* rc) {
        void* x = nullptr;
        if (*rc != BNC_OK) return nullptr;
        if (cudaMalloc(&x, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
            set_error("device allocation of %zu bytes for the state conversion failed", n * sizeof(T));
            *rc = BNC_ERR_ALLOC;
            return nullptr;
        }
        p.push_back(x);
        if (n && cudaMemcpy(x, h, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
            set_error("copy of the host records for the state conversion failed");
            *rc = BNC_ERR_CUDA;
        }
        return (const T*)x;
    }
};

template <typename T>
T* out(DeviceAllocs* a, size_t n, int* rc) {
    if (*rc != BNC_OK) return nullptr;
    T* p = (T*)a->alloc(n * sizeof(T));
    if (!p) {
        set_error("device allocation of %zu bytes failed", n * sizeof(T));
        *rc = BNC_ERR_ALLOC;
    }
    return p;
}

int finish(int rc, const char* what) {
    if (rc != BNC_OK) return rc;
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return BNC_ERR_CUDA;
    }
    return BNC_OK;
}

}  // namespace

int device_convert_state(const HostNet& hn, const std::vector<uint32_t>& perm, const std::vector<uint32_t>& inv,
                         const std::vector<uint32_t>& item_seg, const std::vector<uint8_t>& item_slot, NetDev* dev,
                         DeviceAllocs* allocs, uint32_t* bad_item) {
    *bad_item = UINT32_MAX;
    const uint32_t n = (uint32_t)perm.size();
    const uint32_t NI = (uint32_t)item_seg.size();
    int rc = BNC_OK;
    dev->V = out<float>(allocs, n, &rc);
    dev->ion_in = out<float>(allocs, (size_t)7 * n, &rc);
    dev->ion_out = out<float>(allocs, (size_t)7 * n, &rc);
    dev->intra_nt = out<float>(allocs, (size_t)15 * n, &rc);
    dev->nt = out<float>(allocs, (size_t)15 * n, &rc);
    dev->atp = out<float>(allocs, n, &rc);
    dev->temp = out<float>(allocs, n, &rc);
    dev->txn = out<float>(allocs, n, &rc);
    dev->radius = out<float>(allocs, n, &rc);
    dev->length = out<float>(allocs, n, &rc);
    dev->stype = out<uint8_t>(allocs, n, &rc);
    dev->ibuf = out<double>(allocs, n, &rc);
    dev->cav21_static = out<float2>(allocs, n, &rc);
    dev->it_seg = out<uint32_t>(allocs, NI, &rc);
    dev->it_tf = out<uint16_t>(allocs, NI, &rc);
    dev->it_den = out<float>(allocs, NI, &rc);
    dev->it_st = out<float>(allocs, (size_t)7 * NI, &rc);
    if (rc != BNC_OK || n == 0) return rc;
    TypeTable tt;
    for (int t = 0; t < 256; t++) {
        tt.par[t] = param_mask((uint8_t)t);
        tt.rcp[t] = host_receptor_supported((uint8_t)t) ? 1 : 0;
    }
    std::vector<uint64_t> mod_off(hn.seg.size());
    for (size_t i = 0; i < hn.seg.size(); i++) mod_off[i] = hn.seg[i].mod_off;
    Scratch s;
    const SegLite* d_segs = s.up(hn.seg.data(), hn.seg.size(), &rc);
    const ModLite* d_mods = s.up(hn.mods.data(), hn.mods.size(), &rc);
    const uint32_t* d_perm = s.up(perm.data(), n, &rc);
    const uint64_t* d_off = s.up(mod_off.data(), mod_off.size(), &rc);
    const uint32_t* d_iseg = s.up(item_seg.data(), NI, &rc);
    const uint8_t* d_islot = s.up(item_slot.data(), NI, &rc);
    const uint32_t* d_inv = s.up(inv.data(), inv.size(), &rc);
    unsigned* d_bad = (unsigned*)s.up(bad_item, 1, &rc);
    if (rc != BNC_OK) return rc;
    k_conv_segments<<<(n + 255) / 256, 256>>>(d_segs, d_mods, d_perm, n, dev->V, dev->ion_in, dev->ion_out,
                                              dev->intra_nt, dev->nt, dev->atp, dev->temp, dev->txn, dev->radius,
                                              dev->length, dev->stype, dev->ibuf, dev->cav21_static);
    if (NI)
        k_conv_items<<<(NI + 255) / 256, 256>>>(d_mods, d_off, d_iseg, d_islot, d_inv, NI, tt, dev->it_seg,
                                                dev->it_tf, dev->it_den, dev->it_st, d_bad);
    rc = finish(rc, "state conversion");
    if (rc == BNC_OK && cudaMemcpy(bad_item, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("state conversion: status read failed");
        rc = BNC_ERR_CUDA;
    }
    return rc;
}

int device_convert_synapses(const HostNet& hn, const std::vector<uint32_t>& syn_orig,
                            const std::vector<uint32_t>& inv, const std::vector<uint32_t>& rec_syn,
                            const std::vector<uint8_t>& rec_slot, NetDev* dev, DeviceAllocs* allocs) {
    const uint32_t K = (uint32_t)syn_orig.size();
    const uint32_t NR = (uint32_t)rec_syn.size();
    int rc = BNC_OK;
    SynOut o;
    o.pre = dev->sy_pre = out<uint32_t>(allocs, K, &rc);
    o.id = dev->sy_id = out<uint32_t>(allocs, K, &rc);
    o.prel = dev->sy_prel = out<float>(allocs, K, &rc);
    o.amt = dev->sy_amt = out<float>(allocs, K, &rc);
    o.tauc = dev->sy_tauc = out<float>(allocs, K, &rc);
    o.delay = dev->sy_delay = out<float>(allocs, K, &rc);
    o.prea = dev->sy_pre_area = out<float>(allocs, K, &rc);
    o.posta = dev->sy_post_area = out<float>(allocs, K, &rc);
    o.gK = dev->sy_gK = out<float>(allocs, K, &rc);
    o.gNa = dev->sy_gNa = out<float>(allocs, K, &rc);
    o.refr = dev->sy_refr = out<uint8_t>(allocs, K, &rc);
    o.flags = dev->sy_flags = out<uint8_t>(allocs, K, &rc);
    o.bouton = dev->sy_bouton = out<float>(allocs, K, &rc);
    o.spine = dev->sy_spine = out<float>(allocs, K, &rc);
    o.camkii = dev->sy_camkii = out<float>(allocs, K, &rc);
    o.calcn = dev->sy_calcn = out<float>(allocs, K, &rc);
    o.facil = dev->sy_facil = out<float>(allocs, K, &rc);
    o.weight = dev->sy_weight = out<float>(allocs, K, &rc);
    o.cleft = dev->sy_cleft = out<float>(allocs, K, &rc);
    o.rrp = dev->sy_rrp = out<float>(allocs, K, &rc);
    o.rrpm = dev->sy_rrp_max = out<float>(allocs, K, &rc);
    o.rrpr = dev->sy_rrp_rec = out<float>(allocs, K, &rc);
    o.scale = dev->sy_scale = out<float>(allocs, K, &rc);
    dev->rc_type = out<uint8_t>(allocs, NR, &rc);
    dev->rc_av = out<uint8_t>(allocs, NR, &rc);
    dev->rc_den = out<float>(allocs, NR, &rc);
    dev->rc_st = out<float>(allocs, (size_t)3 * NR, &rc);
    if (rc != BNC_OK || K == 0) return rc;
    SynTable tb;
    for (int t = 0; t < 256; t++) {
        tb.gamma[t] = host_bouton_gamma((uint8_t)t);
        tb.ntr[t] = host_nt_from_receptor((uint8_t)t);
    }
    Scratch s;
    const SynLite* d_syns = s.up(hn.syn.data(), hn.syn.size(), &rc);
    const ModLite* d_recs = s.up(hn.recs.data(), hn.recs.size(), &rc);
    const uint32_t* d_orig = s.up(syn_orig.data(), K, &rc);
    const uint32_t* d_inv = s.up(inv.data(), inv.size(), &rc);
    const uint32_t* d_rsyn = s.up(rec_syn.data(), NR, &rc);
    const uint8_t* d_rslot = s.up(rec_slot.data(), NR, &rc);
    if (rc != BNC_OK) return rc;
    k_conv_synapses<<<(K + 255) / 256, 256>>>(d_syns, d_recs, d_orig, d_inv, K, tb, o);
    if (NR)
        k_conv_receptors<<<(NR + 255) / 256, 256>>>(d_syns, d_recs, d_orig, d_rsyn, d_rslot, NR, dev->rc_type,
                                                    dev->rc_av, dev->rc_den, dev->rc_st);
    return finish(rc, "synapse conversion");
}

}  // namespace bnc
