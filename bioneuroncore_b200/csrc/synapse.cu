// synapse.cu -- the synapse + membrane kernel of a tick (steps 3 and 4).
//
// Thread t handles segment th_seg[t]: first the segments that receive synapses, by
// synapse count descending, then the rest (membrane update only).  Each thread walks
// its segment's incoming synapses in original synapse order, then updates the
// membrane of that segment, so no atomics are involved and every sum keeps the
// reference's order.  Synapse and receptor arrays are stored warp-sliced: the k-th
// synapses of a warp's lanes are adjacent (lanes that still have one form a prefix of
// the warp, since counts descend), and the j-th receptors of a slice's synapses are
// adjacent, so the loads of a loop iteration are coalesced.  All four ionotropic
// receptors run one code path with per-lane constants, so lanes holding different
// receptor types do not serialise.  Presynaptic values come from the record the
// diffusion kernel wrote after step 2.5 (V, Ca_out, the Cav2.1 gate).
#include <cuda_runtime.h>
#include "net.h"
#include "physics.cuh"
#include "receptor.cuh"

namespace bnc {

static bool g_rec_ready[64] = {false};   // per device

__device__ __forceinline__ float xorshift32_rnd(uint32_t seed) {
    uint32_t x = seed;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    return (float)(x & 0x7FFFFFFFu) / (float)0x7FFFFFFFu;
}

// run_tick_common.h:114-122: the slow Ca2+/calmodulin gate of a gap junction
__device__ __forceinline__ float gj_cam_update(float m_slow, float ca_pre, float ca_post, float dt) {
    float ca_avg = 0.5f * (ca_pre + ca_post);
    float cam_act = (ca_avg * ca_avg) / (ca_avg * ca_avg + 0.0003f * 0.0003f);
    m_slow += (cam_act - m_slow) * dt / 100.0f;
    if (m_slow < 0.0f) m_slow = 0.0f;
    if (m_slow > 1.0f) m_slow = 1.0f;
    return m_slow;
}

// run_tick_common.h:79-110: the junction's conductance (nS) from the connexin-36 and
// connexin-43 items of both segments (density from the pre segment's), Cx43's Vj gate
// and the slow gate
__device__ __forceinline__ float gj_g_eff(const NetDev& d, uint32_t gp, uint32_t gq, float m_slow, float Vj) {
    const uint32_t N = d.n_seg, NI = d.n_items;
    float g_gap_ps = 0.0f;
    for (int cx = 0; cx < 2; cx++) {
        const float gamma = cx == 0 ? 14.0f : 100.0f;
        float density = 0.0f;
        float f = 1.0f;
        const uint32_t qp = d.seg_cx[(size_t)cx * N + gp];
        if (qp != UINT32_MAX) {
            density = d.it_den[qp];
            f = (float)((double)f * ((double)d.it_st[qp] * (double)d.it_st[(size_t)4 * NI + qp]));
        }
        const uint32_t qq = d.seg_cx[(size_t)cx * N + gq];
        if (qq != UINT32_MAX) f = (float)((double)f * ((double)d.it_st[qq] * (double)d.it_st[(size_t)4 * NI + qq]));
        if (cx == 1) {
            const float vj_abs = Vj < 0.0f ? -Vj : Vj;
            const float f_vj = (float)(1.0f / (1.0f + dm_exp((double)((vj_abs - 40.0f) / 5.0f))));
            f *= f_vj;
        }
        if (f < 0.01f) f = 0.01f;
        g_gap_ps += density * f * gamma;
    }
    return g_gap_ps * 1e-3f * (1.0f - m_slow);
}

// After step 3: the junctions' state as the post sides left it becomes the next
// tick's starting state.
__global__ void k_gj_commit(NetDev d) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < d.n_gj; g += gridDim.x * blockDim.x) {
        d.gj_dep[g] = d.gj_dep_new[g];
        d.gj_flt[g] = d.gj_flt_new[g];
    }
}

__device__ __forceinline__ void log_release(const NetDev& d, uint32_t k, unsigned long long tick, float amt,
                                         uint32_t slot) {
    const uint32_t at = atomicAdd(d.ev_n, 1u);
    if (at < d.ev_cap) d.ev_buf[at] = make_uint4(k, (uint32_t)tick, __float_as_uint(amt), slot);
}

// kX: the network has release modulators, eCB, glia or gap junctions; the plain
// instantiation leaves their code (and registers) out.
// Step 3's presynaptic half of synapse k (simulation_host.cpp:322-460): delayed
// arrivals, RRP recovery, bouton Ca2+, the Ca2+-dependent release and its delay slot.
// It reads the presynaptic segment's record and the synapse's own state only, so the
// synapses can take it in any order: networks without release modulators, eCB, glia
// and gap junctions run it for all synapses at once (k_release) before the per-segment
// half; the others run it in the segment's synapse loop.
template <bool kX>
__device__ __forceinline__ void presyn_step(const NetDev& d, uint32_t k, uint32_t K, unsigned long long tick, float dt,
                                            float& cleft, float& cleft_e, float& rrp, float& rrp_max, float& bouton,
                                            uint8_t& refr, uint8_t& sf, int& ntt) {
    const uint32_t pre = d.sy_pre[k];
    const float4 pr = d.pre_rec[pre];
    sf = d.sy_flags[k];
    ntt = sf >> 4;
    cleft = d.sy_cleft[k];
    if (kX && d.sy_cleft_ecb) cleft_e = d.sy_cleft_ecb[k];
    const float delay = d.sy_delay[k];
    // delayed releases (delay_buffer.h:31-44)
    if ((d.flags & NF_DELAY) && delay > 0.0f) {
        for (int q = 0; q < 4; q++) {
            unsigned long long arr = d.dl_arr[(size_t)q * K + k];
            if (arr == 0) continue;
            if (arr <= tick) {
                cleft += d.dl_amt[(size_t)q * K + k];
                if (d.ev_buf) log_release(d, k, tick, d.dl_amt[(size_t)q * K + k], q);
                d.dl_arr[(size_t)q * K + k] = 0;
            }
        }
    }
    // RRP recovery (kernel_dispatch.h:612-630); no CaMKII/calcineurin modifiers
    rrp_max = d.sy_rrp_max[k];
    if (rrp_max > 0.0f) rrp = d.sy_rrp[k];
    if (!(rrp_max <= 0.0f || rrp >= rrp_max)) {
        float ca_pre = d.pre_ext[pre].z;
        float ca_f = ca_pre / (0.0005f + ca_pre);
        float priming = d.sy_rrp_rec[k] + 0.0f * 0.02f + 0.0f * 0.01f;
        priming *= ca_f;
        float rec = (rrp_max - rrp) * priming * dt;
        rrp += rec;
        if (rrp > rrp_max) rrp = rrp_max;
    }
    // bouton Ca2+ (modifier_helpers.h:764-806)
    bouton = d.sy_bouton[k];
    const float pre_area = d.sy_pre_area[k];
    {
        const float g_K = d.sy_gK[k], g_Na = d.sy_gNa[k];
        float V_bouton = pr.x;
        if (g_K > 0.0f || g_Na > 0.0f) {
            float4 ex = d.pre_ext[pre];
            float koe = d.pre_ext2[pre];
            float E_K = dp_nernst(ex.y, koe, 1.0f);
            float E_Na = dp_nernst(ex.x, ex.w, 1.0f);
            V_bouton = (float)((300.0f * (double)pr.x + g_K * E_K + g_Na * E_Na) / (300.0f + g_K + g_Na));
        }
        float cav21_dens = 0.0f, mm = 0.0f, h = 0.0f;
        if (pr.z != 0.0f) {
            cav21_dens = pr.z;
            float m_inf = cav21_m_inf(V_bouton);
            float h_inf = cav21_h_inf(V_bouton, bouton * MM_TO_UM);
            mm = m_inf;
            h = (float)(h_inf + ((double)pr.w - h_inf) * dm_exp(-dt / 300.0f));
        }
        float cav21_open = mm * mm * h;
        double P_single = dp_ghk_P(15.0f, 2.0f, GHK_CBAR_CA_MM);
        double flux = dp_ghk_div(V_bouton, bouton, (double)pr.y);
        double I_A = P_single * flux * (cav21_dens * pre_area) * cav21_open;
        float I_Ca = (float)(I_A * A_TO_PA);
        bouton = (float)(bouton - I_Ca * dt * 1000.0f / (2.0f * FARADAY_CONST * 0.1f));
        bouton += (0.0001f - bouton) * dt / 5.0f;
        if (bouton < 0.0f) bouton = 0.0f;
    }
    // Ca2+-dependent release (simulation_host.cpp:421-460)
    refr = d.sy_refr[k];
    if (refr == 0) {
        float Ca_uM = bouton * MM_TO_UM;
        float ca_act = dm_pow(Ca_uM, 4.0f) / (dm_pow(Ca_uM, 4.0f) + dm_pow(10.0f, 4.0f));
        float p = d.sy_prel[k] * ca_act;
        // release modulators of the autoreceptors, in autoreceptor order
        // (kernel_dispatch.h:575-604, receptors_biological.cpp:428-509); the
        // bouton channels take the dispatch's default factor 1
        if (kX && d.md_off) {
            const uint32_t m1 = d.md_off[k + 1];
            for (uint32_t mi = d.md_off[k]; mi < m1; mi++) {
                const uint32_t code = d.md_code[mi];
                const uint32_t kind = code >> 4;
                const int mnt = (int)(code & 15u);
                const float c = mnt == ntt ? cleft : (mnt == 9 ? cleft_e : 0.0f);
                const float activation = c / (c + 0.5f);
                const double scale = d.md_scale[mi];
                float f;
                if (kind == 3) {
                    f = (float)(1.0f + (double)(0.3f * activation) * scale);
                } else {
                    float s0 = d.md_st[mi];
                    s0 = (float)((double)s0 + ((double)activation - (double)s0) * (double)dt /
                                 (kind == 1 ? 50.0 : 30.0));
                    d.md_st[mi] = s0;
                    f = (kind == 1) ? (float)(1.0f - (double)0.7f * (double)s0 * scale)
                                    : (float)(1.0f + (double)0.5f * (double)s0 * scale);
                }
                p *= f;
            }
        }
        uint32_t vbits = (uint32_t)(long long)((double)pr.x * 1000.0f);
        uint32_t seed = d.sy_id[k] ^ (uint32_t)tick ^ vbits;
        if (xorshift32_rnd(seed) < p) {
            const float amt = d.sy_amt[k];
            float release_amt;
            if (rrp_max <= 0.0f) release_amt = amt * p;
            else {
                float avail = amt;
                if (avail > rrp) avail = rrp;
                release_amt = avail * p;
                rrp -= release_amt;
                if (rrp < 0) rrp = 0;
            }
            unsigned long long delay_ticks = (delay <= 0.0f || dt <= 0.0f) ? 0ull
                : (unsigned long long)((delay / dt) + 0.5f);
            if (delay_ticks > 0) {
                for (int q = 0; q < 4; q++) {
                    if (d.dl_arr[(size_t)q * K + k] == 0) {
                        d.dl_arr[(size_t)q * K + k] = tick + delay_ticks;
                        d.dl_amt[(size_t)q * K + k] = release_amt;
                        d.dl_nt[(size_t)q * K + k] = (uint8_t)ntt;
                        break;
                    }
                }
            } else {
                cleft += release_amt;
                if (d.ev_buf) log_release(d, k, tick, release_amt, 4);
            }
            refr = (uint8_t)(uint32_t)(20.0f / dt + 0.5f);
        }
    }
}

// The presynaptic half of every synapse of a network without release modulators, eCB,
// glia or gap junctions, one thread per synapse; k_synapse<false> reads the cleft,
// refractory count, bouton Ca2+ and RRP it leaves.
__global__ void __launch_bounds__(256) k_release(NetDev d, float dt, unsigned long long tick) {
    if (d.clock) tick = d.clock[0];
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.n_syn) return;
    float cleft = 0.0f, cleft_e = 0.0f, rrp = 0.0f, rrp_max = 0.0f, bouton = 0.0f;
    uint8_t refr = 0, sf = 0;
    int ntt = 0;
    presyn_step<false>(d, k, d.n_syn, tick, dt, cleft, cleft_e, rrp, rrp_max, bouton, refr, sf, ntt);
    d.sy_cleft[k] = cleft;
    d.sy_refr[k] = refr;
    d.sy_bouton[k] = bouton;
    if (rrp_max > 0.0f) d.sy_rrp[k] = rrp;
}

template <bool kX>
__global__ void __launch_bounds__(256, 4)
k_synapse(NetDev d, float dt, unsigned long long tick, int first_tick) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t N = d.n_seg;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    if (d.clock) {
        tick = d.clock[0];
        first_tick = d.clock[1] == 0 ? 1 : 0;
    }
    // every lane of the warp takes part in the slice ballots below, valid or not
    const bool valid = t < N;
    const uint32_t i = valid ? d.th_seg[t] : 0u;
    const uint32_t cnt = valid ? (uint32_t)d.th_cnt[t] : 0u;
    const uint32_t maxc = __reduce_max_sync(0xFFFFFFFFu, cnt);
    const uint8_t sfl = valid ? d.sflags[i] : (uint8_t)0;
    const bool syn_on = (d.flags & NF_SYNAPSES) != 0;
    // the neurotransmitters a synapse can deliver: glutamate, GABA, glycine (0, 1, 7)
    float nt_glu = (sfl & SF_NMDA) ? 1.0f : 0.0f;   // bath NMDA (simulation_host.cpp:337-340)
    float nt_gaba = 0.0f, nt_gly = 0.0f, nt_ecb = 0.0f;
    // the segment's eCB-synthesis modifier (its first), whose state[0] each of its
    // synapses draws on in order (simulation_host.cpp:578-589)
    const uint32_t ecb_q = (kX && valid && d.seg_ecb_item) ? d.seg_ecb_item[i] : UINT32_MAX;
    float ecb_st = ecb_q != UINT32_MAX ? d.it_st[ecb_q] : 0.0f;
    double ib = valid ? d.ibuf[i] : 0.0;
    DSeg s;
    s.V = valid ? d.V[i] : 0.0f;
    bool touched = false;
    if (cnt > 0) {
#pragma unroll
        for (int q = 0; q < 7; q++) s.in[q] = d.ion_in[(size_t)q * N + i];
#pragma unroll
        for (int q = 0; q < 4; q++) s.out[q] = d.ion_out[(size_t)q * N + i];
        s.out[4] = s.out[5] = s.out[6] = 0.0f;
        s.atp = 0.0f;
        s.area = d.area[i];
        s.vol = d.vol[i];
        ghk_cache_fill(s.gc, s.V);   // V_m is constant through step 3
    }
    const uint32_t K = d.n_syn;
    const uint32_t NR = d.n_rec;
    uint32_t base = 0, rbase = 0;
    if (maxc > 0) {
        base = d.w_off[t >> 5];
        rbase = d.rw_off[t >> 5];
    }
    for (uint32_t kk = 0; kk < maxc; kk++) {
        const bool act = cnt > kk;
        const uint32_t n_act = __popc(__ballot_sync(0xFFFFFFFFu, act));
        const uint32_t k = base + lane;   // this lane's synapse in the slice (when act)
        // a gap junction's side (simulation_host.cpp:373-402) or a chemical synapse
        const uint32_t gjv = (kX && act && d.sy_gj) ? d.sy_gj[k] : UINT32_MAX;
        const bool chem = act && gjv == UINT32_MAX;
        float cleft = 0.0f, cleft_e = 0.0f, rrp = 0.0f, rrp_max = 0.0f, bouton = 0.0f;
        uint8_t refr = 0, sf = 0;
        int ntt = 0;
        uint32_t n_rc = 0;
        if (chem) {
            if (kX) {
                presyn_step<true>(d, k, K, tick, dt, cleft, cleft_e, rrp, rrp_max, bouton, refr, sf, ntt);
            } else {   // k_release ran the presynaptic half
                sf = d.sy_flags[k];
                ntt = sf >> 4;
                cleft = d.sy_cleft[k];
                refr = d.sy_refr[k];
            }
            // NT into the postsynaptic segment (simulation_host.cpp:463-465)
            if (ntt == 0) nt_glu += cleft;
            else if (ntt == 1) nt_gaba += cleft;
            else nt_gly += cleft;
            if (kX) nt_ecb += cleft_e;
            // glial capture (simulation_host.cpp:467-487): a share of the transmitter
            // goes to the glial segment nearest the post segment in z; k_glia adds the
            // shares to the glial segments in synapse order
            if (kX && d.gl_cap) {
                float cap = 0.0f;
                if (cleft > 0.0f) {
                    const float tau = d.sy_tauc[k] > 0.0f ? d.sy_tauc[k] : 5.0f;
                    cap = (float)((double)cleft * (1.0 - dm_exp(-dt / tau)));
                    cleft -= cap;
                }
                d.gl_cap[k] = cap;
            }
            n_rc = d.rc_cnt[k];
        }
        // receptors (simulation_host.cpp:490-500), j-th receptors of the slice side by side
        float I_syn = 0.0f;
        const float post_area = act ? d.sy_post_area[k] : 0.0f;
        const float scale = act ? d.sy_scale[k] : 0.0f;
        const uint32_t maxr = __reduce_max_sync(0xFFFFFFFFu, n_rc);
        for (uint32_t j = 0; j < maxr; j++) {
            const uint32_t has = __ballot_sync(0xFFFFFFFFu, n_rc > j);
            if (n_rc > j) {
                const uint32_t r = rbase + __popc(has & lt_mask);
                DMod m;
                m.den = d.rc_den[r];
                m.st[0] = d.rc_st[r];
                m.st[1] = d.rc_st[(size_t)NR + r];
                m.st[2] = d.rc_st[(size_t)2 * NR + r];
                m.st[3] = m.st[4] = m.st[5] = m.st[6] = 0.0f;
                m.area = (post_area > 0.0f) ? post_area : s.area;
                m.av = d.rc_av[r];
                const int kind = receptor_kind(d.rc_type[r]);
                const float ntr = kind <= 1 ? nt_glu : (kind == 2 ? nt_gaba : nt_gly);
                I_syn = (float)(I_syn + receptor_current(gRec[kind], m, s, dt, ntr, scale));
                d.rc_st[r] = m.st[0];
                d.rc_st[(size_t)NR + r] = m.st[1];
                d.rc_st[(size_t)2 * NR + r] = m.st[2];
                touched = true;
            }
            rbase += __popc(has);
        }
        if (act && gjv != UINT32_MAX) {
            // gap junction (simulation_host.cpp:373-402): both sides compute the same
            // current from the segments' state as step 3 began (V is constant through
            // step 3, and the builder refuses networks where an earlier synapse could
            // move either segment's Ca2+); the post side records the junction's state
            const uint32_t g = gjv & 0x7FFFFFFFu;
            const uint32_t gp = d.gj_pre[g], gq = d.gj_post[g];
            const float Vj = (float)((double)d.pre_rec[gp].x - (double)d.pre_rec[gq].x);
            const float m_slow = gj_cam_update(d.gj_dep[g], d.pre_ext[gp].z, d.pre_ext[gq].z, dt);
            const float g_eff = gj_g_eff(d, gp, gq, m_slow, Vj);
            const float I_gap_raw = g_eff * Vj;
            const float delay = d.gj_delay[g];
            float I = I_gap_raw;
            if (delay > 0.001f) {
                float I_filtered = d.gj_flt[g];
                I_filtered += (I_gap_raw - I_filtered) * dt / delay;
                I = I_filtered;
            }
            if (gjv >> 31) {
                ib -= I;
            } else {
                ib += I;
                d.gj_dep_new[g] = m_slow;
                if (delay > 0.001f) d.gj_flt_new[g] = I;
            }
        }
        if (chem) {
            ib += I_syn;
            // spine Ca2+ (modifier_helpers.h:808-817)
            float spine = d.sy_spine[k];
            {
                float I_abs = I_syn < 0.0f ? -I_syn : I_syn;
                float I_Ca = I_abs * 0.1f;
                float influx = (float)(I_Ca * dt * 1000.0f / (2.0f * FARADAY_CONST * 0.05f * 100.0f));
                spine += influx;
                spine += (0.0001f - spine) * dt / 50.0f;
                if (spine < 0.0f) spine = 0.0f;
            }
            // clearance (simulation_host.cpp:505-510)
            const auto clear_f = dm_exp(-dt / d.sy_tauc[k]);
            if (!kX || !d.gl_cap) {   // with glia, they take glutamate, GABA and glycine instead
                cleft *= clear_f;
                if (cleft < 0.0f) cleft = 0.0f;
            }
            if (kX) {
                cleft_e *= clear_f;
                if (cleft_e < 0.0f) cleft_e = 0.0f;
            }
            // BCM threshold, spine CaMKII/calcineurin, weight (simulation_host.cpp:527-576)
            float facil = d.sy_facil[k];
            {
                float Ca_uM = spine * 1000.0f;
                float Ca_sq = Ca_uM * Ca_uM;
                facil += (Ca_sq - facil) * dt / 300000.0f;
                if (facil < 0.0f) facil = 0.0f;
            }
            float camkii = d.sy_camkii[k], calcn = d.sy_calcn[k];
            {
                float Ca_uM = spine * MM_TO_UM;
                float Ca4 = Ca_uM * Ca_uM * Ca_uM * Ca_uM;
                float camkii_inf = Ca4 / (Ca4 + 1.0f + 1e-9f);
                camkii += (camkii_inf - camkii) * dt / 2000.0f;
                if (camkii < 0.0f) camkii = 0.0f;
                if (camkii > 1.0f) camkii = 1.0f;
                float Ca2 = Ca_uM * Ca_uM;
                float calcineurin_inf = Ca2 / (Ca2 + 0.05f * 0.05f + 1e-9f);
                calcn += (calcineurin_inf - calcn) * dt / 300.0f;
                if (calcn < 0.0f) calcn = 0.0f;
                if (calcn > 1.0f) calcn = 1.0f;
            }
            float weight = d.sy_weight[k];
            {
                float dw = 0.0f;
                if (camkii > 0.0f) dw += 0.0003f * camkii * dt;
                float pp1_active = 0.5f;
                if (calcn > 0.0f) dw -= 0.0001f * calcn * pp1_active * dt;
                if (sf & 1) dw = -dw;
                weight += dw;
                if (weight != weight) weight = 0.5f;
                if (facil != facil) facil = 0.0f;
                if (weight < 0.01f) weight = 0.01f;
                if (weight > 10.0f) weight = 10.0f;
            }
            // eCB retrograde release (simulation_host.cpp:578-589)
            if (ecb_q != UINT32_MAX) {
                const float ecb = ecb_st;
                if (ecb > 0.0f) {
                    cleft_e += ecb * 0.1f * dt;
                    ecb_st = (float)((double)ecb_st * (double)0.9f);
                }
            }
            if (refr > 0) refr--;
            d.sy_cleft[k] = cleft;
            if (kX && d.sy_cleft_ecb) d.sy_cleft_ecb[k] = cleft_e;
            d.sy_refr[k] = refr;
            if (kX) d.sy_bouton[k] = bouton;   // else k_release stored it
            d.sy_spine[k] = spine;
            d.sy_camkii[k] = camkii;
            d.sy_calcn[k] = calcn;
            d.sy_facil[k] = facil;
            d.sy_weight[k] = weight;
            if (kX && rrp_max > 0.0f) d.sy_rrp[k] = rrp;
        }
        base += n_act;
    }
    if (ecb_q != UINT32_MAX) d.it_st[ecb_q] = ecb_st;
    if (!valid) return;
    // step 4: membrane update (simulation_host.cpp:596-649)
    float V = s.V;
    if (ib != ib) ib = 0.0f;
    if (ib > 10000.0f) ib = 10000.0f;
    if (ib < -10000.0f) ib = -10000.0f;
    const float C_m = d.cm[i];
    const float prev_V = V;
    float dV = (float)(ib / C_m * dt);
    if (dV > 50.0f) dV = 50.0f;
    if (dV < -50.0f) dV = -50.0f;
    V = (float)((double)V + dV);
    if (prev_V <= -40.0f && V > -40.0f) d.spike_count[i]++;
    if (d.vc_off) {
        for (uint32_t q = d.vc_off[i]; q < d.vc_off[i + 1]; q++)
            if (tick >= d.vc_start[q] && tick < d.vc_end[q]) V = d.vc_target[q];
    }
    if (V != V) V = -65.0f;
    else {
        if (V < -120.0f) V = -120.0f;
        if (V > 150.0f) V = 150.0f;
    }
    d.V[i] = V;
    if (touched) {
#pragma unroll
        for (int q = 0; q < 7; q++) d.ion_in[(size_t)q * N + i] = s.in[q];
    }
    if (syn_on) {
        const uint32_t mask = first_tick ? 0x7FFFu : d.nt_used_mask;
#pragma unroll
        for (int q = 0; q < 15; q++)
            if ((mask >> q) & 1u)
                d.nt[(size_t)q * N + i] = q == 0 ? nt_glu : (q == 1 ? nt_gaba : (q == 7 ? nt_gly : (q == 9 ? nt_ecb : 0.0f)));
    } else if (sfl & SF_NMDA) {
        d.nt[i] = 1.0f;
    }
}

cudaError_t prepare_synapse(cudaStream_t stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (g_rec_ready[dev]) return cudaSuccess;
    k_init_receptors<<<1, 1, 0, stream>>>();
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) g_rec_ready[dev] = true;
    return e;
}

// The glial segments' transmitter after step 3: what k_synapse left there (the reset,
// no synapse targets a glial segment) plus each capture, in original synapse order
// (simulation_host.cpp:480-481).  One thread per glial segment.
__global__ void k_glia(NetDev d) {
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= d.n_glia) return;
    const uint32_t g = d.gl_seg[gi];
    const uint32_t N = d.n_seg;
    float glu = d.nt[g], gaba = d.nt[(size_t)1 * N + g], gly = d.nt[(size_t)7 * N + g];
    for (uint32_t x = d.gl_off[gi]; x < d.gl_off[gi + 1]; x++) {
        const uint32_t k = d.gl_syn[x];
        const float c = d.gl_cap[k];
        const int ntt = d.sy_flags[k] >> 4;
        if (ntt == 0) glu += c;
        else if (ntt == 1) gaba += c;
        else gly += c;
    }
    d.nt[g] = glu;
    d.nt[(size_t)1 * N + g] = gaba;
    d.nt[(size_t)7 * N + g] = gly;
}

// Launches of steps 3 and 4 per tick, as launch_synapse issues them.
uint32_t synapse_launches(const NetDev& dev) {
    const bool extras = dev.syn_extras != 0;
    return 1u + ((!extras && dev.n_syn) ? 1u : 0u) + (dev.n_glia ? 1u : 0u) + (dev.n_gj ? 1u : 0u);
}

cudaError_t launch_synapse(const NetDev& dev, float dt, unsigned long long tick, int first_tick,
                           cudaStream_t stream) {
    const bool extras = dev.syn_extras != 0;
    if (extras) k_synapse<true><<<(dev.n_seg + 255) / 256, 256, 0, stream>>>(dev, dt, tick, first_tick);
    else {
        if (dev.n_syn) k_release<<<(dev.n_syn + 255) / 256, 256, 0, stream>>>(dev, dt, tick);
        k_synapse<false><<<(dev.n_seg + 255) / 256, 256, 0, stream>>>(dev, dt, tick, first_tick);
    }
    if (dev.gl_cap) k_glia<<<(dev.n_glia + 127) / 128, 128, 0, stream>>>(dev);
    if (dev.sy_gj) k_gj_commit<<<(dev.n_gj + 255) / 256 < 1184 ? (dev.n_gj + 255) / 256 : 1184, 256, 0, stream>>>(dev);
    return cudaGetLastError();
}

// The device clock of captured tick loops: [0] the tick, [1] ticks run so far.
__global__ void k_set_clock(unsigned long long* clock, unsigned long long tick, unsigned long long ticks_run) {
    clock[0] = tick;
    clock[1] = ticks_run;
}

__global__ void k_advance_clock(unsigned long long* clock) {
    clock[0] += 1;
    clock[1] += 1;
}

cudaError_t launch_set_clock(unsigned long long* clock, unsigned long long tick, unsigned long long ticks_run,
                             cudaStream_t stream) {
    k_set_clock<<<1, 1, 0, stream>>>(clock, tick, ticks_run);
    return cudaGetLastError();
}

cudaError_t launch_advance_clock(unsigned long long* clock, cudaStream_t stream) {
    k_advance_clock<<<1, 1, 0, stream>>>(clock);
    return cudaGetLastError();
}

}  // namespace bnc
