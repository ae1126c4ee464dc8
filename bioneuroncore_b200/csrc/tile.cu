// tile.cu -- step 1 of a tick (modifier currents and stimuli) and the tick launcher.
//
// One tick of the reference (simulation_host.cpp:174-657) is three launches:
//
//  k_modifiers (this file; one CTA per tile of whole neurons, segment state resident
//             in shared memory)
//    step 1   modifier currents: items grouped into phases (each phase holds at most
//             one modifier per segment, phases follow every segment's slot order) and
//             by type within a phase, so warps run one channel model at a time;
//             current stimuli; I_buffer.  Writes the segment state, I_buffer and the
//             Cav2.1 gate the synapses read.
//  k_diffusion (diffuse.cu) step 2.5 electrodiffusion and the presynaptic record.
//  k_synapse (synapse.cu)   steps 3 and 4: synapses in original order per
//             postsynaptic segment, then the membrane update.
#define BNC_MATH_OUTLINE 1   // 26 channel models in one kernel: keep exp/log out of line
#include <cuda_runtime.h>
#include "net.h"
#include "physics.cuh"

namespace bnc {

// state indices each modifier type updates every tick (read + write)
__constant__ uint8_t c_dyn_mask[256];
// state indices each type reads as parameters (default when 0)
__constant__ uint8_t c_par_mask[256];


struct TileSmem {
    double *itot, *vol;
    float *V, *in, *out, *atp, *c21d, *c21h, *area;
    // per-segment GHK factors
    double *gA1, *ge1, *gD1, *gA2, *ge2, *gD2;
    float *gV;
    uint8_t *gm1, *gm2;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline size_t tile_layout(uint32_t S, unsigned char* base, TileSmem* t) {
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align16(off + bytes); return base ? base + o : nullptr; };
    unsigned char* p;
    p = take(8 * (size_t)S); if (t) t->itot = (double*)p;
    p = take(8 * (size_t)S); if (t) t->vol = (double*)p;
    p = take(4 * (size_t)S); if (t) t->V = (float*)p;
    p = take(4 * 7 * (size_t)S); if (t) t->in = (float*)p;
    p = take(4 * 7 * (size_t)S); if (t) t->out = (float*)p;
    p = take(4 * (size_t)S); if (t) t->atp = (float*)p;
    p = take(4 * (size_t)S); if (t) t->c21d = (float*)p;
    p = take(4 * (size_t)S); if (t) t->c21h = (float*)p;
    p = take(4 * (size_t)S); if (t) t->area = (float*)p;
    p = take(8 * (size_t)S); if (t) t->gA1 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->ge1 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->gD1 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->gA2 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->ge2 = (double*)p;
    p = take(8 * (size_t)S); if (t) t->gD2 = (double*)p;
    p = take(4 * (size_t)S); if (t) t->gV = (float*)p;
    p = take((size_t)S); if (t) t->gm1 = (uint8_t*)p;
    p = take((size_t)S); if (t) t->gm2 = (uint8_t*)p;
    return off;
}

size_t tile_smem_bytes(uint32_t max_segs) {
    return tile_layout(max_segs, nullptr, nullptr);
}

template <int kMinCtas>
__global__ void __launch_bounds__(kTileThreads, kMinCtas)
k_modifiers(NetDev d, float dt, unsigned long long tick, uint32_t S) {
    extern __shared__ __align__(16) unsigned char smem[];
    TileSmem t;
    tile_layout(S, smem, &t);
    const int tid = threadIdx.x;
    const int nth = blockDim.x;
    const uint32_t tile = blockIdx.x;
    const uint32_t N = d.n_seg;
    if (d.clock) tick = d.clock[0];
    const uint32_t s0 = d.tile_seg_beg[tile];
    const int ns = (int)(d.tile_seg_beg[tile + 1] - s0);

    // ---- load tile state ----
    for (int i = tid; i < ns; i += nth) {
        uint32_t g = s0 + i;
        t.V[i] = d.V[g];
#pragma unroll
        for (int q = 0; q < 7; q++) {
            t.in[q * S + i] = d.ion_in[(size_t)q * N + g];
            t.out[q * S + i] = d.ion_out[(size_t)q * N + g];
        }
        t.atp[i] = d.atp[g];
        t.area[i] = d.area[g];
        t.vol[i] = d.vol[g];
        t.itot[i] = 0.0;
        float2 c = d.cav21_static[g];
        t.c21d[i] = c.x;
        t.c21h[i] = c.y;
    }
    for (int i = tid; i < ns; i += nth) {   // per-segment GHK factors for step 1
        GhkCache c;
        ghk_cache_fill(c, t.V[i]);
        t.gV[i] = c.Vc; t.gm1[i] = c.m1; t.gm2[i] = c.m2;
        t.gA1[i] = c.A1; t.ge1[i] = c.e1; t.gD1[i] = c.D1;
        t.gA2[i] = c.A2; t.ge2[i] = c.e2; t.gD2[i] = c.D2;
    }
    __syncthreads();

    // ---- step 1: modifier currents (simulation_host.cpp:234-303) ----
    const uint32_t P = d.n_phases;
    const uint32_t NI = d.n_items;
    for (uint32_t p = 0; p < P; p++) {
        const uint32_t b = d.phase_off[(size_t)tile * (P + 1) + p];
        const uint32_t e = d.phase_off[(size_t)tile * (P + 1) + p + 1];
        if (b == e) continue;   // empty for this tile (uniform across the CTA)
        for (uint32_t q = b + tid; q < e; q += nth) {
            const uint32_t meta = d.it_meta[q];
            const int ls = (int)(meta & 0xFFFFu);
            const uint8_t type = (uint8_t)((meta >> 16) & 0xFFu);
            const uint8_t fl = (uint8_t)(meta >> 24);
            DSeg s;
            s.V = t.V[ls];
#pragma unroll
            for (int k = 0; k < 7; k++) { s.in[k] = t.in[k * S + ls]; s.out[k] = t.out[k * S + ls]; }
            s.atp = t.atp[ls];
            s.area = t.area[ls];
            s.vol = t.vol[ls];
            s.gc.Vc = t.gV[ls]; s.gc.m1 = t.gm1[ls]; s.gc.m2 = t.gm2[ls];
            s.gc.A1 = t.gA1[ls]; s.gc.e1 = t.ge1[ls]; s.gc.D1 = t.gD1[ls];
            s.gc.A2 = t.gA2[ls]; s.gc.e2 = t.ge2[ls]; s.gc.D2 = t.gD2[ls];
            DMod m;
            m.den = d.it_den[q];
            m.area = s.area;
            m.av = (fl & 2) ? (uint8_t)((fl >> 2) & 7) : (uint8_t)0;
            uint32_t rm = c_dyn_mask[type] | ((fl & 1) ? c_par_mask[type] : 0u);
            if (fl & 2) rm |= (1u << m.av) & 0x7Fu;
#pragma unroll
            for (int k = 0; k < 7; k++) m.st[k] = ((rm >> k) & 1u) ? d.it_st[(size_t)k * NI + q] : 0.0f;
            float glu = 0.0f, gaba = 0.0f, gly = 0.0f;
            if (type == 8 || type == 9) glu = d.nt[s0 + ls];
            else if (type == 11) gaba = d.nt[(size_t)1 * N + s0 + ls];
            else if (type == 12) gly = d.nt[(size_t)7 * N + s0 + ls];
            double I = dp_dispatch(type, m, s, dt, glu, gaba, gly, (fl & 3) == 0);
            if (s.V != t.V[ls]) {   // a sodium channel clamped V to +-200 mV
                GhkCache c;
                ghk_cache_fill(c, s.V);
                t.gV[ls] = c.Vc; t.gm1[ls] = c.m1; t.gm2[ls] = c.m2;
                t.gA1[ls] = c.A1; t.ge1[ls] = c.e1; t.gD1[ls] = c.D1;
                t.gA2[ls] = c.A2; t.ge2[ls] = c.e2; t.gD2[ls] = c.D2;
            }
            t.V[ls] = s.V;
#pragma unroll
            for (int k = 0; k < 7; k++) { t.in[k * S + ls] = s.in[k]; t.out[k * S + ls] = s.out[k]; }
            t.atp[ls] = s.atp;
            t.itot[ls] += I;
            const uint32_t wm = c_dyn_mask[type];
#pragma unroll
            for (int k = 0; k < 7; k++) if ((wm >> k) & 1u) d.it_st[(size_t)k * NI + q] = m.st[k];
            if (type == 140) { t.c21d[ls] = m.den; t.c21h[ls] = m.st[1]; }
        }
        __syncthreads();
    }
    // current stimuli (simulation_host.cpp:189-209, 247-258): expiry, then add in order
    if (d.cs_off) {
        for (int i = tid; i < ns; i += nth) {
            uint32_t g = s0 + i;
            double I = t.itot[i];
            for (uint32_t k = d.cs_off[g]; k < d.cs_off[g + 1]; k++) {
                if (!d.cs_alive[k]) continue;
                unsigned long long dur = (unsigned long long)(d.cs_dur[k] / dt);
                unsigned long long st = d.cs_start[k];
                if (tick >= st + dur) { d.cs_alive[k] = 0; continue; }
                if (tick >= st && tick < st + dur) I += d.cs_amp[k];
            }
            t.itot[i] = I;
        }
        __syncthreads();
    }

    // ---- output: state after step 1, I_buffer, the Cav2.1 gate of the record ----
    for (int i = tid; i < ns; i += nth) {
        uint32_t g = s0 + i;
        d.V[g] = t.V[i];
#pragma unroll
        for (int q = 0; q < 7; q++) {
            d.ion_in[(size_t)q * N + g] = t.in[q * S + i];
            d.ion_out[(size_t)q * N + g] = t.out[q * S + i];
        }
        d.atp[g] = t.atp[i];
        d.ibuf[g] = t.itot[i];
        d.c21_cur[g] = make_float2(t.c21d[i], t.c21h[i]);
    }
}

static bool g_tables_ready[64] = {false};   // per device: constant memory is per context

static cudaError_t init_tables(cudaStream_t stream) {
    int dev = 0;
    cudaError_t ge = cudaGetDevice(&dev);
    if (ge != cudaSuccess) return ge;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (g_tables_ready[dev]) return cudaSuccess;
    uint8_t dyn[256] = {0}, par[256] = {0};
    dyn[1] = 0x03; par[1] = 0x1C;
    dyn[8] = 0x03; dyn[9] = 0x05; dyn[11] = 0x03; dyn[12] = 0x03;
    dyn[85] = 0x0B; par[85] = 0x34;
    par[98] = 0x06; par[100] = 0x06;
    dyn[102] = 0x02; par[102] = 0x1D;
    dyn[103] = 0x01; par[103] = 0x38;
    dyn[104] = 0x01; par[104] = 0x06;
    dyn[105] = 0x01; par[105] = 0x3E;
    par[106] = 0x08; par[107] = 0x03;
    dyn[112] = 0x01; par[112] = 0x76;
    dyn[123] = 0x01; par[123] = 0x16;
    dyn[129] = 0x01; par[129] = 0x3E;
    par[133] = 0x01;
    dyn[140] = 0x03;
    dyn[141] = 0x03; par[141] = 0x20;
    dyn[142] = 0x03; par[142] = 0x20;
    dyn[150] = 0x07; par[150] = 0x20;
    dyn[200] = 0x03; par[200] = 0x7C;
    cudaError_t e = cudaMemcpyToSymbol(c_dyn_mask, dyn, sizeof(dyn));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_par_mask, par, sizeof(par));
    if (e == cudaSuccess) g_tables_ready[dev] = true;
    return e;
}

cudaError_t prepare_tick(const NetDev& dev, const NetHost& host, cudaStream_t stream) {
    (void)dev;
    cudaError_t e = init_tables(stream);
    if (e != cudaSuccess) return e;
    const size_t smem = tile_smem_bytes(host.max_tile_segs);
    if (smem > 48 * 1024) {
        e = host.opt.mod_ctas == 3
                ? cudaFuncSetAttribute(k_modifiers<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                : cudaFuncSetAttribute(k_modifiers<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    e = prepare_synapse(stream);
    if (e != cudaSuccess) return e;
    return prepare_diffusion(host, stream);
}

static void enqueue_modifiers(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                              cudaStream_t stream) {
    const uint32_t S = host.max_tile_segs;
    if (host.opt.mod_ctas == 3) k_modifiers<3><<<dev.n_tiles, kTileThreads, tile_smem_bytes(S), stream>>>(dev, dt, tick, S);
    else k_modifiers<2><<<dev.n_tiles, kTileThreads, tile_smem_bytes(S), stream>>>(dev, dt, tick, S);
}

cudaError_t launch_modifiers(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                             cudaStream_t stream) {
    cudaError_t e = prepare_tick(dev, host, stream);
    if (e != cudaSuccess) return e;
    enqueue_modifiers(dev, host, dt, tick, stream);
    return cudaGetLastError();
}

cudaError_t launch_diffusion(const NetDev& dev, const NetHost& host, float dt, cudaStream_t stream) {
    cudaError_t e = prepare_tick(dev, host, stream);
    if (e != cudaSuccess) return e;
    enqueue_diffusion(dev, host, dt, stream);
    return cudaGetLastError();
}

cudaError_t enqueue_tick(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick, int first_tick,
                         cudaStream_t stream) {
    enqueue_modifiers(dev, host, dt, tick, stream);
    enqueue_diffusion(dev, host, dt, stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_synapse(dev, dt, tick, first_tick, stream);
}

cudaError_t launch_tick(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick, int first_tick,
                        cudaStream_t stream) {
    cudaError_t e = prepare_tick(dev, host, stream);
    if (e != cudaSuccess) return e;
    return enqueue_tick(dev, host, dt, tick, first_tick, stream);
}

}  // namespace bnc
