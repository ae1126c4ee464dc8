// diffuse.cu -- step 2.5 of a tick, electrodiffusion (diffusion_kernel.h:115-364), and
// the write-back of the tick's segment state.
//
// One CTA per tile of whole components (the same tiles as the modifier kernel), one
// thread per segment and one per connection.  The 300 Jacobi sweeps of a tick (50 for
// phi_e, 5 x 50 for V_m) are latency chains, not bandwidth: each thread keeps its
// segment's stencil -- the incident connections in original connection order, the
// other endpoint, the coefficient -- in registers for all sweeps of a solve, so a
// sweep is a few independent shared-memory loads, the arithmetic and one barrier.
// Every gather sums the segment's incident connections in original connection order,
// the order of the reference's scatter loops, so results are bit-identical to them.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include "net.h"
#include "physics.cuh"

namespace bnc {

// valence, diffusion coefficient and bath concentration per ion (diffusion_kernel.h:23-33)
__constant__ float kNpZ[7] = {1.0f, 1.0f, 2.0f, -1.0f, 2.0f, -1.0f, 1.0f};
__constant__ float kDiffC[7] = {1.33f, 1.96f, 0.22f, 2.03f, 0.10f, 0.0f, 9.31f};
__constant__ float kBathIon[7] = {140.0f, 3.0f, 1.2f, 130.0f, 1.0f, 0.0f, 4.0e-5f};
__device__ float gNtD[15];   // Stokes-Einstein NT diffusion coefficients, set by k_init_ntd

// D = 1.33 * (23/M)^(1/3) (types.h:428-445, nt_diffusion_coeff); the 15th entry has no
// mass in the reference's table (0 -> 1)
__global__ void k_init_ntd() {
    const float mass[15] = {147.0f, 103.0f, 153.0f, 176.0f, 146.0f, 267.0f, 169.0f, 75.0f, 111.0f,
                            348.0f, 507.0f, 232.0f, 24.0f, 162.0f, 0.0f};
    for (int q = 0; q < 15; q++) {
        float ms = mass[q];
        if (ms < 1.0f) ms = 1.0f;
        gNtD[q] = 1.33f * dm_powf(23.0f / ms, 1.0f / 3.0f);   // powf: types.h:442
    }
}

static bool g_ntd_ready[64] = {false};   // per device

namespace {

// incidences held in registers per segment; segments with more use shared memory
constexpr int kDeg = 4;

// a / b rounded to nearest (the IEEE binary64 quotient) for a b that holds a float
// value (a 24-bit significand), given y = 1 / b rounded to nearest.  q0 = a * y is
// within 1.5 units in the last place of a / b; q0 + r * y with r = a - b * q0 (one fma,
// exact) differs from a / b by r * (y - 1/b), under 2^-103 |a / b|.  a - m * b is a
// nonzero multiple of 2^(exponent(a) - 77) for every rounding midpoint m of the binary64
// grid near a / b (m has 54 significant bits, b 24), so a / b lies at least
// 2^-79 |a / b| from any midpoint and fma(r, y, q0) rounds to the same neighbour.
// Zero, non-finite and very small quotients (where r could underflow) take the
// hardware division.  The gathers divide by the segment's volume (a float) every
// substep, ion and incidence: this replaces those divisions with a multiply and two
// fmas.
__device__ __forceinline__ double div_by_float(double a, double b, double y) {
    const double q0 = a * y;
    const double r = fma(-q0, b, a);
    const double aq = fabs(q0);
    if (aq >= 0x1p-900 && aq <= 0x1.fffffffffffffp+1023) return fma(r, y, q0);
    if (aq == 0.0) return q0;
    return a / b;
}

// a / b rounded to nearest in binary32, given y = 1 / b rounded to nearest (Markstein's
// correction, Markstein 1990, IBM J. Res. Dev. 34(1)): q0 = a * y is within an ulp of
// a / b, r = a - b * q0 is then exact (one fma), and fma(r, y, q0) is the correctly
// rounded quotient.  Operands are kept well inside the normal range (|a| in
// [2^-64, 2^64], |b| in [2^-32, 2^32], so q0 and r are normal); outside it the
// hardware division runs.  Used where one divisor serves many divisions (a Jacobi
// solve's diagonal, a segment's volume, a connection's length, the substep).
__device__ __forceinline__ bool div_rn_f_range_b(float b) {
    const float ab = fabsf(b);
    return ab >= 0x1p-32f && ab <= 0x1p32f;
}
__device__ __forceinline__ bool div_rn_f_range_a(float a) {
    const float aa = fabsf(a);
    return aa >= 0x1p-64f && aa <= 0x1p64f;
}
__device__ __forceinline__ float div_rn_f(float a, float b, float y) {
    if (div_rn_f_range_a(a) && div_rn_f_range_b(b)) {
        const float q0 = a * y;
        const float r = __fmaf_rn(-q0, b, a);
        return __fmaf_rn(r, y, q0);
    }
    return a / b;
}

// The same in binary64 (|b| and |q0| in [2^-500, 2^500]).
__device__ __forceinline__ double div_rn_d(double a, double b, double y) {
    const double q0 = a * y;
    const double aq = fabs(q0), ab = fabs(b);
    if (aq >= 0x1p-500 && aq <= 0x1p500 && ab >= 0x1p-500 && ab <= 0x1p500) {
        const double r = __fma_rn(-q0, b, a);
        return __fma_rn(r, y, q0);
    }
    return a / b;
}

// diffusion_kernel.h:108-113
__device__ __forceinline__ float sg_bernoulli(float x) {
    if (fabsf(x) < 1e-3f) return 1.0f - 0.5f * x;
    if (x > 50.0f) return 0.0f;
    if (x < -50.0f) return -x;
    return x / (dm_exp(x) - 1.0f);
}

// valence group of ion q (+1: 0, 1, 6; +2: 2, 4; -1: 3, 5) and the group's factor
// z * 0.03742f of the Scharfetter-Gummel argument, as kNpZ[q] * 0.03742f evaluates it
__device__ __forceinline__ int valence_group(int q) {
    return (q == 2 || q == 4) ? 1 : ((q == 3 || q == 5) ? 2 : 0);
}
__device__ __forceinline__ float valence_factor(int g) {
    return g == 0 ? 1.0f * 0.03742f : (g == 1 ? 2.0f * 0.03742f : -1.0f * 0.03742f);
}

struct DiffSmem {
    double *itot, *phiA, *phiB, *sig, *ed;
    float *V, *in, *out, *atp, *area, *cm, *vf, *vnA, *vnB, *nb;
    float *gax, *dve, *fl, *ie, *earea, *edist;
    float *coef;   // [7][E]: kDiffC[q] * area * dt_sub / dist of each connection
    uint16_t *incoff, *inc, *ea, *eb;
    uint16_t *gsrc;   // ghost g's index in the paired tile
    uint8_t *ei, *es;
};

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline size_t diff_layout(uint32_t S, uint32_t E, unsigned char* base, DiffSmem* t) {
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = al16(off + bytes); return base ? base + o : nullptr; };
    const size_t Ee = E ? E : 1, Ii = 2 * Ee;   // each connection sits in two incidence lists
    unsigned char* p;
    p = take(8 * (size_t)S); if (t) t->itot = (double*)p;
    p = take(8 * (size_t)S); if (t) t->phiA = (double*)p;
    p = take(8 * (size_t)S); if (t) t->phiB = (double*)p;
    p = take(8 * (size_t)S); if (t) t->sig = (double*)p;
    p = take(4 * (size_t)S); if (t) t->V = (float*)p;
    p = take(4 * 7 * (size_t)S); if (t) t->in = (float*)p;
    p = take(4 * 7 * (size_t)S); if (t) t->out = (float*)p;
    p = take(4 * (size_t)S); if (t) t->atp = (float*)p;
    p = take(4 * (size_t)S); if (t) t->area = (float*)p;
    p = take(4 * (size_t)S); if (t) t->cm = (float*)p;
    p = take(4 * (size_t)S); if (t) t->vf = (float*)p;
    p = take(4 * (size_t)S); if (t) t->vnA = (float*)p;
    p = take(4 * (size_t)S); if (t) t->vnB = (float*)p;
    p = take(4 * (size_t)S); if (t) t->nb = (float*)p;
    p = take(2 * ((size_t)S + 1)); if (t) t->incoff = (uint16_t*)p;
    p = take(2 * (size_t)S); if (t) t->gsrc = (uint16_t*)p;
    p = take(2 * Ii); if (t) t->inc = (uint16_t*)p;
    p = take(8 * Ee); if (t) t->ed = (double*)p;
    p = take(4 * Ee); if (t) t->gax = (float*)p;
    p = take(4 * Ee); if (t) t->dve = (float*)p;
    // [7][E] (Fick passes use row 0); during the Jacobi solves of the residual mode the
    // FP64 iterates (2 x S doubles) and the convergence-group bits (130 words)
    const size_t fl_words = 7 * Ee > 4 * (size_t)S + 130 ? 7 * Ee : 4 * (size_t)S + 130;
    p = take(4 * fl_words); if (t) t->fl = (float*)p;
    p = take(4 * 7 * Ee); if (t) t->coef = (float*)p;
    p = take(4 * Ee); if (t) t->ie = (float*)p;
    p = take(4 * Ee); if (t) t->earea = (float*)p;
    p = take(4 * Ee); if (t) t->edist = (float*)p;
    p = take(2 * Ee); if (t) t->ea = (uint16_t*)p;
    p = take(2 * Ee); if (t) t->eb = (uint16_t*)p;
    p = take(Ee); if (t) t->ei = (uint8_t*)p;
    p = take(Ee); if (t) t->es = (uint8_t*)p;
    return off;
}

// A segment's incidences in original connection order: edge index, whether the
// segment is the edge's b end, and the other endpoint.  n < 0: more than kDeg,
// read t.inc instead.
struct Stencil {
    int n;
    uint16_t e[kDeg];
    uint16_t o[kDeg];
    uint8_t bend;   // bit k: the segment is edge e[k]'s b end
};

// Barrier of the threads that share a tile's data: the CTA itself, both CTAs of a
// 2-CTA cluster whose tiles hold the halves of one large component, or -- in a tile
// whose connections all stay inside aligned groups of gm threads -- the thread's own
// group: its warp (gm 32) or its pair of warps, named barrier 1 + tid / 64 (gm 64).
template <int CL>
__device__ __forceinline__ void tile_sync(int gm = 0) {
    if constexpr (CL == 2) {
        cooperative_groups::this_cluster().sync();
    } else {
        if (gm == 32) __syncwarp();
        else if (gm == 64) asm volatile("bar.sync %0, 64;" ::"r"(1 + (int)(threadIdx.x >> 6)) : "memory");
        else __syncthreads();
    }
}

// After a tile_sync that follows an update: copy the paired CTA's values of this
// tile's ghost segments (rows of stride S) into the ghost slots, then make them
// visible to the CTA.  The peer does not change those values again before both
// CTAs have passed another cluster barrier.
template <int CL, typename T>
__device__ __forceinline__ void halo(T* base, int rows, uint32_t S, int ns, int ng, const uint16_t* gsrc, int tid,
                                     int nth) {
    if constexpr (CL == 2) {
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        const T* peer = cl.map_shared_rank(base, cl.block_rank() ^ 1u);
        for (int k = tid; k < rows * ng; k += nth) {
            const int r = k / ng, g = k - r * ng;
            base[(size_t)r * S + ns + g] = peer[(size_t)r * S + gsrc[g]];
        }
        __syncthreads();
    }
}

// Fick pass for a float field in t.nb (diffusion_kernel.h:284-345): per-edge flux,
// then per-segment gather in connection order, updating t.nb in place.
// yvf: 1 / (this segment's volume); rde: 1 / (the length of this thread's connection)
// when each connection has its own thread (edge_reg), else unused.  The thread handles
// connections ef, ef + es, ... below el; gm is the barrier group (tile_sync).
template <int CL, bool kIntraOnly, bool kGradStrict>
__device__ __forceinline__ void fick(const DiffSmem& t, int ns, int ef, int el, int es, int gm, int i,
                                     const Stencil& st, float D, float thresh, float dt, float yvf, bool edge_reg,
                                     float rde) {
    for (int e = ef; e < el; e += es) {
        t.es[e] = 1;
        if (kIntraOnly && !t.ei[e]) continue;
        float dC = t.nb[t.ea[e]] - t.nb[t.eb[e]];
        if (kGradStrict) { if (!(dC > thresh || dC < -thresh)) continue; }
        else if (dC < thresh && dC > -thresh) continue;
        const float num = D * t.earea[e] * dC * dt;
        t.fl[e] = edge_reg ? div_rn_f(num, t.edist[e], rde) : num / t.edist[e];
        t.es[e] = 0;
    }
    tile_sync<CL>(gm);
    // the gather reads only edge fluxes and the segment's own value: update in place
    if (i < ns) {
        const float vf = t.vf[i];
        float acc = 0.0f;
        if (st.n >= 0) {
#pragma unroll
            for (int k = 0; k < kDeg; k++) {
                if (k >= st.n) break;
                const int e = st.e[k];
                if (t.es[e]) continue;
                if ((st.bend >> k) & 1u) acc += div_rn_f(t.fl[e], vf, yvf); else acc -= div_rn_f(t.fl[e], vf, yvf);
            }
        } else {
            for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                const uint16_t ent = t.inc[k];
                const int e = ent & 0x7FFF;
                if (t.es[e]) continue;
                if (ent & 0x8000) acc += div_rn_f(t.fl[e], vf, yvf); else acc -= div_rn_f(t.fl[e], vf, yvf);
            }
        }
        t.nb[i] = t.nb[i] + acc;
    }
    tile_sync<CL>(gm);
}

// ---- residual-controlled Jacobi (NetDev::diff_mode bit 0) ----
// A convergence group is a connected component.  Each sweep updates the segments of
// the groups still iterating; a segment whose value moved by more than jac_tol sets its
// group's bit; a group whose bit stays clear is done (its last sweep kept).  The CTA
// (the cluster, for tile pairs) stops when every group is done or after jac_max sweeps.
struct ResidualBufs {
    double* wa;
    double* wb;
    unsigned* bits;   // [2][64] group bits by sweep parity, then [2] cluster flags
};

__device__ __forceinline__ ResidualBufs residual_bufs(const DiffSmem& t, uint32_t S) {
    ResidualBufs r;
    r.wa = reinterpret_cast<double*>(t.fl);
    r.wb = r.wa + S;
    r.bits = reinterpret_cast<unsigned*>(r.wb + S);
    return r;
}

// OR of a predicate over the CTA, or over both CTAs of a cluster pair (flag[parity] of
// each CTA carries its half; the parity alternates between calls so a value is never
// overwritten before the peer has read it).  A barrier of the tile either way.
template <int CL>
__device__ __forceinline__ bool tile_or(bool pred, unsigned* flag, unsigned parity, int tid) {
    if constexpr (CL == 2) {
        const int local = __syncthreads_or(pred ? 1 : 0);
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        if (tid == 0) flag[parity] = (unsigned)local;
        cl.sync();
        const unsigned* pf = cl.map_shared_rank(flag, cl.block_rank() ^ 1u);
        return local != 0 || pf[parity] != 0u;
    } else {
        return __syncthreads_or(pred ? 1 : 0) != 0;
    }
}

template <int CL>
__device__ __forceinline__ unsigned peer_bits(const unsigned* w) {
    if constexpr (CL == 2) {
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        return *cl.map_shared_rank(const_cast<unsigned*>(w), cl.block_rank() ^ 1u);
    } else {
        return 0u;
    }
}

// Runs one residual-controlled solve starting from rb.wa (own and ghost values set);
// update(w) returns this thread's new value from the iterate w.  Returns the buffer
// holding the result.  slot 0: the V_m solve, 1: the phi_e solve (sweep statistics).
template <int CL, bool kPhi, typename F>
__device__ __forceinline__ const double* residual_solve(const NetDev& d, const DiffSmem& t, ResidualBufs rb,
                                                        uint32_t gw, int i, int ns, int ng, uint32_t S, int tid,
                                                        int nth, F&& update, int slot) {
    (void)kPhi;
    unsigned* bits = rb.bits;
    for (int k = tid; k < 130; k += nth) bits[k] = 0u;
    const uint32_t grp = gw & 0x7FFu;
    const bool leader = (gw & 0x8000u) != 0u;
    const unsigned gbit = 1u << (grp & 31u);
    const uint32_t gword = grp >> 5;
    double* wa = rb.wa;
    double* wb = rb.wb;
    bool done = !(i < ns);
    uint32_t it = 0;
    tile_sync<CL>();
    while (it < d.jac_max) {
        unsigned* cur = bits + (it & 1u) * 64;
        if (i < ns) {
            double nv = wa[i];
            if (!done) {
                nv = update(static_cast<const double*>(wa));
                if (fabs(nv - wa[i]) > d.jac_tol) atomicOr(&cur[gword], gbit);
            }
            wb[i] = nv;
        }
        tile_sync<CL>();
        halo<CL>(wb, 1, S, ns, ng, t.gsrc, tid, nth);
        bool more = false;
        if (!done) {
            const unsigned w = cur[gword] | peer_bits<CL>(cur + gword);
            more = (w & gbit) != 0u;
            if (!more) done = true;
        }
        for (int k = tid; k < 64; k += nth) bits[((it + 1) & 1u) * 64 + k] = 0u;
        it++;
        const bool any = tile_or<CL>(more, bits + 128, it & 1u, tid);
        double* tmp = wa; wa = wb; wb = tmp;
        if (!any) break;
    }
    if (i < ns && leader && !done) atomicAdd(&d.jac_stats[2 + slot], 1u);
    if (tid == 0) atomicMax(&d.jac_stats[slot], it);
    return wa;
}

// Adds a warp's values to a per-CTA FP64 ledger slot (every thread of the CTA calls it).
__device__ __forceinline__ void ledger_add(double* sh, int slot, double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31u) == 0u) atomicAdd(&sh[slot], v);
}

}  // namespace

// OPT 0: the reference's fixed-sweep solves (the default); OPT 1: the options of
// NetDev::diff_mode compiled in (residual-controlled solves, the ion ledger).
// GM: barrier groups (0: the CTA or cluster; 32 or 64: aligned thread groups that hold
// whole components, NetHost::diff_gm).
template <int CL, int OPT, int GM>
__global__ void __launch_bounds__(1024)
k_diffusion(NetDev d, float dt, unsigned long long tick, uint32_t S, uint32_t E) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double sh_ledger[14];   // per ion: FP32 rounding of the NP updates, bath exchange
    if (threadIdx.x < 14) sh_ledger[threadIdx.x] = 0.0;
    DiffSmem t;
    diff_layout(S, E, smem, &t);
    const int tid = threadIdx.x;
    const int nth = blockDim.x;
    const uint32_t tile = blockIdx.x;
    const uint32_t N = d.n_seg;
    const uint32_t s0 = d.tile_seg_beg[tile];
    const int ns = (int)(d.tile_seg_beg[tile + 1] - s0);
    const uint32_t e0 = d.tile_edge_beg[tile];
    const int ne = (int)(d.tile_edge_beg[tile + 1] - e0);
    const uint32_t inc0 = d.inc_off[s0];
    const int ninc = (int)(d.inc_off[s0 + ns] - inc0);
    const int i = tid;   // this thread's segment (when i < ns)
    const uint32_t gh0 = CL == 2 ? d.gh_off[tile] : 0u;
    const int ng = CL == 2 ? (int)(d.gh_off[tile + 1] - gh0) : 0;   // ghost segments (clustered tiles only)
    if (d.clock) tick = d.clock[0];

    // ---- load: state after step 1 (the modifier phases' records), stimuli, statics ----
    float c21d = 0.0f, c21h = 0.0f;
    if (i < ns) {
        const uint32_t g = s0 + i;
        const SegRec* r = d.rec + g;
        t.V[i] = r->V;
#pragma unroll
        for (int q = 0; q < 7; q++) {
            t.in[q * S + i] = r->in[q];
            t.out[q * S + i] = r->out[q];
        }
        t.atp[i] = r->atp;
        t.area[i] = d.area[g];
        t.cm[i] = d.cm[g];
        float vf = (float)r->vol;
        if (vf < 1e-6f) vf = 1e-6f;
        t.vf[i] = vf;
        // current stimuli (simulation_host.cpp:189-209, 247-258): expiry, then add in order
        double I = r->itot;
        if (d.cs_off) {
            for (uint32_t k = d.cs_off[g]; k < d.cs_off[g + 1]; k++) {
                if (!d.cs_alive[k]) continue;
                unsigned long long dur = (unsigned long long)(d.cs_dur[k] / dt);
                unsigned long long st0 = d.cs_start[k];
                if (tick >= st0 + dur) { d.cs_alive[k] = 0; continue; }
                if (tick >= st0 && tick < st0 + dur) I += d.cs_amp[k];
            }
        }
        // ramps (simulation_host.cpp:261-276): the amplitude interpolated in FP32
        if (d.rp_off) {
            for (uint32_t k = d.rp_off[g]; k < d.rp_off[g + 1]; k++) {
                const unsigned long long st0 = d.rp_start[k], en = d.rp_end[k];
                if (tick >= st0 && tick < en) {
                    const float frac = en > st0 ? (float)(tick - st0) / (float)(en - st0) : 1.0f;
                    const float a = d.rp_from[k];
                    const float amp = a + (d.rp_to[k] - a) * frac;
                    I += amp;
                }
            }
        }
        t.itot[i] = I;
        d.ibuf[g] = I;
        t.incoff[i] = (uint16_t)(d.inc_off[g] - inc0);
        const float2 c = d.c21_cur[g];
        c21d = c.x;
        c21h = c.y;
    }
    if (tid == 0) t.incoff[ns] = (uint16_t)ninc;
    for (int e = tid; e < ne; e += nth) {
        t.ea[e] = d.e_a[e0 + e];
        t.eb[e] = d.e_b[e0 + e];
        t.ei[e] = d.e_intra[e0 + e];
        t.earea[e] = d.e_area[e0 + e];
        t.edist[e] = d.e_dist[e0 + e];
    }
    for (int k = tid; k < ninc; k += nth) t.inc[k] = d.inc[inc0 + k];
    for (int g = tid; g < ng; g += nth) {   // ghosts: the paired tile's segments this tile's connections reach
        const SegRec* r = d.rec + d.gh_seg[gh0 + g];
        const int x = ns + g;
        t.V[x] = r->V;
#pragma unroll
        for (int q = 0; q < 7; q++) {
            t.in[q * S + x] = r->in[q];
            t.out[q * S + x] = r->out[q];
        }
        t.atp[x] = r->atp;
        t.phiA[x] = 0.0;
        t.gsrc[g] = (uint16_t)d.gh_src[gh0 + g];
    }
    const float dt_sub = dt / 5;
    const float ydts = 1.0f / dt_sub;
    // Nernst-Planck flux coefficient of each connection and ion: the reference's
    // kDiffC[q] * area * dt_sub / dist, left to right, the same in every substep.
    for (int e = tid; e < ne; e += nth) {
        const float ar = d.e_area[e0 + e], di = d.e_dist[e0 + e];
#pragma unroll
        for (int q = 0; q < 7; q++) t.coef[q * E + e] = kDiffC[q] * ar * dt_sub / di;
    }
    tile_sync<CL>();
    // Barrier group of this tile (tile_sync) and the connections this thread handles:
    // in a grouped tile the one its segment owns (seg_edge), else tid, tid + nth, ...
    constexpr int gm = (CL == 1 && OPT == 0) ? GM : 0;
    int ef = tid, el = ne, es = nth;
    if (gm) {
        const uint16_t me = (i < ns) ? d.seg_edge[s0 + i] : (uint16_t)0xFFFF;
        ef = me != 0xFFFF ? (int)me : 0;
        el = me != 0xFFFF ? (int)me + 1 : 0;
        es = 1;
    }
    // when every connection has its own thread, that thread keeps its connection's
    // extracellular Bernoulli values and reciprocal length in registers for the tick
    const bool edge_reg = gm != 0 || ne <= nth;
    const int my_edge = ef < el ? ef : -1;
    const float rde = (edge_reg && my_edge >= 0) ? 1.0f / t.edist[my_edge] : 1.0f;

    if (d.flags & NF_DIFFUSION) {
        // this segment's incidences in connection order
        Stencil st;
        st.n = 0;
        st.bend = 0;
        if (i < ns) {
            const int k0 = t.incoff[i], k1 = t.incoff[i + 1];
            if (k1 - k0 > kDeg) st.n = -1;
            else {
                st.n = k1 - k0;
#pragma unroll
                for (int k = 0; k < kDeg; k++) {
                    st.e[k] = 0; st.o[k] = 0;
                    if (k < st.n) {
                        const uint16_t ent = t.inc[k0 + k];
                        const int e = ent & 0x7FFF;
                        st.e[k] = (uint16_t)e;
                        if (ent & 0x8000) { st.bend |= (uint8_t)(1u << k); st.o[k] = t.ea[e]; }
                        else st.o[k] = t.eb[e];
                    }
                }
            }
        }

        // ---- phi_e (diffusion_kernel.h:41-104) ----
        if (i < ns) {
            double sacc = 0.0;
#pragma unroll
            for (int q = 0; q < 7; q++) sacc += kNpZ[q] * kNpZ[q] * kDiffC[q] * (double)t.out[q * S + i];
            t.sig[i] = 3.612f * sacc;
            t.phiA[i] = 0.0;
        }
        tile_sync<CL>(gm);
        halo<CL>(t.sig, 1, S, ns, ng, t.gsrc, tid, nth);
        for (int e = ef; e < el; e += es) {
            double g = 0.5 * (t.sig[t.ea[e]] + t.sig[t.eb[e]]) * t.earea[e] / t.edist[e];
            t.ed[e] = g;
        }
        tile_sync<CL>(gm);
        // diagonal and the sweep stencil (connections with g > 0, in order)
        double diag = 0.0, itot = 0.0;
        double pg[kDeg];
        uint16_t po[kDeg];
        int pn_cnt = 0;
        if (i < ns) {
            diag = t.sig[i] * t.area[i] / 1.0f;
            itot = t.itot[i];
            if (st.n >= 0) {
#pragma unroll
                for (int k = 0; k < kDeg; k++) {
                    pg[k] = 0.0; po[k] = 0;
                    if (k < st.n) diag += t.ed[st.e[k]];
                }
#pragma unroll
                for (int k = 0; k < kDeg; k++) {
                    if (k < st.n) {
                        const double g = t.ed[st.e[k]];
                        if (g > 0.0) {
#pragma unroll
                            for (int j = 0; j < kDeg; j++)
                                if (j == pn_cnt) { pg[j] = g; po[j] = st.o[k]; }
                            pn_cnt++;
                        }
                    }
                }
            } else {
                for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) diag += t.ed[t.inc[k] & 0x7FFF];
            }
        }
        const double ydiag = (i < ns && diag > 1e-9) ? 1.0 / diag : 1.0;
        double* phi = t.phiA;
        double* phn = t.phiB;
        if (OPT && (d.diff_mode & 1u)) {
            // residual-controlled: sweeps in phiA/phiB until the group converges; the
            // result is copied into phiA, where the fixed-sweep solve leaves it
            ResidualBufs rb = residual_bufs(t, S);
            rb.wa = t.phiA;
            rb.wb = t.phiB;
            const uint32_t gw = (i < ns) ? d.seg_grp[s0 + i] : 0u;
            const double* res = residual_solve<CL, true>(d, t, rb, gw, i, ns, ng, S, tid, nth, [&](const double* w) {
                double pn = 0.0;
                if (st.n >= 0) {
#pragma unroll
                    for (int k = 0; k < kDeg; k++)
                        if (k < pn_cnt) pn += pg[k] * w[po[k]];
                } else {
                    for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                        const uint16_t ent = t.inc[k];
                        const int e = ent & 0x7FFF;
                        const double g = t.ed[e];
                        if (g <= 0.0) continue;
                        const int o = (ent & 0x8000) ? t.ea[e] : t.eb[e];
                        pn += g * w[o];
                    }
                }
                double v = (diag > 1e-9) ? (pn - itot) / diag : 0.0;
                if (v > 10.0) v = 10.0;
                if (v < -10.0) v = -10.0;
                return v;
            }, 1);
            if (res != t.phiA) {
                if (i < ns) t.phiA[i] = res[i];
                for (int g = tid; g < ng; g += nth) t.phiA[ns + g] = res[ns + g];
            }
            tile_sync<CL>(gm);
        } else
        // Tiles whose every segment has at most two stencil entries (chains and their
        // somata): the same sums over two registers' worth of entries, two sweeps per
        // iteration so the buffers need no swap.  50 sweeps end in phiA either way.
        if (CL == 1 && __syncthreads_and(st.n >= 0 && pn_cnt <= 2)) {
            const bool h0 = pn_cnt > 0, h1 = pn_cnt > 1;
            const double g0 = pg[0], g1 = pg[1];
            const int o0 = po[0], o1 = po[1];
            const bool live = i < ns && diag > 1e-9;
            for (int it = 0; it < 50; it += 2) {
                if (i < ns) {
                    double pn = 0.0;
                    if (h0) pn += g0 * t.phiA[o0];
                    if (h1) pn += g1 * t.phiA[o1];
                    double v = live ? div_rn_d(pn - itot, diag, ydiag) : 0.0;
                    if (v > 10.0) v = 10.0;
                    if (v < -10.0) v = -10.0;
                    t.phiB[i] = v;
                }
                tile_sync<CL>(gm);
                if (i < ns) {
                    double pn = 0.0;
                    if (h0) pn += g0 * t.phiB[o0];
                    if (h1) pn += g1 * t.phiB[o1];
                    double v = live ? div_rn_d(pn - itot, diag, ydiag) : 0.0;
                    if (v > 10.0) v = 10.0;
                    if (v < -10.0) v = -10.0;
                    t.phiA[i] = v;
                }
                tile_sync<CL>(gm);
            }
        } else
        for (int it = 0; it < 50; it++) {
            if (i < ns) {
                double pn = 0.0;
                if (st.n >= 0) {
#pragma unroll
                    for (int k = 0; k < kDeg; k++)
                        if (k < pn_cnt) pn += pg[k] * phi[po[k]];
                } else {
                    for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                        const uint16_t ent = t.inc[k];
                        const int e = ent & 0x7FFF;
                        const double g = t.ed[e];
                        if (g <= 0.0) continue;
                        const int o = (ent & 0x8000) ? t.ea[e] : t.eb[e];
                        pn += g * phi[o];
                    }
                }
                double v = (diag > 1e-9) ? div_rn_d(pn - itot, diag, ydiag) : 0.0;
                if (v > 10.0) v = 10.0;
                if (v < -10.0) v = -10.0;
                phn[i] = v;
            }
            tile_sync<CL>(gm);
            halo<CL>(phn, 1, S, ns, ng, t.gsrc, tid, nth);
            double* tmp = phi; phi = phn; phn = tmp;
        }

        // ---- intracellular Nernst-Planck, 5 substeps (diffusion_kernel.h:152-238) ----
        for (int sub = 0; sub < 5; sub++) {
            for (int e = ef; e < el; e += es) {
                if (!t.ei[e]) continue;
                const int a = t.ea[e], b = t.eb[e];
                float sigma_i = 0.0f;
#pragma unroll
                for (int q = 0; q < 7; q++) {
                    float C_bar = (float)(0.5f * ((double)t.in[q * S + a] + (double)t.in[q * S + b]));
                    sigma_i += kNpZ[q] * kNpZ[q] * kDiffC[q] * C_bar;
                }
                const float gnum = 3.612f * sigma_i * t.earea[e];
                t.gax[e] = edge_reg ? div_rn_f(gnum, t.edist[e], rde) : gnum / t.edist[e];
                t.dve[e] = (float)(((double)t.V[a] + phi[a]) - ((double)t.V[b] + phi[b]));
                t.ie[e] = 0.0f;
            }
            tile_sync<CL>(gm);
            // g_diag, and the V-sweep stencil (intracellular connections, in order)
            float gd = 0.0f;
            float vg[kDeg];
            uint16_t vo[kDeg];
            int vn_cnt = 0;
            if (i < ns) {
                if (st.n >= 0) {
#pragma unroll
                    for (int k = 0; k < kDeg; k++) {
                        vg[k] = 0.0f; vo[k] = 0;
                        if (k < st.n && t.ei[st.e[k]]) {
                            const float g = t.gax[st.e[k]];
                            gd += g;
#pragma unroll
                            for (int j = 0; j < kDeg; j++)
                                if (j == vn_cnt) { vg[j] = g; vo[j] = st.o[k]; }
                            vn_cnt++;
                        }
                    }
                } else {
                    for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                        const int e = t.inc[k] & 0x7FFF;
                        if (t.ei[e]) gd += t.gax[e];
                    }
                }
            }
            // The 7 ions' fluxes in one connection pass (an ion's flux reads only that
            // ion, which no other ion's update touches), then one gather for all 7.
            // Ions of equal valence share x = (z * 0.03742f) * dV and so its Bernoulli values.
            for (int e = ef; e < el; e += es) {
                if (!t.ei[e]) continue;
                const int a = t.ea[e], b = t.eb[e];
                // the z = -1 group's argument is exactly minus the z = +1 group's
                // (x = (-0.03742f) * dV rounds symmetrically), so its two values are
                // the z = +1 group's, swapped
                float bm[3], bp[3];
#pragma unroll
                for (int g = 0; g < 2; g++) {
                    const float x = valence_factor(g) * t.dve[e];
                    bm[g] = sg_bernoulli(-x);
                    bp[g] = sg_bernoulli(x);
                }
                bm[2] = bp[0];
                bp[2] = bm[0];
                float ie = t.ie[e];
#pragma unroll
                for (int q = 0; q < 7; q++) {
                    const float C_a = t.in[q * S + a];
                    const float C_b = t.in[q * S + b];
                    const int g = valence_group(q);
                    const float flux = t.coef[q * E + e] * (C_a * bm[g] - C_b * bp[g]);
                    t.fl[q * E + e] = flux;
                    ie += div_rn_f(kNpZ[q] * 96.485f * flux, dt_sub, ydts);
                }
                t.ie[e] = ie;
            }
            tile_sync<CL>(gm);
            {   // reads connection fluxes and its own concentrations: in place
                const float vf = i < ns ? t.vf[i] : 1.0f;
                const double yv = 1.0 / (double)vf;
#pragma unroll 1
                for (int q = 0; q < 7; q++) {
                    double acc = 0.0, lost = 0.0;
                    if (i < ns) {
                    if (st.n >= 0) {
#pragma unroll
                        for (int k = 0; k < kDeg; k++) {
                            if (k >= st.n) break;
                            const int e = st.e[k];
                            if (!t.ei[e]) continue;
                            const double dq = div_by_float((double)t.fl[q * E + e], (double)vf, yv);
                            if ((st.bend >> k) & 1u) acc += dq;
                            else acc -= dq;
                        }
                    } else {
                        for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                            const uint16_t ent = t.inc[k];
                            const int e = ent & 0x7FFF;
                            if (!t.ei[e]) continue;
                            if (ent & 0x8000) acc += (double)t.fl[q * E + e] / vf;
                            else acc -= (double)t.fl[q * E + e] / vf;
                        }
                    }
                    const float old = t.in[q * S + i];
                    const float upd = (float)((double)old + (double)(float)acc);
                    t.in[q * S + i] = upd;
                    lost = ((double)upd - (double)old - acc) * (double)vf;
                    }
                    if (OPT && (d.diff_mode & 2u)) ledger_add(sh_ledger, q, lost);
                }
            }
            tile_sync<CL>(gm);
            for (int e = ef; e < el; e += es) {
                if (!t.ei[e]) continue;
                t.ie[e] = t.ie[e] - t.gax[e] * t.dve[e];
            }
            tile_sync<CL>(gm);
            float rhs = 0.0f, den = 1.0f, yden = 1.0f, C_dtv = 1.0f, inpv = 0.0f;
            if (i < ns) {
                float inp = 0.0f;
                if (st.n >= 0) {
#pragma unroll
                    for (int k = 0; k < kDeg; k++) {
                        if (k >= st.n) break;
                        const int e = st.e[k];
                        if (!t.ei[e]) continue;
                        if ((st.bend >> k) & 1u) inp -= t.ie[e]; else inp += t.ie[e];
                    }
                } else {
                    for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                        const uint16_t ent = t.inc[k];
                        const int e = ent & 0x7FFF;
                        if (!t.ei[e]) continue;
                        if (ent & 0x8000) inp -= t.ie[e]; else inp += t.ie[e];
                    }
                }
                float C_dt = t.cm[i] / dt_sub;
                if (C_dt < 1e-9f) C_dt = 1e-9f;
                rhs = C_dt * t.V[i] + inp;
                den = C_dt + gd;
                yden = 1.0f / den;
                C_dtv = C_dt;
                inpv = inp;
                t.vnA[i] = t.V[i];
            }
            for (int g = tid; g < ng; g += nth) t.vnA[ns + g] = t.V[ns + g];
            tile_sync<CL>(gm);
            float* vc = t.vnA;
            float* vn = t.vnB;
            if (OPT && (d.diff_mode & 1u)) {
                // residual-controlled FP64 Jacobi: iterates in the (dead) flux buffer, the
                // result rounded to float into vnA
                ResidualBufs rb = residual_bufs(t, S);
                if (i < ns) rb.wa[i] = (double)t.V[i];
                for (int g = tid; g < ng; g += nth) rb.wa[ns + g] = (double)t.V[ns + g];
                const double rhs_d = (double)C_dtv * (double)t.V[i < ns ? i : 0] + (double)inpv;
                const double den_d = (double)C_dtv + (double)gd;
                const uint32_t gw = (i < ns) ? d.seg_grp[s0 + i] : 0u;
                const double* res = residual_solve<CL, false>(d, t, rb, gw, i, ns, ng, S, tid, nth, [&](const double* w) {
                    double off = 0.0;
                    if (st.n >= 0) {
#pragma unroll
                        for (int k = 0; k < kDeg; k++)
                            if (k < vn_cnt) off += (double)vg[k] * w[vo[k]];
                    } else {
                        for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                            const uint16_t ent = t.inc[k];
                            const int e = ent & 0x7FFF;
                            if (!t.ei[e]) continue;
                            const int o = (ent & 0x8000) ? t.ea[e] : t.eb[e];
                            off += (double)t.gax[e] * w[o];
                        }
                    }
                    return (rhs_d + off) / den_d;
                }, 0);
                if (i < ns) t.vnA[i] = (float)res[i];
            } else
            // as for phi_e: two-entry stencils in registers, two sweeps per iteration
            if (CL == 1 && __syncthreads_and(st.n >= 0 && vn_cnt <= 2)) {
                const bool h0 = vn_cnt > 0, h1 = vn_cnt > 1;
                const float g0 = vg[0], g1 = vg[1];
                const int o0 = vo[0], o1 = vo[1];
                for (int it = 0; it < 50; it += 2) {
                    if (i < ns) {
                        float off = 0.0f;
                        if (h0) off += g0 * t.vnA[o0];
                        if (h1) off += g1 * t.vnA[o1];
                        t.vnB[i] = div_rn_f(rhs + off, den, yden);
                    }
                    tile_sync<CL>(gm);
                    if (i < ns) {
                        float off = 0.0f;
                        if (h0) off += g0 * t.vnB[o0];
                        if (h1) off += g1 * t.vnB[o1];
                        t.vnA[i] = div_rn_f(rhs + off, den, yden);
                    }
                    tile_sync<CL>(gm);
                }
            } else
            for (int it = 0; it < 50; it++) {
                if (i < ns) {
                    float off = 0.0f;
                    if (st.n >= 0) {
#pragma unroll
                        for (int k = 0; k < kDeg; k++)
                            if (k < vn_cnt) off += vg[k] * vc[vo[k]];
                    } else {
                        for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                            const uint16_t ent = t.inc[k];
                            const int e = ent & 0x7FFF;
                            if (!t.ei[e]) continue;
                            const int o = (ent & 0x8000) ? t.ea[e] : t.eb[e];
                            off += t.gax[e] * vc[o];
                        }
                    }
                    vn[i] = div_rn_f(rhs + off, den, yden);
                }
                tile_sync<CL>(gm);
                halo<CL>(vn, 1, S, ns, ng, t.gsrc, tid, nth);
                float* tmp = vc; vc = vn; vn = tmp;
            }
            if (i < ns) t.V[i] = vc[i];
            tile_sync<CL>(gm);
            halo<CL>(t.V, 1, S, ns, ng, t.gsrc, tid, nth);
            halo<CL>(t.in, 7, S, ns, ng, t.gsrc, tid, nth);
        }

        // ---- extracellular Nernst-Planck, 5 substeps (diffusion_kernel.h:244-281) ----
        // phi_e is fixed for the tick, so each connection's Bernoulli values are too:
        // x = (float)((z * 0.03742f) * dphi) per valence group.
        float xbm0 = 0.0f, xbm1 = 0.0f, xbm2 = 0.0f, xbp0 = 0.0f, xbp1 = 0.0f, xbp2 = 0.0f;
        if (edge_reg && my_edge >= 0) {
            const double dphi = phi[t.ea[my_edge]] - phi[t.eb[my_edge]];
            float x = (float)(valence_factor(0) * dphi);
            xbm0 = sg_bernoulli(-x); xbp0 = sg_bernoulli(x);
            x = (float)(valence_factor(1) * dphi);
            xbm1 = sg_bernoulli(-x); xbp1 = sg_bernoulli(x);
            xbm2 = xbp0; xbp2 = xbm0;   // the z = -1 argument is minus the z = +1 one
        }
        // The ions in two groups (0-3, 4-6): one connection pass writes a group's
        // fluxes, one gather applies them.  An ion's flux reads only that ion, which no
        // other ion's update touches, so each ion's arithmetic and its order are those
        // of one pass per ion.  The fluxes of a group (4 x E doubles) take the
        // connection buffers the intracellular sub-steps and the phi_e solve have
        // finished with (ed, gax, dve and fl lie contiguous, 44 E bytes in all).
        double* const xfl = t.ed;
        for (int sub = 0; sub < 5; sub++) {
            const float vx_seg = (i < ns ? t.vf[i] : 1.0f) * EXTRA_VOLUME_RATIO;
            const double yx_d = 1.0 / (double)vx_seg;
#pragma unroll 1
            for (int q0 = 0; q0 < 7; q0 += 4) {
                const int nq = q0 == 0 ? 4 : 3;
                for (int e = ef; e < el; e += es) {
                    const int a = t.ea[e], b = t.eb[e];
                    double dphi = 0.0;
                    if (!edge_reg) dphi = phi[a] - phi[b];
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        if (j >= nq) break;
                        const int q = q0 + j;
                        const int g = valence_group(q);
                        const double Ca = t.out[q * S + a];
                        const double Cb = t.out[q * S + b];
                        float bm = g == 0 ? xbm0 : (g == 1 ? xbm1 : xbm2);
                        float bp = g == 0 ? xbp0 : (g == 1 ? xbp1 : xbp2);
                        if (!edge_reg) {
                            const float x = (float)(kNpZ[q] * 0.03742f * dphi);
                            bm = sg_bernoulli(-x);
                            bp = sg_bernoulli(x);
                        }
                        xfl[(size_t)j * E + e] = t.coef[q * E + e] * (Ca * bm - Cb * bp);
                    }
                }
                tile_sync<CL>(gm);
                double lost[4] = {0.0, 0.0, 0.0, 0.0};
                if (i < ns) {   // in place, as above
                    const float vf = t.vf[i];
                    const float vx = vx_seg;
                    const double yx = yx_d;
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        if (j >= nq) break;
                        const int q = q0 + j;
                        const double* fq = xfl + (size_t)j * E;
                        double acc = 0.0;
                        if (st.n >= 0) {
#pragma unroll
                            for (int k = 0; k < kDeg; k++) {
                                if (k >= st.n) break;
                                const int e = st.e[k];
                                const double dq = div_by_float(fq[e], (double)vx, yx);
                                if ((st.bend >> k) & 1u) acc += dq;
                                else acc -= dq;
                            }
                        } else {
                            for (int k = t.incoff[i]; k < t.incoff[i + 1]; k++) {
                                const uint16_t ent = t.inc[k];
                                const int e = ent & 0x7FFF;
                                if (ent & 0x8000) acc += fq[e] / (vf * EXTRA_VOLUME_RATIO);
                                else acc -= fq[e] / (vf * EXTRA_VOLUME_RATIO);
                            }
                        }
                        const float old = t.out[q * S + i];
                        const float upd = (float)((double)old + acc);
                        t.out[q * S + i] = upd;
                        lost[j] = ((double)upd - (double)old - acc) * (double)vx;
                    }
                }
                if (OPT && (d.diff_mode & 2u))   // every thread of the warp takes part
                    for (int j = 0; j < nq; j++) ledger_add(sh_ledger, q0 + j, lost[j]);
                tile_sync<CL>(gm);
                halo<CL>(t.out + (size_t)q0 * S, nq, S, ns, ng, t.gsrc, tid, nth);
            }
        }

        // ---- NT / ATP / heat / transcription (diffusion_kernel.h:284-363) ----
        const float yvf = 1.0f / (i < ns ? t.vf[i] : 1.0f);
        if (d.flags & NF_INTRA_NT) {
            for (int nt = 0; nt < 15; nt++) {
                if (i < ns) t.nb[i] = d.intra_nt[(size_t)nt * N + s0 + i];
                for (int g = tid; g < ng; g += nth) t.nb[ns + g] = d.intra_nt[(size_t)nt * N + d.gh_seg[gh0 + g]];
                tile_sync<CL>(gm);
                fick<CL, true, false>(t, ns, ef, el, es, gm, i, st, gNtD[nt], 1e-12f, dt, yvf, edge_reg, rde);
                if (i < ns) d.intra_nt[(size_t)nt * N + s0 + i] = t.nb[i];
            }
        }
        if (d.flags & NF_NT_DIFFUSE_OUT) {
            for (int nt = 0; nt < 15; nt++) {
                if (i < ns) t.nb[i] = d.nt[(size_t)nt * N + s0 + i];
                for (int g = tid; g < ng; g += nth) t.nb[ns + g] = d.nt[(size_t)nt * N + d.gh_seg[gh0 + g]];
                tile_sync<CL>(gm);
                fick<CL, false, false>(t, ns, ef, el, es, gm, i, st, gNtD[nt], 1e-12f, dt, yvf, edge_reg, rde);
                if (i < ns) d.nt[(size_t)nt * N + s0 + i] = t.nb[i];
            }
        }
        {
            if (i < ns) t.nb[i] = t.atp[i];
            for (int g = tid; g < ng; g += nth) t.nb[ns + g] = t.atp[ns + g];
            tile_sync<CL>(gm);
            fick<CL, true, true>(t, ns, ef, el, es, gm, i, st, 0.14f, 1e-12f, dt, yvf, edge_reg, rde);
            if (i < ns) t.atp[i] = t.nb[i];
        }
        if (d.flags & NF_TEMP) {
            if (i < ns) t.nb[i] = d.temp[s0 + i];
            for (int g = tid; g < ng; g += nth) t.nb[ns + g] = d.temp[d.gh_seg[gh0 + g]];
            tile_sync<CL>(gm);
            fick<CL, true, true>(t, ns, ef, el, es, gm, i, st, 0.0014f, 0.001f, dt, yvf, edge_reg, rde);
            if (i < ns) d.temp[s0 + i] = t.nb[i];
        }
        if (d.flags & NF_TXN) {
            if (i < ns) t.nb[i] = d.txn[s0 + i];
            for (int g = tid; g < ng; g += nth) t.nb[ns + g] = d.txn[d.gh_seg[gh0 + g]];
            tile_sync<CL>(gm);
            fick<CL, true, true>(t, ns, ef, el, es, gm, i, st, 0.01f, 1e-9f, dt, yvf, edge_reg, rde);
            if (i < ns) d.txn[s0 + i] = t.nb[i];
        }
        if (OPT && (d.diff_mode & 2u)) {
            // the same bath relaxation and clamp, with each ion's stored change times the
            // segment's extracellular volume added to the ledger (the bath exchange)
#pragma unroll 1
            for (int q = 0; q < 7; q++) {
                double x = 0.0;
                if (i < ns) {
                    const float old = t.out[q * S + i];
                    double e = (double)old;
                    e += (kBathIon[q] - e) * dt / 1.0f;
                    if (e < 1e-9) e = 1e-9;
                    if (e > 1000.0) e = 1000.0;
                    t.out[q * S + i] = (float)e;
                    x = ((double)t.out[q * S + i] - (double)old) * (double)(t.vf[i] * EXTRA_VOLUME_RATIO);
                }
                ledger_add(sh_ledger, 7 + q, x);
            }
            __syncthreads();
            if (tid < 14) atomicAdd(&d.ledger[tid], sh_ledger[tid]);
        } else if (i < ns) {
#pragma unroll
            for (int q = 0; q < 7; q++) {
                double e = (double)t.out[q * S + i];
                e += (kBathIon[q] - e) * dt / 1.0f;
                if (e < 1e-9) e = 1e-9;
                if (e > 1000.0) e = 1000.0;
                t.out[q * S + i] = (float)e;
            }
        }
    }

    // ---- write back (each thread its own segment: no barrier needed) ----
    if (i < ns) {
        const uint32_t g = s0 + i;
        d.V[g] = t.V[i];
#pragma unroll
        for (int q = 0; q < 7; q++) {
            d.ion_in[(size_t)q * N + g] = t.in[q * S + i];
            d.ion_out[(size_t)q * N + g] = t.out[q * S + i];
        }
        d.atp[g] = t.atp[i];
        d.pre_rec[g] = make_float4(t.V[i], t.out[2 * S + i], c21d, c21h);
        if (d.flags & NF_PRE_EXT) {
            d.pre_ext[g] = make_float4(t.in[i], t.in[S + i], t.in[2 * S + i], t.out[i]);
            d.pre_ext2[g] = t.out[S + i];
        }
    }
}

size_t diffusion_smem_bytes(uint32_t max_segs, uint32_t max_edges) {
    return diff_layout(max_segs, max_edges, nullptr, nullptr);
}

uint32_t diffusion_threads(uint32_t max_segs) {
    uint32_t t = (max_segs + 31) / 32 * 32;
    return t < 32 ? 32 : t;
}

cudaError_t prepare_diffusion(const NetHost& host, cudaStream_t stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!g_ntd_ready[dev]) {
        k_init_ntd<<<1, 1, 0, stream>>>();
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        g_ntd_ready[dev] = true;
    }
    const size_t smem = diffusion_smem_bytes(host.max_tile_stride, host.max_tile_edges);
    if (smem > 48 * 1024) {
        const int a = cudaFuncAttributeMaxDynamicSharedMemorySize;
        if (host.cluster == 2) {
            e = cudaFuncSetAttribute(k_diffusion<2, 0, 0>, (cudaFuncAttribute)a, (int)smem);
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k_diffusion<2, 1, 0>, (cudaFuncAttribute)a, (int)smem);
        } else {
            e = cudaFuncSetAttribute(k_diffusion<1, 0, 0>, (cudaFuncAttribute)a, (int)smem);
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k_diffusion<1, 1, 0>, (cudaFuncAttribute)a, (int)smem);
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k_diffusion<1, 0, 32>, (cudaFuncAttribute)a, (int)smem);
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k_diffusion<1, 0, 64>, (cudaFuncAttribute)a, (int)smem);
        }
        return e;
    }
    return cudaSuccess;
}

// One-shot ion and ligand injections (simulation_host.cpp:279-300), applied after the
// modifier phases wrote the step-1 records and before step 2.5 reads them (ghost
// copies included).  One thread walks the list in upload order, so repeated
// injections into one segment add in the reference's order.
__global__ void k_inject(NetDev d) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t n = *d.inj_n;
    const size_t N = d.n_seg;
    for (uint32_t j = 0; j < n; j++) {
        const uint4 op = d.inj[j];
        const uint32_t g = op.x, what = op.y;
        const float amt = __uint_as_float(op.z);
        if (g >= N) continue;
        if (what < 16u) {
            float* ion = what < 8u ? &d.rec[g].in[what] : &d.rec[g].out[what - 8u];
            *ion = (float)((double)*ion + (double)amt);
        } else if (what < 31u) {
            d.intra_nt[(size_t)(what - 16u) * N + g] += amt;
        } else if (what >= 32u && what < 47u) {
            d.nt[(size_t)(what - 32u) * N + g] += amt;
        }
    }
    *d.inj_n = 0u;
}

cudaError_t enqueue_diffusion(const NetDev& dev, const NetHost& host, float dt, unsigned long long tick,
                              cudaStream_t stream) {
    if (dev.inj) {
        k_inject<<<1, 32, 0, stream>>>(dev);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const uint32_t S = host.max_tile_stride, E = host.max_tile_edges;
    const size_t smem = diffusion_smem_bytes(S, E);
    const uint32_t threads = std::max(host.diff_threads, diffusion_threads(host.max_tile_segs));
    const bool opt = dev.diff_mode != 0u;
    if (host.cluster == 2) {
        // tiles in pairs: one 2-CTA cluster per pair (n_tiles is even)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(dev.n_tiles);
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return opt ? cudaLaunchKernelEx(&cfg, k_diffusion<2, 1, 0>, dev, dt, tick, S, E)
                   : cudaLaunchKernelEx(&cfg, k_diffusion<2, 0, 0>, dev, dt, tick, S, E);
    }
    // barrier groups: only with each segment's connection assignment, and for 64-thread
    // groups only with whole groups of two warps (named barriers 1..15)
    int gm = (opt || !dev.seg_edge) ? 0 : (int)host.diff_gm;
    if (gm == 64 && (threads % 64u != 0u || threads > 960u)) gm = 0;
    if (opt) k_diffusion<1, 1, 0><<<dev.n_tiles, threads, smem, stream>>>(dev, dt, tick, S, E);
    else if (gm == 64) k_diffusion<1, 0, 64><<<dev.n_tiles, threads, smem, stream>>>(dev, dt, tick, S, E);
    else if (gm == 32) k_diffusion<1, 0, 32><<<dev.n_tiles, threads, smem, stream>>>(dev, dt, tick, S, E);
    else k_diffusion<1, 0, 0><<<dev.n_tiles, threads, smem, stream>>>(dev, dt, tick, S, E);
    return cudaGetLastError();
}

}  // namespace bnc
