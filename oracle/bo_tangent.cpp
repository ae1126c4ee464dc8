/*
 * bo_tangent.cpp -- CPU oracle (TEST INFRASTRUCTURE ONLY; never part of the product
 * path): the tick of the reference with its releases replayed from a log, in FP64
 * forward mode.  Every quantity carries its value and one directional derivative
 * with respect to the per-segment conductances (the densities of Nav1.6/Nav1.2 141/
 * 142, Kv delayed rectifier 123, K2P leak 107; Cav1.3 1 and the Na/K pump 7 run with
 * their fixed densities) and the per-synapse receptor density
 * scale, so one run gives the loss and its derivative along a chosen direction.  It
 * is the independent check of the device adjoint's gradients (which must agree with
 * it up to the difference between FP32 and FP64 trajectories) and, against central
 * differences of its own loss, is itself checked on the CPU.
 *
 * The tick restated (simulation_host.cpp:174-657): step 1 with the modifiers in slot
 * order (hh_biological.cpp:193-277, 2763-2797, 3063-3084, 142-187, 57-97 through the
 * GHK helpers of run_tick_common.h:274-312 and modifier_helpers.h:48-76, 132-215,
 * 1008-1018, 1135-1170); the
 * current stimuli; step 2.5 (diffusion_kernel.h:41-364: phi_e Jacobi solve,
 * intracellular and extracellular Nernst-Planck sub-steps with Scharfetter-Gummel
 * fluxes, the backward-Euler V_m sweeps, the bath relaxation); step 3 with the clefts
 * from the log and AMPA / GABA-A / glycine receptors (modifier_helpers.h:1213-1278, with the
 * density scale); step 4 (simulation_host.cpp:596-649).  ATP diffuses (Fick,
 * diffusion_kernel.h:284-345) because the pump reads it; transmitter and heat
 * diffusion are left out: nothing in the modelled networks reads them.  Every
 * arithmetic step is in double (the reference mixes float and double); clamps pass
 * the derivative where inactive and zero where active.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" {
#include "../include/bnc_abi.h"
}

namespace {

struct T {
    double v, d;
    T() : v(0), d(0) {}
    T(double x) : v(x), d(0) {}  // NOLINT
    T(double x, double y) : v(x), d(y) {}
};
inline T operator+(T a, T b) { return T(a.v + b.v, a.d + b.d); }
inline T operator-(T a, T b) { return T(a.v - b.v, a.d - b.d); }
inline T operator-(T a) { return T(-a.v, -a.d); }
inline T operator*(T a, T b) { return T(a.v * b.v, a.d * b.v + a.v * b.d); }
inline T operator/(T a, T b) { double q = a.v / b.v; return T(q, (a.d - q * b.d) / b.v); }
inline T& operator+=(T& a, T b) { a = a + b; return a; }
inline T& operator-=(T& a, T b) { a = a - b; return a; }
inline T texp(T a) { double e = std::exp(a.v); return T(e, e * a.d); }
inline T clampT(T x, double lo, double hi) { return x.v < lo ? T(lo) : (x.v > hi ? T(hi) : x); }
inline T floorT(T x, double lo) { return x.v < lo ? T(lo) : x; }

const double F = 96485.0;
const double R = (double)8.314f;
const double TK = (double)310.15f;
const double EVR = (double)(0.2f / (1.0f - 0.2f));
const double PI = (double)3.14159265f;
const double Z[7] = {1, 1, 2, -1, 2, -1, 1};
const double DC[7] = {(double)1.33f, (double)1.96f, (double)0.22f, (double)2.03f, (double)0.10f, 0.0, (double)9.31f};
const double BATH[7] = {140.0, 3.0, (double)1.2f, 130.0, 1.0, 0.0, (double)4.0e-5f};

// modifier_helpers.h:48-54
double ghk_P(double gamma_pS, double z, double cbar) { return gamma_pS * 1e-12 * (R * TK) / (z * z * F * F * cbar); }
// run_tick_common.h:274-312
T ghk_mono(T V, T ci, T co) {
    T Vn = V * (F * 0.001 / (R * TK));
    if (std::fabs(Vn.v) < 1e-6) return (ci - co) * F;
    T A = V * (F / (R * TK) * F * 0.001);
    if (Vn.v > 20.0) return A * ci;
    if (Vn.v < -20.0) return A * co;
    T e = texp(-Vn);
    return A * (ci - co * e) / (T(1.0) - e);
}
// modifier_helpers.h:132-135
T vtrap(T x, double y) {
    if (std::fabs(x.v / y) < 1e-6) return T(y) * (T(1.0) - x / (2.0 * y));
    return x / (T(1.0) - texp(-x / y));
}
void clamp_ions(T* a) { for (int q = 0; q < 7; q++) a[q] = floorT(a[q], 1e-9); }
// run_tick_common.h:274-312 (divalent cation)
T ghk_div(T V, T ci, T co) {
    T Vn = V * (2.0 * F * 0.001 / (R * TK));
    if (std::fabs(Vn.v) < 1e-6) return (ci - co) * (2.0 * F);
    T A = V * (4.0 * F / (R * TK) * F * 0.001);
    if (Vn.v > 20.0) return A * ci;
    if (Vn.v < -20.0) return A * co;
    T e = texp(-Vn);
    return A * (ci - co * e) / (T(1.0) - e);
}
// modifier_helpers.h:1135-1170 (nak_pump_vnorm, K_m_Na 10, K_m_K 1.5)
T pump_vnorm(T V, T Na, T Ko, T atp) {
    T Na3 = Na * Na * Na, K2 = Ko * Ko;
    T fNa = Na3 / (Na3 + 1000.0), fK = K2 / (K2 + (double)(1.5f * 1.5f));
    if (atp.v < 0.0) atp = T(0.0);
    T fATP = atp / (atp + 0.5);
    T eta = V * (0.8 * F * 0.001 / (R * TK));
    T a2 = texp(eta * 0.5) * 60.0, b2 = texp(-(eta * 0.5)) * 6.0;
    T a1 = fNa * fATP * 200.0, a3 = fK * 200.0;
    if (a1.v == 0.0) return T(0.0);
    T den = a3 / a1 + (b2 + a3) / a2 + 1.0 + a3 / 60.0;
    const double vmax = 200.0 / (200.0 / 200.0 + 1.0 + 200.0 / 60.0);
    return a3 / den / vmax;
}

struct Seg {
    T V, in[7], out[7], atp;
    T gate[5];          // Nav m, h; Kv_DR n; Cav1.3 m, h
    uint8_t type, n_it;
    uint8_t it[5];
    float st[5][7];
    double den[5];      // densities of the items without a fitted conductance
    double area, vol, cm, radius, length;
    uint32_t id;
};

double seg_area(const BncSegment& s) {
    return (s.segment_type == 1 || s.segment_type == 3 || s.segment_type == 4)
               ? (double)(4.0f * 3.14159265f * s.radius * s.radius)
               : (double)(2.0f * 3.14159265f * s.radius * s.length);
}
double seg_volume(const BncSegment& s) {
    if (s.segment_type == 1 || s.segment_type == 3 || s.segment_type == 4)
        return (4.0 / 3.0) * PI * (double)s.radius * (double)s.radius * (double)s.radius;
    return PI * (double)s.radius * (double)s.radius * (double)s.length;
}
bool is_ionotropic(uint8_t t) { return t <= 2 || (t >= 8 && t <= 16) || t == 97 || t == 134 || t == 194; }
// kernel_dispatch.h:283-309
bool myelin_blocked(uint8_t t) {
    static const uint8_t list[] = {107, 151, 152, 153, 133, 85, 202, 203, 204, 150, 205, 206, 207, 154, 156,
                                   157, 159, 112, 123, 121, 105, 195, 84, 96, 191, 200, 201, 140, 158, 168,
                                   129, 130, 131, 132, 103, 209, 104};
    if (is_ionotropic(t)) return true;
    for (uint8_t x : list) if (x == t) return true;
    return false;
}

struct Syn {
    uint32_t post;
    uint8_t n_r, rtype[8], nt;
    double rden[8];
    double r[8], dd[8];   // receptor gates (values: they depend on the clefts only)
    T cdi[8];             // NMDA Ca2+-dependent inactivation gate (state[2]): follows Ca2+, so a tangent
    double cleft, tauc, parea;
    uint32_t ev_b, ev_e;  // log range
};

}  // namespace

extern "C" {

/*
 * Runs `ticks` ticks from the state in `net` (at tick `tick0`) with the clefts fed
 * from the release log (entries sorted by synapse, tick, then slot), parameters
 * p = (gNa, gK, gleak per segment, w per synapse) and direction dp.  Writes the loss
 * (1 / (samples * neurons)) * sum (V_soma - target)^2 and its directional derivative;
 * `soma` lists the loss's segments.  Returns 0, or -1 when the network uses something
 * this restatement does not model.
 */
int bo_tangent_run(const BncBionData* net, const BncCurrentStimulus* stim, uint32_t n_stim,
                   const uint32_t* ev_syn, const uint64_t* ev_tick, const float* ev_amt, uint32_t n_ev,
                   uint64_t tick0, uint32_t ticks, float dt, uint32_t stride,
                   const double* p_gNa, const double* p_gK, const double* p_gleak, const double* p_w,
                   const double* d_gNa, const double* d_gK, const double* d_gleak, const double* d_w,
                   const uint32_t* soma, uint32_t n_soma, const float* target, double* loss, double* dloss) {
    const uint32_t N = net->num_segments, M = net->num_connections, K = net->num_synapses;
    std::vector<Seg> sg(N);
    for (uint32_t i = 0; i < N; i++) {
        const BncSegment& s = net->segments[i];
        Seg& g = sg[i];
        g.V = T(s.V_m);
        for (int q = 0; q < 7; q++) { g.in[q] = T(s.intra_ions[q]); g.out[q] = T(s.extra_ions[q]); }
        g.atp = T((double)s.ATP_level);
        g.type = s.segment_type;
        g.area = seg_area(s);
        g.vol = seg_volume(s);
        g.radius = s.radius; g.length = s.length; g.id = s.id;
        // run_tick_common.h:216-231
        double cm = g.area * (double)0.01f;
        if (cm < 1e-4) cm = 1e-4;
        bool myel = false;
        for (uint32_t j = 0; j < s.modifier_count; j++) if (s.modifiers[j].type == BNC_MOD_MYELIN) myel = true;
        for (uint32_t j = 0; j < s.modifier_count && j < 16; j++)
            if (s.modifiers[j].type == BNC_MOD_MYELIN) {
                double gr = (double)(float)s.modifiers[j].state[0];
                if (gr <= 0.0 || gr >= 1.0) gr = (double)0.6f;
                cm /= 100.0 * (1.0 / gr - 1.0) / (1.0 / (double)0.6f - 1.0);
                break;
            }
        g.cm = cm;
        g.n_it = 0;
        for (uint32_t j = 0; j < s.modifier_count; j++) {
            const BncModifier& m = s.modifiers[j];
            if (myel && m.type != BNC_MOD_MYELIN && myelin_blocked(m.type)) continue;
            if (m.type == BNC_MOD_MYELIN || m.type == BNC_MOD_CAV21) continue;
            if (m.type != BNC_MOD_NAV16 && m.type != BNC_MOD_NAV12 && m.type != BNC_MOD_KV_DR && m.type != BNC_MOD_K2P &&
                m.type != BNC_MOD_CAV13 && m.type != BNC_MOD_PUMP_NAK)
                return -1;
            if (g.n_it >= 5) return -1;
            const int k = g.n_it++;
            g.it[k] = m.type;
            g.den[k] = (double)(float)m.density;
            for (int q = 0; q < 7; q++) g.st[k][q] = (float)m.state[q];
            if (m.type == BNC_MOD_NAV16 || m.type == BNC_MOD_NAV12) { g.gate[0] = T(g.st[k][0]); g.gate[1] = T(g.st[k][1]); }
            if (m.type == BNC_MOD_KV_DR) g.gate[2] = T(g.st[k][0]);
            if (m.type == BNC_MOD_CAV13) { g.gate[3] = T(g.st[k][0]); g.gate[4] = T(g.st[k][1]); }
        }
    }
    std::vector<Syn> sy(K);
    uint32_t ev = 0;
    for (uint32_t k = 0; k < K; k++) {
        const BncSynapse& y = net->synapses[k];
        Syn& s = sy[k];
        if (y.type != BNC_SYN_CHEMICAL || y.post_segment >= N) return -1;
        s.post = y.post_segment;
        bool myel_post = false;
        const BncSegment& ps = net->segments[s.post];
        for (uint32_t j = 0; j < ps.modifier_count; j++) if (ps.modifiers[j].type == BNC_MOD_MYELIN) myel_post = true;
        // transmitter of the first receptor (run_tick_common.h:199-206): 0 glutamate,
        // 1 GABA, 2 glycine (cleft entry BNC_NT_GLYCINE)
        const uint8_t r0 = y.post_receptor_count > 0 ? y.post_receptors[0].type : 0;
        s.nt = r0 == BNC_MOD_GABAA ? 1 : (r0 == BNC_MOD_GLYCINE ? 2 : 0);
        s.n_r = 0;
        for (uint32_t j = 0; j < y.post_receptor_count; j++) {
            const BncModifier& m = y.post_receptors[j];
            if (myel_post && is_ionotropic(m.type)) continue;
            if (m.type != BNC_MOD_AMPA && m.type != BNC_MOD_GABAA && m.type != BNC_MOD_GLYCINE && m.type != BNC_MOD_NMDA)
                return -1;
            s.rtype[s.n_r] = m.type;
            s.rden[s.n_r] = (double)(float)m.density;
            s.r[s.n_r] = (double)(float)m.state[0];
            s.dd[s.n_r] = (double)(float)m.state[1];
            s.cdi[s.n_r] = T((double)(float)m.state[2]);
            s.n_r++;
        }
        s.cleft = y.cleft_neurotransmitter[s.nt == 2 ? BNC_NT_GLYCINE : s.nt];
        s.tauc = y.tau_clearance;
        s.parea = y.post_area;
        s.ev_b = ev;
        while (ev < n_ev && ev_syn[ev] == k) ev++;
        s.ev_e = ev;
    }
    // connections: statics
    struct Edge { uint32_t a, b; bool intra; double area, dist, va, vb; };
    std::vector<Edge> ed(M);
    for (uint32_t e = 0; e < M; e++) {
        const BncIntraConnection& c = net->connections[e];
        Edge& x = ed[e];
        x.a = c.segment_a; x.b = c.segment_b; x.intra = c.is_intracellular != 0;
        if (x.a >= N || x.b >= N) return -1;
        float r_min = std::min(net->segments[x.a].radius, net->segments[x.b].radius);
        float ac = 3.14159265f * r_min * r_min;
        if (ac < 1e-6f) ac = 1e-6f;
        float dist = (net->segments[x.a].length + net->segments[x.b].length) * 0.5f;
        if (dist < 0.1f) dist = 0.1f;
        x.area = ac; x.dist = dist;
        x.va = std::max(sg[x.a].vol, 1e-6);
        x.vb = std::max(sg[x.b].vol, 1e-6);
    }
    auto par = [&](int cls, uint32_t i) {
        const double* p = cls == 0 ? p_gNa : (cls == 1 ? p_gK : p_gleak);
        const double* d = cls == 0 ? d_gNa : (cls == 1 ? d_gK : d_gleak);
        return T(p[i], d[i]);
    };
    const uint32_t n_samples = ticks / stride;
    T L(0.0);
    std::vector<T> ibuf(N), phi(N), phn(N), sig(N), diag(N), gof(M), gdiag(N), inp(N), Vold(N), Vn(N), Vx(N);
    std::vector<T> acc((size_t)N * 7);
    const double dts = (double)(dt / 5);
    for (uint32_t t = 0; t < ticks; t++) {
        const uint64_t tick = tick0 + t;
        // ---- step 1 ----
        for (uint32_t i = 0; i < N; i++) {
            Seg& s = sg[i];
            T I_total(0.0);
            for (int j = 0; j < s.n_it; j++) {
                const uint8_t ty = s.it[j];
                const double cpv = F * s.vol / 1000.0;
                if (ty == BNC_MOD_NAV16 || ty == BNC_MOD_NAV12) {
                    const bool is12 = ty == BNC_MOD_NAV12;
                    s.V = clampT(s.V, -200.0, 200.0);
                    T V = s.V;
                    const double cam = is12 ? 23.0 : 43.0, cah = is12 ? 41.5 : 50.0, cbh = is12 ? 66.5 : 75.0,
                                 chh = is12 ? 63.5 : 72.0;
                    T am = T((double)0.182f) * vtrap(V + cam, 6.0), bm = T((double)0.124f) * vtrap(-(V + cam), 6.0);
                    T ah = T((double)0.024f) * vtrap(V + cah, 5.0), bh = T((double)0.0091f) * vtrap(-(V + cbh), 5.0);
                    T minf = am / (am + bm), mtau = T(1.0) / (am + bm);
                    T hinf = T(1.0) / (T(1.0) + texp((V + chh) / (double)6.2f)), htau = T(1.0) / (ah + bh);
                    T mv = clampT(minf + (s.gate[0] - minf) * texp(T(-(double)dt) / mtau), 0.0, 1.0);
                    T hv = clampT(hinf + (s.gate[1] - hinf) * texp(T(-(double)dt) / htau), 0.0, 1.0);
                    s.gate[0] = mv; s.gate[1] = hv;
                    T open = mv * mv * mv * hv;
                    const double ttx = s.st[j][5] > 0.0f ? (double)s.st[j][5] : 0.0;
                    open = open / (1.0 + ttx / (is12 ? 10.0 : 5.0));
                    if (open.v < 0.0) open = T(0.0);
                    const double P = ghk_P(is12 ? (double)20.8f : (double)20.7f, 1.0, (double)55.964f);
                    T I = T(P) * ghk_mono(V, s.in[0], s.out[0]) * (par(0, i) * s.area) * open * 1e12;
                    s.in[0] = s.in[0] - I * (double)dt / cpv;
                    s.out[0] = s.out[0] + I * (double)dt / (cpv * EVR);
                    clamp_ions(s.in);
                    clamp_ions(s.out);
                    I_total = I_total - I;
                } else if (ty == BNC_MOD_KV_DR) {
                    T V = s.V;
                    const double Vh = s.st[j][1] != 0.0f ? (double)s.st[j][1] : -30.0;
                    const double kk = s.st[j][2] > 0.0f ? (double)s.st[j][2] : 6.0;
                    T tau = s.st[j][4] > 0.0f ? T((double)s.st[j][4])
                                              : clampT(T((double)14.6f) * texp(-(V - Vh) / (double)30.1f), (double)0.3f, 200.0);
                    T minf = T(1.0) / (T(1.0) + texp(-(V - Vh) / (kk + (double)1e-6f)));
                    T nv = clampT(s.gate[2] + (minf - s.gate[2]) * (double)dt / (tau + (double)1e-6f), 0.0, 1.0);
                    s.gate[2] = nv;
                    const double P = ghk_P(12.0, 1.0, (double)40.514f);
                    T I = T(P) * ghk_mono(V, s.in[1], s.out[1]) * (par(1, i) * s.area) * nv * 1e12;
                    s.in[1] = s.in[1] - I * (double)dt / cpv;
                    s.out[1] = s.out[1] + I * (double)dt / (cpv * EVR);
                    clamp_ions(s.in);
                    clamp_ions(s.out);
                    I_total = I_total - I;
                } else if (ty == BNC_MOD_CAV13) {   // hh_biological.cpp:142-187
                    T V = s.V;
                    const double Vh = s.st[j][3] != 0.0f ? -std::fabs((double)s.st[j][3]) : -35.0;
                    const double kk = s.st[j][4] > 0.0f ? (double)s.st[j][4] : 7.0;
                    const double gam = s.st[j][2] > 0.0f ? (double)s.st[j][2] : 25.0;
                    T minf = T(1.0) / (T(1.0) + texp(-(V - Vh) / (kk + (double)1e-6f)));
                    T mv = s.gate[3] + (minf - s.gate[3]) * ((double)dt / 2.0);
                    T hinf = T(1.0) / (T(1.0) + texp((V + 52.0) / 8.0));
                    hinf = hinf * (T(1.0) / (T(1.0) + s.in[2] * (1000.0 / 3.0)));
                    T hv = s.gate[4] + (hinf - s.gate[4]) * ((double)dt / 100.0);
                    mv = clampT(mv, 0.0, 1.0);
                    hv = clampT(hv, 0.0, 1.0);
                    s.gate[3] = mv; s.gate[4] = hv;
                    const double P = ghk_P((double)(float)gam, 2.0, (double)0.12775f);
                    T I = T(P) * ghk_div(V, s.in[2], s.out[2]) * (s.den[j] * s.area) * (mv * mv * hv) * 1e12;
                    s.in[2] = s.in[2] - I * (double)dt / (2.0 * cpv);
                    s.out[2] = s.out[2] - I * (double)dt / (2.0 * cpv * EVR);
                    clamp_ions(s.in);
                    clamp_ions(s.out);
                    I_total = I_total - I;
                } else if (ty == BNC_MOD_PUMP_NAK) {   // hh_biological.cpp:57-97
                    T v = pump_vnorm(s.V, s.in[0], s.out[1], s.atp);
                    const double e = (double)1.602176634e-19f;
                    T I = v * (s.den[j] * s.area * 75.0 * e * 1e12);
                    const double cpm = F * (double)(float)s.vol / 1000.0;
                    T tr = I * ((double)dt / cpm);
                    T na = floorT((s.in[0] - (double)1e-9f) / 3.0, 0.0);
                    T ka = floorT((s.out[1] - (double)1e-9f) * (EVR / 2.0), 0.0);
                    T mx = na.v < ka.v ? na : ka;
                    if (tr.v > mx.v) tr = mx;
                    s.in[0] = s.in[0] - tr * 3.0;
                    s.out[0] = s.out[0] + tr * (3.0 / EVR);
                    s.in[1] = s.in[1] + tr * 2.0;
                    s.out[1] = s.out[1] - tr * (2.0 / EVR);
                    clamp_ions(s.in);
                    clamp_ions(s.out);
                    s.atp = floorT(s.atp - I * ((double)dt * (double)1e-8f), 0.0);
                    I_total = I_total - I;
                } else {   // K2P leak
                    const double gam = s.st[j][0] > 0.0f ? (double)s.st[j][0] : 100.0;
                    const double Po = s.st[j][1] > 0.0f ? (double)s.st[j][1] : (double)0.012f;
                    const double P = ghk_P(gam, 1.0, (double)40.514f);
                    T I = T(P) * ghk_mono(s.V, s.in[1], s.out[1]) * (par(2, i) * s.area) * Po * 1e12;
                    s.in[1] = s.in[1] - I * (double)dt / cpv;
                    s.out[1] = s.out[1] + I * (double)dt / (cpv * EVR);
                    clamp_ions(s.out);
                    I_total = I_total - I;
                }
            }
            for (uint32_t q = 0; q < n_stim; q++) {
                const BncCurrentStimulus& st = stim[q];
                if (st.segment_id != s.id) continue;
                const uint64_t dur = (uint64_t)(st.duration_ms / dt);
                if (tick >= st.start_tick && tick < st.start_tick + dur) I_total += T((double)st.amplitude_pA);
            }
            ibuf[i] = I_total;
        }
        // ---- step 2.5 ----
        if (M > 0) {
            for (uint32_t i = 0; i < N; i++) {
                T s(0.0);
                for (int q = 0; q < 7; q++) s += sg[i].out[q] * (Z[q] * Z[q] * DC[q]);
                sig[i] = s * (double)3.612f;
                diag[i] = sig[i] * sg[i].area;
                phi[i] = T(0.0);
            }
            for (uint32_t e = 0; e < M; e++) {
                gof[e] = (sig[ed[e].a] + sig[ed[e].b]) * (0.5 * ed[e].area / ed[e].dist);
                diag[ed[e].a] += gof[e];
                diag[ed[e].b] += gof[e];
            }
            for (int it = 0; it < 50; it++) {
                for (uint32_t i = 0; i < N; i++) phn[i] = T(0.0);
                for (uint32_t e = 0; e < M; e++) {
                    if (gof[e].v <= 0.0) continue;
                    phn[ed[e].a] += gof[e] * phi[ed[e].b];
                    phn[ed[e].b] += gof[e] * phi[ed[e].a];
                }
                for (uint32_t i = 0; i < N; i++)
                    phi[i] = diag[i].v > 1e-9 ? clampT((phn[i] - ibuf[i]) / diag[i], -10.0, 10.0) : T(0.0);
            }
            for (int sub = 0; sub < 5; sub++) {
                for (auto& x : acc) x = T(0.0);
                for (uint32_t i = 0; i < N; i++) { gdiag[i] = T(0.0); inp[i] = T(0.0); }
                for (uint32_t e = 0; e < M; e++) {
                    const Edge& x = ed[e];
                    if (!x.intra) continue;
                    Seg &A = sg[x.a], &B = sg[x.b];
                    T si(0.0);
                    for (int q = 0; q < 7; q++) si += (A.in[q] + B.in[q]) * (0.5 * Z[q] * Z[q] * DC[q]);
                    T gax = si * ((double)3.612f * x.area / x.dist);
                    gof[e] = gax;
                    gdiag[x.a] += gax;
                    gdiag[x.b] += gax;
                    T dV = (A.V + phi[x.a]) - (B.V + phi[x.b]);
                    T Inp(0.0);
                    for (int q = 0; q < 7; q++) {
                        T xx = dV * (Z[q] * (double)0.03742f);
                        auto bern = [](T y) {
                            if (std::fabs(y.v) < 1e-3) return T(1.0) - y * 0.5;
                            if (y.v > 50.0) return T(0.0);
                            if (y.v < -50.0) return -y;
                            return y / (texp(y) - 1.0);
                        };
                        T flux = (A.in[q] * bern(-xx) - B.in[q] * bern(xx)) * (DC[q] * x.area * dts / x.dist);
                        acc[(size_t)x.a * 7 + q] -= flux / x.va;
                        acc[(size_t)x.b * 7 + q] += flux / x.vb;
                        Inp += flux * (Z[q] * (double)96.485f / dts);
                    }
                    inp[x.a] += Inp - gax * dV;
                    inp[x.b] -= Inp - gax * dV;
                }
                for (uint32_t i = 0; i < N; i++) { Vold[i] = sg[i].V; Vn[i] = sg[i].V; }
                for (int it = 0; it < 50; it++) {
                    for (uint32_t i = 0; i < N; i++) Vx[i] = T(0.0);
                    for (uint32_t e = 0; e < M; e++) {
                        if (!ed[e].intra) continue;
                        Vx[ed[e].a] += gof[e] * Vn[ed[e].b];
                        Vx[ed[e].b] += gof[e] * Vn[ed[e].a];
                    }
                    for (uint32_t i = 0; i < N; i++) {
                        double Cdt = sg[i].cm / dts;
                        if (Cdt < 1e-9) Cdt = 1e-9;
                        Vx[i] = (Vold[i] * Cdt + inp[i] + Vx[i]) / (gdiag[i] + Cdt);
                    }
                    std::swap(Vn, Vx);
                }
                for (uint32_t i = 0; i < N; i++) {
                    sg[i].V = Vn[i];
                    for (int q = 0; q < 7; q++) sg[i].in[q] += acc[(size_t)i * 7 + q];
                }
            }
            for (int sub = 0; sub < 5; sub++) {
                for (auto& x : acc) x = T(0.0);
                for (uint32_t e = 0; e < M; e++) {
                    const Edge& x = ed[e];
                    T dphi = phi[x.a] - phi[x.b];
                    for (int q = 0; q < 7; q++) {
                        T xx = dphi * (Z[q] * (double)0.03742f);
                        auto bern = [](T y) {
                            if (std::fabs(y.v) < 1e-3) return T(1.0) - y * 0.5;
                            if (y.v > 50.0) return T(0.0);
                            if (y.v < -50.0) return -y;
                            return y / (texp(y) - 1.0);
                        };
                        T flux = (sg[x.a].out[q] * bern(-xx) - sg[x.b].out[q] * bern(xx)) * (DC[q] * x.area * dts / x.dist);
                        acc[(size_t)x.a * 7 + q] -= flux / (x.va * EVR);
                        acc[(size_t)x.b * 7 + q] += flux / (x.vb * EVR);
                    }
                }
                for (uint32_t i = 0; i < N; i++)
                    for (int q = 0; q < 7; q++) sg[i].out[q] += acc[(size_t)i * 7 + q];
            }
            // ATP (diffusion_kernel.h:284-345): from the values before the pass, on
            // intracellular connections whose difference exceeds 1e-12
            {
                std::vector<T> da(N);
                for (uint32_t e = 0; e < M; e++) {
                    const Edge& x = ed[e];
                    if (!x.intra) continue;
                    T dC = sg[x.a].atp - sg[x.b].atp;
                    if (!(dC.v > (double)1e-12f || dC.v < -(double)1e-12f)) continue;
                    T f = dC * ((double)0.14f * x.area * (double)dt / x.dist);
                    da[x.a] -= f / (double)(float)x.va;
                    da[x.b] += f / (double)(float)x.vb;
                }
                for (uint32_t i = 0; i < N; i++) sg[i].atp += da[i];
            }
            for (uint32_t i = 0; i < N; i++)
                for (int q = 0; q < 7; q++) {
                    T e = sg[i].out[q];
                    e += (T(BATH[q]) - e) * (double)dt;
                    sg[i].out[q] = clampT(e, 1e-9, 1000.0);
                }
        }
        // ---- step 3 ----
        std::vector<double> nt_glu(N, 0.0), nt_gaba(N, 0.0), nt_gly(N, 0.0);
        for (uint32_t k = 0; k < K; k++) {
            Syn& y = sy[k];
            Seg& s = sg[y.post];
            for (uint32_t q = y.ev_b; q < y.ev_e; q++)
                if (ev_tick[q] == tick) y.cleft += (double)ev_amt[q];
            if (y.nt == 0) nt_glu[y.post] += y.cleft;
            else if (y.nt == 1) nt_gaba[y.post] += y.cleft;
            else nt_gly[y.post] += y.cleft;
            T I_syn(0.0);
            const T w(p_w[k], d_w[k]);
            const double cpm = F * s.vol / 1000.0;
            for (int j = 0; j < y.n_r; j++) {
                // receptors_biological.cpp:42-82: AMPA, NMDA, GABA-A, glycine
                const bool nmda = y.rtype[j] == BNC_MOD_NMDA;
                if (nmda) {
                    // gating on glutamate without desensitisation (EC50 1, rise 5 ms, decay 50
                    // ms); GHK Na+, K+ and Ca2+ currents with the 0.08 / 0.08 / 0.84 split of
                    // 50 pS (modifier_helpers.h:69-76, 1213-1279); the Mg2+ block of the
                    // membrane potential and the Ca2+-dependent inactivation gate that follows
                    // the Ca2+ the receptor has just let in (modifier_helpers.h:1281-1290)
                    const double nt = nt_glu[y.post];
                    const double r_inf = nt / (nt + 1.0);
                    const double tau = r_inf > y.r[j] ? 5.0 : 50.0;
                    y.r[j] = std::min(1.0, std::max(0.0, y.r[j] + (r_inf - y.r[j]) * (double)dt / tau));
                    const double area = y.parea > 0.0 ? y.parea : s.area;
                    const double Nk = y.rden[j] * area * y.r[j];
                    const double cNa = (double)55.964f, cK = (double)40.514f, cCa = (double)0.12775f;
                    const double wsum = (double)0.08f * cNa + (double)0.08f * cK + (double)0.84f * 4.0 * cCa;
                    const double PNa = ghk_P(50.0 * (double)0.08f * cNa / wsum, 1.0, cNa);
                    const double PK = ghk_P(50.0 * (double)0.08f * cK / wsum, 1.0, cK);
                    const double PCa = ghk_P(50.0 * (double)0.84f * 4.0 * cCa / wsum, 2.0, cCa);
                    T INa = T(PNa) * ghk_mono(s.V, s.in[0], s.out[0]) * Nk * w * 1e12;
                    T IK = T(PK) * ghk_mono(s.V, s.in[1], s.out[1]) * Nk * w * 1e12;
                    T ICa = T(PCa) * ghk_div(s.V, s.in[2], s.out[2]) * Nk * w * 1e12;
                    s.in[0] = s.in[0] - INa * (double)dt / cpm;
                    s.in[1] = s.in[1] - IK * (double)dt / cpm;
                    s.in[2] = s.in[2] - ICa * (double)dt / (2.0 * cpm);
                    clamp_ions(s.in);
                    const T mg = T(1.0) / (T(1.0) + T((double)(1.0f / 3.57f)) * texp(s.V * -(double)0.062f));
                    const T ca_uM = s.in[2] * 1000.0;
                    const T cinf = T(1.0) - T((double)0.8f) * ca_uM / (ca_uM + 1.0);
                    const double tcdi = cinf.v < y.cdi[j].v ? 500.0 : 9000.0;
                    y.cdi[j] = clampT(y.cdi[j] + (cinf - y.cdi[j]) * ((double)dt / tcdi), 0.0, 1.0);
                    I_syn = I_syn - (INa + IK + ICa) * mg * y.cdi[j] * (double)(10.0f / 11.0f);
                    continue;
                }
                const bool ampa = y.rtype[j] == BNC_MOD_AMPA, gly = y.rtype[j] == BNC_MOD_GLYCINE;
                const double EC50 = ampa ? 0.5 : (gly ? 0.5 : 1.0), tr = ampa ? 0.5 : (gly ? 0.3 : 1.0),
                             td = ampa ? 3.0 : 5.0, tdes = ampa ? 3.0 : 2000.0;
                const double nt = ampa ? nt_glu[y.post] : (gly ? nt_gly[y.post] : nt_gaba[y.post]);
                const double r_inf = nt / (nt + EC50);
                const double tau = r_inf > y.r[j] ? tr : td;
                y.r[j] = std::min(1.0, std::max(0.0, y.r[j] + (r_inf - y.r[j]) * (double)dt / tau));
                const double d_inf = nt / (nt + EC50);
                y.dd[j] = std::min(1.0, std::max(0.0, y.dd[j] + (d_inf - y.dd[j]) * (double)dt / tdes));
                const double open = y.r[j] * (1.0 - y.dd[j]);
                const double area = y.parea > 0.0 ? y.parea : s.area;
                const double Nk = y.rden[j] * area * open;
                if (ampa) {
                    const double wsum = 0.5 * (double)55.964f + 0.5 * (double)40.514f;
                    const double PNa = ghk_P(8.0 * 0.5 * (double)55.964f / wsum, 1.0, (double)55.964f);
                    const double PK = ghk_P(8.0 * 0.5 * (double)40.514f / wsum, 1.0, (double)40.514f);
                    T INa = T(PNa) * ghk_mono(s.V, s.in[0], s.out[0]) * Nk * w * 1e12;
                    T IK = T(PK) * ghk_mono(s.V, s.in[1], s.out[1]) * Nk * w * 1e12;
                    s.in[0] = s.in[0] - INa * (double)dt / cpm;
                    s.in[1] = s.in[1] - IK * (double)dt / cpm;
                    clamp_ions(s.in);
                    I_syn = I_syn - (INa + IK);
                } else {
                    const double PCl = ghk_P(gly ? 60.0 : 28.0, 1.0, (double)36.20f);
                    T ICl = T(PCl) * ghk_mono(s.V, s.out[3], s.in[3]) * Nk * w * 1e12;
                    s.in[3] = s.in[3] + ICl * (double)dt / cpm;
                    clamp_ions(s.in);
                    I_syn = I_syn - ICl;
                }
            }
            ibuf[y.post] += I_syn;
            y.cleft *= std::exp(-(double)dt / y.tauc);
            if (y.cleft < 0.0) y.cleft = 0.0;
        }
        // ---- step 4 ----
        for (uint32_t i = 0; i < N; i++) {
            Seg& s = sg[i];
            T ib = clampT(ibuf[i], -10000.0, 10000.0);
            T dV = clampT(ib / s.cm * (double)dt, -50.0, 50.0);
            s.V = clampT(s.V + dV, -120.0, 150.0);
        }
        if ((t + 1) % stride == 0) {
            const uint32_t smp = (t + 1) / stride - 1;
            for (uint32_t n = 0; n < n_soma; n++) {
                T diff = sg[soma[n]].V - (double)target[(size_t)smp * n_soma + n];
                L += diff * diff;
            }
        }
    }
    const double norm = 1.0 / ((double)n_samples * (double)n_soma);
    *loss = L.v * norm;
    *dloss = L.d * norm;
    return 0;
}

}  // extern "C"
