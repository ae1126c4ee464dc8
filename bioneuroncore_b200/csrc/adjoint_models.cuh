// adjoint_models.cuh -- local derivatives of the pointwise pieces of a tick, for the
// reverse tick in adjoint.cu.
//
// Each function restates one model of physics.cuh / synapse.cu over a forward-mode
// dual number (value + N partial derivatives, double precision): evaluated once with
// every input seeded, it yields the model's local Jacobian at the forward point, and
// the reverse tick applies its transpose.  The values are not used for the forward
// trajectory (that keeps the bit-exact device functions); only the derivatives are.
// Float roundings of the forward code are identities here, clamps are subgradient
// masks (derivative 0 where the clamp is active).
#pragma once
#include <cstdint>
#include <cmath>

namespace bnc {
namespace adj {

#ifndef BNC_ADJ_NOINLINE
#define BNC_ADJ_NOINLINE __device__ __noinline__
#endif
// One out-of-line copy of the double exponential for every dual-number use.
BNC_ADJ_NOINLINE double adj_exp(double x) { return exp(x); }

template <int N>
struct Dual {
    double v;
    double d[N];
    __device__ __forceinline__ Dual() : v(0.0) {
#pragma unroll
        for (int k = 0; k < N; k++) d[k] = 0.0;
    }
    __device__ __forceinline__ Dual(double x) : v(x) {   // NOLINT: constants promote implicitly
#pragma unroll
        for (int k = 0; k < N; k++) d[k] = 0.0;
    }
    __device__ __forceinline__ static Dual seed(double x, int k) {
        Dual r(x);
        r.d[k] = 1.0;
        return r;
    }
};

#define BNC_DUAL_OP(OP, EXPR_V, EXPR_D)                                                        \
    template <int N>                                                                           \
    __device__ __forceinline__ Dual<N> operator OP(const Dual<N>& a, const Dual<N>& b) {       \
        Dual<N> r;                                                                             \
        r.v = EXPR_V;                                                                          \
        _Pragma("unroll") for (int k = 0; k < N; k++) r.d[k] = EXPR_D;                         \
        return r;                                                                              \
    }
BNC_DUAL_OP(+, a.v + b.v, a.d[k] + b.d[k])
BNC_DUAL_OP(-, a.v - b.v, a.d[k] - b.d[k])
BNC_DUAL_OP(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
#undef BNC_DUAL_OP
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = -a.d[k];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) { return a * (1.0 / b); }
template <int N> __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }
template <int N>
__device__ __forceinline__ Dual<N> dexp(const Dual<N>& a) {
    Dual<N> r;
    r.v = adj_exp(a.v);
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = r.v * a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dconst(const Dual<N>& a) { return Dual<N>(a.v); }   // a clamp in effect

// clamp(x, lo, hi) with the derivative masked where the clamp is active
template <int N>
__device__ __forceinline__ Dual<N> dclamp(const Dual<N>& x, double lo, double hi) {
    if (x.v < lo) return Dual<N>(lo);
    if (x.v > hi) return Dual<N>(hi);
    return x;
}
template <int N>
__device__ __forceinline__ Dual<N> dfloor(const Dual<N>& x, double lo) { return (x.v < lo) ? Dual<N>(lo) : x; }

/* ---- constants: the same literals as physics.cuh ---- */
constexpr double kF = 96485.0;
constexpr double kR = (double)8.314f;
constexpr double kT = (double)310.15f;
constexpr double kEVR = (double)(0.2f / (1.0f - 0.2f));

// run_tick_common.h:274-312 (GHK flux, monovalent cation / anion) as a function of
// (V, c_in, c_out); branch choice by value, as the forward code takes it.
template <int N>
__device__ __forceinline__ Dual<N> ghk_mono(const Dual<N>& V, const Dual<N>& cin, const Dual<N>& cout) {
    const double kk = kF / (kR * kT);
    Dual<N> Vn = V * (kF * 0.001 / (kR * kT));
    if (fabs(Vn.v) < 1e-6) return (cin - cout) * kF;
    Dual<N> A = V * (kk * kF * 0.001);
    if (Vn.v > 20.0) return A * cin;
    if (Vn.v < -20.0) return A * cout;
    Dual<N> e = dexp(-Vn);
    return A * (cin - cout * e) / (1.0 - e);
}
template <int N>
__device__ __forceinline__ Dual<N> ghk_anion(const Dual<N>& V, const Dual<N>& cin, const Dual<N>& cout) {
    return ghk_mono(V, cout, cin);
}

// modifier_helpers.h:132-135
template <int N>
__device__ __forceinline__ Dual<N> vtrap(const Dual<N>& x, double y) {
    if (fabs(x.v / y) < 1e-6) return y * (1.0 - x / (2.0 * y));
    return x / (1.0 - dexp(-x / y));
}

// Nav1.6 / Nav1.2 gating (modifier_helpers.h:145-215)
struct NavK { double am, bm, ah, bh, hh; };
__device__ __forceinline__ NavK nav_consts(int is12) {
    return is12 ? NavK{(double)23.0f, (double)23.0f, (double)41.5f, (double)66.5f, (double)63.5f}
                : NavK{(double)43.0f, (double)43.0f, (double)50.0f, (double)75.0f, (double)72.0f};
}

// Local Jacobians of the modifier items.  Inputs (seed order):
//   0 V, 1 gate0, 2 gate1, 3 c_in, 4 c_out, 5 density
// Outputs: V' (the Nav clamp), gate0', gate1', c_in', c_out', I (the returned current).
struct ItemJac {
    double dV[6], dg0[6], dg1[6], dcin[6], dcout[6], dI[6];
};

template <int N>
__device__ __forceinline__ void store_row(double* row, const Dual<N>& x) {
#pragma unroll
    for (int k = 0; k < 6; k++) row[k] = (k < N) ? x.d[k] : 0.0;
}

// hh_biological.cpp:193-277 (dp_nav_current): c = Na
__device__ __forceinline__ void jac_nav(ItemJac& J, float V0, float m0, float h0, float cin0, float cout0, float den0,
                                        float area, double vol, float dt, int is12, float ttx) {
    typedef Dual<6> D;
    D V = D::seed(V0, 0), m = D::seed(m0, 1), h = D::seed(h0, 2);
    D cin = D::seed(cin0, 3), cout = D::seed(cout0, 4), den = D::seed(den0, 5);
    V = dclamp(V, -200.0, 200.0);
    const NavK c = nav_consts(is12);
    D am = (double)0.182f * vtrap(V + c.am, 6.0), bm = (double)0.124f * vtrap(-(V + c.bm), 6.0);
    D ah = (double)0.024f * vtrap(V + c.ah, 5.0), bh = (double)0.0091f * vtrap(-(V + c.bh), 5.0);
    D minf = am / (am + bm), mtau = 1.0 / (am + bm);
    D hinf = 1.0 / (1.0 + dexp((V + c.hh) / (double)6.2f)), htau = 1.0 / (ah + bh);
    D mv = dclamp(minf + (m - minf) * dexp(-(double)dt / mtau), 0.0, 1.0);
    D hv = dclamp(hinf + (h - hinf) * dexp(-(double)dt / htau), 0.0, 1.0);
    D open = mv * mv * mv * hv;
    double ttxd = ttx > 0.0f ? (double)ttx : 0.0;
    open = open / (1.0 + ttxd / (is12 ? 10.0 : 5.0));
    if (open.v < 0.0) open = D(0.0);
    const double gamma = is12 ? (double)20.8f : (double)20.7f;
    const double P = gamma * 1e-12 * (kR * kT) / (kF * kF * (double)55.964f);
    D flux = ghk_mono(V, cin, cout);
    D I_Na = P * flux * (den * (double)area) * open * 1e12;
    const double cpv = kF * vol / 1000.0;
    D cin1 = dfloor(cin - (I_Na * (double)dt) / cpv, 1e-9);
    D cout1 = dfloor(cout + (I_Na * (double)dt) / (cpv * kEVR), 1e-9);
    store_row(J.dV, V); store_row(J.dg0, mv); store_row(J.dg1, hv);
    store_row(J.dcin, cin1); store_row(J.dcout, cout1); store_row(J.dI, -I_Na);
}

// hh_biological.cpp:2763-2797 (dp_kvdr_current): gate0 = n, c = K
__device__ __forceinline__ void jac_kvdr(ItemJac& J, float V0, float n0, float cin0, float cout0, float den0,
                                         float area, double vol, float dt, const float* st) {
    typedef Dual<6> D;
    D V = D::seed(V0, 0), n = D::seed(n0, 1);
    D cin = D::seed(cin0, 3), cout = D::seed(cout0, 4), den = D::seed(den0, 5);
    const double V_half = (st[1] != 0.0f) ? (double)st[1] : -30.0;
    const double k = (st[2] > 0.0f) ? (double)st[2] : 6.0;
    D tau;
    if (st[4] > 0.0f) tau = D((double)st[4]);
    else {
        tau = (double)14.6f * dexp(-(V - (double)(float)V_half) / (double)30.1f);
        tau = dclamp(tau, (double)0.3f, 200.0);
    }
    D minf = 1.0 / (1.0 + dexp(-(V - V_half) / (k + (double)1e-6f)));
    D nv = dclamp(n + (minf - n) * (double)dt / (tau + (double)1e-6f), 0.0, 1.0);
    const double P = 12.0 * 1e-12 * (kR * kT) / (kF * kF * (double)40.514f);
    D I_K = P * ghk_mono(V, cin, cout) * (den * (double)area) * nv * 1e12;
    const double cpmv = (double)(float)(kF * vol / 1000.0);
    D cin1 = dfloor(cin - (I_K * (double)dt) / cpmv, 1e-9);
    D cout1 = dfloor(cout + (I_K * (double)dt) / (cpmv * kEVR), 1e-9);
    store_row(J.dV, V); store_row(J.dg0, nv); store_row(J.dg1, D(0.0));
    store_row(J.dcin, cin1); store_row(J.dcout, cout1); store_row(J.dI, -I_K);
}

// hh_biological.cpp:3063-3084 (dp_k2p_current): c = K, no gates
__device__ __forceinline__ void jac_k2p(ItemJac& J, float V0, float cin0, float cout0, float den0,
                                        float area, double vol, float dt, const float* st) {
    typedef Dual<6> D;
    D V = D::seed(V0, 0);
    D cin = D::seed(cin0, 3), cout = D::seed(cout0, 4), den = D::seed(den0, 5);
    const double gamma = (st[0] > 0.0f) ? (double)st[0] : 100.0;
    const double Po = (st[1] > 0.0f) ? (double)st[1] : (double)0.012f;
    const double P = (double)(float)gamma * 1e-12 * (kR * kT) / (kF * kF * (double)40.514f);
    D I_K = P * ghk_mono(V, cin, cout) * (den * (double)area) * Po * 1e12;
    const double cpv = kF * vol / 1000.0;
    D cin1 = cin - (I_K * (double)dt) / cpv;   // dp_k_flux clamps the extracellular side only
    D cout1 = dfloor(cout + (I_K * (double)dt) / (cpv * kEVR), 1e-9);
    store_row(J.dV, V); store_row(J.dg0, D(0.0)); store_row(J.dg1, D(0.0));
    store_row(J.dcin, cin1); store_row(J.dcout, cout1); store_row(J.dI, -I_K);
}

// Ionotropic receptor (modifier_helpers.h:1213-1278) with its gates given.  Inputs:
//   0 V, 1 in[0], 2 in[1], 3 in[3], 4 out[0], 5 out[1], 6 out[3], 7 weight scale
// Outputs: in[0]', in[1]', in[3]', I.
struct RecJac {
    double din0[8], din1[8], din3[8], dI[8];
    double v0, v1, v3;   // the updated ions (values)
};
__device__ __forceinline__ void jac_receptor(RecJac& J, int anion, double P_a, double P_b, float V0,
                                             const float* in, const float* out, float w0, float den,
                                             float area, float open, double vol, float dt) {
    typedef Dual<8> D;
    D V = D::seed(V0, 0), i0 = D::seed(in[0], 1), i1 = D::seed(in[1], 2), i3 = D::seed(in[3], 3);
    D o0 = D::seed(out[0], 4), o1 = D::seed(out[1], 5), o3 = D::seed(out[3], 6), w = D::seed(w0, 7);
    const double cpm = kF * vol / 1000.0;
    const double Nk = (double)den * (double)area * (double)open;
    D n0 = i0, n1 = i1, n3 = i3, I;
    if (anion) {
        D I_Cl = P_a * ghk_anion(V, i3, o3) * Nk * w * 1e12;
        n3 = dfloor(i3 + (I_Cl * (double)dt) / cpm, 1e-9);
        I = -I_Cl;
    } else {
        D I_Na = P_a * ghk_mono(V, i0, o0) * Nk * w * 1e12;
        D I_K = P_b * ghk_mono(V, i1, o1) * Nk * w * 1e12;
        n0 = dfloor(i0 - (I_Na * (double)dt) / cpm, 1e-9);
        n1 = dfloor(i1 - (I_K * (double)dt) / cpm, 1e-9);
        I = -(I_Na + I_K);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) { J.din0[k] = n0.d[k]; J.din1[k] = n1.d[k]; J.din3[k] = n3.d[k]; J.dI[k] = I.d[k]; }
    J.v0 = n0.v; J.v1 = n1.v; J.v3 = n3.v;
}

// ---- vector-Jacobian products of the items and receptors ----
// The reverse tick needs lambda^T J, not J: these contract on the fly.  Quantities that
// depend on V alone (gating rates, the GHK prefactor and exponential) carry a one-
// component dual number; the rest of the chain rule is written out.

// GHK flux (run_tick_common.h:274-312) and its partials in V, c_in, c_out.
struct GhkD { double F, dV, dci, dco; };
__device__ __forceinline__ GhkD ghk_mono_d(double Vd, double ci, double co) {
    const double kk = kF / (kR * kT);
    const double c1 = kF * 0.001 / (kR * kT);
    const double Vn = Vd * c1;
    GhkD r;
    if (fabs(Vn) < 1e-6) { r.F = kF * (ci - co); r.dV = 0.0; r.dci = kF; r.dco = -kF; return r; }
    const double A = Vd * (kk * kF * 0.001), dA = kk * kF * 0.001;
    if (Vn > 20.0) { r.F = A * ci; r.dV = dA * ci; r.dci = A; r.dco = 0.0; return r; }
    if (Vn < -20.0) { r.F = A * co; r.dV = dA * co; r.dci = 0.0; r.dco = A; return r; }
    const double e = adj_exp(-Vn), de = -e * c1;
    const double D = 1.0 - e, Nn = ci - co * e;
    r.F = A * Nn / D;
    r.dV = dA * Nn / D + A * de * (ci - co) / (D * D);
    r.dci = A / D;
    r.dco = -A * e / D;
    return r;
}

// lo = adjoints of (V', gate0', gate1', c_in', c_out', returned I); lx = adjoints of
// (V, gate0, gate1, c_in, c_out, density).
__device__ __forceinline__ void vjp_nav(const double* lo, double* lx, float V0, float m0, float h0, float cin,
                                        float cout, float den, float area, double vol, float dt, int is12, float ttx) {
    typedef Dual<1> D;
    const bool mV = (double)V0 >= -200.0 && (double)V0 <= 200.0;
    const double Vc = mV ? (double)V0 : ((double)V0 < -200.0 ? -200.0 : 200.0);
    const D V = D::seed(Vc, 0);
    const NavK c = nav_consts(is12);
    const D am = (double)0.182f * vtrap(V + c.am, 6.0), bm = (double)0.124f * vtrap(-(V + c.bm), 6.0);
    const D ah = (double)0.024f * vtrap(V + c.ah, 5.0), bh = (double)0.0091f * vtrap(-(V + c.bh), 5.0);
    const D minf = am / (am + bm), mtau = 1.0 / (am + bm);
    const D hinf = 1.0 / (1.0 + dexp((V + c.hh) / (double)6.2f)), htau = 1.0 / (ah + bh);
    const D Em = dexp(-(double)dt / mtau), Eh = dexp(-(double)dt / htau);
    const double mu_ = minf.v + ((double)m0 - minf.v) * Em.v, hu_ = hinf.v + ((double)h0 - hinf.v) * Eh.v;
    const bool mm = mu_ >= 0.0 && mu_ <= 1.0, mh = hu_ >= 0.0 && hu_ <= 1.0;
    const double mv = mm ? mu_ : (mu_ < 0.0 ? 0.0 : 1.0), hv = mh ? hu_ : (hu_ < 0.0 ? 0.0 : 1.0);
    const double dm_dV = mm ? minf.d[0] * (1.0 - Em.v) + ((double)m0 - minf.v) * Em.d[0] : 0.0;
    const double dh_dV = mh ? hinf.d[0] * (1.0 - Eh.v) + ((double)h0 - hinf.v) * Eh.d[0] : 0.0;
    const double dm_dm = mm ? Em.v : 0.0, dh_dh = mh ? Eh.v : 0.0;
    const double cdiv = 1.0 + (ttx > 0.0f ? (double)ttx : 0.0) / (is12 ? 10.0 : 5.0);
    const double open = mv * mv * mv * hv / cdiv;
    const double do_dm = 3.0 * mv * mv * hv / cdiv, do_dh = mv * mv * mv / cdiv;
    const double gamma = is12 ? (double)20.8f : (double)20.7f;
    const double Kc = gamma * 1e-12 * (kR * kT) / (kF * kF * (double)55.964f) * 1e12 * (double)area;
    const GhkD G = ghk_mono_d(Vc, cin, cout);
    const double I = Kc * G.F * (double)den * open;
    const double cpv = kF * vol / 1000.0;
    const bool mci = (double)cin - I * (double)dt / cpv >= 1e-9;
    const bool mco = (double)cout + I * (double)dt / (cpv * kEVR) >= 1e-9;
    const double lI = -lo[5] - (mci ? lo[3] * (double)dt / cpv : 0.0) + (mco ? lo[4] * (double)dt / (cpv * kEVR) : 0.0);
    const double lopen = lI * Kc * G.F * (double)den;
    const double lF = lI * Kc * (double)den * open;
    const double lmv = lo[1] + lopen * do_dm, lhv = lo[2] + lopen * do_dh;
    const double lVc = lo[0] + lF * G.dV + lmv * dm_dV + lhv * dh_dV;
    lx[0] = mV ? lVc : 0.0;
    lx[1] = lmv * dm_dm;
    lx[2] = lhv * dh_dh;
    lx[3] = (mci ? lo[3] : 0.0) + lF * G.dci;
    lx[4] = (mco ? lo[4] : 0.0) + lF * G.dco;
    lx[5] = lI * Kc * G.F * open;
}

__device__ __forceinline__ void vjp_kvdr(const double* lo, double* lx, float V0, float n0, float cin, float cout,
                                         float den, float area, double vol, float dt, const float* st) {
    typedef Dual<1> D;
    const D V = D::seed((double)V0, 0);
    const double V_half = (st[1] != 0.0f) ? (double)st[1] : -30.0;
    const double k = (st[2] > 0.0f) ? (double)st[2] : 6.0;
    D tau;
    if (st[4] > 0.0f) tau = D((double)st[4]);
    else tau = dclamp((double)14.6f * dexp(-(V - (double)(float)V_half) / (double)30.1f), (double)0.3f, 200.0);
    const D minf = 1.0 / (1.0 + dexp(-(V - V_half) / (k + (double)1e-6f)));
    const double tt = tau.v + (double)1e-6f;
    const double nu = (double)n0 + (minf.v - (double)n0) * (double)dt / tt;
    const bool mn = nu >= 0.0 && nu <= 1.0;
    const double nv = mn ? nu : (nu < 0.0 ? 0.0 : 1.0);
    const double dn_dV = mn ? (minf.d[0] * (double)dt / tt - (minf.v - (double)n0) * (double)dt * tau.d[0] / (tt * tt)) : 0.0;
    const double dn_dn = mn ? 1.0 - (double)dt / tt : 0.0;
    const double Kc = 12.0 * 1e-12 * (kR * kT) / (kF * kF * (double)40.514f) * 1e12 * (double)area;
    const GhkD G = ghk_mono_d((double)V0, cin, cout);
    const double I = Kc * G.F * (double)den * nv;
    const double cpmv = (double)(float)(kF * vol / 1000.0);
    const bool mci = (double)cin - I * (double)dt / cpmv >= 1e-9;
    const bool mco = (double)cout + I * (double)dt / (cpmv * kEVR) >= 1e-9;
    const double lI = -lo[5] - (mci ? lo[3] * (double)dt / cpmv : 0.0) + (mco ? lo[4] * (double)dt / (cpmv * kEVR) : 0.0);
    const double lF = lI * Kc * (double)den * nv;
    const double lnv = lo[1] + lI * Kc * G.F * (double)den;
    lx[0] = lo[0] + lF * G.dV + lnv * dn_dV;
    lx[1] = lnv * dn_dn;
    lx[2] = 0.0;
    lx[3] = (mci ? lo[3] : 0.0) + lF * G.dci;
    lx[4] = (mco ? lo[4] : 0.0) + lF * G.dco;
    lx[5] = lI * Kc * G.F * nv;
}

__device__ __forceinline__ void vjp_k2p(const double* lo, double* lx, float V0, float cin, float cout, float den,
                                        float area, double vol, float dt, const float* st) {
    const double gamma = (st[0] > 0.0f) ? (double)st[0] : 100.0;
    const double Po = (st[1] > 0.0f) ? (double)st[1] : (double)0.012f;
    const double Kc = (double)(float)gamma * 1e-12 * (kR * kT) / (kF * kF * (double)40.514f) * 1e12 * (double)area * Po;
    const GhkD G = ghk_mono_d((double)V0, cin, cout);
    const double I = Kc * G.F * (double)den;
    const double cpv = kF * vol / 1000.0;
    const bool mco = (double)cout + I * (double)dt / (cpv * kEVR) >= 1e-9;
    const double lI = -lo[5] - lo[3] * (double)dt / cpv + (mco ? lo[4] * (double)dt / (cpv * kEVR) : 0.0);
    const double lF = lI * Kc * (double)den;
    lx[0] = lo[0] + lF * G.dV;
    lx[1] = lx[2] = 0.0;
    lx[3] = lo[3] + lF * G.dci;
    lx[4] = (mco ? lo[4] : 0.0) + lF * G.dco;
    lx[5] = lI * Kc * G.F;
}

// Ionotropic receptor with its open probability given.  lo = adjoints of (in[0]',
// in[1]', in[3]', returned I); lx = adjoints of (V, in[0], in[1], in[3], out[0],
// out[1], out[3], weight scale).  nv0/nv1/nv3 receive the updated ions (values).
__device__ __forceinline__ void vjp_receptor(const double* lo, double* lx, int anion, double P_a, double P_b, float V0,
                                             const float* in, const float* out, float w, float den, float area,
                                             float open, double vol, float dt, float* nv) {
    const double cpm = kF * vol / 1000.0;
    const double Nk = (double)den * (double)area * (double)open * 1e12;
    for (int k = 0; k < 8; k++) lx[k] = 0.0;
    nv[0] = in[0]; nv[1] = in[1]; nv[2] = in[3];
    if (anion) {
        const GhkD G = ghk_mono_d((double)V0, out[3], in[3]);   // anion flux: c_in and c_out swapped
        const double I = P_a * G.F * Nk * (double)w;
        const double n3 = (double)in[3] + I * (double)dt / cpm;
        const bool m3 = n3 >= 1e-9;
        nv[2] = (float)(m3 ? n3 : 1e-9);
        const double lI = -lo[3] + (m3 ? lo[2] * (double)dt / cpm : 0.0);
        const double lF = lI * P_a * Nk * (double)w;
        lx[0] = lF * G.dV;
        lx[1] = lo[0]; lx[2] = lo[1];
        lx[3] = (m3 ? lo[2] : 0.0) + lF * G.dco;
        lx[6] = lF * G.dci;
        lx[7] = lI * P_a * G.F * Nk;
        return;
    }
    const GhkD Ga = ghk_mono_d((double)V0, in[0], out[0]);
    const GhkD Gb = ghk_mono_d((double)V0, in[1], out[1]);
    const double Ia = P_a * Ga.F * Nk * (double)w, Ib = P_b * Gb.F * Nk * (double)w;
    const double n0 = (double)in[0] - Ia * (double)dt / cpm, n1 = (double)in[1] - Ib * (double)dt / cpm;
    const bool m0 = n0 >= 1e-9, m1 = n1 >= 1e-9;
    nv[0] = (float)(m0 ? n0 : 1e-9);
    nv[1] = (float)(m1 ? n1 : 1e-9);
    const double lIa = -lo[3] - (m0 ? lo[0] * (double)dt / cpm : 0.0);
    const double lIb = -lo[3] - (m1 ? lo[1] * (double)dt / cpm : 0.0);
    const double lFa = lIa * P_a * Nk * (double)w, lFb = lIb * P_b * Nk * (double)w;
    lx[0] = lFa * Ga.dV + lFb * Gb.dV;
    lx[1] = (m0 ? lo[0] : 0.0) + lFa * Ga.dci;
    lx[2] = (m1 ? lo[1] : 0.0) + lFb * Gb.dci;
    lx[3] = lo[2];
    lx[4] = lFa * Ga.dco;
    lx[5] = lFb * Gb.dco;
    lx[7] = (lIa * P_a * Ga.F + lIb * P_b * Gb.F) * Nk;
}

// The NMDA receptor (receptors_biological.cpp:48-70): GHK Na+, K+ and Ca2+ currents of
// the open receptors, each moving its ion (the ions clamped at 1e-9 as masks), the Mg2+
// block of the membrane potential, and the Ca2+-dependent inactivation gate cdi
// (modifier_helpers.h:1281-1290), which relaxes toward a value set by the Ca2+ the
// receptor has just let in and scales the returned current with the co-agonist factor.
// The divalent GHK flux is 2 x the monovalent one at 2V.  Float roundings are
// identities and the gate's time constant is the branch the forward took.
// lo = adjoints of (c_in Na', K', Ca', returned I, cdi'); lx = adjoints of (V, c_in Na,
// K, Ca, c_out Na, K, Ca, weight, cdi); nv = c_in Na', K', Ca' as the forward leaves them.
__device__ __forceinline__ void vjp_nmda(const double* lo, double* lx, double P_Na, double P_K, double P_Ca, float V0,
                                         const float* in, const float* out, float w, float den, float area, float open,
                                         float cdi0, double vol, float dt, float* nv) {
    const double cpm = kF * vol / 1000.0;
    const double Nk = (double)den * (double)area * (double)open * 1e12;
    const double W = (double)w, T = (double)dt;
    for (int k = 0; k < 9; k++) lx[k] = 0.0;
    const GhkD Ga = ghk_mono_d((double)V0, in[0], out[0]);
    const GhkD Gb = ghk_mono_d((double)V0, in[1], out[1]);
    const GhkD Gh = ghk_mono_d(2.0 * (double)V0, in[2], out[2]);
    const double Fc = 2.0 * Gh.F, dVc = 4.0 * Gh.dV, dcic = 2.0 * Gh.dci, dcoc = 2.0 * Gh.dco;
    const double Ia = P_Na * Ga.F * Nk * W, Ib = P_K * Gb.F * Nk * W, Ic = P_Ca * Fc * Nk * W;
    const double n0 = (double)in[0] - Ia * T / cpm, n1 = (double)in[1] - Ib * T / cpm;
    const double n2 = (double)in[2] - Ic * T / (2.0 * cpm);
    const bool m0 = n0 >= 1e-9, m1 = n1 >= 1e-9, m2 = n2 >= 1e-9;
    nv[0] = (float)(m0 ? n0 : 1e-9);
    nv[1] = (float)(m1 ? n1 : 1e-9);
    nv[2] = (float)(m2 ? n2 : 1e-9);
    const double I0 = -(Ia + Ib + Ic);
    // Mg2+ block: 1 / (1 + e^(-0.062 V) / 3.57)
    const double a = (double)(1.0f / 3.57f), b = (double)0.062f;
    const double ex = adj_exp(-b * (double)V0);
    const double mg = 1.0 / (1.0 + a * ex);
    const double dmg = mg * mg * a * b * ex;
    // inactivation gate from the Ca2+ after the receptor's own influx
    const double u = (double)nv[2] * 1000.0;
    const double cinf = 1.0 - (double)0.8f * u / (u + 1.0);
    const double tau = (cinf < (double)cdi0) ? 500.0 : 9000.0;
    const double craw = (double)cdi0 + (cinf - (double)cdi0) * T / tau;
    const bool mc = craw >= 0.0 && craw <= 1.0;
    const double cnew = mc ? craw : (craw < 0.0 ? 0.0 : 1.0);
    const double coag = (double)(10.0f / 11.0f);
    const double lI = lo[3];
    const double lcnew = lo[4] + lI * I0 * mg * coag;
    lx[0] = lI * I0 * cnew * coag * dmg;
    const double lI0 = lI * mg * cnew * coag;
    const double lcraw = mc ? lcnew : 0.0;
    lx[8] = lcraw * (1.0 - T / tau);
    const double lu = lcraw * (T / tau) * (-(double)0.8f / ((u + 1.0) * (u + 1.0)));
    const double ln0 = lo[0], ln1 = lo[1], ln2 = lo[2] + lu * 1000.0;
    const double lIa = -lI0 - (m0 ? ln0 * T / cpm : 0.0);
    const double lIb = -lI0 - (m1 ? ln1 * T / cpm : 0.0);
    const double lIc = -lI0 - (m2 ? ln2 * T / (2.0 * cpm) : 0.0);
    const double lFa = lIa * P_Na * Nk * W, lFb = lIb * P_K * Nk * W, lFc = lIc * P_Ca * Nk * W;
    lx[0] += lFa * Ga.dV + lFb * Gb.dV + lFc * dVc;
    lx[1] = (m0 ? ln0 : 0.0) + lFa * Ga.dci;
    lx[2] = (m1 ? ln1 : 0.0) + lFb * Gb.dci;
    lx[3] = (m2 ? ln2 : 0.0) + lFc * dcic;
    lx[4] = lFa * Ga.dco;
    lx[5] = lFb * Gb.dco;
    lx[6] = lFc * dcoc;
    lx[7] = (lIa * P_Na * Ga.F + lIb * P_K * Gb.F + lIc * P_Ca * Fc) * Nk;
}

// ---- the same products in single precision ----
// The reverse tick's hot path.  Differences that cancel near zero -- 1 - e^-u in
// vtrap and in the GHK flux -- are formed with expm1f, so they keep full relative
// precision; the products agree with the double-precision ones above to ~1e-5.
struct GhkF { float F, dV, dci, dco; };
__device__ __forceinline__ GhkF ghk_mono_f(float V, float ci, float co) {
    const float c1 = (float)(kF * 0.001 / (kR * kT));
    const float dA = (float)(kF / (kR * kT) * kF * 0.001);
    const float Vn = V * c1;
    GhkF r;
    if (fabsf(Vn) < 1e-6f) { r.F = (float)kF * (ci - co); r.dV = 0.0f; r.dci = (float)kF; r.dco = -(float)kF; return r; }
    const float A = V * dA;
    if (Vn > 20.0f) { r.F = A * ci; r.dV = dA * ci; r.dci = A; r.dco = 0.0f; return r; }
    if (Vn < -20.0f) { r.F = A * co; r.dV = dA * co; r.dci = 0.0f; r.dco = A; return r; }
    const float D = -expm1f(-Vn);      // 1 - e^-Vn
    const float e = 1.0f - D;
    const float Nn = ci - co * e;
    r.F = A * Nn / D;
    if (fabsf(Vn) < 1e-2f) {
        // F = kappa (ci g(Vn) - co g(-Vn)), g(u) = u / (1 - e^-u): the two terms of the
        // closed-form derivative cancel here, so take g'(u) = 1/2 + u/6 - u^3/180
        const float kappa = dA / c1;
        const float g1 = 0.5f + Vn / 6.0f - Vn * Vn * Vn / 180.0f, g2 = 0.5f - Vn / 6.0f + Vn * Vn * Vn / 180.0f;
        r.dV = c1 * kappa * (ci * g1 + co * g2);
    } else {
        r.dV = dA * Nn / D - A * e * c1 * (ci - co) / (D * D);
    }
    r.dci = A / D;
    r.dco = -A * e / D;
    return r;
}

// vtrap(x, y) (modifier_helpers.h:132-135) and its derivative in x
__device__ __forceinline__ void vtrap_f(float x, float y, float* v, float* dv) {
    const float u = x / y;
    if (fabsf(u) < 1e-6f) { *v = y * (1.0f - x / (2.0f * y)); *dv = -0.5f; return; }
    const float D = -expm1f(-u);       // 1 - e^-u
    *v = x / D;
    // d/dx = g'(u), g(u) = u / (1 - e^-u); near 0 the closed form cancels
    *dv = (fabsf(u) < 1e-2f) ? 0.5f + u / 6.0f - u * u * u / 180.0f : (D - u * (1.0f - D)) / (D * D);
}
// 1 / (1 + e^z) and its derivative in z
__device__ __forceinline__ void logistic_f(float z, float* v, float* dv) {
    const float ez = expf(z);
    const float den = 1.0f + ez;
    *v = 1.0f / den;
    *dv = -ez / (den * den);
}

// Cav1.3 (hh_biological.cpp:142-187): lambda^T J in single precision, contracted by
// hand.  The divalent GHK flux is 2 x the monovalent one at 2V (the thresholds of
// run_tick_common.h:274-312 coincide), so ghk_mono_f gives its value and partials
// without cancellation near 0.  lo = adjoints of (V', m', h', Ca_in', Ca_out',
// returned I); lx = adjoints of (V, m, h, Ca_in, Ca_out, density) -- the density is
// not fitted and its entry is 0.
__device__ __noinline__ void vjp_cav13(const float* lo, float* lx, float V, float m0, float h0, float cin, float cout,
                                      float den, float area, double vol, float dt, const float* st) {
    const float Vhalf = (st[3] != 0.0f) ? -fabsf(st[3]) : -35.0f;
    const float kk = ((st[4] > 0.0f) ? st[4] : 7.0f) + 1e-6f;
    const float gamma = (st[2] > 0.0f) ? st[2] : 25.0f;
    const float a = dt / 2.0f, b = dt / 100.0f;
    float mi, dmi, hi0, dhi0;
    logistic_f(-(V - Vhalf) / kk, &mi, &dmi);   // d mi / dV = -dmi / kk
    logistic_f((V + 52.0f) / 8.0f, &hi0, &dhi0);  // d hi0 / dV = dhi0 / 8
    const float m1 = m0 + (mi - m0) * a;
    const float hc = 1.0f / (1.0f + cin * (1000.0f / 3.0f));
    const float h1 = h0 + (hi0 * hc - h0) * b;
    const bool mm = m1 >= 0.0f && m1 <= 1.0f, mh = h1 >= 0.0f && h1 <= 1.0f;
    const float mc = fminf(fmaxf(m1, 0.0f), 1.0f), hcl = fminf(fmaxf(h1, 0.0f), 1.0f);
    const float open = mc * mc * hcl;
    const GhkF g = ghk_mono_f(2.0f * V, cin, cout);
    const float flux = 2.0f * g.F, fV = 4.0f * g.dV, fci = 2.0f * g.dci, fco = 2.0f * g.dco;
    const float G = (float)((double)gamma * 1e-12 * (kR * kT) / (4.0 * kF * kF * (double)0.12775f) * 1e12) * den * area;
    const float I = G * flux * open;
    const float cpm = (float)(kF * vol / 1000.0);
    const float s_in = dt / (2.0f * cpm), s_out = dt / (2.0f * cpm * (float)kEVR);
    const float lcin1 = (cin - I * s_in >= 1e-9f) ? lo[3] : 0.0f, lcout1 = (cout - I * s_out >= 1e-9f) ? lo[4] : 0.0f;
    const float lI = -lo[5] - lcin1 * s_in - lcout1 * s_out;
    const float lopen = lI * G * flux, lflux = lI * G * open;
    const float lm1 = mm ? (lo[1] + lopen * 2.0f * mc * hcl) : 0.0f;
    const float lh1 = mh ? (lo[2] + lopen * mc * mc) : 0.0f;
    const float lmi = lm1 * a, lhi = lh1 * b;
    lx[0] = lo[0] - lmi * dmi / kk + lhi * hc * dhi0 / 8.0f + lflux * fV;
    lx[1] = lm1 * (1.0f - a);
    lx[2] = lh1 * (1.0f - b);
    lx[3] = lcin1 + lflux * fci - lhi * hi0 * hc * hc * (1000.0f / 3.0f);
    lx[4] = lcout1 + lflux * fco;
    lx[5] = 0.0f;
}

// The Na/K pump (hh_biological.cpp:57-97, nak_pump_vnorm modifier_helpers.h:1135-1170)
// reversed in single precision.  Inputs V, Na_in, K_out, ATP; outputs Na_in', Na_out',
// K_in', K_out', ATP' and the returned current.  lp holds the adjoints of (V', Na_in',
// Na_out', K_in', K_out', ATP', I) on entry and those of (V, Na_in, Na_out, K_in, K_out,
// ATP) on exit (Na_out and K_in pass through; V is not changed).  The transport cap (the
// available Na and K) is a branch by value; the ion floors of 1e-9 are not reached by
// a capped transport and are left out.
__device__ __noinline__ void vjp_pump(float* lp, float V, float Na, float Ko, float atp0, float den, float area,
                                     double vol, float dt) {
    const float Na3 = Na * Na * Na, K2 = Ko * Ko, KK2 = 1.5f * 1.5f;
    const float fNa = Na3 / (Na3 + 1000.0f), fK = K2 / (K2 + KK2);
    const float dfNa = 3000.0f * Na * Na / ((Na3 + 1000.0f) * (Na3 + 1000.0f));
    const float dfK = 2.0f * Ko * KK2 / ((K2 + KK2) * (K2 + KK2));
    const bool atp_pos = atp0 >= 0.0f;
    const float at = atp_pos ? atp0 : 0.0f;
    const float fATP = at / (at + 0.5f), dfATP = atp_pos ? 0.5f / ((at + 0.5f) * (at + 0.5f)) : 0.0f;
    const float cV = (float)(0.8 * kF * 0.001 / (kR * kT));
    const float a2 = 60.0f * expf(0.5f * cV * V), b2 = 6.0f * expf(-0.5f * cV * V);
    const float a1 = 200.0f * fNa * fATP, a3 = 200.0f * fK;
    const float vmax = 200.0f / (200.0f / 200.0f + 1.0f + 200.0f / 60.0f);
    float dv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    float vn = 0.0f;
    if (a1 != 0.0f) {
        const float dn = a3 / a1 + (b2 + a3) / a2 + 1.0f + a3 / 60.0f;
        const float tv = a3 / dn, q = tv / dn;
        vn = tv / vmax;
        const float t_a1 = q * a3 / (a1 * a1), t_a2 = q * (b2 + a3) / (a2 * a2);
        const float t_a3 = 1.0f / dn - q * (1.0f / a1 + 1.0f / a2 + 1.0f / 60.0f), t_b2 = -q / a2;
        dv[0] = 0.5f * cV * (t_a2 * a2 - t_b2 * b2) / vmax;
        dv[1] = t_a1 * 200.0f * dfNa * fATP / vmax;
        dv[2] = t_a3 * 200.0f * dfK / vmax;
        dv[3] = t_a1 * 200.0f * fNa * dfATP / vmax;
    }
    const float cI = (float)((double)den * (double)area * 75.0 * (double)1.602176634e-19f * 1e12);
    const float I = vn * cI;
    const float cdt = dt / (float)(kF * (double)(float)vol / 1000.0);
    const float tr_raw = I * cdt;
    float na = (Na - 1e-9f) / 3.0f, ka = (Ko - 1e-9f) * (float)(kEVR / 2.0);
    const bool na_on = na >= 0.0f, ka_on = ka >= 0.0f;
    na = fmaxf(na, 0.0f);
    ka = fmaxf(ka, 0.0f);
    float dtr[4];
    if (tr_raw > fminf(na, ka)) {   // capped by the available Na or K
        dtr[0] = dtr[3] = 0.0f;
        dtr[1] = (na < ka && na_on) ? 1.0f / 3.0f : 0.0f;
        dtr[2] = (na >= ka && ka_on) ? (float)(kEVR / 2.0) : 0.0f;
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) dtr[k] = dv[k] * cI * cdt;
    }
    const float la1 = (atp0 - I * (dt * 1e-8f) >= 0.0f) ? lp[5] : 0.0f;
    const float lt = -3.0f * lp[1] + (float)(3.0 / kEVR) * lp[2] + 2.0f * lp[3] - (float)(2.0 / kEVR) * lp[4];
    const float lI = -lp[6] - la1 * (dt * 1e-8f);
    float lx[4];
#pragma unroll
    for (int k = 0; k < 4; k++) lx[k] = lt * dtr[k] + lI * dv[k] * cI;
    lp[0] += lx[0];
    lp[1] += lx[1];
    lp[4] += lx[2];
    lp[5] = la1 + lx[3];
}

__device__ __forceinline__ void vjp_nav_f(const float* lo, float* lx, float V0, float m0, float h0, float cin, float cout,
                                          float den, float area, double vol, float dt, int is12, float ttx) {
    const bool mV = V0 >= -200.0f && V0 <= 200.0f;
    const float V = mV ? V0 : (V0 < -200.0f ? -200.0f : 200.0f);
    const float cam = is12 ? 23.0f : 43.0f, cah = is12 ? 41.5f : 50.0f, cbh = is12 ? 66.5f : 75.0f,
                chh = is12 ? 63.5f : 72.0f;
    float am, dam, bm, dbm, ah, dah, bh, dbh;
    vtrap_f(V + cam, 6.0f, &am, &dam); am *= 0.182f; dam *= 0.182f;
    vtrap_f(-(V + cam), 6.0f, &bm, &dbm); bm *= 0.124f; dbm *= -0.124f;
    vtrap_f(V + cah, 5.0f, &ah, &dah); ah *= 0.024f; dah *= 0.024f;
    vtrap_f(-(V + cbh), 5.0f, &bh, &dbh); bh *= 0.0091f; dbh *= -0.0091f;
    const float sm = am + bm, sh = ah + bh;
    const float minf = am / sm, dminf = (dam * bm - am * dbm) / (sm * sm);
    const float mtau = 1.0f / sm, dmtau = -(dam + dbm) / (sm * sm);
    float hinf, dhinf;
    logistic_f((V + chh) / 6.2f, &hinf, &dhinf);
    dhinf /= 6.2f;
    const float htau = 1.0f / sh, dhtau = -(dah + dbh) / (sh * sh);
    const float Em = expf(-dt / mtau), dEm = Em * dt / (mtau * mtau) * dmtau;
    const float Eh = expf(-dt / htau), dEh = Eh * dt / (htau * htau) * dhtau;
    const float mu_ = minf + (m0 - minf) * Em, hu_ = hinf + (h0 - hinf) * Eh;
    const bool mm = mu_ >= 0.0f && mu_ <= 1.0f, mh = hu_ >= 0.0f && hu_ <= 1.0f;
    const float mv = mm ? mu_ : (mu_ < 0.0f ? 0.0f : 1.0f), hv = mh ? hu_ : (hu_ < 0.0f ? 0.0f : 1.0f);
    const float dm_dV = mm ? dminf * (1.0f - Em) + (m0 - minf) * dEm : 0.0f;
    const float dh_dV = mh ? dhinf * (1.0f - Eh) + (h0 - hinf) * dEh : 0.0f;
    const float dm_dm = mm ? Em : 0.0f, dh_dh = mh ? Eh : 0.0f;
    const float cdiv = 1.0f + (ttx > 0.0f ? ttx : 0.0f) / (is12 ? 10.0f : 5.0f);
    const float open = mv * mv * mv * hv / cdiv;
    const float do_dm = 3.0f * mv * mv * hv / cdiv, do_dh = mv * mv * mv / cdiv;
    const float gamma = is12 ? 20.8f : 20.7f;
    const float Kc = (float)((double)gamma * 1e-12 * (kR * kT) / (kF * kF * (double)55.964f) * 1e12) * area;
    const GhkF G = ghk_mono_f(V, cin, cout);
    const float I = Kc * G.F * den * open;
    const float cpv = (float)(kF * vol / 1000.0);
    const bool mci = cin - I * dt / cpv >= 1e-9f;
    const bool mco = cout + I * dt / (cpv * (float)kEVR) >= 1e-9f;
    const float lI = -lo[5] - (mci ? lo[3] * dt / cpv : 0.0f) + (mco ? lo[4] * dt / (cpv * (float)kEVR) : 0.0f);
    const float lopen = lI * Kc * G.F * den;
    const float lF = lI * Kc * den * open;
    const float lmv = lo[1] + lopen * do_dm, lhv = lo[2] + lopen * do_dh;
    const float lVc = lo[0] + lF * G.dV + lmv * dm_dV + lhv * dh_dV;
    lx[0] = mV ? lVc : 0.0f;
    lx[1] = lmv * dm_dm;
    lx[2] = lhv * dh_dh;
    lx[3] = (mci ? lo[3] : 0.0f) + lF * G.dci;
    lx[4] = (mco ? lo[4] : 0.0f) + lF * G.dco;
    lx[5] = lI * Kc * G.F * open;
}

__device__ __forceinline__ void vjp_kvdr_f(const float* lo, float* lx, float V, float n0, float cin, float cout,
                                           float den, float area, double vol, float dt, const float* st) {
    const float V_half = (st[1] != 0.0f) ? st[1] : -30.0f;
    const float k = (st[2] > 0.0f) ? st[2] : 6.0f;
    float tau, dtau;
    if (st[4] > 0.0f) { tau = st[4]; dtau = 0.0f; }
    else {
        const float t0 = 14.6f * expf(-(V - V_half) / 30.1f);
        if (t0 < 0.3f) { tau = 0.3f; dtau = 0.0f; }
        else if (t0 > 200.0f) { tau = 200.0f; dtau = 0.0f; }
        else { tau = t0; dtau = -t0 / 30.1f; }
    }
    float minf, dminf;
    logistic_f(-(V - V_half) / (k + 1e-6f), &minf, &dminf);
    dminf *= -1.0f / (k + 1e-6f);
    const float tt = tau + 1e-6f;
    const float nu = n0 + (minf - n0) * dt / tt;
    const bool mn = nu >= 0.0f && nu <= 1.0f;
    const float nv = mn ? nu : (nu < 0.0f ? 0.0f : 1.0f);
    const float dn_dV = mn ? (dminf * dt / tt - (minf - n0) * dt * dtau / (tt * tt)) : 0.0f;
    const float dn_dn = mn ? 1.0f - dt / tt : 0.0f;
    const float Kc = (float)(12.0 * 1e-12 * (kR * kT) / (kF * kF * (double)40.514f) * 1e12) * area;
    const GhkF G = ghk_mono_f(V, cin, cout);
    const float I = Kc * G.F * den * nv;
    const float cpmv = (float)(kF * vol / 1000.0);
    const bool mci = cin - I * dt / cpmv >= 1e-9f;
    const bool mco = cout + I * dt / (cpmv * (float)kEVR) >= 1e-9f;
    const float lI = -lo[5] - (mci ? lo[3] * dt / cpmv : 0.0f) + (mco ? lo[4] * dt / (cpmv * (float)kEVR) : 0.0f);
    const float lF = lI * Kc * den * nv;
    const float lnv = lo[1] + lI * Kc * G.F * den;
    lx[0] = lo[0] + lF * G.dV + lnv * dn_dV;
    lx[1] = lnv * dn_dn;
    lx[2] = 0.0f;
    lx[3] = (mci ? lo[3] : 0.0f) + lF * G.dci;
    lx[4] = (mco ? lo[4] : 0.0f) + lF * G.dco;
    lx[5] = lI * Kc * G.F * nv;
}

__device__ __forceinline__ void vjp_k2p_f(const float* lo, float* lx, float V, float cin, float cout, float den,
                                          float area, double vol, float dt, const float* st) {
    const double gamma = (st[0] > 0.0f) ? (double)st[0] : 100.0;
    const double Po = (st[1] > 0.0f) ? (double)st[1] : (double)0.012f;
    const float Kc = (float)((double)(float)gamma * 1e-12 * (kR * kT) / (kF * kF * (double)40.514f) * 1e12 * Po) * area;
    const GhkF G = ghk_mono_f(V, cin, cout);
    const float I = Kc * G.F * den;
    const float cpv = (float)(kF * vol / 1000.0);
    const bool mco = cout + I * dt / (cpv * (float)kEVR) >= 1e-9f;
    const float lI = -lo[5] - lo[3] * dt / cpv + (mco ? lo[4] * dt / (cpv * (float)kEVR) : 0.0f);
    const float lF = lI * Kc * den;
    lx[0] = lo[0] + lF * G.dV;
    lx[1] = lx[2] = 0.0f;
    lx[3] = lo[3] + lF * G.dci;
    lx[4] = (mco ? lo[4] : 0.0f) + lF * G.dco;
    lx[5] = lI * Kc * G.F;
}

// Scharfetter-Gummel Bernoulli function B(x) = x / (e^x - 1) and B'(x) in single
// precision, one exponential for both; B(-x) = B(x) + x and B'(-x) = -(B'(x) + 1).
__device__ __forceinline__ void bern_pair(float x, float ex, float* B, float* dB) {
    if (fabsf(x) < 1e-3f) { *B = 1.0f - 0.5f * x; *dB = -0.5f; return; }
    if (x > 50.0f) { *B = 0.0f; *dB = 0.0f; return; }
    if (x < -50.0f) { *B = -x; *dB = -1.0f; return; }
    const float em = ex - 1.0f;
    *B = x / em;
    *dB = (em - x * ex) / (em * em);
}

// diffusion_kernel.h:108-113 and its derivative
__device__ __forceinline__ float bern(float x, float ex) {   // ex = exp(x) when needed
    if (fabsf(x) < 1e-3f) return 1.0f - 0.5f * x;
    if (x > 50.0f) return 0.0f;
    if (x < -50.0f) return -x;
    return x / (ex - 1.0f);
}
__device__ __forceinline__ double bern_d(float x) {
    if (fabsf(x) < 1e-3f) return -0.5;
    if (x > 50.0f) return 0.0;
    if (x < -50.0f) return -1.0;
    const double e = exp((double)x), em = e - 1.0;
    return (em - (double)x * e) / (em * em);
}

}  // namespace adj
}  // namespace bnc
