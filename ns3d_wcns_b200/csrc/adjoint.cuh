// adjoint.cuh -- hand-written reverse mode (vector-Jacobian products) of the
// face flux and of the pointwise viscous flux.
//
// Every function recomputes its forward intermediates and propagates the
// adjoint back through them; branches (entropy fix, |lambda| signs, WENO
// nonlinear weights) are differentiated where they are active.  All of it is
// __host__ __device__ so the same code is verified against finite
// differences on the host (tests/test_adjoint_cpu.py through
// ns3d_debug_face_vjp) and runs in the adjoint kernels.
//
// Supported: WENO5, MDCD_LINEAR and MDCD_HYBRID component-wise
// interpolation; Roe, Rusanov, HLL and HLLC fluxes.  MDCD_HYBRID's detector
// is a switch: its derivative is zero, and the active branch (linear or
// WENO) is differentiated.  The state differentiated is the conserved U (the
// c2p/p2c round trip of runge_kutta_3 is the identity mathematically).
#pragma once

#include <math.h>

#include "common.cuh"
#include "schemes.cuh"

#ifndef NS3D_HD
#define NS3D_HD __host__ __device__ __forceinline__
#endif

namespace ns3d {
namespace adj {

// ----------------------------------------------------------- interpolation

// Forward WENO5 (same function as schemes.cuh's weno5) and its VJP:
// f[0..4] -> q; fb[0..4] += dq/df * qb.
template <typename R>
NS3D_HD R weno5_fwd(const R *f) {
    const R eps = R(1e-6), c13 = R(13.0 / 12.0);
    R t0 = f[0] - R(2) * f[1] + f[2], u0 = f[0] - R(4) * f[1] + R(3) * f[2];
    R t1 = f[1] - R(2) * f[2] + f[3], u1 = f[1] - f[3];
    R t2 = f[2] - R(2) * f[3] + f[4], u2 = R(3) * f[2] - R(4) * f[3] + f[4];
    R b0 = c13 * t0 * t0 + R(0.25) * u0 * u0, b1 = c13 * t1 * t1 + R(0.25) * u1 * u1;
    R b2 = c13 * t2 * t2 + R(0.25) * u2 * u2;
    R s0 = (eps + b0) * (eps + b0), s1 = (eps + b1) * (eps + b1), s2 = (eps + b2) * (eps + b2);
    R a0 = R(1.0 / 16.0) * s1 * s2, a1 = R(5.0 / 8.0) * s0 * s2, a2 = R(5.0 / 16.0) * s0 * s1;
    R p0 = R(3) * f[0] - R(10) * f[1] + R(15) * f[2];
    R p1 = -f[1] + R(6) * f[2] + R(3) * f[3];
    R p2 = R(3) * f[2] + R(6) * f[3] - f[4];
    return (a0 * p0 + a1 * p1 + a2 * p2) / (R(8) * (a0 + a1 + a2));
}

template <typename R>
NS3D_HD void weno5_vjp(const R *f, R qb, R *fb) {
    const R eps = R(1e-6), c13 = R(13.0 / 12.0);
    R t0 = f[0] - R(2) * f[1] + f[2], u0 = f[0] - R(4) * f[1] + R(3) * f[2];
    R t1 = f[1] - R(2) * f[2] + f[3], u1 = f[1] - f[3];
    R t2 = f[2] - R(2) * f[3] + f[4], u2 = R(3) * f[2] - R(4) * f[3] + f[4];
    R b0 = c13 * t0 * t0 + R(0.25) * u0 * u0, b1 = c13 * t1 * t1 + R(0.25) * u1 * u1;
    R b2 = c13 * t2 * t2 + R(0.25) * u2 * u2;
    R e0 = eps + b0, e1 = eps + b1, e2 = eps + b2;
    R s0 = e0 * e0, s1 = e1 * e1, s2 = e2 * e2;
    R a0 = R(1.0 / 16.0) * s1 * s2, a1 = R(5.0 / 8.0) * s0 * s2, a2 = R(5.0 / 16.0) * s0 * s1;
    R A = a0 + a1 + a2;
    R w0 = a0 / A, w1 = a1 / A, w2 = a2 / A;  // normalised weights
    R p0 = (R(3) * f[0] - R(10) * f[1] + R(15) * f[2]) * R(0.125);
    R p1 = (-f[1] + R(6) * f[2] + R(3) * f[3]) * R(0.125);
    R p2 = (R(3) * f[2] + R(6) * f[3] - f[4]) * R(0.125);
    R q = w0 * p0 + w1 * p1 + w2 * p2;
    // candidates
    R pb0 = w0 * qb, pb1 = w1 * qb, pb2 = w2 * qb;
    fb[0] += R(0.375) * pb0;
    fb[1] += R(-1.25) * pb0 - R(0.125) * pb1;
    fb[2] += R(1.875) * pb0 + R(0.75) * pb1 + R(0.375) * pb2;
    fb[3] += R(0.375) * pb1 + R(0.75) * pb2;
    fb[4] += R(-0.125) * pb2;
    // weights: alpha_k = d_k / e_k^2, d q / d beta_k = -2 w_k (p_k - q) / e_k
    R bb0 = R(-2) * qb * w0 * (p0 - q) / e0;
    R bb1 = R(-2) * qb * w1 * (p1 - q) / e1;
    R bb2 = R(-2) * qb * w2 * (p2 - q) / e2;
    R tb, ub;
    tb = R(2) * c13 * t0 * bb0; ub = R(0.5) * u0 * bb0;
    fb[0] += tb + ub; fb[1] += R(-2) * tb - R(4) * ub; fb[2] += tb + R(3) * ub;
    tb = R(2) * c13 * t1 * bb1; ub = R(0.5) * u1 * bb1;
    fb[1] += tb + ub; fb[2] += R(-2) * tb; fb[3] += tb - ub;
    tb = R(2) * c13 * t2 * bb2; ub = R(0.5) * u2 * bb2;
    fb[2] += tb + R(3) * ub; fb[3] += R(-2) * tb - R(4) * ub; fb[4] += tb + ub;
}

// MDCD_HYBRID's WENO branch (mdcd_weno_branch, interpolation.cpp:170-208)
// VJP: q = sum al_k q_k / (8 sum al_k), al_k = d_k (20 + tau6/(beta_k + 1e-40))^2,
// tau6 = |beta3 - (beta0 + 4 beta1 + beta2)/6|; fb[0..5] += dq/df * qb.
template <typename R>
NS3D_HD void mdcd_weno_vjp(const R *f, const R *hd, R qb, R *fb) {
    const R c13 = R(13.0 / 12.0), es = R(1e-40);
    const R t0 = f[0] - R(2) * f[1] + f[2], u0 = f[0] - R(4) * f[1] + R(3) * f[2];
    const R t1 = f[1] - R(2) * f[2] + f[3], u1 = f[1] - f[3];
    const R t2 = f[2] - R(2) * f[3] + f[4], u2 = R(3) * f[2] - R(4) * f[3] + f[4];
    const R be[4] = {c13 * (t0 * t0) + R(0.25) * (u0 * u0), c13 * (t1 * t1) + R(0.25) * (u1 * u1),
                     c13 * (t2 * t2) + R(0.25) * (u2 * u2), mdcd_beta3(f[0], f[1], f[2], f[3], f[4], f[5])};
    const R qk[4] = {R(3) * f[0] - R(10) * f[1] + R(15) * f[2], -f[1] + R(6) * f[2] + R(3) * f[3],
                     R(3) * f[2] + R(6) * f[3] - f[4], R(15) * f[3] - R(10) * f[4] + R(3) * f[5]};
    const R D = be[3] - (be[0] + R(4) * be[1] + be[2]) / R(6);
    const R tau = fabs(D);
    R g[4], al[4], A = R(0), Q = R(0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        g[k] = R(20) + tau / (be[k] + es);
        al[k] = hd[k] * (g[k] * g[k]);
        A += al[k];
        Q += al[k] * qk[k];
    }
    const R q = Q / (R(8) * A);
    R qkb[4], beb[4], taub = R(0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        qkb[k] = qb * al[k] / (R(8) * A);
        const R alb = qb * (qk[k] * R(0.125) - q) / A;
        const R gb = alb * R(2) * hd[k] * g[k];
        const R ib = R(1) / (be[k] + es);
        taub += gb * ib;
        beb[k] = -gb * tau * ib * ib;
    }
    const R Db = D >= R(0) ? taub : -taub;
    beb[3] += Db;
    beb[0] -= Db / R(6);
    beb[1] -= R(4) * Db / R(6);
    beb[2] -= Db / R(6);
    // candidates
    fb[0] += R(3) * qkb[0];
    fb[1] += R(-10) * qkb[0] - qkb[1];
    fb[2] += R(15) * qkb[0] + R(6) * qkb[1] + R(3) * qkb[2];
    fb[3] += R(3) * qkb[1] + R(6) * qkb[2] + R(15) * qkb[3];
    fb[4] += -qkb[2] - R(10) * qkb[3];
    fb[5] += R(3) * qkb[3];
    // beta0..beta2
    R tb = R(2) * c13 * t0 * beb[0], ub = R(0.5) * u0 * beb[0];
    fb[0] += tb + ub; fb[1] += R(-2) * tb - R(4) * ub; fb[2] += tb + R(3) * ub;
    tb = R(2) * c13 * t1 * beb[1]; ub = R(0.5) * u1 * beb[1];
    fb[1] += tb + ub; fb[2] += R(-2) * tb; fb[3] += tb - ub;
    tb = R(2) * c13 * t2 * beb[2]; ub = R(0.5) * u2 * beb[2];
    fb[2] += tb + R(3) * ub; fb[3] += R(-2) * tb - R(4) * ub; fb[4] += tb + ub;
    // beta3: gradient of the quadratic form of interpolation.cpp:193-200
    const R b3 = beb[3] / R(120960);
    fb[0] += b3 * (R(543598) * f[0] - R(2380800) * f[1] + R(4086352) * f[2] - R(3462252) * f[3] +
                   R(1458762) * f[4] - R(245620) * f[5]);
    fb[1] += b3 * (R(-2380800) * f[0] + R(11306634) * f[1] - R(20427884) * f[2] + R(17905032) * f[3] -
                   R(7727988) * f[4] + R(1325006) * f[5]);
    fb[2] += b3 * (R(4086352) * f[0] - R(20427884) * f[1] + R(39021944) * f[2] - R(35817664) * f[3] +
                   R(15929912) * f[4] - R(2792660) * f[5]);
    fb[3] += b3 * (R(-3462252) * f[0] + R(17905032) * f[1] - R(35817664) * f[2] + R(34391304) * f[3] -
                   R(15880404) * f[4] + R(2863984) * f[5]);
    fb[4] += b3 * (R(1458762) * f[0] - R(7727988) * f[1] + R(15929912) * f[2] - R(15880404) * f[3] +
                   R(7649694) * f[4] - R(1429976) * f[5]);
    fb[5] += b3 * (R(-245620) * f[0] + R(1325006) * f[1] - R(2792660) * f[2] + R(2863984) * f[3] -
                   R(1429976) * f[4] + R(279266) * f[5]);
}

// Left and right interpolated states of one variable at a face from its
// stencil f[0..5] (cells i-2 .. i+3) -- INTERP 0 WENO5, 2 MDCD_LINEAR,
// 3 MDCD_HYBRID (the decision of both sides is the detector at cells i and
// i+1, as in the sweeps) -- and their VJP into gb[0..5].
template <typename R, int INTERP>
NS3D_HD void interp_pair_fwd(const R *f, const R *lin, const R *hd, R &l, R &r) {
    const R fr[6] = {f[5], f[4], f[3], f[2], f[1], f[0]};
    if constexpr (INTERP == 0) {
        l = weno5_fwd(f);
        r = weno5_fwd(fr);
        return;
    }
    if constexpr (INTERP == 3) {
        if (!(mdcd_smooth(f[0], f[1], f[2], f[3], f[4]) && mdcd_smooth(f[1], f[2], f[3], f[4], f[5]))) {
            l = mdcd_weno_branch(hd, f[0], f[1], f[2], f[3], f[4], f[5]);
            r = mdcd_weno_branch(hd, fr[0], fr[1], fr[2], fr[3], fr[4], fr[5]);
            return;
        }
    }
    l = R(0);
    r = R(0);
#pragma unroll
    for (int m = 0; m < 6; ++m) { l += lin[m] * f[m]; r += lin[m] * fr[m]; }
}

template <typename R, int INTERP>
NS3D_HD void interp_pair_vjp(const R *f, const R *lin, const R *hd, R lb, R rb, R *gb) {
#pragma unroll
    for (int m = 0; m < 6; ++m) gb[m] = R(0);
    if constexpr (INTERP == 0) {
        R fbl[5] = {0, 0, 0, 0, 0}, fbr[5] = {0, 0, 0, 0, 0};
        weno5_vjp(f, lb, fbl);
        const R fr[5] = {f[5], f[4], f[3], f[2], f[1]};
        weno5_vjp(fr, rb, fbr);
        gb[0] = fbl[0]; gb[5] = fbr[0];
#pragma unroll
        for (int m = 1; m < 5; ++m) gb[m] = fbl[m] + fbr[5 - m];
        return;
    }
    if constexpr (INTERP == 3) {
        if (!(mdcd_smooth(f[0], f[1], f[2], f[3], f[4]) && mdcd_smooth(f[1], f[2], f[3], f[4], f[5]))) {
            R fbr[6] = {0, 0, 0, 0, 0, 0};
            const R fr[6] = {f[5], f[4], f[3], f[2], f[1], f[0]};
            mdcd_weno_vjp(f, hd, lb, gb);
            mdcd_weno_vjp(fr, hd, rb, fbr);
#pragma unroll
            for (int m = 0; m < 6; ++m) gb[m] += fbr[5 - m];
            return;
        }
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) gb[m] = lin[m] * lb + lin[5 - m] * rb;
}

// ------------------------------------------------------------ Riemann VJPs

template <typename R>
struct SideF {
    R r, ir, u, v, w, E, q2, p;
};

template <typename R>
NS3D_HD SideF<R> side_fwd(const R *U, R g) {
    SideF<R> s;
    s.r = U[0]; s.ir = R(1) / s.r;
    s.u = U[1] * s.ir; s.v = U[2] * s.ir; s.w = U[3] * s.ir; s.E = U[4];
    s.q2 = s.u * s.u + s.v * s.v + s.w * s.w;
    s.p = (s.E - R(0.5) * s.r * s.q2) * (g - R(1));
    return s;
}

// adjoint of (u, v, w, p, E-direct, r-direct) back to U
template <typename R>
NS3D_HD void side_vjp(const SideF<R> &s, R g, R ub, R vb, R wb, R pb, R Eb, R rb, R *Ub) {
    // p = (E - 0.5 r q2)(g-1)
    Eb += pb * (g - R(1));
    rb -= R(0.5) * s.q2 * (g - R(1)) * pb;
    R q2b = R(-0.5) * s.r * (g - R(1)) * pb;
    ub += R(2) * s.u * q2b; vb += R(2) * s.v * q2b; wb += R(2) * s.w * q2b;
    // u = U1 * ir, ir = 1/r
    Ub[1] += ub * s.ir; Ub[2] += vb * s.ir; Ub[3] += wb * s.ir;
    R irb = ub * s.u * s.r + vb * s.v * s.r + wb * s.w * s.r;  // U1 = u r
    rb += -irb * s.ir * s.ir;
    Ub[0] += rb;
    Ub[4] += Eb;
}

// physical flux F(U) along direction DIR and its VJP into (u,v,w,p,E,r) adjoints
template <int DIR, typename R>
NS3D_HD void pflux_fwd(const SideF<R> &s, R *F) {
    R un = DIR == 0 ? s.u : (DIR == 1 ? s.v : s.w);
    R m = s.r * un;
    F[0] = m;
    F[1] = m * s.u + (DIR == 0 ? s.p : R(0));
    F[2] = m * s.v + (DIR == 1 ? s.p : R(0));
    F[3] = m * s.w + (DIR == 2 ? s.p : R(0));
    F[4] = (s.E + s.p) * un;
}

template <int DIR, typename R>
NS3D_HD void pflux_vjp(const SideF<R> &s, const R *Fb, R &ub, R &vb, R &wb, R &pb, R &Eb, R &rb) {
    R un = DIR == 0 ? s.u : (DIR == 1 ? s.v : s.w);
    R m = s.r * un;
    R mb = Fb[0] + Fb[1] * s.u + Fb[2] * s.v + Fb[3] * s.w;
    ub += Fb[1] * m; vb += Fb[2] * m; wb += Fb[3] * m;
    pb += (DIR == 0 ? Fb[1] : DIR == 1 ? Fb[2] : Fb[3]) + Fb[4] * un;
    Eb += Fb[4] * un;
    R unb = Fb[4] * (s.E + s.p) + mb * s.r;
    rb += mb * un;
    if (DIR == 0) ub += unb; else if (DIR == 1) vb += unb; else wb += unb;
}

// entropy fix of Roe_Riemann_solver (InviscousFlux.cpp:364-373) on |lambda|
template <typename R>
NS3D_HD R efix(R l, R d) { return l < d ? (l * l + d * d) / (R(2) * d) : l; }

// Roe flux: same function as schemes.cuh roe_flux; VJP accumulates ULb, URb.
template <int DIR, typename R>
NS3D_HD void roe_vjp(const R *UL, const R *UR, R g, const R *Fb, R *ULb, R *URb) {
    const R gm1 = g - R(1), kfac = g / gm1;
    SideF<R> L = side_fwd(UL, g), Rs = side_fwd(UR, g);
    R HL = R(0.5) * L.q2 + kfac * L.p * L.ir, HR = R(0.5) * Rs.q2 + kfac * Rs.p * Rs.ir;
    R sL = sqrt(L.r), sR = sqrt(Rs.r);
    R den = R(1) / (sL + sR);
    R ub = (sL * L.u + sR * Rs.u) * den, vb = (sL * L.v + sR * Rs.v) * den, wb = (sL * L.w + sR * Rs.w) * den;
    R Hb = (sL * HL + sR * HR) * den;
    R q2b = ub * ub + vb * vb + wb * wb;
    R c2 = gm1 * (Hb - R(0.5) * q2b);
    R c = sqrt(c2);
    R V = DIR == 0 ? ub : (DIR == 1 ? vb : wb);
    R phi = R(0.5) * gm1 * q2b;
    R dU[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) dU[n] = UR[n] - UL[n];
    const R dUn = dU[1 + DIR];
    R t = phi * dU[0] + gm1 * (dU[4] - ub * dU[1] - vb * dU[2] - wb * dU[3]);
    R s = c * (V * dU[0] - dUn);
    R i2c2 = R(1) / (R(2) * c2);
    R A0 = (t + s) * i2c2, A4 = (t - s) * i2c2;
    R l0 = fabs(V - c), lv = fabs(V), l4 = fabs(V + c);
    R delta = R(0.1) * (lv + c);
    R l0f = efix(l0, delta), lvf = efix(lv, delta), l4f = efix(l4, delta);
    R k0 = (l0f - lvf) * A0, k4 = (l4f - lvf) * A4;
    const R e0 = DIR == 0 ? R(1) : R(0), e1 = DIR == 1 ? R(1) : R(0), e2 = DIR == 2 ? R(1) : R(0);
    // ---- reverse
    R Db[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) Db[n] = R(-0.5) * Fb[n];
    R FLb[5], FRb[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) { FLb[n] = R(0.5) * Fb[n]; FRb[n] = R(0.5) * Fb[n]; }
    R dUb[5];
    R lvfb = R(0);
#pragma unroll
    for (int n = 0; n < 5; ++n) { lvfb += Db[n] * dU[n]; dUb[n] = lvf * Db[n]; }
    R k0b = Db[0] + Db[1] * (ub - c * e0) + Db[2] * (vb - c * e1) + Db[3] * (wb - c * e2) + Db[4] * (Hb - c * V);
    R k4b = Db[0] + Db[1] * (ub + c * e0) + Db[2] * (vb + c * e1) + Db[3] * (wb + c * e2) + Db[4] * (Hb + c * V);
    R ubb = (k0 + k4) * Db[1], vbb = (k0 + k4) * Db[2], wbb = (k0 + k4) * Db[3], Hbb = (k0 + k4) * Db[4];
    R Dbn = DIR == 0 ? Db[1] : (DIR == 1 ? Db[2] : Db[3]);
    R cb = (k4 - k0) * (Dbn + V * Db[4]);
    R Vb = c * (k4 - k0) * Db[4];
    R l0fb = k0b * A0, l4fb = k4b * A4;
    lvfb -= k0b * A0 + k4b * A4;
    R A0b = k0b * (l0f - lvf), A4b = k4b * (l4f - lvf);
    // entropy fix
    R deltab = R(0);
    auto fixb = [&](R l, R lfb) -> R {  // returns lb, accumulates deltab
        if (l < delta) {
            deltab += lfb * (R(0.5) - l * l / (R(2) * delta * delta));
            return lfb * l / delta;
        }
        return lfb;
    };
    R l0b = fixb(l0, l0fb), lvb = fixb(lv, lvfb), l4b = fixb(l4, l4fb);
    lvb += R(0.1) * deltab;
    cb += R(0.1) * deltab;
    R sg0 = (V - c) >= R(0) ? R(1) : R(-1), sgv = V >= R(0) ? R(1) : R(-1), sg4 = (V + c) >= R(0) ? R(1) : R(-1);
    Vb += sg0 * l0b + sgv * lvb + sg4 * l4b;
    cb += -sg0 * l0b + sg4 * l4b;
    R tb = (A0b + A4b) * i2c2, sb = (A0b - A4b) * i2c2;
    R i2c2b = A0b * (t + s) + A4b * (t - s);
    R c2b = i2c2b * (R(-2) * i2c2 * i2c2);
    // s = c (V dU0 - dUn)
    cb += sb * (V * dU[0] - dUn);
    Vb += sb * c * dU[0];
    dUb[0] += sb * c * V;
    dUb[1 + DIR] -= sb * c;
    // t = phi dU0 + gm1 (dU4 - ub dU1 - vb dU2 - wb dU3)
    R phib = tb * dU[0];
    dUb[0] += tb * phi;
    dUb[4] += tb * gm1;
    dUb[1] -= tb * gm1 * ub; dUb[2] -= tb * gm1 * vb; dUb[3] -= tb * gm1 * wb;
    ubb -= tb * gm1 * dU[1]; vbb -= tb * gm1 * dU[2]; wbb -= tb * gm1 * dU[3];
    R q2bb = R(0.5) * gm1 * phib;
    if (DIR == 0) ubb += Vb; else if (DIR == 1) vbb += Vb; else wbb += Vb;
    c2b += cb / (R(2) * c);
    Hbb += gm1 * c2b;
    q2bb -= R(0.5) * gm1 * c2b;
    ubb += R(2) * ub * q2bb; vbb += R(2) * vb * q2bb; wbb += R(2) * wb * q2bb;
    // Roe averages
    R sLb = den * (ubb * L.u + vbb * L.v + wbb * L.w + Hbb * HL);
    R sRb = den * (ubb * Rs.u + vbb * Rs.v + wbb * Rs.w + Hbb * HR);
    R denb = ubb * (sL * L.u + sR * Rs.u) + vbb * (sL * L.v + sR * Rs.v) + wbb * (sL * L.w + sR * Rs.w) +
             Hbb * (sL * HL + sR * HR);
    sLb -= denb * den * den;
    sRb -= denb * den * den;
    R uLb = ubb * sL * den, vLb = vbb * sL * den, wLb = wbb * sL * den, HLb = Hbb * sL * den;
    R uRb = ubb * sR * den, vRb = vbb * sR * den, wRb = wbb * sR * den, HRb = Hbb * sR * den;
    R rLb = sLb / (R(2) * sL), rRb = sRb / (R(2) * sR);
    // H = 0.5 q2 + kfac p ir
    R pLb = kfac * L.ir * HLb, pRb = kfac * Rs.ir * HRb;
    uLb += L.u * HLb; vLb += L.v * HLb; wLb += L.w * HLb;   // d(0.5 q2)/du = u
    uRb += Rs.u * HRb; vRb += Rs.v * HRb; wRb += Rs.w * HRb;
    R irLb = kfac * L.p * HLb, irRb = kfac * Rs.p * HRb;
    rLb += -irLb * L.ir * L.ir;
    rRb += -irRb * Rs.ir * Rs.ir;
    R ELb = R(0), ERb = R(0);
    pflux_vjp<DIR, R>(L, FLb, uLb, vLb, wLb, pLb, ELb, rLb);
    pflux_vjp<DIR, R>(Rs, FRb, uRb, vRb, wRb, pRb, ERb, rRb);
    side_vjp(L, g, uLb, vLb, wLb, pLb, ELb, rLb, ULb);
    side_vjp(Rs, g, uRb, vRb, wRb, pRb, ERb, rRb, URb);
#pragma unroll
    for (int n = 0; n < 5; ++n) { URb[n] += dUb[n]; ULb[n] -= dUb[n]; }
}

// Rusanov flux (InviscousFlux.cpp:270-311) VJP.
template <int DIR, typename R>
NS3D_HD void rusanov_vjp(const R *UL, const R *UR, R g, const R *Fb, R *ULb, R *URb) {
    SideF<R> L = side_fwd(UL, g), Rs = side_fwd(UR, g);
    R unL = DIR == 0 ? L.u : (DIR == 1 ? L.v : L.w), unR = DIR == 0 ? Rs.u : (DIR == 1 ? Rs.v : Rs.w);
    R aL = sqrt(g * L.p * L.ir), aR = sqrt(g * Rs.p * Rs.ir);
    R sl = fabs(unL) + aL, sr = fabs(unR) + aR;
    bool left = !(sl < sr);  // std::max(a,b) returns a unless a < b
    R smax = left ? sl : sr;
    R FLb[5], FRb[5], smaxb = R(0);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
        FLb[n] = R(0.5) * Fb[n]; FRb[n] = R(0.5) * Fb[n];
        smaxb += R(-0.5) * Fb[n] * (UR[n] - UL[n]);
        URb[n] += R(-0.5) * smax * Fb[n];
        ULb[n] += R(0.5) * smax * Fb[n];
    }
    R uLb = 0, vLb = 0, wLb = 0, pLb = 0, ELb = 0, rLb = 0, uRb = 0, vRb = 0, wRb = 0, pRb = 0, ERb = 0, rRb = 0;
    // smax = |un| + sqrt(g p / r)
    if (left) {
        R unb = (unL >= R(0) ? R(1) : R(-1)) * smaxb;
        if (DIR == 0) uLb += unb; else if (DIR == 1) vLb += unb; else wLb += unb;
        R ab = smaxb, x = g * L.p * L.ir;
        R xb = ab / (R(2) * aL);
        pLb += xb * g * L.ir;
        rLb += -(xb * g * L.p) * L.ir * L.ir;
        (void)x;
    } else {
        R unb = (unR >= R(0) ? R(1) : R(-1)) * smaxb;
        if (DIR == 0) uRb += unb; else if (DIR == 1) vRb += unb; else wRb += unb;
        R xb = smaxb / (R(2) * aR);
        pRb += xb * g * Rs.ir;
        rRb += -(xb * g * Rs.p) * Rs.ir * Rs.ir;
    }
    pflux_vjp<DIR, R>(L, FLb, uLb, vLb, wLb, pLb, ELb, rLb);
    pflux_vjp<DIR, R>(Rs, FRb, uRb, vRb, wRb, pRb, ERb, rRb);
    side_vjp(L, g, uLb, vLb, wLb, pLb, ELb, rLb, ULb);
    side_vjp(Rs, g, uRb, vRb, wRb, pRb, ERb, rRb, URb);
}

// HLL flux (InviscousFlux.cpp:384-447) VJP.
template <int DIR, typename R>
NS3D_HD void hll_vjp(const R *UL, const R *UR, R g, const R *Fb, R *ULb, R *URb) {
    SideF<R> L = side_fwd(UL, g), Rs = side_fwd(UR, g);
    R unL = DIR == 0 ? L.u : (DIR == 1 ? L.v : L.w), unR = DIR == 0 ? Rs.u : (DIR == 1 ? Rs.v : Rs.w);
    R aL = sqrt(g * L.p * L.ir), aR = sqrt(g * Rs.p * Rs.ir);
    R a = unL - aL, b = unR - aR;
    bool sl_right = b < a;  // SL = min -> b when b < a
    R SL = sl_right ? b : a;
    a = unL + aL; b = unR + aR;
    bool sr_right = a < b;  // SR = max -> b when a < b
    R SR = sr_right ? b : a;
    R FL[5], FR[5];
    pflux_fwd<DIR, R>(L, FL);
    pflux_fwd<DIR, R>(Rs, FR);
    R uLb = 0, vLb = 0, wLb = 0, pLb = 0, ELb = 0, rLb = 0, uRb = 0, vRb = 0, wRb = 0, pRb = 0, ERb = 0, rRb = 0;
    R FLb[5] = {0, 0, 0, 0, 0}, FRb[5] = {0, 0, 0, 0, 0};
    if (SL >= R(0)) {
#pragma unroll
        for (int n = 0; n < 5; ++n) FLb[n] = Fb[n];
    } else if (SR <= R(0)) {
#pragma unroll
        for (int n = 0; n < 5; ++n) FRb[n] = Fb[n];
    } else {
        R id = R(1) / (SR - SL);
        R SLb = 0, SRb = 0;
#pragma unroll
        for (int n = 0; n < 5; ++n) {
            R dUn = UR[n] - UL[n];
            R F = (SR * FL[n] - SL * FR[n] + SL * SR * dUn) * id;
            FLb[n] = SR * id * Fb[n];
            FRb[n] = -SL * id * Fb[n];
            URb[n] += SL * SR * id * Fb[n];
            ULb[n] -= SL * SR * id * Fb[n];
            // d/dSR: (FL + SL dU) id - F id ; d/dSL: (-FR + SR dU) id + F id
            SRb += Fb[n] * ((FL[n] + SL * dUn) * id - F * id);
            SLb += Fb[n] * ((-FR[n] + SR * dUn) * id + F * id);
        }
        // SL, SR -> un and a of the selected sides
        auto add_speed = [&](bool rightside, R sgn_a, R sb) {
            // speed = un + sgn_a * a
            if (!rightside) {
                if (DIR == 0) uLb += sb; else if (DIR == 1) vLb += sb; else wLb += sb;
                R xb = sgn_a * sb / (R(2) * aL);
                pLb += xb * g * L.ir;
                rLb += -(xb * g * L.p) * L.ir * L.ir;
            } else {
                if (DIR == 0) uRb += sb; else if (DIR == 1) vRb += sb; else wRb += sb;
                R xb = sgn_a * sb / (R(2) * aR);
                pRb += xb * g * Rs.ir;
                rRb += -(xb * g * Rs.p) * Rs.ir * Rs.ir;
            }
        };
        add_speed(sl_right, R(-1), SLb);
        add_speed(sr_right, R(1), SRb);
    }
    pflux_vjp<DIR, R>(L, FLb, uLb, vLb, wLb, pLb, ELb, rLb);
    pflux_vjp<DIR, R>(Rs, FRb, uRb, vRb, wRb, pRb, ERb, rRb);
    side_vjp(L, g, uLb, vLb, wLb, pLb, ELb, rLb, ULb);
    side_vjp(Rs, g, uRb, vRb, wRb, pRb, ERb, rRb, URb);
}

// HLLC flux (HLLC_Riemann_solver, InviscousFlux.cpp:449-592, as hllc_flux of
// schemes.cuh evaluates it) VJP: Davis wave speeds S_L = min(un_L - a_L,
// un_R - a_R), S_R = max(un_L + a_L, un_R + a_R) (the active arm
// differentiated), the Batten contact speed S_M (or its Roe-average
// fallback) and the upwind side's star state.
template <int DIR, typename R>
NS3D_HD void hllc_vjp(const R *UL, const R *UR, R g, const R *Fb, R *ULb, R *URb) {
    SideF<R> L = side_fwd(UL, g), Rs = side_fwd(UR, g);
    const R unL = DIR == 0 ? L.u : (DIR == 1 ? L.v : L.w), unR = DIR == 0 ? Rs.u : (DIR == 1 ? Rs.v : Rs.w);
    const R aL = sqrt(g * L.p * L.ir), aR = sqrt(g * Rs.p * Rs.ir);
    R a = unL - aL, b = unR - aR;
    const bool sl_right = b < a;
    const R SL = sl_right ? b : a;
    a = unL + aL; b = unR + aR;
    const bool sr_right = a < b;
    const R SR = sr_right ? b : a;
    R uLb = 0, vLb = 0, wLb = 0, pLb = 0, ELb = 0, rLb = 0, irLb = 0;
    R uRb = 0, vRb = 0, wRb = 0, pRb = 0, ERb = 0, rRb = 0, irRb = 0;
    if (SL >= R(0) || SR <= R(0)) {
        const bool left = SL >= R(0);
        if (left) pflux_vjp<DIR, R>(L, Fb, uLb, vLb, wLb, pLb, ELb, rLb);
        else pflux_vjp<DIR, R>(Rs, Fb, uRb, vRb, wRb, pRb, ERb, rRb);
        side_vjp(L, g, uLb, vLb, wLb, pLb, ELb, rLb, ULb);
        side_vjp(Rs, g, uRb, vRb, wRb, pRb, ERb, rRb, URb);
        return;
    }
    const R num = Rs.r * unR * (SR - unR) - L.r * unL * (SL - unL) + L.p - Rs.p;
    const R den = Rs.r * (SR - unR) - L.r * (SL - unL);
    const bool batten = fabs(den) > R(1e-12);
    R SM;
    const R sqL = sqrt(L.r), sqR = sqrt(Rs.r);
    if (batten) SM = num / den;
    else SM = (sqL * unL + sqR * unR) / (sqL + sqR);
    // the upwind side K and its star state
    const bool left = SM >= R(0);
    const SideF<R> &K = left ? L : Rs;
    const R *UK = left ? UL : UR;
    R *UKb = left ? ULb : URb;
    const R unK = left ? unL : unR, Sk = left ? SL : SR;
    const R dk = Sk - unK, W = Sk - SM, P = K.r * dk;
    const R rs = K.r * dk / W;
    const R Z = K.p / P, X = SM - unK, Y = SM + Z;
    const R Es = K.E * K.ir + X * Y;
    const R vs[5] = {R(1), DIR == 0 ? SM : K.u, DIR == 1 ? SM : K.v, DIR == 2 ? SM : K.w, Es};
    // F_n = FK_n + Sk (rs vs_n - UK_n)
    R Skb = R(0), rsb = R(0), vsb[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
        Skb += Fb[n] * (rs * vs[n] - UK[n]);
        rsb += Sk * Fb[n] * vs[n];
        vsb[n] = Sk * rs * Fb[n];
        UKb[n] -= Sk * Fb[n];
    }
    R uKb = 0, vKb = 0, wKb = 0, pKb = 0, EKb = 0, rKb = 0, irKb = 0, unKb = 0, SMb = 0, dkb = 0;
    if (DIR == 0) SMb += vsb[1]; else uKb += vsb[1];
    if (DIR == 1) SMb += vsb[2]; else vKb += vsb[2];
    if (DIR == 2) SMb += vsb[3]; else wKb += vsb[3];
    // Es = E ir + X Y, X = SM - un, Y = SM + p / (r dk)
    const R Esb = vsb[4];
    EKb += Esb * K.ir;
    irKb += Esb * K.E;
    const R Xb = Esb * Y, Yb = Esb * X;
    SMb += Xb + Yb;
    unKb -= Xb;
    pKb += Yb / P;
    const R Pb = -Yb * K.p / (P * P);
    rKb += Pb * dk;
    dkb += Pb * K.r;
    // rs = r dk / (Sk - SM)
    rKb += rsb * dk / W;
    dkb += rsb * K.r / W;
    const R Wb = -rsb * K.r * dk / (W * W);
    Skb += Wb;
    SMb -= Wb;
    // dk = Sk - un
    Skb += dkb;
    unKb -= dkb;
    // the physical flux of side K
    pflux_vjp<DIR, R>(K, Fb, uKb, vKb, wKb, pKb, EKb, rKb);
    if (DIR == 0) uKb += unKb; else if (DIR == 1) vKb += unKb; else wKb += unKb;
    if (left) {
        uLb += uKb; vLb += vKb; wLb += wKb; pLb += pKb; ELb += EKb; rLb += rKb; irLb += irKb;
    } else {
        uRb += uKb; vRb += vKb; wRb += wKb; pRb += pKb; ERb += EKb; rRb += rKb; irRb += irKb;
    }
    R SLb = left ? Skb : R(0), SRb = left ? R(0) : Skb;
    R unLb = 0, unRb = 0;
    if (batten) {
        const R numb = SMb / den, denb = -SMb * SM / den;
        rRb += numb * unR * (SR - unR) + denb * (SR - unR);
        unRb += numb * Rs.r * (SR - R(2) * unR) - denb * Rs.r;
        SRb += numb * Rs.r * unR + denb * Rs.r;
        rLb -= numb * unL * (SL - unL) + denb * (SL - unL);
        unLb -= numb * L.r * (SL - R(2) * unL) - denb * L.r;
        SLb -= numb * L.r * unL + denb * L.r;
        pLb += numb;
        pRb -= numb;
    } else {
        const R S = sqL + sqR, N = sqL * unL + sqR * unR;
        const R Nb = SMb / S, Sb = -SMb * N / (S * S);
        unLb += Nb * sqL;
        unRb += Nb * sqR;
        rLb += (Nb * unL + Sb) / (R(2) * sqL);
        rRb += (Nb * unR + Sb) / (R(2) * sqR);
    }
    // wave speeds: S_L = un - a of the minimising side, S_R = un + a of the maximising side
    R aLb = 0, aRb = 0;
    if (sl_right) { unRb += SLb; aRb -= SLb; } else { unLb += SLb; aLb -= SLb; }
    if (sr_right) { unRb += SRb; aRb += SRb; } else { unLb += SRb; aLb += SRb; }
    // a = sqrt(g p ir)
    if (aL > R(0)) { const R xb = aLb / (R(2) * aL); pLb += xb * g * L.ir; irLb += xb * g * L.p; }
    if (aR > R(0)) { const R xb = aRb / (R(2) * aR); pRb += xb * g * Rs.ir; irRb += xb * g * Rs.p; }
    if (DIR == 0) { uLb += unLb; uRb += unRb; }
    else if (DIR == 1) { vLb += unLb; vRb += unRb; }
    else { wLb += unLb; wRb += unRb; }
    // ir = 1 / r
    rLb -= irLb * L.ir * L.ir;
    rRb -= irRb * Rs.ir * Rs.ir;
    side_vjp(L, g, uLb, vLb, wLb, pLb, ELb, rLb, ULb);
    side_vjp(Rs, g, uRb, vRb, wRb, pRb, ERb, rRb, URb);
}

// Riemann VJP by code: 0 Roe, 1 Rusanov, 2 HLL, 3 HLLC.
template <int DIR, typename R, int RS>
NS3D_HD void riemann_vjp(const R *UL, const R *UR, R g, const R *Fb, R *ULb, R *URb) {
    if constexpr (RS == 0) roe_vjp<DIR, R>(UL, UR, g, Fb, ULb, URb);
    else if constexpr (RS == 1) rusanov_vjp<DIR, R>(UL, UR, g, Fb, ULb, URb);
    else if constexpr (RS == 2) hll_vjp<DIR, R>(UL, UR, g, Fb, ULb, URb);
    else hllc_vjp<DIR, R>(UL, UR, g, Fb, ULb, URb);
}

// VJP code of a public riemann_solver value (NS3D_ROE 0, NS3D_RUSANOV 1,
// NS3D_HLLC 2, NS3D_HLL 3), -1 when it has no VJP.
NS3D_HD int adj_riemann_code(int rs) {
    return rs == 0 ? 0 : rs == 1 ? 1 : rs == 3 ? 2 : rs == 2 ? 3 : -1;
}

// ------------------------------------------------------------ face VJP

// Component-wise WCNS face flux (WCNS_Riemann_InviscidFlux, InviscousFlux.cpp:
// 146-268 with char_recon = false): U[n][m], m = cells i-2..i+3.
// INTERP: 0 WENO5, 2 MDCD_LINEAR (lin = its six coefficients), 3 MDCD_HYBRID
// (also hd = its WENO weights d0..d3); RS: a riemann_vjp code.
template <int DIR, typename R, int INTERP, int RS>
NS3D_HD void face_vjp_t(const R *lin, const R *hd, R g, const R U[5][6], const R *Fb, R Ub[5][6]) {
    R UL[5], UR[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) interp_pair_fwd<R, INTERP>(U[n], lin, hd, UL[n], UR[n]);
    R ULb[5] = {0, 0, 0, 0, 0}, URb[5] = {0, 0, 0, 0, 0};
    riemann_vjp<DIR, R, RS>(UL, UR, g, Fb, ULb, URb);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
        R gb[6];
        interp_pair_vjp<R, INTERP>(U[n], lin, hd, ULb[n], URb[n], gb);
#pragma unroll
        for (int m = 0; m < 6; ++m) Ub[n][m] += gb[m];
    }
}

// run-time selection (interp 0 WENO5 / 2 MDCD_LINEAR / 3 MDCD_HYBRID; rcode a
// riemann_vjp code)
template <int DIR, typename R, int INTERP>
NS3D_HD void face_vjp_i(int rcode, const R *lin, const R *hd, R g, const R U[5][6], const R *Fb, R Ub[5][6]) {
    if (rcode == 0) face_vjp_t<DIR, R, INTERP, 0>(lin, hd, g, U, Fb, Ub);
    else if (rcode == 1) face_vjp_t<DIR, R, INTERP, 1>(lin, hd, g, U, Fb, Ub);
    else if (rcode == 2) face_vjp_t<DIR, R, INTERP, 2>(lin, hd, g, U, Fb, Ub);
    else face_vjp_t<DIR, R, INTERP, 3>(lin, hd, g, U, Fb, Ub);
}

template <int DIR, typename R>
NS3D_HD void face_vjp(int interp, int rcode, const R *lin, const R *hd, R g, const R U[5][6], const R *Fb,
                      R Ub[5][6]) {
    if (interp == 0) face_vjp_i<DIR, R, 0>(rcode, lin, hd, g, U, Fb, Ub);
    else if (interp == 2) face_vjp_i<DIR, R, 2>(rcode, lin, hd, g, U, Fb, Ub);
    else face_vjp_i<DIR, R, 3>(rcode, lin, hd, g, U, Fb, Ub);
}

// ------------------------------------------------------------ viscous VJP

// Pointwise node viscous flux (compute_viscous_flux, ViscousFlux.cpp:151-208)
// of direction d's four components for rhou, rhov, rhow, E, and its VJP.
// x = (u, v, w, T), g[4][3] = gradients; returns xb (u,v,w,T) and gb.
template <typename R>
NS3D_HD void visc_flux_all(R mu0, R S, R cpr, const R *x, const R g[4][3], R V[9]) {
    const R T = x[3];
    const R mu = mu0 * (T * sqrt(T)) * (R(1) + S) / (T + S);
    const R div = g[0][0] + g[1][1] + g[2][2];
    const R m2 = R(2) * mu, m23 = R(2.0 / 3.0) * mu * div;
    const R txx = m2 * g[0][0] - m23, tyy = m2 * g[1][1] - m23, tzz = m2 * g[2][2] - m23;
    const R txy = mu * (g[0][1] + g[1][0]), txz = mu * (g[0][2] + g[2][0]), tyz = mu * (g[1][2] + g[2][1]);
    const R kq = mu * cpr;
    V[0] = txx; V[1] = tyy; V[2] = tzz; V[3] = txy; V[4] = txz; V[5] = tyz;
    V[6] = x[0] * txx + x[1] * txy + x[2] * txz + kq * g[3][0];
    V[7] = x[0] * txy + x[1] * tyy + x[2] * tyz + kq * g[3][1];
    V[8] = x[0] * txz + x[1] * tyz + x[2] * tzz + kq * g[3][2];
}

template <typename R>
NS3D_HD void visc_flux_vjp(R mu0, R S, R cpr, const R *x, const R g[4][3], const R *Vb, R *xb, R gb[4][3]) {
    const R T = x[3];
    const R sq = sqrt(T);
    const R num = mu0 * (T * sq) * (R(1) + S);
    const R mu = num / (T + S);
    const R div = g[0][0] + g[1][1] + g[2][2];
    const R txx = R(2) * mu * g[0][0] - R(2.0 / 3.0) * mu * div;
    const R tyy = R(2) * mu * g[1][1] - R(2.0 / 3.0) * mu * div;
    const R tzz = R(2) * mu * g[2][2] - R(2.0 / 3.0) * mu * div;
    const R txy = mu * (g[0][1] + g[1][0]), txz = mu * (g[0][2] + g[2][0]), tyz = mu * (g[1][2] + g[2][1]);
    // energy components
    R txxb = Vb[0] + x[0] * Vb[6], tyyb = Vb[1] + x[1] * Vb[7], tzzb = Vb[2] + x[2] * Vb[8];
    R txyb = Vb[3] + x[1] * Vb[6] + x[0] * Vb[7];
    R txzb = Vb[4] + x[2] * Vb[6] + x[0] * Vb[8];
    R tyzb = Vb[5] + x[2] * Vb[7] + x[1] * Vb[8];
    xb[0] += Vb[6] * txx + Vb[7] * txy + Vb[8] * txz;
    xb[1] += Vb[6] * txy + Vb[7] * tyy + Vb[8] * tyz;
    xb[2] += Vb[6] * txz + Vb[7] * tyz + Vb[8] * tzz;
    R kqb = Vb[6] * g[3][0] + Vb[7] * g[3][1] + Vb[8] * g[3][2];
    gb[3][0] += Vb[6] * mu * cpr; gb[3][1] += Vb[7] * mu * cpr; gb[3][2] += Vb[8] * mu * cpr;
    R mub = kqb * cpr;
    // stresses
    mub += txxb * (R(2) * g[0][0] - R(2.0 / 3.0) * div) + tyyb * (R(2) * g[1][1] - R(2.0 / 3.0) * div) +
           tzzb * (R(2) * g[2][2] - R(2.0 / 3.0) * div) + txyb * (g[0][1] + g[1][0]) +
           txzb * (g[0][2] + g[2][0]) + tyzb * (g[1][2] + g[2][1]);
    R divb = R(-2.0 / 3.0) * mu * (txxb + tyyb + tzzb);
    gb[0][0] += R(2) * mu * txxb + divb; gb[1][1] += R(2) * mu * tyyb + divb; gb[2][2] += R(2) * mu * tzzb + divb;
    gb[0][1] += mu * txyb; gb[1][0] += mu * txyb;
    gb[0][2] += mu * txzb; gb[2][0] += mu * txzb;
    gb[1][2] += mu * tyzb; gb[2][1] += mu * tyzb;
    // mu = mu0 T^1.5 (1+S)/(T+S)
    const R dmu = mu0 * (R(1) + S) * (R(1.5) * sq * (T + S) - T * sq) / ((T + S) * (T + S));
    xb[3] += mub * dmu;
    (void)num;
}

}  // namespace adj
}  // namespace ns3d
