// schemes.cuh -- WCNS interpolation and approximate Riemann solvers on the
// device, templated on the arithmetic type (double: plain path, float: mixed
// path) and on the sweep direction, so the face normal is a compile-time unit
// vector and the tangential terms vanish instead of being multiplied by zero.
//
// The formulas are those of interpolation.cpp and InviscousFlux.cpp; where a
// form below is rearranged (common-denominator WENO weights, the Roe
// dissipation through the eigen-projectors of the two acoustic waves) the
// result is mathematically identical and differs only in rounding.
#pragma once

#include <cstring>

#include "common.cuh"

#ifndef NS3D_HD
#define NS3D_HD __host__ __device__ __forceinline__
#endif

namespace ns3d {

enum { I_WENO5 = 0, I_ZERO = 1, I_MDCD_LINEAR = 2, I_MDCD_HYBRID = 3 };
enum { R_ROE = 0, R_RUSANOV = 1, R_HLLC = 2, R_HLL = 3, R_HLLC_P = 4, R_AUSM = 5, R_STEGER_WARMING = 6 };
constexpr int RUNTIME = -1;

template <typename R>
struct SchemeParams {
    R gamma;
    R lin[6];           // MDCD linear coefficients (interpolation.cpp:130-132)
    R hd[4];            // MDCD-WENO linear weights d0..d3 (interpolation.cpp:179-182)
    int interp, riemann, char_recon;  // runtime selection for the generic kernel
};

// ------------------------------------------------------------ interpolation

// weno5_interpolate, interpolation.cpp:86-115: WCNS-E5 midpoint value from
// the 5 left-biased points f0..f4, weights 1/16, 5/8, 5/16, eps = 1e-6.
// The three divisions of the normalised weights are folded into one.
template <typename R>
NS3D_HD R weno5(R f0, R f1, R f2, R f3, R f4) {
    const R eps = R(1e-6);
    const R c13 = R(13.0 / 12.0);
    R t, u;
    t = f0 - R(2) * f1 + f2; u = f0 - R(4) * f1 + R(3) * f2;
    R b0 = c13 * t * t + R(0.25) * u * u;
    t = f1 - R(2) * f2 + f3; u = f1 - f3;
    R b1 = c13 * t * t + R(0.25) * u * u;
    t = f2 - R(2) * f3 + f4; u = R(3) * f2 - R(4) * f3 + f4;
    R b2 = c13 * t * t + R(0.25) * u * u;
    R s0 = (eps + b0) * (eps + b0), s1 = (eps + b1) * (eps + b1), s2 = (eps + b2) * (eps + b2);
    // alpha_k = d_k / s_k; multiply every alpha by s0*s1*s2
    R a0 = R(1.0 / 16.0) * s1 * s2;
    R a1 = R(5.0 / 8.0) * s0 * s2;
    R a2 = R(5.0 / 16.0) * s0 * s1;
    R p0 = R(3) * f0 - R(10) * f1 + R(15) * f2;
    R p1 = -f1 + R(6) * f2 + R(3) * f3;
    R p2 = R(3) * f2 + R(6) * f3 - f4;
    return (a0 * p0 + a1 * p1 + a2 * p2) / (R(8) * (a0 + a1 + a2));
}

// mdcd_linear_interpolate, interpolation.cpp:118-133.
template <typename R>
NS3D_HD R mdcd_linear(const R *c, R f0, R f1, R f2, R f3, R f4, R f5) {
    return c[0] * f0 + c[1] * f1 + c[2] * f2 + c[3] * f3 + c[4] * f4 + c[5] * f5;
}

// beta3 of mdcd_hybrid_interpolate (interpolation.cpp:193-200).  The
// reference's expanded quadratic form is kept for the FP64 path.  Its row
// sums are (20,0,0,0,0,0), so beta3(f) = Q(f - f0) + f0^2/6048 exactly; the
// FP32 path evaluates that split form, which avoids the cancellation of the
// expanded form (terms ~1e3 f^2 summing to ~1e-4 f^2).
NS3D_HD double mdcd_beta3(double f0, double f1, double f2, double f3, double f4,
                                             double f5) {
    return (271799.0 * (f0 * f0) +
            f0 * (-2380800.0 * f1 + 4086352.0 * f2 - 3462252.0 * f3 + 1458762.0 * f4 - 245620.0 * f5) +
            f1 * (5653317.0 * f1 - 20427884.0 * f2 + 17905032.0 * f3 - 7727988.0 * f4 + 1325006.0 * f5) +
            f2 * (19510972.0 * f2 - 35817664.0 * f3 + 15929912.0 * f4 - 2792660.0 * f5) +
            f3 * (17195652.0 * f3 - 15880404.0 * f4 + 2863984.0 * f5) +
            f4 * (3824847.0 * f4 - 1429976.0 * f5) + 139633.0 * (f5 * f5)) / 120960.0;
}
NS3D_HD float mdcd_beta3(float f0, float f1, float f2, float f3, float f4, float f5) {
    const float d1 = f1 - f0, d2 = f2 - f0, d3 = f3 - f0, d4 = f4 - f0, d5 = f5 - f0;
    float q = d1 * (5653317.f * d1 - 20427884.f * d2 + 17905032.f * d3 - 7727988.f * d4 + 1325006.f * d5) +
              d2 * (19510972.f * d2 - 35817664.f * d3 + 15929912.f * d4 - 2792660.f * d5) +
              d3 * (17195652.f * d3 - 15880404.f * d4 + 2863984.f * d5) +
              d4 * (3824847.f * d4 - 1429976.f * d5) + 139633.f * (d5 * d5);
    return q * (1.f / 120960.f) + f0 * f0 * (1.f / 6048.f);
}

// mdcd_hybrid_interpolate, interpolation.cpp:135-209, split into its
// detector and its WENO branch.
//
// Detector: with a_j = |f_j - f_{j-1}| + |f_j - 2 f_{j-1} + f_{j-2}| and
// b_j = |f_j - f_{j+1}| + |f_j - 2 f_{j+1} + f_{j+2}| at the two central
// points j = 2, 3 of the stencil, the linear scheme is used when
// min(sai(a_2, b_2), sai(a_3, b_3)) > 0.4 with sai(a, b) = (2ab + eps)/(a^2 +
// b^2 + eps), evaluated as cross-multiplied comparisons (the denominators are
// positive).  sai is symmetric in (a, b), and the reversed stencil of the
// right state swaps a_j and b_j of the same two points with the same
// operation order, so both states of a face take the same decision:
// smooth(cell i) && smooth(cell i+1) for the face i+1/2.
//
// The detector is the one discontinuous decision of the scheme, so the FP64
// build takes the reference's decision exactly: the cross-multiplied test
// (whose products the compiler may fuse) decides every case whose two sides
// lie at least two units apart in their high 32-bit words (more than 2^-21
// relative, far beyond the test's few-ulp rounding; an integer test, so the
// FP64 pipe does no extra work), and the rest are decided by the reference's
// own quotient, term by term with unfused IEEE operations (mdcd_sai_ref).  a
// and b themselves round as in the reference: 2 f is exact, so a fused
// f0 - 2 fm1 gives the same bits.
NS3D_HD double mdcd_sai_ref(double a, double b) {
    const double eps = 0.9 * 0.4 / (1.0 - 0.9 * 0.4) * 1e-4;
#ifdef __CUDA_ARCH__
    const double num = __dadd_rn(__dmul_rn(__dmul_rn(2.0, a), b), eps);
    const double den = __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), eps);
    return __ddiv_rn(num, den);
#else
    volatile double aa = a * a, bb = b * b, ab2 = 2.0 * a * b;
    return (ab2 + eps) / (aa + bb + eps);
#endif
}

// high 32 bits of an FP64 value (sign, exponent, top 20 mantissa bits)
NS3D_HD int f64_hi_word(double x) {
#ifdef __CUDA_ARCH__
    return __double2hiint(x);
#else
    unsigned long long u;
    std::memcpy(&u, &x, sizeof u);
    return (int)(u >> 32);
#endif
}

template <typename R>
NS3D_HD bool mdcd_smooth(R fm2, R fm1, R f0, R fp1, R fp2) {
    const R eps = R(0.9 * 0.4 / (1.0 - 0.9 * 0.4) * 1e-4);
    R a = fabs(f0 - fm1) + fabs(f0 - R(2) * fm1 + fm2);
    R b = fabs(f0 - fp1) + fabs(f0 - R(2) * fp1 + fp2);
    const R lhs = R(2) * a * b + eps, rhs = R(0.4) * (a * a + b * b + eps);
    if constexpr (sizeof(R) == 8) {
        // lhs, rhs > 0, so their high words order as the values do
        if ((unsigned)(f64_hi_word(lhs) - f64_hi_word(rhs) + 1) <= 2u) return mdcd_sai_ref(a, b) > 0.4;
    }
    return lhs > rhs;
}

// The cross-multiplied decision alone, without a branch: near is set (FP64)
// where the two sides are too close for it, and the caller then takes
// mdcd_smooth's decision instead (once for all the detectors of a cell, so
// the common path has no branch per detector).  Wherever near stays clear the
// value equals mdcd_smooth's.
template <typename R>
NS3D_HD bool mdcd_smooth_fast(R fm2, R fm1, R f0, R fp1, R fp2, bool &near) {
    const R eps = R(0.9 * 0.4 / (1.0 - 0.9 * 0.4) * 1e-4);
    R a = fabs(f0 - fm1) + fabs(f0 - R(2) * fm1 + fm2);
    R b = fabs(f0 - fp1) + fabs(f0 - R(2) * fp1 + fp2);
    const R lhs = R(2) * a * b + eps, rhs = R(0.4) * (a * a + b * b + eps);
    if constexpr (sizeof(R) == 8) near |= (unsigned)(f64_hi_word(lhs) - f64_hi_word(rhs) + 1) <= 2u;
    return lhs > rhs;
}

// The non-linear branch: 4-stencil WENO with weights d_k (20 + tau6/(beta_k +
// 1e-40))^2 (interpolation.cpp:170-208).
template <typename R>
NS3D_HD R mdcd_weno_branch(const R *hd, R f0, R f1, R f2, R f3, R f4, R f5) {
    const R eps_small = sizeof(R) == 8 ? R(1e-40) : R(1e-40f);
    const R c13 = R(13.0 / 12.0);
    R t, u;
    t = f0 - R(2) * f1 + f2; u = f0 - R(4) * f1 + R(3) * f2;
    R be0 = c13 * (t * t) + R(0.25) * (u * u);
    t = f1 - R(2) * f2 + f3; u = f1 - f3;
    R be1 = c13 * (t * t) + R(0.25) * (u * u);
    t = f2 - R(2) * f3 + f4; u = R(3) * f2 - R(4) * f3 + f4;
    R be2 = c13 * (t * t) + R(0.25) * (u * u);
    R be3 = mdcd_beta3(f0, f1, f2, f3, f4, f5);
    R q0 = R(3) * f0 - R(10) * f1 + R(15) * f2;
    R q1 = -f1 + R(6) * f2 + R(3) * f3;
    R q2 = R(3) * f2 + R(6) * f3 - f4;
    R q3 = R(15) * f3 - R(10) * f4 + R(3) * f5;
    // The weights span far more than the FP32 range: FP32 inputs quantise a
    // smooth stencil to beta == 0 exactly, and (tau6 * 1e40)^2 overflows to
    // inf (inf/inf = NaN).  So the FP32 build forms the weights and the
    // normalisation in FP64, like the reference; this branch is the rare one
    // (most faces take the linear scheme).
    using Wt = double;
    Wt tau6 = fabs((Wt)be3 - ((Wt)be0 + Wt(4) * (Wt)be1 + (Wt)be2) / Wt(6));
    const Wt es = sizeof(R) == 8 ? (Wt)eps_small : Wt(1e-40);
    Wt g0 = Wt(20) + tau6 / ((Wt)be0 + es);
    Wt g1 = Wt(20) + tau6 / ((Wt)be1 + es);
    Wt g2 = Wt(20) + tau6 / ((Wt)be2 + es);
    Wt g3 = Wt(20) + tau6 / ((Wt)be3 + es);
    Wt al0 = (Wt)hd[0] * (g0 * g0), al1 = (Wt)hd[1] * (g1 * g1), al2 = (Wt)hd[2] * (g2 * g2),
       al3 = (Wt)hd[3] * (g3 * g3);
    return (R)((al0 * (Wt)q0 + al1 * (Wt)q1 + al2 * (Wt)q2 + al3 * (Wt)q3) / (Wt(8) * (al0 + al1 + al2 + al3)));
}

template <typename R>
NS3D_HD R mdcd_hybrid(const R *lin, const R *hd, R f0, R f1, R f2, R f3, R f4, R f5) {
    if (mdcd_smooth(f0, f1, f2, f3, f4) && mdcd_smooth(f1, f2, f3, f4, f5))
        return mdcd_linear(lin, f0, f1, f2, f3, f4, f5);
    return mdcd_weno_branch(hd, f0, f1, f2, f3, f4, f5);
}

// interpolate_select, interpolation.cpp:13-77, for the left state (flag +1,
// stencil f[0..5]) or the right state (flag -1, reversed stencil).
template <typename R, int INTERP>
NS3D_HD R interp_side(const SchemeParams<R> &sp, const R *f, bool right) {
    const int it = INTERP == RUNTIME ? sp.interp : INTERP;
    R g0, g1, g2, g3, g4, g5;
    if (!right) { g0 = f[0]; g1 = f[1]; g2 = f[2]; g3 = f[3]; g4 = f[4]; g5 = f[5]; }
    else { g0 = f[5]; g1 = f[4]; g2 = f[3]; g3 = f[2]; g4 = f[1]; g5 = f[0]; }
    if (it == I_WENO5) return weno5(g0, g1, g2, g3, g4);
    if (it == I_MDCD_LINEAR) return mdcd_linear(sp.lin, g0, g1, g2, g3, g4, g5);
    return mdcd_hybrid(sp.lin, sp.hd, g0, g1, g2, g3, g4, g5);
}

// Left and right states of one conserved variable at face i+1/2 from the
// stencil f[0..5] = cells i-2 .. i+3 (component-wise interpolation).  For
// MDCD_HYBRID the detector is evaluated once for both sides (see
// mdcd_smooth); every value equals interp_side's.
template <typename R, int INTERP>
NS3D_HD void face_pair(const SchemeParams<R> &sp, const R *f, R &L, R &Rr) {
    const int it = INTERP == RUNTIME ? sp.interp : INTERP;
    if (it == I_MDCD_HYBRID) {
        if (mdcd_smooth(f[0], f[1], f[2], f[3], f[4]) && mdcd_smooth(f[1], f[2], f[3], f[4], f[5])) {
            L = mdcd_linear(sp.lin, f[0], f[1], f[2], f[3], f[4], f[5]);
            Rr = mdcd_linear(sp.lin, f[5], f[4], f[3], f[2], f[1], f[0]);
        } else {
            L = mdcd_weno_branch(sp.hd, f[0], f[1], f[2], f[3], f[4], f[5]);
            Rr = mdcd_weno_branch(sp.hd, f[5], f[4], f[3], f[2], f[1], f[0]);
        }
        return;
    }
    L = interp_side<R, INTERP>(sp, f, false);
    Rr = interp_side<R, INTERP>(sp, f, true);
}

// ------------------------------------------------------------ Riemann solvers

template <int DIR, typename R>
struct Side {
    R r, ir, u, v, w, E, p, un;
    NS3D_HD void load(const R *U, R g) {
        r = U[0]; ir = R(1) / r;
        u = U[1] * ir; v = U[2] * ir; w = U[3] * ir; E = U[4];
        p = (E - R(0.5) * r * (u * u + v * v + w * w)) * (g - R(1));
        un = DIR == 0 ? u : (DIR == 1 ? v : w);
    }
    // physical flux of the state along the face normal (InviscousFlux.cpp:333-346)
    NS3D_HD void flux(R *F) const {
        R m = r * un;
        F[0] = m;
        F[1] = m * u + (DIR == 0 ? p : R(0));
        F[2] = m * v + (DIR == 1 ? p : R(0));
        F[3] = m * w + (DIR == 2 ? p : R(0));
        F[4] = (E + p) * un;
    }
};

// Roe_Riemann_solver, InviscousFlux.cpp:313-382.  The eigen-system is the
// Blazek form of build_eigen_matrices (:888-987) with L R = I, so the three
// degenerate waves (eigenvalue V) contribute |V|(dU - a0 R0 - a4 R4): only
// the two acoustic projections are formed.  Harten entropy fix with
// delta = 0.1 max|lambda| = 0.1 (|V| + c) as the reference.
template <int DIR, typename R>
NS3D_HD void roe_flux(const R *UL, const R *UR, R g, R *F) {
    Side<DIR, R> L, Rt;
    L.load(UL, g); Rt.load(UR, g);
    R FL[5], FR[5];
    L.flux(FL); Rt.flux(FR);
    const R gm1 = g - R(1);
    const R kfac = g / gm1;
    R HL = R(0.5) * (L.u * L.u + L.v * L.v + L.w * L.w) + kfac * L.p * L.ir;
    R HR = R(0.5) * (Rt.u * Rt.u + Rt.v * Rt.v + Rt.w * Rt.w) + kfac * Rt.p * Rt.ir;
    R sL = sqrt(L.r), sR = sqrt(Rt.r);
    R den = R(1) / (sL + sR);
    R ub = (sL * L.u + sR * Rt.u) * den;
    R vb = (sL * L.v + sR * Rt.v) * den;
    R wb = (sL * L.w + sR * Rt.w) * den;
    R Hb = (sL * HL + sR * HR) * den;
    R q2 = ub * ub + vb * vb + wb * wb;
    R c2 = gm1 * (Hb - R(0.5) * q2);
    R c = sqrt(c2);
    R V = DIR == 0 ? ub : (DIR == 1 ? vb : wb);
    R phi = R(0.5) * gm1 * q2;
    R dU[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) dU[n] = UR[n] - UL[n];
    const R dUn = dU[1 + DIR];
    R t = phi * dU[0] + gm1 * (dU[4] - ub * dU[1] - vb * dU[2] - wb * dU[3]);
    R s = c * (V * dU[0] - dUn);
    R i2c2 = R(1) / (R(2) * c2);
    R A0 = (t + s) * i2c2;   // acoustic wave V - c: alpha0 * a3
    R A4 = (t - s) * i2c2;   // acoustic wave V + c
    R l0 = fabs(V - c), lv = fabs(V), l4 = fabs(V + c);
    R delta = R(0.1) * (lv + c);
    // (l^2 + delta^2) / (2 delta) below delta, through one reciprocal and
    // selects (no divergent division per eigenvalue)
    const R i2d = R(1) / (R(2) * delta), d2 = delta * delta;
    l0 = l0 < delta ? (l0 * l0 + d2) * i2d : l0;
    lv = lv < delta ? (lv * lv + d2) * i2d : lv;
    l4 = l4 < delta ? (l4 * l4 + d2) * i2d : l4;
    R k0 = (l0 - lv) * A0, k4 = (l4 - lv) * A4;
    // R0 = (1, u-nc, v-nc, w-nc, H-cV), R4 = (1, u+nc, v+nc, w+nc, H+cV)
    R cx = DIR == 0 ? c : R(0), cy = DIR == 1 ? c : R(0), cz = DIR == 2 ? c : R(0);
    R D0 = lv * dU[0] + k0 + k4;
    R D1 = lv * dU[1] + k0 * (ub - cx) + k4 * (ub + cx);
    R D2 = lv * dU[2] + k0 * (vb - cy) + k4 * (vb + cy);
    R D3 = lv * dU[3] + k0 * (wb - cz) + k4 * (wb + cz);
    R D4 = lv * dU[4] + k0 * (Hb - c * V) + k4 * (Hb + c * V);
    F[0] = R(0.5) * (FL[0] + FR[0]) - R(0.5) * D0;
    F[1] = R(0.5) * (FL[1] + FR[1]) - R(0.5) * D1;
    F[2] = R(0.5) * (FL[2] + FR[2]) - R(0.5) * D2;
    F[3] = R(0.5) * (FL[3] + FR[3]) - R(0.5) * D3;
    F[4] = R(0.5) * (FL[4] + FR[4]) - R(0.5) * D4;
}

// Rusanov_Riemann_solver, InviscousFlux.cpp:270-311.
template <int DIR, typename R>
NS3D_HD void rusanov_flux(const R *UL, const R *UR, R g, R *F) {
    Side<DIR, R> L, Rt;
    L.load(UL, g); Rt.load(UR, g);
    R FL[5], FR[5];
    L.flux(FL); Rt.flux(FR);
    R aL = sqrt(g * L.p * L.ir), aR = sqrt(g * Rt.p * Rt.ir);
    R smax = fmax(fabs(L.un) + aL, fabs(Rt.un) + aR);
#pragma unroll
    for (int n = 0; n < 5; ++n) F[n] = R(0.5) * (FL[n] + FR[n]) - R(0.5) * smax * (UR[n] - UL[n]);
}

// HLL_Riemann_solver, InviscousFlux.cpp:384-447 (Davis wave speeds).
template <int DIR, typename R>
NS3D_HD void hll_flux(const R *UL, const R *UR, R g, R *F) {
    Side<DIR, R> L, Rt;
    L.load(UL, g); Rt.load(UR, g);
    R FL[5], FR[5];
    L.flux(FL); Rt.flux(FR);
    R aL = sqrt(g * L.p * L.ir), aR = sqrt(g * Rt.p * Rt.ir);
    R SL = fmin(L.un - aL, Rt.un - aR);
    R SR = fmax(L.un + aL, Rt.un + aR);
    if (SL >= R(0)) {
#pragma unroll
        for (int n = 0; n < 5; ++n) F[n] = FL[n];
    } else if (SR <= R(0)) {
#pragma unroll
        for (int n = 0; n < 5; ++n) F[n] = FR[n];
    } else {
        R id = R(1) / (SR - SL);
#pragma unroll
        for (int n = 0; n < 5; ++n) F[n] = (SR * FL[n] - SL * FR[n] + SL * SR * (UR[n] - UL[n])) * id;
    }
}

// HLLC star-region flux, InviscousFlux.cpp:537-591 (and :663-715 for HLLC_p).
template <int DIR, typename R>
NS3D_HD void hllc_star(const Side<DIR, R> &S, const R *U, const R *Fs, R Sk, R SM,
                                          R *F) {
    R dk = Sk - S.un;
    R rs = S.r * dk / (Sk - SM);
    R us = DIR == 0 ? SM : S.u, vs = DIR == 1 ? SM : S.v, ws = DIR == 2 ? SM : S.w;
    R Es = S.E * S.ir + (SM - S.un) * (SM + S.p / (S.r * dk));
    F[0] = Fs[0] + Sk * (rs - U[0]);
    F[1] = Fs[1] + Sk * (rs * us - U[1]);
    F[2] = Fs[2] + Sk * (rs * vs - U[2]);
    F[3] = Fs[3] + Sk * (rs * ws - U[3]);
    F[4] = Fs[4] + Sk * (rs * Es - U[4]);
}

// HLLC_Riemann_solver, InviscousFlux.cpp:449-592: Davis S_L/S_R, Batten S_M
// (Roe-averaged normal velocity when the S_M denominator is below 1e-12).
template <int DIR, typename R>
NS3D_HD void hllc_flux(const R *UL, const R *UR, R g, R *F) {
    Side<DIR, R> L, Rt;
    L.load(UL, g); Rt.load(UR, g);
    R aL = sqrt(g * L.p * L.ir), aR = sqrt(g * Rt.p * Rt.ir);
    R SL = fmin(L.un - aL, Rt.un - aR);
    R SR = fmax(L.un + aL, Rt.un + aR);
    if (SL >= R(0)) { L.flux(F); return; }
    if (SR <= R(0)) { Rt.flux(F); return; }
    R num = Rt.r * Rt.un * (SR - Rt.un) - L.r * L.un * (SL - L.un) + L.p - Rt.p;
    R den = Rt.r * (SR - Rt.un) - L.r * (SL - L.un);
    R SM;
    if (fabs(den) > R(1e-12)) {
        SM = num / den;
    } else {
        R sL = sqrt(L.r), sR = sqrt(Rt.r);
        SM = (sL * L.un + sR * Rt.un) / (sL + sR);
    }
    // the star state of the upwind side: selected, not branched, so faces of
    // one warp with different signs of S_M do not diverge
    const bool left = SM >= R(0);
    Side<DIR, R> S;
    S.r = left ? L.r : Rt.r; S.ir = left ? L.ir : Rt.ir;
    S.u = left ? L.u : Rt.u; S.v = left ? L.v : Rt.v; S.w = left ? L.w : Rt.w;
    S.E = left ? L.E : Rt.E; S.p = left ? L.p : Rt.p; S.un = left ? L.un : Rt.un;
    R Us[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) Us[n] = left ? UL[n] : UR[n];
    R Fs[5];
    S.flux(Fs);
    hllc_star<DIR, R>(S, Us, Fs, left ? SL : SR, SM, F);
}

// HLLC_p_Riemann_solver, InviscousFlux.cpp:594-717: PVRS p*, Toro speeds.
template <int DIR, typename R>
NS3D_HD void hllc_p_flux(const R *UL, const R *UR, R g, R *F) {
    Side<DIR, R> L, Rt;
    L.load(UL, g); Rt.load(UR, g);
    R aL = sqrt(g * L.p * L.ir), aR = sqrt(g * Rt.p * Rt.ir);
    R ps = R(0.5) * (L.p + Rt.p) - R(0.125) * (Rt.un - L.un) * (L.r + Rt.r) * (aL + aR);
    ps = fmax(R(0), ps);
    const R c1 = (g + R(1)) / (R(2) * g), c2 = (g - R(1)) / (R(2) * g);
    R SL = ps <= L.p ? L.un - aL : L.un - aL * sqrt(c1 * ps / L.p + c2);
    R SR = ps <= Rt.p ? Rt.un + aR : Rt.un + aR * sqrt(c1 * ps / Rt.p + c2);
    if (SL >= R(0)) { L.flux(F); return; }
    if (SR <= R(0)) { Rt.flux(F); return; }
    R SM = (Rt.p - L.p + L.r * L.un * (SL - L.un) - Rt.r * Rt.un * (SR - Rt.un)) /
           (L.r * (SL - L.un) - Rt.r * (SR - Rt.un));
    R Fs[5];
    if (SM >= R(0)) { L.flux(Fs); hllc_star<DIR, R>(L, UL, Fs, SL, SM, F); }
    else { Rt.flux(Fs); hllc_star<DIR, R>(Rt, UR, Fs, SR, SM, F); }
}

// AUSM_Riemann_solver, InviscousFlux.cpp:719-846 (AUSM+-up style, Kp = 0.25,
// Ku = 0.75, pressure clamped at 1e-12; the pressure diffusion uses the
// x-velocity difference u_R - u_L in every direction, as the reference).
template <int DIR, typename R>
NS3D_HD void ausm_flux(const R *UL, const R *UR, R g, R *F) {
    const R Kp = R(0.25), Ku = R(0.75);
    Side<DIR, R> L, Rt;
    L.load(UL, g); Rt.load(UR, g);
    R pL = fmax(L.p, R(1e-12)), pR = fmax(Rt.p, R(1e-12));
    R aL = sqrt(g * pL * L.ir), aR = sqrt(g * pR * Rt.ir);
    R HL = (L.E + pL) * L.ir, HR = (Rt.E + pR) * Rt.ir;
    R ab = R(0.5) * (aL + aR), rb = R(0.5) * (L.r + Rt.r);
    R iab = R(1) / ab;
    R ML = L.un * iab, MR = Rt.un * iab;
    R Mb2 = (L.un * L.un + Rt.un * Rt.un) * (R(0.5) * iab * iab);
    R Mo2 = fmin(R(1), fmax(Mb2, R(0.5)));
    R fa = Mo2 * (R(2) - Mo2);
    R Mp = fabs(ML) >= R(1) ? R(0.5) * (ML + fabs(ML)) : R(0.25) * (ML + R(1)) * (ML + R(1));
    R Mm = fabs(MR) >= R(1) ? R(0.5) * (MR - fabs(MR)) : R(-0.25) * (MR - R(1)) * (MR - R(1));
    R Mh = Mp + Mm - Kp / fa * fmax(R(1) - Mb2, R(0)) * ((pR - pL) / (rb * ab * ab));
    R md = ab * Mh * (Mh >= R(0) ? L.r : Rt.r);
    R pp = fabs(ML) >= R(1) ? R(0.5) * (R(1) + (ML > R(0) ? R(1) : R(-1)))
                            : R(0.25) * (ML + R(1)) * (ML + R(1)) * (R(2) - ML);
    R pm = fabs(MR) >= R(1) ? R(0.5) * (R(1) - (MR > R(0) ? R(1) : R(-1)))
                            : R(0.25) * (MR - R(1)) * (MR - R(1)) * (R(2) + MR);
    R ph = pp * pL + pm * pR - Ku * pm * pp * (L.r + Rt.r) * fa * (Rt.u - L.u) * ab;
    bool up = md >= R(0);
    R uf = up ? L.u : Rt.u, vf = up ? L.v : Rt.v, wf = up ? L.w : Rt.w, Hf = up ? HL : HR;
    F[0] = md;
    F[1] = md * uf + (DIR == 0 ? ph : R(0));
    F[2] = md * vf + (DIR == 1 ? ph : R(0));
    F[3] = md * wf + (DIR == 2 ? ph : R(0));
    F[4] = md * Hf;
}

// Steger-Warming flux-vector splitting (J. L. Steger, R. F. Warming, J.
// Comput. Phys. 40 (1981) 263-293) as a face flux: F = F+(U_L) + F-(U_R).
// With the eigenvalues l1 = u_n, l2 = u_n + c, l3 = u_n - c of the normal
// velocity u_n and their positive / negative parts l+- = (l +- |l|)/2,
//   F+- = rho/(2 gamma) [ 2(g-1) l1 + l2 + l3,
//                         2(g-1) l1 V + l2 (V + c n) + l3 (V - c n),
//                         (g-1) l1 |V|^2 + l2 ((u_n + c)^2 + |V_t|^2)/2 + l3 ((u_n - c)^2 + |V_t|^2)/2
//                           + (3 - g)(l2 + l3) c^2 / (2 (g-1)) ]
// (all l's taken +- alike), with V_t the tangential velocity.  F+ + F- is
// the physical flux.  The reference declares this splitting
// (field_structures.h:113-119, initialization.cpp:80-84) but implements no
// formula, so this one has no reference output to match.
template <int DIR, typename R>
NS3D_HD void sw_split(const R *U, R g, R sgn, R *F) {
    Side<DIR, R> S;
    S.load(U, g);
    const R c2 = g * S.p * S.ir, c = sqrt(c2);
    auto part = [&](R l) { return R(0.5) * (l + sgn * fabs(l)); };
    const R l1 = part(S.un), l2 = part(S.un + c), l3 = part(S.un - c);
    const R k = S.r / (R(2) * g);
    const R gm1 = g - R(1);
    const R vt2 = S.u * S.u + S.v * S.v + S.w * S.w - S.un * S.un;
    const R up = S.un + c, um = S.un - c;
    const R m = R(2) * gm1 * l1 + l2 + l3;
    F[0] = k * m;
    F[1] = k * (m * S.u + (DIR == 0 ? c * (l2 - l3) : R(0)));
    F[2] = k * (m * S.v + (DIR == 1 ? c * (l2 - l3) : R(0)));
    F[3] = k * (m * S.w + (DIR == 2 ? c * (l2 - l3) : R(0)));
    F[4] = k * (gm1 * l1 * (S.un * S.un + vt2) + R(0.5) * l2 * (up * up + vt2) + R(0.5) * l3 * (um * um + vt2) +
                (R(3) - g) * (l2 + l3) * c2 / (R(2) * gm1));
}

template <int DIR, typename R>
NS3D_HD void steger_warming_flux(const R *UL, const R *UR, R g, R *F) {
    R Fp[5], Fm[5];
    sw_split<DIR, R>(UL, g, R(1), Fp);
    sw_split<DIR, R>(UR, g, R(-1), Fm);
#pragma unroll
    for (int n = 0; n < 5; ++n) F[n] = Fp[n] + Fm[n];
}

template <int DIR, typename R, int RS>
NS3D_HD void riemann(const SchemeParams<R> &sp, const R *UL, const R *UR, R *F) {
    const int rs = RS == RUNTIME ? sp.riemann : RS;
    const R g = sp.gamma;
    if (RS == R_ROE || (RS == RUNTIME && rs == R_ROE)) roe_flux<DIR, R>(UL, UR, g, F);
    else if (RS == R_HLLC || (RS == RUNTIME && rs == R_HLLC)) hllc_flux<DIR, R>(UL, UR, g, F);
    else if (RS == R_HLL || (RS == RUNTIME && rs == R_HLL)) hll_flux<DIR, R>(UL, UR, g, F);
    else if (RS == R_HLLC_P || (RS == RUNTIME && rs == R_HLLC_P)) hllc_p_flux<DIR, R>(UL, UR, g, F);
    else if (RS == R_RUSANOV || (RS == RUNTIME && rs == R_RUSANOV)) rusanov_flux<DIR, R>(UL, UR, g, F);
    else if (RS == R_STEGER_WARMING || (RS == RUNTIME && rs == R_STEGER_WARMING))
        steger_warming_flux<DIR, R>(UL, UR, g, F);
    else ausm_flux<DIR, R>(UL, UR, g, F);
}

// ------------------------------------------------------- characteristic basis

// build_eigen_matrices for the Roe average of a cell state with itself, as
// WCNS_Riemann_InviscidFlux does for characteristic interpolation
// (InviscousFlux.cpp:166-231 with :849-987).  w = primitive (rho,u,v,w,p).
template <int DIR, typename R>
NS3D_HD void cell_eigen(const R *w, R g, R Lm[5][5], R Rm[5][5]) {
    const R nx = DIR == 0 ? R(1) : R(0), ny = DIR == 1 ? R(1) : R(0), nz = DIR == 2 ? R(1) : R(0);
    const R gm1 = g - R(1);
    R r = w[0], u = w[1], v = w[2], ww = w[3], p = w[4];
    R E = r * (R(0.5) * (u * u + v * v + ww * ww) + p / (gm1 * r));
    R sq = sqrt(r);
    R rb = sq * sq;
    R den = R(1) / (sq + sq);
    R ub = (sq * u + sq * u) * den, vb = (sq * v + sq * v) * den, wb = (sq * ww + sq * ww) * den;
    R H = (E + p) / r;
    R Hb = (sq * H + sq * H) * den;
    R c = sqrt(gm1 * (Hb - R(0.5) * (ub * ub + vb * vb + wb * wb)));
    R V = nx * ub + ny * vb + nz * wb;
    R phi = R(0.5) * gm1 * (ub * ub + vb * vb + wb * wb);
    R a1 = gm1;
    R a2 = R(1) / (sqrt(R(2)) * rb * c);
    R a3 = rb / (sqrt(R(2)) * c);
    R a4 = (phi + c * c) / gm1;
    R ic2 = R(1) / (c * c), irb = R(1) / rb;
    R a5 = R(1) - phi * ic2;
    R a6 = phi / gm1;
    Lm[0][0] = a2 * (phi + c * V); Lm[0][1] = -a2 * (a1 * ub + nx * c); Lm[0][2] = -a2 * (a1 * vb + ny * c);
    Lm[0][3] = -a2 * (a1 * wb + nz * c); Lm[0][4] = a1 * a2;
    Lm[1][0] = nx * a5 - (nz * vb - ny * wb) * irb; Lm[1][1] = nx * a1 * ub * ic2;
    Lm[1][2] = nx * a1 * vb * ic2 + nz * irb; Lm[1][3] = nx * a1 * wb * ic2 - ny * irb; Lm[1][4] = -nx * a1 * ic2;
    Lm[2][0] = nz * a5 - (ny * ub - nx * vb) * irb; Lm[2][1] = nz * a1 * ub * ic2 + ny * irb;
    Lm[2][2] = nz * a1 * vb * ic2 - nx * irb; Lm[2][3] = nz * a1 * wb * ic2; Lm[2][4] = -nz * a1 * ic2;
    Lm[3][0] = ny * a5 - (nx * wb - nz * ub) * irb; Lm[3][1] = ny * a1 * ub * ic2 - nz * irb;
    Lm[3][2] = ny * a1 * vb * ic2; Lm[3][3] = ny * a1 * wb * ic2 + nx * irb; Lm[3][4] = -ny * a1 * ic2;
    Lm[4][0] = a2 * (phi - c * V); Lm[4][1] = -a2 * (a1 * ub - nx * c); Lm[4][2] = -a2 * (a1 * vb - ny * c);
    Lm[4][3] = -a2 * (a1 * wb - nz * c); Lm[4][4] = a1 * a2;
    Rm[0][0] = a3; Rm[1][0] = a3 * (ub - nx * c); Rm[2][0] = a3 * (vb - ny * c); Rm[3][0] = a3 * (wb - nz * c);
    Rm[4][0] = a3 * (a4 - c * V);
    Rm[0][1] = nx; Rm[1][1] = nx * ub; Rm[2][1] = nx * vb + nz * rb; Rm[3][1] = nx * wb - ny * rb;
    Rm[4][1] = nx * a6 + rb * (nz * vb - ny * wb);
    Rm[0][2] = nz; Rm[1][2] = nz * ub + ny * rb; Rm[2][2] = nz * vb - nx * rb; Rm[3][2] = nz * wb;
    Rm[4][2] = nz * a6 + rb * (ny * ub - nx * vb);
    Rm[0][3] = ny; Rm[1][3] = ny * ub - nz * rb; Rm[2][3] = ny * vb; Rm[3][3] = ny * wb + nx * rb;
    Rm[4][3] = ny * a6 + rb * (nx * wb - nz * ub);
    Rm[0][4] = a3; Rm[1][4] = a3 * (ub + nx * c); Rm[2][4] = a3 * (vb + ny * c); Rm[3][4] = a3 * (wb + nz * c);
    Rm[4][4] = a3 * (a4 + c * V);
}

// WCNS_Riemann_InviscidFlux, InviscousFlux.cpp:146-268.
// U[n][m]: conserved stencil of cells i-2..i+3; wi / wi1: primitives of the
// cells i and i+1 (characteristic bases of the left / right states).
template <int DIR, typename R, int INTERP, int RS, int CHAR>
NS3D_HD void wcns_face(const SchemeParams<R> &sp, const R U[5][6], const R *wi,
                                          const R *wi1, R *F) {
    R UL[5], UR[5];
    const bool ch = CHAR == RUNTIME ? (sp.char_recon != 0) : (CHAR != 0);
    if (!ch) {
#pragma unroll
        for (int n = 0; n < 5; ++n) face_pair<R, INTERP>(sp, U[n], UL[n], UR[n]);
    } else if (CHAR != 0) {
        R Lm[5][5], Rm[5][5], Q[5], Wc[6];
#pragma unroll 1
        for (int side = 0; side < 2; ++side) {
            cell_eigen<DIR, R>(side == 0 ? wi : wi1, sp.gamma, Lm, Rm);
#pragma unroll
            for (int n = 0; n < 5; ++n) {
#pragma unroll
                for (int m = 0; m < 6; ++m) {
                    R s = R(0);
#pragma unroll
                    for (int r = 0; r < 5; ++r) s += Lm[n][r] * U[r][m];
                    Wc[m] = s;
                }
                Q[n] = interp_side<R, INTERP>(sp, Wc, side == 1);
            }
#pragma unroll
            for (int n = 0; n < 5; ++n) {
                R s = R(0);
#pragma unroll
                for (int r = 0; r < 5; ++r) s += Rm[n][r] * Q[r];
                if (side == 0) UL[n] = s; else UR[n] = s;
            }
        }
    }
    riemann<DIR, R, RS>(sp, UL, UR, F);
}

}  // namespace ns3d
