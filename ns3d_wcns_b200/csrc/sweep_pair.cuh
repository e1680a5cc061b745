// sweep_pair.cuh -- the mixed path's FP32 sweep with two lines per thread.
//
// Same algorithm, chunked shared-memory buffers and boundary handling as
// sweep_kernel<DIR, float, ...> (sweep.cuh); the difference is the unit of
// work.  Every thread carries the same face -- and later the same cell -- of
// two neighbouring lines in the two halves of a float2, so that
//   * the MDCD detector and linear interpolation, the 6th-order half-node
//     difference and the viscous derivative run as sm_100's paired FP32
//     instructions (add / mul / fma on f32x2: one instruction for both lines),
//   * every shared-memory access moves a 64-bit word (both lines at once), and
//   * along y and z the two lines are x-neighbours, so the global loads,
//     stores and cp.async copies are 8 bytes (16 for the FP64 state; along z
//     the staging copies take four lines, 16 bytes, past L1).
// HLLC runs paired too (hllc_flux2); the other Riemann solvers and the rare
// WENO branch of the hybrid scheme run per line on the unpacked halves.  The
// arithmetic of each half is the scalar kernel's; only the placement of fused
// multiply-adds differs, so results agree with it to FP32 rounding (the mixed
// path has an accuracy bound, not a bitwise contract).
//
// Requires an even number of lines across the block's bundle (ny along x,
// nx along y and z), so a pair never straddles the end of the domain and the
// 8-byte accesses stay aligned; sweep_select_f32 falls back to the scalar
// kernel otherwise and for characteristic reconstruction.
#pragma once

#include <cstdlib>
#include <cstring>

#include "sweep.cuh"

namespace ns3d {

__device__ __forceinline__ float2 p2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b, rounded once (b * -1 is exact)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

__device__ __forceinline__ void cp_async8(float2 *smem_dst, const float *gsrc) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// 16-byte copy of two float2 (four neighbouring lines), bypassing L1
__device__ __forceinline__ void cp_async16f(float2 *smem_dst, const float *gsrc) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async16(double2 *smem_dst, const double *gsrc) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}

// MDCD linear coefficients, each duplicated into both halves
struct PairConsts {
    float2 lin[6];
};

// sum_k c_k f_k (mdcd_linear) for both lines
__device__ __forceinline__ float2 mdcd_linear2(const float2 *c, float2 f0, float2 f1, float2 f2, float2 f3,
                                               float2 f4, float2 f5) {
    float2 s = mul2(c[0], f0);
    s = fma2(c[1], f1, s);
    s = fma2(c[2], f2, s);
    s = fma2(c[3], f3, s);
    s = fma2(c[4], f4, s);
    return fma2(c[5], f5, s);
}

// mdcd_smooth for both lines (the detector of interpolation.cpp:135-209 at
// one stencil centre): a and b, the sums of two absolute differences, are
// formed per half (absolute values fold into the scalar adds).
__device__ __forceinline__ void mdcd_smooth2(float2 fm2, float2 fm1, float2 f0, float2 fp1, float2 fp2, bool &sa,
                                             bool &sb) {
    const float eps = float(0.9 * 0.4 / (1.0 - 0.9 * 0.4) * 1e-4);
    const float2 dm = sub2(f0, fm1), tm = add2(fma2(p2(-2.f), fm1, f0), fm2);
    const float2 dp = sub2(f0, fp1), tp = add2(fma2(p2(-2.f), fp1, f0), fp2);
    const float2 A = make_float2(fabsf(dm.x) + fabsf(tm.x), fabsf(dm.y) + fabsf(tm.y));
    const float2 B = make_float2(fabsf(dp.x) + fabsf(tp.x), fabsf(dp.y) + fabsf(tp.y));
    const float2 lhs = fma2(mul2(p2(2.f), A), B, p2(eps));
    const float2 rhs = mul2(p2(0.4f), add2(fma2(A, A, mul2(B, B)), p2(eps)));
    sa = lhs.x > rhs.x;
    sb = lhs.y > rhs.y;
}

// hllc_flux (HLLC_Riemann_solver, InviscousFlux.cpp:449-592) for both lines:
// the side states, wave speeds, S_M and the star flux of the upwind side in
// paired arithmetic; reciprocals, square roots, divisions, minima and the
// side selection per half.  Faces with S_L >= 0 or S_R <= 0 (supersonic,
// rare) and S_M denominators below 1e-12 take the scalar forms per half.
template <int DIR>
__device__ __forceinline__ void hllc_flux2(const float2 *UL, const float2 *UR, float g, float2 *F) {
    const float2 rL = UL[0], rR = UR[0], EL = UL[4], ER = UR[4];
    const float2 irL = make_float2(1.f / rL.x, 1.f / rL.y), irR = make_float2(1.f / rR.x, 1.f / rR.y);
    const float2 uL = mul2(UL[1], irL), vL = mul2(UL[2], irL), wL = mul2(UL[3], irL);
    const float2 uR = mul2(UR[1], irR), vR = mul2(UR[2], irR), wR = mul2(UR[3], irR);
    const float2 gm1 = p2(g - 1.f), mh = p2(-0.5f);
    const float2 pL = mul2(fma2(mul2(mh, rL), fma2(wL, wL, fma2(vL, vL, mul2(uL, uL))), EL), gm1);
    const float2 pR = mul2(fma2(mul2(mh, rR), fma2(wR, wR, fma2(vR, vR, mul2(uR, uR))), ER), gm1);
    const float2 unL = DIR == 0 ? uL : (DIR == 1 ? vL : wL), unR = DIR == 0 ? uR : (DIR == 1 ? vR : wR);
    const float2 tL = mul2(mul2(p2(g), pL), irL), tR = mul2(mul2(p2(g), pR), irR);
    const float2 aL = make_float2(sqrtf(tL.x), sqrtf(tL.y)), aR = make_float2(sqrtf(tR.x), sqrtf(tR.y));
    const float2 dL = sub2(unL, aL), dR = sub2(unR, aR), eL = add2(unL, aL), eR = add2(unR, aR);
    const float2 SL = make_float2(fminf(dL.x, dR.x), fminf(dL.y, dR.y));
    const float2 SR = make_float2(fmaxf(eL.x, eR.x), fmaxf(eL.y, eR.y));
    const float2 cR = sub2(SR, unR), cL = sub2(SL, unL);
    const float2 num = add2(sub2(mul2(mul2(rR, unR), cR), mul2(mul2(rL, unL), cL)), sub2(pL, pR));
    const float2 den = sub2(mul2(rR, cR), mul2(rL, cL));
    float2 SM;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const float n_ = h ? num.y : num.x, d_ = h ? den.y : den.x;
        float sm;
        if (fabsf(d_) > 1e-12f) {
            sm = n_ / d_;
        } else {
            const float sL = sqrtf(h ? rL.y : rL.x), sR = sqrtf(h ? rR.y : rR.x);
            sm = (sL * (h ? unL.y : unL.x) + sR * (h ? unR.y : unR.x)) / (sL + sR);
        }
        if (h) SM.y = sm; else SM.x = sm;
    }
    // the star state of the upwind side, per half
    const bool lx = SM.x >= 0.f, ly = SM.y >= 0.f;
    auto sel = [&](float2 l, float2 r) { return make_float2(lx ? l.x : r.x, ly ? l.y : r.y); };
    const float2 r = sel(rL, rR), ir = sel(irL, irR), u = sel(uL, uR), v = sel(vL, vR), w = sel(wL, wR);
    const float2 E = sel(EL, ER), p = sel(pL, pR), un = sel(unL, unR), Sk = sel(SL, SR);
    const float2 U1 = sel(UL[1], UR[1]), U2 = sel(UL[2], UR[2]), U3 = sel(UL[3], UR[3]);
    const float2 m = mul2(r, un);
    const float2 zero = p2(0.f);
    const float2 Fs0 = m;
    const float2 Fs1 = fma2(m, u, DIR == 0 ? p : zero);
    const float2 Fs2 = fma2(m, v, DIR == 1 ? p : zero);
    const float2 Fs3 = fma2(m, w, DIR == 2 ? p : zero);
    const float2 Fs4 = mul2(add2(E, p), un);
    const float2 dk = sub2(Sk, un), rdk = mul2(r, dk), dS = sub2(Sk, SM);
    const float2 rs = make_float2(rdk.x / dS.x, rdk.y / dS.y);
    const float2 pr = make_float2(p.x / rdk.x, p.y / rdk.y);
    const float2 Es = fma2(sub2(SM, un), add2(SM, pr), mul2(E, ir));
    const float2 us = DIR == 0 ? SM : u, vs = DIR == 1 ? SM : v, ws = DIR == 2 ? SM : w;
    F[0] = fma2(Sk, sub2(rs, r), Fs0);
    F[1] = fma2(Sk, sub2(mul2(rs, us), U1), Fs1);
    F[2] = fma2(Sk, sub2(mul2(rs, vs), U2), Fs2);
    F[3] = fma2(Sk, sub2(mul2(rs, ws), U3), Fs3);
    F[4] = fma2(Sk, sub2(mul2(rs, Es), E), Fs4);
    // supersonic faces: the physical flux of the upwind state
    if (SL.x >= 0.f || SR.x <= 0.f || SL.y >= 0.f || SR.y <= 0.f) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float sl = h ? SL.y : SL.x, sr = h ? SR.y : SR.x;
            if (sl >= 0.f || sr <= 0.f) {
                const float2 *Us = sl >= 0.f ? UL : UR;
                float Uh[5], Fh[5];
#pragma unroll
                for (int q = 0; q < 5; ++q) Uh[q] = h ? Us[q].y : Us[q].x;
                Side<DIR, float> S;
                S.load(Uh, g);
                S.flux(Fh);
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    if (h) F[q].y = Fh[q]; else F[q].x = Fh[q];
                }
            }
        }
    }
}

// Chunk geometry: C faces of NL = 2 NP lines per chunk, one thread per
// (line pair, face).  Buffers hold float2 (both lines of a pair):
//   cells  position p <-> cell fc - 2 + p, p in [0, NU)
//   faces  position p <-> face fc - 5 + p, p in [0, NF)
//   visc   position p <-> cell fc - 5 + p, p in [0, NV)
// Along x a warp owns one pair ([pair][pos]); along y/z the 16 pairs of a
// bundle span half a warp ([pos][pair]); both give conflict-free 64-bit
// accesses.
template <int DIR>
struct PairGeom {
    static constexpr int C = DIR == 0 ? 32 : 16;   // faces per chunk
    static constexpr int NP = DIR == 0 ? 8 : 16;   // line pairs per block
    static constexpr int NL = 2 * NP;              // lines per block
    static constexpr int CH = C * NP;              // threads
    static constexpr int NU = C + 5, NF = C + 7, NV = C + 8;
    template <int NPOS>
    __device__ __forceinline__ static int idx(int pair, int pos) {
        return DIR == 0 ? pair * NPOS + pos : pos * NP + pair;
    }
    __device__ __forceinline__ static int tidx(int pair, int slot) {
        return DIR == 0 ? pair * C + slot : slot * NP + pair;
    }
};
static_assert(PairGeom<2>::NL == SweepGeom<2, float>::NLINE, "the fused stage's CFL partials assume one z-sweep grid");

// float2 units: U(5) F(5) V(4), staging W(5)+V(4), old RHS(5); z-sweep:
// FP64 U0 (5 double2), the FP32 stage increments (5 float2) and the deferred
// primitives of the first five cells of periodic lines (6 x 5 x NP float2)
template <int DIR>
constexpr size_t pair_smem_bytes() {
    using G = PairGeom<DIR>;
    return 8 * ((size_t)G::NP * (5 * G::NU + 5 * G::NF + 4 * G::NV) + (size_t)14 * G::CH) +
           (DIR == 2 ? (size_t)5 * G::CH * 16 + (size_t)5 * G::CH * 8 + (size_t)6 * 5 * G::NP * 8 : 0);
}
static_assert((PairGeom<2>::NP * (5 * PairGeom<2>::NU + 5 * PairGeom<2>::NF + 4 * PairGeom<2>::NV) +
               14 * PairGeom<2>::CH) % 2 == 0, "double2 staging must start 16-byte aligned");

// resident blocks per SM requested from the register allocator: three along
// x (80 registers, 63 KB of shared memory; 0.50 -> 0.46 ms at 256^3), two
// along y and z (the z-sweep's fused stage needs its registers, and 111 KB of
// shared memory per block allow two).  The shared-memory carveout is left to
// the driver: forcing the largest one (smallest L1) slowed the x and y
// sweeps by 10-25 %.
template <int DIR>
constexpr int pair_min_blocks() { return DIR == 0 ? 3 : 2; }

template <int DIR, int INTERP, int RS>
__global__ void __launch_bounds__(256, pair_min_blocks<DIR>()) sweep_pair_kernel(SweepArgs<float> a, PairConsts pc) {
    using G = PairGeom<DIR>;
    constexpr int C = G::C, NP = G::NP, NL = G::NL, CH = G::CH, NU = G::NU, NF = G::NF, NV = G::NV;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *const sU = reinterpret_cast<float2 *>(smem_raw);  // [5][NP*NU]
    float2 *const sF = sU + 5 * NP * NU;                       // [5][NP*NF]
    float2 *const sV = sF + 5 * NP * NF;                       // [4][NP*NV]
    float2 *const stg = sV + 4 * NP * NV;                      // [9][CH]
    float2 *const srold = stg + 9 * CH;                        // [5][CH]
    double2 *const sUf = reinterpret_cast<double2 *>(srold + 5 * CH);  // [5][CH] z: U0
    float2 *const sDs = reinterpret_cast<float2 *>(sUf + 5 * CH);      // [5][CH] z: stage increment
    float2 *const sDef = sDs + 5 * CH;                                 // [6][5][NP] z: deferred W, T
    // periodic x-lines: faces 0 .. 4 of each pair, kept from the first chunk
    // for faces n .. n+4 (the same wrapped cells, so the same bits)
    __shared__ float2 sWrapF[DIR == 0 ? 25 * NP : 1];

    if (a.done && *a.done) return;  // uniform over the grid
    const Layout &L = a.L;
    const double fdt = (DIR == 2 && a.fs.stage) ? (a.fs.dt_dev ? *a.fs.dt_dev : a.fs.dt) : 0.0;
    double cfl_acc = 0.0, ke_acc = 0.0, ke_c = 0.0;  // largest wave speed, kinetic energy
    const double irg = (DIR == 2 && a.fs.stage) ? 1.0 / a.fs.Rgas : 0.0;  // T = p / (rho Rgas)
    bool has_def = false;
    const int slot = DIR == 0 ? threadIdx.x : threadIdx.y;
    const int pr = DIR == 0 ? threadIdx.y : threadIdx.x;
    const int ta0 = blockIdx.x * NL + 2 * pr, tb0 = blockIdx.y + (DIR == 2 ? 0 : a.zlo);  // first line of the pair
    const bool line_ok = ta0 < (DIR == 0 ? L.ny : L.nx);          // both lines (even count)
    const int n = DIR == 0 ? L.nx : (DIR == 1 ? L.ny : L.nz);
    // padded-layout address of cell c of the first line; the second line is
    // lpair (vpair for the node fluxes) further on
    long lbase, lstride, lpair, vbase, vstride, vpair;
    if (DIR == 0) {
        lbase = L.at(0, ta0 + NG, tb0 + NG); lstride = 1; lpair = L.px;
        vbase = ((long)tb0 * L.ny + ta0) * L.nx; vstride = 1; vpair = L.nx;
    } else if (DIR == 1) {
        lbase = L.at(ta0 + NG, 0, tb0 + NG); lstride = L.px; lpair = 1;
        vbase = (long)tb0 * L.ny * L.nx + ta0; vstride = L.nx; vpair = 1;
    } else {
        lbase = L.at(ta0 + NG, tb0 + NG, 0); lstride = (long)L.px * L.sy; lpair = 1;
        vbase = (long)tb0 * L.nx + ta0; vstride = (long)L.nx * L.ny; vpair = 1;
    }
    const bool per = a.periodic != 0;
    const bool visc = a.visc != 0;
    const bool rmw = a.first == 0;
    const int fb = per ? 0 : NG - 1;
    const int fe = per ? n + 5 : n + NG;
    const int cell_end = per ? n + 8 : n + 6;
    const int chunk_end = n + NG + 2;
    const int ti = G::tidx(pr, slot);
    const float gm1 = a.sp.gamma - 1.f;
    // z with nx a multiple of 4: the even pair copies its own and the next
    // pair's values (four x-neighbouring lines, 16 bytes, past L1); the two
    // pairs share line_ok and every staging condition.  The z-sweep's 111 KB
    // of shared memory per block leave little L1 for 8-byte cp.async.ca
    // copies (0.81 -> 0.69 ms at 256^3); along y, with a large L1, the
    // 8-byte copies are faster (0.43 against 0.47 ms).
    const bool wide = DIR == 2 && (L.nx & 3) == 0;
    const bool lead = !wide || (pr & 1) == 0;

    auto wrap = [&](int c) { return per ? (c < NG ? c + n : (c >= n + NG ? c - n : c)) : c; };
    auto vis_pos = [&](int c) -> int {
        if (c < 0) return -1;
        int ci = c - NG;
        if (per) { if (ci < 0) ci += n; else if (ci >= n) ci -= n; return ci; }
        return (ci >= 0 && ci < n) ? ci : -1;
    };
    auto ld2 = [&](const float *p, long off) -> float2 {
        if (DIR == 0) return make_float2(p[0], p[off]);
        return *reinterpret_cast<const float2 *>(p);
    };
    auto cp2 = [&](float2 *dst, const float *src, long off) {
        if (DIR == 0) { cp_async(&dst->x, src); cp_async(&dst->y, src + off); }
        else cp_async8(dst, src);
    };
    auto cpw = [&](float2 *dst, const float *src, long off) {
        if (wide) { if (lead) cp_async16f(dst, src); }
        else cp2(dst, src, off);
    };
    auto st2 = [&](float *p, long off, float2 v) {
        if (DIR == 0) { p[0] = v.x; p[off] = v.y; }
        else *reinterpret_cast<float2 *>(p) = v;
    };
    auto put_cell = [&](int pu, int pv, const float2 *w5, const float2 *vf) {
        float Ua[5], Ub[5];
        p2c_f(w5[0].x, w5[1].x, w5[2].x, w5[3].x, w5[4].x, gm1, Ua);
        p2c_f(w5[0].y, w5[1].y, w5[2].y, w5[3].y, w5[4].y, gm1, Ub);
        const int s = G::template idx<NU>(pr, pu);
#pragma unroll
        for (int q = 0; q < 5; ++q) sU[q * NP * NU + s] = make_float2(Ua[q], Ub[q]);
        if (visc && pv >= 0) {
            const int sv = G::template idx<NV>(pr, pv);
#pragma unroll
            for (int q = 0; q < 4; ++q) sV[q * NP * NV + sv] = vf[q];
        }
    };

    // ---- first chunk: visc positions [0, NV) = cells fb-5 .., cell
    //      positions [0, NU) = cells fb-2 .. (position p-3 of the same cell)
    if (line_ok) {
        for (int p = slot; p < NV; p += C) {
            const int c = fb - 5 + p;
            float2 vf[4] = {p2(0.f), p2(0.f), p2(0.f), p2(0.f)};
            if (visc) {
                const int ci = vis_pos(c);
                if (ci >= 0) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) vf[q] = ld2(a.V[q] + vbase + ci * vstride, vpair);
                }
            }
            if (p >= 3 && c < cell_end) {
                const long id = lbase + wrap(c) * lstride;
                float2 w5[5];
#pragma unroll
                for (int q = 0; q < 5; ++q) w5[q] = ld2(a.W[q] + id, lpair);
                put_cell(p - 3, p, w5, vf);
            } else if (visc) {
                const int sv = G::template idx<NV>(pr, p);
#pragma unroll
                for (int q = 0; q < 4; ++q) sV[q * NP * NV + sv] = vf[q];
            }
        }
    }

    for (int fc = fb; fc < chunk_end; fc += C) {
        // cell updated by this thread (both lines) in this chunk
        const int cu = fc - 2 + slot;
        const bool upd = line_ok && cu >= NG && cu < n + NG && (DIR != 2 || (cu - NG >= a.zlo && cu - NG < a.zhi));
        const long cid = lbase + cu * lstride;
        if (rmw && upd) {
#pragma unroll
            for (int q = 0; q < 5; ++q) cpw(&srold[q * CH + ti], a.Rhs[q] + cid, lpair);
        }
        if constexpr (DIR == 2) {
            if (a.fs.stage && upd) {  // the FP64 state of the two cells this thread updates
                const long c64 = a.fs.L64.at(ta0 + NG, tb0 + NG, cu);
#pragma unroll
                for (int q = 0; q < 5; ++q) cp_async16(&sUf[q * CH + ti], a.fs.U0[q] + c64);
                if (a.fs.stage > 1) {
#pragma unroll
                    for (int q = 0; q < 5; ++q) cpw(&sDs[q * CH + ti], a.fs.D[q] + cid, lpair);
                }
            }
        }
        cp_async_commit();
        // stage the next chunk's new cell (cell and visc positions 5+slot, 8+slot)
        const int cn = fc + C + 3 + slot;
        const bool stage = fc + C < chunk_end && line_ok && cn < cell_end;
        if (stage) {
            const long id = lbase + wrap(cn) * lstride;
#pragma unroll
            for (int q = 0; q < 5; ++q) cpw(&stg[q * CH + ti], a.W[q] + id, lpair);
            if (visc) {
                const int ci = vis_pos(cn);
                if (ci >= 0) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) cpw(&stg[(5 + q) * CH + ti], a.V[q] + vbase + ci * vstride, vpair);
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) stg[(5 + q) * CH + ti] = p2(0.f);
                }
            }
        }
        cp_async_commit();
        __syncthreads();  // buffers of this chunk complete

        // ---- face f = fc + slot of both lines: cell positions slot .. slot+5
        const int f = fc + slot;
        if (DIR == 0 && per && fc >= n) {
            // the last chunk of a periodic x-line holds only faces n .. n+4
            // (fc >= n: uniform over the block): copies of faces 0 .. 4
            if (line_ok && f < fe) {
#pragma unroll
                for (int q = 0; q < 5; ++q)
                    sF[q * NP * NF + G::template idx<NF>(pr, slot + 5)] = sWrapF[(q * NP + pr) * 5 + (f - n)];
            }
        } else if (line_ok && f < fe) {
            // one variable's stencil at a time (its registers die with it);
            // the rare WENO branch re-reads its stencil from shared memory
            float2 UL[5], UR[5];
            unsigned wa = 0, wb = 0;
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                float2 sq[6];
#pragma unroll
                for (int m = 0; m < 6; ++m) sq[m] = sU[q * NP * NU + G::template idx<NU>(pr, slot + m)];
                if constexpr (INTERP == I_MDCD_HYBRID || INTERP == I_MDCD_LINEAR) {
                    UL[q] = mdcd_linear2(pc.lin, sq[0], sq[1], sq[2], sq[3], sq[4], sq[5]);
                    UR[q] = mdcd_linear2(pc.lin, sq[5], sq[4], sq[3], sq[2], sq[1], sq[0]);
                }
                if constexpr (INTERP == I_MDCD_HYBRID) {
                    // detectors of both lines at the face's two central cells
                    bool a2, b2, a3, b3;
                    mdcd_smooth2(sq[0], sq[1], sq[2], sq[3], sq[4], a2, b2);
                    mdcd_smooth2(sq[1], sq[2], sq[3], sq[4], sq[5], a3, b3);
                    wa |= ((a2 && a3) ? 0u : 1u) << q;
                    wb |= ((b2 && b3) ? 0u : 1u) << q;
                } else if constexpr (INTERP != I_MDCD_LINEAR) {
                    float sa[6], sb[6];
#pragma unroll
                    for (int m = 0; m < 6; ++m) { sa[m] = sq[m].x; sb[m] = sq[m].y; }
                    face_pair<float, INTERP>(a.sp, sa, UL[q].x, UR[q].x);
                    face_pair<float, INTERP>(a.sp, sb, UL[q].y, UR[q].y);
                }
            }
            if constexpr (INTERP == I_MDCD_HYBRID) {
                if (wa | wb) {  // the WENO branch of the lines whose detector rejected the linear scheme
#pragma unroll
                    for (int q = 0; q < 5; ++q) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            if ((h ? wb : wa) & (1u << q)) {
                                const volatile float *vq = reinterpret_cast<const volatile float *>(sU + q * NP * NU);
                                float f[6];
#pragma unroll
                                for (int m = 0; m < 6; ++m) f[m] = vq[2 * G::template idx<NU>(pr, slot + m) + h];
                                const float l = mdcd_weno_branch(a.sp.hd, f[0], f[1], f[2], f[3], f[4], f[5]);
                                const float r = mdcd_weno_branch(a.sp.hd, f[5], f[4], f[3], f[2], f[1], f[0]);
                                if (h) { UL[q].y = l; UR[q].y = r; } else { UL[q].x = l; UR[q].x = r; }
                            }
                        }
                    }
                }
            }
            const int s = G::template idx<NF>(pr, slot + 5);
            if constexpr (RS == R_HLLC) {
                float2 F[5];
                hllc_flux2<DIR>(UL, UR, a.sp.gamma, F);
#pragma unroll
                for (int q = 0; q < 5; ++q) sF[q * NP * NF + s] = F[q];
            } else {
                float ULa[5], URa[5], ULb[5], URb[5], Fa[5], Fb[5];
#pragma unroll
                for (int q = 0; q < 5; ++q) { ULa[q] = UL[q].x; URa[q] = UR[q].x; ULb[q] = UL[q].y; URb[q] = UR[q].y; }
                riemann<DIR, float, RS>(a.sp, ULa, URa, Fa);
                riemann<DIR, float, RS>(a.sp, ULb, URb, Fb);
#pragma unroll
                for (int q = 0; q < 5; ++q) sF[q * NP * NF + s] = make_float2(Fa[q], Fb[q]);
            }
            if (DIR == 0 && per && f < 5) {  // first chunk (fb = 0 on periodic lines)
#pragma unroll
                for (int q = 0; q < 5; ++q) sWrapF[(q * NP + pr) * 5 + f] = sF[q * NP * NF + s];
            }
        }
        cp_async_wait<1>();  // this thread's old-RHS / FP64-state copies landed
        __syncthreads();     // faces of this chunk complete
        float2 rold[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) rold[q] = (rmw && upd) ? srold[q * CH + ti] : p2(0.f);

        // ---- cell cu of both lines: faces cu-3 .. cu+2 at positions slot ..
        //      slot+5, node fluxes cu-3 .. cu+3 at visc positions slot .. slot+6
        if (upd) {
            const bool edge = !per && (cu - NG < 3 || cu - NG >= n - 3);
            float2 d[5], vd[4] = {p2(0.f), p2(0.f), p2(0.f), p2(0.f)};
            if (!edge) {
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    const float2 *fq = sF + q * NP * NF;
                    auto F_ = [&](int m) { return fq[G::template idx<NF>(pr, slot + m)]; };
                    // diff_6th_central_half, InviscousFlux.cpp:990-992
                    float2 t = mul2(sub2(F_(3), F_(2)), p2(float(75.0 / 64.0)));
                    t = fma2(sub2(F_(4), F_(1)), p2(float(-25.0 / 384.0)), t);
                    t = fma2(sub2(F_(5), F_(0)), p2(float(3.0 / 640.0)), t);
                    d[q] = mul2(t, p2(a.inv_h));
                }
                if (visc) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float2 *vq = sV + q * NP * NV;
                        auto V_ = [&](int off) { return vq[G::template idx<NV>(pr, slot + 3 + off)]; };
                        float2 t = fma2(p2(-9.f), V_(2), V_(3));
                        t = fma2(p2(45.f), V_(1), t);
                        t = fma2(p2(-45.f), V_(-1), t);
                        t = fma2(p2(9.f), V_(-2), t);
                        vd[q] = mul2(sub2(t, V_(-3)), p2(a.dinv[2]));
                    }
                }
            } else {
                // within 3 cells of a non-periodic boundary: ghost faces and
                // reduced viscous orders as the scalar kernel, per line
                const int pf_lo = (NG - 1) - (fc - 5), pf_hi = (n + NG - 1) - (fc - 5);
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    float2 fv[6];
#pragma unroll
                    for (int m = 0; m < 6; ++m) {
                        int pm = slot + m;
                        bool zero = false;
                        const int ff = cu - 3 + m;
                        if (ff < NG - 1) { if (a.outflow_lo) pm = pf_lo; else zero = true; }
                        else if (ff > n + NG - 1) { if (a.outflow_hi) pm = pf_hi; else zero = true; }
                        fv[m] = zero ? p2(0.f) : sF[q * NP * NF + G::template idx<NF>(pr, pm)];
                    }
                    float2 t = mul2(sub2(fv[3], fv[2]), p2(float(75.0 / 64.0)));
                    t = fma2(sub2(fv[4], fv[1]), p2(float(-25.0 / 384.0)), t);
                    t = fma2(sub2(fv[5], fv[0]), p2(float(3.0 / 640.0)), t);
                    d[q] = mul2(t, p2(a.inv_h));
                }
                if (visc) {
                    const int o = visc_order(cu - NG, n, false);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float2 *vq = sV + q * NP * NV;
                        vd[q].x = dstencil_inv<float>(
                            [&](int off) { return vq[G::template idx<NV>(pr, slot + 3 + off)].x; }, o, a.dinv);
                        vd[q].y = dstencil_inv<float>(
                            [&](int off) { return vq[G::template idx<NV>(pr, slot + 3 + off)].y; }, o, a.dinv);
                    }
                }
            }
            float2 rq[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                rq[q] = sub2(rold[q], d[q]);
                if (q > 0) rq[q] = add2(rq[q], vd[q - 1]);
            }
            bool fused = false;
            if constexpr (DIR == 2) {
                if (a.fs.stage) {
                    // runge_kutta_3's update of both cells (range_kutta.cpp:53-91) in
                    // increment form: U_s = U0 + D_s with the FP32 increments
                    // D_1 = dt L0 and D_2 = (D_1 + dt L1) / 4 kept between stages,
                    // and U_3 = U0 + 2/3 (D_2 + dt L2) in FP64
                    const FusedStage &fs = a.fs;
                    const long c64 = fs.L64.at(ta0 + NG, tb0 + NG, cu);
                    double2 Uo[5];
                    float2 Wn[5], Tn, Dn[5];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        double U[5];
#pragma unroll
                        for (int q = 0; q < 5; ++q) {
                            const double rr = (double)(h ? rq[q].y : rq[q].x);
                            const double2 s0 = sUf[q * CH + ti];
                            const double u0 = h ? s0.y : s0.x;
                            double dp = 0.0;
                            if (fs.stage > 1) { const float2 d = sDs[q * CH + ti]; dp = (double)(h ? d.y : d.x); }
                            if (fs.stage == 3) {
                                U[q] = u0 + (2.0 / 3.0) * (dp + fdt * rr);
                            } else {
                                const float dn = (float)(fs.stage == 1 ? fdt * rr : 0.25 * (dp + fdt * rr));
                                if (h) Dn[q].y = dn; else Dn[q].x = dn;
                                U[q] = u0 + (double)dn;
                            }
                        }
                        if (U[0] <= 0.0) U[0] = 1e-12;
                        double W[5], ir;
                        c2p_fast(U, fs.gamma, W, ir);
                        const float t = (float)(W[4] * ir * irg);
#pragma unroll
                        for (int q = 0; q < 5; ++q) {
                            if (h) { Uo[q].y = U[q]; Wn[q].y = (float)W[q]; }
                            else { Uo[q].x = U[q]; Wn[q].x = (float)W[q]; }
                        }
                        if (h) Tn.y = t; else Tn.x = t;
                        if (fs.stage == 3) {
                            cfl_acc = fmax(cfl_acc, cfl_speed(U, fs.gamma));
                            const double y = 0.5 * W[0] * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) * fs.vol - ke_c;
                            const double tk = __dadd_rn(ke_acc, y);
                            ke_c = __dsub_rn(__dsub_rn(tk, ke_acc), y);
                            ke_acc = tk;
                        }
                    }
                    if (fs.stage == 3) {
#pragma unroll
                        for (int q = 0; q < 5; ++q) *reinterpret_cast<double2 *>(fs.Uout[q] + c64) = Uo[q];
                    } else {
#pragma unroll
                        for (int q = 0; q < 5; ++q) *reinterpret_cast<float2 *>(fs.D[q] + cid) = Dn[q];
                    }
                    if (per && cu < NG + 5) {  // re-read by the line's wrapped end: write after the line
                        has_def = true;
                        const int dp = (cu - NG) * NP + pr;
#pragma unroll
                        for (int q = 0; q < 5; ++q) sDef[q * 5 * NP + dp] = Wn[q];
                        sDef[5 * 5 * NP + dp] = Tn;
                    } else {
#pragma unroll
                        for (int q = 0; q < 5; ++q) *reinterpret_cast<float2 *>(fs.W32out[q] + cid) = Wn[q];
                        *reinterpret_cast<float2 *>(fs.T32out + cid) = Tn;
                    }
                    fused = true;
                }
            }
            if (!fused || a.fs.keep_rhs) {  // keep_rhs: the last stage's complete RHS as well
#pragma unroll
                for (int q = 0; q < 5; ++q) st2(a.Rhs[q] + cid, lpair, rq[q]);
            }
        }
        cp_async_wait<0>();
        __syncthreads();  // buffer reads of this chunk done; staged cells landed

        // ---- move the tails to the front, append the staged cell
        if (line_ok && fc + C < chunk_end) {
            if (visc && slot >= C - 8) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    sV[q * NP * NV + G::template idx<NV>(pr, slot - C + 8)] =
                        sV[q * NP * NV + G::template idx<NV>(pr, slot + 8)];
            }
            if (slot >= C - 5) {
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    sU[q * NP * NU + G::template idx<NU>(pr, slot - C + 5)] =
                        sU[q * NP * NU + G::template idx<NU>(pr, slot + 5)];
                    sF[q * NP * NF + G::template idx<NF>(pr, slot - C + 5)] =
                        sF[q * NP * NF + G::template idx<NF>(pr, slot + 5)];
                }
            }
            if (stage) {
                float2 w5[5], v4[4] = {p2(0.f), p2(0.f), p2(0.f), p2(0.f)};
#pragma unroll
                for (int q = 0; q < 5; ++q) w5[q] = stg[q * CH + ti];
                if (visc) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) v4[q] = stg[(5 + q) * CH + ti];
                }
                put_cell(5 + slot, 8 + slot, w5, v4);
            }
        }
    }
    if constexpr (DIR == 2) {
        if (has_def) {  // the line is done: nothing reads these cells any more
            // the thread deferred its cells of the first chunk: cu = fb - 2 + slot
            const int cu = fb - 2 + slot;
            const long cid = lbase + cu * lstride;
            const int dp = (cu - NG) * NP + pr;
#pragma unroll
            for (int q = 0; q < 5; ++q) *reinterpret_cast<float2 *>(a.fs.W32out[q] + cid) = sDef[q * 5 * NP + dp];
            *reinterpret_cast<float2 *>(a.fs.T32out + cid) = sDef[5 * 5 * NP + dp];
        }
        if (a.fs.stage == 3)  // uniform: every thread of the block arrives
            block_speed_sum_n<CH>(cfl_acc, ke_acc - ke_c, a.fs.dx,
                                  a.fs.cfl_part + (long)blockIdx.y * gridDim.x + blockIdx.x,
                                  a.fs.ke_part + (long)blockIdx.y * gridDim.x + blockIdx.x);
    }
}

template <int DIR, int INTERP, int RS>
inline cudaError_t launch_pair(const SweepArgs<float> &a, cudaStream_t st) {
    using G = PairGeom<DIR>;
    dim3 block(DIR == 0 ? G::C : G::NP, DIR == 0 ? G::NP : G::C);
    dim3 grid(((DIR == 0 ? a.L.ny : a.L.nx) + G::NL - 1) / G::NL, DIR == 2 ? a.L.ny : a.zhi - a.zlo);
    const size_t smem = pair_smem_bytes<DIR>();
    static unsigned configured = 0;  // one bit per device ordinal
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(configured & (1u << (dev & 31)))) {
        cudaError_t e = cudaFuncSetAttribute(sweep_pair_kernel<DIR, INTERP, RS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured |= 1u << (dev & 31);
    }
    PairConsts pc;
    for (int k = 0; k < 6; ++k) pc.lin[k] = make_float2(a.sp.lin[k], a.sp.lin[k]);
    sweep_pair_kernel<DIR, INTERP, RS><<<grid, block, smem, st>>>(a, pc);
    return cudaGetLastError();
}

// NS3D_SWEEP32=scalar selects the one-line-per-thread FP32 kernel (kept for
// characteristic reconstruction and odd line counts, and for comparison).
inline bool sweep32_scalar_forced() {
    const char *v = std::getenv("NS3D_SWEEP32");
    return v && std::strcmp(v, "scalar") == 0;
}

template <int DIR>
inline cudaError_t sweep_select_f32(const SweepArgs<float> &a, cudaStream_t st) {
    const auto &sp = a.sp;
    const int across = DIR == 0 ? a.L.ny : a.L.nx;
    if (sp.char_recon || (across & 1) || sweep32_scalar_forced()) return sweep_select<DIR, float>(a, st);
    if (sp.interp == I_WENO5 && sp.riemann == R_ROE) return launch_pair<DIR, I_WENO5, R_ROE>(a, st);
    if (sp.interp == I_MDCD_HYBRID && sp.riemann == R_HLLC) return launch_pair<DIR, I_MDCD_HYBRID, R_HLLC>(a, st);
    if (sp.interp == I_MDCD_LINEAR && sp.riemann == R_HLLC) return launch_pair<DIR, I_MDCD_LINEAR, R_HLLC>(a, st);
    return launch_pair<DIR, RUNTIME, RUNTIME>(a, st);
}

}  // namespace ns3d
