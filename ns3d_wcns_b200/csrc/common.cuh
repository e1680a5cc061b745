// common.cuh -- device layout and the exact-rounding state conversions shared
// by every kernel of the B200 ns3d_wcns path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ns3d {

constexpr int NG = 3;  // ghost layers for WENO5/MDCD (initialization.cpp:175-192)

// Padded device layout of one Field3D array: element (i,j,k), i in [0,sx),
// lives at ((k*sy + j)*px + i + off).  off puts the first interior cell
// (i = 3) on a 32-byte sector boundary; px keeps every row sector aligned.
struct Layout {
    int nx, ny, nz;     // interior
    int sx, sy, sz;     // with ghosts
    int px, off;        // pitch and x offset (elements)
    long plane;         // elements of one padded array (sz*sy*px, rounded)
    __host__ __device__ __forceinline__ long at(int i, int j, int k) const {
        return ((long)k * sy + j) * px + i + off;
    }
};

template <typename T>
inline Layout make_layout(int nx, int ny, int nz) {
    Layout L;
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.sx = nx + 2 * NG; L.sy = ny + 2 * NG; L.sz = nz + 2 * NG;
    const int per_sector = 32 / (int)sizeof(T);
    L.off = per_sector - NG;  // (NG + off) * sizeof(T) == 32
    L.px = ((L.sx + L.off + per_sector - 1) / per_sector) * per_sector;
    long n = (long)L.sz * L.sy * L.px;
    const long align = 256 / (long)sizeof(T);
    L.plane = ((n + align - 1) / align) * align;
    return L;
}

// Device-resident time-advance state (the dt schedule of time_advance,
// maincycle.cpp:18-56, run on the device so that many steps need no host
// round trip).  While `done` is set every kernel of a step returns at once.
struct DevClock {
    double t, dt, t_end, cfl_min;
    int done, steps, budget, err;
};

// Physical constants (initialization.cpp:194-197, field_structures.h:95).
struct Phys {
    double gamma, Rgas, Cp, Pr, mu, S;
    double inv_dx, inv_dy, inv_dz;
    double dx, dy, dz;
    double mdcd_disp, mdcd_diss;
};

// ---------------------------------------------------------------------------
// Conversions with the reference's rounding.  The reference compiles without
// fused multiply-add, so these use the _rn intrinsics (no contraction) and
// IEEE division: for identical inputs they return identical bits.
// ---------------------------------------------------------------------------

// Field3D::primitiveToConserved, field_structures.h:468-488.
__device__ __forceinline__ void p2c_exact(double r, double u, double v, double w, double p,
                                          double gamma, double U[5]) {
    double rr = r <= 0.0 ? 1e-12 : r;
    U[0] = rr;
    U[1] = __dmul_rn(rr, u);
    U[2] = __dmul_rn(rr, v);
    U[3] = __dmul_rn(rr, w);
    double kin = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w)));
    double e = p / __dmul_rn(gamma - 1.0, rr);
    U[4] = __dmul_rn(rr, __dadd_rn(e, kin));
}

// Field3D::conservedToPrimitive, field_structures.h:444-465 (density clamp).
__device__ __forceinline__ void c2p_exact(const double U[5], double gamma, double W[5]) {
    double rr = U[0] <= 0.0 ? 1e-12 : U[0];
    double u = U[1] / rr, v = U[2] / rr, w = U[3] / rr;
    double kin = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w)));
    double e = __dsub_rn(U[4] / rr, kin);
    W[0] = rr; W[1] = u; W[2] = v; W[3] = w;
    W[4] = __dmul_rn(__dmul_rn(gamma - 1.0, rr), e);
}

// Mixed path: conserved -> primitive in FP64 with one reciprocal (the mixed
// path has an accuracy bound, not a bitwise contract); the pressure
// recovery p = (gamma-1)(E - rho |u|^2 / 2), which cancels at low Mach, stays
// FP64.  Density clamp as field_structures.h:444-465.
__device__ __forceinline__ void c2p_fast(const double U[5], double gamma, double W[5], double &irho) {
    const double rr = U[0] <= 0.0 ? 1e-12 : U[0];
    irho = 1.0 / rr;
    const double u = U[1] * irho, v = U[2] * irho, w = U[3] * irho;
    W[0] = rr; W[1] = u; W[2] = v; W[3] = w;
    W[4] = (gamma - 1.0) * (U[4] - 0.5 * rr * (u * u + v * v + w * w));
}

// Float versions for the mixed path (no parity contract).
__device__ __forceinline__ void p2c_f(float r, float u, float v, float w, float p, float gm1,
                                      float U[5]) {
    float rr = r <= 0.f ? 1e-12f : r;
    U[0] = rr; U[1] = rr * u; U[2] = rr * v; U[3] = rr * w;
    U[4] = p / gm1 + 0.5f * rr * (u * u + v * v + w * w);
}

}  // namespace ns3d

namespace ns3d {
// Asynchronous global -> shared copies (LDGSTS), used to stage the next chunk
// of a sweep while the current one computes.
__device__ __forceinline__ void cp_async(double *smem_dst, const double *gsrc) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async(float *smem_dst, const float *gsrc) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
}  // namespace ns3d
