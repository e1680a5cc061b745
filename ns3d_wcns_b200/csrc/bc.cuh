// bc.cuh -- the ghost fill of apply_boundary as a per-cell source lookup, and
// the RK3 stage combination with the reference's rounding (shared by the
// single-domain stage kernels and the batched kernel).
#pragma once

#include "common.cuh"

namespace ns3d {

struct BcInfo {
    int periodic[3];
    int bc[6];   // NS3D_* boundary types
};

enum { SRC_CELL = 0, SRC_ZERO = 1, SRC_INFLOW = 2 };
enum { BC_PERIODIC = 0, BC_WALL = 1, BC_SYMMETRY = 2, BC_OUTFLOW = 3, BC_INFLOW = 4 };

// Resolve cell c (ghost-inclusive coordinates) to its source.  flip bit d set
// => negate velocity component d.
__device__ __forceinline__ int resolve_source(const Layout &L, const BcInfo &b, int c[3], int &flip) {
    const int ext[3] = {L.sx, L.sy, L.sz};
    const int n[3] = {L.nx, L.ny, L.nz};
    flip = 0;
#pragma unroll
    for (int face = 5; face >= 0; --face) {
        const int d = face >> 1, hi = face & 1;
        if (b.periodic[d]) continue;
        const int t = b.bc[face];
        if (t == BC_PERIODIC) continue;  // Periodic side without a periodic partner: no fill
        const bool in = hi ? (c[d] >= ext[d] - NG) : (c[d] < NG);
        if (!in) continue;
        if (t == BC_INFLOW) return SRC_INFLOW;
        if (t == BC_OUTFLOW) c[d] = hi ? ext[d] - NG - 1 : NG;
        else { c[d] = hi ? 2 * (ext[d] - NG) - 1 - c[d] : 2 * NG - 1 - c[d]; flip ^= 1 << d; }
    }
    // exchange_halos_physical: ghost in exactly one dimension, interior in the others
    int gd = -1, ng = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
        if (c[d] < NG || c[d] >= NG + n[d]) { gd = d; ++ng; }
    if (ng == 1) {
        if (!b.periodic[gd]) return SRC_ZERO;
        c[gd] += c[gd] < NG ? n[gd] : -n[gd];
    }
    return SRC_CELL;
}

__device__ __forceinline__ bool is_interior(const Layout &L, const int c[3]) {
    return c[0] >= NG && c[0] < NG + L.nx && c[1] >= NG && c[1] < NG + L.ny && c[2] >= NG && c[2] < NG + L.nz;
}

// Constant states of the ghost fill (after primitiveToConserved's clamp).
__device__ __forceinline__ void special_state(int kind, double W[5]) {
    if (kind == SRC_INFLOW) { W[0] = 1.0; W[1] = 1.0; W[2] = 0.0; W[3] = 0.0; W[4] = 1.0; }  // boundary.cpp:188
    else { W[0] = 1e-12; W[1] = 0.0; W[2] = 0.0; W[3] = 0.0; W[4] = 0.0; }
}

__device__ __forceinline__ void apply_flips(int flip, double W[5]) {
    if (flip & 1) W[1] = -W[1];
    if (flip & 2) W[2] = -W[2];
    if (flip & 4) W[3] = -W[3];
}

// RK coefficients of runge_kutta_3 (range_kutta.cpp:55, 69, 83) with the
// reference's rounding (no contraction).
__device__ __forceinline__ double rk_combine(int stage, double u0, double u, double r, double dt) {
    if (stage == 1) return __dadd_rn(u0, __dmul_rn(dt, r));
    if (stage == 2) return __dadd_rn(__dmul_rn(0.75, u0), __dmul_rn(0.25, __dadd_rn(u, __dmul_rn(dt, r))));
    return __dadd_rn(__dmul_rn(1.0 / 3.0, u0), __dmul_rn(2.0 / 3.0, __dadd_rn(u, __dmul_rn(dt, r))));
}

}  // namespace ns3d
