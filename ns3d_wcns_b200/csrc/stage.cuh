// stage.cuh -- RK3 stage update with the state round trip and the ghost fill,
// plus the global reductions (CFL time step, kinetic energy, dissipation).
//
// The reference performs, after every RK stage (range_kutta.cpp:53-91):
//   U = a U0 + b (U + dt rhs) on all cells (rhs = 0 in ghosts),
//   conservedToPrimitive on all cells (density clamp),
//   apply_boundary: periodic exchange (or, in non-periodic dimensions, the
//     unpack of never-received zero buffers) on interior-tangential ghost
//     slabs, then the Wall/Symmetry/Outflow/Inflow fills face by face over
//     full tangential extents (boundary.cpp:14-205),
//   primitiveToConserved on all cells.
// Here one thread per output cell walks that sequence backwards to the cell
// whose stage value it receives (with velocity sign flips, or a constant
// Inflow / zero state), computes that cell's stage update and conversion, and
// writes the result: one pass, no separate ghost kernel, no grid barrier.
#pragma once

#include "bc.cuh"
#include "common.cuh"
#include "reduce.cuh"

namespace ns3d {

// --------------------------------------------------------------- plain FP64

struct StageArgs64 {
    const double *W0[5];    // step-start state
    const double *Wc[5];    // current stage state
    const double *Rhs[5];
    double *Wout[5];
    double *Tout;           // T = p/(rho Rgas) of the new state (field_structures.h:486)
    Layout L;
    BcInfo b;
    double dt, gamma, Rgas;
    int stage;              // 1, 2, 3; 0 = ghost fill only (copy of Wc)
    double *cfl_part;       // non-null: per-block minimum CFL bound of the new state
    double *ke_part;        // with cfl_part: per-block kinetic energy of the new state
    double dx, vol;
    const double *dt_dev;   // non-null: dt from the device time loop (replaces dt)
    const int *done;        // non-null: skip the launch while *done
};

constexpr int STAGE_THREADS = 128;

// The CFL bound of the next step and the kinetic energy of the new state
// ride on the last stage: each block writes the minimum of dx/(|u| + a)
// (timestep.cpp:12-20, from the conserved state as compute_timestep sees it)
// and the sum of rho |u|^2 / 2 dV (postprocess.cpp:103-128) over its interior
// cells.  The minimum of the same per-cell values is the same number whatever
// the partition; the sum is fixed-order (deterministic).
__device__ __forceinline__ void stage_partials(double *cfl_part, double *ke_part, double m, double ke) {
    const long b = ((long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    block_min_sum_n<STAGE_THREADS>(m, ke, cfl_part + b, ke_part + b);
}

__global__ void __launch_bounds__(STAGE_THREADS) stage_kernel64(StageArgs64 a) {
    if (a.done && *a.done) return;  // uniform over the grid
    const double dt = a.dt_dev ? *a.dt_dev : a.dt;
    const Layout &L = a.L;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    double cfl = 1e9;  // the initial minimum of the CFL reduction kernels
    double ke = 0.0;
    if (i < L.sx) {
    int c[3] = {i, j, k};
    int flip;
    const int kind = resolve_source(L, a.b, c, flip);
    double W[5];
    if (kind != SRC_CELL) {
        special_state(kind, W);
    } else {
        const long s = L.at(c[0], c[1], c[2]);
        if (a.stage == 0) {
#pragma unroll
            for (int q = 0; q < 5; ++q) W[q] = a.Wc[q][s];
            if (W[0] <= 0.0) W[0] = 1e-12;
        } else {
            double U0[5], U[5];
            p2c_exact(a.W0[0][s], a.W0[1][s], a.W0[2][s], a.W0[3][s], a.W0[4][s], a.gamma, U0);
            if (a.stage == 1) {
#pragma unroll
                for (int q = 0; q < 5; ++q) U[q] = U0[q];
            } else {
                p2c_exact(a.Wc[0][s], a.Wc[1][s], a.Wc[2][s], a.Wc[3][s], a.Wc[4][s], a.gamma, U);
            }
            const bool inner = is_interior(L, c);
            double Un[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double r = inner ? a.Rhs[q][s] : 0.0;
                Un[q] = rk_combine(a.stage, U0[q], U[q], r, dt);
            }
            c2p_exact(Un, a.gamma, W);
        }
    }
    apply_flips(flip, W);
    const long o = L.at(i, j, k);
#pragma unroll
    for (int q = 0; q < 5; ++q) a.Wout[q][o] = W[q];
    a.Tout[o] = W[4] / __dmul_rn(W[0], a.Rgas);
    if (a.cfl_part) {
        const int co[3] = {i, j, k};
        if (is_interior(L, co)) {
            double Un[5];
            p2c_exact(W[0], W[1], W[2], W[3], W[4], a.gamma, Un);
            cfl = cfl_bound(Un, a.gamma, a.dx);
            ke = 0.5 * W[0] * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) * a.vol;
        }
    }
    }
    if (a.cfl_part) stage_partials(a.cfl_part, a.ke_part, cfl, ke);
}

// --------------------------------------------------------------- mixed path

struct StageArgsMixed {
    const double *U0[5];    // step-start conserved state (FP64)
    const double *Uc[5];    // current stage conserved state (FP64)
    const float *Rhs[5];    // FP32 right-hand side
    double *Uout[5];        // next conserved state (FP64)
    float *Wout[5];         // FP32 primitives for the stencil kernels
    float *Tout;            // FP32 temperature
    Layout L;               // FP64 layout
    Layout L32;             // FP32 layout
    BcInfo b;
    double dt, gamma, Rgas;
    int stage;              // 1, 2, 3; 0 = ghost fill only
    double *cfl_part;       // non-null: per-block minimum CFL bound of the new state
    double *ke_part;        // with cfl_part: per-block kinetic energy of the new state
    double dx, vol;
    const double *dt_dev;   // non-null: dt from the device time loop (replaces dt)
    const int *done;        // non-null: skip the launch while *done
    const float *D[5];      // ghost kernel after the fused z-sweep: stage increments (FP32 layout)
};

__global__ void __launch_bounds__(STAGE_THREADS) stage_kernel_mixed(StageArgsMixed a) {
    if (a.done && *a.done) return;  // uniform over the grid
    const double dt = a.dt_dev ? *a.dt_dev : a.dt;
    const Layout &L = a.L;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    double cfl = 1e9;  // the initial minimum of the CFL reduction kernels
    double ke = 0.0;
    if (i < L.sx) {
    int c[3] = {i, j, k};
    int flip;
    const int kind = resolve_source(L, a.b, c, flip);
    double U[5], W[5];
    if (kind != SRC_CELL) {
        special_state(kind, W);
        apply_flips(flip, W);
        p2c_exact(W[0], W[1], W[2], W[3], W[4], a.gamma, U);
    } else {
        const long s = L.at(c[0], c[1], c[2]);
        if (a.stage == 0) {
#pragma unroll
            for (int q = 0; q < 5; ++q) U[q] = a.Uc[q][s];
        } else {
            const bool inner = is_interior(L, c);
            const long s32 = a.L32.at(c[0], c[1], c[2]);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double r = inner ? (double)a.Rhs[q][s32] : 0.0;
                const double u0 = a.U0[q][s];
                const double u = a.stage == 1 ? u0 : a.Uc[q][s];
                U[q] = a.stage == 1 ? u0 + dt * r
                     : a.stage == 2 ? 0.75 * u0 + 0.25 * (u + dt * r)
                                    : (1.0 / 3.0) * u0 + (2.0 / 3.0) * (u + dt * r);
            }
        }
        if (U[0] <= 0.0) U[0] = 1e-12;
        if (flip & 1) U[1] = -U[1];
        if (flip & 2) U[2] = -U[2];
        if (flip & 4) U[3] = -U[3];
        c2p_exact(U, a.gamma, W);  // FP64 pressure recovery
    }
    const long o = L.at(i, j, k);
#pragma unroll
    for (int q = 0; q < 5; ++q) a.Uout[q][o] = U[q];
    const long o32 = a.L32.at(i, j, k);
#pragma unroll
    for (int q = 0; q < 5; ++q) a.Wout[q][o32] = (float)W[q];
    a.Tout[o32] = (float)(W[4] / (W[0] * a.Rgas));
    if (a.cfl_part) {
        const int co[3] = {i, j, k};
        if (is_interior(L, co)) {
            cfl = cfl_bound(U, a.gamma, a.dx);
            ke = 0.5 * W[0] * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) * a.vol;
        }
    }
    }
    if (a.cfl_part) stage_partials(a.cfl_part, a.ke_part, cfl, ke);
}

// ----------------------------------------------------- ghost fill after a fused stage

// Ghost cells only, one thread each: t enumerates the two z-slabs (full x-y
// planes), then the y-slabs of the interior planes, then the x-ghosts of the
// interior rows.
// Ghost cell number t: the two z-slabs (3 planes each, full sy x sx), then the
// y-slabs of the interior planes, then the x-slabs of the interior rows.  The
// decode runs in 32-bit unsigned arithmetic (the host checks ghost_count <
// 2^31): 64-bit divisions are several times slower.
__device__ __forceinline__ bool ghost_cell(const Layout &L, long t64, int &i, int &j, int &k) {
    const unsigned sx = (unsigned)L.sx, sy = (unsigned)L.sy, nz = (unsigned)L.nz, ny = (unsigned)L.ny;
    const unsigned gz = 6u * sy * sx, gy = 6u * nz * sx, gx = 6u * nz * ny;
    if (t64 < 0 || t64 >= (long)gz + gy + gx) return false;
    unsigned t = (unsigned)t64;
    if (t < gz) {
        const unsigned pl = sy * sx, sl = t / pl, rem = t - sl * pl, jj = rem / sx;
        k = sl < 3 ? (int)sl : L.nz + (int)sl; j = (int)jj; i = (int)(rem - jj * sx);
        return true;
    }
    t -= gz;
    if (t < gy) {
        const unsigned rw = 6u * sx, kk = t / rw, rem = t - kk * rw, sl = rem / sx;
        k = (int)kk + NG;
        j = sl < 3 ? (int)sl : L.ny + (int)sl; i = (int)(rem - sl * sx);
        return true;
    }
    t -= gy;
    const unsigned row = t / 6u, sl = t - row * 6u, kk = row / ny;
    k = (int)kk + NG; j = (int)(row - kk * ny) + NG;
    i = sl < 3 ? (int)sl : L.nx + (int)sl;
    return true;
}

__host__ __device__ inline long ghost_count(const Layout &L) {
    return 6L * L.sy * L.sx + 6L * L.nz * L.sx + 6L * L.nz * L.ny;
}

// After the z-sweep wrote the new interior state (fused stage), the ghost
// cells receive exactly what stage_kernel64 gives them: a copy (with sign
// flips) of their source's new value when the source is interior, the stage
// combination with a zero right-hand side when it is a ghost, or a constant.
__global__ void __launch_bounds__(256) stage_ghost_kernel64(StageArgs64 a) {
    if (a.done && *a.done) return;
    const Layout &L = a.L;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!ghost_cell(L, t, i, j, k)) return;
    const double dt = a.dt_dev ? *a.dt_dev : a.dt;
    int c[3] = {i, j, k};
    int flip;
    const int kind = resolve_source(L, a.b, c, flip);
    double W[5];
    if (kind != SRC_CELL) {
        special_state(kind, W);
    } else {
        const long s = L.at(c[0], c[1], c[2]);
        if (is_interior(L, c)) {
#pragma unroll
            for (int q = 0; q < 5; ++q) W[q] = a.Wout[q][s];
        } else {
            double U0[5], U[5], Un[5];
            p2c_exact(a.W0[0][s], a.W0[1][s], a.W0[2][s], a.W0[3][s], a.W0[4][s], a.gamma, U0);
            if (a.stage == 1) {
#pragma unroll
                for (int q = 0; q < 5; ++q) U[q] = U0[q];
            } else {
                p2c_exact(a.Wc[0][s], a.Wc[1][s], a.Wc[2][s], a.Wc[3][s], a.Wc[4][s], a.gamma, U);
            }
#pragma unroll
            for (int q = 0; q < 5; ++q) Un[q] = rk_combine(a.stage, U0[q], U[q], 0.0, dt);
            c2p_exact(Un, a.gamma, W);
        }
    }
    apply_flips(flip, W);
    const long o = L.at(i, j, k);
#pragma unroll
    for (int q = 0; q < 5; ++q) a.Wout[q][o] = W[q];
    a.Tout[o] = W[4] / __dmul_rn(W[0], a.Rgas);
}

// Ghost cells after the mixed path's fused z-sweep (increment form, see
// FusedStage): a ghost whose source is an interior cell gets that cell's new
// state -- U0 + D after stages 1 and 2 (the conversion the sweep applies, so
// the same FP32 primitives), the FP64 state after stage 3 -- with sign flips;
// a ghost whose source is a ghost keeps its step-start state (its right-hand
// side is zero in every stage); special states are constants.  Only stage 3
// writes the FP64 state's ghosts.
__global__ void __launch_bounds__(256) stage_ghost_kernel_mixed(StageArgsMixed a) {
    if (a.done && *a.done) return;
    const Layout &L = a.L;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!ghost_cell(L, t, i, j, k)) return;
    int c[3] = {i, j, k};
    int flip;
    const int kind = resolve_source(L, a.b, c, flip);
    double U[5], W[5], ir;
    if (kind != SRC_CELL) {
        special_state(kind, W);
        apply_flips(flip, W);
        p2c_exact(W[0], W[1], W[2], W[3], W[4], a.gamma, U);
        ir = 1.0 / W[0];
    } else {
        const long s = L.at(c[0], c[1], c[2]);
        if (is_interior(L, c)) {
            if (a.stage == 3) {
#pragma unroll
                for (int q = 0; q < 5; ++q) U[q] = a.Uout[q][s];  // new value, already clamped
            } else {
                const long s32 = a.L32.at(c[0], c[1], c[2]);
#pragma unroll
                for (int q = 0; q < 5; ++q) U[q] = a.U0[q][s] + (double)a.D[q][s32];
                if (U[0] <= 0.0) U[0] = 1e-12;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 5; ++q) U[q] = a.U0[q][s];
            if (U[0] <= 0.0) U[0] = 1e-12;
        }
        if (flip & 1) U[1] = -U[1];
        if (flip & 2) U[2] = -U[2];
        if (flip & 4) U[3] = -U[3];
        c2p_fast(U, a.gamma, W, ir);  // the conversion the fused z-sweep gives the interior cells
    }
    if (a.stage == 3) {
        const long o = L.at(i, j, k);
#pragma unroll
        for (int q = 0; q < 5; ++q) a.Uout[q][o] = U[q];
    }
    const long o32 = a.L32.at(i, j, k);
#pragma unroll
    for (int q = 0; q < 5; ++q) a.Wout[q][o32] = (float)W[q];
    a.Tout[o32] = (float)(W[4] * ir * (1.0 / a.Rgas));  // as the z-sweep
}

}  // namespace ns3d
