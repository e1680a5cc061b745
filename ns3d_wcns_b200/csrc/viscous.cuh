// viscous.cuh -- node viscous fluxes.
//
// viscous_flux_kernel: at every interior node, the 12 derivatives of u, v, w, T
// with the order chosen by distance to a non-periodic boundary
// (compute_gradients + choose_scheme, ViscousFlux.cpp:15-148), Sutherland mu
// (field_structures.h:96-106), stresses and heat flux, stored as the nine
// distinct node fluxes txx tyy tzz txy txz tyz ex ey ez
// (compute_viscous_flux, ViscousFlux.cpp:151-208; F_v = (txx,txy,txz,ex),
// H_v = (txy,tyy,tyz,ey), G_v = (txz,tyz,tzz,ez)).
//
// A block owns a 32 x 8 column of nodes and marches along z; the plane tiles
// with their halo arrive by TMA (see the kernel).
// T is the array the stage kernel stores (p/(rho Rgas)).
//
// The divergence of these fluxes (compute_vis_flux, ViscousFlux.cpp:210-255)
// is added by the three sweeps, each differencing its direction's fluxes
// along the lines it already stages (sweep.cuh).  In periodic directions that
// stencil wraps to the interior node, which is what
// exchange_halos_viscous_flux (field_structures.h:877-932) copies into the
// ghosts; in non-periodic directions the orders keep the stencil inside.
#pragma once

#include "common.cuh"
#include "reduce.cuh"
#include "tma.cuh"

namespace ns3d {

template <typename R>
struct ViscArgs {
    const R *W[5];          // primitives (padded layout)
    const R *T;             // temperature (padded layout)
    R *V[9];                // node fluxes, interior layout (k*ny + j)*nx + i
    Layout L;
    int periodic[3];
    R h[3];
    R dinv[3][3];           // per direction: 1/(2h), 1/(12h), 1/(60h)
    R mu0, S, cp_over_pr;
    int *err;               // device error word (a bounded wait that ran out)
    const int *done;        // non-null: skip the launch while *done (device time loop)
    int zlo, zhi;           // interior z-planes whose node fluxes are computed
    // non-null: also the turbulence sums of ns3d_diagnostics over the nodes of
    // planes [rlo, rhi), five per block in the order of diag_kernel:
    // 0.5 rho |u|^2 vol, sum_ij (du_i/dx_j)^2, mu(T), rho, |u|^2
    double *red;
    int rlo, rhi;
    double vol;
};

// choose_scheme, ViscousFlux.cpp:33-50 (idx relative to the first interior node)
__device__ __forceinline__ int visc_order(int idx, int n, bool periodic) {
    if (periodic) return 6;
    if (idx == 0) return 1;
    if (idx == n - 1) return -1;
    int d = min(idx, n - 1 - idx);
    return d == 1 ? 2 : (d == 2 ? 4 : 6);
}

// diff_2nd_forward / 2nd / 4th / 6th central, ViscousFlux.cpp:15-29.
// f(o) returns the value at offset o.  Order -1 reproduces the reference's
// backward form, which evaluates to -df/dx.
template <typename R, typename F>
__device__ __forceinline__ R dstencil(F f, int order, R h) {
    if (order == 1 || order == -1)
        return (R(-3) * f(0) + R(4) * f(order) - f(2 * order)) / (R(2) * h);
    if (order == 2) return (f(1) - f(-1)) / (R(2) * h);
    if (order == 4) return (-f(2) + R(8) * f(1) - R(8) * f(-1) + f(-2)) / (R(12) * h);
    return (f(3) - R(9) * f(2) + R(45) * f(1) - R(45) * f(-1) + R(9) * f(-2) - f(-3)) / (R(60) * h);
}

// Sutherland's law mu0 T^1.5 (1+S)/(T+S), with T^1.5 evaluated as T sqrt(T).
template <typename R>
__device__ __forceinline__ R sutherland(R mu0, R S, R T) {
    return mu0 * (T * sqrt(T)) * (R(1) + S) / (T + S);
}

constexpr int VTX = 32, VTY = 8, VH = NG, VZC = 32;

// First derivative of the window value f(o), o in [-3, 3], with a block-
// uniform order; the offsets stay compile-time so the window lives in
// registers.  dinv = 1/(2h), 1/(12h), 1/(60h) (ViscousFlux.cpp:15-29; order
// -1 is the reference's backward form, which evaluates to -df/dx).
template <typename R, typename F>
__device__ __forceinline__ R dwindow(F f, int order, const R *dinv) {
    switch (order) {
        case 6: return (f(3) - R(9) * f(2) + R(45) * f(1) - R(45) * f(-1) + R(9) * f(-2) - f(-3)) * dinv[2];
        case 4: return (-f(2) + R(8) * f(1) - R(8) * f(-1) + f(-2)) * dinv[1];
        case 2: return (f(1) - f(-1)) * dinv[0];
        case 1: return (R(-3) * f(0) + R(4) * f(1) - f(2)) * dinv[0];
        default: return (R(-3) * f(0) + R(4) * f(-1) - f(-2)) * dinv[0];
    }
}

template <typename R, typename F>
__device__ __forceinline__ R dtile(F f, int order, const R *dinv) {
    if (order == 6)
        return (f(3) - R(9) * f(2) + R(45) * f(1) - R(45) * f(-1) + R(9) * f(-2) - f(-3)) * dinv[2];
    if (order == 1 || order == -1) return (R(-3) * f(0) + R(4) * f(order) - f(2 * order)) * dinv[0];
    if (order == 2) return (f(1) - f(-1)) * dinv[0];
    return (-f(2) + R(8) * f(1) - R(8) * f(-1) + f(-2)) * dinv[1];
}

// A block owns a 32 x 8 column of nodes and marches up VZC planes: each
// thread keeps its node's (u, v, w, T) of planes k-3 .. k+3 in registers and
// loads one new plane per step (prefetched a step ahead); the x/y derivatives
// read the plane's tile with its 3-cell halo, which one thread requests as
// four TMA boxes a plane ahead (double buffer, mbarrier completion, bounded
// waits).
// Tensor maps of u, v, w, T of the state being differenced (3-D: x = padded
// element index, y = ghost-inclusive row, z = ghost-inclusive plane).
struct ViscMaps {
    CUtensorMap m[4];
};

// Plane tile as loaded by TMA: rows y0 .. y0+13 (ghost-inclusive), elements
// x0 + off - 1 .. x0 + off + 38 of each row, so a node's ghost-inclusive x0 + t
// sits in column t + 1.  Starting one element early puts the box's x
// coordinate on a 16-byte boundary for both element sizes (FP64: off = 1,
// FP32: off = 5).
constexpr int VBX = 40, VBY = VTY + 2 * VH;
template <typename R>
constexpr int vtile_stride() {  // elements per tile, 128-byte aligned tiles
    return (int)(((VBX * VBY * sizeof(R) + 127) / 128) * 128 / sizeof(R));
}

// P6: every direction periodic, so every derivative is the 6th-order central
// one (choose_scheme's order for periodic directions) and the order dispatch
// compiles away.
// DIAG: the ns3d_diagnostics sums (a.red) from the same gradient tiles, and
// no node fluxes; a separate instantiation, so the kernel of the RK stages
// carries none of it.
template <typename R, bool P6, bool DIAG>
__global__ void __launch_bounds__(VTX * VTY) viscous_flux_kernel(ViscArgs<R> a, const __grid_constant__ ViscMaps tm) {
    constexpr int TS = vtile_stride<R>();
    __shared__ __align__(128) R sm[2 * 4 * TS];  // two plane tiles of u, v, w, T
    __shared__ __align__(8) uint64_t bar[2];
    if (a.done && *a.done) return;  // uniform over the grid
    const Layout &L = a.L;
    const int x0 = blockIdx.x * VTX, y0 = blockIdx.y * VTY;
    const int kb = a.zlo + blockIdx.z * VZC, ke = min(kb + VZC, a.zhi);
    const int i = x0 + threadIdx.x, j = y0 + threadIdx.y;
    const int tid = threadIdx.y * VTX + threadIdx.x;
    const bool in = i < L.nx && j < L.ny;
    const R *src[4] = {a.W[1], a.W[2], a.W[3], a.T};
    const long zs = (long)L.px * L.sy;
    const long col = L.at(min(i, L.nx - 1) + NG, min(j, L.ny - 1) + NG, 0);  // ghost-inclusive plane 0
    const int ox = P6 ? 6 : visc_order(i, L.nx, a.periodic[0]);
    const int oy = P6 ? 6 : visc_order(j, L.ny, a.periodic[1]);
    const int cx = threadIdx.x + VH + 1, cy = threadIdx.y + VH;
    auto tile = [&](int buf, int q) { return sm + (buf * 4 + q) * TS; };
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    auto issue = [&](int buf, int k) {  // one thread: four boxes of plane k
        mbar_arrive_expect_tx(&bar[buf], 4u * VBX * VBY * (unsigned)sizeof(R));
#pragma unroll
        for (int q = 0; q < 4; ++q) tma_load_3d(tile(buf, q), &tm.m[q], x0 + L.off - 1, y0, k + NG, &bar[buf]);
    };
    unsigned phase = 0u;  // bit b: parity of buffer b's next completion
    if (tid == 0) issue(0, kb);
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // ns3d_diagnostics sums (DIAG)
    // window: win[q][m] = value at interior plane k - 3 + m (ghost-inclusive k + m)
    R win[4][7], nxt[4];
#pragma unroll
    for (int m = 0; m < 6; ++m)
#pragma unroll
        for (int q = 0; q < 4; ++q) win[q][m] = src[q][col + (long)(kb + m) * zs];
#pragma unroll
    for (int q = 0; q < 4; ++q) nxt[q] = src[q][col + (long)(kb + 6) * zs];
#pragma unroll 7  // the window shift becomes register renaming (7 planes)
    for (int k = kb; k < ke; ++k) {
        const int buf = (k - kb) & 1;
        const bool more = k + 1 < ke;
        if (more && tid == 0) {
            fence_proxy_async_smem();  // the tile's last readers finished at the previous barrier
            issue(buf ^ 1, k + 1);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) win[q][6] = nxt[q];
        if (more) {
#pragma unroll
            for (int q = 0; q < 4; ++q) nxt[q] = src[q][col + (long)(k + 7) * zs];
        }
        const unsigned par = (phase >> buf) & 1u;
        const bool ok = mbar_wait_bounded(&bar[buf], par, a.err);
        phase ^= 1u << buf;
        if (__syncthreads_or(!ok)) {
            // a tile did not arrive in time (the error word is set): issue
            // nothing more, and let both copies in flight land (bounded)
            // before the block retires
            if (tid == 0) {
                mbar_drain(&bar[buf], par);
                if (more) mbar_drain(&bar[buf ^ 1], (phase >> (buf ^ 1)) & 1u);
            }
            __syncthreads();
            return;
        }
        if (in) {
            const R *tu = tile(buf, 0), *tv = tile(buf, 1), *tw = tile(buf, 2), *tT = tile(buf, 3);
            const R *tq[4] = {tu, tv, tw, tT};
            const int oz = P6 ? 6 : visc_order(k, L.nz, a.periodic[2]);
            R g[4][3];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const R *t = tq[q];
                g[q][0] = dtile<R>([&](int o) { return t[cy * VBX + cx + o]; }, ox, a.dinv[0]);
                g[q][1] = dtile<R>([&](int o) { return t[(cy + o) * VBX + cx]; }, oy, a.dinv[1]);
                g[q][2] = dwindow<R>([&](int o) { return win[q][3 + o]; }, oz, a.dinv[2]);
            }
            const R T = win[3][3];
            const R mu = sutherland(a.mu0, a.S, T);
            const R ux = g[0][0], uy = g[0][1], uz = g[0][2], vx = g[1][0], vy = g[1][1], vz = g[1][2];
            const R wx = g[2][0], wy = g[2][1], wz = g[2][2], Tx = g[3][0], Ty = g[3][1], Tz = g[3][2];
            const R div = ux + vy + wz;
            const R m2 = R(2) * mu, m23 = R(2.0 / 3.0) * mu * div;
            const R txx = m2 * ux - m23, tyy = m2 * vy - m23, tzz = m2 * wz - m23;
            const R txy = mu * (uy + vx), txz = mu * (uz + wx), tyz = mu * (vz + wy);
            const R kq = mu * a.cp_over_pr;
            const R u = win[0][3], v = win[1][3], w = win[2][3];
            const long o = ((long)k * L.ny + j) * L.nx + i;
            if (!DIAG) {
                a.V[0][o] = txx; a.V[1][o] = tyy; a.V[2][o] = tzz;
                a.V[3][o] = txy; a.V[4][o] = txz; a.V[5][o] = tyz;
                a.V[6][o] = u * txx + v * txy + w * txz + kq * Tx;
                a.V[7][o] = u * txy + v * tyy + w * tyz + kq * Ty;
                a.V[8][o] = u * txz + v * tyz + w * tzz + kq * Tz;
            }
            if (DIAG && k >= a.rlo && k < a.rhi) {
                const double rho = (double)a.W[0][col + (long)(k + NG) * zs];
                const double du = u, dv = v, dw = w, uu = du * du + dv * dv + dw * dw;
                acc[0] += 0.5 * rho * uu * a.vol;
                double g2 = 0.0;
#pragma unroll
                for (int q = 0; q < 3; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) g2 += (double)g[q][d] * (double)g[q][d];
                acc[1] += g2;
                acc[2] += (double)mu;
                acc[3] += rho;
                acc[4] += uu;
            }
        }
#pragma unroll
        for (int m = 0; m < 6; ++m)
#pragma unroll
            for (int q = 0; q < 4; ++q) win[q][m] = win[q][m + 1];
        __syncthreads();  // this tile's reads done before it is refilled
    }
    if (DIAG)  // uniform: every thread of the block arrives
        block_sum_n<5, VTX * VTY>(acc, a.red + 5 * ((long)(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x));
}

// All 12 derivatives at interior node (i,j,k) (ghost-inclusive indices), for
// the reductions.
template <typename R>
__device__ __forceinline__ void node_gradients(const ViscArgs<R> &a, int i, int j, int k, R g[12]) {
    const Layout &L = a.L;
    const int o[3] = {visc_order(i - NG, L.nx, a.periodic[0]), visc_order(j - NG, L.ny, a.periodic[1]),
                      visc_order(k - NG, L.nz, a.periodic[2])};
    const long stride[3] = {1, (long)L.px, (long)L.px * L.sy};
    const long c = L.at(i, j, k);
    const R *src[4] = {a.W[1], a.W[2], a.W[3], a.T};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const long s = stride[d];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const R *f = src[q];
            g[3 * q + d] = dstencil<R>([&](int off) { return f[c + off * s]; }, o[d], a.h[d]);
        }
    }
}

}  // namespace ns3d
