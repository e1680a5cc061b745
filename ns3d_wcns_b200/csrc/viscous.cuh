// viscous.cuh -- viscous terms of the RHS.
//
// Kernel 1 (viscous_flux_kernel): at every interior node, the 12 derivatives
// of u, v, w, T with the order chosen by distance to a non-periodic boundary
// (compute_gradients + choose_scheme, ViscousFlux.cpp:15-148), Sutherland mu
// (field_structures.h:96-106), stresses and heat flux, stored as the nine
// distinct node fluxes txx tyy tzz txy txz tyz ex ey ez
// (compute_viscous_flux, ViscousFlux.cpp:151-208; F_v = (txx,txy,txz,ex),
// H_v = (txy,tyy,tyz,ey), G_v = (txz,tyz,tzz,ez)).
//
// Kernel 2 (viscous_div_kernel): rhs += D_x F_v + D_y H_v + D_z G_v with the
// same boundary orders (compute_vis_flux, ViscousFlux.cpp:210-255).  In
// periodic directions the stencil wraps to the interior node, which is what
// exchange_halos_viscous_flux (field_structures.h:877-932) copies into the
// ghosts; in non-periodic directions the orders keep the stencil inside.
#pragma once

#include "common.cuh"

namespace ns3d {

template <typename R>
struct ViscArgs {
    const R *W[5];          // primitives (padded layout)
    R *Rhs[5];              // RHS (padded layout)
    R *V[9];                // node fluxes, interior-only layout (k*ny + j)*nx + i
    Layout L;
    int periodic[3];
    R inv_h[3];             // 1/(2h), 1/(12h), 1/(60h) are formed from these
    R h[3];
    R Rgas, mu0, S, cp_over_pr;
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

template <typename R>
__device__ __forceinline__ R temp_at(const ViscArgs<R> &a, long id) {
    return a.W[4][id] / (a.W[0][id] * a.Rgas);  // T = p/(rho Rgas), field_structures.h:486
}

// All 12 derivatives at interior node (i,j,k) (ghost-inclusive indices).
template <typename R>
__device__ __forceinline__ void node_gradients(const ViscArgs<R> &a, int i, int j, int k, R g[12]) {
    const Layout &L = a.L;
    const int o[3] = {visc_order(i - NG, L.nx, a.periodic[0]), visc_order(j - NG, L.ny, a.periodic[1]),
                      visc_order(k - NG, L.nz, a.periodic[2])};
    const long stride[3] = {1, (long)L.px, (long)L.px * L.sy};
    const long c = L.at(i, j, k);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const long s = stride[d];
        const R h = a.h[d];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const R *f = a.W[1 + q];
            g[3 * q + d] = dstencil<R>([&](int off) { return f[c + off * s]; }, o[d], h);
        }
        g[9 + d] = dstencil<R>([&](int off) { return temp_at(a, c + off * s); }, o[d], h);
    }
}

template <typename R>
__global__ void __launch_bounds__(256) viscous_flux_kernel(ViscArgs<R> a) {
    const Layout &L = a.L;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= L.nx) return;
    R g[12];
    node_gradients(a, i + NG, j + NG, k + NG, g);
    const long c = L.at(i + NG, j + NG, k + NG);
    const R T = temp_at(a, c);
    // SolverParams::get_mu, field_structures.h:96-106
    const R mu = a.mu0 * pow(T, R(1.5)) * (R(1) + a.S) / (T + a.S);
    const R ux = g[0], uy = g[1], uz = g[2], vx = g[3], vy = g[4], vz = g[5];
    const R wx = g[6], wy = g[7], wz = g[8], Tx = g[9], Ty = g[10], Tz = g[11];
    const R div = ux + vy + wz;
    const R m2 = R(2) * mu, m23 = R(2.0 / 3.0) * mu * div;
    const R txx = m2 * ux - m23, tyy = m2 * vy - m23, tzz = m2 * wz - m23;
    const R txy = mu * (uy + vx), txz = mu * (uz + wx), tyz = mu * (vz + wy);
    const R kq = mu * a.cp_over_pr;
    const R u = a.W[1][c], v = a.W[2][c], w = a.W[3][c];
    const long o = ((long)k * L.ny + j) * L.nx + i;
    a.V[0][o] = txx; a.V[1][o] = tyy; a.V[2][o] = tzz;
    a.V[3][o] = txy; a.V[4][o] = txz; a.V[5][o] = tyz;
    a.V[6][o] = u * txx + v * txy + w * txz + kq * Tx;
    a.V[7][o] = u * txy + v * tyy + w * tyz + kq * Ty;
    a.V[8][o] = u * txz + v * tyz + w * tzz + kq * Tz;
}

template <typename R>
__global__ void __launch_bounds__(256) viscous_div_kernel(ViscArgs<R> a) {
    const Layout &L = a.L;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= L.nx) return;
    const int n[3] = {L.nx, L.ny, L.nz};
    const int p[3] = {i, j, k};
    int o[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) o[d] = visc_order(p[d], n[d], a.periodic[d]);
    // interior-layout index of the node shifted by off along d (wrapped if periodic)
    auto at = [&](int d, int off) -> long {
        int q[3] = {i, j, k};
        int x = q[d] + off;
        if (a.periodic[d]) { if (x < 0) x += n[d]; else if (x >= n[d]) x -= n[d]; }
        q[d] = x;
        return ((long)q[2] * L.ny + q[1]) * L.nx + q[0];
    };
    auto D = [&](int comp, int d) -> R {
        const R *f = a.V[comp];
        return dstencil<R>([&](int off) { return f[at(d, off)]; }, o[d], a.h[d]);
    };
    const long c = L.at(i + NG, j + NG, k + NG);
    // momentum x: F_v momx = txx, H_v momx = txy, G_v momx = txz
    R r = a.Rhs[1][c]; r += D(0, 0); r += D(3, 1); r += D(4, 2); a.Rhs[1][c] = r;
    r = a.Rhs[2][c]; r += D(3, 0); r += D(1, 1); r += D(5, 2); a.Rhs[2][c] = r;
    r = a.Rhs[3][c]; r += D(4, 0); r += D(5, 1); r += D(2, 2); a.Rhs[3][c] = r;
    r = a.Rhs[4][c]; r += D(6, 0); r += D(7, 1); r += D(8, 2); a.Rhs[4][c] = r;
}

}  // namespace ns3d
