// adjoint.cu -- adjoint (VJP) kernels of the RHS and of the RK3 stage update,
// plain FP64 path, periodic domains.
//
// All adjoint arrays use the interior layout (k*ny + j)*nx + i: with periodic
// boundaries every ghost value is a copy of an interior value, so the ghost
// fill's adjoint is the periodic wrap of the stencils.
//
// RHS adjoint = inviscid part per direction (face-flux VJPs through the
// transposed 6th-order half-node difference, then a gather of the six face
// contributions of each cell, deterministic) + viscous part (transposed
// divergence stencils -> pointwise VJP of the node flux -> transposed gradient
// stencils -> chain rule through u = m/rho, T = p/(rho Rgas)).
#include <cuda_runtime.h>

#include <type_traits>

#include "adjoint.cuh"
#include "adjoint_api.cuh"
#include "common.cuh"
#include "schemes.cuh"

namespace ns3d {

namespace {

constexpr double C1 = 75.0 / 64.0, C3 = -25.0 / 384.0, C5 = 3.0 / 640.0;
// 6th-order central first-derivative weights for offsets -3..3 (ViscousFlux.cpp:27-29)
__device__ __constant__ double D6[7] = {-1.0 / 60.0, 9.0 / 60.0, -45.0 / 60.0, 0.0, 45.0 / 60.0, -9.0 / 60.0,
                                        1.0 / 60.0};

__device__ __forceinline__ int wrapn(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

struct Idx {
    int nx, ny, nz;
    __device__ __forceinline__ long at(int i, int j, int k) const { return ((long)k * ny + j) * nx + i; }
};

// interior (i,j,k) shifted by o along d, periodic
__device__ __forceinline__ long shifted(const Idx &I, int i, int j, int k, int d, int o) {
    if (d == 0) i = wrapn(i + o, I.nx);
    else if (d == 1) j = wrapn(j + o, I.ny);
    else k = wrapn(k + o, I.nz);
    return I.at(i, j, k);
}

__device__ __forceinline__ void cons_at(const AdjArgs &a, int i, int j, int k, double U[5]) {
    const long c = a.L.at(i + NG, j + NG, k + NG);
    p2c_exact(a.W[0][c], a.W[1][c], a.W[2][c], a.W[3][c], a.W[4][c], a.gamma, U);
}

// ---------------------------------------------------------------- inviscid

// One thread per face.  The stencil and the face states are staged in the
// thread's own shared-memory column, so the per-variable interpolation
// passes run as rolled loops without local-memory arrays; the Riemann VJP
// (all five variables coupled) runs in registers in between.
constexpr int ADJ_T = 128;

template <int DIR, int INTERP, int RS>
__global__ void __launch_bounds__(ADJ_T) adj_face_kernel(AdjArgs a) {
    __shared__ double sSt[30][ADJ_T];  // conserved stencil, row q*6 + m
    __shared__ double sLR[10][ADJ_T];  // UL, UR; then their adjoints
    const int tid = threadIdx.x;
    const Idx I{a.L.nx, a.L.ny, a.L.nz};
    const long nface = (long)I.nx * I.ny * I.nz;
    const long t = (long)blockIdx.x * blockDim.x + tid;
    if (t >= nface) return;
    const int i = (int)(t % I.nx), j = (int)((t / I.nx) % I.ny), k = (int)(t / ((long)I.nx * I.ny));
    // face j' + 1/2 along DIR with j' = the cell coordinate along DIR
    const double ih = a.inv_h[DIR];
    double Fb[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const double *r = a.Rb[q];
        auto R = [&](int o) { return r[shifted(I, i, j, k, DIR, o)]; };
        Fb[q] = -ih * a.rbs * (C1 * (R(0) - R(1)) + C3 * (R(-1) - R(2)) + C5 * (R(-2) - R(3)));
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        int ii = i, jj = j, kk = k;
        if (DIR == 0) ii = wrapn(i + m - 2, I.nx);
        else if (DIR == 1) jj = wrapn(j + m - 2, I.ny);
        else kk = wrapn(k + m - 2, I.nz);
        double Uc[5];
        cons_at(a, ii, jj, kk, Uc);
#pragma unroll
        for (int q = 0; q < 5; ++q) sSt[q * 6 + m][tid] = Uc[q];
    }
    // forward interpolation, one variable at a time
#pragma unroll 1
    for (int q = 0; q < 5; ++q) {
        double f[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) f[m] = sSt[q * 6 + m][tid];
        double l, r;
        adj::interp_pair_fwd<double, INTERP>(f, a.lin, a.hd, l, r);
        sLR[q][tid] = l;
        sLR[5 + q][tid] = r;
    }
    double UL[5], UR[5], ULb[5] = {0, 0, 0, 0, 0}, URb[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int q = 0; q < 5; ++q) { UL[q] = sLR[q][tid]; UR[q] = sLR[5 + q][tid]; }
    adj::riemann_vjp<DIR, double, RS>(UL, UR, a.gamma, Fb, ULb, URb);
#pragma unroll
    for (int q = 0; q < 5; ++q) { sLR[q][tid] = ULb[q]; sLR[5 + q][tid] = URb[q]; }
    // interpolation VJP, one variable at a time, straight into the face store
#pragma unroll 1
    for (int q = 0; q < 5; ++q) {
        double f[6], gb[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) f[m] = sSt[q * 6 + m][tid];
        const double lb = sLR[q][tid], rb = sLR[5 + q][tid];
        adj::interp_pair_vjp<double, INTERP>(f, a.lin, a.hd, lb, rb, gb);
#pragma unroll
        for (int m = 0; m < 6; ++m) a.G[m * 5 + q][t] = gb[m];
    }
}

// Whole periodic lines in one block (line length n <= 256): the block
// converts its cells once, computes the face VJPs of the line (same
// arithmetic as adj_face_kernel) into shared memory and gathers them, in
// the same order as adj_face_gather_kernel, so the per-face store never
// reaches global memory.  lpb lines per block; threads = lpb * n.
template <int DIR, int INTERP, int RS>
__global__ void __launch_bounds__(256) adj_line_kernel(AdjArgs a, int lpb, int first) {
    extern __shared__ __align__(16) double smem_adj[];
    const Idx I{a.L.nx, a.L.ny, a.L.nz};
    const int n = DIR == 0 ? I.nx : (DIR == 1 ? I.ny : I.nz);
    const int T = lpb * n;
    double *sU = smem_adj, *sR = sU + 5 * T, *sG = sR + 5 * T, *sLR = sG + 30 * T;
    const int l = DIR == 0 ? threadIdx.y : threadIdx.x;
    const int c = DIR == 0 ? threadIdx.x : threadIdx.y;
    // [line][pos] along x, [pos][line] across lines: warps read contiguous words
    auto sidx = [&](int cc) { return DIR == 0 ? l * n + cc : cc * lpb + l; };
    auto at = [&](int cc) { return sidx(wrapn(cc, n)); };
    const int tid = sidx(c);
    const long nlines = DIR == 0 ? (long)I.ny * I.nz : (DIR == 1 ? (long)I.nx * I.nz : (long)I.nx * I.ny);
    const long g = (long)blockIdx.x * lpb + l;
    const bool ok = g < nlines;
    int i, j, k;
    if (DIR == 0) { i = c; j = (int)(g % I.ny); k = (int)(g / I.ny); }
    else if (DIR == 1) { i = (int)(g % I.nx); j = c; k = (int)(g / I.nx); }
    else { i = (int)(g % I.nx); j = (int)(g / I.nx); k = c; }
    const long tc = ok ? I.at(i, j, k) : 0;
    if (ok) {
        double Uc[5];
        cons_at(a, i, j, k, Uc);
#pragma unroll
        for (int q = 0; q < 5; ++q) { sU[q * T + tid] = Uc[q]; sR[q * T + tid] = a.rbs * a.Rb[q][tc]; }
    }
    __syncthreads();
    if (ok) {
        // face c + 1/2
        const double ih = a.inv_h[DIR];
        double Fb[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            auto R = [&](int o) { return sR[q * T + at(c + o)]; };
            Fb[q] = -ih * (C1 * (R(0) - R(1)) + C3 * (R(-1) - R(2)) + C5 * (R(-2) - R(3)));
        }
#pragma unroll 1
        for (int q = 0; q < 5; ++q) {
            double f[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) f[m] = sU[q * T + at(c - 2 + m)];
            double lv, rv;
            adj::interp_pair_fwd<double, INTERP>(f, a.lin, a.hd, lv, rv);
            sLR[q * T + tid] = lv;
            sLR[(5 + q) * T + tid] = rv;
        }
        double UL[5], UR[5], ULb[5] = {0, 0, 0, 0, 0}, URb[5] = {0, 0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < 5; ++q) { UL[q] = sLR[q * T + tid]; UR[q] = sLR[(5 + q) * T + tid]; }
        adj::riemann_vjp<DIR, double, RS>(UL, UR, a.gamma, Fb, ULb, URb);
#pragma unroll
        for (int q = 0; q < 5; ++q) { sLR[q * T + tid] = ULb[q]; sLR[(5 + q) * T + tid] = URb[q]; }
#pragma unroll 1
        for (int q = 0; q < 5; ++q) {
            double f[6], gb[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) f[m] = sU[q * T + at(c - 2 + m)];
            const double lb = sLR[q * T + tid], rb = sLR[(5 + q) * T + tid];
            adj::interp_pair_vjp<double, INTERP>(f, a.lin, a.hd, lb, rb, gb);
#pragma unroll
            for (int m = 0; m < 6; ++m) sG[(m * 5 + q) * T + tid] = gb[m];
        }
    }
    __syncthreads();
    if (ok) {
        // cell c gathers the m-th contribution of face c - m + 2
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            double s = first ? 0.0 : a.Ub[q][tc];
#pragma unroll
            for (int m = 0; m < 6; ++m) s += sG[(m * 5 + q) * T + at(c + 2 - m)];
            a.Ub[q][tc] = s;
        }
    }
}

template <int DIR, int INTERP, int RS>
cudaError_t launch_line(const AdjArgs &a, int first, cudaStream_t st) {
    const int n = DIR == 0 ? a.L.nx : (DIR == 1 ? a.L.ny : a.L.nz);
    const int lpb = n <= 128 ? 128 / n : 1;
    const long nlines = DIR == 0 ? (long)a.L.ny * a.L.nz : (DIR == 1 ? (long)a.L.nx * a.L.nz : (long)a.L.nx * a.L.ny);
    const size_t smem = (size_t)50 * lpb * n * sizeof(double);
    static unsigned configured = 0;  // one bit per device ordinal
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(configured & (1u << (dev & 31)))) {
        cudaError_t e = cudaFuncSetAttribute(adj_line_kernel<DIR, INTERP, RS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 50 * 256 * 8);
        if (e != cudaSuccess) return e;
        configured |= 1u << (dev & 31);
    }
    dim3 block(DIR == 0 ? n : lpb, DIR == 0 ? lpb : n);
    adj_line_kernel<DIR, INTERP, RS><<<(unsigned)((nlines + lpb - 1) / lpb), block, smem, st>>>(a, lpb, first);
    return cudaGetLastError();
}

// cell c gathers m-th stencil contributions of faces c - m + 2
template <int DIR>
__global__ void __launch_bounds__(128) adj_face_gather_kernel(AdjArgs a, int first) {
    const Idx I{a.L.nx, a.L.ny, a.L.nz};
    const long ncell = (long)I.nx * I.ny * I.nz;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell) return;
    const int i = (int)(t % I.nx), j = (int)((t / I.nx) % I.ny), k = (int)(t / ((long)I.nx * I.ny));
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        double s = first ? 0.0 : a.Ub[q][t];
#pragma unroll
        for (int m = 0; m < 6; ++m) s += a.G[m * 5 + q][shifted(I, i, j, k, DIR, 2 - m)];
        a.Ub[q][t] = s;
    }
}

// ---------------------------------------------------------------- viscous

// primitives (u, v, w, T) at interior node
__device__ __forceinline__ void prim4(const AdjArgs &a, int i, int j, int k, double x[4]) {
    const long c = a.L.at(i + NG, j + NG, k + NG);
    x[0] = a.W[1][c]; x[1] = a.W[2][c]; x[2] = a.W[3][c];
    x[3] = a.W[4][c] / (a.W[0][c] * a.Rgas);
}

__global__ void __launch_bounds__(128) adj_visc_node_kernel(AdjArgs a) {
    const Idx I{a.L.nx, a.L.ny, a.L.nz};
    const long ncell = (long)I.nx * I.ny * I.nz;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell) return;
    const int i = (int)(t % I.nx), j = (int)((t / I.nx) % I.ny), k = (int)(t / ((long)I.nx * I.ny));
    // node-flux adjoint: transpose of D_d (antisymmetric) applied to rhs adjoints
    auto DT = [&](const double *r, int d) {
        double s = 0.0;
#pragma unroll
        for (int o = -3; o <= 3; ++o) s += D6[o + 3] * r[shifted(I, i, j, k, d, -o)];
        return s * (a.inv_h[d] * a.rbs);
    };
    double Vb[9];
    Vb[0] = DT(a.Rb[1], 0);                    // txx: x-term of rhou
    Vb[1] = DT(a.Rb[2], 1);                    // tyy: y-term of rhov
    Vb[2] = DT(a.Rb[3], 2);                    // tzz: z-term of rhow
    Vb[3] = DT(a.Rb[2], 0) + DT(a.Rb[1], 1);   // txy
    Vb[4] = DT(a.Rb[3], 0) + DT(a.Rb[1], 2);   // txz
    Vb[5] = DT(a.Rb[3], 1) + DT(a.Rb[2], 2);   // tyz
    Vb[6] = DT(a.Rb[4], 0);                    // ex
    Vb[7] = DT(a.Rb[4], 1);                    // ey
    Vb[8] = DT(a.Rb[4], 2);                    // ez
    double x[4];
    prim4(a, i, j, k, x);
    double g[4][3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double s[4] = {0, 0, 0, 0};
#pragma unroll
        for (int o = -3; o <= 3; ++o) {
            if (o == 0) continue;
            int ii = i, jj = j, kk = k;
            if (d == 0) ii = wrapn(i + o, I.nx); else if (d == 1) jj = wrapn(j + o, I.ny); else kk = wrapn(k + o, I.nz);
            double y[4];
            prim4(a, ii, jj, kk, y);
#pragma unroll
            for (int q = 0; q < 4; ++q) s[q] += D6[o + 3] * y[q];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) g[q][d] = s[q] * a.inv_h[d];
    }
    double xb[4] = {0, 0, 0, 0}, gb[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    adj::visc_flux_vjp<double>(a.mu0, a.S, a.cpr, x, g, Vb, xb, gb);
#pragma unroll
    for (int q = 0; q < 4; ++q) a.X[q][t] = xb[q];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int d = 0; d < 3; ++d) a.X[4 + 3 * q + d][t] = gb[q][d];
}

__global__ void __launch_bounds__(128) adj_visc_gather_kernel(AdjArgs a) {
    const Idx I{a.L.nx, a.L.ny, a.L.nz};
    const long ncell = (long)I.nx * I.ny * I.nz;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell) return;
    const int i = (int)(t % I.nx), j = (int)((t / I.nx) % I.ny), k = (int)(t / ((long)I.nx * I.ny));
    double xb[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double s = a.X[q][t];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double *gbar = a.X[4 + 3 * q + d];
            double acc = 0.0;
#pragma unroll
            for (int o = -3; o <= 3; ++o) acc += D6[o + 3] * gbar[shifted(I, i, j, k, d, -o)];
            s += acc * a.inv_h[d];
        }
        xb[q] = s;
    }
    // chain rule u = m/rho, T = (g-1)(E - |m|^2/(2 rho)) / (rho Rgas)
    const long c = a.L.at(i + NG, j + NG, k + NG);
    const double rho = a.W[0][c], u = a.W[1][c], v = a.W[2][c], w = a.W[3][c], p = a.W[4][c];
    const double gm1 = a.gamma - 1.0;
    const double E = p / gm1 + 0.5 * rho * (u * u + v * v + w * w);
    const double irR = 1.0 / (rho * a.Rgas);
    a.Ub[0][t] += -(u * xb[0] + v * xb[1] + w * xb[2]) / rho + xb[3] * gm1 * irR * (u * u + v * v + w * w - E / rho);
    a.Ub[1][t] += xb[0] / rho - xb[3] * gm1 * u * irR;
    a.Ub[2][t] += xb[1] / rho - xb[3] * gm1 * v * irR;
    a.Ub[3][t] += xb[2] / rho - xb[3] * gm1 * w * irR;
    a.Ub[4][t] += xb[3] * gm1 * irR;
}

// ---------------------------------------------------------------- pointwise

__global__ void axpby_kernel(double *const *y, const double *const *x, double alpha, double beta, long n) {
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
#pragma unroll
        for (int q = 0; q < 5; ++q) y[q][t] = beta * y[q][t] + alpha * x[q][t];
}

__global__ void ke_seed_kernel(AdjArgs a, double vol, double *const *Ub) {
    const Idx I{a.L.nx, a.L.ny, a.L.nz};
    const long ncell = (long)I.nx * I.ny * I.nz;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % I.nx), j = (int)((t / I.nx) % I.ny), k = (int)(t / ((long)I.nx * I.ny));
        const long c = a.L.at(i + NG, j + NG, k + NG);
        const double u = a.W[1][c], v = a.W[2][c], w = a.W[3][c];
        // J = sum 0.5 |m|^2 / rho * vol (postprocess.cpp:119-122)
        Ub[0][t] = -0.5 * (u * u + v * v + w * w) * vol;
        Ub[1][t] = u * vol; Ub[2][t] = v * vol; Ub[3][t] = w * vol;
        Ub[4][t] = 0.0;
    }
}

// conserved adjoint -> adjoint of the initial velocity at fixed rho and p
__global__ void velocity_grad_kernel(AdjArgs a, const double *const *Ub, double *const *gvel) {
    const Idx I{a.L.nx, a.L.ny, a.L.nz};
    const long ncell = (long)I.nx * I.ny * I.nz;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % I.nx), j = (int)((t / I.nx) % I.ny), k = (int)(t / ((long)I.nx * I.ny));
        const long c = a.L.at(i + NG, j + NG, k + NG);
        const double rho = a.W[0][c];
        for (int q = 0; q < 3; ++q) gvel[q][t] = rho * Ub[1 + q][t] + rho * a.W[1 + q][c] * Ub[4][t];
    }
}

int blocks_for(long n, int t) { return (int)((n + t - 1) / t); }

// tab[5*slot + q]: slot 0 UB (adjoint of the step's result / of its input),
// 1 ACC, 2 SB, 3 RB
__global__ void step_combine_kernel(int which, double *const *tab, double dt, long n) {
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            double *UB = tab[q], *ACC = tab[5 + q], *SB = tab[10 + q], *RB = tab[15 + q];
            if (which == 1) {
                const double u = UB[t];
                ACC[t] = u * (1.0 / 3.0);
                SB[t] = u * (2.0 / 3.0);
            } else if (which == 2) {
                const double sb = SB[t], s4 = 0.25 * sb;
                ACC[t] += 0.75 * sb;
                SB[t] = s4;
                RB[t] = dt * s4;
            } else {
                UB[t] = ACC[t] + SB[t];
            }
        }
}

}  // namespace

cudaError_t adj_rhs_vjp(const AdjArgs &a, cudaStream_t st, long *launches) {
    const long n = (long)a.L.nx * a.L.ny * a.L.nz;
    const int nb = blocks_for(n, 128);
    // riemann_vjp codes: 0 Roe, 1 Rusanov, 2 HLL, 3 HLLC (from the public value)
    const int rs = adj::adj_riemann_code(a.riemann);
    auto face = [&](auto dir_tag) {
        constexpr int D = decltype(dir_tag)::value;
        auto go = [&](auto it) {
            constexpr int I = decltype(it)::value;
            if (rs == 0) adj_face_kernel<D, I, 0><<<nb, 128, 0, st>>>(a);
            else if (rs == 1) adj_face_kernel<D, I, 1><<<nb, 128, 0, st>>>(a);
            else if (rs == 2) adj_face_kernel<D, I, 2><<<nb, 128, 0, st>>>(a);
            else adj_face_kernel<D, I, 3><<<nb, 128, 0, st>>>(a);
        };
        if (a.interp == 0) go(std::integral_constant<int, 0>{});
        else if (a.interp == 2) go(std::integral_constant<int, 2>{});
        else go(std::integral_constant<int, 3>{});
    };
    auto line = [&](auto dir_tag, int first) -> cudaError_t {
        constexpr int D = decltype(dir_tag)::value;
        auto go = [&](auto it) -> cudaError_t {
            constexpr int I = decltype(it)::value;
            if (rs == 0) return launch_line<D, I, 0>(a, first, st);
            if (rs == 1) return launch_line<D, I, 1>(a, first, st);
            if (rs == 2) return launch_line<D, I, 2>(a, first, st);
            return launch_line<D, I, 3>(a, first, st);
        };
        if (a.interp == 0) return go(std::integral_constant<int, 0>{});
        if (a.interp == 2) return go(std::integral_constant<int, 2>{});
        return go(std::integral_constant<int, 3>{});
    };
    const bool fused = a.L.nx <= 256 && a.L.ny <= 256 && a.L.nz <= 256;
    if (fused) {
        cudaError_t e;
        if ((e = line(std::integral_constant<int, 0>{}, a.first)) != cudaSuccess) return e;
        if ((e = line(std::integral_constant<int, 1>{}, 0)) != cudaSuccess) return e;
        if ((e = line(std::integral_constant<int, 2>{}, 0)) != cudaSuccess) return e;
        *launches += 3;
    } else {
        face(std::integral_constant<int, 0>{});
        adj_face_gather_kernel<0><<<nb, 128, 0, st>>>(a, a.first);
        face(std::integral_constant<int, 1>{});
        adj_face_gather_kernel<1><<<nb, 128, 0, st>>>(a, 0);
        face(std::integral_constant<int, 2>{});
        adj_face_gather_kernel<2><<<nb, 128, 0, st>>>(a, 0);
        *launches += 6;
    }
    if (a.mu0 != 0.0) {
        adj_visc_node_kernel<<<nb, 128, 0, st>>>(a);
        adj_visc_gather_kernel<<<nb, 128, 0, st>>>(a);
        *launches += 2;
    }
    return cudaGetLastError();
}

cudaError_t adj_axpby(double *const *y, const double *const *x, double alpha, double beta, long n, cudaStream_t st) {
    axpby_kernel<<<blocks_for(n, 256) < 4096 ? blocks_for(n, 256) : 4096, 256, 0, st>>>(y, x, alpha, beta, n);
    return cudaGetLastError();
}

cudaError_t adj_step_combine(int which, double *const *tab, double dt, long n, cudaStream_t st) {
    step_combine_kernel<<<blocks_for(n, 256) < 4096 ? blocks_for(n, 256) : 4096, 256, 0, st>>>(which, tab, dt, n);
    return cudaGetLastError();
}

cudaError_t adj_ke_seed(const AdjArgs &a, double vol, double *const *Ub, cudaStream_t st) {
    const long n = (long)a.L.nx * a.L.ny * a.L.nz;
    ke_seed_kernel<<<blocks_for(n, 256) < 4096 ? blocks_for(n, 256) : 4096, 256, 0, st>>>(a, vol, Ub);
    return cudaGetLastError();
}

cudaError_t adj_velocity_grad(const AdjArgs &a, const double *const *Ub, double *const *gvel, cudaStream_t st) {
    const long n = (long)a.L.nx * a.L.ny * a.L.nz;
    velocity_grad_kernel<<<blocks_for(n, 256) < 4096 ? blocks_for(n, 256) : 4096, 256, 0, st>>>(a, Ub, gvel);
    return cudaGetLastError();
}

}  // namespace ns3d

// ------------------------------------------------- host evaluation for tests

namespace ns3d {
template <int DIR>
void riemann_flux_host(const SchemeParams<double> &sp, const double *UL, const double *UR, double *F) {
    riemann<DIR, double, RUNTIME>(sp, UL, UR, F);
}
}  // namespace ns3d

extern "C" int ns3d_debug_face_vjp(int direction, int interpolation, int riemann, double gamma,
                                   const double *lin, const double *U30, const double *Fbar5, double *out30,
                                   double *flux5) {
    using namespace ns3d;
    if (!U30 || !Fbar5 || !out30 || direction < 0 || direction > 2) return -1;
    if (interpolation != 0 && interpolation != 2 && interpolation != 3) return -2;
    if (interpolation != 0 && !lin) return -1;
    const int rs = adj::adj_riemann_code(riemann);
    if (rs < 0) return -2;
    double U[5][6], Ub[5][6] = {};
    for (int q = 0; q < 5; ++q)
        for (int m = 0; m < 6; ++m) U[q][m] = U30[q * 6 + m];
    const double zero6[6] = {0, 0, 0, 0, 0, 0};
    const double *li = lin ? lin : zero6, *hd = interpolation == 3 ? lin + 6 : zero6;
    if (direction == 0) adj::face_vjp<0, double>(interpolation, rs, li, hd, gamma, U, Fbar5, Ub);
    else if (direction == 1) adj::face_vjp<1, double>(interpolation, rs, li, hd, gamma, U, Fbar5, Ub);
    else adj::face_vjp<2, double>(interpolation, rs, li, hd, gamma, U, Fbar5, Ub);
    for (int q = 0; q < 5; ++q)
        for (int m = 0; m < 6; ++m) out30[q * 6 + m] = Ub[q][m];
    if (flux5) {
        // forward face flux with the production functions (schemes.cuh)
        SchemeParams<double> sp;
        sp.gamma = gamma;
        for (int m = 0; m < 6; ++m) sp.lin[m] = li[m];
        for (int m = 0; m < 4; ++m) sp.hd[m] = interpolation == 3 ? hd[m] : 0.0;
        sp.interp = interpolation; sp.riemann = riemann; sp.char_recon = 0;
        double wi[5] = {0, 0, 0, 0, 0};
        if (direction == 0) wcns_face<0, double, RUNTIME, RUNTIME, 0>(sp, U, wi, wi, flux5);
        else if (direction == 1) wcns_face<1, double, RUNTIME, RUNTIME, 0>(sp, U, wi, wi, flux5);
        else wcns_face<2, double, RUNTIME, RUNTIME, 0>(sp, U, wi, wi, flux5);
    }
    return 0;
}

extern "C" int ns3d_debug_visc_vjp(double mu0, double S, double cpr, const double *x4, const double *g12,
                                   const double *Vbar9, double *xb4, double *gb12, double *V9) {
    using namespace ns3d;
    double g[4][3], gb[4][3] = {};
    for (int q = 0; q < 4; ++q)
        for (int d = 0; d < 3; ++d) g[q][d] = g12[3 * q + d];
    double xb[4] = {0, 0, 0, 0};
    adj::visc_flux_vjp<double>(mu0, S, cpr, x4, g, Vbar9, xb, gb);
    for (int q = 0; q < 4; ++q) xb4[q] = xb[q];
    for (int q = 0; q < 4; ++q)
        for (int d = 0; d < 3; ++d) gb12[3 * q + d] = gb[q][d];
    if (V9) adj::visc_flux_all<double>(mu0, S, cpr, x4, g, V9);
    return 0;
}

extern "C" int ns3d_debug_riemann(int direction, int riemann, double gamma, const double UL[5], const double UR[5],
                                  double F[5]) {
    using namespace ns3d;
    if (!UL || !UR || !F || direction < 0 || direction > 2 || riemann < 0 || riemann > 6) return -1;
    SchemeParams<double> sp;
    sp.gamma = gamma;
    for (int m = 0; m < 6; ++m) sp.lin[m] = 0.0;
    for (int m = 0; m < 4; ++m) sp.hd[m] = 0.0;
    sp.interp = 0; sp.riemann = riemann; sp.char_recon = 0;
    if (direction == 0) riemann_flux_host<0>(sp, UL, UR, F);
    else if (direction == 1) riemann_flux_host<1>(sp, UL, UR, F);
    else riemann_flux_host<2>(sp, UL, UR, F);
    return 0;
}
