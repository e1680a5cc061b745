// reduce.cuh -- block reductions for the global scalars (CFL time step,
// kinetic energy, dissipation) and the per-cell CFL bound.
#pragma once

#include "common.cuh"

namespace ns3d {

// Reduction kernels write one partial per block; a single-block kernel then
// combines the partials in a fixed order, so results are deterministic.
constexpr int RED_THREADS = 256;

template <int NV>
__device__ __forceinline__ void block_sum(double v[NV], double *partial_out) {
    __shared__ double sh[NV][RED_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0.0;
            for (int w = 0; w < RED_THREADS / 32; ++w) s += sh[q][w];
            partial_out[q] = s;
        }
    }
}

// Sums of v[0..NV) over a block of NT threads of any shape (NT a multiple of
// 32, every thread calling), in a fixed order; thread 0 writes them.
template <int NV, int NT>
__device__ __forceinline__ void block_sum_n(double v[NV], double *out) {
    __shared__ double sh[NV][NT / 32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[q][wid] = x;
    }
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0.0;
            for (int w = 0; w < NT / 32; ++w) s += sh[q][w];
            out[q] = s;
        }
    }
}

// Sums of s[0..NV) and maxima of m[0..NV) over a block of RED_THREADS
// threads, in a fixed order; thread 0 writes s then m (2 NV values).
template <int NV>
__device__ __forceinline__ void block_sum_max(double s[NV], double m[NV], double *partial_out) {
    __shared__ double sh[2 * NV][RED_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double x = s[q], y = m[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_down_sync(0xffffffffu, x, o);
            y = fmax(y, __shfl_down_sync(0xffffffffu, y, o));
        }
        if (lane == 0) { sh[q][wid] = x; sh[NV + q][wid] = y; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < RED_THREADS / 32; ++w) { a += sh[q][w]; b = fmax(b, sh[NV + q][w]); }
            partial_out[q] = a;
            partial_out[NV + q] = b;
        }
    }
}

__device__ __forceinline__ double block_min(double x, double *partial_out) {
    __shared__ double sh[RED_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_down_sync(0xffffffffu, x, o));
    if (lane == 0) sh[wid] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = sh[0];
        for (int w = 1; w < RED_THREADS / 32; ++w) m = fmin(m, sh[w]);
        *partial_out = m;
    }
    return x;
}

// Minimum over a block of NT threads (NT a multiple of 32, every thread
// calling); thread 0 writes it.
template <int NT>
__device__ __forceinline__ void block_min_n(double x, double *out) {
    __shared__ double sh[NT / 32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_down_sync(0xffffffffu, x, o));
    if (lane == 0) sh[wid] = x;
    __syncthreads();
    if (tid == 0) {
        double m = sh[0];
#pragma unroll
        for (int w = 1; w < NT / 32; ++w) m = fmin(m, sh[w]);
        *out = m;
    }
}

// Minimum of m and sum of v over a block of NT threads (NT a multiple of 32,
// every thread calling), in a fixed order; thread 0 writes both.
template <int NT>
__device__ __forceinline__ void block_min_sum_n(double m, double v, double *out_min, double *out_sum) {
    __shared__ double shm[NT / 32], shs[NT / 32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m = fmin(m, __shfl_down_sync(0xffffffffu, m, o));
        v += __shfl_down_sync(0xffffffffu, v, o);
    }
    if (lane == 0) { shm[wid] = m; shs[wid] = v; }
    __syncthreads();
    if (tid == 0) {
        double a = shm[0], b = shs[0];
#pragma unroll
        for (int w = 1; w < NT / 32; ++w) { a = fmin(a, shm[w]); b += shs[w]; }
        *out_min = a;
        *out_sum = b;
    }
}

// The CFL bound of a block from its largest wave speed: min_i fl(dx / s_i)
// equals fl(dx / max_i s_i) bit for bit (correctly rounded division by a
// positive speed is monotone; fmin and fmax both skip NaN), so the fused
// stage keeps max s per thread and divides once per block.  Capped at 1e9,
// the initial value of the per-cell minimum.  Thread 0 writes both results.
template <int NT>
__device__ __forceinline__ void block_speed_sum_n(double s, double v, double dx, double *out_min,
                                                  double *out_sum) {
    __shared__ double shm[NT / 32], shs[NT / 32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s = fmax(s, __shfl_down_sync(0xffffffffu, s, o));
        v += __shfl_down_sync(0xffffffffu, v, o);
    }
    if (lane == 0) { shm[wid] = s; shs[wid] = v; }
    __syncthreads();
    if (tid == 0) {
        double a = shm[0], b = shs[0];
#pragma unroll
        for (int w = 1; w < NT / 32; ++w) { a = fmax(a, shm[w]); b += shs[w]; }
        *out_min = fmin(1e9, dx / a);
        *out_sum = b;
    }
}

// Per-cell CFL bound of compute_timestep (timestep.cpp:12-20) from the FP64
// conserved state: u = rhou/rho, p = (gamma-1)(E - 0.5 rho u^2) (v, w are not
// used), a = sqrt(gamma p / rho), bound = dx / (|u| + a).
__device__ __forceinline__ double cfl_bound(const double U[5], double gamma, double dx) {
    double rho = U[0];
    double u = U[1] / rho;
    double p = __dmul_rn(gamma - 1., __dsub_rn(U[4], __dmul_rn(__dmul_rn(__dmul_rn(0.5, rho), u), u)));
    double a = sqrt(__dmul_rn(gamma, p) / rho);
    return dx / __dadd_rn(fabs(u), a);
}

// The wave speed |u| + a of cfl_bound (cfl_bound = dx / cfl_speed, same bits).
__device__ __forceinline__ double cfl_speed(const double U[5], double gamma) {
    double rho = U[0];
    double u = U[1] / rho;
    double p = __dmul_rn(gamma - 1., __dsub_rn(U[4], __dmul_rn(__dmul_rn(__dmul_rn(0.5, rho), u), u)));
    double a = sqrt(__dmul_rn(gamma, p) / rho);
    return __dadd_rn(fabs(u), a);
}

}  // namespace ns3d
