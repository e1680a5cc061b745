// sweep.cuh -- fused inviscid sweep along one direction.
//
// One kernel per direction performs, for every interior line of the domain:
//   primitive -> conserved conversion (field_structures.h:468-488),
//   WCNS interpolation to the half nodes and the Riemann flux
//     (compute_invis_flux / WCNS_Riemann_InviscidFlux, InviscousFlux.cpp:10-268),
//   the half-node ghost faces (apply_boundary_halfnode_flux, boundary.cpp:207-300),
//   the 6th-order half-node difference accumulated into the RHS
//     (compute_invis_dflux, InviscousFlux.cpp:990-1056).
//
// A thread block owns a bundle of lines and marches along them in chunks of C
// faces.  Conserved cells and face fluxes live in shared-memory rings, so each
// cell is loaded and converted once and each face flux is computed once per
// line (plus a 5-face halo at the line ends).  In periodic directions the
// wrapped faces are computed from wrapped cells (identical inputs, identical
// values to the reference's face exchange); in non-periodic directions the
// ghost faces are the Outflow copies or zero, as the reference leaves them.
//
// Thread mapping keeps global accesses coalesced: along x the 32 lanes of a
// warp march along the line; along y and z the lanes span 32 neighbouring
// x-lines and the warps march.
#pragma once

#include "common.cuh"
#include "schemes.cuh"

namespace ns3d {

template <typename R>
struct SweepArgs {
    const R *W[5];      // primitives rho,u,v,w,p (padded layout)
    R *Rhs[5];          // right-hand side (padded layout)
    Layout L;
    int periodic;       // this direction
    int outflow_lo, outflow_hi;  // ghost faces copy the boundary face (else zero)
    R inv_h;            // 1/dx of this direction
    SchemeParams<R> sp;
    int first;          // 1: write -d (first direction), 0: accumulate
};

template <int DIR>
struct SweepGeom {
    static constexpr int C = DIR == 0 ? 32 : 8;        // faces per chunk
    static constexpr int NLINE = DIR == 0 ? 8 : 32;    // lines per block
    static constexpr int RING = DIR == 0 ? 64 : 16;    // ring length (power of 2, > C+4)
    static constexpr int SIZE = NLINE * RING;
    __device__ __forceinline__ static int sidx(int line, int r) {
        return DIR == 0 ? line * RING + (r & (RING - 1)) : (r & (RING - 1)) * NLINE + line;
    }
};

template <typename R>
__device__ __forceinline__ void load_conserved(const SweepArgs<R> &a, long id, R *U, R *W) {
    R r = a.W[0][id], u = a.W[1][id], v = a.W[2][id], w = a.W[3][id], p = a.W[4][id];
    if constexpr (sizeof(R) == 8) {
        p2c_exact(r, u, v, w, p, a.sp.gamma, U);
    } else {
        p2c_f(r, u, v, w, p, a.sp.gamma - 1.f, U);
    }
    W[0] = r <= R(0) ? R(1e-12) : r; W[1] = u; W[2] = v; W[3] = w; W[4] = p;
}

template <int DIR, typename R, int INTERP, int RS, int CHAR>
__global__ void __launch_bounds__(256)
sweep_kernel(SweepArgs<R> a) {
    using G = SweepGeom<DIR>;
    constexpr int C = G::C;
    constexpr bool USE_W = (CHAR != 0);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R (*sU)[G::SIZE] = reinterpret_cast<R (*)[G::SIZE]>(smem_raw);
    R (*sF)[G::SIZE] = sU + 5;
    R (*sW)[G::SIZE] = sU + 10;  // only with characteristic interpolation

    const Layout &L = a.L;
    const int slot = DIR == 0 ? threadIdx.x : threadIdx.y;
    const int line = DIR == 0 ? threadIdx.y : threadIdx.x;
    // tangential coordinates of this thread's line (interior indices + NG)
    int ta, tb;
    bool line_ok;
    if (DIR == 0) { ta = blockIdx.x * G::NLINE + line; tb = blockIdx.y; line_ok = ta < L.ny; }
    else if (DIR == 1) { ta = blockIdx.x * G::NLINE + line; tb = blockIdx.y; line_ok = ta < L.nx; }
    else { ta = blockIdx.x * G::NLINE + line; tb = blockIdx.y; line_ok = ta < L.nx; }
    ta += NG; tb += NG;
    const int n = DIR == 0 ? L.nx : (DIR == 1 ? L.ny : L.nz);
    // address of cell c (march coordinate, with ghosts) of this line
    auto cell_id = [&](int c) -> long {
        if (DIR == 0) return L.at(c, ta, tb);
        if (DIR == 1) return L.at(ta, c, tb);
        return L.at(ta, tb, c);
    };
    const bool per = a.periodic != 0;
    const int fb = per ? 0 : NG - 1;           // first face computed from cells
    const int fe = per ? n + 5 : n + NG;       // one past the last
    const int cell_end = per ? n + 8 : n + 6;  // one past the last cell needed
    int loaded = fb - 2;

    const bool char_rt = CHAR == RUNTIME ? (a.sp.char_recon != 0) : (CHAR != 0);

    for (int fc = fb; fc < fe; fc += C) {
        // ---- stage the cells needed by faces [fc, fc+C): cells up to fc+C+2
        const int need = min(fc + C + 3, cell_end);
        for (int c = loaded + slot; c < need; c += C) {
            if (line_ok) {
                int cc = c;
                if (per) { if (cc < NG) cc += n; else if (cc >= n + NG) cc -= n; }
                R U[5], W[5];
                load_conserved(a, cell_id(cc), U, W);
                const int s = G::sidx(line, c);
#pragma unroll
                for (int q = 0; q < 5; ++q) sU[q][s] = U[q];
                if (USE_W && char_rt) {
#pragma unroll
                    for (int q = 0; q < 5; ++q) sW[q][s] = W[q];
                }
            }
        }
        loaded = need;
        __syncthreads();
        // ---- face flux of face f (between cells f and f+1): cells f-2 .. f+3
        const int f = fc + slot;
        if (line_ok && f < fe) {
            R st[5][6];
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                const int s = G::sidx(line, f - 2 + m);
#pragma unroll
                for (int q = 0; q < 5; ++q) st[q][m] = sU[q][s];
            }
            R wi[5], wi1[5];
            if (USE_W && char_rt) {
                const int s0 = G::sidx(line, f), s1 = G::sidx(line, f + 1);
#pragma unroll
                for (int q = 0; q < 5; ++q) { wi[q] = sW[q][s0]; wi1[q] = sW[q][s1]; }
            }
            R F[5];
            wcns_face<DIR, R, INTERP, RS, CHAR>(a.sp, st, wi, wi1, F);
            const int s = G::sidx(line, f);
#pragma unroll
            for (int q = 0; q < 5; ++q) sF[q][s] = F[q];
        }
        __syncthreads();
        // ---- cells whose six faces (c-3 .. c+2) are now available
        const bool last = fc + C >= fe;
        const int c_lo = max(fc - 2, NG);
        const int c_hi = last ? n + NG : min(fc + C - 2, n + NG);
        for (int c = c_lo + slot; c < c_hi; c += C) {
            if (!line_ok) continue;
            R fv[5][6];
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                int ff = c - 3 + m;
                bool zero = false;
                if (!per) {
                    if (ff < NG - 1) { if (a.outflow_lo) ff = NG - 1; else zero = true; }
                    else if (ff > n + NG - 1) { if (a.outflow_hi) ff = n + NG - 1; else zero = true; }
                }
                const int s = G::sidx(line, ff);
#pragma unroll
                for (int q = 0; q < 5; ++q) fv[q][m] = zero ? R(0) : sF[q][s];
            }
            const long id = cell_id(c);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                // diff_6th_central_half, InviscousFlux.cpp:990-992
                R d = ((fv[q][3] - fv[q][2]) * R(75.0 / 64.0) + (fv[q][4] - fv[q][1]) * R(-25.0 / 384.0) +
                       (fv[q][5] - fv[q][0]) * R(3.0 / 640.0)) * a.inv_h;
                if (a.first) a.Rhs[q][id] = R(0) - d;
                else a.Rhs[q][id] = a.Rhs[q][id] - d;
            }
        }
    }
}

template <int DIR, typename R, int INTERP, int RS, int CHAR>
inline cudaError_t launch_sweep(const SweepArgs<R> &a, cudaStream_t st) {
    using G = SweepGeom<DIR>;
    dim3 block(DIR == 0 ? G::C : G::NLINE, DIR == 0 ? G::NLINE : G::C);
    dim3 grid;
    if (DIR == 0) grid = dim3((a.L.ny + G::NLINE - 1) / G::NLINE, a.L.nz);
    else if (DIR == 1) grid = dim3((a.L.nx + G::NLINE - 1) / G::NLINE, a.L.nz);
    else grid = dim3((a.L.nx + G::NLINE - 1) / G::NLINE, a.L.ny);
    const size_t smem = (size_t)(CHAR != 0 ? 15 : 10) * G::SIZE * sizeof(R);
    static unsigned configured = 0;  // one bit per device ordinal
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(configured & (1u << (dev & 31)))) {
        cudaError_t e = cudaFuncSetAttribute(sweep_kernel<DIR, R, INTERP, RS, CHAR>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured |= 1u << (dev & 31);
    }
    sweep_kernel<DIR, R, INTERP, RS, CHAR><<<grid, block, smem, st>>>(a);
    return cudaGetLastError();
}

// Dispatch entry points, one translation unit per direction (sweep_x/y/z.cu).
template <typename R>
cudaError_t sweep_dispatch(int dir, const SweepArgs<R> &a, cudaStream_t st);

cudaError_t sweep_x(const SweepArgs<double> &, cudaStream_t);
cudaError_t sweep_y(const SweepArgs<double> &, cudaStream_t);
cudaError_t sweep_z(const SweepArgs<double> &, cudaStream_t);
cudaError_t sweep_x(const SweepArgs<float> &, cudaStream_t);
cudaError_t sweep_y(const SweepArgs<float> &, cudaStream_t);
cudaError_t sweep_z(const SweepArgs<float> &, cudaStream_t);

// Specialised instantiations for the benchmark schemes, generic otherwise.
template <int DIR, typename R>
inline cudaError_t sweep_select(const SweepArgs<R> &a, cudaStream_t st) {
    const auto &sp = a.sp;
    if (!sp.char_recon) {
        if (sp.interp == I_WENO5 && sp.riemann == R_ROE) return launch_sweep<DIR, R, I_WENO5, R_ROE, 0>(a, st);
        if (sp.interp == I_MDCD_HYBRID && sp.riemann == R_HLLC)
            return launch_sweep<DIR, R, I_MDCD_HYBRID, R_HLLC, 0>(a, st);
        if (sp.interp == I_MDCD_LINEAR && sp.riemann == R_HLLC)
            return launch_sweep<DIR, R, I_MDCD_LINEAR, R_HLLC, 0>(a, st);
        return launch_sweep<DIR, R, RUNTIME, RUNTIME, 0>(a, st);
    }
    return launch_sweep<DIR, R, RUNTIME, RUNTIME, 1>(a, st);
}

}  // namespace ns3d
