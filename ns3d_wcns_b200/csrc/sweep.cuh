// sweep.cuh -- fused inviscid + viscous sweep along one direction.
//
// One kernel per direction performs, for every interior line of the domain:
//   primitive -> conserved conversion (field_structures.h:468-488),
//   WCNS interpolation to the half nodes and the Riemann flux
//     (compute_invis_flux / WCNS_Riemann_InviscidFlux, InviscousFlux.cpp:10-268),
//   the half-node ghost faces (apply_boundary_halfnode_flux, boundary.cpp:207-300),
//   the 6th-order half-node difference (compute_invis_dflux, InviscousFlux.cpp:990-1056),
//   and this direction's term of the viscous divergence: the derivative of the
//   node viscous fluxes along the line with the reference's boundary orders
//   (compute_vis_flux, ViscousFlux.cpp:210-255),
// accumulated into the RHS.
//
// A thread block owns a bundle of lines and marches along them in chunks of C
// faces.  Conserved cells, viscous node fluxes and face fluxes live in
// shared-memory rings, so each cell is loaded and converted once and each face
// flux is computed once per line (plus a 5-face halo at the line ends).  The
// next chunk's cells and viscous fluxes, and the current chunk's old RHS
// values, are copied with cp.async while the face fluxes compute.  In periodic
// directions the wrapped faces are computed from wrapped cells (identical
// inputs, identical values to the reference's face exchange); in non-periodic
// directions the ghost faces are the Outflow copies or zero, as the reference
// leaves them.
//
// Thread mapping keeps global accesses coalesced: along x the 32 lanes of a
// warp march along the line; along y and z the lanes span 32 neighbouring
// x-lines and the warps march.
#pragma once

#include "common.cuh"
#include "schemes.cuh"
#include "viscous.cuh"

namespace ns3d {

template <typename R>
struct SweepArgs {
    const R *W[5];      // primitives rho,u,v,w,p (padded layout)
    R *Rhs[5];          // right-hand side (padded layout)
    const R *V[4];      // this direction's node viscous fluxes (interior layout)
                        // for rhou, rhov, rhow, E
    Layout L;
    int periodic;       // this direction
    int outflow_lo, outflow_hi;  // ghost faces copy the boundary face (else zero)
    R inv_h;            // 1/h of this direction
    R h;                // h (viscous stencils divide by k*h as the reference)
    SchemeParams<R> sp;
    int first;          // 1: write (first direction), 0: accumulate
    int visc;           // 1: add the viscous divergence term
};

template <int DIR>
struct SweepGeom {
    static constexpr int C = DIR == 0 ? 32 : 8;        // faces per chunk
    static constexpr int NLINE = DIR == 0 ? 8 : 32;    // lines per block
    static constexpr int RING = DIR == 0 ? 64 : 16;    // ring length (power of 2, >= C+8)
    static constexpr int SIZE = NLINE * RING;
    static constexpr int CH = C * NLINE;               // cells per chunk = threads
    __device__ __forceinline__ static int sidx(int line, int r) {
        return DIR == 0 ? line * RING + (r & (RING - 1)) : (r & (RING - 1)) * NLINE + line;
    }
    __device__ __forceinline__ static int tidx(int line, int slot) {
        return DIR == 0 ? line * C + slot : slot * NLINE + line;
    }
};

// rings U(5) F(5) V(4) [W(5) with characteristic bases], staging W(5)+V(4), old RHS(5)
template <int DIR, typename R, bool CHARW>
constexpr size_t sweep_smem_bytes() {
    using G = SweepGeom<DIR>;
    return sizeof(R) * ((size_t)(14 + (CHARW ? 5 : 0)) * G::SIZE + (size_t)14 * G::CH);
}

template <typename R>
__device__ __forceinline__ void to_conserved(const SweepArgs<R> &a, R r, R u, R v, R w, R p, R *U) {
    if constexpr (sizeof(R) == 8) {
        p2c_exact(r, u, v, w, p, a.sp.gamma, U);
    } else {
        p2c_f(r, u, v, w, p, a.sp.gamma - 1.f, U);
    }
}

template <int DIR, typename R, int INTERP, int RS, int CHAR>
__global__ void __launch_bounds__(256)
sweep_kernel(SweepArgs<R> a) {
    using G = SweepGeom<DIR>;
    constexpr int C = G::C, SZ = G::SIZE, CH = G::CH;
    constexpr bool USE_W = (CHAR != 0);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *base = reinterpret_cast<R *>(smem_raw);
    R (*sU)[SZ] = reinterpret_cast<R (*)[SZ]>(base);
    R (*sF)[SZ] = sU + 5;
    R (*sV)[SZ] = sU + 10;
    R (*sW)[SZ] = sU + 14;  // characteristic bases only
    R (*stg)[CH] = reinterpret_cast<R (*)[CH]>(base + (14 + (USE_W ? 5 : 0)) * SZ);  // [9][CH]
    R (*rold)[CH] = stg + 9;                                                          // [5][CH]

    const Layout &L = a.L;
    const int slot = DIR == 0 ? threadIdx.x : threadIdx.y;
    const int line = DIR == 0 ? threadIdx.y : threadIdx.x;
    int ta = blockIdx.x * G::NLINE + line, tb = blockIdx.y;
    const bool line_ok = ta < (DIR == 0 ? L.ny : L.nx);
    ta += NG; tb += NG;
    const int n = DIR == 0 ? L.nx : (DIR == 1 ? L.ny : L.nz);
    auto cell_id = [&](int c) -> long {
        if (DIR == 0) return L.at(c, ta, tb);
        if (DIR == 1) return L.at(ta, c, tb);
        return L.at(ta, tb, c);
    };
    // interior-layout index of interior position ci along the line
    auto vis_id = [&](int ci) -> long {
        const int a0 = ta - NG, b0 = tb - NG;
        if (DIR == 0) return ((long)b0 * L.ny + a0) * L.nx + ci;
        if (DIR == 1) return ((long)b0 * L.ny + ci) * L.nx + a0;
        return ((long)ci * L.ny + b0) * L.nx + a0;
    };
    const bool per = a.periodic != 0;
    const bool visc = a.visc != 0;
    const bool rmw = a.first == 0;
    const int fb = per ? 0 : NG - 1;           // first face computed from cells
    const int fe = per ? n + 5 : n + NG;       // one past the last
    const int cell_end = per ? n + 8 : n + 6;  // one past the last cell needed
    const bool char_rt = CHAR == RUNTIME ? (a.sp.char_recon != 0) : (CHAR != 0);
    const int ti = G::tidx(line, slot);

    auto wrap = [&](int c) { return per ? (c < NG ? c + n : (c >= n + NG ? c - n : c)) : c; };
    // interior index of the viscous node flux of cell c; -1 outside a
    // non-periodic interior (never read there: the orders stay inside)
    auto vis_pos = [&](int c) -> int {
        int ci = c - NG;
        if (per) { if (ci < 0) ci += n; else if (ci >= n) ci -= n; return ci; }
        return (ci >= 0 && ci < n) ? ci : -1;
    };
    // one converted cell into the rings
    auto put_cell = [&](int c, R r, R u, R v, R w, R p, const R *vf) {
        R U[5];
        to_conserved(a, r, u, v, w, p, U);
        const int s = G::sidx(line, c);
#pragma unroll
        for (int q = 0; q < 5; ++q) sU[q][s] = U[q];
        if (USE_W && char_rt) {
            sW[0][s] = r <= R(0) ? R(1e-12) : r; sW[1][s] = u; sW[2][s] = v; sW[3][s] = w; sW[4][s] = p;
        }
        if (visc) {
#pragma unroll
            for (int q = 0; q < 4; ++q) sV[q][s] = vf[q];
        }
    };
    // asynchronous staging of cell c (primitives + viscous fluxes)
    auto stage_cell = [&](int c) {
        const long id = cell_id(wrap(c));
#pragma unroll
        for (int q = 0; q < 5; ++q) cp_async(&stg[q][ti], a.W[q] + id);
        if (visc) {
            const int ci = vis_pos(c);
            if (ci >= 0) {
                const long vid = vis_id(ci);
#pragma unroll
                for (int q = 0; q < 4; ++q) cp_async(&stg[5 + q][ti], a.V[q] + vid);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) stg[5 + q][ti] = R(0);
            }
        }
    };

    // ---- first chunk: the cells of faces [fb, fb+C) are loaded directly
    int loaded = fb - 2;
    {
        const int need = min(fb + C + 3, cell_end);
        for (int c = loaded + slot; c < need; c += C) {
            if (!line_ok) continue;
            const long id = cell_id(wrap(c));
            R vf[4] = {R(0), R(0), R(0), R(0)};
            if (visc) {
                const int ci = vis_pos(c);
                if (ci >= 0) {
                    const long vid = vis_id(ci);
#pragma unroll
                    for (int q = 0; q < 4; ++q) vf[q] = a.V[q][vid];
                }
            }
            put_cell(c, a.W[0][id], a.W[1][id], a.W[2][id], a.W[3][id], a.W[4][id], vf);
        }
        loaded = need;
    }

    for (int fc = fb; fc < fe; fc += C) {
        const bool last = fc + C >= fe;
        const int c_hi = last ? n + NG : min(fc + C - 2, n + NG);
        // ---- asynchronous fetches: the old RHS of this slot's first cell
        //      (group 1) and the next chunk's new cell (group 2)
        const int rc = fc - 2 + slot;
        if (rmw && line_ok && rc >= NG && rc < c_hi) {
            const long id = cell_id(rc);
#pragma unroll
            for (int q = 0; q < 5; ++q) cp_async(&rold[q][ti], a.Rhs[q] + id);
        }
        cp_async_commit();
        const int nfc = fc + C;
        const int next_need = min(nfc + C + 3, cell_end);
        const int pc = loaded + slot;
        const bool prefetch = nfc < fe && line_ok && pc < next_need;
        if (prefetch) stage_cell(pc);
        cp_async_commit();
        __syncthreads();  // rings of this chunk complete
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
        cp_async_wait<1>();  // this thread's old-RHS copies have landed
        __syncthreads();     // face fluxes complete
        // ---- cells whose six faces (c-3 .. c+2) are now available
        for (int c = rc; c < c_hi; c += C) {
            if (!line_ok || c < NG) continue;
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
            R vd[4] = {R(0), R(0), R(0), R(0)};
            if (visc) {
                const int o = visc_order(c - NG, n, per);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    vd[q] = dstencil<R>([&](int off) { return sV[q][G::sidx(line, c + off)]; }, o, a.h);
            }
            const long id = cell_id(c);
            const bool staged = c == rc;
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                // diff_6th_central_half, InviscousFlux.cpp:990-992
                R d = ((fv[q][3] - fv[q][2]) * R(75.0 / 64.0) + (fv[q][4] - fv[q][1]) * R(-25.0 / 384.0) +
                       (fv[q][5] - fv[q][0]) * R(3.0 / 640.0)) * a.inv_h;
                R old = R(0);
                if (rmw) old = staged ? rold[q][ti] : a.Rhs[q][id];
                R r = old - d;
                if (q > 0) r += vd[q - 1];
                a.Rhs[q][id] = r;
            }
        }
        // ---- commit the staged next-chunk cell into the rings
        cp_async_wait<0>();
        __syncthreads();  // staging complete; face-flux and ring reads of this chunk done
        if (prefetch) {
            R v4[4] = {R(0), R(0), R(0), R(0)};
            if (visc) {
#pragma unroll
                for (int q = 0; q < 4; ++q) v4[q] = stg[5 + q][ti];
            }
            put_cell(pc, stg[0][ti], stg[1][ti], stg[2][ti], stg[3][ti], stg[4][ti], v4);
        }
        loaded = next_need;
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
    const size_t smem = sweep_smem_bytes<DIR, R, CHAR != 0>();
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
