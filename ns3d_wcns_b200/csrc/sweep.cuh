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
// chunk-relative shared-memory buffers, so each cell is loaded and converted
// once and each face flux is computed once per line (plus a 5-face halo at
// the line ends).  The next chunk's cells and viscous fluxes are copied with
// cp.async, and the old RHS values loaded, while the face fluxes compute.  In periodic
// directions the wrapped faces are computed from wrapped cells (identical
// inputs, identical values to the reference's face exchange); in non-periodic
// directions the ghost faces are the Outflow copies or zero, as the reference
// leaves them.
//
// Thread mapping keeps global accesses coalesced: along x the 32 lanes of a
// warp march along the line; along y and z the lanes span 32 neighbouring
// x-lines and the warps march.
#pragma once

#include "bc.cuh"
#include "common.cuh"
#include "reduce.cuh"
#include "schemes.cuh"
#include "viscous.cuh"

namespace ns3d {

// The RK stage fused into the last (z) sweep: for every interior cell the
// sweep holds the final right-hand side in registers and the current state,
// so it applies runge_kutta_3's update (range_kutta.cpp:53-91) itself and
// writes the new state instead of the right-hand side; a ghost kernel then
// fills the ghost cells.  stage 0: no fusion (the sweep writes the RHS).
//   plain FP64 path: W0 -> Wout, Tout; the current conserved state is the
//     sweep's exact p2c of W (shared buffer), so the bits equal the separate
//     stage kernel's;
//   mixed path, in increment form: the FP64 step-start state U0 and the FP32
//     stage increment D (both staged with cp.async) give U_s = U0 + D_s;
//     stages 1 and 2 store the next increment (D_1 = dt L0, D_2 = (D_1 +
//     dt L1) / 4) in D, stage 3 the FP64 state U0 + 2/3 (D_2 + dt L2) in
//     Uout.  The FP32 primitives / temperature of U_s are rewritten in place
//     (W32out, T32out): the first five cells of a periodic line are re-read
//     by its wrapped end, so their new primitives are written after the line.
struct FusedStage {
    int stage;
    const double *W0[5];
    double *Wout[5];
    double *Tout;
    const double *U0[5];
    float *D[5];            // mixed: stage increments (FP32 layout), read and rewritten
    double *Uout[5];
    float *W32out[5];
    float *T32out;
    Layout L64;             // layout of the FP64 arrays
    double dt;
    const double *dt_dev;   // non-null: dt from the device time loop
    double gamma, Rgas, dx, vol;
    double *cfl_part, *ke_part;  // stage 3: per-block CFL minimum and kinetic energy
    int keep_rhs;                // also write the complete RHS (the handle's keep_rhs, stage 3 only)
};

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
    R dinv[3];          // 1/(2h), 1/(12h), 1/(60h): the viscous stencils' divisors
    SchemeParams<R> sp;
    int first;          // 1: write (first direction), 0: accumulate
    int visc;           // 1: add the viscous divergence term
    const int *done;    // non-null: skip the launch while *done (device time loop)
    int zlo, zhi;       // owned interior z-planes [zlo, zhi): the x/y sweeps run over them, the
                        // z-sweep updates only them (the rest of a z-slab's planes are halo)
    FusedStage fs;      // z-sweep only
};

// Chunk geometry.  A chunk holds C faces of every line of the block.  Its
// shared-memory buffers are indexed relative to the chunk (no ring wrap):
//   cells  position p <-> cell fc - 2 + p, p in [0, NU)  (conserved state)
//   faces  position p <-> face fc - 5 + p, p in [0, NF)
//   visc   position p <-> cell fc - 5 + p, p in [0, NV)  (node fluxes)
// At the end of a chunk the tails are moved to the front and the staged next
// cells appended, so every stencil read is a fixed offset from the thread's
// own position.
// FP64 y/z chunk geometry (faces per chunk, lines per block; C * NLINE = 256)
#ifndef NS3D_SWEEP64_YZ_C
#define NS3D_SWEEP64_YZ_C 8
#endif
#ifndef NS3D_SWEEP64_YZ_NL
#define NS3D_SWEEP64_YZ_NL 32
#endif
template <int DIR, typename R>
struct SweepGeom {
    static constexpr bool F64 = sizeof(R) == 8;
    static constexpr int C = DIR == 0 ? 32 : (F64 ? NS3D_SWEEP64_YZ_C : 8);        // faces per chunk
    static constexpr int NLINE = DIR == 0 ? 8 : (F64 ? NS3D_SWEEP64_YZ_NL : 32);  // lines per block
    static constexpr int CH = C * NLINE;               // threads
    static constexpr int NU = C + 5, NF = C + 7, NV = C + 8;
    // along x a warp owns one line ([line][pos]); along y/z the lanes span
    // neighbouring lines ([pos][line]); both are conflict-free
    template <int NP>
    __device__ __forceinline__ static int idx(int line, int pos) {
        return DIR == 0 ? line * NP + pos : pos * NLINE + line;
    }
    __device__ __forceinline__ static int tidx(int line, int slot) {
        return DIR == 0 ? line * C + slot : slot * NLINE + line;
    }
};

// The old RHS of the updated cell is staged in shared memory with the next
// chunk's cells (true) or loaded into registers (false).
constexpr bool kRoldSmem = true;
// minimum resident blocks per SM requested from the register allocator
#ifndef NS3D_SWEEP64_MINB
#define NS3D_SWEEP64_MINB 2
#endif
template <int DIR, typename R>
constexpr int sweep_min_blocks() { return sizeof(R) == 8 ? NS3D_SWEEP64_MINB : 2; }

// buffers U(5) F(5) V(4) [W(5) for characteristic bases], staging W(5)+V(4)
// [+ old RHS(5)]
template <int DIR, typename R, bool CHARW>
constexpr size_t sweep_smem_bytes() {
    using G = SweepGeom<DIR, R>;
    return sizeof(R) * ((size_t)G::NLINE * (5 * G::NU + 5 * G::NF + 4 * G::NV + (CHARW ? 5 * G::NU : 0)) +
                        (size_t)(kRoldSmem ? 14 : 9) * G::CH) +
           (DIR == 2 ? (size_t)5 * G::CH * (sizeof(double) + (sizeof(R) == 4 ? sizeof(float) : 0)) : 0);  // fused stage
}

template <typename R>
__device__ __forceinline__ void to_conserved(const SweepArgs<R> &a, R r, R u, R v, R w, R p, R *U) {
    if constexpr (sizeof(R) == 8) {
        p2c_exact(r, u, v, w, p, a.sp.gamma, U);
    } else {
        p2c_f(r, u, v, w, p, a.sp.gamma - 1.f, U);
    }
}

// first derivative along the line, ViscousFlux.cpp:15-29 with the order of
// choose_scheme; dinv = 1/(2h), 1/(12h), 1/(60h).  Order -1 reproduces the
// reference's backward form, which evaluates to -df/dx.
template <typename R, typename F>
__device__ __forceinline__ R dstencil_inv(F f, int order, const R *dinv) {
    if (order == 6)
        return (f(3) - R(9) * f(2) + R(45) * f(1) - R(45) * f(-1) + R(9) * f(-2) - f(-3)) * dinv[2];
    if (order == 1 || order == -1) return (R(-3) * f(0) + R(4) * f(order) - f(2 * order)) * dinv[0];
    if (order == 2) return (f(1) - f(-1)) * dinv[0];
    return (-f(2) + R(8) * f(1) - R(8) * f(-1) + f(-2)) * dinv[1];
}

// Stage update of interior cell c (padded FP64 index) from its final
// right-hand side r and current conserved state Uc (the sweep's exact p2c of
// W): the operations of stage_kernel64 for an interior cell, so the same bits.
// w0: the cell's step-start primitives (staged by the sweep; stages 2 and 3
// only -- in stage 1 the step-start state is the current one, whose exact p2c
// the sweep already holds).
__device__ __forceinline__ void fused_stage_cell(const FusedStage &f, double dt, long c, const double *r,
                                                 const double *Ucur, const double *w0, double &smax, double &ke,
                                                 double &kc) {
    double U0[5], U[5], W[5];
    if (f.stage == 1) {
#pragma unroll
        for (int q = 0; q < 5; ++q) U0[q] = Ucur[q];
    } else {
        p2c_exact(w0[0], w0[1], w0[2], w0[3], w0[4], f.gamma, U0);
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) U[q] = rk_combine(f.stage, U0[q], f.stage == 1 ? U0[q] : Ucur[q], r[q], dt);
    c2p_exact(U, f.gamma, W);
#pragma unroll
    for (int q = 0; q < 5; ++q) f.Wout[q][c] = W[q];
    f.Tout[c] = W[4] / __dmul_rn(W[0], f.Rgas);
    if (f.stage == 3) {
        double Un[5];
        p2c_exact(W[0], W[1], W[2], W[3], W[4], f.gamma, Un);
        smax = fmax(smax, cfl_speed(Un, f.gamma));  // largest wave speed: one division per block
        // a thread adds one cell per chunk along its line: compensated
        // (Kahan) summation keeps its partial exact to rounding
        const double y = 0.5 * W[0] * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) * f.vol - kc;
        const double t = __dadd_rn(ke, y);
        kc = __dsub_rn(__dsub_rn(t, ke), y);
        ke = t;
    }
}

// The detector bits of a cell (and of the line's first cell) again with
// mdcd_smooth's exact decisions, for the rare cell where one of the
// cross-multiplied tests was too close to call.  Stencils re-read from shared
// memory, so no registers stay alive across the common path.
template <typename R, int NL, int NU, typename G>
__device__ __noinline__ uint2 detect_exact(const R *sU, int line, int slot, bool first) {
    unsigned r3 = 0, r2f = 0;  // as in the sweep: bit q for cell f+1 / f
    for (int q = 0; q < 5; ++q) {
        R sq[6];
        for (int m = 0; m < 6; ++m) sq[m] = sU[q * NL * NU + G::template idx<NU>(line, slot + m)];
        r3 |= (mdcd_smooth(sq[1], sq[2], sq[3], sq[4], sq[5]) ? 0u : 1u) << q;
        if (first) r2f |= (mdcd_smooth(sq[0], sq[1], sq[2], sq[3], sq[4]) ? 0u : 1u) << q;
    }
    return make_uint2(r3, r2f);
}

template <int DIR, typename R, int INTERP, int RS, int CHAR>
__global__ void __launch_bounds__(256, sweep_min_blocks<DIR, R>())
sweep_kernel(SweepArgs<R> a) {
    using G = SweepGeom<DIR, R>;
    constexpr int C = G::C, NL = G::NLINE, CH = G::CH, NU = G::NU, NF = G::NF, NV = G::NV;
    constexpr bool USE_W = (CHAR != 0);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *const sU = reinterpret_cast<R *>(smem_raw);  // [5][NL*NU]
    R *const sF = sU + 5 * NL * NU;                  // [5][NL*NF]
    R *const sV = sF + 5 * NL * NF;                  // [4][NL*NV]
    R *const sW = sV + 4 * NL * NV;                  // [5][NL*NU] characteristic bases only
    R *const stg = sW + (USE_W ? 5 * NL * NU : 0);   // [9][CH]
    R *const srold = stg + 9 * CH;                   // [5][CH] (kRoldSmem)
    // fused stage (z-sweep): staged FP64 step-start state, and (mixed) the FP32 increment
    double *const sUf = reinterpret_cast<double *>(srold + 5 * CH);  // z fused stage: [5][CH] FP64
    float *const sDs = reinterpret_cast<float *>(sUf + 5 * CH);       // mixed: [5][CH] stage increment

    if (a.done && *a.done) return;  // uniform over the grid
    const Layout &L = a.L;
    // fused stage (z-sweep): dt, and the thread's largest wave speed / kinetic energy
    const double fdt = (DIR == 2 && a.fs.stage) ? (a.fs.dt_dev ? *a.fs.dt_dev : a.fs.dt) : 0.0;
    double cfl_acc = 0.0, ke_acc = 0.0, ke_c = 0.0;  // largest wave speed, kinetic energy
    const double irg = (DIR == 2 && sizeof(R) == 4 && a.fs.stage) ? 1.0 / a.fs.Rgas : 0.0;  // mixed: T = p / (rho Rgas)
    // mixed fused stage: the deferred new primitives of one of a periodic line's first five cells
    bool has_def = false;
    long def_id = 0;
    unsigned det_carry = 0;  // x-sweep detector bits of the previous chunk's last face (cell fc)
    // y/z-sweep detector bits, position p <-> cell fc + p (MDCD_HYBRID)
    __shared__ unsigned char sDet[(DIR != 0 && CHAR == 0 && INTERP == I_MDCD_HYBRID) ? (C + 1) * NL : 1];
    // periodic x-lines: faces 0 .. 4 of each line, kept from the first chunk
    // for faces n .. n+4 (the same wrapped cells, so the same bits)
    __shared__ R sWrapF[(DIR == 0 && CHAR == 0 && INTERP == I_MDCD_HYBRID) ? 25 * NL : 1];
    float def_w[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, def_t = 0.f;
    const int slot = DIR == 0 ? threadIdx.x : threadIdx.y;
    const int line = DIR == 0 ? threadIdx.y : threadIdx.x;
    const int ta0 = blockIdx.x * NL + line, tb0 = blockIdx.y + (DIR == 2 ? 0 : a.zlo);
    const bool line_ok = ta0 < (DIR == 0 ? L.ny : L.nx);
    const int n = DIR == 0 ? L.nx : (DIR == 1 ? L.ny : L.nz);
    // padded-layout address of cell c (ghost-inclusive index along the line)
    long lbase, lstride, vbase, vstride;
    if (DIR == 0) {
        lbase = L.at(0, ta0 + NG, tb0 + NG); lstride = 1;
        vbase = ((long)tb0 * L.ny + ta0) * L.nx; vstride = 1;
    } else if (DIR == 1) {
        lbase = L.at(ta0 + NG, 0, tb0 + NG); lstride = L.px;
        vbase = (long)tb0 * L.ny * L.nx + ta0; vstride = L.nx;
    } else {
        lbase = L.at(ta0 + NG, tb0 + NG, 0); lstride = (long)L.px * L.sy;
        vbase = (long)tb0 * L.nx + ta0; vstride = (long)L.nx * L.ny;
    }
    const bool per = a.periodic != 0;
    const bool visc = a.visc != 0;
    const bool rmw = a.first == 0;
    const int fb = per ? 0 : NG - 1;           // first face computed from cells
    const int fe = per ? n + 5 : n + NG;       // one past the last computed face
    const int cell_end = per ? n + 8 : n + 6;  // one past the last cell needed
    const int chunk_end = n + NG + 2;          // chunks run while fc - 2 < n + NG
    const bool char_rt = CHAR == RUNTIME ? (a.sp.char_recon != 0) : (CHAR != 0);
    const int ti = G::tidx(line, slot);

    auto wrap = [&](int c) { return per ? (c < NG ? c + n : (c >= n + NG ? c - n : c)) : c; };
    // interior index of the node flux of cell c, or -1 (outside a
    // non-periodic interior, or before the first needed cell: never read)
    auto vis_pos = [&](int c) -> int {
        if (c < 0) return -1;
        int ci = c - NG;
        if (per) { if (ci < 0) ci += n; else if (ci >= n) ci -= n; return ci; }
        return (ci >= 0 && ci < n) ? ci : -1;
    };
    auto put_cell = [&](int pu, int pv, R r, R u, R v, R w, R p, const R *vf) {
        R U[5];
        to_conserved(a, r, u, v, w, p, U);
        const int s = G::template idx<NU>(line, pu);
#pragma unroll
        for (int q = 0; q < 5; ++q) sU[q * NL * NU + s] = U[q];
        if (USE_W && char_rt) {
            R *w5 = sW + s;
            w5[0] = r <= R(0) ? R(1e-12) : r; w5[NL * NU] = u; w5[2 * NL * NU] = v;
            w5[3 * NL * NU] = w; w5[4 * NL * NU] = p;
        }
        if (visc && pv >= 0) {
            const int sv = G::template idx<NV>(line, pv);
#pragma unroll
            for (int q = 0; q < 4; ++q) sV[q * NL * NV + sv] = vf[q];
        }
    };

    // ---- first chunk: visc positions [0, NV) = cells fb-5 .., cell
    //      positions [0, NU) = cells fb-2 .. (position p-3 of the same cell)
    if (line_ok) {
        for (int p = slot; p < NV; p += C) {
            const int c = fb - 5 + p;
            R vf[4] = {R(0), R(0), R(0), R(0)};
            if (visc) {
                const int ci = vis_pos(c);
                if (ci >= 0) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) vf[q] = a.V[q][vbase + ci * vstride];
                }
            }
            if (p >= 3 && c < cell_end) {
                const long id = lbase + wrap(c) * lstride;
                put_cell(p - 3, p, a.W[0][id], a.W[1][id], a.W[2][id], a.W[3][id], a.W[4][id], vf);
            } else if (visc) {
                const int sv = G::template idx<NV>(line, p);
#pragma unroll
                for (int q = 0; q < 4; ++q) sV[q * NL * NV + sv] = vf[q];
            }
        }
    }

    for (int fc = fb; fc < chunk_end; fc += C) {
        // cell updated by this thread in this chunk; its old RHS (plain
        // loads, consumed after the face phase)
        const int cu = fc - 2 + slot;
        const bool upd = line_ok && cu >= NG && cu < n + NG && (DIR != 2 || (cu - NG >= a.zlo && cu - NG < a.zhi));
        const long cid = lbase + cu * lstride;
        R rold[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) rold[q] = R(0);
        if (rmw && upd) {
            if constexpr (kRoldSmem) {
#pragma unroll
                for (int q = 0; q < 5; ++q) cp_async(&srold[q * CH + ti], a.Rhs[q] + cid);
            } else {
#pragma unroll
                for (int q = 0; q < 5; ++q) rold[q] = a.Rhs[q][cid];
            }
        }
        if constexpr (DIR == 2 && sizeof(R) == 8) {
            if (a.fs.stage > 1 && upd) {  // the step-start primitives of the cell this thread updates
#pragma unroll
                for (int q = 0; q < 5; ++q) cp_async(&sUf[q * CH + ti], a.fs.W0[q] + cid);
            }
        }
        if constexpr (DIR == 2 && sizeof(R) == 4) {
            if (a.fs.stage && upd) {  // the FP64 state of the cell this thread updates
                const long c64 = a.fs.L64.at(ta0 + NG, tb0 + NG, cu);
#pragma unroll
                for (int q = 0; q < 5; ++q) cp_async(&sUf[q * CH + ti], a.fs.U0[q] + c64);
                if (a.fs.stage > 1) {
#pragma unroll
                    for (int q = 0; q < 5; ++q) cp_async(&sDs[q * CH + ti], a.fs.D[q] + cid);
                }
            }
        }
        if constexpr (kRoldSmem) cp_async_commit();
        // stage the next chunk's new cell (cell and visc positions 5+slot, 8+slot)
        const int cn = fc + C + 3 + slot;
        const bool stage = fc + C < chunk_end && line_ok && cn < cell_end;
        if (stage) {
            const long id = lbase + wrap(cn) * lstride;
#pragma unroll
            for (int q = 0; q < 5; ++q) cp_async(&stg[q * CH + ti], a.W[q] + id);
            if (visc) {
                const int ci = vis_pos(cn);
                if (ci >= 0) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) cp_async(&stg[(5 + q) * CH + ti], a.V[q] + vbase + ci * vstride);
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) stg[(5 + q) * CH + ti] = R(0);
                }
            }
        }
        cp_async_commit();
        __syncthreads();  // buffers of this chunk complete

        // ---- face f = fc + slot (between cells f and f+1): cell positions slot .. slot+5
        const int f = fc + slot;
        if constexpr (DIR == 0 && CHAR == 0 && INTERP == I_MDCD_HYBRID) {
            // Along x a warp is one line and its lanes are consecutive faces.
            // The detector at a face's right-hand centre (cell f+1) is the
            // left-hand centre of the next face, so each lane evaluates one
            // centre and takes the other from the lane before it (lane 0: from
            // lane 31 of the previous chunk; in the first chunk it evaluates
            // both).  Same values as evaluating both centres per face.
            if (line_ok && per && fc >= n) {
                // the last chunk of a periodic line holds only faces n .. n+4
                // (fc >= n: uniform over the block): copies of faces 0 .. 4
                if (f < fe) {
#pragma unroll
                    for (int q = 0; q < 5; ++q)
                        sF[q * NL * NF + G::template idx<NF>(line, slot + 5)] = sWrapF[(q * NL + line) * 5 + (f - n)];
                }
            } else if (line_ok) {  // uniform over the warp
                // one variable's stencil at a time (its registers die with it);
                // the rare WENO branch re-reads its stencil from shared memory
                R UL[5], UR[5];
                unsigned r3 = 0, r2f = 0;  // bit q: the detector rejects the linear scheme at cell f+1 / f
                bool near = false;
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    R sq[6];
#pragma unroll
                    for (int m = 0; m < 6; ++m) sq[m] = sU[q * NL * NU + G::template idx<NU>(line, slot + m)];
                    r3 |= (mdcd_smooth_fast(sq[1], sq[2], sq[3], sq[4], sq[5], near) ? 0u : 1u) << q;
                    if (fc == fb && slot == 0)
                        r2f |= (mdcd_smooth_fast(sq[0], sq[1], sq[2], sq[3], sq[4], near) ? 0u : 1u) << q;
                    UL[q] = mdcd_linear(a.sp.lin, sq[0], sq[1], sq[2], sq[3], sq[4], sq[5]);
                    UR[q] = mdcd_linear(a.sp.lin, sq[5], sq[4], sq[3], sq[2], sq[1], sq[0]);
                }
                if (near) {
                    const uint2 e = detect_exact<R, NL, NU, G>(sU, line, slot, fc == fb && slot == 0);
                    r3 = e.x;
                    r2f = e.y;
                }
                unsigned r2 = __shfl_up_sync(0xffffffffu, r3, 1);
                if (slot == 0) r2 = fc == fb ? r2f : det_carry;
                det_carry = __shfl_sync(0xffffffffu, r3, 31);
                if (f < fe) {
                    const unsigned weno = r2 | r3;
                    if (weno) {
#pragma unroll
                        for (int q = 0; q < 5; ++q)
                            if (weno & (1u << q)) {
                                const volatile R *vq = sU + q * NL * NU;
                                R sq[6];
#pragma unroll
                                for (int m = 0; m < 6; ++m) sq[m] = vq[G::template idx<NU>(line, slot + m)];
                                UL[q] = mdcd_weno_branch(a.sp.hd, sq[0], sq[1], sq[2], sq[3], sq[4], sq[5]);
                                UR[q] = mdcd_weno_branch(a.sp.hd, sq[5], sq[4], sq[3], sq[2], sq[1], sq[0]);
                            }
                    }
                    R F[5];
                    riemann<DIR, R, RS>(a.sp, UL, UR, F);
                    const int s = G::template idx<NF>(line, slot + 5);
#pragma unroll
                    for (int q = 0; q < 5; ++q) sF[q * NL * NF + s] = F[q];
                    if (per && f < 5) {  // first chunk (fb = 0 on periodic lines)
#pragma unroll
                        for (int q = 0; q < 5; ++q) sWrapF[(q * NL + line) * 5 + f] = F[q];
                    }
                }
            }
        } else if constexpr (DIR != 0 && CHAR == 0 && INTERP == I_MDCD_HYBRID) {
            // Along y and z the faces of a line are spread over the warps:
            // each face evaluates the detector at its right-hand centre (cell
            // f+1) into shared memory and, after a barrier, reads its
            // left-hand centre (cell f) written by the face before it.  Cell
            // fc comes from the previous chunk's last face (moved with the
            // tails); the first chunk's first face evaluates it.
            const bool act = line_ok && f < fe;
            // one variable's stencil at a time (its registers die with it);
            // the rare WENO branch re-reads its stencil from shared memory
            R UL[5], UR[5];
            unsigned r3 = 0;
            if (act) {
                unsigned r2f = 0;
                bool near = false;
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    R sq[6];
#pragma unroll
                    for (int m = 0; m < 6; ++m) sq[m] = sU[q * NL * NU + G::template idx<NU>(line, slot + m)];
                    r3 |= (mdcd_smooth_fast(sq[1], sq[2], sq[3], sq[4], sq[5], near) ? 0u : 1u) << q;
                    if (fc == fb && slot == 0)
                        r2f |= (mdcd_smooth_fast(sq[0], sq[1], sq[2], sq[3], sq[4], near) ? 0u : 1u) << q;
                    UL[q] = mdcd_linear(a.sp.lin, sq[0], sq[1], sq[2], sq[3], sq[4], sq[5]);
                    UR[q] = mdcd_linear(a.sp.lin, sq[5], sq[4], sq[3], sq[2], sq[1], sq[0]);
                }
                if (near) {
                    const uint2 e = detect_exact<R, NL, NU, G>(sU, line, slot, fc == fb && slot == 0);
                    r3 = e.x;
                    r2f = e.y;
                }
                sDet[(slot + 1) * NL + line] = (unsigned char)r3;
                if (fc == fb && slot == 0) sDet[line] = (unsigned char)r2f;
            }
            __syncthreads();  // detector bits of this chunk's cells complete
            if (act) {
                const unsigned weno = r3 | sDet[slot * NL + line];
                if (weno) {
#pragma unroll
                    for (int q = 0; q < 5; ++q)
                        if (weno & (1u << q)) {
                            const volatile R *vq = sU + q * NL * NU;
                            R sq[6];
#pragma unroll
                            for (int m = 0; m < 6; ++m) sq[m] = vq[G::template idx<NU>(line, slot + m)];
                            UL[q] = mdcd_weno_branch(a.sp.hd, sq[0], sq[1], sq[2], sq[3], sq[4], sq[5]);
                            UR[q] = mdcd_weno_branch(a.sp.hd, sq[5], sq[4], sq[3], sq[2], sq[1], sq[0]);
                        }
                }
                R F[5];
                riemann<DIR, R, RS>(a.sp, UL, UR, F);
                const int s = G::template idx<NF>(line, slot + 5);
#pragma unroll
                for (int q = 0; q < 5; ++q) sF[q * NL * NF + s] = F[q];
            }
        } else if (CHAR == 0 && line_ok && f < fe) {
            R st[5][6];
#pragma unroll
            for (int q = 0; q < 5; ++q)
#pragma unroll
                for (int m = 0; m < 6; ++m) st[q][m] = sU[q * NL * NU + G::template idx<NU>(line, slot + m)];
            R UL[5], UR[5];
            if constexpr (INTERP == I_MDCD_HYBRID) {
                // detector of every variable, the linear states of all, then
                // the WENO branch only where a detector rejected the linear
                // scheme (rare): the common path has no divergent branch
                unsigned weno = 0;
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    const bool lin = mdcd_smooth(st[q][0], st[q][1], st[q][2], st[q][3], st[q][4]) &&
                                     mdcd_smooth(st[q][1], st[q][2], st[q][3], st[q][4], st[q][5]);
                    weno |= (lin ? 0u : 1u) << q;
                    UL[q] = mdcd_linear(a.sp.lin, st[q][0], st[q][1], st[q][2], st[q][3], st[q][4], st[q][5]);
                    UR[q] = mdcd_linear(a.sp.lin, st[q][5], st[q][4], st[q][3], st[q][2], st[q][1], st[q][0]);
                }
                if (weno) {
#pragma unroll
                    for (int q = 0; q < 5; ++q)
                        if (weno & (1u << q)) {
                            UL[q] = mdcd_weno_branch(a.sp.hd, st[q][0], st[q][1], st[q][2], st[q][3], st[q][4], st[q][5]);
                            UR[q] = mdcd_weno_branch(a.sp.hd, st[q][5], st[q][4], st[q][3], st[q][2], st[q][1], st[q][0]);
                        }
                }
            } else {
#pragma unroll
                for (int q = 0; q < 5; ++q) face_pair<R, INTERP>(a.sp, st[q], UL[q], UR[q]);
            }
            R F[5];
            riemann<DIR, R, RS>(a.sp, UL, UR, F);
            const int s = G::template idx<NF>(line, slot + 5);
#pragma unroll
            for (int q = 0; q < 5; ++q) sF[q * NL * NF + s] = F[q];
        } else if (line_ok && f < fe) {
            R st[5][6];
#pragma unroll
            for (int q = 0; q < 5; ++q)
#pragma unroll
                for (int m = 0; m < 6; ++m) st[q][m] = sU[q * NL * NU + G::template idx<NU>(line, slot + m)];
            R wi[5], wi1[5];
            if (USE_W && char_rt) {
                const int s0 = G::template idx<NU>(line, slot + 2), s1 = G::template idx<NU>(line, slot + 3);
#pragma unroll
                for (int q = 0; q < 5; ++q) { wi[q] = sW[q * NL * NU + s0]; wi1[q] = sW[q * NL * NU + s1]; }
            }
            R F[5];
            wcns_face<DIR, R, INTERP, RS, CHAR>(a.sp, st, wi, wi1, F);
            const int s = G::template idx<NF>(line, slot + 5);
#pragma unroll
            for (int q = 0; q < 5; ++q) sF[q * NL * NF + s] = F[q];
        }
        if constexpr (kRoldSmem) cp_async_wait<1>();  // this thread's old-RHS copies landed
        __syncthreads();  // faces of this chunk complete
        if constexpr (DIR != 0 && CHAR == 0 && INTERP == I_MDCD_HYBRID) {
            // the last face's bits (cell fc + C) become the next chunk's cell fc
            if (line_ok && slot == C - 1) sDet[line] = sDet[C * NL + line];
        }
        if constexpr (kRoldSmem) {
            if (rmw && upd) {
#pragma unroll
                for (int q = 0; q < 5; ++q) rold[q] = srold[q * CH + ti];
            }
        }

        // ---- cell cu: faces cu-3 .. cu+2 at positions slot .. slot+5,
        //      node fluxes cu-3 .. cu+3 at visc positions slot .. slot+6
        if (upd) {
            // within 3 cells of a non-periodic boundary the reference's ghost
            // faces (Outflow copy of the boundary face, else zero) and the
            // reduced viscous orders apply; everywhere else one straight path
            const bool edge = !per && (cu - NG < 3 || cu - NG >= n - 3);
            R d[5], vd[4] = {R(0), R(0), R(0), R(0)};
            if (!edge) {
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    const R *fq = sF + q * NL * NF;
                    auto F_ = [&](int m) { return fq[G::template idx<NF>(line, slot + m)]; };
                    // diff_6th_central_half, InviscousFlux.cpp:990-992
                    d[q] = ((F_(3) - F_(2)) * R(75.0 / 64.0) + (F_(4) - F_(1)) * R(-25.0 / 384.0) +
                            (F_(5) - F_(0)) * R(3.0 / 640.0)) * a.inv_h;
                }
                if (visc) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const R *vq = sV + q * NL * NV;
                        auto V_ = [&](int off) { return vq[G::template idx<NV>(line, slot + 3 + off)]; };
                        vd[q] = (V_(3) - R(9) * V_(2) + R(45) * V_(1) - R(45) * V_(-1) + R(9) * V_(-2) - V_(-3)) *
                                a.dinv[2];
                    }
                }
            } else {
                const int pf_lo = (NG - 1) - (fc - 5), pf_hi = (n + NG - 1) - (fc - 5);
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    R fv[6];
#pragma unroll
                    for (int m = 0; m < 6; ++m) {
                        int pm = slot + m;
                        bool zero = false;
                        const int ff = cu - 3 + m;
                        if (ff < NG - 1) { if (a.outflow_lo) pm = pf_lo; else zero = true; }
                        else if (ff > n + NG - 1) { if (a.outflow_hi) pm = pf_hi; else zero = true; }
                        fv[m] = zero ? R(0) : sF[q * NL * NF + G::template idx<NF>(line, pm)];
                    }
                    d[q] = ((fv[3] - fv[2]) * R(75.0 / 64.0) + (fv[4] - fv[1]) * R(-25.0 / 384.0) +
                            (fv[5] - fv[0]) * R(3.0 / 640.0)) * a.inv_h;
                }
                if (visc) {
                    const int o = visc_order(cu - NG, n, false);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        vd[q] = dstencil_inv<R>(
                            [&](int off) { return sV[q * NL * NV + G::template idx<NV>(line, slot + 3 + off)]; },
                            o, a.dinv);
                }
            }
            R rq[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                rq[q] = rold[q] - d[q];
                if (q > 0) rq[q] += vd[q - 1];
            }
            bool fused = false;
            if constexpr (DIR == 2 && sizeof(R) == 8) {
                if (a.fs.stage) {
                    double Uc[5], rr[5];
#pragma unroll
                    for (int q = 0; q < 5; ++q) {
                        Uc[q] = sU[q * NL * NU + G::template idx<NU>(line, slot)];
                        rr[q] = rq[q];
                    }
                    double w0[5];
#pragma unroll
                    for (int q = 0; q < 5; ++q) w0[q] = a.fs.stage > 1 ? sUf[q * CH + ti] : 0.0;
                    fused_stage_cell(a.fs, fdt, cid, rr, Uc, w0, cfl_acc, ke_acc, ke_c);
                    fused = true;
                }
            }
            if constexpr (DIR == 2 && sizeof(R) == 4) {
                if (a.fs.stage) {
                    const FusedStage &f = a.fs;
                    double U[5];
#pragma unroll
                    for (int q = 0; q < 5; ++q) {
                        const double rr = (double)rq[q];
                        const double u0 = sUf[q * CH + ti];
                        const double dp = f.stage == 1 ? 0.0 : (double)sDs[q * CH + ti];
                        if (f.stage == 3) {
                            U[q] = u0 + (2.0 / 3.0) * (dp + fdt * rr);
                        } else {
                            const float dn = (float)(f.stage == 1 ? fdt * rr : 0.25 * (dp + fdt * rr));
                            f.D[q][cid] = dn;
                            U[q] = u0 + (double)dn;
                        }
                    }
                    if (U[0] <= 0.0) U[0] = 1e-12;
                    double W[5], ir;
                    c2p_fast(U, f.gamma, W, ir);
                    if (f.stage == 3) {
                        const long c64 = f.L64.at(ta0 + NG, tb0 + NG, cu);
#pragma unroll
                        for (int q = 0; q < 5; ++q) f.Uout[q][c64] = U[q];
                    }
                    if (per && cu < NG + 5) {  // re-read by the line's wrapped end: write after the line
                        has_def = true; def_id = cid;
#pragma unroll
                        for (int q = 0; q < 5; ++q) def_w[q] = (float)W[q];
                        def_t = (float)(W[4] * ir * irg);
                    } else {
#pragma unroll
                        for (int q = 0; q < 5; ++q) f.W32out[q][cid] = (float)W[q];
                        f.T32out[cid] = (float)(W[4] * ir * irg);
                    }
                    if (f.stage == 3) {
                        cfl_acc = fmax(cfl_acc, cfl_speed(U, f.gamma));
                        const double y = 0.5 * W[0] * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) * f.vol - ke_c;
                        const double t = __dadd_rn(ke_acc, y);
                        ke_c = __dsub_rn(__dsub_rn(t, ke_acc), y);
                        ke_acc = t;
                    }
                    fused = true;
                }
            }
            if (!fused || a.fs.keep_rhs) {  // keep_rhs: the last stage's complete RHS as well
#pragma unroll
                for (int q = 0; q < 5; ++q) a.Rhs[q][cid] = rq[q];
            }
        }
        cp_async_wait<0>();
        __syncthreads();  // buffer reads of this chunk done; staged cells landed

        // ---- move the tails to the front, append the staged cell
        if (line_ok && fc + C < chunk_end) {
            if (visc && slot >= C - 8) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    sV[q * NL * NV + G::template idx<NV>(line, slot - C + 8)] =
                        sV[q * NL * NV + G::template idx<NV>(line, slot + 8)];
            }
            if (slot >= C - 5) {
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    sU[q * NL * NU + G::template idx<NU>(line, slot - C + 5)] =
                        sU[q * NL * NU + G::template idx<NU>(line, slot + 5)];
                    sF[q * NL * NF + G::template idx<NF>(line, slot - C + 5)] =
                        sF[q * NL * NF + G::template idx<NF>(line, slot + 5)];
                    if (USE_W && char_rt)
                        sW[q * NL * NU + G::template idx<NU>(line, slot - C + 5)] =
                            sW[q * NL * NU + G::template idx<NU>(line, slot + 5)];
                }
            }
            if (stage) {
                R v4[4] = {R(0), R(0), R(0), R(0)};
                if (visc) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) v4[q] = stg[(5 + q) * CH + ti];
                }
                put_cell(5 + slot, 8 + slot, stg[ti], stg[CH + ti], stg[2 * CH + ti], stg[3 * CH + ti],
                         stg[4 * CH + ti], v4);
            }
        }
    }
    if constexpr (DIR == 2 && sizeof(R) == 4) {
        if (has_def) {  // the line is done: nothing reads these cells any more
#pragma unroll
            for (int q = 0; q < 5; ++q) a.fs.W32out[q][def_id] = def_w[q];
            a.fs.T32out[def_id] = def_t;
        }
    }
    if (DIR == 2 && a.fs.stage == 3)  // uniform: every thread of the block arrives
        block_speed_sum_n<CH>(cfl_acc, ke_acc - ke_c, a.fs.dx,
                              a.fs.cfl_part + (long)blockIdx.y * gridDim.x + blockIdx.x,
                              a.fs.ke_part + (long)blockIdx.y * gridDim.x + blockIdx.x);
}

template <int DIR, typename R, int INTERP, int RS, int CHAR>
inline cudaError_t launch_sweep(const SweepArgs<R> &a, cudaStream_t st) {
    using G = SweepGeom<DIR, R>;
    dim3 block(DIR == 0 ? G::C : G::NLINE, DIR == 0 ? G::NLINE : G::C);
    dim3 grid;
    if (DIR == 0) grid = dim3((a.L.ny + G::NLINE - 1) / G::NLINE, a.zhi - a.zlo);
    else if (DIR == 1) grid = dim3((a.L.nx + G::NLINE - 1) / G::NLINE, a.zhi - a.zlo);
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
