// batch.cu -- many independent small problems (e.g. quasi-1D shock tubes of
// uneven length) in one persistent launch.
//
// Each problem is a complete ns3d_wcns run on its own grid: its own CFL time
// step every step (timestep.cpp:5-23), the dt schedule of time_advance
// (maincycle.cpp:18-56: clip to t_end, stop when dt <= 1e-12), and full
// runge_kutta_3 steps with the device ghost fill, the same face fluxes and the
// same stage arithmetic as the single-domain path.
//
// Scheduling: the grid is a set of thread-block clusters; a cluster takes the
// next problem from an atomic work counter (problems are sorted by decreasing
// cost, so this is longest-processing-time-first list scheduling) and
// integrates it to its end time; the cluster's CTAs split the problem's x
// range and meet at hardware cluster barriers between phases.  There is no
// software spin-wait anywhere.  The cluster size and CTA width are chosen by
// ns3d_batch_autotune (timed trial launches); the launch (counter reset +
// kernel) is captured once in a CUDA graph and replayed.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ns3d_b200.h"
#include "common.cuh"
#include "bc.cuh"
#include "reduce.cuh"
#include "schemes.cuh"

namespace cg = cooperative_groups;
using namespace ns3d;

namespace {

struct Inst {
    Layout L;
    long base;        // offset (elements) of this problem's arrays in the pool
    double dx, dy, dz, inv_dx, inv_dy, inv_dz;
    double t_end;
    int bc[6];
    int periodic[3];
};

// per-problem array offsets relative to Inst::base (units of L.plane):
// W buffers 0..14 (3 x 5), face fluxes X 15..19, Y 20..24, Z 25..29, and the
// conserved state U = p2c(W) of each W buffer 30..44 (every cell, ghosts
// included), kept beside W so that each cell is converted once per stage
// instead of once per stencil that reads it
constexpr int NARR = 45;
constexpr int UOFF = 30;

struct BatchArgs {
    const Inst *inst;
    double *pool;
    int n_inst;
    int *counter;        // work queue
    double *t_out;       // per-problem final time
    int *steps_out;      // per-problem steps taken
    int *state_out;      // per-problem: index of the W buffer holding the final state
    int *status_out;     // 0 ok, 1 stopped on dt <= 1e-12, 2 max_steps reached
    double *partials;    // per-problem CFL partial minima, [n_inst][16]
    int max_steps;
    double cfl, gamma;
    SchemeParams<double> sp;
};

__device__ __forceinline__ double *arr(const BatchArgs &a, const Inst &I, int q) {
    return a.pool + I.base + (long)q * I.L.plane;
}

// Which stored x-face gives the flux of face g of a line in the half-node
// difference: periodic x wraps (face nx is face 0: the same stencil cells);
// otherwise a face beyond the domain takes the boundary face's flux at an
// outflow side and zero elsewhere (-1), the reference's ghost faces.
__device__ __forceinline__ int batch_xface(const Inst &I, int g) {
    const int nx = I.L.nx;
    if (I.periodic[0]) return g < 0 ? g + nx : (g > nx ? g - nx : g);
    if (g < 0) return I.bc[0] == BC_OUTFLOW ? 0 : -1;
    if (g > nx) return I.bc[1] == BC_OUTFLOW ? nx : -1;
    return g;
}

// Face flux of x-face g (between interior cells g-1 and g; g in [0, nx]) /
// y-face, z-face g (between interior g and g+1, periodic wrap) of line (j,k),
// from the stored conserved state U
template <int DIR, int INTERP, int RS>
__device__ __forceinline__ void face_flux(const BatchArgs &a, const Inst &I, const double *Uc, int g, int t1,
                                          int t2, double F[5]) {
    const Layout &L = I.L;
    const int n = DIR == 0 ? L.nx : (DIR == 1 ? L.ny : L.nz);
    long id[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        // ghost-inclusive cell along DIR: face g sits between cells (g-1+NG) and (g+NG) for x;
        // periodic directions: between g+NG and g+1+NG, stencil wrapped into [0, n+6)
        int c;
        if (DIR == 0) c = g + NG - 1 - 2 + m;
        else {
            c = g + NG - 2 + m;
            if (c < NG) c += n; else if (c >= n + NG) c -= n;
        }
        id[m] = DIR == 0 ? L.at(c, t1, t2) : (DIR == 1 ? L.at(t1, c, t2) : L.at(t1, t2, c));
    }
    // one variable's stencil at a time (WCNS_Riemann_InviscidFlux, component-wise)
    double UL[5], UR[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        double f[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) f[m] = Uc[(long)q * L.plane + id[m]];
        face_pair<double, INTERP>(a.sp, f, UL[q], UR[q]);
    }
    riemann<DIR, double, RS>(a.sp, UL, UR, F);
}

// INTERP / RS: compile-time scheme (RUNTIME: from a.sp); MINB: resident CTAs
// per SM the register allocation is sized for (one of the autotuned knobs)
template <int INTERP, int RS, int MINB>
__global__ void __launch_bounds__(256, MINB) batch_kernel(BatchArgs a) {
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int csize = (int)cluster.num_blocks();
    __shared__ int s_inst;
    __shared__ double s_red[32];
    const int tid = threadIdx.x, nth = blockDim.x;
    // minimum over the block (any multiple of 32 threads)
    auto block_min_any = [&](double x, double *out) {
        for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_down_sync(0xffffffffu, x, o));
        if ((tid & 31) == 0) s_red[tid >> 5] = x;
        __syncthreads();
        if (tid == 0) {
            double mn = s_red[0];
            for (int w = 1; w < nth / 32; ++w) mn = fmin(mn, s_red[w]);
            *out = mn;
        }
        __syncthreads();
    };

    for (;;) {
        if (crank == 0 && tid == 0) s_inst = atomicAdd(a.counter, 1);
        cluster.sync();
        const int pi = *cluster.map_shared_rank(&s_inst, 0);
        cluster.sync();  // everyone has read the leader's slot before it changes
        if (pi >= a.n_inst) return;
        const Inst I = a.inst[pi];
        const Layout &L = I.L;
        // this CTA's share of the interior x range
        const int x0 = (int)((long)L.nx * crank / csize), x1 = (int)((long)L.nx * (crank + 1) / csize);
        // the problem's arrays, addressed from one base (no pointer tables in
        // registers): array q of the list in NARR's comment at base + q * plane
        double *const P0 = a.pool + I.base;
        const long pl = L.plane;
        auto W = [&](int b, int q) { return P0 + (long)(5 * b + q) * pl; };
        auto U = [&](int b, int q) { return P0 + (long)(UOFF + 5 * b + q) * pl; };
        auto FX = [&](int q) { return P0 + (long)(15 + q) * pl; };
        auto FY = [&](int q) { return P0 + (long)(20 + q) * pl; };
        auto FZ = [&](int q) { return P0 + (long)(25 + q) * pl; };
        const int cells_yz = L.ny * L.nz;
        // this CTA's share of the ghost-inclusive x range (the end CTAs take the x ghost slabs)
        const int gx0 = crank == 0 ? 0 : x0 + NG, gx1 = crank == csize - 1 ? L.sx : x1 + NG;
        const long gcells = (long)(gx1 - gx0) * L.sy * L.sz;
        // conserved state of the initial buffer, every cell
        for (long e = tid; e < gcells; e += nth) {
            const int ci = gx0 + (int)(e % (gx1 - gx0));
            const long r2 = e / (gx1 - gx0);
            const long o = L.at(ci, (int)(r2 % L.sy), (int)(r2 / L.sy));
            double Uo[5];
            p2c_exact(W(0, 0)[o], W(0, 1)[o], W(0, 2)[o], W(0, 3)[o], W(0, 4)[o], a.gamma, Uo);
            for (int q = 0; q < 5; ++q) U(0, q)[o] = Uo[q];
        }
        cluster.sync();
        int s0 = 0;
        double t = 0.0;
        int steps = 0, status = 2;
        for (int step = 1; step <= a.max_steps; ++step) {
            if (fabs(I.t_end - t) <= 1e-12) { status = 0; break; }
            // ---- CFL: this CTA's minimum over its cells, then the cluster minimum
            double m = 1e9;
            for (long e = tid; e < (long)(x1 - x0) * cells_yz; e += nth) {
                const int i = x0 + (int)(e % (x1 - x0)), jk = (int)(e / (x1 - x0));
                const long c = L.at(i + NG, jk % L.ny + NG, jk / L.ny + NG);
                const double Us[5] = {U(s0, 0)[c], U(s0, 1)[c], U(s0, 2)[c], U(s0, 3)[c], U(s0, 4)[c]};
                m = fmin(m, cfl_bound(Us, a.gamma, I.dx));
            }
            block_min_any(m, &a.partials[(long)pi * 16 + crank]);
            cluster.sync();
            double mm = 1e9;
            for (int r = 0; r < csize; ++r) mm = fmin(mm, a.partials[(long)pi * 16 + r]);
            double dt = a.cfl * mm;
            if (t + dt > I.t_end) dt = I.t_end - t;
            if (dt <= 1e-12) { status = 1; cluster.sync(); break; }
            t += dt;
            // ---- three RK stages
            const int b1 = (s0 + 1) % 3, b2 = (s0 + 2) % 3;
            for (int stage = 1; stage <= 3; ++stage) {
                const int src = stage == 1 ? s0 : (stage == 2 ? b1 : b2);
                const int dst = stage == 2 ? b2 : b1;
                const double *const Uc = U(src, 0);
                // faces: x-faces g in [x0, x1) (+ g = nx for the last CTA), y/z faces per column
                const int gx_hi = (crank == csize - 1) ? x1 + 1 : x1;
                for (long e = tid; e < (long)(gx_hi - x0) * cells_yz; e += nth) {
                    const int g = x0 + (int)(e % (gx_hi - x0)), jk = (int)(e / (gx_hi - x0));
                    const int j = jk % L.ny, k = jk / L.ny;
                    double F[5];
                    face_flux<0, INTERP, RS>(a, I, Uc, g, j + NG, k + NG, F);
                    const long o = ((long)k * L.ny + j) * (L.nx + 1) + g;
                    for (int q = 0; q < 5; ++q) FX(q)[o] = F[q];
                }
                for (long e = tid; e < (long)(x1 - x0) * cells_yz; e += nth) {
                    const int i = x0 + (int)(e % (x1 - x0)), jk = (int)(e / (x1 - x0));
                    const int j = jk % L.ny, k = jk / L.ny;
                    double F[5];
                    const long o = ((long)k * L.ny + j) * L.nx + i;
                    face_flux<1, INTERP, RS>(a, I, Uc, j, i + NG, k + NG, F);
                    for (int q = 0; q < 5; ++q) FY(q)[o] = F[q];
                    face_flux<2, INTERP, RS>(a, I, Uc, k, i + NG, j + NG, F);
                    for (int q = 0; q < 5; ++q) FZ(q)[o] = F[q];
                }
                cluster.sync();
                // RHS + stage update of this CTA's interior cells
                for (long e = tid; e < (long)(x1 - x0) * cells_yz; e += nth) {
                    const int i = x0 + (int)(e % (x1 - x0)), jk = (int)(e / (x1 - x0));
                    const int j = jk % L.ny, k = jk / L.ny;
                    double R[5];
                    for (int q = 0; q < 5; ++q) {
                        auto fx = [&](int g) -> double {
                            g = batch_xface(I, g);
                            return g < 0 ? 0.0 : FX(q)[((long)k * L.ny + j) * (L.nx + 1) + g];
                        };
                        // cell i uses faces i-3 .. i+2 (ghost-inclusive), x-face g = f - (NG - 1)
                        auto dh = [](double f0, double f1, double f2, double f3, double f4, double f5, double ih) {
                            return ((f3 - f2) * (75.0 / 64.0) + (f4 - f1) * (-25.0 / 384.0) + (f5 - f0) * (3.0 / 640.0)) * ih;
                        };
                        double r = 0.0 - dh(fx(i - 2), fx(i - 1), fx(i), fx(i + 1), fx(i + 2), fx(i + 3), I.inv_dx);
                        auto fy = [&](int jj) {
                            jj = jj < 0 ? jj + L.ny : (jj >= L.ny ? jj - L.ny : jj);
                            return FY(q)[((long)k * L.ny + jj) * L.nx + i];
                        };
                        auto fz = [&](int kk) {
                            kk = kk < 0 ? kk + L.nz : (kk >= L.nz ? kk - L.nz : kk);
                            return FZ(q)[((long)kk * L.ny + j) * L.nx + i];
                        };
                        // periodic y/z: face jj + 1/2 between interior jj and jj+1; cell j uses jj = j-3 .. j+2
                        r = r - dh(fy(j - 3), fy(j - 2), fy(j - 1), fy(j), fy(j + 1), fy(j + 2), I.inv_dy);
                        r = r - dh(fz(k - 3), fz(k - 2), fz(k - 1), fz(k), fz(k + 1), fz(k + 2), I.inv_dz);
                        R[q] = r;
                    }
                    const long c = L.at(i + NG, j + NG, k + NG);
                    double Un[5], Wn[5], Ud[5];
                    for (int q = 0; q < 5; ++q) Un[q] = rk_combine(stage, U(s0, q)[c], Uc[q * pl + c], R[q], dt);
                    c2p_exact(Un, a.gamma, Wn);
                    // runge_kutta_3's c2p -> p2c round trip: the stored conserved state is p2c(W)
                    p2c_exact(Wn[0], Wn[1], Wn[2], Wn[3], Wn[4], a.gamma, Ud);
                    for (int q = 0; q < 5; ++q) { W(dst, q)[c] = Wn[q]; U(dst, q)[c] = Ud[q]; }
                }
                cluster.sync();
                // ghost fill of the new state: cells in this CTA's x range (and the x ghost
                // slabs for the end CTAs) that are not interior
                BcInfo b;
                for (int d = 0; d < 3; ++d) b.periodic[d] = I.periodic[d];
                for (int f = 0; f < 6; ++f) b.bc[f] = I.bc[f];
                for (long e = tid; e < gcells; e += nth) {
                    const int ci = gx0 + (int)(e % (gx1 - gx0));
                    const long r2 = e / (gx1 - gx0);
                    const int cj = (int)(r2 % L.sy), ck = (int)(r2 / L.sy);
                    int cc[3] = {ci, cj, ck};
                    if (is_interior(L, cc)) continue;
                    int flip;
                    const int kind = resolve_source(L, b, cc, flip);
                    double Wn[5];
                    if (kind != SRC_CELL) {
                        special_state(kind, Wn);
                    } else if (is_interior(L, cc)) {
                        const long s = L.at(cc[0], cc[1], cc[2]);
                        for (int q = 0; q < 5; ++q) Wn[q] = W(dst, q)[s];
                    } else {
                        // a ghost cell no fill reaches keeps its own stage update with rhs = 0
                        const long s = L.at(cc[0], cc[1], cc[2]);
                        double Un[5];
                        for (int q = 0; q < 5; ++q) Un[q] = rk_combine(stage, U(s0, q)[s], Uc[q * pl + s], 0.0, dt);
                        c2p_exact(Un, a.gamma, Wn);
                    }
                    apply_flips(flip, Wn);
                    const long o = L.at(ci, cj, ck);
                    double Ud[5];
                    p2c_exact(Wn[0], Wn[1], Wn[2], Wn[3], Wn[4], a.gamma, Ud);
                    for (int q = 0; q < 5; ++q) { W(dst, q)[o] = Wn[q]; U(dst, q)[o] = Ud[q]; }
                }
                cluster.sync();
            }
            s0 = (s0 + 1) % 3;  // stage 3 wrote b1
            steps = step;
            if (t >= I.t_end) { status = 0; break; }
        }
        if (crank == 0 && tid == 0) {
            a.t_out[pi] = t; a.steps_out[pi] = steps; a.state_out[pi] = s0; a.status_out[pi] = status;
        }
    }
}

// ------------------------------------------------- wavefront schedule
//
// Every active problem advances one step per sweep of a few flat launches:
// each launch covers the cells of all stepping problems (a table maps block
// b to a problem and a 256-cell tile of it), so the whole GPU works on every
// phase however uneven the problem sizes are, and no problem's critical path
// is bounded by the few CTAs of one cluster.  Each problem keeps its own
// time, CFL time step, step count and status; the same face, update and
// ghost-fill arithmetic as the persistent kernel, so the same bits.  Problems
// that finish stop stepping and leave the tile tables when the host next
// compacts them.
struct WaveArgs {
    const Inst *inst;
    double *pool;
    const int *tile_prob;        // block -> problem (sorted position)
    const int *tile_off;         // block -> first cell of its tile
    double cfl, gamma;
    SchemeParams<double> sp;
    unsigned long long *minbits; // per problem: bits of the CFL minimum (positive doubles order as integers)
    double *t, *dt;              // per problem
    int *steps, *status, *state_out, *stepping;
    int max_steps;
    int s0, stage;               // buffer holding the step-start state (same for all), stage 1..3
    // (problem, box cell) lists, wave_ghost_list_kernel: [0] the ghost cells a
    // stage fills, [1] the ghost cells no fill reaches that are their own
    // source, [2] those whose source is another such cell (kind 1)
    const int2 *ghosts;
    int n_ghost[3], ghost_base[3];
    int *ghost_count;            // [3]: entries found (list building)
    double *dt_hist;             // [WAVE_WINDOW][n]: dt of each step of the window, -1: did not step
    int hist_slot, n_prob;
};

// Ghost cells no fill reaches evolve by their own zero-RHS stage updates and
// are read by nothing else, so they are advanced in windows of WAVE_WINDOW
// steps (wave_unreached_kernel, registers only) from the recorded dt values
// instead of through memory at every stage.
constexpr int WAVE_WINDOW = 16;

// Problems whose cross-section has at most BRICK_COLS cells take the fused
// face + update kernel (wave_brick_kernel) on bricks of 256 / (ny nz) x-cells
// by the whole cross-section; larger cross-sections the separate kernels.
constexpr int BRICK_COLS = 64;
#ifndef NS3D_BRICK_CELLS
#define NS3D_BRICK_CELLS 512
#endif
constexpr int BRICK_CELLS = NS3D_BRICK_CELLS;  // cells per brick (256 threads: two cells each)
__host__ __device__ __forceinline__ bool brick_ok(const Layout &L) { return L.ny * L.nz <= BRICK_COLS; }
__host__ __device__ __forceinline__ int brick_width(const Layout &L) { return BRICK_CELLS / (L.ny * L.nz); }

__device__ __forceinline__ double *warr(const WaveArgs &a, const Inst &I, int q) {
    return a.pool + I.base + (long)q * I.L.plane;
}

// CFL minimum of each stepping problem over its interior cells (timestep.cpp:5-23)
__global__ void __launch_bounds__(256) wave_cfl_kernel(WaveArgs a) {
    const int p = a.tile_prob[blockIdx.x];
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    const long e = (long)a.tile_off[blockIdx.x] + threadIdx.x;
    double m = 1e9;
    if (e < (long)L.nx * L.ny * L.nz) {
        const int i = (int)(e % L.nx), jk = (int)(e / L.nx);
        const long c = L.at(i + NG, jk % L.ny + NG, jk / L.ny + NG);
        const double Us[5] = {warr(a, I, UOFF + 5 * a.s0)[c], warr(a, I, UOFF + 5 * a.s0 + 1)[c],
                              warr(a, I, UOFF + 5 * a.s0 + 2)[c], warr(a, I, UOFF + 5 * a.s0 + 3)[c],
                              warr(a, I, UOFF + 5 * a.s0 + 4)[c]};
        m = cfl_bound(Us, a.gamma, I.dx);
    }
    __shared__ double mm;
    block_min_n<256>(m, &mm);
    // the bounds are positive (or the 1e9 cap), so their bit patterns order as the values
    if (threadIdx.x == 0) atomicMin(&a.minbits[p], (unsigned long long)__double_as_longlong(mm));
}

// time_advance's schedule (maincycle.cpp:18-56) per problem, before a step
__global__ void wave_schedule_kernel(WaveArgs a, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    a.stepping[p] = 0;
    a.dt_hist[(long)a.hist_slot * n + p] = -1.0;
    if (a.status[p] != 2 || a.steps[p] >= a.max_steps) { a.minbits[p] = ~0ull; return; }  // done
    const double t = a.t[p], t_end = a.inst[p].t_end;
    const double m = __longlong_as_double((long long)a.minbits[p]);
    a.minbits[p] = ~0ull;  // reset for the next step
    if (fabs(t_end - t) <= 1e-12) { a.status[p] = 0; return; }
    double dt = a.cfl * m;
    if (t + dt > t_end) dt = t_end - t;
    if (dt <= 1e-12) { a.status[p] = 1; return; }
    a.t[p] = t + dt;
    a.dt[p] = dt;
    a.dt_hist[(long)a.hist_slot * n + p] = dt;
    a.stepping[p] = 1;
}

// after a step: the count, the end test, and where the state is
__global__ void wave_post_kernel(WaveArgs a, int n, int s_new) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || !a.stepping[p]) return;
    const int st = a.steps[p] + 1;
    a.steps[p] = st;
    a.state_out[p] = s_new;
    if (a.t[p] >= a.inst[p].t_end) a.status[p] = 0;
}

// face fluxes of the stage's state: x-face g = i (and g = nx for the last
// cell of a line), y-face j + 1/2, z-face k + 1/2 of interior cell (i, j, k)
template <int INTERP, int RS>
__global__ void __launch_bounds__(256) wave_face_kernel(WaveArgs a) {
    const int p = a.tile_prob[blockIdx.x];
    if (!a.stepping[p]) return;
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    if (brick_ok(L)) return;  // wave_brick_kernel's
    const long e = (long)a.tile_off[blockIdx.x] + threadIdx.x;
    if (e >= (long)L.nx * L.ny * L.nz) return;
    const int i = (int)(e % L.nx), jk = (int)(e / L.nx), j = jk % L.ny, k = jk / L.ny;
    const int src = a.stage == 1 ? a.s0 : (a.stage == 2 ? (a.s0 + 1) % 3 : (a.s0 + 2) % 3);
    const double *Uc = warr(a, I, UOFF + 5 * src);
    BatchArgs b;
    b.sp = a.sp;
    b.gamma = a.gamma;
    double F[5];
    face_flux<0, INTERP, RS>(b, I, Uc, i, j + NG, k + NG, F);
    long o = ((long)k * L.ny + j) * (L.nx + 1) + i;
    for (int q = 0; q < 5; ++q) warr(a, I, 15 + q)[o] = F[q];
    if (i == L.nx - 1) {
        face_flux<0, INTERP, RS>(b, I, Uc, L.nx, j + NG, k + NG, F);
        for (int q = 0; q < 5; ++q) warr(a, I, 15 + q)[o + 1] = F[q];
    }
    o = ((long)k * L.ny + j) * L.nx + i;
    face_flux<1, INTERP, RS>(b, I, Uc, j, i + NG, k + NG, F);
    for (int q = 0; q < 5; ++q) warr(a, I, 20 + q)[o] = F[q];
    face_flux<2, INTERP, RS>(b, I, Uc, k, i + NG, j + NG, F);
    for (int q = 0; q < 5; ++q) warr(a, I, 25 + q)[o] = F[q];
}

// RHS of one variable at interior cell (i, j, k) from its face fluxes: the
// 6th-order half-node difference in x, then y, then z (fx: x-face g with the
// boundary rule for g outside [0, nx]; fy / fz: periodic face index)
template <class FX, class FY, class FZ>
__device__ __forceinline__ double wave_rhs(const Inst &I, int i, int j, int k, FX fx, FY fy, FZ fz) {
    auto dh = [](double f0, double f1, double f2, double f3, double f4, double f5, double ih) {
        return ((f3 - f2) * (75.0 / 64.0) + (f4 - f1) * (-25.0 / 384.0) + (f5 - f0) * (3.0 / 640.0)) * ih;
    };
    double r = 0.0 - dh(fx(i - 2), fx(i - 1), fx(i), fx(i + 1), fx(i + 2), fx(i + 3), I.inv_dx);
    r = r - dh(fy(j - 3), fy(j - 2), fy(j - 1), fy(j), fy(j + 1), fy(j + 2), I.inv_dy);
    r = r - dh(fz(k - 3), fz(k - 2), fz(k - 1), fz(k), fz(k + 1), fz(k + 2), I.inv_dz);
    return r;
}

// the stage update of interior cell c from its RHS and runge_kutta_3's
// c2p -> p2c round trip (range_kutta.cpp:53-91)
__device__ __forceinline__ void wave_finish(const WaveArgs &a, const Inst &I, long c, int dst, int src,
                                            const double r[5], double dt) {
    double Un[5], Wn[5], Ud[5];
    for (int q = 0; q < 5; ++q)
        Un[q] = rk_combine(a.stage, warr(a, I, UOFF + 5 * a.s0 + q)[c], warr(a, I, UOFF + 5 * src + q)[c], r[q], dt);
    c2p_exact(Un, a.gamma, Wn);
    p2c_exact(Wn[0], Wn[1], Wn[2], Wn[3], Wn[4], a.gamma, Ud);
    for (int q = 0; q < 5; ++q) { warr(a, I, 5 * dst + q)[c] = Wn[q]; warr(a, I, UOFF + 5 * dst + q)[c] = Ud[q]; }
}

__device__ __forceinline__ int wave_src(const WaveArgs &a) {
    return a.stage == 1 ? a.s0 : (a.stage == 2 ? (a.s0 + 1) % 3 : (a.s0 + 2) % 3);
}
__device__ __forceinline__ int wave_dst(const WaveArgs &a) {
    return a.stage == 2 ? (a.s0 + 2) % 3 : (a.s0 + 1) % 3;
}

// RHS of interior cell (i, j, k) from the face fluxes and the stage update
__global__ void __launch_bounds__(256) wave_update_kernel(WaveArgs a) {
    const int p = a.tile_prob[blockIdx.x];
    if (!a.stepping[p]) return;
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    if (brick_ok(L)) return;  // wave_brick_kernel's
    const long e = (long)a.tile_off[blockIdx.x] + threadIdx.x;
    if (e >= (long)L.nx * L.ny * L.nz) return;
    const int i = (int)(e % L.nx), jk = (int)(e / L.nx), j = jk % L.ny, k = jk / L.ny;
    double r[5];
    for (int q = 0; q < 5; ++q) {
        const double *FX = warr(a, I, 15 + q), *FY = warr(a, I, 20 + q), *FZ = warr(a, I, 25 + q);
        auto fx = [&](int g) -> double {
            g = batch_xface(I, g);
            return g < 0 ? 0.0 : FX[((long)k * L.ny + j) * (L.nx + 1) + g];
        };
        auto fy = [&](int jj) {
            jj = jj < 0 ? jj + L.ny : (jj >= L.ny ? jj - L.ny : jj);
            return FY[((long)k * L.ny + jj) * L.nx + i];
        };
        auto fz = [&](int kk) {
            kk = kk < 0 ? kk + L.nz : (kk >= L.nz ? kk - L.nz : kk);
            return FZ[((long)kk * L.ny + j) * L.nx + i];
        };
        r[q] = wave_rhs(I, i, j, k, fx, fy, fz);
    }
    wave_finish(a, I, L.at(i + NG, j + NG, k + NG), wave_dst(a), wave_src(a), r, a.dt[p]);
}

// Faces and update of one brick -- bx = BRICK_CELLS / (ny nz) x-cells by the
// whole ny x nz cross-section of one problem -- in one kernel: the brick's
// x-faces (with the 2 + 3 faces beyond its ends the difference stencil
// needs), y-faces and z-faces go to shared memory, then the threads update
// the brick's cells from them.
// The same face_flux and update arithmetic as wave_face_kernel +
// wave_update_kernel, so the same bits, without the global face arrays'
// round trip and one launch per stage fewer.  Registers are capped for three
// resident blocks per SM (80 registers, a few spills): measured faster than
// two blocks at 98 registers on the 512-tube benchmark.
template <int INTERP, int RS>
__global__ void __launch_bounds__(256, 3) wave_brick_kernel(WaveArgs a) {
    extern __shared__ double sfl[];
    const int p = a.tile_prob[blockIdx.x];
    if (!a.stepping[p]) return;
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    const int ncol = L.ny * L.nz, x0 = a.tile_off[blockIdx.x];
    const int bx = min(brick_width(L), L.nx - x0);
    // x-faces x0-2 .. x0+bx+2; without periodic x those beyond the domain
    // follow the boundary rule in the update instead
    const bool px = I.periodic[0] != 0;
    const int gl = px ? x0 - 2 : max(0, x0 - 2), gh = px ? x0 + bx + 2 : min(L.nx, x0 + bx + 2);
    const int nfx = gh - gl + 1;
    const int ncell = bx * ncol;
    // [q][col][face] x-faces, then [q][cell] y- and z-faces (cell = i + bx (j + ny k))
    double *sX = sfl, *sY = sX + 5 * nfx * ncol, *sZ = sY + 5 * ncell;
    const int src = wave_src(a);
    const double *Uc = warr(a, I, UOFF + 5 * src);
    BatchArgs b;
    b.sp = a.sp;
    b.gamma = a.gamma;
    double F[5];
    for (int t = threadIdx.x; t < nfx * ncol; t += blockDim.x) {
        const int g = gl + t % nfx, col = t / nfx;
        face_flux<0, INTERP, RS>(b, I, Uc, batch_xface(I, g), col % L.ny + NG, col / L.ny + NG, F);
        for (int q = 0; q < 5; ++q) sX[(q * ncol + col) * nfx + (g - gl)] = F[q];
    }
    for (int t = threadIdx.x; t < ncell; t += blockDim.x) {
        const int i = x0 + t % bx, col = t / bx, j = col % L.ny, k = col / L.ny;
        face_flux<1, INTERP, RS>(b, I, Uc, j, i + NG, k + NG, F);
        for (int q = 0; q < 5; ++q) sY[q * ncell + t] = F[q];
        face_flux<2, INTERP, RS>(b, I, Uc, k, i + NG, j + NG, F);
        for (int q = 0; q < 5; ++q) sZ[q * ncell + t] = F[q];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < ncell; t += blockDim.x) {
        const int il = t % bx, col = t / bx, j = col % L.ny, k = col / L.ny, i = x0 + il;
        double r[5];
        for (int q = 0; q < 5; ++q) {
            const double *X = sX + (q * ncol + col) * nfx, *Y = sY + q * ncell, *Z = sZ + q * ncell;
            auto fx = [&](int g) -> double {
                if (!px) g = batch_xface(I, g);
                return !px && g < 0 ? 0.0 : X[g - gl];
            };
            auto fy = [&](int jj) {
                jj = jj < 0 ? jj + L.ny : (jj >= L.ny ? jj - L.ny : jj);
                return Y[il + bx * (jj + L.ny * k)];
            };
            auto fz = [&](int kk) {
                kk = kk < 0 ? kk + L.nz : (kk >= L.nz ? kk - L.nz : kk);
                return Z[il + bx * (j + L.ny * kk)];
            };
            r[q] = wave_rhs(I, i, j, k, fx, fy, fz);
        }
        wave_finish(a, I, L.at(i + NG, j + NG, k + NG), wave_dst(a), src, r, a.dt[p]);
    }
}

// shared memory of wave_brick_kernel for a problem (the largest brick)
inline size_t brick_smem(const Layout &L) {
    const int bx = std::min(brick_width(L), L.nx), ncol = L.ny * L.nz;
    return sizeof(double) * 5 * ((size_t)(bx + 5) * ncol + 2 * (size_t)bx * ncol);
}

// Within a run only two kinds of ghost cell are read: the x ghosts of
// interior lines (by the x-face stencils) and the ghosts no fill reaches (by
// their own zero-RHS update).  The others -- copies of interior cells,
// constants -- are a function of the current state alone, so one fill at the
// end of the run (wave_final_fill_kernel) gives them the values the per-stage
// fill would have left.  This kernel lists the first two kinds once per run
// (count only while list is null), in any order: each entry is filled
// independently of the others.
__global__ void __launch_bounds__(256) wave_ghost_list_kernel(WaveArgs a, int2 *list) {
    const int p = a.tile_prob[blockIdx.x];
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    const long e = (long)a.tile_off[blockIdx.x] + threadIdx.x;
    if (e >= (long)L.sx * L.sy * L.sz) return;
    int cc[3] = {(int)(e % L.sx), (int)((e / L.sx) % L.sy), (int)(e / ((long)L.sx * L.sy))};
    if (is_interior(L, cc)) return;
    const bool x_ghost_line = (cc[0] < NG || cc[0] >= L.nx + NG) && cc[1] >= NG && cc[1] < L.ny + NG &&
                              cc[2] >= NG && cc[2] < L.nz + NG;
    BcInfo b;
    for (int d = 0; d < 3; ++d) b.periodic[d] = I.periodic[d];
    for (int f = 0; f < 6; ++f) b.bc[f] = I.bc[f];
    int flip;
    const int c0[3] = {cc[0], cc[1], cc[2]};
    const int kind = resolve_source(L, b, cc, flip);
    const bool unreached = kind == SRC_CELL && !is_interior(L, cc);
    if (!x_ghost_line && !unreached) return;
    // x ghosts of interior lines always resolve to an interior cell or a constant
    const int cls = !unreached ? 0 : (cc[0] == c0[0] && cc[1] == c0[1] && cc[2] == c0[2] ? 1 : 2);
    const int slot = atomicAdd(a.ghost_count + cls, 1);
    if (list && slot < a.n_ghost[cls]) list[a.ghost_base[cls] + slot] = make_int2(p, (int)e);
}

// ghost fill of the stage's new state over the listed cells: the persistent
// kernel's ghost phase for the cells a stage reads
__global__ void __launch_bounds__(256) wave_ghost_kernel(WaveArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n_ghost[0]) return;
    const int2 pe = a.ghosts[t];
    const int p = pe.x;
    if (!a.stepping[p]) return;
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    const long e = pe.y;
    int cc[3] = {(int)(e % L.sx), (int)((e / L.sx) % L.sy), (int)(e / ((long)L.sx * L.sy))};
    const long o = L.at(cc[0], cc[1], cc[2]);
    const int dst = wave_dst(a);
    BcInfo b;
    for (int d = 0; d < 3; ++d) b.periodic[d] = I.periodic[d];
    for (int f = 0; f < 6; ++f) b.bc[f] = I.bc[f];
    int flip;
    const int kind = resolve_source(L, b, cc, flip);
    double Wn[5];
    if (kind != SRC_CELL) {
        special_state(kind, Wn);
    } else {
        const long s = L.at(cc[0], cc[1], cc[2]);
        for (int q = 0; q < 5; ++q) Wn[q] = warr(a, I, 5 * dst + q)[s];
    }
    apply_flips(flip, Wn);
    double Ud[5];
    p2c_exact(Wn[0], Wn[1], Wn[2], Wn[3], Wn[4], a.gamma, Ud);
    for (int q = 0; q < 5; ++q) { warr(a, I, 5 * dst + q)[o] = Wn[q]; warr(a, I, UOFF + 5 * dst + q)[o] = Ud[q]; }
}

// The window's steps of the ghost cells no fill reaches that are their own
// source: per step the three stage updates with rhs = 0 and runge_kutta_3's
// c2p -> p2c round trip, as every stage of the persistent kernel applies them,
// from the step-start buffer of the window (s_begin) into the buffer holding
// the problem's state at the window's end.  With rhs = 0 a stage adds
// dt * 0 = +0 whatever dt is, so a step is one fixed map of the cell's state;
// once a step returns the state it started from (bit for bit), every later
// step does too, and the loop stops there with the same result.
__global__ void __launch_bounds__(256) wave_unreached_kernel(WaveArgs a, int nsteps, int s_begin) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n_ghost[1]) return;
    const int2 pe = a.ghosts[a.ghost_base[1] + t];
    const int p = pe.x;
    if (nsteps < 1 || a.dt_hist[p] < 0.0) return;  // the problem did not step in this window
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    const long e = pe.y;
    const long o = L.at((int)(e % L.sx), (int)((e / L.sx) % L.sy), (int)(e / ((long)L.sx * L.sy)));
    double U0[5], U[5], Wn[5];
    for (int q = 0; q < 5; ++q) U0[q] = warr(a, I, UOFF + 5 * s_begin + q)[o];
    for (int w = 0; w < nsteps; ++w) {
        const double dt = a.dt_hist[(long)w * a.n_prob + p];
        if (dt < 0.0) break;
        for (int q = 0; q < 5; ++q) U[q] = U0[q];
        for (int stage = 1; stage <= 3; ++stage) {
            double Un[5];
            for (int q = 0; q < 5; ++q) Un[q] = rk_combine(stage, U0[q], U[q], 0.0, dt);
            c2p_exact(Un, a.gamma, Wn);
            p2c_exact(Wn[0], Wn[1], Wn[2], Wn[3], Wn[4], a.gamma, U);
        }
        bool same = true;
        for (int q = 0; q < 5; ++q) {
            same = same && __double_as_longlong(U[q]) == __double_as_longlong(U0[q]);
            U0[q] = U[q];
        }
        if (same) break;  // a fixed point of the step
    }
    const int buf = a.state_out[p];
    for (int q = 0; q < 5; ++q) { warr(a, I, 5 * buf + q)[o] = Wn[q]; warr(a, I, UOFF + 5 * buf + q)[o] = U0[q]; }
}

// The ghost cells no fill reaches whose source is another such cell: its last
// stage's state with the sign flips, after wave_unreached_kernel
__global__ void __launch_bounds__(256) wave_unreached_copy_kernel(WaveArgs a, int nsteps) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n_ghost[2]) return;
    const int2 pe = a.ghosts[a.ghost_base[2] + t];
    const int p = pe.x;
    if (nsteps < 1 || a.dt_hist[p] < 0.0) return;
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    const long e = pe.y;
    int cc[3] = {(int)(e % L.sx), (int)((e / L.sx) % L.sy), (int)(e / ((long)L.sx * L.sy))};
    const long o = L.at(cc[0], cc[1], cc[2]);
    BcInfo b;
    for (int d = 0; d < 3; ++d) b.periodic[d] = I.periodic[d];
    for (int f = 0; f < 6; ++f) b.bc[f] = I.bc[f];
    int flip;
    resolve_source(L, b, cc, flip);
    const long s = L.at(cc[0], cc[1], cc[2]);
    const int buf = a.state_out[p];
    double Wn[5], Ud[5];
    for (int q = 0; q < 5; ++q) Wn[q] = warr(a, I, 5 * buf + q)[s];
    apply_flips(flip, Wn);
    p2c_exact(Wn[0], Wn[1], Wn[2], Wn[3], Wn[4], a.gamma, Ud);
    for (int q = 0; q < 5; ++q) { warr(a, I, 5 * buf + q)[o] = Wn[q]; warr(a, I, UOFF + 5 * buf + q)[o] = Ud[q]; }
}

// The ghost cells the per-stage fill leaves out, once at the end of a run:
// copies of (the final state's) interior cells with their sign flips, and
// constants -- the values the last stage's fill would have given them.
__global__ void __launch_bounds__(256) wave_final_fill_kernel(WaveArgs a) {
    const int p = a.tile_prob[blockIdx.x];
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    const long e = (long)a.tile_off[blockIdx.x] + threadIdx.x;
    if (e >= (long)L.sx * L.sy * L.sz || a.steps[p] == 0) return;
    int cc[3] = {(int)(e % L.sx), (int)((e / L.sx) % L.sy), (int)(e / ((long)L.sx * L.sy))};
    if (is_interior(L, cc)) return;
    const long o = L.at(cc[0], cc[1], cc[2]);
    BcInfo b;
    for (int d = 0; d < 3; ++d) b.periodic[d] = I.periodic[d];
    for (int f = 0; f < 6; ++f) b.bc[f] = I.bc[f];
    int flip;
    const int kind = resolve_source(L, b, cc, flip);
    if (kind == SRC_CELL && !is_interior(L, cc)) return;  // evolved by its own updates
    const int buf = a.state_out[p];
    double Wn[5];
    if (kind != SRC_CELL) {
        special_state(kind, Wn);
    } else {
        const long s = L.at(cc[0], cc[1], cc[2]);
        for (int q = 0; q < 5; ++q) Wn[q] = warr(a, I, 5 * buf + q)[s];
    }
    apply_flips(flip, Wn);
    double Ud[5];
    p2c_exact(Wn[0], Wn[1], Wn[2], Wn[3], Wn[4], a.gamma, Ud);
    for (int q = 0; q < 5; ++q) { warr(a, I, 5 * buf + q)[o] = Wn[q]; warr(a, I, UOFF + 5 * buf + q)[o] = Ud[q]; }
}

// the conserved state of the initial buffer (every cell) and the per-problem
// counters, before the first step
__global__ void __launch_bounds__(256) wave_init_kernel(WaveArgs a) {
    const int p = a.tile_prob[blockIdx.x];
    const Inst &I = a.inst[p];
    const Layout &L = I.L;
    const long e = (long)a.tile_off[blockIdx.x] + threadIdx.x;
    if (e == 0) {
        a.t[p] = 0.0; a.steps[p] = 0; a.status[p] = 2; a.state_out[p] = 0; a.minbits[p] = ~0ull;
        a.stepping[p] = 0;
    }
    if (e >= (long)L.sx * L.sy * L.sz) return;
    const long o = L.at((int)(e % L.sx), (int)((e / L.sx) % L.sy), (int)(e / ((long)L.sx * L.sy)));
    double Uo[5];
    p2c_exact(warr(a, I, 0)[o], warr(a, I, 1)[o], warr(a, I, 2)[o], warr(a, I, 3)[o], warr(a, I, 4)[o], a.gamma, Uo);
    for (int q = 0; q < 5; ++q) warr(a, I, UOFF + q)[o] = Uo[q];
}

__global__ void batch_scatter_interior(const double *src, double *dst, Layout L) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.nx) return;
    dst[L.at(i + NG, j + NG, k + NG)] = src[((long)k * L.ny + j) * L.nx + i];
}

// ghost fill of one problem's freshly uploaded state (stage 0 of stage_kernel64)
__global__ void batch_fill_kernel(const double *const *Wc, double *const *Wout, Layout L, BcInfo b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.sx) return;
    int c[3] = {i, j, k};
    int flip;
    const int kind = resolve_source(L, b, c, flip);
    double W[5];
    if (kind != SRC_CELL) special_state(kind, W);
    else {
        const long s = L.at(c[0], c[1], c[2]);
        for (int q = 0; q < 5; ++q) W[q] = Wc[q][s];
        if (W[0] <= 0.0) W[0] = 1e-12;
    }
    apply_flips(flip, W);
    const long o = L.at(i, j, k);
    for (int q = 0; q < 5; ++q) Wout[q][o] = W[q];
}

}  // namespace

// =============================================================== host side

struct ns3d_batch {
    ns3d_params P;
    int n = 0;
    std::vector<Inst> inst;      // sorted by decreasing cost
    std::vector<int> order;      // user index -> sorted position
    double *pool = nullptr;      // all problem arrays
    size_t pool_bytes = 0;
    void *meta = nullptr;        // device: Inst table, counters, outputs, partials, pointer tables
    Inst *d_inst = nullptr;
    int *d_counter = nullptr, *d_steps = nullptr, *d_state = nullptr, *d_status = nullptr;
    double *d_t = nullptr, *d_partials = nullptr;
    double **d_tab = nullptr;    // scratch pointer table (10 pointers)
    cudaStream_t stream = nullptr;
    int device = 0;
    int cluster = 4, threads = 256, minb = 1;  // cluster 0: the wavefront schedule
    // wavefront schedule: per-problem counters and the tile tables
    void *wave = nullptr;
    unsigned long long *w_minbits = nullptr;
    double *w_dt = nullptr;
    int *w_stepping = nullptr, *w_tiles = nullptr;  // tiles: [interior prob | off | box prob | off | brick prob | x0]
    long w_tile_cap = 0;
    int2 *w_ghosts = nullptr;    // WaveArgs::ghosts (wave_ghost_list_kernel), built once
    int w_n_ghost[3] = {-1, 0, 0};
    int *w_ghost_count = nullptr;
    double *w_dt_hist = nullptr;
    size_t w_brick_smem = 0;     // wave_brick_kernel's dynamic shared memory (largest brick)
    cudaGraphExec_t graph = nullptr;
    int graph_max_steps = -1;
    SchemeParams<double> sp;
    std::string err;
    std::vector<double> init;    // copy of the uploaded pool (for re-runs after tuning)
};

namespace {

int bfail(ns3d_batch *b, int code, const std::string &m) {
    if (b) b->err = m;
    return code;
}

#define BCK(b, call, what)                                                                          \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return bfail(b, NS3D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

BatchArgs batch_args(ns3d_batch *b, int max_steps) {
    BatchArgs a;
    a.inst = b->d_inst; a.pool = b->pool; a.n_inst = b->n; a.counter = b->d_counter;
    a.t_out = b->d_t; a.steps_out = b->d_steps; a.state_out = b->d_state; a.status_out = b->d_status;
    a.partials = b->d_partials; a.max_steps = max_steps; a.cfl = b->P.cfl; a.gamma = b->P.gamma;
    a.sp = b->sp;
    return a;
}

typedef void (*BatchKernel)(BatchArgs);

// the instantiation for the scheme and the resident-CTA target: WENO5 + Roe
// (the shock-tube benchmark) compiled in, any other pair selected at run time
template <int MINB>
BatchKernel batch_kernel_for(const SchemeParams<double> &sp) {
    if (sp.interp == I_WENO5 && sp.riemann == R_ROE) return batch_kernel<I_WENO5, R_ROE, MINB>;
    return batch_kernel<RUNTIME, RUNTIME, MINB>;
}

BatchKernel select_kernel(const SchemeParams<double> &sp, int minb) {
    return minb >= 3 ? batch_kernel_for<3>(sp) : (minb == 2 ? batch_kernel_for<2>(sp) : batch_kernel_for<1>(sp));
}

int launch_batch(ns3d_batch *b, int max_steps, int cluster, int threads, int minb) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    BatchArgs a = batch_args(b, max_steps);
    const BatchKernel kern = select_kernel(b->sp, minb);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr; cfg.numAttrs = 1;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = b->stream;
    // persistent grid: as many clusters as fit at once (clusters pull work)
    int max_clusters = 0;
    cfg.gridDim = dim3(cluster * sms);
    if (cudaOccupancyMaxActiveClusters(&max_clusters, (void *)kern, &cfg) != cudaSuccess || max_clusters < 1) {
        cudaGetLastError();
        max_clusters = std::max(1, sms / cluster);
    }
    const int nclusters = std::min(max_clusters, b->n);
    cfg.gridDim = dim3(cluster * std::max(1, nclusters));
    BCK(b, cudaMemsetAsync(b->d_counter, 0, sizeof(int), b->stream), "counter reset");
    BCK(b, cudaLaunchKernelEx(&cfg, kern, a), "batch launch");
    return NS3D_OK;
}

WaveArgs wave_args(ns3d_batch *b, int max_steps) {
    WaveArgs a;
    a.inst = b->d_inst; a.pool = b->pool; a.cfl = b->P.cfl; a.gamma = b->P.gamma; a.sp = b->sp;
    a.minbits = b->w_minbits; a.t = b->d_t; a.dt = b->w_dt; a.steps = b->d_steps; a.status = b->d_status;
    a.state_out = b->d_state; a.stepping = b->w_stepping; a.max_steps = max_steps;
    a.s0 = 0; a.stage = 0;
    a.tile_prob = nullptr; a.tile_off = nullptr;
    a.ghosts = b->w_ghosts;
    a.ghost_count = b->w_ghost_count;
    for (int k = 0, base = 0; k < 3; ++k) {
        a.n_ghost[k] = std::max(0, b->w_n_ghost[k]);
        a.ghost_base[k] = base;
        base += a.n_ghost[k];
    }
    a.dt_hist = b->w_dt_hist;
    a.hist_slot = 0;
    a.n_prob = b->n;
    return a;
}

// Tile tables of the listed problems: 256 cells per block, interior cells
// (CFL, and faces + update of problems too wide for bricks), whole boxes
// (initial conversion, ghost list, final fill), and bricks of brick_width
// x-cells by the cross-section (wave_brick_kernel).
struct WaveTiles {
    int n_int = 0, n_box = 0, n_brick = 0;
    bool general = false;  // a listed problem takes the separate face and update kernels
};

int wave_tables(ns3d_batch *b, const std::vector<int> &probs, WaveTiles &wt) {
    std::vector<int> ip, io, bp, bo, kp, ko;
    wt.general = false;
    for (int p : probs) {
        const Layout &L = b->inst[p].L;
        const long ni = (long)L.nx * L.ny * L.nz, nb = (long)L.sx * L.sy * L.sz;
        for (long o = 0; o < ni; o += 256) { ip.push_back(p); io.push_back((int)o); }
        for (long o = 0; o < nb; o += 256) { bp.push_back(p); bo.push_back((int)o); }
        if (brick_ok(L)) {
            for (int x0 = 0; x0 < L.nx; x0 += brick_width(L)) { kp.push_back(p); ko.push_back(x0); }
        } else {
            wt.general = true;
        }
    }
    wt.n_int = (int)ip.size();
    wt.n_box = (int)bp.size();
    wt.n_brick = (int)kp.size();
    if ((long)(wt.n_int + wt.n_box + wt.n_brick) * 2 > b->w_tile_cap) return bfail(b, NS3D_ERR_STATE, "tile table capacity");
    std::vector<int> all;
    all.reserve(2 * (wt.n_int + wt.n_box + wt.n_brick));
    for (const std::vector<int> *v : {&ip, &io, &bp, &bo, &kp, &ko}) all.insert(all.end(), v->begin(), v->end());
    if (!all.empty())
        BCK(b, cudaMemcpyAsync(b->w_tiles, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream),
            "tile tables");
    BCK(b, cudaStreamSynchronize(b->stream), "synchronize");  // the host vector goes out of scope
    return NS3D_OK;
}

int ensure_wave(ns3d_batch *b) {
    if (b->wave) return NS3D_OK;
    long tiles = 0;
    size_t smem = 0;
    for (const Inst &I : b->inst) {
        const Layout &L = I.L;
        tiles += ((long)L.nx * L.ny * L.nz + 255) / 256 + ((long)L.sx * L.sy * L.sz + 255) / 256;
        if (brick_ok(L)) {
            tiles += (L.nx + brick_width(L) - 1) / brick_width(L);
            smem = std::max(smem, brick_smem(L));
        }
    }
    b->w_tile_cap = 2 * tiles;
    const size_t n = (size_t)b->n;
    const size_t bytes = n * 8 + n * 8 + n * 4 + 256 + n * 8 * WAVE_WINDOW + 256 + (size_t)b->w_tile_cap * 4 + 4 * 256;
    BCK(b, cudaMalloc(&b->wave, bytes), "wavefront tables");
    char *p = (char *)b->wave;
    b->w_minbits = (unsigned long long *)p; p += (n * 8 + 255) / 256 * 256;
    b->w_dt = (double *)p; p += (n * 8 + 255) / 256 * 256;
    b->w_stepping = (int *)p; p += (n * 4 + 255) / 256 * 256;
    b->w_ghost_count = (int *)p; p += 256;
    b->w_dt_hist = (double *)p; p += (n * 8 * WAVE_WINDOW + 255) / 256 * 256;
    b->w_tiles = (int *)p;
    b->w_brick_smem = smem;
    if (smem > 48 * 1024) {
        BCK(b, cudaFuncSetAttribute(wave_brick_kernel<I_WENO5, R_ROE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
            "brick shared memory");
        BCK(b, cudaFuncSetAttribute(wave_brick_kernel<RUNTIME, RUNTIME>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem),
            "brick shared memory");
    }
    return NS3D_OK;
}

// the ghost-cell lists (once per batch: they depend on the layouts and
// boundary types only); the box tiles of every problem are set
int build_ghost_list(ns3d_batch *b, WaveArgs &a, int n_box) {
    if (b->w_n_ghost[0] >= 0) return NS3D_OK;
    int count[3] = {0, 0, 0};
    for (int pass = 0; pass < 2; ++pass) {
        BCK(b, cudaMemsetAsync(b->w_ghost_count, 0, 3 * sizeof(int), b->stream), "ghost count");
        a.ghost_count = b->w_ghost_count;
        for (int k = 0, base = 0; k < 3; ++k) { a.n_ghost[k] = count[k]; a.ghost_base[k] = base; base += count[k]; }
        wave_ghost_list_kernel<<<n_box, 256, 0, b->stream>>>(a, pass ? b->w_ghosts : nullptr);
        BCK(b, cudaGetLastError(), "ghost list");
        BCK(b, cudaMemcpyAsync(count, b->w_ghost_count, 3 * sizeof(int), cudaMemcpyDeviceToHost, b->stream),
            "ghost count");
        BCK(b, cudaStreamSynchronize(b->stream), "synchronize");
        const size_t total = (size_t)count[0] + count[1] + count[2];
        if (pass == 0 && total == 0) break;
        if (pass == 0) BCK(b, cudaMalloc(&b->w_ghosts, sizeof(int2) * total), "ghost list");
    }
    for (int k = 0; k < 3; ++k) b->w_n_ghost[k] = count[k];
    a = wave_args(b, a.max_steps);
    return NS3D_OK;
}

// The wavefront schedule to every problem's t_end (or max_steps): one step of
// every active problem per round of launches; every 16 steps the host reads
// the statuses and drops the finished problems from the tile tables.
int run_wave(ns3d_batch *b, int max_steps) {
    int r = ensure_wave(b);
    if (r) return r;
    WaveArgs a = wave_args(b, max_steps);
    std::vector<int> active(b->n);
    for (int p = 0; p < b->n; ++p) active[p] = p;
    WaveTiles wt;
    if ((r = wave_tables(b, active, wt))) return r;
    // table views: 0 interior, 1 box, 2 brick
    auto set_tables = [&](int which) {
        const int off[3] = {0, 2 * wt.n_int, 2 * (wt.n_int + wt.n_box)};
        const int len[3] = {wt.n_int, wt.n_box, wt.n_brick};
        a.tile_prob = b->w_tiles + off[which];
        a.tile_off = b->w_tiles + off[which] + len[which];
    };
    set_tables(1);
    wave_init_kernel<<<wt.n_box, 256, 0, b->stream>>>(a);
    BCK(b, cudaGetLastError(), "wavefront init");
    if ((r = build_ghost_list(b, a, wt.n_box))) return r;
    set_tables(1);
    const unsigned pblocks = (unsigned)((b->n + 127) / 128);
    const unsigned gblocks = (unsigned)((a.n_ghost[0] + 255) / 256);
    // the unreached ghost cells' steps since the last catch-up, from the
    // step-start buffer at that point
    int s_begin = 0, wsteps = 0;
    auto catch_up = [&]() {
        if (wsteps == 0) return;
        if (a.n_ghost[1]) wave_unreached_kernel<<<(a.n_ghost[1] + 255) / 256, 256, 0, b->stream>>>(a, wsteps, s_begin);
        if (a.n_ghost[2]) wave_unreached_copy_kernel<<<(a.n_ghost[2] + 255) / 256, 256, 0, b->stream>>>(a, wsteps);
        wsteps = 0;
    };
    const bool weno_roe = b->sp.interp == I_WENO5 && b->sp.riemann == R_ROE;
    std::vector<int> status(b->n), steps(b->n);
    int s0 = 0;
    for (int step = 0; step < max_steps; ++step) {
        if (step > 0 && step % WAVE_WINDOW == 0) {
            catch_up();
            s_begin = s0;
            BCK(b, cudaMemcpyAsync(status.data(), b->d_status, sizeof(int) * b->n, cudaMemcpyDeviceToHost, b->stream),
                "statuses");
            BCK(b, cudaMemcpyAsync(steps.data(), b->d_steps, sizeof(int) * b->n, cudaMemcpyDeviceToHost, b->stream),
                "steps");
            BCK(b, cudaStreamSynchronize(b->stream), "synchronize");
            std::vector<int> act;
            for (int p : active)
                if (status[p] == 2 && steps[p] < max_steps) act.push_back(p);
            if (act.empty()) break;
            if (act.size() != active.size()) {
                active.swap(act);
                if ((r = wave_tables(b, active, wt))) return r;
            }
        }
        a.s0 = s0;
        a.hist_slot = wsteps;
        set_tables(0);
        wave_cfl_kernel<<<wt.n_int, 256, 0, b->stream>>>(a);
        wave_schedule_kernel<<<pblocks, 128, 0, b->stream>>>(a, b->n);
        for (int stage = 1; stage <= 3; ++stage) {
            a.stage = stage;
            if (wt.n_brick) {
                set_tables(2);
                if (weno_roe) wave_brick_kernel<I_WENO5, R_ROE><<<wt.n_brick, 256, b->w_brick_smem, b->stream>>>(a);
                else wave_brick_kernel<RUNTIME, RUNTIME><<<wt.n_brick, 256, b->w_brick_smem, b->stream>>>(a);
            }
            if (wt.general) {
                set_tables(0);
                if (weno_roe) wave_face_kernel<I_WENO5, R_ROE><<<wt.n_int, 256, 0, b->stream>>>(a);
                else wave_face_kernel<RUNTIME, RUNTIME><<<wt.n_int, 256, 0, b->stream>>>(a);
                wave_update_kernel<<<wt.n_int, 256, 0, b->stream>>>(a);
            }
            if (gblocks) wave_ghost_kernel<<<gblocks, 256, 0, b->stream>>>(a);
        }
        s0 = (s0 + 1) % 3;
        wave_post_kernel<<<pblocks, 128, 0, b->stream>>>(a, b->n, s0);
        BCK(b, cudaGetLastError(), "wavefront step");
        ++wsteps;
    }
    catch_up();
    // the ghost cells left out of the per-stage fills, every problem
    std::vector<int> all(b->n);
    for (int p = 0; p < b->n; ++p) all[p] = p;
    if ((r = wave_tables(b, all, wt))) return r;
    set_tables(1);
    wave_final_fill_kernel<<<wt.n_box, 256, 0, b->stream>>>(a);
    BCK(b, cudaGetLastError(), "final ghost fill");
    BCK(b, cudaStreamSynchronize(b->stream), "synchronize");
    return NS3D_OK;
}

}  // namespace

extern "C" {

int ns3d_batch_create(const ns3d_params *params, int n_inst, const ns3d_grid *grids, const double *t_end,
                      ns3d_batch **out) {
    if (!params || !grids || !t_end || !out || n_inst < 1) return NS3D_ERR_INVALID_ARG;
    *out = nullptr;
    if (params->precision != NS3D_FP64 || params->char_recon) return NS3D_ERR_CONFIG;
    if (params->interpolation == NS3D_ZERO || params->interpolation < 0 || params->interpolation > 3) return NS3D_ERR_CONFIG;
    if (params->riemann_solver < 0 || params->riemann_solver > 6) return NS3D_ERR_CONFIG;
    if (!std::isinf(params->Re)) return NS3D_ERR_CONFIG;  // batched problems are inviscid (Re = inf)
    // y and z must be periodic (the quasi-1D cross-section); x takes any boundary type
    for (int f = 2; f < 6; ++f)
        if (params->bc[f] != NS3D_PERIODIC) return NS3D_ERR_CONFIG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NS3D_ERR_NO_DEVICE;
    ns3d_batch *b = new (std::nothrow) ns3d_batch();
    if (!b) return NS3D_ERR_OOM;
    b->P = *params;
    b->n = n_inst;
    b->device = params->device;
    cudaSetDevice(b->device);
    // cost ~ nx^2 * ny * nz (cells x steps); sort decreasing
    std::vector<int> idx(n_inst);
    for (int i = 0; i < n_inst; ++i) {
        const ns3d_grid &g = grids[i];
        if (g.nx < 3 || g.ny < 3 || g.nz < 3 || !(t_end[i] > 0)) { delete b; return NS3D_ERR_INVALID_ARG; }
        idx[i] = i;
    }
    std::stable_sort(idx.begin(), idx.end(), [&](int p, int q) {
        double cp = (double)grids[p].nx * grids[p].nx * grids[p].ny * grids[p].nz;
        double cq = (double)grids[q].nx * grids[q].nx * grids[q].ny * grids[q].nz;
        return cp > cq;
    });
    b->order.assign(n_inst, 0);
    long base = 0;
    for (int s = 0; s < n_inst; ++s) {
        const int u = idx[s];
        b->order[u] = s;
        const ns3d_grid &g = grids[u];
        Inst I;
        I.L = make_layout<double>(g.nx, g.ny, g.nz);
        // face arrays need (nx+1)*ny*nz <= plane: true since plane >= (nx+6)*(ny+6)*(nz+6)
        I.base = base;
        base += (long)NARR * I.L.plane;
        I.dx = g.Lx / g.nx; I.dy = g.Ly / g.ny; I.dz = g.Lz / g.nz;
        I.inv_dx = 1.0 / I.dx; I.inv_dy = 1.0 / I.dy; I.inv_dz = 1.0 / I.dz;
        I.t_end = t_end[u];
        for (int f = 0; f < 6; ++f) I.bc[f] = params->bc[f];
        for (int d = 0; d < 3; ++d) I.periodic[d] = params->bc[2 * d] == NS3D_PERIODIC && params->bc[2 * d + 1] == NS3D_PERIODIC;
        b->inst.push_back(I);
    }
    b->pool_bytes = (size_t)base * 8;
    const size_t meta_bytes = sizeof(Inst) * n_inst + 4 * 256 + (size_t)n_inst * (8 + 3 * 4) + (size_t)n_inst * 16 * 8 + 1024;
    if (cudaMalloc(&b->pool, b->pool_bytes) != cudaSuccess || cudaMalloc(&b->meta, meta_bytes) != cudaSuccess) {
        cudaGetLastError();
        if (b->pool) cudaFree(b->pool);
        delete b;
        return NS3D_ERR_OOM;
    }
    char *p = (char *)b->meta;
    b->d_inst = (Inst *)p; p += ((sizeof(Inst) * n_inst + 255) / 256) * 256;
    b->d_counter = (int *)p; p += 256;
    b->d_t = (double *)p; p += ((size_t)n_inst * 8 + 255) / 256 * 256;
    b->d_steps = (int *)p; p += ((size_t)n_inst * 4 + 255) / 256 * 256;
    b->d_state = (int *)p; p += ((size_t)n_inst * 4 + 255) / 256 * 256;
    b->d_status = (int *)p; p += ((size_t)n_inst * 4 + 255) / 256 * 256;
    b->d_partials = (double *)p; p += ((size_t)n_inst * 16 * 8 + 255) / 256 * 256;
    b->d_tab = (double **)p;
    cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    cudaMemcpy(b->d_inst, b->inst.data(), sizeof(Inst) * n_inst, cudaMemcpyHostToDevice);
    cudaMemset(b->pool, 0, b->pool_bytes);
    // Field3D::allocate defaults: rho = 1 in every buffer
    std::vector<double> ones;
    for (int s = 0; s < n_inst; ++s) {
        const Inst &I = b->inst[s];
        ones.assign(I.L.plane, 1.0);
        for (int buf = 0; buf < 3; ++buf)
            cudaMemcpy(b->pool + I.base + (long)(5 * buf) * I.L.plane, ones.data(), I.L.plane * 8, cudaMemcpyHostToDevice);
    }
    // scheme constants (interpolation.cpp:130-132, 179-182)
    const double disp = params->mdcd_disp, diss = params->mdcd_diss;
    const double lin[6] = {(3.0 * disp + 3.0 * diss) / 8.0, (-18.0 * disp - 30 * diss - 1.0) / 16.0,
                           (12.0 * disp + 60.0 * diss + 9.0) / 16.0, (12.0 * disp - 60.0 * diss + 9.0) / 16.0,
                           (-18.0 * disp + 30.0 * diss - 1.0) / 16.0, (3.0 * disp - 3.0 * diss) / 8.0};
    const double hd[4] = {1.5 * (disp + diss), 0.5 - 1.5 * (disp - 3 * diss), 0.5 - 1.5 * (disp + 3 * diss),
                          1.5 * (disp - diss)};
    b->sp.gamma = params->gamma;
    for (int q = 0; q < 6; ++q) b->sp.lin[q] = lin[q];
    for (int q = 0; q < 4; ++q) b->sp.hd[q] = hd[q];
    b->sp.interp = params->interpolation; b->sp.riemann = params->riemann_solver; b->sp.char_recon = 0;
    if (cudaDeviceSynchronize() != cudaSuccess) { ns3d_batch_destroy(b); return NS3D_ERR_CUDA; }
    *out = b;
    return NS3D_OK;
}

int ns3d_batch_destroy(ns3d_batch *b) {
    if (!b) return NS3D_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->stream) { cudaStreamSynchronize(b->stream); cudaStreamDestroy(b->stream); }
    if (b->pool) cudaFree(b->pool);
    if (b->meta) cudaFree(b->meta);
    if (b->wave) cudaFree(b->wave);
    if (b->w_ghosts) cudaFree(b->w_ghosts);
    delete b;
    return NS3D_OK;
}

const char *ns3d_batch_last_error(const ns3d_batch *b) { return b ? b->err.c_str() : "null batch"; }

int ns3d_batch_set_interior_primitives(ns3d_batch *b, int problem, const double *const fields[5]) {
    if (!b || !fields || problem < 0 || problem >= b->n) return NS3D_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    const Inst &I = b->inst[b->order[problem]];
    const Layout &L = I.L;
    const size_t nb = (size_t)L.nx * L.ny * L.nz * 8;
    double *W0[5], *W1[5], *stg = b->pool + I.base + 15L * L.plane;  // face-flux area as staging
    for (int q = 0; q < 5; ++q) { W0[q] = b->pool + I.base + (long)q * L.plane; W1[q] = b->pool + I.base + (long)(5 + q) * L.plane; }
    for (int q = 0; q < 5; ++q) {
        BCK(b, cudaMemcpyAsync(stg, fields[q], nb, cudaMemcpyHostToDevice, b->stream), "upload");
        batch_scatter_interior<<<dim3((L.nx + 127) / 128, L.ny, L.nz), 128, 0, b->stream>>>(stg, W1[q], L);
    }
    // ghost fill (apply_boundary + primitiveToConserved, main.cpp:98-99) into buffer 0
    BcInfo bi;
    for (int d = 0; d < 3; ++d) bi.periodic[d] = I.periodic[d];
    for (int f = 0; f < 6; ++f) bi.bc[f] = I.bc[f];
    BCK(b, cudaMemcpyAsync(b->d_tab, W1, sizeof(W1), cudaMemcpyHostToDevice, b->stream), "table");
    BCK(b, cudaMemcpyAsync(b->d_tab + 5, W0, sizeof(W0), cudaMemcpyHostToDevice, b->stream), "table");
    batch_fill_kernel<<<dim3((L.sx + 127) / 128, L.sy, L.sz), 128, 0, b->stream>>>(b->d_tab, b->d_tab + 5, L, bi);
    BCK(b, cudaGetLastError(), "fill");
    BCK(b, cudaStreamSynchronize(b->stream), "synchronize");
    return NS3D_OK;
}

int ns3d_batch_run(ns3d_batch *b, int max_steps) {
    if (!b || max_steps < 1) return NS3D_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    if (b->cluster == 0) return run_wave(b, max_steps);
    if (!b->graph || b->graph_max_steps != max_steps) {
        if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
        cudaGraph_t g;
        BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "capture");
        int r = launch_batch(b, max_steps, b->cluster, b->threads, b->minb);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (r) return r;
        if (e != cudaSuccess) return bfail(b, NS3D_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return bfail(b, NS3D_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
        b->graph_max_steps = max_steps;
    }
    BCK(b, cudaGraphLaunch(b->graph, b->stream), "graph launch");
    BCK(b, cudaStreamSynchronize(b->stream), "synchronize");
    return NS3D_OK;
}

int ns3d_batch_autotune(ns3d_batch *b, int trial_steps, int out[3]) {
    if (!b || trial_steps < 1) return NS3D_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    // save the state (a device copy), try each configuration for trial_steps
    // steps -- cluster size, CTA width and resident CTAs per SM (the register
    // budget of the instantiation) -- and restore
    double *save = nullptr;
    BCK(b, cudaMalloc(&save, b->pool_bytes), "autotune save buffer");
    cudaError_t se = cudaMemcpyAsync(save, b->pool, b->pool_bytes, cudaMemcpyDeviceToDevice, b->stream);
    if (se != cudaSuccess) { cudaFree(save); return bfail(b, NS3D_ERR_CUDA, "autotune save"); }
    // cluster 0: the wavefront schedule (one configuration)
    const int clusters[5] = {0, 1, 2, 4, 8}, widths[2] = {128, 256}, minbs[3] = {1, 2, 3};
    float best = 1e30f;
    int bc = b->cluster, bw = b->threads, bm = b->minb;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    for (int ci = 0; ci < 5; ++ci)
        for (int wi = 0; wi < 2; ++wi)
            for (int mi = 0; mi < 3; ++mi) {
                if (clusters[ci] == 0 && (wi || mi)) continue;
                if (cudaMemcpyAsync(b->pool, save, b->pool_bytes, cudaMemcpyDeviceToDevice, b->stream) != cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                cudaEventRecord(e0, b->stream);
                int r = clusters[ci] == 0 ? run_wave(b, trial_steps)
                                          : launch_batch(b, trial_steps, clusters[ci], widths[wi], minbs[mi]);
                cudaEventRecord(e1, b->stream);
                if (r || cudaStreamSynchronize(b->stream) != cudaSuccess) { cudaGetLastError(); continue; }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) {
                    best = ms;
                    bc = clusters[ci]; bw = clusters[ci] ? widths[wi] : 256; bm = clusters[ci] ? minbs[mi] : 1;
                }
            }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    se = cudaMemcpyAsync(b->pool, save, b->pool_bytes, cudaMemcpyDeviceToDevice, b->stream);
    if (se == cudaSuccess) se = cudaStreamSynchronize(b->stream);
    cudaFree(save);
    if (se != cudaSuccess) return bfail(b, NS3D_ERR_CUDA, "autotune restore");
    b->cluster = bc; b->threads = bw; b->minb = bm;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    if (out) { out[0] = bc; out[1] = bw; out[2] = bm; }
    return NS3D_OK;
}

int ns3d_batch_set_config(ns3d_batch *b, int cluster, int threads, int ctas_per_sm) {
    if (!b || (cluster != 0 && cluster != 1 && cluster != 2 && cluster != 4 && cluster != 8) ||
        (threads != 128 && threads != 256) || ctas_per_sm < 1 || ctas_per_sm > 3)
        return NS3D_ERR_INVALID_ARG;
    b->cluster = cluster; b->threads = threads; b->minb = ctas_per_sm;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    return NS3D_OK;
}

int ns3d_batch_query(ns3d_batch *b, int problem, double *time, int *steps, int *status) {
    if (!b || problem < 0 || problem >= b->n) return NS3D_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    const int s = b->order[problem];
    double t = 0; int st = 0, stat = 0;
    BCK(b, cudaMemcpy(&t, b->d_t + s, 8, cudaMemcpyDeviceToHost), "query");
    BCK(b, cudaMemcpy(&st, b->d_steps + s, 4, cudaMemcpyDeviceToHost), "query");
    BCK(b, cudaMemcpy(&stat, b->d_status + s, 4, cudaMemcpyDeviceToHost), "query");
    if (time) *time = t;
    if (steps) *steps = st;
    if (status) *status = stat;
    return NS3D_OK;
}

// Primitive (rho,u,v,w,p) Field3D arrays of problem i after ns3d_batch_run.
int ns3d_batch_download(ns3d_batch *b, int problem, double *const out[5]) {
    if (!b || !out || problem < 0 || problem >= b->n) return NS3D_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    const int s = b->order[problem];
    const Inst &I = b->inst[s];
    int buf = 0;
    BCK(b, cudaMemcpy(&buf, b->d_state + s, 4, cudaMemcpyDeviceToHost), "query");
    if (buf < 0 || buf > 2) buf = 0;
    const Layout &L = I.L;
    for (int q = 0; q < 5; ++q) {
        const double *src = b->pool + I.base + (long)(5 * buf + q) * L.plane;
        BCK(b, cudaMemcpy2D(out[q], (size_t)L.sx * 8, src + L.off, (size_t)L.px * 8, (size_t)L.sx * 8,
                            (size_t)L.sy * L.sz, cudaMemcpyDeviceToHost), "download");
    }
    return NS3D_OK;
}

}  // extern "C"
