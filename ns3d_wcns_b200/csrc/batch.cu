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

// Face flux of x-face g (between interior cells g-1 and g; g in [0, nx]) /
// y-face, z-face g (between interior g and g+1, periodic wrap) of line (j,k),
// from the stored conserved state U
template <int DIR, int INTERP, int RS>
__device__ __forceinline__ void face_flux(const BatchArgs &a, const Inst &I, const double *Uc, int g, int t1,
                                          int t2, double F[5]) {
    const Layout &L = I.L;
    const int n = DIR == 0 ? L.nx : (DIR == 1 ? L.ny : L.nz);
    double st[5][6];
    for (int m = 0; m < 6; ++m) {
        // ghost-inclusive cell along DIR: face g sits between cells (g-1+NG) and (g+NG) for x;
        // periodic directions: between g+NG and g+1+NG, stencil wrapped into [0, n+6)
        int c;
        if (DIR == 0) c = g + NG - 1 - 2 + m;
        else {
            c = g + NG - 2 + m;
            if (c < NG) c += n; else if (c >= n + NG) c -= n;
        }
        long id = DIR == 0 ? L.at(c, t1, t2) : (DIR == 1 ? L.at(t1, c, t2) : L.at(t1, t2, c));
        for (int q = 0; q < 5; ++q) st[q][m] = Uc[(long)q * L.plane + id];
    }
    double wi[5] = {0, 0, 0, 0, 0};
    wcns_face<DIR, double, INTERP, RS, 0>(a.sp, st, wi, wi, F);
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
                            if (g < 0) { if (I.bc[0] == BC_OUTFLOW) g = 0; else return 0.0; }
                            if (g > L.nx) { if (I.bc[1] == BC_OUTFLOW) g = L.nx; else return 0.0; }
                            return FX(q)[((long)k * L.ny + j) * (L.nx + 1) + g];
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
    int cluster = 4, threads = 256, minb = 1;
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

int ns3d_batch_autotune(ns3d_batch *b, int trial_steps, int out[2]) {
    if (!b || trial_steps < 1) return NS3D_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    // save the state (a device copy), try each configuration for trial_steps
    // steps -- cluster size, CTA width and resident CTAs per SM (the register
    // budget of the instantiation) -- and restore
    double *save = nullptr;
    BCK(b, cudaMalloc(&save, b->pool_bytes), "autotune save buffer");
    cudaError_t se = cudaMemcpyAsync(save, b->pool, b->pool_bytes, cudaMemcpyDeviceToDevice, b->stream);
    if (se != cudaSuccess) { cudaFree(save); return bfail(b, NS3D_ERR_CUDA, "autotune save"); }
    const int clusters[4] = {1, 2, 4, 8}, widths[2] = {128, 256}, minbs[3] = {1, 2, 3};
    float best = 1e30f;
    int bc = b->cluster, bw = b->threads, bm = b->minb;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    for (int ci = 0; ci < 4; ++ci)
        for (int wi = 0; wi < 2; ++wi)
            for (int mi = 0; mi < 3; ++mi) {
                if (cudaMemcpyAsync(b->pool, save, b->pool_bytes, cudaMemcpyDeviceToDevice, b->stream) != cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                cudaEventRecord(e0, b->stream);
                int r = launch_batch(b, trial_steps, clusters[ci], widths[wi], minbs[mi]);
                cudaEventRecord(e1, b->stream);
                if (r || cudaStreamSynchronize(b->stream) != cudaSuccess) { cudaGetLastError(); continue; }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) { best = ms; bc = clusters[ci]; bw = widths[wi]; bm = minbs[mi]; }
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
    if (!b || (cluster != 1 && cluster != 2 && cluster != 4 && cluster != 8) || (threads != 128 && threads != 256) ||
        ctas_per_sm < 1 || ctas_per_sm > 3)
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
