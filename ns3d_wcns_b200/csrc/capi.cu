// capi.cu -- the C ABI (include/ns3d_b200.h): handle, device memory, launch
// sequencing of compute_rhs / runge_kutta_3 / compute_timestep /
// compute_total_energy, and the reductions.
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ns3d_b200.h"
#include "isotropic.cuh"
#include "adjoint_api.cuh"
#include "common.cuh"
#include "schemes.cuh"
#include "stage.cuh"
#include "sweep.cuh"
#include "viscous.cuh"

using namespace ns3d;

// --------------------------------------------------------------- reductions

// Sums over interior cells: [0] KE (0.5 rho |u|^2 dV, postprocess.cpp:119-122),
// [1] sum |grad u|^2, [2] sum mu(T), [3] sum rho, [4] sum |u|^2.
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) diag_kernel(ViscArgs<R> a, double vol, double *partials, int zlo,
                                                            int nzo) {
    const Layout &L = a.L;
    const long ncell = (long)L.nx * L.ny * nzo;
    double acc[5] = {0, 0, 0, 0, 0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % L.nx), j = (int)((t / L.nx) % L.ny), k = zlo + (int)(t / ((long)L.nx * L.ny));
        const long c = L.at(i + NG, j + NG, k + NG);
        const double rho = a.W[0][c], u = a.W[1][c], v = a.W[2][c], w = a.W[3][c];
        const double kinetic = 0.5 * rho * (u * u + v * v + w * w);
        acc[0] += kinetic * vol;
        R g[12];
        node_gradients(a, i + NG, j + NG, k + NG, g);
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) s += (double)g[q] * (double)g[q];
        acc[1] += s;
        const double T = (double)a.T[c];
        acc[2] += sutherland((double)a.mu0, (double)a.S, T);
        acc[3] += rho;
        acc[4] += u * u + v * v + w * w;
    }
    block_sum<5>(acc, partials + 5 * blockIdx.x);
}

// Minimum CFL bound over interior cells (compute_timestep, timestep.cpp:5-23).
__global__ void __launch_bounds__(RED_THREADS) dt_kernel64(const double *const *Wp, Layout L, double gamma,
                                                           double dx, double *partials, int zlo, int nzo) {
    const long ncell = (long)L.nx * L.ny * nzo;
    double m = 1e9;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % L.nx), j = (int)((t / L.nx) % L.ny), k = zlo + (int)(t / ((long)L.nx * L.ny));
        const long c = L.at(i + NG, j + NG, k + NG);
        double U[5];
        p2c_exact(Wp[0][c], Wp[1][c], Wp[2][c], Wp[3][c], Wp[4][c], gamma, U);
        m = fmin(m, cfl_bound(U, gamma, dx));
    }
    block_min(m, partials + blockIdx.x);
}

__global__ void __launch_bounds__(RED_THREADS) dt_kernel_mixed(const double *const *Up, Layout L, double gamma,
                                                               double dx, double *partials, int zlo, int nzo) {
    const long ncell = (long)L.nx * L.ny * nzo;
    double m = 1e9;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % L.nx), j = (int)((t / L.nx) % L.ny), k = zlo + (int)(t / ((long)L.nx * L.ny));
        const long c = L.at(i + NG, j + NG, k + NG);
        double U[5] = {Up[0][c], Up[1][c], Up[2][c], Up[3][c], Up[4][c]};
        m = fmin(m, cfl_bound(U, gamma, dx));
    }
    block_min(m, partials + blockIdx.x);
}

// Sum of n partials, deterministic: each block of 256 threads sums a strided
// share into out[blockIdx.x] in a fixed order (a second launch with one block
// finishes).
__global__ void __launch_bounds__(256) sum_combine_kernel(const double *part, long n, double *out) {
    double s = 0.0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) s += part[t];
    double v[1] = {s};
    block_sum<1>(v, out + blockIdx.x);
}

// One step of time_advance's dt schedule (maincycle.cpp:18-56) on the
// device, same operations as the host loop: stop when |t_end - t| <= eps, when
// the previous step reached t_end or when the step budget is spent; dt from the
// CFL minimum (adaptive) or dt_fixed, clipped to t_end; dt <= eps is the
// reference's error.
__global__ void schedule_kernel(DevClock *c, double cfl, double dt_fixed, double eps) {
    if (c->done) return;
    if (c->steps >= c->budget || fabs(c->t_end - c->t) <= eps || (c->steps > 0 && c->t >= c->t_end)) {
        c->done = 1;
        return;
    }
    double dt = dt_fixed >= 0.0 ? dt_fixed : cfl * c->cfl_min;
    if (c->t + dt > c->t_end) dt = c->t_end - c->t;
    if (dt <= eps) {
        c->done = 1;
        c->err = 1;
        return;
    }
    c->t += dt;
    c->dt = dt;
    c->steps += 1;
}

// Minimum of n partials: each block of 256 threads reduces a strided share
// into out[blockIdx.x] (a second launch with one block finishes).
__global__ void __launch_bounds__(256) min_combine_kernel(const double *part, long n, double *out) {
    double m = 1e9;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
        m = fmin(m, part[t]);
    block_min_n<256>(m, out + blockIdx.x);
}

// Non-finite / non-positive state detector: counts interior cells with a
// non-finite value or rho <= 0 or p <= 0.
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) check_kernel(const R *const *Wp, Layout L, double *partials, int zlo,
                                                             int nzo) {
    const long ncell = (long)L.nx * L.ny * nzo;
    double bad = 0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % L.nx), j = (int)((t / L.nx) % L.ny), k = zlo + (int)(t / ((long)L.nx * L.ny));
        const long c = L.at(i + NG, j + NG, k + NG);
        bool ok = true;
#pragma unroll
        for (int q = 0; q < 5; ++q) ok = ok && isfinite((double)Wp[q][c]);
        ok = ok && Wp[0][c] > R(0) && Wp[4][c] > R(0);
        bad += ok ? 0.0 : 1.0;
    }
    double v[1] = {bad};
    block_sum<1>(v, partials + blockIdx.x);
}

// Residual norms of a step (compute_diagnostics, postprocess.cpp:7-98, with
// Field3D::updateResiduals, field_structures.h:500-508): per conserved
// variable, the sum over interior cells of (U - U0)^2 dx^3 and the largest
// |U|, U the state after the step and U0 the state it started from (plain
// path: both the exact p2c of the stored primitives, so the same bits as the
// reference's arrays; mixed path: the stored FP64 conserved states).
template <bool MIXED>
__global__ void __launch_bounds__(RED_THREADS) residual_kernel(const double *const *Sn, const double *const *S0,
                                                               Layout L, double gamma, double dx3,
                                                               double *partials, int zlo, int nzo) {
    const long ncell = (long)L.nx * L.ny * nzo;
    double sq[5] = {0, 0, 0, 0, 0}, mx[5] = {0, 0, 0, 0, 0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % L.nx), j = (int)((t / L.nx) % L.ny), k = zlo + (int)(t / ((long)L.nx * L.ny));
        const long c = L.at(i + NG, j + NG, k + NG);
        double U[5], U0[5];
        if constexpr (MIXED) {
#pragma unroll
            for (int q = 0; q < 5; ++q) { U[q] = Sn[q][c]; U0[q] = S0[q][c]; }
        } else {
            p2c_exact(Sn[0][c], Sn[1][c], Sn[2][c], Sn[3][c], Sn[4][c], gamma, U);
            p2c_exact(S0[0][c], S0[1][c], S0[2][c], S0[3][c], S0[4][c], gamma, U0);
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double r = U[q] - U0[q];
            sq[q] += r * r * dx3;
            mx[q] = fmax(mx[q], fabs(U[q]));
        }
    }
    block_sum_max<5>(sq, mx, partials + 10 * blockIdx.x);
}

// Fixed-order combination of the residual partials: sums of values 0-4,
// maxima of values 5-9.
__global__ void residual_combine_kernel(const double *partials, int nblocks, double *out) {
    if (threadIdx.x >= 10) return;
    const int q = threadIdx.x;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        const double x = partials[(long)b * 10 + q];
        s = q < 5 ? s + x : fmax(s, x);
    }
    out[q] = s;
}

// Fixed-order combination of per-block partials (nv values per block).
// mode 0: sums, mode 1: minimum of value 0.
__global__ void combine_kernel(const double *partials, int nblocks, int nv, int mode, double *out) {
    if (threadIdx.x >= nv) return;
    const int q = threadIdx.x;
    double s = mode == 1 ? 1e300 : 0.0;
    for (int b = 0; b < nblocks; ++b) {
        const double x = partials[(long)b * nv + q];
        s = mode == 1 ? fmin(s, x) : s + x;
    }
    out[q] = s;
}

// Interior upload helpers: host interior block (nx*ny*nz) -> padded state.
template <typename T>
__global__ void scatter_interior(const double *src, T *dst, Layout L) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.nx) return;
    dst[L.at(i + NG, j + NG, k + NG)] = (T)src[((long)k * L.ny + j) * L.nx + i];
}

// Conserved FP64 state from FP64 primitives (mixed path set-up).
__global__ void prim_to_cons_kernel(const double *const *Wp, double *const *Up, Layout L, double gamma) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.sx) return;
    const long c = L.at(i, j, k);
    double U[5];
    p2c_exact(Wp[0][c], Wp[1][c], Wp[2][c], Wp[3][c], Wp[4][c], gamma, U);
#pragma unroll
    for (int q = 0; q < 5; ++q) Up[q][c] = U[q];
}

// Group download conversions (device padded -> device scratch in Field3D
// order is done by cudaMemcpy2D; these produce derived groups in place).
__global__ void derive_kernel64(const double *const *Wp, double *const *Out, Layout L, double gamma,
                                double Rgas, int what) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.sx) return;
    const long c = L.at(i, j, k);
    if (what == NS3D_CONSERVED) {
        double U[5];
        p2c_exact(Wp[0][c], Wp[1][c], Wp[2][c], Wp[3][c], Wp[4][c], gamma, U);
#pragma unroll
        for (int q = 0; q < 5; ++q) Out[q][c] = U[q];
    } else {  // temperature, field_structures.h:486
        double rr = Wp[0][c] <= 0.0 ? 1e-12 : Wp[0][c];
        Out[0][c] = Wp[4][c] / __dmul_rn(rr, Rgas);
    }
}

__global__ void derive_kernel_mixed(const double *const *Up, double *const *Out, Layout L, double gamma,
                                    double Rgas, int what) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.sx) return;
    const long c = L.at(i, j, k);
    double U[5] = {Up[0][c], Up[1][c], Up[2][c], Up[3][c], Up[4][c]};
    double W[5];
    c2p_exact(U, gamma, W);
    if (what == NS3D_PRIMITIVE) {
#pragma unroll
        for (int q = 0; q < 5; ++q) Out[q][c] = W[q];
    } else {
        Out[0][c] = W[4] / __dmul_rn(W[0], Rgas);
    }
}

// T = p/(rho Rgas) of every cell (after a full-field upload).
__global__ void temp_kernel64(const double *const *Wp, double *T, Layout L, double Rgas) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.sx) return;
    const long c = L.at(i, j, k);
    const double rr = Wp[0][c] <= 0.0 ? 1e-12 : Wp[0][c];
    T[c] = Wp[4][c] / __dmul_rn(rr, Rgas);
}

template <typename T>
__global__ void widen_kernel(const T *src, double *dst, Layout Ls, Layout Ld) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= Ls.sx) return;
    dst[Ld.at(i, j, k)] = (double)src[Ls.at(i, j, k)];
}

template <typename T>
__global__ void fill_kernel(T *dst, long n, T v) {
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) dst[t] = v;
}

// --------------------------------------------------------------- the handle

struct ns3d_handle {
    ns3d_params P;
    ns3d_grid G;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool mixed = false;
    Layout L64, L32;
    Phys ph;
    BcInfo bc;
    SchemeParams<double> sp64;
    SchemeParams<float> sp32;
    // one allocation for every array
    void *pool = nullptr;
    size_t pool_bytes = 0;
    // plain: S[b][q] primitive state buffers; mixed: S[b][q] FP64 conserved
    double *S[3][5] = {};
    int s0 = 0;          // buffer holding the current state
    double *rhs64[5] = {};
    double *T64 = nullptr;
    float *w32[5] = {};
    float *rhs32[5] = {};
    float *T32 = nullptr;
    void *visc[9] = {};  // double (plain) or float (mixed), interior layout
    double *scratch[5] = {};   // download staging (points into a state buffer)
    double **dptr = nullptr;   // device array of pointer tables
    double *partials = nullptr;
    int *dev_err = nullptr;       // device error word (a bounded device wait ran out)
    // TMA tensor maps of (u, v, w) per state buffer and of T (FP64 path), or of
    // the FP32 primitives and T (mixed path)
    CUtensorMap tmW64[3][3], tmT64, tmW32[3], tmT32;
    double *cfl_part = nullptr;   // per-block CFL minima written by the last RK stage
    double *ke_part = nullptr;    // per-block kinetic energy written by the last RK stage
    long cfl_nblocks = 0;         // capacity of cfl_part / ke_part
    long cfl_count = 0;           // partials the last stage-3 launch wrote
    bool cfl_valid = false;       // cfl_part describes the current state
    bool rhs_complete = false;    // the RHS buffer holds a complete right-hand side
    bool prev_valid = false;      // buffer (s0 + 2) % 3 holds the state the last step started from
    int zlo = 0, zhi = 0;         // owned interior z-planes (a z-slab's halo planes lie outside)
    bool visc_valid = false;      // the node viscous fluxes describe the current state
    bool diag_separate = false;   // ns3d_diagnostics by its separate gradient pass (NS3D_DIAG_SEPARATE=1)
    double *visc_red = nullptr;   // per-block diagnostics sums of the viscous kernel (5 per block)
    long visc_nblocks = 0;
    int step_start = -1;          // ns3d_rk3_stage: buffer the current step started from
    bool slab_z_periodic = false; // a z-slab of a domain periodic in z
    double *scalars = nullptr;
    int red_blocks = 0;
    bool has_state = false;
    long launches = 0;
    std::string err;
    DevClock *clock = nullptr;           // device time-advance state
    bool dev_loop = false;               // kernels being captured read dt / done from clock
    cudaGraphExec_t adv_graph[3][3] = {};  // [length index][starting buffer rotation]
    double graph_dt = 0.0;
    int graph_s0 = -1;
    // per-kernel CUDA-event timing (ns3d_profile)
    bool profiling = false;
    struct Prof { const char *name; std::vector<cudaEvent_t> ev; long launches; double ms; };
    std::vector<Prof> prof;
    int prof_open = -1;
    // adjoint workspace (allocated on first use): Ub, Acc, Sb, Rb (interior
    // layout), face-VJP scratch G, viscous scratch X, velocity gradient
    void *adj_pool = nullptr;
    size_t adj_bytes = 0;
    double *ab[4][5] = {};
    double *adjG[30] = {};
    double *adjX[16] = {};
    double *gvel[3] = {};
    double **adj_tab = nullptr;  // device tables: [5*b + q] for ab[b][q], [20..22] gvel
};

namespace {

int fail(ns3d_handle *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    return code;
}

int cuda_fail(ns3d_handle *h, cudaError_t e, const char *what) {
    return fail(h, NS3D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(h, call, what)                                   \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, what); \
    } while (0)

dim3 cell_grid(const Layout &L, bool with_ghosts, int bx = 128) {
    int nx = with_ghosts ? L.sx : L.nx;
    return dim3((nx + bx - 1) / bx, with_ghosts ? L.sy : L.ny, with_ghosts ? L.sz : L.nz);
}

double *const *state_table(ns3d_handle *h, int b) { return h->dptr + 5 * b; }

int set_device(ns3d_handle *h) {
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    return NS3D_OK;
}

// Kernel timing: prof_begin/prof_end bracket one launch with events on the
// handle's stream; ns3d_profile_report resolves the elapsed times.
void prof_begin(ns3d_handle *h, const char *name) {
    if (!h->profiling) return;
    int idx = -1;
    for (size_t q = 0; q < h->prof.size(); ++q)
        if (std::strcmp(h->prof[q].name, name) == 0) idx = (int)q;
    if (idx < 0) { h->prof.push_back({name, {}, 0, 0.0}); idx = (int)h->prof.size() - 1; }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, h->stream);
    h->prof[idx].ev.push_back(a);
    h->prof[idx].ev.push_back(b);
    h->prof_open = idx;
}

void prof_end(ns3d_handle *h) {
    if (!h->profiling || h->prof_open < 0) return;
    cudaEventRecord(h->prof[h->prof_open].ev.back(), h->stream);
    h->prof[h->prof_open].launches += 1;
    h->prof_open = -1;
}

template <typename R>
SweepArgs<R> sweep_args(ns3d_handle *h, int dir) {
    SweepArgs<R> a;
    const bool m = sizeof(R) == 4;
    for (int q = 0; q < 5; ++q) {
        if constexpr (sizeof(R) == 8) { a.W[q] = h->S[h->s0][q]; a.Rhs[q] = h->rhs64[q]; }
        else { a.W[q] = h->w32[q]; a.Rhs[q] = h->rhs32[q]; }
    }
    a.L = m ? h->L32 : h->L64;
    a.periodic = h->bc.periodic[dir];
    a.outflow_lo = h->P.bc[2 * dir] == NS3D_OUTFLOW;
    a.outflow_hi = h->P.bc[2 * dir + 1] == NS3D_OUTFLOW;
    a.inv_h = (R)(dir == 0 ? h->ph.inv_dx : dir == 1 ? h->ph.inv_dy : h->ph.inv_dz);
    const double hd = dir == 0 ? h->ph.dx : dir == 1 ? h->ph.dy : h->ph.dz;
    a.dinv[0] = (R)(1.0 / (2.0 * hd)); a.dinv[1] = (R)(1.0 / (12.0 * hd)); a.dinv[2] = (R)(1.0 / (60.0 * hd));
    if constexpr (sizeof(R) == 8) a.sp = h->sp64; else a.sp = h->sp32;
    a.first = dir == 0;
    a.visc = h->ph.mu != 0.0;
    // node fluxes of this direction for rhou, rhov, rhow, E: F_v, H_v, G_v
    static const int comp[3][4] = {{0, 3, 4, 6}, {3, 1, 5, 7}, {4, 5, 2, 8}};
    for (int q = 0; q < 4; ++q) a.V[q] = (const R *)h->visc[comp[dir][q]];
    a.done = h->dev_loop ? &h->clock->done : nullptr;
    a.zlo = h->zlo; a.zhi = h->zhi;
    a.fs = FusedStage{};  // stage 0: the sweep writes the right-hand side
    return a;
}

// 3-D tensor map over one padded array (x = padded element index, y = row, z
// = plane) with the viscous kernel's plane-tile box.
bool encode_plane_map(CUtensorMap *m, const void *base, bool f64, const Layout &L) {
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (!enc) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            return false;
        }
        enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t esz = f64 ? 8 : 4;
    const cuuint64_t dims[3] = {(cuuint64_t)L.px, (cuuint64_t)L.sy, (cuuint64_t)L.sz};
    const cuuint64_t strides[2] = {(cuuint64_t)L.px * esz, (cuuint64_t)L.px * L.sy * esz};
    const cuuint32_t box[3] = {(cuuint32_t)VBX, (cuuint32_t)VBY, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(base),
               dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The plane-tile box starts at element x0 + off - 1 with x0 a multiple of 32:
// its byte offset must be a multiple of 16 (a TMA rule nothing checks at run
// time), as must the row pitch.
bool plane_box_aligned(const Layout &L, size_t esz) {
    return ((size_t)(L.off - 1) * esz) % 16 == 0 && ((size_t)VTX * esz) % 16 == 0 &&
           ((size_t)L.px * esz) % 16 == 0 && L.off >= 1;
}

template <typename R>
ViscArgs<R> visc_args(ns3d_handle *h) {
    ViscArgs<R> a;
    for (int q = 0; q < 5; ++q) {
        if constexpr (sizeof(R) == 8) a.W[q] = h->S[h->s0][q];
        else a.W[q] = h->w32[q];
    }
    for (int q = 0; q < 9; ++q) a.V[q] = (R *)h->visc[q];
    if constexpr (sizeof(R) == 8) a.T = h->T64; else a.T = h->T32;
    a.L = sizeof(R) == 8 ? h->L64 : h->L32;
    for (int d = 0; d < 3; ++d) a.periodic[d] = h->bc.periodic[d];
    a.h[0] = (R)h->ph.dx; a.h[1] = (R)h->ph.dy; a.h[2] = (R)h->ph.dz;
    const double hh[3] = {h->ph.dx, h->ph.dy, h->ph.dz};
    for (int d = 0; d < 3; ++d) {
        a.dinv[d][0] = (R)(1.0 / (2.0 * hh[d])); a.dinv[d][1] = (R)(1.0 / (12.0 * hh[d]));
        a.dinv[d][2] = (R)(1.0 / (60.0 * hh[d]));
    }
    a.mu0 = (R)h->ph.mu; a.S = (R)h->ph.S;
    a.err = h->dev_err;
    a.done = h->dev_loop ? &h->clock->done : nullptr;
    a.cp_over_pr = (R)(h->ph.Cp / h->ph.Pr);
    // the owned planes and the three either side whose fluxes the z-divergence reads
    a.zlo = h->zlo > 0 ? h->zlo - 3 : 0;
    a.zhi = h->zhi < a.L.nz ? h->zhi + 3 : a.L.nz;
    // a slab of a z-periodic domain: over the planes it computes (three or
    // more from its ends) every z derivative is the 6th-order one, as in that
    // domain, and the kernel instantiation is the one the whole periodic
    // domain uses (same bits); a slab of a bounded domain keeps its local
    // non-periodic instantiation, as the bounded domain does
    if (h->slab_z_periodic) a.periodic[2] = 1;
    a.red = nullptr;
    a.rlo = h->zlo; a.rhi = h->zhi;
    a.vol = h->ph.dx * h->ph.dy * h->ph.dz;
    return a;
}

template <typename R>
int visc_launch(ns3d_handle *h, double *red, long *nblocks = nullptr) {
    ViscArgs<R> va = visc_args<R>(h);
    va.red = red;
    dim3 g((va.L.nx + VTX - 1) / VTX, (va.L.ny + VTY - 1) / VTY, (va.zhi - va.zlo + VZC - 1) / VZC);
    if (nblocks) *nblocks = (long)g.x * g.y * g.z;
    ViscMaps maps;
    for (int q = 0; q < 3; ++q) maps.m[q] = sizeof(R) == 8 ? h->tmW64[h->s0][q] : h->tmW32[q];
    maps.m[3] = sizeof(R) == 8 ? h->tmT64 : h->tmT32;
    prof_begin(h, "viscous_flux");
    const bool p6 = va.periodic[0] && va.periodic[1] && va.periodic[2];
    if (red) {
        if (p6) viscous_flux_kernel<R, true, true><<<g, dim3(VTX, VTY), 0, h->stream>>>(va, maps);
        else viscous_flux_kernel<R, false, true><<<g, dim3(VTX, VTY), 0, h->stream>>>(va, maps);
    } else {
        if (p6) viscous_flux_kernel<R, true, false><<<g, dim3(VTX, VTY), 0, h->stream>>>(va, maps);
        else viscous_flux_kernel<R, false, false><<<g, dim3(VTX, VTY), 0, h->stream>>>(va, maps);
    }
    prof_end(h);
    h->launches += 1;
    CK(h, cudaGetLastError(), "viscous kernel");
    return NS3D_OK;
}

template <typename R>
int rhs_impl(ns3d_handle *h, const FusedStage *fs = nullptr) {
    cudaStream_t st = h->stream;
    cudaError_t e;
    // the node fluxes of this state may be there already (ns3d_diagnostics
    // computes them with its sums); never inside a captured time loop
    const bool have_visc = h->visc_valid && !h->dev_loop;
    h->visc_valid = false;
    if (h->ph.mu != 0.0 && !have_visc) {  // Re = inf: the viscous terms are exactly zero
        const int r = visc_launch<R>(h, nullptr);
        if (r) return r;
    }
    prof_begin(h, "sweep_x");
    e = sweep_x(sweep_args<R>(h, 0), st); if (e != cudaSuccess) return cuda_fail(h, e, "sweep_x");
    prof_end(h);
    prof_begin(h, "sweep_y");
    e = sweep_y(sweep_args<R>(h, 1), st); if (e != cudaSuccess) return cuda_fail(h, e, "sweep_y");
    prof_end(h);
    SweepArgs<R> az = sweep_args<R>(h, 2);
    if (fs) az.fs = *fs;
    prof_begin(h, fs ? "sweep_z_stage" : "sweep_z");
    e = sweep_z(az, st); if (e != cudaSuccess) return cuda_fail(h, e, "sweep_z");
    prof_end(h);
    h->launches += 3;
    return NS3D_OK;
}

int compute_rhs_async(ns3d_handle *h) {
    const int r = h->mixed ? rhs_impl<float>(h) : rhs_impl<double>(h);
    h->rhs_complete = r == NS3D_OK;
    h->visc_valid = r == NS3D_OK && h->ph.mu != 0.0 && !h->dev_loop;  // node fluxes of the current state
    return r;
}

// stage: 1..3 RK stages, 0 = ghost fill of the current state.
int stage_async(ns3d_handle *h, int stage, int src0, int srcc, int dst, double dt) {
    cudaStream_t st = h->stream;
    h->visc_valid = false;
    dim3 g = cell_grid(h->L64, true, STAGE_THREADS);
    double *cfl = stage == 3 ? h->cfl_part : nullptr;  // the next step's CFL bound
    if (!h->mixed) {
        StageArgs64 a;
        for (int q = 0; q < 5; ++q) {
            a.W0[q] = h->S[src0][q]; a.Wc[q] = h->S[srcc][q]; a.Rhs[q] = h->rhs64[q]; a.Wout[q] = h->S[dst][q];
        }
        a.L = h->L64; a.b = h->bc; a.dt = dt; a.gamma = h->ph.gamma; a.stage = stage;
        a.Tout = h->T64; a.Rgas = h->ph.Rgas;
        a.cfl_part = cfl; a.ke_part = h->ke_part; a.dx = h->ph.dx;
        a.vol = h->ph.dx * h->ph.dy * h->ph.dz;
        a.dt_dev = h->dev_loop ? &h->clock->dt : nullptr;
        a.done = h->dev_loop ? &h->clock->done : nullptr;
        prof_begin(h, "stage");
        stage_kernel64<<<g, STAGE_THREADS, 0, st>>>(a);
        prof_end(h);
    } else {
        StageArgsMixed a;
        for (int q = 0; q < 5; ++q) {
            a.U0[q] = h->S[src0][q]; a.Uc[q] = h->S[srcc][q]; a.Rhs[q] = h->rhs32[q]; a.D[q] = nullptr;
            a.Uout[q] = h->S[dst][q]; a.Wout[q] = h->w32[q];
        }
        a.L = h->L64; a.L32 = h->L32; a.b = h->bc; a.dt = dt; a.gamma = h->ph.gamma; a.stage = stage;
        a.Tout = h->T32; a.Rgas = h->ph.Rgas;
        a.cfl_part = cfl; a.ke_part = h->ke_part; a.dx = h->ph.dx;
        a.vol = h->ph.dx * h->ph.dy * h->ph.dz;
        a.dt_dev = h->dev_loop ? &h->clock->dt : nullptr;
        a.done = h->dev_loop ? &h->clock->done : nullptr;
        prof_begin(h, "stage");
        stage_kernel_mixed<<<g, STAGE_THREADS, 0, st>>>(a);
        prof_end(h);
    }
    h->launches += 1;
    h->cfl_valid = false;
    CK(h, cudaGetLastError(), "stage kernel");
    h->cfl_valid = stage == 3;
    if (stage == 3) h->cfl_count = (long)g.x * g.y * g.z;
    return NS3D_OK;
}

// One RK stage: right-hand side and update, fused into the z-sweep
// (FusedStage), then a ghost kernel for the ghost cells.  Plain FP64 path: the
// same bits as the separate stage kernel.  Mixed path: increment form -- the
// FP32 increments of stages 1 and 2 live in the state buffer that is free
// during the step (neither src0 nor the step's result), and only stage 3
// writes the FP64 state.  src0 = step-start state, srcc = this stage's state
// (the sweeps read h->s0, which the caller has set to srcc), dst = new state.
int rk_stage_async(ns3d_handle *h, int stage, int src0, int srcc, int dst, double dt) {
    if (h->mixed) {
        // rk3_async's buffers: (1: s0, s0 -> b1), (2: s0, b1 -> b2), (3: s0, b2 -> b1)
        const int free_buf = 3 - src0 - (stage == 2 ? srcc : dst);
        if (free_buf < 0 || free_buf > 2 || free_buf == src0 || (stage != 2 && free_buf == dst)) return NS3D_ERR_STATE;
        FusedStage f{};
        f.stage = stage;
        for (int q = 0; q < 5; ++q) {
            f.U0[q] = h->S[src0][q]; f.Uout[q] = h->S[dst][q];
            f.D[q] = reinterpret_cast<float *>(h->S[free_buf][q]);  // FP32 layout inside an FP64 plane
            f.W32out[q] = h->w32[q];  // in place (the sweep defers the cells its wrap re-reads)
        }
        f.T32out = h->T32;
        f.L64 = h->L64;
        f.dt = dt;
        f.dt_dev = h->dev_loop ? &h->clock->dt : nullptr;
        f.gamma = h->ph.gamma; f.Rgas = h->ph.Rgas; f.dx = h->ph.dx;
        f.vol = h->ph.dx * h->ph.dy * h->ph.dz;
        f.cfl_part = stage == 3 ? h->cfl_part : nullptr;
        f.ke_part = stage == 3 ? h->ke_part : nullptr;
        f.keep_rhs = stage == 3 && h->P.keep_rhs;
        h->cfl_valid = false;
        h->rhs_complete = false;
        int r = rhs_impl<float>(h, &f);
        if (r) return r;
        h->rhs_complete = f.keep_rhs != 0;
        StageArgsMixed a;
        for (int q = 0; q < 5; ++q) {
            a.U0[q] = h->S[src0][q]; a.Uc[q] = nullptr; a.Rhs[q] = h->rhs32[q];
            a.Uout[q] = h->S[dst][q]; a.Wout[q] = h->w32[q]; a.D[q] = f.D[q];
        }
        a.L = h->L64; a.L32 = h->L32; a.b = h->bc; a.dt = dt; a.gamma = h->ph.gamma; a.stage = stage;
        a.Tout = h->T32; a.Rgas = h->ph.Rgas;
        a.cfl_part = nullptr; a.ke_part = nullptr; a.dx = h->ph.dx; a.vol = f.vol;
        a.dt_dev = f.dt_dev;
        a.done = h->dev_loop ? &h->clock->done : nullptr;
        const long ng = ghost_count(h->L64);
        prof_begin(h, "ghost_fill");
        stage_ghost_kernel_mixed<<<(unsigned)((ng + 255) / 256), 256, 0, h->stream>>>(a);
        prof_end(h);
        h->launches += 1;
        CK(h, cudaGetLastError(), "ghost kernel");
        if (stage == 3) {
            const int gx = (h->L32.nx + SweepGeom<2, float>::NLINE - 1) / SweepGeom<2, float>::NLINE;
            h->cfl_count = (long)gx * h->L32.ny;  // z-sweep blocks
            h->cfl_valid = true;
        }
        return NS3D_OK;
    }
    FusedStage f{};
    f.stage = stage;
    for (int q = 0; q < 5; ++q) { f.W0[q] = h->S[src0][q]; f.Wout[q] = h->S[dst][q]; }
    f.Tout = h->T64;
    f.L64 = h->L64;
    f.dt = dt;
    f.dt_dev = h->dev_loop ? &h->clock->dt : nullptr;
    f.gamma = h->ph.gamma; f.Rgas = h->ph.Rgas; f.dx = h->ph.dx;
    f.vol = h->ph.dx * h->ph.dy * h->ph.dz;
    f.cfl_part = stage == 3 ? h->cfl_part : nullptr;
    f.ke_part = stage == 3 ? h->ke_part : nullptr;
    f.keep_rhs = stage == 3 && h->P.keep_rhs;
    h->cfl_valid = false;
    h->rhs_complete = false;
    int r = rhs_impl<double>(h, &f);
    if (r) return r;
    h->rhs_complete = f.keep_rhs != 0;
    StageArgs64 a;
    for (int q = 0; q < 5; ++q) {
        a.W0[q] = h->S[src0][q]; a.Wc[q] = h->S[srcc][q]; a.Rhs[q] = h->rhs64[q]; a.Wout[q] = h->S[dst][q];
    }
    a.L = h->L64; a.b = h->bc; a.dt = dt; a.gamma = h->ph.gamma; a.stage = stage;
    a.Tout = h->T64; a.Rgas = h->ph.Rgas;
    a.cfl_part = nullptr; a.ke_part = nullptr; a.dx = h->ph.dx; a.vol = f.vol;
    a.dt_dev = f.dt_dev;
    a.done = h->dev_loop ? &h->clock->done : nullptr;
    const long ng = ghost_count(h->L64);
    prof_begin(h, "ghost_fill");
    stage_ghost_kernel64<<<(unsigned)((ng + 255) / 256), 256, 0, h->stream>>>(a);
    prof_end(h);
    h->launches += 1;
    CK(h, cudaGetLastError(), "ghost kernel");
    if (stage == 3) {
        const int gx = (h->L64.nx + SweepGeom<2, double>::NLINE - 1) / SweepGeom<2, double>::NLINE;
        h->cfl_count = (long)gx * h->L64.ny;  // z-sweep blocks
        h->cfl_valid = true;
    }
    return NS3D_OK;
}

// One RK3 step (no synchronisation).  Buffers: state s0 -> stage 1 -> b1,
// stage 2 -> b2, stage 3 -> b1; the new state is b1 (recordConservedTo0 is
// the pointer rotation).
int rk3_async(ns3d_handle *h, double dt) {
    const int s0 = h->s0, b1 = (s0 + 1) % 3, b2 = (s0 + 2) % 3;
    auto fail_reset = [&](int r) {  // back to the step's start buffer
        h->s0 = s0;
        return r;
    };
    int r;
    if ((r = rk_stage_async(h, 1, s0, s0, b1, dt)) != NS3D_OK) return fail_reset(r);
    h->s0 = b1;  // RHS of stage 2 reads the stage-1 state
    if ((r = rk_stage_async(h, 2, s0, b1, b2, dt)) != NS3D_OK) return fail_reset(r);
    h->s0 = b2;
    if ((r = rk_stage_async(h, 3, s0, b2, b1, dt)) != NS3D_OK) return fail_reset(r);
    h->s0 = b1;
    return NS3D_OK;
}

int reduce_combine(ns3d_handle *h, int nv, int mode, double *host_out, const double *part = nullptr,
                   long nblocks = 0) {
    combine_kernel<<<1, 32, 0, h->stream>>>(part ? part : h->partials, part ? (int)nblocks : h->red_blocks, nv, mode,
                                            h->scalars);
    h->launches += 1;
    CK(h, cudaGetLastError(), "combine");
    CK(h, cudaMemcpyAsync(host_out, h->scalars, sizeof(double) * nv, cudaMemcpyDeviceToHost, h->stream), "copy scalars");
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    return NS3D_OK;
}

int check_state(ns3d_handle *h) {
    if (!h->mixed)
        check_kernel<double><<<h->red_blocks, RED_THREADS, 0, h->stream>>>(state_table(h, h->s0), h->L64, h->partials, h->zlo, h->zhi - h->zlo);
    else
        check_kernel<float><<<h->red_blocks, RED_THREADS, 0, h->stream>>>((const float *const *)(h->dptr + 25), h->L32,
                                                                           h->partials, h->zlo, h->zhi - h->zlo);
    h->launches += 1;
    CK(h, cudaGetLastError(), "check kernel");
    double bad = 0;
    int r = reduce_combine(h, 1, 0, &bad);
    if (r != NS3D_OK) return r;
    if (bad > 0) return fail(h, NS3D_ERR_NONFINITE, "state has " + std::to_string((long)bad) +
                                                       " interior cells with non-finite values or rho/p <= 0");
    return NS3D_OK;
}


// ----------------------------------------------------------------- adjoint

__global__ void to_interior_kernel(const double *src, double *dst, Layout L) {
    // contiguous Field3D array -> interior layout
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.nx) return;
    dst[((long)k * L.ny + j) * L.nx + i] = src[((long)(k + NG) * L.sy + (j + NG)) * L.sx + (i + NG)];
}

__global__ void from_interior_kernel(const double *src, double *dst, Layout L) {
    // interior layout -> contiguous Field3D array (ghost entries zero)
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.sx) return;
    const bool in = i >= NG && i < NG + L.nx && j >= NG && j < NG + L.ny && k >= NG && k < NG + L.nz;
    dst[((long)k * L.sy + j) * L.sx + i] = in ? src[((long)(k - NG) * L.ny + (j - NG)) * L.nx + (i - NG)] : 0.0;
}

bool is_slab(const ns3d_handle *h) { return h->zlo != 0 || h->zhi != h->G.nz; }

bool adjoint_supported(const ns3d_handle *h, std::string &why) {
    if (h->mixed) { why = "adjoint: plain FP64 path only"; return false; }
    if (is_slab(h)) { why = "adjoint: whole domains only (not a z-slab)"; return false; }
    if (!(h->bc.periodic[0] && h->bc.periodic[1] && h->bc.periodic[2])) {
        why = "adjoint: periodic boundaries in all directions only"; return false;
    }
    if (h->P.char_recon) { why = "adjoint: component-wise interpolation only"; return false; }
    if (h->P.interpolation != NS3D_WENO5 && h->P.interpolation != NS3D_MDCD_LINEAR &&
        h->P.interpolation != NS3D_MDCD_HYBRID) {
        why = "adjoint: WENO5, MDCD_LINEAR or MDCD_HYBRID interpolation only"; return false;
    }
    const int rs = h->P.riemann_solver;
    if (rs != NS3D_ROE && rs != NS3D_RUSANOV && rs != NS3D_HLL && rs != NS3D_HLLC) {
        why = "adjoint: Roe, Rusanov, HLL or HLLC flux only"; return false;
    }
    return true;
}

int ensure_adjoint(ns3d_handle *h) {
    if (h->adj_pool) return NS3D_OK;
    const long n = (long)h->L64.nx * h->L64.ny * h->L64.nz;
    const long n_al = ((n + 31) / 32) * 32;
    const size_t arrays = 20 + 30 + 16 + 3;
    const size_t bytes = arrays * n_al * 8 + 4096;
    cudaError_t e = cudaMalloc(&h->adj_pool, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); h->adj_pool = nullptr; return fail(h, NS3D_ERR_OOM, "adjoint workspace"); }
    h->adj_bytes = bytes;
    double *p = (double *)h->adj_pool;
    for (int b = 0; b < 4; ++b)
        for (int q = 0; q < 5; ++q) { h->ab[b][q] = p; p += n_al; }
    for (int q = 0; q < 30; ++q) { h->adjG[q] = p; p += n_al; }
    for (int q = 0; q < 16; ++q) { h->adjX[q] = p; p += n_al; }
    for (int q = 0; q < 3; ++q) { h->gvel[q] = p; p += n_al; }
    h->adj_tab = (double **)p;
    void *tab[23];
    for (int b = 0; b < 4; ++b)
        for (int q = 0; q < 5; ++q) tab[5 * b + q] = h->ab[b][q];
    for (int q = 0; q < 3; ++q) tab[20 + q] = h->gvel[q];
    CK(h, cudaMemcpy(h->adj_tab, tab, sizeof(tab), cudaMemcpyHostToDevice), "adjoint tables");
    return NS3D_OK;
}

AdjArgs adj_args(ns3d_handle *h, double *const W[5], const double *const Rb[5], double *const Ub[5]) {
    AdjArgs a;
    for (int q = 0; q < 5; ++q) { a.W[q] = W[q]; a.Rb[q] = Rb[q]; a.Ub[q] = Ub[q]; }
    for (int q = 0; q < 30; ++q) a.G[q] = h->adjG[q];
    for (int q = 0; q < 16; ++q) a.X[q] = h->adjX[q];
    a.L = h->L64;
    a.inv_h[0] = h->ph.inv_dx; a.inv_h[1] = h->ph.inv_dy; a.inv_h[2] = h->ph.inv_dz;
    a.gamma = h->ph.gamma; a.Rgas = h->ph.Rgas; a.mu0 = h->ph.mu; a.S = h->ph.S; a.cpr = h->ph.Cp / h->ph.Pr;
    a.interp = h->P.interpolation; a.riemann = h->P.riemann_solver == NS3D_HLL ? 3 : h->P.riemann_solver;
    for (int m = 0; m < 6; ++m) a.lin[m] = h->sp64.lin[m];
    for (int m = 0; m < 4; ++m) a.hd[m] = h->sp64.hd[m];
    a.first = 0;
    a.rbs = 1.0;
    return a;
}

// Ub_target += (dR/dU at W)^T (rbs * Rb)
int vjp_rhs_async(ns3d_handle *h, double *const W[5], int rb_slot, int target_slot, double rbs = 1.0) {
    AdjArgs a = adj_args(h, W, h->ab[rb_slot], h->ab[target_slot]);
    a.rbs = rbs;
    cudaError_t e = adj_rhs_vjp(a, h->stream, &h->launches);
    if (e != cudaSuccess) return cuda_fail(h, e, "adjoint kernels");
    return NS3D_OK;
}

// y = beta*y + alpha*x on adjoint slots
int axpby_slot(ns3d_handle *h, int y, int x, double alpha, double beta) {
    const long n = (long)h->L64.nx * h->L64.ny * h->L64.nz;
    cudaError_t e = adj_axpby(h->adj_tab + 5 * y, h->adj_tab + 5 * x, alpha, beta, n, h->stream);
    h->launches += 1;
    if (e != cudaSuccess) return cuda_fail(h, e, "axpby");
    return NS3D_OK;
}

// Backward through one RK3 step whose stage states are W0, W1, W2.
// Slot 0 holds the adjoint of the step's result on entry and of its input on
// exit; slots 1 (accumulator ACC), 2 (stage adjoint SB), 3 (RHS adjoint RB)
// are scratch.
//   U1 = U0 + dt R(U0); U2 = 3/4 U0 + 1/4 (U1 + dt R(U1)); U3 = 1/3 U0 + 2/3 (U2 + dt R(U2))
// The scalings of the RHS adjoints ride on the VJP kernels' input scale, so
// one step costs three fused combinations and three RHS VJPs.
int vjp_step_async(ns3d_handle *h, double *const W0[5], double *const W1[5], double *const W2[5], double dt) {
    int r;
    enum { UB = 0, ACC = 1, SB = 2, RB = 3 };
    const long n = (long)h->L64.nx * h->L64.ny * h->L64.nz;
    auto combine = [&](int which) -> int {
        cudaError_t e = adj_step_combine(which, h->adj_tab, dt, n, h->stream);
        h->launches += 1;
        return e == cudaSuccess ? NS3D_OK : cuda_fail(h, e, "adjoint combination");
    };
    if ((r = combine(1))) return r;                                    // ACC = UB/3, SB = 2 UB/3
    if ((r = vjp_rhs_async(h, W2, UB, SB, (2.0 / 3.0) * dt))) return r;  // SB = adjoint of U2
    if ((r = combine(2))) return r;                                    // ACC += 3/4 SB, SB /= 4, RB = dt SB
    if ((r = vjp_rhs_async(h, W1, RB, SB))) return r;                  // SB = adjoint of U1
    if ((r = combine(3))) return r;                                    // UB = ACC + SB
    return vjp_rhs_async(h, W0, SB, UB, dt);                           // UB = adjoint of U0
}

// One forward step that also stores its three stage states.
int rk3_async_store(ns3d_handle *h, double dt, double *const st[3][5]) {
    const size_t bytes = (size_t)h->L64.plane * 8;
    const int s0 = h->s0, b1 = (s0 + 1) % 3, b2 = (s0 + 2) % 3;
    int r;
    for (int q = 0; q < 5; ++q) CK(h, cudaMemcpyAsync(st[0][q], h->S[s0][q], bytes, cudaMemcpyDeviceToDevice, h->stream), "store");
    if ((r = rk_stage_async(h, 1, s0, s0, b1, dt))) return r;
    for (int q = 0; q < 5; ++q) CK(h, cudaMemcpyAsync(st[1][q], h->S[b1][q], bytes, cudaMemcpyDeviceToDevice, h->stream), "store");
    h->s0 = b1;
    if ((r = rk_stage_async(h, 2, s0, b1, b2, dt))) { h->s0 = s0; return r; }
    for (int q = 0; q < 5; ++q) CK(h, cudaMemcpyAsync(st[2][q], h->S[b2][q], bytes, cudaMemcpyDeviceToDevice, h->stream), "store");
    h->s0 = b2;
    if ((r = rk_stage_async(h, 3, s0, b2, b1, dt))) { h->s0 = s0; return r; }
    h->s0 = b1;
    return NS3D_OK;
}

// T of the current state (after the state buffer was overwritten by a copy)
int refresh_T(ns3d_handle *h) {
    h->visc_valid = false;
    dim3 g = cell_grid(h->L64, true, 128);
    temp_kernel64<<<g, 128, 0, h->stream>>>(state_table(h, h->s0), h->T64, h->L64, h->ph.Rgas);
    h->launches += 1;
    CK(h, cudaGetLastError(), "temperature");
    return NS3D_OK;
}

int upload_interior_slot(ns3d_handle *h, const double *const host[5], int slot) {
    const Layout &L = h->L64;
    const size_t n = (size_t)L.sx * L.sy * L.sz;
    const int stg = (h->s0 + 1) % 3;
    for (int q = 0; q < 5; ++q) {
        CK(h, cudaMemcpyAsync(h->S[stg][q], host[q], n * 8, cudaMemcpyHostToDevice, h->stream), "upload adjoint");
        to_interior_kernel<<<cell_grid(L, false, 128), 128, 0, h->stream>>>(h->S[stg][q], h->ab[slot][q], L);
        h->launches += 1;
    }
    CK(h, cudaGetLastError(), "to_interior");
    return NS3D_OK;
}

int download_interior_slot(ns3d_handle *h, int slot, double *const host[5]) {
    const Layout &L = h->L64;
    const size_t n = (size_t)L.sx * L.sy * L.sz;
    const int stg = (h->s0 + 1) % 3;
    for (int q = 0; q < 5; ++q) {
        from_interior_kernel<<<cell_grid(L, true, 128), 128, 0, h->stream>>>(h->ab[slot][q], h->S[stg][q], L);
        h->launches += 1;
        CK(h, cudaMemcpyAsync(host[q], h->S[stg][q], n * 8, cudaMemcpyDeviceToHost, h->stream), "download adjoint");
    }
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    return NS3D_OK;
}

bool valid_params(const ns3d_params *p, const ns3d_grid *g, std::string &why) {
    if (p->interpolation == NS3D_ZERO) {
        why = "ZERO interpolation sets ghost_layers=1 while the flux difference and viscous stencils read "
              "+-3 points (initialization.cpp:180-183); unsupported";
        return false;
    }
    if (p->interpolation != NS3D_WENO5 && p->interpolation != NS3D_MDCD_LINEAR && p->interpolation != NS3D_MDCD_HYBRID) {
        why = "unknown interpolation"; return false;
    }
    if (p->riemann_solver < 0 || p->riemann_solver > 6) { why = "unknown Riemann solver"; return false; }
    for (int f = 0; f < 6; ++f)
        if (p->bc[f] < 0 || p->bc[f] > 4) { why = "unknown boundary type"; return false; }
    if (p->precision != NS3D_FP64 && p->precision != NS3D_MIXED) { why = "unknown precision"; return false; }
    if (g->nx < 3 || g->ny < 3 || g->nz < 3) { why = "each dimension needs at least 3 interior cells"; return false; }
    if ((long)g->nx * g->ny * g->nz > (1L << 31)) { why = "grid too large"; return false; }
    if (!(g->Lx > 0 && g->Ly > 0 && g->Lz > 0)) { why = "domain lengths must be positive"; return false; }
    if (!(p->gamma > 1.0) || !(p->Ma > 0) || !(p->Pr > 0) || !(p->Re > 0)) { why = "invalid physical constants"; return false; }
    return true;
}

}  // namespace

// =============================================================== C ABI

extern "C" {

void ns3d_params_default(ns3d_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->gamma = 1.4; p->Pr = 0.71; p->Ma = 0.4; p->Re = 500.0; p->cfl = 0.1; p->dt_fixed = -1.0;
    p->mdcd_diss = 0.01; p->mdcd_disp = 0.0463783; p->sutherland_s = 110.4 / 288.15;
    p->interpolation = NS3D_WENO5; p->riemann_solver = NS3D_ROE; p->char_recon = 0;
    for (int f = 0; f < 6; ++f) p->bc[f] = NS3D_PERIODIC;
    p->precision = NS3D_FP64; p->device = 0; p->check_state = 0;
}

const char *ns3d_status_string(int s) {
    switch (s) {
        case NS3D_OK: return "ok";
        case NS3D_ERR_INVALID_ARG: return "invalid argument";
        case NS3D_ERR_CONFIG: return "unsupported configuration";
        case NS3D_ERR_OOM: return "out of device memory";
        case NS3D_ERR_CUDA: return "CUDA error";
        case NS3D_ERR_NONFINITE: return "non-finite state";
        case NS3D_ERR_NO_DEVICE: return "no CUDA device";
        case NS3D_ERR_STATE: return "no state uploaded";
        case NS3D_ERR_DT: return "time step too small";
        case NS3D_ERR_TIMEOUT: return "device wait timed out";
        default: return "unknown status";
    }
}

static thread_local std::string g_create_error;

const char *ns3d_last_error(const ns3d_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int ns3d_create(const ns3d_params *params, const ns3d_grid *grid, ns3d_handle **out) {
    if (!params || !grid || !out) return NS3D_ERR_INVALID_ARG;
    *out = nullptr;
    std::string why;
    if (!valid_params(params, grid, why)) {
        g_create_error = why;
        return NS3D_ERR_CONFIG;
    }
    g_create_error.clear();
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NS3D_ERR_NO_DEVICE;
    if (params->device < 0 || params->device >= ndev) return NS3D_ERR_INVALID_ARG;
    ns3d_handle *h = new (std::nothrow) ns3d_handle();
    if (!h) return NS3D_ERR_OOM;
    h->P = *params;
    h->G = *grid;
    h->device = params->device;
    h->mixed = params->precision == NS3D_MIXED;
    if (cudaSetDevice(h->device) != cudaSuccess) { delete h; return NS3D_ERR_NO_DEVICE; }
    h->L64 = make_layout<double>(grid->nx, grid->ny, grid->nz);
    h->L32 = make_layout<float>(grid->nx, grid->ny, grid->nz);
    h->zlo = 0;
    h->zhi = grid->nz;
    if (ghost_count(h->L64) >= (1L << 31)) { delete h; return NS3D_ERR_SIZE; }  // 32-bit ghost decode
    // the mixed path's FP32 stage increments live inside an FP64 state plane
    if ((size_t)h->L32.plane * 4 > (size_t)h->L64.plane * 8) { delete h; return NS3D_ERR_CONFIG; }
    // derived constants, initialization.cpp:170-172, 194-197
    Phys &ph = h->ph;
    ph.gamma = params->gamma;
    ph.Rgas = 1.0 / (params->Ma * params->Ma * params->gamma);
    const double Cv = 1.0 / (params->gamma * (params->gamma - 1.0) * params->Ma * params->Ma);
    ph.Cp = Cv * params->gamma;
    ph.Pr = params->Pr;
    ph.mu = std::isinf(params->Re) ? 0.0 : 1.0 / params->Re;
    ph.S = params->sutherland_s;
    ph.dx = grid->Lx / grid->nx; ph.dy = grid->Ly / grid->ny; ph.dz = grid->Lz / grid->nz;
    ph.inv_dx = 1.0 / ph.dx; ph.inv_dy = 1.0 / ph.dy; ph.inv_dz = 1.0 / ph.dz;
    ph.mdcd_disp = params->mdcd_disp; ph.mdcd_diss = params->mdcd_diss;
    for (int d = 0; d < 3; ++d)
        h->bc.periodic[d] = params->bc[2 * d] == NS3D_PERIODIC && params->bc[2 * d + 1] == NS3D_PERIODIC;
    for (int f = 0; f < 6; ++f) h->bc.bc[f] = params->bc[f];
    // interpolation coefficients, interpolation.cpp:130-132, 179-182
    const double disp = params->mdcd_disp, diss = params->mdcd_diss;
    const double lin[6] = {(3.0 * disp + 3.0 * diss) / 8.0, (-18.0 * disp - 30 * diss - 1.0) / 16.0,
                           (12.0 * disp + 60.0 * diss + 9.0) / 16.0, (12.0 * disp - 60.0 * diss + 9.0) / 16.0,
                           (-18.0 * disp + 30.0 * diss - 1.0) / 16.0, (3.0 * disp - 3.0 * diss) / 8.0};
    const double hd[4] = {1.5 * (disp + diss), 0.5 - 1.5 * (disp - 3 * diss), 0.5 - 1.5 * (disp + 3 * diss),
                          1.5 * (disp - diss)};
    h->sp64.gamma = params->gamma; h->sp32.gamma = (float)params->gamma;
    for (int q = 0; q < 6; ++q) { h->sp64.lin[q] = lin[q]; h->sp32.lin[q] = (float)lin[q]; }
    for (int q = 0; q < 4; ++q) { h->sp64.hd[q] = hd[q]; h->sp32.hd[q] = (float)hd[q]; }
    h->sp64.interp = h->sp32.interp = params->interpolation;
    h->sp64.riemann = h->sp32.riemann = params->riemann_solver;
    h->sp64.char_recon = h->sp32.char_recon = params->char_recon;

    // memory plan (bytes, each array 256-byte aligned)
    const long p64 = h->L64.plane * 8, p32 = h->L32.plane * 4;
    const long ncell = (long)grid->nx * grid->ny * grid->nz;
    const long vis_elems = ((ncell + 63) / 64) * 64;
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, h->device);
    h->red_blocks = dev_sms * 4;
    size_t bytes = 15 * p64;                                   // three state buffers
    bytes += h->mixed ? 11 * p32 : 6 * p64;                    // (w32 + rhs32 + T32) or (rhs64 + T64)
    bytes += 9 * vis_elems * (h->mixed ? 4 : 8);               // viscous node fluxes
    bytes += 256 * 32;                                         // pointer tables
    bytes += ((size_t)h->red_blocks * 10 * 8 + 255) / 256 * 256;  // partials
    bytes += 256;                                              // scalars
    {
        const dim3 sg = cell_grid(h->L64, true, STAGE_THREADS);
        h->cfl_nblocks = (long)sg.x * sg.y * sg.z;
    }
    bytes += 2 * (((size_t)h->cfl_nblocks * 8 + 255) / 256 * 256);  // stage CFL minima, kinetic energy
    bytes += 256;                                              // device clock
    {
        const long vb = (long)((grid->nx + VTX - 1) / VTX) * ((grid->ny + VTY - 1) / VTY) * ((grid->nz + VZC - 1) / VZC);
        h->visc_nblocks = vb;
        bytes += ((size_t)vb * 5 * 8 + 255) / 256 * 256;      // viscous-kernel diagnostics sums
    }
    cudaError_t e = cudaMalloc(&h->pool, bytes);
    if (e != cudaSuccess) { delete h; cudaGetLastError(); return NS3D_ERR_OOM; }
    h->pool_bytes = bytes;
    char *p = (char *)h->pool;
    for (int b = 0; b < 3; ++b)
        for (int q = 0; q < 5; ++q) { h->S[b][q] = (double *)p; p += p64; }
    if (h->mixed) {
        for (int q = 0; q < 5; ++q) { h->w32[q] = (float *)p; p += p32; }
        for (int q = 0; q < 5; ++q) { h->rhs32[q] = (float *)p; p += p32; }
        h->T32 = (float *)p; p += p32;
    } else {
        for (int q = 0; q < 5; ++q) { h->rhs64[q] = (double *)p; p += p64; }
        h->T64 = (double *)p; p += p64;
    }
    for (int q = 0; q < 9; ++q) { h->visc[q] = p; p += vis_elems * (h->mixed ? 4 : 8); }
    h->dptr = (double **)p; p += 256 * 32;
    h->partials = (double *)p; p += ((size_t)h->red_blocks * 10 * 8 + 255) / 256 * 256;
    h->scalars = (double *)p;
    h->dev_err = (int *)((char *)p + 128);
    p += 256;
    h->cfl_part = (double *)p;
    p += ((size_t)h->cfl_nblocks * 8 + 255) / 256 * 256;
    h->ke_part = (double *)p;
    p += ((size_t)h->cfl_nblocks * 8 + 255) / 256 * 256;
    h->clock = (DevClock *)p;
    p += 256;
    h->visc_red = (double *)p;
    {
        const char *ds = std::getenv("NS3D_DIAG_SEPARATE");  // the separate gradient pass, for comparison
        h->diag_separate = ds && ds[0] == '1';
    }
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { cudaFree(h->pool); delete h; return NS3D_ERR_CUDA; }
    h->own_stream = true;
    // pointer tables: [0..14] state buffers, [15..19] scratch, [20..24] rhs64, [25..29] w32
    void *tab[30] = {};
    for (int b = 0; b < 3; ++b)
        for (int q = 0; q < 5; ++q) tab[5 * b + q] = h->S[b][q];
    for (int q = 0; q < 5; ++q) {
        tab[20 + q] = h->rhs64[q];
        tab[25 + q] = h->w32[q];
    }
    e = cudaMemcpy(h->dptr, tab, sizeof(tab), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(h->pool, 0, (size_t)((char *)h->dptr - (char *)h->pool));
    if (e == cudaSuccess) e = cudaMemset(h->dev_err, 0, sizeof(int));
    if (e != cudaSuccess) { ns3d_destroy(h); return NS3D_ERR_CUDA; }
    // TMA tensor maps of the viscous kernel's plane tiles
    {
        bool ok = plane_box_aligned(h->mixed ? h->L32 : h->L64, h->mixed ? 4 : 8);
        if (!h->mixed) {
            for (int b = 0; b < 3 && ok; ++b)
                for (int q = 0; q < 3 && ok; ++q) ok = encode_plane_map(&h->tmW64[b][q], h->S[b][q + 1], true, h->L64);
            if (ok) ok = encode_plane_map(&h->tmT64, h->T64, true, h->L64);
        } else {
            for (int q = 0; q < 3 && ok; ++q) ok = encode_plane_map(&h->tmW32[q], h->w32[q + 1], false, h->L32);
            if (ok) ok = encode_plane_map(&h->tmT32, h->T32, false, h->L32);
        }
        if (!ok) {
            ns3d_destroy(h);
            g_create_error = "TMA tensor maps of the viscous tiles could not be encoded";
            return NS3D_ERR_CUDA;
        }
    }
    // Field3D::allocate: rho = 1 everywhere (field_structures.h:257)
    for (int b = 0; b < 3; ++b) {
        fill_kernel<double><<<256, 256, 0, h->stream>>>(h->S[b][0], h->L64.plane, 1.0);
    }
    if (h->mixed) fill_kernel<float><<<256, 256, 0, h->stream>>>(h->w32[0], h->L32.plane, 1.0f);
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { ns3d_destroy(h); return NS3D_ERR_CUDA; }
    *out = h;
    return NS3D_OK;
}

int ns3d_destroy(ns3d_handle *h) {
    if (!h) return NS3D_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    for (auto &row : h->adv_graph)
        for (auto &g : row)
            if (g) cudaGraphExecDestroy(g);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto &p : h->prof)
        for (auto e : p.ev) cudaEventDestroy(e);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    if (h->pool) cudaFree(h->pool);
    if (h->adj_pool) cudaFree(h->adj_pool);
    delete h;
    return NS3D_OK;
}

int ns3d_field_dims(const ns3d_handle *h, int out[3]) {
    if (!h || !out) return NS3D_ERR_INVALID_ARG;
    out[0] = h->L64.sx; out[1] = h->L64.sy; out[2] = h->L64.sz;
    return NS3D_OK;
}

int ns3d_set_stream(ns3d_handle *h, void *stream) {
    if (!h) return NS3D_ERR_INVALID_ARG;
    int r = set_device(h); if (r) return r;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    if (h->own_stream) cudaStreamDestroy(h->stream);
    if (stream) { h->stream = (cudaStream_t)stream; h->own_stream = false; }
    else { CK(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream"); h->own_stream = true; }
    for (auto &row : h->adv_graph)
        for (auto &g : row)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    return NS3D_OK;
}

int ns3d_synchronize(ns3d_handle *h) {
    if (!h) return NS3D_ERR_INVALID_ARG;
    int r = set_device(h); if (r) return r;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    return NS3D_OK;
}

int ns3d_last_launch_count(const ns3d_handle *h, long *count) {
    if (!h || !count) return NS3D_ERR_INVALID_ARG;
    *count = h->launches;
    return NS3D_OK;
}

// host Field3D array (sx*sy*sz doubles) -> padded device array
// Host Field3D arrays move as one contiguous copy each (full link bandwidth;
// a pitched 2-D copy of ~2 KB rows is several times slower) through a
// contiguous device staging array, repacked on the device.
__global__ void repack_kernel(const double *src, double *dst, Layout L, int to_padded) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.sx) return;
    const long flat = ((long)k * L.sy + j) * L.sx + i;
    if (to_padded) dst[L.at(i, j, k)] = src[flat];
    else dst[flat] = src[L.at(i, j, k)];
}

static int upload_plane(ns3d_handle *h, double *dst, const double *src, double *staging) {
    const Layout &L = h->L64;
    const size_t n = (size_t)L.sx * L.sy * L.sz;
    CK(h, cudaMemcpyAsync(staging, src, n * 8, cudaMemcpyHostToDevice, h->stream), "upload");
    repack_kernel<<<cell_grid(L, true, 128), 128, 0, h->stream>>>(staging, dst, L, 1);
    h->launches += 1;
    CK(h, cudaGetLastError(), "repack");
    return NS3D_OK;
}

static int download_plane(ns3d_handle *h, double *dst, const double *src, double *staging) {
    const Layout &L = h->L64;
    const size_t n = (size_t)L.sx * L.sy * L.sz;
    repack_kernel<<<cell_grid(L, true, 128), 128, 0, h->stream>>>(src, staging, L, 0);
    h->launches += 1;
    CK(h, cudaGetLastError(), "pack");
    CK(h, cudaMemcpyAsync(dst, staging, n * 8, cudaMemcpyDeviceToHost, h->stream), "download");
    return NS3D_OK;
}

// FP64 primitives of the full field sit in buffer b.  Plain path: b becomes
// the state (after the ghost fill when apply_bc).  Mixed path: FP64
// conserved state + FP32 primitives are derived from it.
__global__ void upload_mixed_kernel(const double *const *Wp, double *const *Up, float *const *W32, float *T32,
                                    Layout L, Layout L32, double gamma, double Rgas) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.sx) return;
    const long c = L.at(i, j, k), c32 = L32.at(i, j, k);
    double U[5];
    p2c_exact(Wp[0][c], Wp[1][c], Wp[2][c], Wp[3][c], Wp[4][c], gamma, U);
    double W[5];
    c2p_exact(U, gamma, W);
#pragma unroll
    for (int q = 0; q < 5; ++q) { Up[q][c] = U[q]; W32[q][c32] = (float)W[q]; }
    T32[c32] = (float)(W[4] / (W[0] * Rgas));
}

// The reference's built-in initialisers (initialization.cpp:516-638) on the
// device, writing primitives into a padded FP64 state buffer: the same
// cells, formulas and operation order (x = (ox + i - ngx + 0.5) dx with
// ox = 0 on one rank).  riemann_2d fills every cell including the ghosts;
// the others fill the interior only.
__global__ void init_kernel(double *const *Wp, Layout L, int kind, double dx, double dy, double Lx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.sx) return;
    const bool interior = i >= NG && i < NG + L.nx && j >= NG && j < NG + L.ny && k >= NG && k < NG + L.nz;
    double rho, u, v, w, p;
    const double x = ((double)(i - NG) + 0.5) * dx;
    if (kind == NS3D_INIT_RIEMANN_2D) {
        // initialize_riemann_2d, initialization.cpp:516-566 (four quadrants about (0.5, 0.5))
        const double y = ((double)(j - NG) + 0.5) * dy;
        w = 0.0;
        if (x >= 0.5 && y >= 0.5) { rho = 1.1; u = 0.0; v = 0.0; p = 1.1; }
        else if (x < 0.5 && y >= 0.5) { rho = 0.5065; u = 0.8939; v = 0.0; p = 0.35; }
        else if (x < 0.5 && y < 0.5) { rho = 1.1; u = 0.8939; v = 0.8939; p = 1.1; }
        else { rho = 0.5065; u = 0.0; v = 0.8939; p = 0.35; }
    } else {
        if (!interior) return;
        if (kind == NS3D_INIT_SOD) {
            // initialize_sod_shock_tube, initialization.cpp:568-596 (x_mid = 0.5 nx dx)
            const double x_mid = 0.5 * L.nx * dx;
            v = 0.0; w = 0.0; u = 0.0;
            if (x < x_mid) { rho = 1.0; p = 1.0; } else { rho = 0.125; p = 0.1; }
        } else if (kind == NS3D_INIT_UNIFORM) {
            // initialize_uniform_field, initialization.cpp:598-617
            rho = 1.0; u = 1.0; v = 1.0; w = 1.0; p = 1.0;
        } else {
            // initialize_sine_x_field, initialization.cpp:619-638: u = sin(2 pi x / Lx)
            rho = 1.0; v = 0.0; w = 0.0; p = 1.0;
            u = sin(2.0 * M_PI * x / Lx);
        }
    }
    const long c = L.at(i, j, k);
    Wp[0][c] = rho; Wp[1][c] = u; Wp[2][c] = v; Wp[3][c] = w; Wp[4][c] = p;
}

static int finish_upload(ns3d_handle *h, int b, bool apply_bc) {
    const int dst = (b + 1) % 3, dst2 = (b + 2) % 3;
    int r;
    h->visc_valid = false;
    if (!h->mixed) {
        if (!apply_bc) {
            dim3 g = cell_grid(h->L64, true, 128);
            temp_kernel64<<<g, 128, 0, h->stream>>>(state_table(h, b), h->T64, h->L64, h->ph.Rgas);
            h->launches += 1;
            CK(h, cudaGetLastError(), "temperature");
            h->s0 = b;
            return NS3D_OK;
        }
        if ((r = stage_async(h, 0, b, b, dst, 0.0))) return r;
        h->s0 = dst;
        return NS3D_OK;
    }
    dim3 g = cell_grid(h->L64, true, 128);
    upload_mixed_kernel<<<g, 128, 0, h->stream>>>(state_table(h, b), state_table(h, dst),
                                                  (float *const *)(h->dptr + 25), h->T32, h->L64, h->L32,
                                                  h->ph.gamma, h->ph.Rgas);
    h->launches += 1;
    CK(h, cudaGetLastError(), "upload conversion");
    h->s0 = dst;
    if (!apply_bc) return NS3D_OK;
    if ((r = stage_async(h, 0, dst, dst, dst2, 0.0))) return r;
    h->s0 = dst2;
    return NS3D_OK;
}

int ns3d_upload_primitives(ns3d_handle *h, const double *const fields[5]) {
    if (!h || !fields) return NS3D_ERR_INVALID_ARG;
    h->prev_valid = false;  // the free state buffers are scratch here
    for (int q = 0; q < 5; ++q) if (!fields[q]) return NS3D_ERR_INVALID_ARG;
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    const int b = (h->s0 + 1) % 3;
    const int stg = (h->s0 + 2) % 3;
    for (int q = 0; q < 5; ++q) if ((r = upload_plane(h, h->S[b][q], fields[q], h->S[stg][q]))) return r;
    if ((r = finish_upload(h, b, false))) return r;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    h->has_state = true;
    h->cfl_valid = false;
    return NS3D_OK;
}

int ns3d_set_interior_primitives(ns3d_handle *h, const double *const fields[5]) {
    if (!h || !fields) return NS3D_ERR_INVALID_ARG;
    h->prev_valid = false;  // the free state buffers are scratch here
    for (int q = 0; q < 5; ++q) if (!fields[q]) return NS3D_ERR_INVALID_ARG;
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    const Layout &L = h->L64;
    const size_t nb = (size_t)L.nx * L.ny * L.nz * 8;
    // stage the interior blocks in the RHS/viscous area? use the free state buffer
    const int b = (h->s0 + 1) % 3, tmp = (h->s0 + 2) % 3;
    // plain: the current state keeps its ghosts (initially the allocate defaults)
    // mixed: the current FP64 primitives are recomputed from the conserved state
    if (h->mixed) {
        dim3 g = cell_grid(L, true, 128);
        derive_kernel_mixed<<<g, 128, 0, h->stream>>>(state_table(h, h->s0), state_table(h, b), L, h->ph.gamma,
                                                       h->ph.Rgas, NS3D_PRIMITIVE);
        h->launches += 1;
    } else {
        for (int q = 0; q < 5; ++q)
            CK(h, cudaMemcpyAsync(h->S[b][q], h->S[h->s0][q], L.plane * 8, cudaMemcpyDeviceToDevice, h->stream), "copy");
    }
    for (int q = 0; q < 5; ++q) {
        double *stage_buf = h->S[tmp][q];
        CK(h, cudaMemcpyAsync(stage_buf, fields[q], nb, cudaMemcpyHostToDevice, h->stream), "upload interior");
        scatter_interior<double><<<cell_grid(L, false, 128), 128, 0, h->stream>>>(stage_buf, h->S[b][q], L);
        h->launches += 1;
    }
    CK(h, cudaGetLastError(), "scatter");
    // apply_boundary + primitiveToConserved (main.cpp:98-99)
    if ((r = finish_upload(h, b, true))) return r;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    h->has_state = true;
    h->cfl_valid = false;
    return NS3D_OK;
}

int ns3d_initialize(ns3d_handle *h, int kind) {
    if (!h || kind < NS3D_INIT_RIEMANN_2D || kind > NS3D_INIT_ISOTROPIC) return NS3D_ERR_INVALID_ARG;
    h->prev_valid = false;  // the free state buffers are scratch here
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    const Layout &L = h->L64;
    const int b = (h->s0 + 1) % 3;
    // the cells the initialiser does not write keep their current values
    // (initially the Field3D::allocate defaults), as in the reference
    if (h->mixed) {
        dim3 g = cell_grid(L, true, 128);
        derive_kernel_mixed<<<g, 128, 0, h->stream>>>(state_table(h, h->s0), state_table(h, b), L, h->ph.gamma,
                                                       h->ph.Rgas, NS3D_PRIMITIVE);
        h->launches += 1;
    } else {
        for (int q = 0; q < 5; ++q)
            CK(h, cudaMemcpyAsync(h->S[b][q], h->S[h->s0][q], L.plane * 8, cudaMemcpyDeviceToDevice, h->stream), "copy");
    }
    if (kind == NS3D_INIT_ISOTROPIC) {
        if ((r = isotropic_fill(state_table(h, b), L, h->ph.Rgas, h->stream, h->err))) return r;
    } else {
        init_kernel<<<cell_grid(L, true, 128), 128, 0, h->stream>>>(state_table(h, b), L, kind, h->ph.dx, h->ph.dy,
                                                                     h->G.Lx);
        h->launches += 1;
    }
    CK(h, cudaGetLastError(), "initialiser");
    // apply_boundary + primitiveToConserved (main.cpp:98-99)
    if ((r = finish_upload(h, b, true))) return r;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    h->has_state = true;
    h->cfl_valid = false;
    return NS3D_OK;
}

int ns3d_download(ns3d_handle *h, int what, double *const out[]) {
    if (!h || !out) return NS3D_ERR_INVALID_ARG;
    h->prev_valid = false;  // the free state buffers are scratch here
    if (what < NS3D_PRIMITIVE || what > NS3D_TEMPERATURE) return NS3D_ERR_INVALID_ARG;
    const int nq = what == NS3D_TEMPERATURE ? 1 : 5;
    for (int q = 0; q < nq; ++q) if (!out[q]) return NS3D_ERR_INVALID_ARG;
    if (!h->has_state && what != NS3D_RHS) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    int r = set_device(h); if (r) return r;
    const Layout &L = h->L64;
    const int free_b = (h->s0 + 1) % 3, free2 = (h->s0 + 2) % 3;
    // scratch for derived groups: the free state buffers (their contents are dead between steps)
    double *const *scr = state_table(h, free_b);
    dim3 g = cell_grid(L, true, 128);
    if (what == NS3D_RHS) {
        if (!h->rhs_complete)
            return fail(h, NS3D_ERR_STATE,
                        "the RHS buffer holds no complete right-hand side: an RK3 step's last stage stores "
                        "it only when the handle was created with keep_rhs = 1 (else call ns3d_compute_rhs)");
        if (!h->mixed) {
            for (int q = 0; q < 5; ++q) if ((r = download_plane(h, out[q], h->rhs64[q], h->S[free_b][q]))) return r;
        } else {
            for (int q = 0; q < 5; ++q)
                widen_kernel<float><<<g, 128, 0, h->stream>>>(h->rhs32[q], h->S[free_b][q], h->L32, L);
            for (int q = 0; q < 5; ++q) if ((r = download_plane(h, out[q], h->S[free_b][q], h->S[free2][q]))) return r;
        }
    } else if (!h->mixed) {
        if (what == NS3D_PRIMITIVE) {
            for (int q = 0; q < 5; ++q) if ((r = download_plane(h, out[q], h->S[h->s0][q], h->S[free_b][q]))) return r;
        } else {
            derive_kernel64<<<g, 128, 0, h->stream>>>(state_table(h, h->s0), scr, L, h->ph.gamma, h->ph.Rgas, what);
            CK(h, cudaGetLastError(), "derive");
            for (int q = 0; q < nq; ++q) if ((r = download_plane(h, out[q], h->S[free_b][q], h->S[free2][q]))) return r;
        }
    } else {
        if (what == NS3D_CONSERVED) {
            for (int q = 0; q < 5; ++q) if ((r = download_plane(h, out[q], h->S[h->s0][q], h->S[free_b][q]))) return r;
        } else {
            derive_kernel_mixed<<<g, 128, 0, h->stream>>>(state_table(h, h->s0), scr, L, h->ph.gamma, h->ph.Rgas, what);
            CK(h, cudaGetLastError(), "derive");
            for (int q = 0; q < nq; ++q) if ((r = download_plane(h, out[q], h->S[free_b][q], h->S[free2][q]))) return r;
        }
    }
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    return NS3D_OK;
}

int ns3d_apply_boundary(ns3d_handle *h) {
    if (!h) return NS3D_ERR_INVALID_ARG;
    h->prev_valid = false;  // the free state buffers are scratch here
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    const int dst = (h->s0 + 1) % 3;
    if ((r = stage_async(h, 0, h->s0, h->s0, dst, 0.0))) return r;
    h->s0 = dst;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    return NS3D_OK;
}

int check_device_error(ns3d_handle *h);

int ns3d_compute_rhs(ns3d_handle *h) {
    if (!h) return NS3D_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    if ((r = compute_rhs_async(h))) return r;
    return check_device_error(h);
}

// The kernels' bounded waits record a non-zero error word instead of
// spinning for ever; read it after the work of an entry point.
int check_device_error(ns3d_handle *h) {
    int code = 0;
    CK(h, cudaMemcpyAsync(&code, h->dev_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "error word");
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    if (code) {
        cudaMemsetAsync(h->dev_err, 0, sizeof(int), h->stream);
        return fail(h, NS3D_ERR_TIMEOUT, "a device-side wait for a TMA tile ran out (error word " +
                                             std::to_string(code) + ")");
    }
    return NS3D_OK;
}

int ns3d_rk3_step(ns3d_handle *h, double dt) {
    if (!h) return NS3D_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    if (is_slab(h))
        return fail(h, NS3D_ERR_STATE, "a z-slab steps stage by stage (ns3d_rk3_stage) with a halo exchange between");
    if (!std::isfinite(dt)) return fail(h, NS3D_ERR_INVALID_ARG, "dt is not finite");
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    h->prev_valid = false;
    if ((r = rk3_async(h, dt))) return r;
    h->prev_valid = true;
    if ((r = check_device_error(h))) return r;
    if (h->P.check_state) return check_state(h);
    return NS3D_OK;
}

// One step per graph launch; the step graph is captured for the buffer
// rotation state it starts from, so three consecutive graphs cover a cycle.
int ns3d_rk3_steps(ns3d_handle *h, int nsteps, double dt) {
    if (!h || nsteps < 0) return NS3D_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    if (is_slab(h))
        return fail(h, NS3D_ERR_STATE, "a z-slab steps stage by stage (ns3d_rk3_stage) with a halo exchange between");
    if (!std::isfinite(dt)) return fail(h, NS3D_ERR_INVALID_ARG, "dt is not finite");
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    for (int s = 0; s < nsteps; ++s) {
        h->prev_valid = false;
        if ((r = rk3_async(h, dt))) return r;
        h->prev_valid = true;
    }
    if ((r = check_device_error(h))) return r;
    if (h->P.check_state) return check_state(h);
    return NS3D_OK;
}

int ns3d_compute_timestep(ns3d_handle *h, double *dt_out) {
    if (!h || !dt_out) return NS3D_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    if (h->cfl_valid) {
        // the last RK stage left the per-block minima of this state
        prof_begin(h, "cfl_combine");
        const int nb = h->red_blocks;  // partials holds at least red_blocks values
        min_combine_kernel<<<nb, 256, 0, h->stream>>>(h->cfl_part, h->cfl_count, h->partials);
        min_combine_kernel<<<1, 256, 0, h->stream>>>(h->partials, nb, h->scalars);
        prof_end(h);
        h->launches += 2;
        CK(h, cudaGetLastError(), "cfl combine");
        double m = 0;
        CK(h, cudaMemcpyAsync(&m, h->scalars, sizeof(double), cudaMemcpyDeviceToHost, h->stream), "copy dt");
        CK(h, cudaStreamSynchronize(h->stream), "synchronize");
        *dt_out = h->P.cfl * m;
        return NS3D_OK;
    }
    prof_begin(h, "cfl_dt");
    if (!h->mixed)
        dt_kernel64<<<h->red_blocks, RED_THREADS, 0, h->stream>>>(state_table(h, h->s0), h->L64, h->ph.gamma,
                                                                  h->ph.dx, h->partials, h->zlo, h->zhi - h->zlo);
    else
        dt_kernel_mixed<<<h->red_blocks, RED_THREADS, 0, h->stream>>>(state_table(h, h->s0), h->L64, h->ph.gamma,
                                                                      h->ph.dx, h->partials, h->zlo, h->zhi - h->zlo);
    prof_end(h);
    h->launches += 1;
    CK(h, cudaGetLastError(), "dt kernel");
    double m = 0;
    if ((r = reduce_combine(h, 1, 1, &m))) return r;
    *dt_out = h->P.cfl * m;
    return NS3D_OK;
}

int ns3d_diagnostics(ns3d_handle *h, double out[6]) {
    if (!h || !out) return NS3D_ERR_INVALID_ARG;
    h->prev_valid = false;  // the free state buffers are scratch here
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    const double vol = h->ph.dx * h->ph.dy * h->ph.dz;
    double s[5];
    if (!h->mixed && h->ph.mu != 0.0 && !h->diag_separate) {
        // the viscous kernel's gradient pass (TMA plane tiles, register
        // windows) with the sums instead of the node fluxes
        long nb = 0;
        if ((r = visc_launch<double>(h, h->visc_red, &nb))) return r;
        if ((r = reduce_combine(h, 5, 0, s, h->visc_red, nb))) return r;
        if ((r = check_device_error(h))) return r;
    } else if (!h->mixed) {
        diag_kernel<double><<<h->red_blocks, RED_THREADS, 0, h->stream>>>(visc_args<double>(h), vol, h->partials,
                                                                           h->zlo, h->zhi - h->zlo);
    } else {
        // FP64 primitives of the current conserved state for the reductions
        const int b = (h->s0 + 1) % 3;
        dim3 g = cell_grid(h->L64, true, 128);
        derive_kernel_mixed<<<g, 128, 0, h->stream>>>(state_table(h, h->s0), state_table(h, b), h->L64, h->ph.gamma,
                                                       h->ph.Rgas, NS3D_PRIMITIVE);
        const int bt = (h->s0 + 2) % 3;
        derive_kernel_mixed<<<g, 128, 0, h->stream>>>(state_table(h, h->s0), state_table(h, bt), h->L64, h->ph.gamma,
                                                       h->ph.Rgas, NS3D_TEMPERATURE);
        h->launches += 1;
        ViscArgs<double> a = visc_args<double>(h);
        for (int q = 0; q < 5; ++q) a.W[q] = h->S[b][q];
        a.T = h->S[bt][0];
        a.L = h->L64;
        diag_kernel<double><<<h->red_blocks, RED_THREADS, 0, h->stream>>>(a, vol, h->partials, h->zlo, h->zhi - h->zlo);
        h->launches += 1;
    }
    if (h->mixed || h->ph.mu == 0.0 || h->diag_separate) {
        h->launches += 1;
        CK(h, cudaGetLastError(), "diagnostics");
        if ((r = reduce_combine(h, 5, 0, s))) return r;
    }
    const double N = (double)h->G.nx * h->G.ny * (h->zhi - h->zlo);  // the owned cells
    const double mean_mu = s[2] / N, mean_rho = s[3] / N;
    out[0] = s[0];
    out[1] = s[1] / N;
    out[2] = mean_mu;
    out[3] = mean_rho;
    out[4] = (mean_mu / mean_rho) * (s[1] / N);
    out[5] = std::sqrt(s[4] / (3.0 * N));
    return NS3D_OK;
}

int ns3d_residuals(ns3d_handle *h, double out[5]) {
    if (!h || !out) return NS3D_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    if (!h->prev_valid)
        return fail(h, NS3D_ERR_STATE,
                    "no step-start state to difference against: call right after an RK3 step or "
                    "ns3d_time_advance, before any download or upload");
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    const int prev = (h->s0 + 2) % 3;
    const double dx3 = h->ph.dx * h->ph.dx * h->ph.dx;  // compute_diagnostics weights by dx^3
    if (!h->mixed)
        residual_kernel<false><<<h->red_blocks, RED_THREADS, 0, h->stream>>>(
            state_table(h, h->s0), state_table(h, prev), h->L64, h->ph.gamma, dx3, h->partials, h->zlo, h->zhi - h->zlo);
    else
        residual_kernel<true><<<h->red_blocks, RED_THREADS, 0, h->stream>>>(
            state_table(h, h->s0), state_table(h, prev), h->L64, h->ph.gamma, dx3, h->partials, h->zlo, h->zhi - h->zlo);
    residual_combine_kernel<<<1, 32, 0, h->stream>>>(h->partials, h->red_blocks, h->scalars);
    h->launches += 2;
    CK(h, cudaGetLastError(), "residuals");
    double v[10];
    CK(h, cudaMemcpyAsync(v, h->scalars, sizeof(v), cudaMemcpyDeviceToHost, h->stream), "copy residuals");
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    for (int q = 0; q < 5; ++q) out[q] = std::sqrt(v[q]) / v[5 + q];
    return NS3D_OK;
}

int ns3d_total_energy(ns3d_handle *h, double *ke_out) {
    if (!h || !ke_out) return NS3D_ERR_INVALID_ARG;
    if (h->cfl_valid) {
        // the last RK stage left the per-block kinetic energies of this state
        int r = set_device(h); if (r) return r;
        h->launches = 0;
        const int nb = h->red_blocks;
        sum_combine_kernel<<<nb, 256, 0, h->stream>>>(h->ke_part, h->cfl_count, h->partials);
        sum_combine_kernel<<<1, 256, 0, h->stream>>>(h->partials, nb, h->scalars);
        h->launches += 2;
        CK(h, cudaGetLastError(), "kinetic energy combine");
        CK(h, cudaMemcpyAsync(ke_out, h->scalars, sizeof(double), cudaMemcpyDeviceToHost, h->stream), "copy energy");
        CK(h, cudaStreamSynchronize(h->stream), "synchronize");
        return NS3D_OK;
    }
    double d[6];
    int r = ns3d_diagnostics(h, d);
    if (r) return r;
    *ke_out = d[0];
    return NS3D_OK;
}

// time_advance's dt schedule (maincycle.cpp:18-56) without output.
// Steps per captured time-advance graph.  A launch executes the longest
// graph that fits the remaining step budget, so a budgeted run wastes no
// launches; only the launch in which t_end is reached may carry steps that
// return at once (a no-op step still costs about 0.1 ms of block scheduling).
constexpr int ADV_LENS[3] = {12, 3, 1};

// The CFL minimum of the current state into clock->cfl_min: from the last
// stage's per-block minima when they describe it, else the separate reduction.
int seed_cfl_min(ns3d_handle *h) {
    if (h->cfl_valid) {
        min_combine_kernel<<<h->red_blocks, 256, 0, h->stream>>>(h->cfl_part, h->cfl_count, h->partials);
    } else if (!h->mixed) {
        dt_kernel64<<<h->red_blocks, RED_THREADS, 0, h->stream>>>(state_table(h, h->s0), h->L64, h->ph.gamma,
                                                                  h->ph.dx, h->partials, h->zlo, h->zhi - h->zlo);
    } else {
        dt_kernel_mixed<<<h->red_blocks, RED_THREADS, 0, h->stream>>>(state_table(h, h->s0), h->L64, h->ph.gamma,
                                                                      h->ph.dx, h->partials, h->zlo, h->zhi - h->zlo);
    }
    min_combine_kernel<<<1, 256, 0, h->stream>>>(h->partials, h->red_blocks, &h->clock->cfl_min);
    h->launches += 2;
    CK(h, cudaGetLastError(), "cfl seed");
    return NS3D_OK;
}

// Capture ADV_LENS[li] device-scheduled steps starting from buffer rotation s0:
// schedule -> three (RHS, stage) pairs reading dt from the clock -> the CFL
// minimum of the new state into the clock for the next step.
int capture_adv_graph(ns3d_handle *h, int li, int s0) {
    // one ordinary RHS first: every kernel's attributes are set and its
    // launch checked before any of it is captured (it only writes the RHS
    // scratch arrays)
    int rr = compute_rhs_async(h);
    if (rr) return rr;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    const int keep = h->s0;
    const bool keep_valid = h->cfl_valid;  // capturing executes nothing: the stored minima stay as they were
    const bool keep_rhs_flag = h->rhs_complete, keep_visc = h->visc_valid;
    h->s0 = s0;
    h->dev_loop = true;
    cudaGraph_t g = nullptr;
    int r = NS3D_OK;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (int n = 0; n < ADV_LENS[li] && r == NS3D_OK; ++n) {
            schedule_kernel<<<1, 1, 0, h->stream>>>(h->clock, h->P.cfl, h->P.dt_fixed, 1e-12);
            r = rk3_async(h, 0.0);
            if (r == NS3D_OK) {
                min_combine_kernel<<<h->red_blocks, 256, 0, h->stream>>>(h->cfl_part, h->cfl_count, h->partials);
                min_combine_kernel<<<1, 256, 0, h->stream>>>(h->partials, h->red_blocks, &h->clock->cfl_min);
            }
        }
        cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
        if (e == cudaSuccess) e = e2;
    }
    h->dev_loop = false;
    h->s0 = keep;
    h->cfl_valid = keep_valid;
    h->rhs_complete = keep_rhs_flag;
    h->visc_valid = keep_visc;
    if (r == NS3D_OK && e == cudaSuccess) e = cudaGraphInstantiate(&h->adv_graph[li][s0], g, 0);
    if (g) cudaGraphDestroy(g);
    if (r != NS3D_OK) return r;
    if (e != cudaSuccess) { h->adv_graph[li][s0] = nullptr; return cuda_fail(h, e, "time-advance graph"); }
    return NS3D_OK;
}

// time_advance with the dt schedule on the device: up to 12 steps per graph
// launch, one host synchronisation per launch.  Same dt sequence and state as
// the host loop below, bit for bit.
int time_advance_device(ns3d_handle *h, double t_end, int max_steps, double *time, int *steps_done) {
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    // all graphs are captured at the first call of a handle, so no capture
    // (and its set-up synchronisation) falls inside a later run
    for (int li = 0; li < 3; ++li)
        for (int b = 0; b < 3; ++b)
            if (!h->adv_graph[li][b] && (r = capture_adv_graph(h, li, b))) return r;
    DevClock c{*time, 0.0, t_end, 0.0, 0, 0, max_steps, 0};
    CK(h, cudaMemcpyAsync(h->clock, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream), "clock");
    if (h->P.dt_fixed < 0.0 && (r = seed_cfl_min(h))) return r;
    int total = 0;
    while (true) {
        const int s0 = h->s0;
        const int left = max_steps - total;
        const int li = left >= ADV_LENS[0] ? 0 : (left >= ADV_LENS[1] ? 1 : 2);
        CK(h, cudaGraphLaunch(h->adv_graph[li][s0], h->stream), "graph launch");
        h->launches += (long)ADV_LENS[li] * (3 + 3 * ((h->ph.mu != 0.0 ? 1 : 0) + 4));
        CK(h, cudaMemcpyAsync(&c, h->clock, sizeof(c), cudaMemcpyDeviceToHost, h->stream), "clock");
        CK(h, cudaStreamSynchronize(h->stream), "synchronize");
        const int ran = c.steps - total;  // steps this launch executed (the rest returned at once)
        total = c.steps;
        h->s0 = (s0 + ran) % 3;
        if (ran > 0) {
            h->visc_valid = false;
            h->cfl_valid = true;
            h->rhs_complete = h->P.keep_rhs != 0;
            h->prev_valid = true;
        }
        if ((r = check_device_error(h))) break;
        if (c.err) { r = fail(h, NS3D_ERR_DT, "dt too small or zero"); break; }
        if (h->P.check_state && ran > 0 && (r = check_state(h))) break;
        if (c.done) break;
    }
    *time = c.t;
    if (steps_done) *steps_done = total;
    return r;
}

int ns3d_time_advance(ns3d_handle *h, double t_end, int max_steps, double *time, int *steps_done) {
    if (!h || !time) return NS3D_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    if (is_slab(h))
        return fail(h, NS3D_ERR_STATE, "a z-slab steps stage by stage (ns3d_rk3_stage) with a halo exchange between");
    // per-kernel event profiling cannot sit inside a captured graph
    if (!h->profiling && max_steps > 0) return time_advance_device(h, t_end, max_steps, time, steps_done);
    const double eps = 1e-12;
    int done = 0, r = NS3D_OK;
    double t = *time;
    for (int step = 1; step <= max_steps; ++step) {
        if (std::fabs(t_end - t) <= eps) break;
        double dt = h->P.dt_fixed;
        if (h->P.dt_fixed < 0.0 && (r = ns3d_compute_timestep(h, &dt))) break;
        if (t + dt > t_end) dt = t_end - t;
        if (dt <= eps) { r = fail(h, NS3D_ERR_DT, "dt too small or zero"); break; }
        t += dt;
        if ((r = ns3d_rk3_step(h, dt))) break;
        ++done;
        if (t >= t_end) break;
    }
    *time = t;
    if (steps_done) *steps_done = done;
    return r;
}

int ns3d_set_slab(ns3d_handle *h, int z_begin, int z_end, double dz, int z_periodic) {
    if (!h || z_begin < 0 || z_end > h->G.nz || z_end - z_begin < 1) return NS3D_ERR_INVALID_ARG;
    if (z_periodic && (z_begin == 0 || z_end == h->G.nz))
        return fail(h, NS3D_ERR_INVALID_ARG, "a slab of a z-periodic domain has halos on both z sides");
    if (!(dz > 0.0) && dz != 0.0) return NS3D_ERR_INVALID_ARG;
    const bool slab = z_begin != 0 || z_end != h->G.nz;
    if (slab && ((z_begin != 0 && z_begin < 6) || (z_end != h->G.nz && h->G.nz - z_end < 6) || z_end - z_begin < 6))
        return fail(h, NS3D_ERR_INVALID_ARG, "a z-slab needs six halo planes on each bordering side and six owned planes");
    if (slab && h->bc.periodic[2])
        return fail(h, NS3D_ERR_CONFIG, "a z-slab's local z boundaries are its halos: give them a non-periodic type");
    int r = set_device(h); if (r) return r;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    // captured time-advance graphs hold the old launch geometry
    for (auto &row : h->adv_graph)
        for (auto &g : row)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    h->zlo = z_begin;
    h->zhi = z_end;
    h->slab_z_periodic = z_periodic != 0;
    h->visc_valid = false;
    if (dz > 0.0) { h->ph.dz = dz; h->ph.inv_dz = 1.0 / dz; }
    h->cfl_valid = false;
    h->prev_valid = false;
    h->step_start = -1;
    return NS3D_OK;
}

int ns3d_rk3_stage(ns3d_handle *h, int stage, double dt) {
    if (!h || stage < 1 || stage > 3) return NS3D_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    if (!std::isfinite(dt)) return fail(h, NS3D_ERR_INVALID_ARG, "dt is not finite");
    if (stage != 1 && (h->step_start < 0 || h->s0 != (h->step_start + stage - 1) % 3))
        return fail(h, NS3D_ERR_STATE, "RK3 stages run in order 1, 2, 3");
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    if (stage == 1) {
        h->prev_valid = false;
        h->step_start = h->s0;
    }
    // rk3_async's buffers: (1: s0, s0 -> b1), (2: s0, b1 -> b2), (3: s0, b2 -> b1)
    const int s0 = h->step_start, b1 = (s0 + 1) % 3, b2 = (s0 + 2) % 3;
    const int srcc = stage == 1 ? s0 : (stage == 2 ? b1 : b2);
    const int dst = stage == 2 ? b2 : b1;
    if ((r = rk_stage_async(h, stage, s0, srcc, dst, dt))) {
        h->s0 = s0;
        h->step_start = -1;
        return r;
    }
    h->s0 = dst;
    if (stage == 3) {
        h->step_start = -1;
        h->prev_valid = true;
        if ((r = check_device_error(h))) return r;
        if (h->P.check_state) return check_state(h);
    }
    return NS3D_OK;
}

int ns3d_device_fields(ns3d_handle *h, int what, void *ptrs[5], long layout[6]) {
    if (!h || !ptrs || !layout) return NS3D_ERR_INVALID_ARG;
    const Layout *L = &h->L64;
    long esz = 8;
    if (what == NS3D_PRIMITIVE && !h->mixed) {
        for (int q = 0; q < 5; ++q) ptrs[q] = h->S[h->s0][q];
    } else if (what == NS3D_PRIMITIVE && h->mixed) {
        for (int q = 0; q < 5; ++q) ptrs[q] = h->w32[q];
        L = &h->L32; esz = 4;
    } else if (what == NS3D_CONSERVED && h->mixed) {
        for (int q = 0; q < 5; ++q) ptrs[q] = h->S[h->s0][q];
    } else if (what == NS3D_RHS) {
        for (int q = 0; q < 5; ++q) ptrs[q] = h->mixed ? (void *)h->rhs32[q] : (void *)h->rhs64[q];
        if (h->mixed) { L = &h->L32; esz = 4; }
    } else if (what == NS3D_TEMPERATURE) {
        ptrs[0] = h->mixed ? (void *)h->T32 : (void *)h->T64;
        for (int q = 1; q < 5; ++q) ptrs[q] = nullptr;
        if (h->mixed) { L = &h->L32; esz = 4; }
    } else {
        return fail(h, NS3D_ERR_INVALID_ARG, "group not resident on the device in this precision");
    }
    layout[0] = L->sx; layout[1] = L->sy; layout[2] = L->sz; layout[3] = L->px; layout[4] = L->off; layout[5] = esz;
    return NS3D_OK;
}

int ns3d_vjp_rhs(ns3d_handle *h, const double *const rbar[5], double *const ubar[5]) {
    if (!h || !rbar || !ubar) return NS3D_ERR_INVALID_ARG;
    h->visc_valid = false;
    h->prev_valid = false;  // the free state buffers are scratch here
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    std::string why;
    if (!adjoint_supported(h, why)) return fail(h, NS3D_ERR_CONFIG, why);
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    if ((r = ensure_adjoint(h))) return r;
    if ((r = upload_interior_slot(h, rbar, 3))) return r;
    if ((r = axpby_slot(h, 0, 0, 0.0, 0.0))) return r;
    if ((r = vjp_rhs_async(h, h->S[h->s0], 3, 0))) return r;
    return download_interior_slot(h, 0, ubar);
}

int ns3d_vjp_rk3_step(ns3d_handle *h, double dt, const double *const ubar_next[5], double *const ubar[5]) {
    if (!h || !ubar_next || !ubar) return NS3D_ERR_INVALID_ARG;
    h->visc_valid = false;
    h->prev_valid = false;  // the free state buffers are scratch here
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    std::string why;
    if (!adjoint_supported(h, why)) return fail(h, NS3D_ERR_CONFIG, why);
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    if ((r = ensure_adjoint(h))) return r;
    // stage states of the step from the current state; the state is restored
    const size_t bytes = (size_t)h->L64.plane * 8;
    double *buf = nullptr;
    CK(h, cudaMalloc(&buf, 15 * bytes), "stage buffers");
    double *st[3][5];
    for (int b = 0; b < 3; ++b)
        for (int q = 0; q < 5; ++q) st[b][q] = buf + (size_t)(5 * b + q) * h->L64.plane;
    const int s_keep = h->s0;
    r = rk3_async_store(h, dt, st);
    if (!r) {
        for (int q = 0; q < 5; ++q)
            cudaMemcpyAsync(h->S[s_keep][q], st[0][q], bytes, cudaMemcpyDeviceToDevice, h->stream);
        h->s0 = s_keep;
        h->cfl_valid = false;
        r = refresh_T(h);
        if (!r) r = upload_interior_slot(h, ubar_next, 0);
    }
    if (!r) r = vjp_step_async(h, st[0], st[1], st[2], dt);
    if (!r) r = download_interior_slot(h, 0, ubar);
    cudaStreamSynchronize(h->stream);
    cudaFree(buf);
    return r;
}

int ns3d_adjoint_kinetic_energy(ns3d_handle *h, int nsteps, double dt, int checkpoint_every, double *J,
                                double *const grad[3], double stats[4]) {
    if (!h || !J || !grad || nsteps < 1 || checkpoint_every < 1) return NS3D_ERR_INVALID_ARG;
    h->visc_valid = false;
    h->prev_valid = false;
    if (!h->has_state) return fail(h, NS3D_ERR_STATE, "no state uploaded");
    std::string why;
    if (!adjoint_supported(h, why)) return fail(h, NS3D_ERR_CONFIG, why);
    int r = set_device(h); if (r) return r;
    h->launches = 0;
    if ((r = ensure_adjoint(h))) return r;
    const int ce = checkpoint_every;
    const int nck = (nsteps + ce - 1) / ce;
    const size_t plane = (size_t)h->L64.plane, bytes = plane * 8;
    // checkpoints (nck states) + one segment of stage states (ce x 3 states)
    const size_t store_bytes = (size_t)(nck + 3 * ce) * 5 * bytes;
    double *store = nullptr;
    CK(h, cudaMalloc(&store, store_bytes), "checkpoint storage");
    auto ck = [&](int c, int q) { return store + ((size_t)c * 5 + q) * plane; };
    auto seg = [&](int step, int stage, int q) { return store + ((size_t)(nck + 3 * step + stage) * 5 + q) * plane; };
    cudaEvent_t e0, e1, em, e2;
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&em); cudaEventCreate(&e2);
    const int s_init = h->s0;
    double Jv = 0.0;
    cudaEventRecord(e0, h->stream);
    // ---- forward with checkpoints every ce steps
    for (int n = 0; n < nsteps && !r; ++n) {
        if (n % ce == 0)
            for (int q = 0; q < 5; ++q)
                if (cudaMemcpyAsync(ck(n / ce, q), h->S[h->s0][q], bytes, cudaMemcpyDeviceToDevice, h->stream))
                    r = fail(h, NS3D_ERR_CUDA, "checkpoint copy");
        if (r) break;
        const int n0_last = (nck - 1) * ce;
        if (n >= n0_last) {
            // the last segment keeps its stage states from this pass: the
            // backward sweep starts there without recomputing it
            double *st[3][5];
            for (int b = 0; b < 3; ++b)
                for (int q = 0; q < 5; ++q) st[b][q] = seg(n - n0_last, b, q);
            r = rk3_async_store(h, dt, st);
        } else {
            r = rk3_async(h, dt);
        }
    }
    cudaEventRecord(e1, h->stream);
    long recomputed = 0;
    if (!r) {
        // objective of the final state and its adjoint seed
        AdjArgs a = adj_args(h, h->S[h->s0], h->ab[3], h->ab[0]);
        cudaError_t e = adj_ke_seed(a, h->ph.dx * h->ph.dy * h->ph.dz, h->adj_tab, h->stream);
        if (e != cudaSuccess) r = cuda_fail(h, e, "seed");
    }
    if (!r) {
        double d[6];
        r = ns3d_diagnostics(h, d);
        Jv = d[0];
    }
    cudaEventRecord(em, h->stream);  // backward pass starts here
    // ---- backward: per segment recompute the stage states, then step back
    for (int c = nck - 1; c >= 0 && !r; --c) {
        const int n0 = c * ce, n1 = (n0 + ce < nsteps) ? n0 + ce : nsteps;
        const bool stored = c == nck - 1;  // stage states kept by the forward pass
        if (!stored) {
            for (int q = 0; q < 5; ++q)
                cudaMemcpyAsync(h->S[h->s0][q], ck(c, q), bytes, cudaMemcpyDeviceToDevice, h->stream);
            r = refresh_T(h);
        }
        for (int n = n0; n < n1 && !r && !stored; ++n) {
            double *st[3][5];
            for (int b = 0; b < 3; ++b)
                for (int q = 0; q < 5; ++q) st[b][q] = seg(n - n0, b, q);
            r = rk3_async_store(h, dt, st);
            ++recomputed;
        }
        for (int n = n1 - 1; n >= n0 && !r; --n) {
            double *W0[5], *W1[5], *W2[5];
            for (int q = 0; q < 5; ++q) { W0[q] = seg(n - n0, 0, q); W1[q] = seg(n - n0, 1, q); W2[q] = seg(n - n0, 2, q); }
            r = vjp_step_async(h, W0, W1, W2, dt);
        }
    }
    cudaEventRecord(e2, h->stream);
    if (!r) {
        // initial state back into the handle, gradient w.r.t. the initial velocity
        for (int q = 0; q < 5; ++q)
            cudaMemcpyAsync(h->S[s_init][q], ck(0, q), bytes, cudaMemcpyDeviceToDevice, h->stream);
        h->s0 = s_init;
        h->cfl_valid = false;
        AdjArgs a = adj_args(h, h->S[h->s0], h->ab[3], h->ab[0]);
        cudaError_t e = adj_velocity_grad(a, h->adj_tab, h->adj_tab + 20, h->stream);
        if (e != cudaSuccess) r = cuda_fail(h, e, "velocity gradient");
        const size_t nb = (size_t)h->L64.nx * h->L64.ny * h->L64.nz * 8;
        for (int q = 0; q < 3 && !r; ++q)
            if (cudaMemcpyAsync(grad[q], h->gvel[q], nb, cudaMemcpyDeviceToHost, h->stream))
                r = fail(h, NS3D_ERR_CUDA, "gradient copy");
        // T of the restored state for the next RHS
        if (!r) r = refresh_T(h);
    }
    cudaStreamSynchronize(h->stream);
    float fwd_ms = 0.f, adj_ms = 0.f;
    cudaEventElapsedTime(&fwd_ms, e0, e1);
    cudaEventElapsedTime(&adj_ms, em, e2);
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(em); cudaEventDestroy(e2);
    cudaFree(store);
    if (r) return r;
    *J = Jv;
    if (stats) {
        stats[0] = fwd_ms; stats[1] = adj_ms;
        stats[2] = (double)(store_bytes + h->adj_bytes);
        stats[3] = (double)recomputed;
    }
    return NS3D_OK;
}

int ns3d_profile(ns3d_handle *h, int enable) {
    if (!h) return NS3D_ERR_INVALID_ARG;
    int r = set_device(h); if (r) return r;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    for (auto &p : h->prof)
        for (auto e : p.ev) cudaEventDestroy(e);
    h->prof.clear();
    h->profiling = enable != 0;
    return NS3D_OK;
}

int ns3d_profile_report(ns3d_handle *h, char *buf, long len) {
    if (!h || !buf || len <= 0) return NS3D_ERR_INVALID_ARG;
    int r = set_device(h); if (r) return r;
    CK(h, cudaStreamSynchronize(h->stream), "synchronize");
    std::string out;
    for (auto &p : h->prof) {
        double ms = 0.0;
        for (size_t q = 0; q + 1 < p.ev.size(); q += 2) {
            float t = 0.f;
            CK(h, cudaEventElapsedTime(&t, p.ev[q], p.ev[q + 1]), "event time");
            ms += t;
        }
        char line[160];
        std::snprintf(line, sizeof(line), "%s %ld %.6f\n", p.name, p.launches, ms);
        out += line;
    }
    if ((long)out.size() + 1 > len) return fail(h, NS3D_ERR_INVALID_ARG, "report buffer too small");
    std::memcpy(buf, out.c_str(), out.size() + 1);
    return NS3D_OK;
}

}  // extern "C"
