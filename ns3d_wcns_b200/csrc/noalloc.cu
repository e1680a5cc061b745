// noalloc.cu -- CFL time step over caller-owned device arrays with no device
// allocation at all.
//
// Some host codes cannot let a library call cudaMalloc: solvers that carve
// every device byte out of their own pre-sized pool (a stray allocation breaks
// their memory accounting, or fails once the pool has taken the GPU's
// memory).  For them this entry
// point does the work of ns3d_compute_timestep without a handle: its only
// scratch, the per-block partial minima of the reduction, is a fixed
// file-scope device array that every GPU which loads the library keeps until
// the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/ns3d_b200.h"
#include "common.cuh"
#include "reduce.cuh"

using namespace ns3d;

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_CELLS_PER_THREAD = 32;
static_assert((long)NS3D_NOALLOC_MAX_BLOCKS * NOALLOC_THREADS * NOALLOC_CELLS_PER_THREAD == NS3D_NOALLOC_MAX_CELLS,
              "header limits out of step with the kernel");

// Partial minima, one per block of the reduction.  Each call writes the
// entries it then reads, so nothing has to be cleared between calls.
static __device__ __align__(256) double g_noalloc_partials[NS3D_NOALLOC_MAX_BLOCKS];

// Device address of g_noalloc_partials, looked up once per CUDA context: in
// host code the array's name is only a host-side stand-in, not a device
// address.  The cache is keyed on the context's unique id (cuCtxGetId), not
// on the device ordinal: after cudaDeviceReset, or under another context on
// the same device, the module is loaded anew at another address, and a
// context id is never reused within a process.
constexpr int ADDR_CACHE = 64;
struct AddrEntry {
    unsigned long long ctx_id;
    double *addr;
};
AddrEntry g_addr_cache[ADDR_CACHE] = {};
int g_addr_next = 0;
std::mutex g_setup_mutex;

typedef int (*CtxGetCurrentFn)(void **);
typedef int (*CtxGetIdFn)(void *, unsigned long long *);

// Unique id of the calling thread's current context (0: none, or the driver
// does not offer the query).
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *f1 = nullptr, *f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess)
            get_current = (CtxGetCurrentFn)f1;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)f2;
        cudaGetLastError();
        looked_up = true;
    }
    if (!get_current || !get_id) return 0;
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

struct FieldPtrs {
    const double *p[5];  // rho, u, v, w, p
};

// Fixed block -> cells assignment (no grid-stride loop), so the number of
// partials equals the number of blocks: 256 * 32 cells per block.
__global__ void __launch_bounds__(NOALLOC_THREADS)
cfl_partials_kernel(FieldPtrs W, Layout L, double gamma, double dx, double *partials) {
    const long ncell = (long)L.nx * L.ny * L.nz;
    const long first = (long)blockIdx.x * NOALLOC_THREADS * NOALLOC_CELLS_PER_THREAD + threadIdx.x;
    double m = 1e9;  // dt_local's initial value, timestep.cpp:6
    for (int r = 0; r < NOALLOC_CELLS_PER_THREAD; ++r) {
        const long t = first + (long)r * NOALLOC_THREADS;
        if (t >= ncell) break;
        const int i = (int)(t % L.nx), j = (int)((t / L.nx) % L.ny), k = (int)(t / ((long)L.nx * L.ny));
        const long c = L.at(i + NG, j + NG, k + NG);
        double U[5];
        p2c_exact(W.p[0][c], W.p[1][c], W.p[2][c], W.p[3][c], W.p[4][c], gamma, U);
        m = fmin(m, cfl_bound(U, gamma, dx));
    }
    block_min(m, partials + blockIdx.x);
}

// One block: strided minimum over the partials, then a block minimum.  The
// minimum does not depend on the order, so the result is the same bits as a
// sequential pass.
__global__ void __launch_bounds__(NOALLOC_THREADS)
cfl_combine_kernel(const double *partials, int nblocks, double cfl, double *dt_out) {
    __shared__ double m_out;
    double m = 1e300;
    for (int b = threadIdx.x; b < nblocks; b += NOALLOC_THREADS) m = fmin(m, partials[b]);
    block_min_n<NOALLOC_THREADS>(m, &m_out);
    if (threadIdx.x == 0) *dt_out = cfl * m_out;
}

}  // namespace

extern "C" int ns3d_compute_timestep_noalloc(const double *const d_fields[5], int nx, int ny, int nz, double gamma,
                                             double cfl, double dx, double *d_dt_out, void *stream) {
    if (!d_fields || !d_dt_out || nx < 1 || ny < 1 || nz < 1) return NS3D_ERR_INVALID_ARG;
    FieldPtrs W;
    for (int q = 0; q < 5; ++q) {
        if (!d_fields[q]) return NS3D_ERR_INVALID_ARG;
        W.p[q] = d_fields[q];
    }
    const long ncell = (long)nx * ny * nz;
    if (ncell > NS3D_NOALLOC_MAX_CELLS) return NS3D_ERR_SIZE;
    const long per_block = (long)NOALLOC_THREADS * NOALLOC_CELLS_PER_THREAD;
    const int nblocks = (int)((ncell + per_block - 1) / per_block);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return NS3D_ERR_NO_DEVICE;
    }
    double *partials = nullptr;
    {
        // one-time set-up for the caller's current context (device)
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        unsigned long long id = current_context_id();
        for (int e = 0; id && e < ADDR_CACHE; ++e)
            if (g_addr_cache[e].ctx_id == id) partials = g_addr_cache[e].addr;
        if (!partials) {
            // the look-up also makes the device's primary context current
            // when the thread has none yet
            if (cudaGetSymbolAddress((void **)&partials, g_noalloc_partials) != cudaSuccess || !partials) {
                cudaGetLastError();
                return NS3D_ERR_CUDA;
            }
            if (!id) id = current_context_id();
            if (id) {
                g_addr_cache[g_addr_next] = {id, partials};
                g_addr_next = (g_addr_next + 1) % ADDR_CACHE;
            }
        }
    }
    Layout L;
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.sx = nx + 2 * NG; L.sy = ny + 2 * NG; L.sz = nz + 2 * NG;
    L.px = L.sx; L.off = 0;  // caller arrays: unpadded Field3D layout
    L.plane = (long)L.sx * L.sy * L.sz;
    cudaStream_t st = (cudaStream_t)stream;
    cfl_partials_kernel<<<nblocks, NOALLOC_THREADS, 0, st>>>(W, L, gamma, dx, partials);
    cfl_combine_kernel<<<1, NOALLOC_THREADS, 0, st>>>(partials, nblocks, cfl, d_dt_out);
    return cudaGetLastError() == cudaSuccess ? NS3D_OK : NS3D_ERR_CUDA;
}
