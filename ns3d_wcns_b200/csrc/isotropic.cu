// isotropic.cu -- the reference's isotropic-turbulence initial field on the
// device: generate_full_turbulence (isotropic_ini.cpp:26-126) and the
// interior assignment of init_isotropic_turbulence (isotropic_ini.cpp:131-193).
//
// The reference draws three random phases per Fourier mode from a
// std::mt19937_64 seeded with 123 (rnd01, isotropic_ini.cpp:16-20), builds a
// solenoidal spectrum with amplitude sqrt(2/3) sqrt(A k^2 exp(-2 k^2/k0^2) /
// (4 pi)), k0 = 8, A = 0.00013, transforms it back with an unnormalised
// inverse FFT (FFTW_BACKWARD), keeps the real parts and scales them to the
// kinetic energy Ek0 = 3A/64 sqrt(2 pi) k0^5.  Here the phases come from the
// same generator on the host (one z-plane of modes at a time), the spectrum is
// built on the device, and the inverse transform is a direct DFT along each
// axis in turn (any grid size; O(n) work per output, a few ms at 256^3): the
// same sums as the FFT, in another order, so the field agrees with the
// reference to rounding.  The spectra use the reference's array order, index
// (i*NY + j)*NZ + k (z fastest).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ns3d_b200.h"
#include "common.cuh"
#include "isotropic.cuh"

namespace ns3d {
namespace {

constexpr double ISO_PI = 3.14159265358979323846;
constexpr int ISO_K0 = 8;
constexpr double ISO_A = 0.00013;
constexpr int ISO_MAX_N = 2048;  // longest line of the direct DFT (shared memory)

// MT19937-64 (M. Matsumoto and T. Nishimura, ACM TOMACS 8 (1998) 3-30; the
// 64-bit parameters that the C++ standard gives std::mt19937_64).
class Mt64 {
public:
    explicit Mt64(uint64_t seed) {
        mt_[0] = seed;
        for (int i = 1; i < N; ++i) mt_[i] = 6364136223846793005ULL * (mt_[i - 1] ^ (mt_[i - 1] >> 62)) + (uint64_t)i;
        idx_ = N;
    }
    uint64_t next() {
        if (idx_ >= N) twist();
        uint64_t y = mt_[idx_++];
        y ^= (y >> 29) & 0x5555555555555555ULL;
        y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
        y ^= (y << 37) & 0xFFF7EEE000000000ULL;
        y ^= y >> 43;
        return y;
    }
    // uniform_real_distribution<double>(0, 1) as libstdc++ draws it: one 64-bit
    // output rounded to double and scaled by 2^-64 (generate_canonical with 53
    // bits), kept below 1
    double uniform01() {
        const double r = (double)next() * 0x1p-64;
        return r >= 1.0 ? std::nextafter(1.0, 0.0) : r;
    }

private:
    static constexpr int N = 312, M = 156;
    void twist() {
        const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
        for (int i = 0; i < N; ++i) {
            const uint64_t x = (mt_[i] & upper) | (mt_[(i + 1) % N] & lower);
            uint64_t xa = x >> 1;
            if (x & 1ULL) xa ^= 0xB5026F5AA96619E9ULL;
            mt_[i] = mt_[(i + M) % N] ^ xa;
        }
        idx_ = 0;
    }
    uint64_t mt_[N];
    int idx_;
};

// The modes of z-plane k from the plane's phases (three per mode, [j][i][3],
// in the reference's draw order): the solenoidal projection of three random
// complex vectors (isotropic_ini.cpp:43-79)
__global__ void iso_modes_kernel(const double *phase, double2 *U, double2 *V, double2 *W, int NX, int NY, int NZ,
                                 int k) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= NX) return;
    const long id = ((long)i * NY + j) * NZ + k;
    const int k1 = i <= NX / 2 ? i : i - NX, k2 = j <= NY / 2 ? j : j - NY, k3 = k <= NZ / 2 ? k : k - NZ;
    const int kk = k1 * k1 + k2 * k2 + k3 * k3;
    if (kk == 0) {
        U[id] = make_double2(0.0, 0.0); V[id] = make_double2(0.0, 0.0); W[id] = make_double2(0.0, 0.0);
        return;
    }
    const double Ak = sqrt(2.0 / 3.0) * sqrt(ISO_A * kk * exp(-2.0 * kk / (double)(ISO_K0 * ISO_K0)) / (4.0 * ISO_PI));
    const double *ph = phase + 3 * ((long)j * NX + i);
    const double a1 = 2 * ISO_PI * ph[0], a2 = 2 * ISO_PI * ph[1], a3 = 2 * ISO_PI * ph[2];
    const double v1r = Ak * sin(a1), v1i = Ak * cos(a1);
    const double v2r = Ak * sin(a2), v2i = Ak * cos(a2);
    const double v3r = Ak * sin(a3), v3i = Ak * cos(a3);
    const double vkr = k1 * v1r + k2 * v2r + k3 * v3r;
    const double vki = k1 * v1i + k2 * v2i + k3 * v3i;
    U[id] = make_double2(k1 * vkr / kk - v1r, k1 * vki / kk - v1i);
    V[id] = make_double2(k2 * vkr / kk - v2r, k2 * vki / kk - v2i);
    W[id] = make_double2(k3 * vkr / kk - v3r, k3 * vki / kk - v3i);
}

// In-place unnormalised inverse DFT, exponent +1 (FFTW_BACKWARD), of every
// line along one axis of the (NX, NY, NZ) array: out[x] = sum_t in[t] e^{2 pi i t x / n}.
// One block per line; the line and the n twiddles e^{2 pi i m / n} sit in
// shared memory, each thread sums the outputs x = tid, tid + blockDim, ...
constexpr int DFT_THREADS = 256;
constexpr int DFT_MAX_OUT = ISO_MAX_N / DFT_THREADS;

__global__ void __launch_bounds__(DFT_THREADS) iso_dft_kernel(double2 *a, int axis, int NX, int NY, int NZ) {
    extern __shared__ double2 sh[];
    const int n = axis == 0 ? NX : (axis == 1 ? NY : NZ);
    double2 *line = sh, *tw = sh + n;
    const long l = blockIdx.x;
    long base, stride;
    if (axis == 2) { base = l * NZ; stride = 1; }                                   // lines (i, j)
    else if (axis == 1) { base = (l / NZ) * (long)NY * NZ + l % NZ; stride = NZ; }  // lines (i, k)
    else { base = l; stride = (long)NY * NZ; }                                      // lines (j, k)
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        line[t] = a[base + t * stride];
        double s, c;
        sincospi(2.0 * t / n, &s, &c);
        tw[t] = make_double2(c, s);
    }
    __syncthreads();
    double2 out[DFT_MAX_OUT];
    int nout = 0;
    for (int x = threadIdx.x; x < n; x += blockDim.x, ++nout) {
        double re = 0.0, im = 0.0;
        int m = 0;  // t * x mod n
        for (int t = 0; t < n; ++t) {
            const double2 v = line[t], w = tw[m];
            re += v.x * w.x - v.y * w.y;
            im += v.x * w.y + v.y * w.x;
            m += x;
            if (m >= n) m -= n;
        }
        out[nout] = make_double2(re, im);
    }
    nout = 0;
    for (int x = threadIdx.x; x < n; x += blockDim.x, ++nout) a[base + x * stride] = out[nout];
}

// per-block sums of 0.5 (u^2 + v^2 + w^2) over the real parts
__global__ void __launch_bounds__(256) iso_energy_kernel(const double2 *U, const double2 *V, const double2 *W, long N,
                                                         double *part) {
    __shared__ double s[256];
    double acc = 0.0;
    for (long id = (long)blockIdx.x * blockDim.x + threadIdx.x; id < N; id += (long)gridDim.x * blockDim.x) {
        const double u = U[id].x, v = V[id].x, w = W[id].x;
        acc += 0.5 * (u * u + v * v + w * w);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// the interior of the handle's primitive arrays (init_isotropic_turbulence:
// rho = 1, T = 1, p = Rgas rho T, the scaled velocity)
__global__ void iso_write_kernel(double *const *Wp, Layout L, const double2 *U, const double2 *V, const double2 *W,
                                 double scale, double Rgas) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.nx) return;
    const long id = ((long)i * L.ny + j) * L.nz + k;
    const long c = L.at(i + NG, j + NG, k + NG);
    Wp[0][c] = 1.0;
    Wp[1][c] = U[id].x * scale;
    Wp[2][c] = V[id].x * scale;
    Wp[3][c] = W[id].x * scale;
    Wp[4][c] = Rgas * 1.0 * 1.0;
}

}  // namespace

int isotropic_fill(double *const *Wp, const Layout &L, double Rgas, cudaStream_t st, std::string &err) {
    const int NX = L.nx, NY = L.ny, NZ = L.nz;
    if (NX > ISO_MAX_N || NY > ISO_MAX_N || NZ > ISO_MAX_N) {
        err = "isotropic initialiser: at most 2048 cells along each axis";
        return NS3D_ERR_CONFIG;
    }
    const long N = (long)NX * NY * NZ;
    double2 *spec = nullptr;
    double *phase = nullptr, *part = nullptr;
    constexpr int EBLOCKS = 1024;
    auto fail = [&](const char *what, cudaError_t e) {
        err = std::string("isotropic initialiser: ") + what + ": " + cudaGetErrorString(e);
        cudaFree(spec); cudaFree(phase); cudaFree(part);
        return e == cudaErrorMemoryAllocation ? NS3D_ERR_OOM : NS3D_ERR_CUDA;
    };
    cudaError_t e = cudaMalloc(&spec, sizeof(double2) * 3 * (size_t)N);
    if (e != cudaSuccess) return fail("spectra", e);
    if ((e = cudaMalloc(&phase, sizeof(double) * 3 * (size_t)NX * NY)) != cudaSuccess) return fail("phases", e);
    if ((e = cudaMalloc(&part, sizeof(double) * EBLOCKS)) != cudaSuccess) return fail("partials", e);
    double2 *U = spec, *V = spec + N, *W = spec + 2 * N;

    // the phases in the reference's draw order: k, then j, then i; none for the zero mode
    Mt64 rng(123);
    std::vector<double> host(3 * (size_t)NX * NY);
    const dim3 mgrid((NX + 127) / 128, NY);
    for (int k = 0; k < NZ; ++k) {
        const int k3 = k <= NZ / 2 ? k : k - NZ;
        for (int j = 0; j < NY; ++j) {
            const int k2 = j <= NY / 2 ? j : j - NY;
            for (int i = 0; i < NX; ++i) {
                const int k1 = i <= NX / 2 ? i : i - NX;
                double *ph = &host[3 * ((size_t)j * NX + i)];
                if (k1 * k1 + k2 * k2 + k3 * k3 == 0) { ph[0] = ph[1] = ph[2] = 0.0; continue; }
                ph[0] = rng.uniform01(); ph[1] = rng.uniform01(); ph[2] = rng.uniform01();
            }
        }
        // the kernel of the previous plane reads the staging buffer: copy after it
        if ((e = cudaMemcpyAsync(phase, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, st)) !=
            cudaSuccess)
            return fail("phase upload", e);
        iso_modes_kernel<<<mgrid, 128, 0, st>>>(phase, U, V, W, NX, NY, NZ, k);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail("modes", e);
    }
    // inverse transform of each component along z, y, x
    const int maxn = std::max(NX, std::max(NY, NZ));
    const size_t smem = 2 * sizeof(double2) * (size_t)maxn;
    if (smem > 48 * 1024 &&
        (e = cudaFuncSetAttribute(iso_dft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return fail("DFT shared memory", e);
    for (double2 *c : {U, V, W}) {
        iso_dft_kernel<<<(unsigned)((long)NX * NY), DFT_THREADS, 2 * sizeof(double2) * NZ, st>>>(c, 2, NX, NY, NZ);
        iso_dft_kernel<<<(unsigned)((long)NX * NZ), DFT_THREADS, 2 * sizeof(double2) * NY, st>>>(c, 1, NX, NY, NZ);
        iso_dft_kernel<<<(unsigned)((long)NY * NZ), DFT_THREADS, 2 * sizeof(double2) * NX, st>>>(c, 0, NX, NY, NZ);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail("DFT", e);
    // normalise the kinetic energy to Ek0 (isotropic_ini.cpp:108-123)
    iso_energy_kernel<<<EBLOCKS, 256, 0, st>>>(U, V, W, N, part);
    std::vector<double> hp(EBLOCKS);
    if ((e = cudaMemcpyAsync(hp.data(), part, sizeof(double) * EBLOCKS, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return fail("energy", e);
    double Er = 0.0;
    for (double x : hp) Er += x;
    Er /= (double)N;
    const double Ek0 = 3.0 * ISO_A / 64.0 * std::sqrt(2 * ISO_PI) * std::pow(ISO_K0, 5);
    const double scale = std::sqrt(Ek0 / Er);
    iso_write_kernel<<<dim3((NX + 127) / 128, NY, NZ), 128, 0, st>>>(Wp, L, U, V, W, scale, Rgas);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return fail("write", e);
    cudaFree(spec); cudaFree(phase); cudaFree(part);
    return NS3D_OK;
}

}  // namespace ns3d
