// debug_detector.cu -- the MDCD_HYBRID discontinuity detector evaluated by
// the device, for tests of its decision against the reference's quotient
// form (interpolation.cpp:149-160) on near-threshold stencils.
#include <cuda_runtime.h>

#include "../../include/ns3d_b200.h"
#include "schemes.cuh"

namespace ns3d {
namespace {

__global__ void detector_kernel(const double *__restrict__ s5, long n, int *__restrict__ out) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double *s = s5 + 5 * i;
        out[i] = mdcd_smooth<double>(s[0], s[1], s[2], s[3], s[4]) ? 1 : 0;
    }
}

}  // namespace
}  // namespace ns3d

extern "C" int ns3d_debug_mdcd_detector(int device, long n, const double *stencils, int *smooth_out) {
    using namespace ns3d;
    if (n < 0 || (n > 0 && (!stencils || !smooth_out)) || n > (1L << 26)) return NS3D_ERR_INVALID_ARG;
    if (n == 0) return NS3D_OK;
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return NS3D_ERR_CUDA; }
    double *ds = nullptr;
    int *dout = nullptr;
    if (cudaMalloc(&ds, sizeof(double) * 5 * n) != cudaSuccess) { cudaGetLastError(); return NS3D_ERR_OOM; }
    if (cudaMalloc(&dout, sizeof(int) * n) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(ds);
        return NS3D_ERR_OOM;
    }
    cudaError_t e = cudaMemcpy(ds, stencils, sizeof(double) * 5 * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const long blocks = (n + 255) / 256;
        detector_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256>>>(ds, n, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(smooth_out, dout, sizeof(int) * n, cudaMemcpyDeviceToHost);
    cudaFree(ds);
    cudaFree(dout);
    return e == cudaSuccess ? NS3D_OK : NS3D_ERR_CUDA;
}
