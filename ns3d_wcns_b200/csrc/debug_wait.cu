// debug_wait.cu -- exercise of the bounded mbarrier wait on the device.
//
// A block arms an mbarrier for 16 bytes that no copy will deliver, so its
// phase never completes; the bounded wait gives up after `polls` polls,
// writes the device error word and the block returns.  Nothing faults or
// hangs: this is how the tests check the failure path of the TMA waits.
#include <cuda_runtime.h>

#include "../../include/ns3d_b200.h"
#include "tma.cuh"

namespace ns3d {
namespace {

__global__ void wait_timeout_kernel(unsigned polls, int *err, int *finished) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16);  // bytes that never arrive
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0u, err, polls);
    __syncthreads();
    if (threadIdx.x == 0 && !ok) atomicAdd(finished, 1);
}

}  // namespace
}  // namespace ns3d

extern "C" int ns3d_debug_wait_timeout(int device, unsigned polls, int *code_out) {
    using namespace ns3d;
    if (!code_out || polls == 0) return NS3D_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return NS3D_ERR_CUDA; }
    int *d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(int)) != cudaSuccess) { cudaGetLastError(); return NS3D_ERR_OOM; }
    int h[2] = {0, 0};
    cudaError_t e = cudaMemset(d, 0, 2 * sizeof(int));
    if (e == cudaSuccess) {
        wait_timeout_kernel<<<4, 64>>>(polls, d, d + 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return NS3D_ERR_CUDA;
    *code_out = h[0];
    // every block gave up and returned on its own
    return (h[0] != 0 && h[1] == 4) ? NS3D_ERR_TIMEOUT : NS3D_OK;
}
