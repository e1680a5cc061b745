// sweep_x.cu -- instantiations of the fused inviscid sweep along x
// (one translation unit per direction so the builds run in parallel).
#include "sweep_pair.cuh"

namespace ns3d {
cudaError_t sweep_x(const SweepArgs<double> &a, cudaStream_t st) { return sweep_select<0, double>(a, st); }
cudaError_t sweep_x(const SweepArgs<float> &a, cudaStream_t st) { return sweep_select_f32<0>(a, st); }
}  // namespace ns3d
