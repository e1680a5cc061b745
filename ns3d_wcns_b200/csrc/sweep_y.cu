// sweep_y.cu -- instantiations of the fused inviscid sweep along y
// (one translation unit per direction so the builds run in parallel).
#include "sweep_pair.cuh"

namespace ns3d {
cudaError_t sweep_y(const SweepArgs<double> &a, cudaStream_t st) { return sweep_select<1, double>(a, st); }
cudaError_t sweep_y(const SweepArgs<float> &a, cudaStream_t st) { return sweep_select_f32<1>(a, st); }
}  // namespace ns3d
