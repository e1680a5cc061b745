// sweep_z.cu -- instantiations of the fused inviscid sweep along z
// (one translation unit per direction so the builds run in parallel).
#include "sweep_pair.cuh"

namespace ns3d {
cudaError_t sweep_z(const SweepArgs<double> &a, cudaStream_t st) { return sweep_select<2, double>(a, st); }
cudaError_t sweep_z(const SweepArgs<float> &a, cudaStream_t st) { return sweep_select_f32<2>(a, st); }
}  // namespace ns3d
