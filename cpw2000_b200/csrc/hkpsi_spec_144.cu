// Local H|psi> kernels instantiated for a cubic 144^3 box (radix split 12 x 12), with the
// z stage in 32- and 16-column tiles.
#include "hkpsi_kernels.cuh"

namespace cpwb {
CPWB_INSTANTIATE(double, 12, 12, 12, 12, 12, 12, 32, 32)
CPWB_INSTANTIATE(float, 12, 12, 12, 12, 12, 12, 32, 32)
template cudaError_t kern::launch_impl<double, 12, 12, 12, 12, 12, 12, 32, 16>(CPWB_LAUNCH_ARGS(double));
template cudaError_t kern::launch_impl<float, 12, 12, 12, 12, 12, 12, 32, 16>(CPWB_LAUNCH_ARGS(float));
}  // namespace cpwb
