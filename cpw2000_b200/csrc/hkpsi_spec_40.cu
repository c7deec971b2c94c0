// Local H|psi> kernels instantiated for a cubic 40^3 box (radix split 5 x 8).
#include "hkpsi_kernels.cuh"

namespace cpwb {
CPWB_INSTANTIATE(double, 5, 8, 5, 8, 5, 8, 32, 32)
CPWB_INSTANTIATE(float, 5, 8, 5, 8, 5, 8, 32, 32)
}  // namespace cpwb
