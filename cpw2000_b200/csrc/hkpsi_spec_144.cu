// Local H|psi> kernels instantiated for a cubic 144^3 box (radix split 12 x 12).
#include "hkpsi_kernels.cuh"

namespace cpwb {
CPWB_INSTANTIATE(double, 12, 12, 12, 12, 12, 12, 32, 32)
CPWB_INSTANTIATE(float, 12, 12, 12, 12, 12, 12, 32, 32)
}  // namespace cpwb
