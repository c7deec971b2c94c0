// Local H|psi> kernels instantiated for a cubic 32^3 box (radix split 4 x 8).
#include "hkpsi_kernels.cuh"

namespace cpwb {
CPWB_INSTANTIATE(double, 4, 8, 4, 8, 4, 8, 32, 32)
CPWB_INSTANTIATE(float, 4, 8, 4, 8, 4, 8, 32, 32)
}  // namespace cpwb
