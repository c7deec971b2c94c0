// Local H|psi> kernels instantiated for a cubic 96^3 box (radix split 8 x 12).
#include "hkpsi_kernels.cuh"

namespace cpwb {
CPWB_INSTANTIATE(double, 8, 12, 8, 12, 8, 12, 32, 32)
CPWB_INSTANTIATE(float, 8, 12, 8, 12, 8, 12, 32, 32)
}  // namespace cpwb
