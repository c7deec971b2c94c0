// Local H|psi> kernels instantiated for any supported box (run-time radices).
#include "hkpsi_kernels.cuh"

namespace cpwb {
CPWB_INSTANTIATE(double, 0, 0, 0, 0, 0, 0, 0, 0)
CPWB_INSTANTIATE(float, 0, 0, 0, 0, 0, 0, 0, 0)
}  // namespace cpwb
