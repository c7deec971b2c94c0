// Dispatch of the local H|psi> to a compile-time specialised kernel set when the
// box is cubic with a known radix split and the batches are 32 wide, otherwise
// to the generic (run-time radix) set.
#include "hkpsi_kernels.cuh"

namespace cpwb {

namespace kern {
// specialisations compiled in hkpsi_spec_*.cu
#define CPWB_DECLARE(T, RX1, RX2, RY1, RY2, RZ1, RZ2, TC, CB)                                                  \
  extern template cudaError_t launch_impl<T, RX1, RX2, RY1, RY2, RZ1, RZ2, TC, CB>(CPWB_LAUNCH_ARGS(T));        \
  extern template cudaError_t launch_inv_impl<T, RX1, RX2, RY1, RY2, TC>(CPWB_INV_ARGS(T));
CPWB_DECLARE(double, 4, 8, 4, 8, 4, 8, 32, 32)
CPWB_DECLARE(float, 4, 8, 4, 8, 4, 8, 32, 32)
CPWB_DECLARE(double, 5, 8, 5, 8, 5, 8, 32, 32)
CPWB_DECLARE(float, 5, 8, 5, 8, 5, 8, 32, 32)
CPWB_DECLARE(double, 8, 12, 8, 12, 8, 12, 32, 32)
CPWB_DECLARE(float, 8, 12, 8, 12, 8, 12, 32, 32)
CPWB_DECLARE(double, 12, 12, 12, 12, 12, 12, 32, 32)
CPWB_DECLARE(double, 12, 12, 12, 12, 12, 12, 32, 16)
CPWB_DECLARE(float, 12, 12, 12, 12, 12, 12, 32, 16)
CPWB_DECLARE(float, 12, 12, 12, 12, 12, 12, 32, 32)
CPWB_DECLARE(double, 0, 0, 0, 0, 0, 0, 0, 0)
CPWB_DECLARE(float, 0, 0, 0, 0, 0, 0, 0, 0)
}  // namespace kern

static bool is_split(const FftDim& d, int r1, int r2) { return d.r1 == r1 && d.r2 == r2; }

template <typename T>
cudaError_t launch_local(CPWB_LAUNCH_ARGS(T)) {
  // 144^3 with the z stage in 16-column tiles
  if (p.n1 == p.n2 && p.n2 == p.n3 && p.tcol == 32 && p.cb == 16 && is_split(p.dx, 12, 12))
    return kern::launch_impl<T, 12, 12, 12, 12, 12, 12, 32, 16>(p, nbc, band0, psi, ldpsi, hpsi, ldh, plane_start,
                                                               pw_idx, pw_pos, ekpg, vr, twx, twy, twz, W, st, ev);
  const bool cubic = p.n1 == p.n2 && p.n2 == p.n3 && p.tcol == 32 && p.cb == 32;
  if (cubic && is_split(p.dx, 8, 12))
    return kern::launch_impl<T, 8, 12, 8, 12, 8, 12, 32, 32>(p, nbc, band0, psi, ldpsi, hpsi, ldh, plane_start,
                                                            pw_idx, pw_pos, ekpg, vr, twx, twy, twz, W, st, ev);
  if (cubic && is_split(p.dx, 12, 12))
    return kern::launch_impl<T, 12, 12, 12, 12, 12, 12, 32, 32>(p, nbc, band0, psi, ldpsi, hpsi, ldh, plane_start,
                                                               pw_idx, pw_pos, ekpg, vr, twx, twy, twz, W, st, ev);
  if (cubic && is_split(p.dx, 4, 8))
    return kern::launch_impl<T, 4, 8, 4, 8, 4, 8, 32, 32>(p, nbc, band0, psi, ldpsi, hpsi, ldh, plane_start,
                                                         pw_idx, pw_pos, ekpg, vr, twx, twy, twz, W, st, ev);
  if (cubic && is_split(p.dx, 5, 8))
    return kern::launch_impl<T, 5, 8, 5, 8, 5, 8, 32, 32>(p, nbc, band0, psi, ldpsi, hpsi, ldh, plane_start,
                                                         pw_idx, pw_pos, ekpg, vr, twx, twy, twz, W, st, ev);
  return kern::launch_impl<T, 0, 0, 0, 0, 0, 0, 0, 0>(p, nbc, band0, psi, ldpsi, hpsi, ldh, plane_start, pw_idx,
                                                     pw_pos, ekpg, vr, twx, twy, twz, W, st, ev);
}

template cudaError_t launch_local<double>(CPWB_LAUNCH_ARGS(double));
template cudaError_t launch_local<float>(CPWB_LAUNCH_ARGS(float));

template <typename T>
cudaError_t launch_inverse_xy(CPWB_INV_ARGS(T)) {
  const bool cubic = p.n1 == p.n2 && p.n2 == p.n3 && p.tcol == 32;   // kernel A does not depend on the z tile
  if (cubic && is_split(p.dx, 8, 12))
    return kern::launch_inv_impl<T, 8, 12, 8, 12, 32>(p, nbc, band0, psi, ldpsi, plane_start, pw_idx, pw_pos, twx,
                                                     twy, W, st);
  if (cubic && is_split(p.dx, 12, 12))
    return kern::launch_inv_impl<T, 12, 12, 12, 12, 32>(p, nbc, band0, psi, ldpsi, plane_start, pw_idx, pw_pos, twx,
                                                       twy, W, st);
  if (cubic && is_split(p.dx, 4, 8))
    return kern::launch_inv_impl<T, 4, 8, 4, 8, 32>(p, nbc, band0, psi, ldpsi, plane_start, pw_idx, pw_pos, twx, twy,
                                                   W, st);
  if (cubic && is_split(p.dx, 5, 8))
    return kern::launch_inv_impl<T, 5, 8, 5, 8, 32>(p, nbc, band0, psi, ldpsi, plane_start, pw_idx, pw_pos, twx, twy,
                                                   W, st);
  return kern::launch_inv_impl<T, 0, 0, 0, 0, 0>(p, nbc, band0, psi, ldpsi, plane_start, pw_idx, pw_pos, twx, twy, W,
                                                st);
}
template cudaError_t launch_inverse_xy<double>(CPWB_INV_ARGS(double));
template cudaError_t launch_inverse_xy<float>(CPWB_INV_ARGS(float));

}  // namespace cpwb
