// The Lanczos three-term update of one complex entry (single_lanczos_iteration,
// eigen/src/lanczos.c:708-738), written with explicitly rounded operations so
// that every kernel that applies it -- k_update after a product, and the
// product that regenerates recurrence segments with the update fused -- gives
// the same bits:  r = w - (alpha q + beta_prev p), q = rc * iq, p = rp * ip,
// where iq = 1 / beta_prev and ip = 1 / beta_prevprev (0 at the first step).
#pragma once

namespace tbgpu {

__device__ __forceinline__ double2 lanczos_update_entry(double2 w, double2 rc, double2 rp,
                                                       double al, double bprev, double iq,
                                                       double ip) {
  const double qx = __dmul_rn(rc.x, iq), qy = __dmul_rn(rc.y, iq);
  const double px = __dmul_rn(rp.x, ip), py = __dmul_rn(rp.y, ip);
  return make_double2(__dsub_rn(w.x, __fma_rn(al, qx, __dmul_rn(bprev, px))),
                      __dsub_rn(w.y, __fma_rn(al, qy, __dmul_rn(bprev, py))));
}

}  // namespace tbgpu
