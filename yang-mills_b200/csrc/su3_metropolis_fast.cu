// su3_metropolis_fast.cu -- the tiled SU(3) FP64 sub-sweep in its fast form
// (ym_ensemble_set_fast_sweeps; no reference counterpart): the kernels of
// su3_tiled.cuh compiled with fused multiply-adds and with cos_sin_horner
// rotations.  Links, staple, action change and accept test stay binary64 and
// the algorithm, streams and decisions are the exact form's; a product
// rounded once instead of twice and the Horner rotation move a link by a few
// ulps per update (on a 16^4 lattice from a Haar start: at most 9.3e-16
// after one sweep and 3.2e-15 after ten, with every accept decision the
// exact form's), so a decision changes only when its uniform lies within
// that distance of exp(-dS).
#define YM_TILED_FAST 1
#include "su3_tiled.cuh"

namespace ym {

cudaError_t launch_su3_metropolis_fast(ym_ensemble *e, int parity, int mu, double angle, int uniform) {
    return tiled_fast::tiled_launch(e, parity, mu, angle, uniform);
}

cudaError_t launch_su3_metropolis_measure_fast(ym_ensemble *e, int mu, double angle, double *tr_partial) {
    return tiled_fast::tiled_launch_measure(e, mu, angle, tr_partial);
}

}  // namespace ym
