// Kernel instances of the mixed-precision optimizer (R = float terms and
// vectors, A = double reductions).  Split per precision so the instances
// compile in parallel.
#include "mmff_kernels.cuh"

namespace mmffb {

// The instance a plan selects: CTA size, register-cached H columns, matrix in
// shared memory or in a global slot, dense BFGS or L-BFGS.
template <class Fn>
static int with_instance(const Plan &pl, bool lb, const Fn &fn) {
    using R = float;
    using A = double;
    if (lb) {
        if (pl.nt == 512) return fn.template run<R, A, 512, 0, false, true>();   // 16 warps, global slot
        if (!pl.msm) return pl.nc == 0 ? fn.template run<R, A, 256, 0, false, true>()   // 128 registers
                                       : fn.template run<R, A, 256, 2, false, true>();
        return pl.nc == 0 ? fn.template run<R, A, 256, 0, true, true>()     // 128 registers, 2 CTAs/SM
                          : fn.template run<R, A, 256, 2, true, true>();
    }
    if (!pl.msm) {
        if (pl.nc == 0) return pl.nt == 512 ? fn.template run<R, A, 512, 0, false, false>()
                                            : fn.template run<R, A, 256, 0, false, false>();
        return fn.template run<R, A, 256, 16, false, false>();
    }
    if (pl.nt == 64) return fn.template run<R, A, 64, 4, true, false>();
    if (pl.nt == 128) return fn.template run<R, A, 128, 8, true, false>();
    if (pl.nc == 0) return fn.template run<R, A, 256, 0, true, false>();     // 128 registers, 2 CTAs/SM
    return fn.template run<R, A, 256, 8, true, false>();
}

int minimize_mixed(const Params &P, const Plan &pl, cudaStream_t st) {
    return with_instance(pl, P.hist_m > 0, LaunchFn{P, pl, st});
}

int occupancy_mixed(const Plan &pl, bool lb) { return with_instance(pl, lb, OccFn{pl}); }

int energy_grad_mixed(const Params &P, float *grad, cudaStream_t st) {
    return launch_eg<float, double, 128>(P, grad, st);
}

}  // namespace mmffb
