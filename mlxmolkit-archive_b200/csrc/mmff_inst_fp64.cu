// Kernel instances of the fp64-precision optimizer (R = double terms and
// vectors, A = double reductions).  Split per precision so the instances
// compile in parallel.
#include "mmff_kernels.cuh"

namespace mmffb {

// The instance a plan selects: CTA size, register-cached H columns, matrix in
// shared memory or in a global slot, dense BFGS or L-BFGS.
template <class Fn>
static int with_instance(const Plan &pl, bool lb, const Fn &fn) {
    using R = double;
    using A = double;
    if (lb) return pl.msm ? fn.template run<R, A, 256, 2, true, true>()
                          : fn.template run<R, A, 256, 2, false, true>();
    if (!pl.msm) return fn.template run<R, A, 256, 16, false, false>();
    return fn.template run<R, A, 256, 8, true, false>();
}

int minimize_fp64(const Params &P, const Plan &pl, cudaStream_t st) {
    return with_instance(pl, P.hist_m > 0, LaunchFn{P, pl, st});
}

int occupancy_fp64(const Plan &pl, bool lb) { return with_instance(pl, lb, OccFn{pl}); }

int energy_grad_fp64(const Params &P, float *grad, cudaStream_t st) {
    return launch_eg<double, double, 128>(P, grad, st);
}

int check_fp64(const Params &P, const double *e_in, double *e64, double *derr, double *grms, cudaStream_t st) {
    constexpr int NT = 128;
    Layout L = make_eval_layout(P.nmax, NT / 32, 8, 8, P.b.max_classes);
    auto k = check64_kernel<NT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    k<<<P.c.n_conf, NT, L.total, st>>>(P, e_in, e64, derr, grms);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "check64_kernel launch");
    return 0;
}

}  // namespace mmffb
