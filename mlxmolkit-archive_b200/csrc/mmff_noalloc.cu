// mmffb_minimize_noalloc: the persistent minimiser with its scratch taken from
// a fixed device array in this file instead of a buffer the caller allocates.
//
// Callers that cannot allocate device memory at call time use it: a serving
// loop whose other streams must keep running (cudaMalloc and cudaFree can
// synchronise the device), or a host whose device memory is reserved up front
// by another framework's pool.  Nothing here calls an allocator.
#include <cstring>

#include "mmff_kernels.cuh"

namespace mmffb {

// Same layout as mmffb_minimize's scratch: work counter (int at byte 0), error
// word (int at byte 4), then one inverse-Hessian slot per CTA from byte 256.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MMFFB_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr size_t kHead = 256;

// Device address of the array on the calling thread's current device, looked up
// with that device current.  The lookup allocates nothing; the first one on a
// device loads this library's module there (set-up).  It is repeated on every
// call, so the address stays right after the caller resets the device
// (cudaDeviceReset reloads the module, possibly elsewhere).
int scratch_address(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    *out = static_cast<unsigned char *>(p);
    return 0;
}

}  // namespace
}  // namespace mmffb

using namespace mmffb;

extern "C" int mmffb_minimize_noalloc(const MMFFBatchDev *batch, const MMFFConfDev *confs,
                                      const MMFFOptParams *opt, float *pos, double *energy, int32_t *status,
                                      int32_t *iters, int32_t *ls_evals, mmffb_stream_t stream) {
    // Resolve the array first, so that any call (an empty batch included)
    // performs the per-device set-up.
    unsigned char *scratch = nullptr;
    int r = scratch_address(&scratch);
    if (r) return r;
    r = check_batch(batch, confs);
    if (r) return r;
    if (!opt || !pos || !energy || !status || !iters) return fail(MMFFB_EINVAL, "null argument");
    r = check_opt(opt);
    if (r) return r;
    if (confs->n_conf == 0) return 0;
    Plan pl;
    r = plan_minimize(batch, confs, opt, &pl);
    if (r) return r;
    if (!pl.msm) {
        // One slot per CTA of the persistent grid; the CTAs pull conformers
        // from the work counter, so fewer CTAs give the same results.
        const size_t slot = pl.gslot * pl.rsz;
        if (kHead + slot > MMFFB_NOALLOC_SCRATCH_BYTES)
            return fail(MMFFB_ESCRATCH,
                        "one inverse-Hessian slot of %zu B (%d atoms) plus %zu B exceeds the %zu B "
                        "no-alloc scratch; use mmffb_minimize with a caller buffer",
                        slot, confs->max_atoms, kHead, (size_t)MMFFB_NOALLOC_SCRATCH_BYTES);
        const size_t fit = (MMFFB_NOALLOC_SCRATCH_BYTES - kHead) / slot;
        if ((size_t)pl.grid > fit) pl.grid = (int)fit;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    Params P = make_params(batch, confs, opt, pl, pos, energy, status, iters, ls_evals, scratch);
    // the array keeps the previous call's contents: the work counter and the error
    // word start at zero again
    r = prepare_minimize(P, st);
    if (r) return r;
    if (opt->precision == MMFFB_PREC_FP64) return minimize_fp64(P, pl, st);
    if (opt->precision == MMFFB_PREC_FP32) return minimize_fp32(P, pl, st);
    return minimize_mixed(P, pl, st);
}
