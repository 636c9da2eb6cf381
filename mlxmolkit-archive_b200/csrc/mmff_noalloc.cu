// mmffb_minimize_noalloc: the persistent minimiser with its scratch taken from
// a fixed device array in this file instead of a buffer the caller allocates.
//
// Callers that cannot allocate device memory at call time use it: a serving
// loop whose other streams must keep running (cudaMalloc and cudaFree can
// synchronise the device), or a host whose device memory is reserved up front
// by another framework's pool.  Nothing here calls an allocator.
#include <cstring>
#include <mutex>

#include "mmff_kernels.cuh"

namespace mmffb {

// Same layout as mmffb_minimize's scratch: work counter (int at byte 0), error
// word (int at byte 4), then one inverse-Hessian slot per CTA from byte 256.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MMFFB_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr size_t kHead = 256;
constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
unsigned char *g_addr[kMaxDevices];

// Device address of the array on the calling thread's current device.  The
// first call for a device resolves it with that device current; later calls
// read the cache.
int scratch_address(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices)
        return fail(MMFFB_EINVAL, "device %d is beyond the %d devices mmffb_minimize_noalloc tracks", dev,
                    kMaxDevices);
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_addr[dev];
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
    if (opt->max_iters < 0) return fail(MMFFB_EINVAL, "max_iters must be >= 0");
    if (opt->consts[5] < 1) return fail(MMFFB_EINVAL, "MAX_LS must be >= 1");
    if (opt->exit_test != MMFFB_EXIT_TG && opt->exit_test != MMFFB_EXIT_ATOM_NORM)
        return fail(MMFFB_EINVAL, "unknown exit_test %d", opt->exit_test);
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
    // the work counter and the error word start at zero
    cudaError_t e = cudaMemsetAsync(scratch, 0, kHead, st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(no-alloc scratch)");
    Params P;
    memset(&P, 0, sizeof P);
    P.b = *batch;
    P.c = *confs;
    P.md = to_mode(opt->mode);
    P.K = to_consts(opt->consts);
    P.max_iters = opt->max_iters;
    P.hist_m = opt->history_m;
    P.grad_tol = opt->grad_tol;
    P.exit_test = opt->exit_test;
    P.check_every = opt->check_every;
    P.atom_grad_scale = opt->atom_grad_scale;
    P.max_restarts = opt->max_restarts < 0 ? 0 : opt->max_restarts;
    P.polish64 = opt->precision == MMFFB_PREC_MIXED && opt->polish64 != 0;
    P.ls_evals = ls_evals;
    P.nmax = confs->max_atoms;
    P.pos = pos;
    P.energy = energy;
    P.status = status;
    P.iters = iters;
    P.counter = reinterpret_cast<int *>(scratch);
    P.err = reinterpret_cast<int *>(scratch) + 1;
    P.gmat = scratch + kHead;
    P.gslot = pl.gslot;
    if (opt->precision == MMFFB_PREC_FP64) return minimize_fp64(P, pl, st);
    if (opt->precision == MMFFB_PREC_FP32) return minimize_fp32(P, pl, st);
    return minimize_mixed(P, pl, st);
}
