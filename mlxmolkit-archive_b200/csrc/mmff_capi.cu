// C ABI entry points and launch planning (host code).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "mmff_kernels.cuh"

namespace mmffb {

static thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *where) {
    return fail(MMFFB_ECUDA, "%s: %s", where, cudaGetErrorString(e));
}

static int device_props(int *sms, int *smem_optin) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    e = cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
    e = cudaDeviceGetAttribute(smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(smem)");
    return 0;
}

int check_batch(const MMFFBatchDev *b, const MMFFConfDev *c) {
    if (!b || !c) return fail(MMFFB_EINVAL, "null batch or conformer descriptor");
    if (c->n_conf < 0 || b->n_mols < 0) return fail(MMFFB_EINVAL, "negative count");
    if (c->n_conf > 0 && (!b->mol_desc || !b->bonded || !b->atom_cls || !b->atom_q || !b->cls_tab ||
                          !b->pair_mask || !c->conf_mol || !c->conf_coord))
        return fail(MMFFB_EINVAL, "null device pointer in batch");
    if (c->max_atoms <= 0 && c->n_conf > 0) return fail(MMFFB_EINVAL, "max_atoms must be positive");
    if (c->max_atoms > kMaxAtoms) return fail(MMFFB_ETOOBIG, "molecule of %d atoms exceeds %d", c->max_atoms, kMaxAtoms);
    if (b->max_classes < 1 || b->max_classes > 64)
        return fail(MMFFB_EINVAL, "max_classes must be in 1..64 (got %d)", b->max_classes);
    return 0;
}

TermMode to_mode(const double *mode) {
    TermMode md;
    md.cb = mode[0]; md.kang = mode[1]; md.ksbg = mode[2]; md.lin = mode[3] != 0.0;
    return md;
}

KConst to_consts(const double *k) {
    KConst K;
    K.tolx = k[0]; K.functol = k[1]; K.movetol = k[2]; K.eps = k[3]; K.maxstep = k[4];
    K.maxls = (int)k[5]; K.gscale = k[6]; K.gcap = k[7];
    return K;
}

// Pick the kernel instance (CTA size, register-cached H columns, matrix in
// shared or global memory) and the persistent grid for these conformers.
int plan_minimize(const MMFFBatchDev *b, const MMFFConfDev *c, const MMFFOptParams *o, Plan *pl) {
    int sms = 0, optin = 0;
    int r = device_props(&sms, &optin);
    if (r) return r;
    const int nmax = c->max_atoms;
    const int n = 3 * nmax;
    const bool mixed = o->precision == MMFFB_PREC_MIXED;
    if (o->precision < 0 || o->precision > 2) return fail(MMFFB_EINVAL, "unknown precision %d", o->precision);
    const size_t rs = o->precision == MMFFB_PREC_FP64 ? 8 : 4;
    const size_t as = o->precision == MMFFB_PREC_FP32 ? 4 : 8;
    if (o->history_m < 0 || o->history_m > kMaxHist) return fail(MMFFB_EINVAL, "history_m out of range");
    const bool lb = o->history_m > 0;
    int nt = o->threads;
    // default CTA size: 128 threads for 25-48 atoms, 256 otherwise (measured per size class on
    // B200; for up to 24 atoms 256 threads beat 64 by finishing each conformer sooner)
    if (nt == 0) nt = (nmax > 24 && nmax <= 48) ? 128 : 256;
    if (nt != 64 && nt != 128 && nt != 256 && nt != 512)
        return fail(MMFFB_EINVAL, "threads must be 64, 128, 256 or 512");
    if (!mixed || lb) nt = 256;
    if (!lb && n > 512) return fail(MMFFB_ETOOBIG, "dense BFGS supports up to 170 atoms (got %d); use L-BFGS", nmax);
    const int mc = b->max_classes;
    if (nt == 512 && (lb || !mixed)) nt = 256;
    // L-BFGS decides from the atom bound alone (the full 64-entry class table), so that every
    // launch of one atom bound -- whatever its molecules' class counts -- runs the same instance
    Layout Ls = make_layout(nmax, nt / 32, o->history_m, true, rs, as, lb ? 64 : mc);
    bool msm = Ls.total <= (size_t)optin;
    // mixed-precision dense BFGS above 48 atoms: the register-lean streamed instance (H in a
    // global slot, 2 CTAs/SM) beats a shared-memory H that leaves one CTA of 8 warps per SM
    if (mixed && !lb && nmax > 48) msm = false;
    int nc = 2;
    if (!lb) {
        if (msm) {
            if (nt == 512) nt = 256;
            if (nt == 64 && n > 128) nt = 128;
            nc = nt == 64 ? 4 : 8;
            // mixed precision with the CTA size left to the plan: the register-capped 256-thread
            // instance (H columns read from shared memory, 128 registers, 2 CTAs and 16 warps per
            // SM) -- the register-cached columns take 230 registers and leave 8 warps per SM
            if (mixed && o->threads == 0) {
                nt = 256;
                nc = 0;
            }
            if (nc > 0 && n > 32 * nc) msm = false;   // register-cached columns cover 32 * nc
        }
        if (!msm) {
            // streamed H: register-cached columns (1 CTA/SM), or the register-lean form
            // (columns from shared memory) at 2 CTAs/SM (256 threads) or 512 threads
            const bool lean = mixed && (o->hpass_lean || nt == 512);
            if (nt != 512) nt = 256;
            nc = lean ? 0 : 16;
        }
    }
    Layout L = make_layout(nmax, nt / 32, o->history_m, msm, rs, as, mc);
    if (L.total > (size_t)optin)
        return fail(MMFFB_ETOOBIG, "molecule of %d atoms needs %zu B of shared memory", nmax, L.total);
    pl->nt = nt;
    pl->nc = nc;
    pl->msm = msm;
    pl->smem = L.total;
    pl->rsz = rs;
    pl->gslot = mat_elems(nmax, o->history_m);
    auto occupancy = [&]() {
        return o->precision == MMFFB_PREC_FP64 ? occupancy_fp64(*pl, lb)
             : o->precision == MMFFB_PREC_FP32 ? occupancy_fp32(*pl, lb) : occupancy_mixed(*pl, lb);
    };
    int fit = occupancy();
    if (fit < 0) return fit;
    // mixed-precision L-BFGS with the history in shared memory: the register-capped instance
    // (128 registers a thread) where two of its CTAs fit an SM by shared memory -- measured on
    // the 150-170-atom class; where only one fits, the cap only adds spills (170-400 atoms
    // measured 25 % slower).  Decided at the atom bound with a 32-entry class table (the
    // serving classes' bound), so the instance does not depend on the launch's molecules; a
    // launch whose tables are larger still runs, with the CTAs that fit.
    if (mixed && lb && o->threads == 0) {
        // the register-capped instance with the history where it is: in shared memory if two
        // CTAs fit so, else in a global slot if two fit that way (up to about 290 atoms; the
        // slots of a full grid take a few tens of MB, L2-resident), else the uncapped one
        bool capped = false;
        for (int where = msm ? 1 : 0; where >= 0 && !capped; --where) {
            pl->nc = 0;
            pl->msm = where == 1;
            pl->smem = make_layout(nmax, nt / 32, o->history_m, where == 1, rs, as, 32).total;
            const int fit2 = occupancy();
            if (fit2 < 0) return fit2;
            capped = fit2 >= 2;
        }
        if (capped) {
            msm = pl->msm;
            L = make_layout(nmax, nt / 32, o->history_m, msm, rs, as, mc);
            pl->smem = L.total;
            fit = occupancy();
            if (fit < 0) return fit;
        } else {
            pl->nc = nc;
            pl->msm = msm;
            pl->smem = L.total;
        }
    }
    // mixed-precision L-BFGS where no two CTAs fit an SM (289 atoms and up): one CTA of 16 warps
    // with the history in a global slot, where that layout fits (to about 410 atoms; decided
    // with the full class table) -- 2 % faster on the large workload than 8 warps with the
    // history in shared memory
    if (mixed && lb && o->threads == 0 && pl->nc != 0) {
        const Layout L16 = make_layout(nmax, 16, o->history_m, false, rs, as, 64);
        if (L16.total <= (size_t)optin) {
            pl->nt = 512;
            pl->nc = 0;
            pl->msm = false;
            msm = false;
            L = make_layout(nmax, 16, o->history_m, false, rs, as, mc);
            pl->smem = L.total;
            fit = occupancy();
            if (fit < 0) return fit;
        }
    }
    if (o->ctas_per_sm > 0 && o->ctas_per_sm < fit) fit = o->ctas_per_sm;
    int grid = sms * fit;
    if (grid > c->n_conf) grid = c->n_conf > 0 ? c->n_conf : 1;
    pl->grid = grid;
    return 0;
}


int check_opt(const MMFFOptParams *o) {
    if (o->max_iters < 0) return fail(MMFFB_EINVAL, "max_iters must be >= 0");
    if (o->consts[5] < 1) return fail(MMFFB_EINVAL, "MAX_LS must be >= 1");
    if (o->exit_test != MMFFB_EXIT_TG && o->exit_test != MMFFB_EXIT_ATOM_NORM)
        return fail(MMFFB_EINVAL, "unknown exit_test %d", o->exit_test);
    return 0;
}

Params make_params(const MMFFBatchDev *b, const MMFFConfDev *c, const MMFFOptParams *o, const Plan &pl,
                   float *pos, double *energy, int32_t *status, int32_t *iters, int32_t *ls_evals,
                   unsigned char *scratch) {
    Params P;
    memset(&P, 0, sizeof P);
    P.b = *b;
    P.c = *c;
    P.md = to_mode(o->mode);
    P.K = to_consts(o->consts);
    P.max_iters = o->max_iters;
    P.hist_m = o->history_m;
    P.grad_tol = o->grad_tol;
    P.exit_test = o->exit_test;
    P.check_every = o->check_every;
    P.atom_grad_scale = o->atom_grad_scale;
    P.max_restarts = o->max_restarts < 0 ? 0 : o->max_restarts;
    P.polish64 = o->precision == MMFFB_PREC_MIXED && o->polish64 != 0;
    P.wait_spins = o->give_up_waits ? 0u : o->wait_spins ? o->wait_spins : kMaxWaitSpins;
    P.ls_evals = ls_evals;
    P.nmax = c->max_atoms;
    P.pos = pos;
    P.energy = energy;
    P.status = status;
    P.iters = iters;
    P.counter = reinterpret_cast<int *>(scratch);
    P.err = o->err_word ? reinterpret_cast<int *>(o->err_word) : reinterpret_cast<int *>(scratch) + 1;
    P.scratch_err = reinterpret_cast<int *>(scratch) + 1;
    P.gmat = scratch + 256;
    P.gslot = pl.gslot;
    return P;
}

static __global__ void zero_err_kernel(const Params P) {
    *P.err = 0;
    *P.scratch_err = 0;
}

static __global__ void prepare_kernel(const Params P) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        *P.counter = 0;
        *P.err = 0;
        *P.scratch_err = 0;
    }
    for (int i = t; i < P.c.n_conf; i += gridDim.x * blockDim.x) {
        const int conf = P.c.order ? P.c.order[i] : i;
        P.status[conf] = MMFFB_ST_TIMEOUT;
        P.iters[conf] = 0;
        P.energy[conf] = __longlong_as_double(0x7ff8000000000000LL);   // quiet NaN
        if (P.ls_evals) P.ls_evals[conf] = 0;
    }
}

int prepare_minimize(const Params &P, cudaStream_t st) {
    int blocks = (P.c.n_conf + 255) / 256;
    blocks = blocks < 1 ? 1 : (blocks > 148 ? 148 : blocks);
    prepare_kernel<<<blocks, 256, 0, st>>>(P);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "prepare_kernel launch");
    return 0;
}

}  // namespace mmffb

using namespace mmffb;

extern "C" {

int mmffb_version(void) { return 1; }

const char *mmffb_last_error(void) { return g_err.c_str(); }

int mmffb_energy_grad(const MMFFBatchDev *batch, const MMFFConfDev *confs, int32_t precision,
                      const double *mode, const float *pos, double *energy, float *grad,
                      mmffb_stream_t stream) {
    int r = check_batch(batch, confs);
    if (r) return r;
    if (!mode || !pos || !energy) return fail(MMFFB_EINVAL, "null mode, pos or energy");
    if (confs->n_conf == 0) return 0;
    Params P;
    memset(&P, 0, sizeof P);
    P.b = *batch;
    P.c = *confs;
    P.md = to_mode(mode);
    P.nmax = confs->max_atoms;
    P.pos = const_cast<float *>(pos);
    P.energy = energy;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (precision == MMFFB_PREC_FP64) return energy_grad_fp64(P, grad, st);
    if (precision == MMFFB_PREC_FP32) return energy_grad_fp32(P, grad, st);
    if (precision != MMFFB_PREC_MIXED) return fail(MMFFB_EINVAL, "unknown precision %d", precision);
    return energy_grad_mixed(P, grad, st);
}

int mmffb_fp64_check(const MMFFBatchDev *batch, const MMFFConfDev *confs, const double *mode, const float *pos,
                     const double *energy, double *e64, double *err, double *grad_rms, mmffb_stream_t stream) {
    int r = check_batch(batch, confs);
    if (r) return r;
    if (!mode || !pos || !e64) return fail(MMFFB_EINVAL, "null mode, pos or e64");
    if (err && !energy) return fail(MMFFB_EINVAL, "err needs the returned energies");
    if (confs->n_conf == 0) return 0;
    Params P;
    memset(&P, 0, sizeof P);
    P.b = *batch;
    P.c = *confs;
    P.md = to_mode(mode);
    P.nmax = confs->max_atoms;
    P.pos = const_cast<float *>(pos);
    return check_fp64(P, energy, e64, err, grad_rms, reinterpret_cast<cudaStream_t>(stream));
}

size_t mmffb_minimize_scratch_bytes(const MMFFBatchDev *batch, const MMFFConfDev *confs,
                                    const MMFFOptParams *opt) {
    if (check_batch(batch, confs) || !opt) return 0;
    Plan pl;
    if (plan_minimize(batch, confs, opt, &pl)) return 0;
    size_t b = 256;
    if (!pl.msm) b += (size_t)pl.grid * pl.gslot * pl.rsz;
    return b;
}

int mmffb_minimize(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                   float *pos, double *energy, int32_t *status, int32_t *iters, int32_t *ls_evals,
                   void *scratch, size_t scratch_bytes, mmffb_stream_t stream) {
    int r = check_batch(batch, confs);
    if (r) return r;
    if (!opt || !pos || !energy || !status || !iters) return fail(MMFFB_EINVAL, "null argument");
    r = check_opt(opt);
    if (r) return r;
    if (confs->n_conf == 0) return 0;
    Plan pl;
    r = plan_minimize(batch, confs, opt, &pl);
    if (r) return r;
    size_t need = 256 + (pl.msm ? 0 : (size_t)pl.grid * pl.gslot * pl.rsz);
    if (!scratch || scratch_bytes < need)
        return fail(MMFFB_ESCRATCH, "scratch of %zu B given, %zu B needed", scratch_bytes, need);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    Params P = make_params(batch, confs, opt, pl, pos, energy, status, iters, ls_evals,
                           reinterpret_cast<unsigned char *>(scratch));
    r = prepare_minimize(P, st);
    if (r) return r;
    if (opt->precision == MMFFB_PREC_FP64) return minimize_fp64(P, pl, st);
    if (opt->precision == MMFFB_PREC_FP32) return minimize_fp32(P, pl, st);
    return minimize_mixed(P, pl, st);
}

int mmffb_host_alloc_mapped(size_t bytes, void **host, void **device) {
    if (!host || !device || bytes == 0) return fail(MMFFB_EINVAL, "null pointer or zero size");
    cudaError_t e = cudaHostAlloc(host, bytes, cudaHostAllocMapped);
    if (e != cudaSuccess) return cuda_fail(e, "cudaHostAlloc(mapped)");
    std::memset(*host, 0, bytes);
    e = cudaHostGetDevicePointer(device, *host, 0);
    if (e != cudaSuccess) {
        cudaFreeHost(*host);
        *host = nullptr;
        return cuda_fail(e, "cudaHostGetDevicePointer");
    }
    return 0;
}

int mmffb_host_free(void *host) {
    cudaError_t e = cudaFreeHost(host);
    return e == cudaSuccess ? 0 : cuda_fail(e, "cudaFreeHost");
}

int32_t mmffb_minimize_ctas(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt) {
    int r = check_batch(batch, confs);
    if (r) return r;
    if (!opt) return fail(MMFFB_EINVAL, "null options");
    Plan pl;
    r = plan_minimize(batch, confs, opt, &pl);
    return r ? r : pl.grid;
}

size_t mmffb_queue_scratch_bytes(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                                 int32_t max_ctas) {
    if (check_batch(batch, confs) || !opt) return 0;
    Plan pl;
    if (plan_minimize(batch, confs, opt, &pl)) return 0;
    if (max_ctas > 0 && pl.grid > max_ctas) pl.grid = max_ctas;
    return 256 + (pl.msm ? 0 : (size_t)pl.grid * pl.gslot * pl.rsz);
}

int mmffb_minimize_queue(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                         const MMFFQueueDev *queue, float *pos, double *energy, int32_t *status, int32_t *iters,
                         int32_t max_ctas, void *scratch, size_t scratch_bytes, mmffb_stream_t stream) {
    int r = check_batch(batch, confs);
    if (r) return r;
    if (!opt || !queue || !pos || !energy || !status || !iters) return fail(MMFFB_EINVAL, "null argument");
    if (!queue->head || !queue->tail || !queue->close || !queue->done)
        return fail(MMFFB_EINVAL, "null queue pointer");
    if (confs->order) return fail(MMFFB_EINVAL, "queue slots are taken in index order (order must be NULL)");
    r = check_opt(opt);
    if (r) return r;
    if (confs->n_conf == 0) return 0;
    Plan pl;
    r = plan_minimize(batch, confs, opt, &pl);
    if (r) return r;
    if (max_ctas > 0 && pl.grid > max_ctas) pl.grid = max_ctas;
    const size_t need = 256 + (pl.msm ? 0 : (size_t)pl.grid * pl.gslot * pl.rsz);
    if (!scratch || scratch_bytes < need)
        return fail(MMFFB_ESCRATCH, "scratch of %zu B given, %zu B needed", scratch_bytes, need);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    Params P = make_params(batch, confs, opt, pl, pos, energy, status, iters, nullptr,
                           reinterpret_cast<unsigned char *>(scratch));
    P.q_head = queue->head;
    P.q_tail = queue->tail;
    P.q_close = queue->close;
    P.q_done = queue->done;
    P.q_idle_polls = queue->idle_polls;
    P.q_sleep_ns = queue->sleep_ns;
    zero_err_kernel<<<1, 1, 0, st>>>(P);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "zero_err_kernel launch");
    if (opt->precision == MMFFB_PREC_FP64) return minimize_fp64(P, pl, st);
    if (opt->precision == MMFFB_PREC_FP32) return minimize_fp32(P, pl, st);
    return minimize_mixed(P, pl, st);
}

}  // extern "C"
