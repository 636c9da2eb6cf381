/*
 * mmffb200 -- C ABI of the B200-native batched MMFF94/94s conformer optimizer.
 *
 * Plain C types only: every pointer below is a CUDA device pointer owned by
 * the caller (a PyTorch tensor, a cudaMalloc arena, ...), every call is
 * ordered on the given stream and returns 0 on success or a negative
 * MMFFB_E* code; mmffb_last_error() gives the message of the calling thread's
 * last failure.
 *
 * Data layout (written by mlxmolkit_b200/pack.py):
 *   mol_desc   int32[n_mols * MMFFB_MOL_DESC_INTS], fields MMFFB_MD_*
 *   bonded     16-byte records in chunks of 32 terms per term type; within
 *              a chunk no two terms share an atom in the same role
 *   atom_cls   int32 per atom: non-bonded class (index into the molecule's
 *              ncls x ncls (R*, eps) table at cls_tab + 2*cls_off)
 *   atom_q     float64 per atom: MMFF partial charge (|q| <= 1e-10 stored as 0)
 *   pair_mask  uint32 bit rows: N rows x ceil(N/32) words of "non-bonded
 *              pair (i<j)" bits, then the same for "1-4 pair" bits
 *   positions  float32, conformer c's 3N coordinates at pos + conf_coord[c]
 */
#ifndef MMFFB200_H
#define MMFFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *mmffb_stream_t; /* = cudaStream_t */

enum {
    MMFFB_OK = 0,
    MMFFB_EINVAL = -1,   /* bad argument (size, pointer, unsupported option) */
    MMFFB_ECUDA = -2,    /* CUDA runtime error (message in mmffb_last_error) */
    MMFFB_ESCRATCH = -3, /* scratch buffer smaller than mmffb_*_scratch_bytes */
    MMFFB_ETOOBIG = -4   /* molecule larger than the kernel supports */
};

/* molecule descriptor fields */
enum {
    MMFFB_MD_N = 0, MMFFB_MD_ATOM_OFF, MMFFB_MD_NCLS, MMFFB_MD_CLS_OFF, MMFFB_MD_MASK_OFF,
    MMFFB_MD_DIEL, MMFFB_MD_B_OFF, MMFFB_MD_B_NCH, MMFFB_MD_A_OFF, MMFFB_MD_A_NCH,
    MMFFB_MD_S_OFF, MMFFB_MD_S_NCH, MMFFB_MD_O_OFF, MMFFB_MD_O_NCH, MMFFB_MD_T_OFF,
    MMFFB_MD_T_NCH, MMFFB_MOL_DESC_INTS
};

/* per-conformer exit status; 0, 2, 3 and 5 are the reference's status 0 ("done") */
enum {
    MMFFB_ST_GRAD = 0,       /* gradient test passed */
    MMFFB_ST_MAXIT = 1,      /* iteration cap reached (the reference's status 1) */
    MMFFB_ST_TOLX = 2,       /* step below TOLX */
    MMFFB_ST_SLOPE = 3,      /* no descent direction (slope >= 0) */
    MMFFB_ST_NONFINITE = 4,  /* energy or gradient not finite */
    MMFFB_ST_LSFAIL = 5,     /* line search found no decrease; position restored */
    MMFFB_ST_TIMEOUT = 6     /* no valid result: a bounded wait on a data copy inside the kernel
                                gave up in this conformer's CTA (positions and energy are those of
                                the iterate reached), or no CTA reached the conformer afterwards
                                (energy NaN, 0 iterations, positions as given); the error word is
                                set (never expected) */
};

/* arithmetic of the optimizer */
enum {
    MMFFB_PREC_MIXED = 0, /* FP32 terms, gradients, BFGS update; FP64 energy sums, Armijo, tests */
    MMFFB_PREC_FP64 = 1,  /* everything FP64 (the GPU oracle) */
    MMFFB_PREC_FP32 = 2   /* everything FP32 */
};

typedef struct {
    int32_t n_mols;
    int32_t max_atoms;           /* largest N in the batch */
    int32_t max_classes;         /* largest per-molecule class count (<= 64) */
    const int32_t *mol_desc;
    const void *bonded;          /* 16-byte aligned records */
    const int32_t *atom_cls;
    const double *atom_q;
    const float *cls_tab;        /* (R*, eps) float pairs */
    const uint32_t *pair_mask;
} MMFFBatchDev;

typedef struct {
    int32_t n_conf;
    int32_t max_atoms;           /* largest N among these conformers */
    const int32_t *conf_mol;     /* molecule of each conformer */
    const int64_t *conf_coord;   /* float offset of each conformer's coordinates */
    const int32_t *order;        /* processing order (largest first) or NULL */
} MMFFConfDev;

typedef struct {
    int32_t max_iters;
    int32_t history_m;           /* 0: dense BFGS; > 0: L-BFGS with that many pairs */
    int32_t precision;           /* MMFFB_PREC_* */
    int32_t threads;             /* CTA size 64, 128, 256 or 512 (512: streamed H only); 0 = auto */
    int32_t ctas_per_sm;         /* persistent CTAs per SM; 0 = as many as fit */
    float grad_tol;
    double consts[8];            /* TOLX FUNCTOL MOVETOL EPS MAXSTEP_FACTOR MAX_LS GRAD_SCALE GRAD_CAP */
    double mode[4];              /* cb (per degree), angle/oop prefactor, stretch-bend gradient prefactor, honour linear */
    int32_t exit_test;           /* MMFFB_EXIT_* */
    int32_t check_every;         /* MMFFB_EXIT_ATOM_NORM: test every k-th iteration (0 = every) */
    float atom_grad_scale;       /* MMFFB_EXIT_ATOM_NORM: factor on the raw gradient */
    int32_t max_restarts;        /* 0: exit on a failed line search or an uphill direction, like the
                                    reference; > 0: reset the inverse Hessian (or L-BFGS history) to the
                                    identity and continue, at most this many times per conformer */
    int32_t polish64;            /* MMFFB_PREC_MIXED: when the FP32 line-search energies stall (no
                                    Armijo decrease or a step below TOLX), continue with FP64 term
                                    energies of the same FP32 coordinates for the line search (the
                                    Python host turns it on for L-BFGS and leaves it off for dense BFGS) */
    int32_t hpass_lean;          /* inverse Hessian in global memory: read its column vectors from
                                    shared memory instead of registers (2 CTAs per SM) */
    uint32_t wait_spins;         /* inverse Hessian in global memory: tests of a row copy's completion
                                    before its wait gives up (0 = 2^22) */
    int32_t give_up_waits;       /* test switch, 0 in normal use: 1 = every wait for a row copy gives up
                                    before testing, as if the copy never completed, which exercises the
                                    timeout path (the kernel drains the copies in flight, its conformers
                                    end MMFFB_ST_TIMEOUT and the error word is set) */
    int32_t *err_word;           /* optional device int32, zeroed by the call; 1 once the launch is done
                                    if a bounded wait gave up (the affected conformers then have status
                                    MMFFB_ST_TIMEOUT).  With or without it, mmffb_minimize's scratch
                                    keeps the same word at byte 4 */
} MMFFOptParams;

/* convergence test of mmffb_minimize */
enum {
    MMFFB_EXIT_TG = 0,        /* max|g_i|*max(|x_i|,1)/max(E*gradScale,1) < grad_tol (tg.metal:300-316) */
    MMFFB_EXIT_ATOM_NORM = 1  /* max over atoms |g_atom|*atom_grad_scale <= grad_tol, every check_every
                                 iterations (mmff_metal_optimizer.py:334-359, 405-416) */
};

int mmffb_version(void);
const char *mmffb_last_error(void);

/*
 * Energy and (if grad != NULL) gradient of every conformer at pos.
 * Replaces the mega kernel mmff_energy_grad_metal_mega
 * (mlxmolkit/mmff_metal_kernel.py:713-744) and the serial/parallel energy
 * macros of the in-kernel optimizer (mlxmolkit/mmff_bfgs_source_tg.metal:54-113).
 * energy: float64[n_conf]; grad: float32 laid out like pos.
 */
int mmffb_energy_grad(const MMFFBatchDev *batch, const MMFFConfDev *confs, int32_t precision,
                      const double *mode, const float *pos, double *energy, float *grad,
                      mmffb_stream_t stream);

/*
 * FP64 check of returned conformers: each conformer's energy and gradient
 * re-evaluated in FP64 at pos (typically right after mmffb_minimize, on the
 * same stream).  e64: float64[n_conf] FP64 energy; err (may be NULL):
 * energy[c] - e64[c], the returned energy's error against the FP64
 * evaluation; grad_rms (may be NULL): root mean square of the 3N components of
 * the FP64 gradient (kcal/mol/A), the stationarity of the returned point.
 * No counterpart in the reference, whose results carry FP32 energies only
 * (mlxmolkit/mmff_metal_optimizer.py:34-44, mmff_minimize.py:346).
 */
int mmffb_fp64_check(const MMFFBatchDev *batch, const MMFFConfDev *confs, const double *mode, const float *pos,
                     const double *energy, double *e64, double *err, double *grad_rms, mmffb_stream_t stream);

/* Bytes of device scratch mmffb_minimize needs for these conformers and options. */
size_t mmffb_minimize_scratch_bytes(const MMFFBatchDev *batch, const MMFFConfDev *confs,
                                    const MMFFOptParams *opt);

/*
 * Minimise every conformer in place (one persistent, work-queued launch):
 * dense BFGS (history_m == 0) or L-BFGS, backtracking line search, TOLX and
 * gradient exits inside the kernel.  Replaces the in-kernel optimizers behind
 * mmff_minimize_nk (mlxmolkit/mmff_minimize.py:231-346;
 * mmff_bfgs_source_tg.metal, mmff_lbfgs_source_tg.metal).
 * energy: float64[n_conf]; status, iters: int32[n_conf]; ls_evals (may be
 * NULL): int32[n_conf] energy-only line-search evaluations per conformer.
 */
int mmffb_minimize(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                   float *pos, double *energy, int32_t *status, int32_t *iters, int32_t *ls_evals,
                   void *scratch, size_t scratch_bytes, mmffb_stream_t stream);

/*
 * The reference's own design restated in CUDA, kept as the measured
 * "plain one-launch-per-batch FP32 GPU path": 32 threads per conformer,
 * serial thread-0 gradient, 32-wide energy, inverse Hessian in global memory,
 * one launch for the batch (mlxmolkit/mmff_bfgs_source_tg.metal:1-372).
 */
size_t mmffb_plain_scratch_bytes(const MMFFBatchDev *batch, const MMFFConfDev *confs);
int mmffb_plain_minimize(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                         float *pos, double *energy, int32_t *status, int32_t *iters,
                         void *scratch, size_t scratch_bytes, mmffb_stream_t stream);

/*
 * Barzilai-Borwein steepest descent with the energy guard and per-atom step
 * cap of the reference's fused optimizer (mlxmolkit/mmff_metal_kernel.py:792-1150),
 * behind mmff_optimize_metal_fused_multi_mol.  opt->max_iters iterations;
 * sd[0] = max_step (A), sd[1] = grad_lr.
 */
int mmffb_fused_sd(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                   const float *sd, float *pos, double *energy, mmffb_stream_t stream);

/*
 * Host-side packing helper (no device work; unlike the calls above, every pointer
 * here is host memory): chunk ids of a term type's terms,
 * the bonded-table layout above.  Greedy first fit in term order, at most 32
 * terms per chunk and no atom twice in one role of a chunk; with flip_perm
 * (the role permutation of the term's equivalent reversed form, or NULL) a term
 * may enter a chunk reversed, flagged in flipped_out (may be NULL).
 * role_atoms: int32[n_terms * roles], atoms < n_atoms.  Returns the number of
 * chunks or a negative MMFFB_E* code.  Replaces the host packing loops of
 * mlxmolkit/mmff_minimize.py:40-173 and mmff_metal_kernel.py:512-687.
 */
int32_t mmffb_pack_chunk(int32_t n_terms, int32_t roles, const int32_t *role_atoms, const int32_t *flip_perm,
                         int32_t n_atoms, int64_t *chunk_out, uint8_t *flipped_out);

/*
 * Host-side packing of whole batches (no device work; every pointer is host
 * memory): the device layout above, built from the molecules' extracted term
 * lists on host threads.  Replaces the reference's per-call host packing
 * (mlxmolkit/mmff_minimize.py:40-173 _pack_mmff_for_nk,
 * mlxmolkit/mmff_metal_kernel.py:594-687 pack_multi_mol_for_metal), with one
 * copy of the tables per molecule instead of one per conformer.
 *
 * Input: the MMFFParams fields of n_mols molecules, each field concatenated
 * over the molecules in molecule order.  term_start[7 * m + t] is the index of
 * molecule m's first term of type t (bond, angle, stretch-bend, out-of-plane,
 * torsion, vdW pair, electrostatic pair) in the arrays of that type;
 * term_start[7 * n_mols + t] is the total.  Atom indices are molecule-local.
 */
typedef struct {
    int32_t n_mols;
    const int32_t *n_atoms;          /* [n_mols] */
    const int32_t *diel;             /* [n_mols] ele_diel_model (2: distance-dependent) */
    const int64_t *term_start;       /* [7 * (n_mols + 1)] */
    const int32_t *bond_i, *bond_j;
    const float *bond_kb, *bond_r0;
    const int32_t *angle_i, *angle_j, *angle_k, *angle_linear;
    const float *angle_ka, *angle_theta0;
    const int32_t *sb_i, *sb_j, *sb_k;
    const float *sb_kba_ijk, *sb_kba_kji, *sb_r0_ij, *sb_r0_kj, *sb_theta0;
    const int32_t *oop_i, *oop_j, *oop_k, *oop_l;
    const float *oop_koop;
    const int32_t *tor_i, *tor_j, *tor_k, *tor_l;
    const float *tor_v1, *tor_v2, *tor_v3;
    const int32_t *vdw_i, *vdw_j;
    const float *vdw_rstar, *vdw_eps;
    const int32_t *ele_i, *ele_j, *ele_is14;
    const float *ele_charge;
    const int64_t *atom_type;        /* [sum n_atoms] MMFF atom type */
    const double *atom_charge;       /* [sum n_atoms] float64 partial charge */
} MMFFTermsHost;

typedef struct {
    int64_t bonded_rows;             /* 16-byte records */
    int64_t atoms;                   /* atom_cls / atom_q entries */
    int64_t cls_pairs;               /* (R*, eps) float pairs */
    int64_t mask_words;
} MMFFPackSizes;

/*
 * Pack in two steps.  mmffb_pack_begin builds every molecule's tables on
 * n_threads host threads (0: all cores), checks them like pack.py does
 * (vdW parameters a function of the atom types, charge terms float32(q_i q_j),
 * ...), fills *sizes and returns a handle, or NULL with the reason in
 * mmffb_last_error().  mmffb_pack_finish writes the batch into the caller's
 * arrays (mol_desc int32[16 * n_mols], bonded uint32[4 * bonded_rows],
 * atom_cls int32[atoms], atom_q float64[atoms], cls_tab float32[2 * cls_pairs],
 * pair_mask uint32[mask_words]) and frees the handle; mmffb_pack_free frees it
 * unused.
 */
void *mmffb_pack_begin(const MMFFTermsHost *terms, int32_t n_threads, MMFFPackSizes *sizes);
int mmffb_pack_finish(void *handle, int32_t *mol_desc, uint32_t *bonded, int32_t *atom_cls, double *atom_q,
                      float *cls_tab, uint32_t *pair_mask);
void mmffb_pack_free(void *handle);

/*
 * The reference's multi-molecule L-BFGS optimizer (mlxmolkit/mmff_metal_optimizer.py:217-535,
 * behind mmff_optimize_metal_multi_mol), run as device-resident chunks: each
 * mmffb_multimol_step launch advances every conformer by n_iters iterations of
 * two-loop L-BFGS on the grad_scale-scaled gradient, a per-atom step cap of
 * max_step_per_atom and no line search; energies use the given term mode (the
 * reference uses its mega-kernel constants).  All state lives in the caller's
 * device buffers below, laid out like the positions where noted.
 */
typedef struct {
    float *x;               /* positions (like pos) */
    float *g;               /* grad_scale * dE/dx at x (like pos) */
    float *best_x;          /* best-seen positions (like pos) */
    double *e;              /* energy at x, per conformer */
    double *best_e;         /* best-seen energy, per conformer */
    float *hist;            /* per conformer mmffb_multimol_hist_floats(): S rows, then Y rows */
    float *rho;             /* per conformer history_m curvature factors */
    int32_t *hcount;        /* pairs pushed so far, per conformer */
    int32_t *converged;     /* main loop: met grad_tol at a check point (sticky) */
    int32_t *conv_iter;     /* iteration of that check point (max_iters if never) */
    int32_t *pending;       /* one counter: conformers that fail the test of the launch's check;
                               the caller zeroes it before a checking launch */
} MMFFMultiMolState;

typedef struct {
    int32_t history_m;      /* L-BFGS pairs, 1..16 (the reference's lbfgs_m) */
    float grad_scale;
    float max_step_per_atom;
    float grad_tol;         /* largest per-atom norm of the scaled gradient */
    double mode[4];         /* term constants, as MMFFOptParams.mode */
    int32_t threads;        /* threads per conformer: 64, 128 or 256; 0 = chosen from the batch */
} MMFFMultiMolParams;

enum {
    MMFFB_MM_START = 0,        /* E, g at x; best = x; history, converged and conv_iter reset */
    MMFFB_MM_REVERT = 1,       /* x = best_x; E, g at x; history reset (the polish pass start) */
    MMFFB_MM_RUN = 2,          /* n_iters iterations, no check */
    MMFFB_MM_MAIN_CHECK = 3,   /* n_iters iterations, then best-seen update and the sticky test
                                  (conv_iter = it_end); pending += conformers not converged */
    MMFFB_MM_POLISH_CHECK = 4  /* n_iters iterations, then best-seen update; pending +=
                                  conformers over grad_tol now */
};

/* Floats of history per conformer (2 * history_m rows of the padded coordinate count). */
size_t mmffb_multimol_hist_floats(const MMFFConfDev *confs, int32_t history_m);
int mmffb_multimol_step(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFMultiMolParams *params,
                        const MMFFMultiMolState *state, int32_t phase, int32_t n_iters, int32_t it_end,
                        int32_t max_iters, mmffb_stream_t stream);

/*
 * Serving worker: one persistent launch of the minimiser that takes conformer
 * slots from a work queue while it runs, so that conformers published while
 * others are being optimised start as soon as a CTA frees up.  No counterpart
 * in the reference, whose multi-molecule loop runs each batch in lockstep
 * (mlxmolkit/mmff_metal_optimizer.py:255-260).
 *
 * The queue's slots are the conformers of confs (n_conf = capacity, order
 * NULL): slot s is conformer s of the arrays there and of pos / energy /
 * status / iters.  The host publishes slots in index order by writing, after
 * the slots' tables, descriptors and coordinates are in device memory, the
 * number of published slots to *tail with a copy ordered on the stream that
 * carried that data (never on the worker's stream).  The launch claims slots
 * from *head, writes each slot's results, then sets done[s] = 1 in host
 * memory.  It ends when *close is set and every published slot is claimed,
 * or after idle_polls polls of an empty queue (sleep_ns apart): every wait is
 * bounded.  Device memory that a running worker has read must not be written
 * again until it ends (the caches of a launch are not refreshed).
 */
typedef struct {
    int32_t *head;           /* device int32: next slot to claim; zero before the queue's first launch */
    const int32_t *tail;     /* device int32: slots published */
    const int32_t *close;    /* device int32: nonzero once no more slots will be published */
    int32_t *done;           /* int32[capacity] of host memory mapped for the device (cudaHostAlloc
                                with cudaHostAllocMapped; its device address) */
    uint32_t idle_polls;     /* empty polls before the launch ends */
    uint32_t sleep_ns;       /* pause between empty polls */
} MMFFQueueDev;

/* Host memory the device can write (for MMFFQueueDev.done): zeroed; *device is its device address. */
int mmffb_host_alloc_mapped(size_t bytes, void **host, void **device);
int mmffb_host_free(void *host);

/* CTAs of the persistent grid mmffb_minimize would launch for these conformers and options
 * (as many as fit on the device, at most one per conformer), or a negative MMFFB_E* code. */
int32_t mmffb_minimize_ctas(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt);

/* Bytes of device scratch mmffb_minimize_queue needs (max_ctas: 0 = as many CTAs as fit). */
size_t mmffb_queue_scratch_bytes(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                                 int32_t max_ctas);
int mmffb_minimize_queue(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                         const MMFFQueueDev *queue, float *pos, double *energy, int32_t *status, int32_t *iters,
                         int32_t max_ctas, void *scratch, size_t scratch_bytes, mmffb_stream_t stream);

/* Size of the fixed per-device scratch array behind mmffb_minimize_noalloc. */
#define MMFFB_NOALLOC_SCRATCH_BYTES ((size_t)64 << 20)

/*
 * mmffb_minimize with no scratch argument and no device allocation.  This
 * entry point has no counterpart in the reference.
 *
 * It is for callers that cannot allocate device memory at call time:
 * - a serving loop whose other streams must keep running, since cudaMalloc
 *   and cudaFree can synchronise the device;
 * - a host whose device memory is reserved up front by another framework's
 *   pool, where a cudaMalloc would fail or take memory the pool expects.
 *
 * Scratch comes from a fixed array inside this library,
 * MMFFB_NOALLOC_SCRATCH_BYTES (64 MiB) per device.  It holds the work
 * counter, the error word and one inverse-Hessian slot per CTA.  A dense BFGS
 * slot is 3N x 3N elements (N = max_atoms): 4 B each for mixed and fp32,
 * 8 B for fp64.  The call itself allocates nothing.
 *
 * - Set-up: every call looks up the array's device address on the current
 *   device (a lookup, no allocation).  The first call on a device also loads
 *   this library's module there, so make that first call before any stream
 *   capture.  Since the lookup is repeated, calls stay valid after a
 *   cudaDeviceReset.
 * - Errors inside the launch: the array's error word is not reachable by the
 *   caller; pass opt->err_word to learn whether a bounded wait gave up.
 * - Limit: if the persistent grid's slots do not all fit in the array, the
 *   grid shrinks to the slots that fit.  Results are unchanged; batches of
 *   large molecules run on fewer CTAs (about 80 for 150 atoms in mixed
 *   precision).  If even one slot plus 256 B does not fit, the call returns
 *   MMFFB_ESCRATCH.
 * - Concurrency: each device has one array.  Calls whose kernels overlap on
 *   the GPU race on it and give wrong results; this happens with calls on
 *   different streams or from several host threads.  Issue such calls on one
 *   stream, or use mmffb_minimize with one scratch buffer per stream.
 *
 * Otherwise the arguments, results and error codes are those of
 * mmffb_minimize.
 */
int mmffb_minimize_noalloc(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                           float *pos, double *energy, int32_t *status, int32_t *iters,
                           int32_t *ls_evals, mmffb_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* MMFFB200_H */
