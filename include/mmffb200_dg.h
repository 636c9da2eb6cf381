/*
 * mmffb200_dg -- C ABI of the embedding stages: distance geometry (DG) and the
 * experimental-torsion (ETK) refinement.
 *
 * Same conventions as mmffb200.h (whose error codes, mmffb_stream_t and
 * mmffb_last_error() it shares; both are exported by libmmffb200.so): every
 * pointer is a CUDA device pointer owned by the caller, calls are ordered on
 * the given stream and return 0 or a negative MMFFB_E* code.
 *
 * The stage minimises the reference's DG error function (distance-bound
 * violations, chiral-volume violations and a fourth-dimension penalty) per
 * conformer with the reference's L-BFGS and backtracking line search
 * (mlxmolkit/conformer_metal.py:196-547).  It replaces the reference's kernel
 * dispatch in dg_minimize_shared (mlxmolkit/conformer_metal.py:618-736), whose
 * inputs are a SharedConstraintBatch (mlxmolkit/shared_batch.py:23-96).
 *
 * Data layout (written by mlxmolkit_b200/shared_batch.py, DGDeviceBatch):
 *   positions      float32, conformer c's n*dim coordinates (atom-major) at
 *                  pos + conf_atom_starts[c]*dim, dim = 3 or 4
 *   dist_rec       16-byte records {i | j << 16 (int32 bits), lb^2, ub^2, weight},
 *                  molecule m's terms at [dist_starts[m], dist_starts[m+1]),
 *                  local atom indices
 *   dinc_rec       the same terms listed once under each of their two atoms:
 *                  {other atom (int32 bits), lb^2, ub^2, weight}; atom a of
 *                  molecule m owns [dinc_starts[r], dinc_starts[r+1]) with
 *                  r = mol_atom_base[m] + a
 *   chiral_quads   int32[4] per term (local), chiral_bounds float32[2] {lower, upper}
 *   cinc_rec       int32[2] {term index, role 0..3} listed under each of the
 *                  term's four atoms, rows as for dinc_rec
 *   fourth_count   int32 per atom row: how many fourth-dimension terms name it
 *
 * The ETK stage (mlxmolkit/etk_metal.py:27-536, replacing the kernel dispatch of
 * etk_minimize_shared, :567-683) runs the same L-BFGS in 3-D without the first-gradient
 * scaling on MMFFETKTermsDev terms (written by shared_batch.etk_device_arrays):
 *   fb_rec         flat-bottom distance terms {i | j << 16, lb, ub, weight} (bounds in A):
 *                  a molecule's 1-2, 1-3 and 1-4 terms; fbinc_rec lists them per atom as
 *                  {other, lb, ub, weight}
 *   tor_quads      int32[4] and tor_coef float32[12] {V0..V5, s0..s5} per 6-term Fourier
 *                  torsion; a molecule's torsions, then its impropers (V1 = w, s1 = -1);
 *                  tinc_rec lists them per atom as {term, role}
 * The conformer map (conf_*, mol_n_atoms, mol_atom_base, dim = 3) comes from an
 * MMFFDGBatchDev whose DG term pointers are not read.
 */
#ifndef MMFFB200_DG_H
#define MMFFB200_DG_H

#include "mmffb200.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { MMFFB_DG_CONVERGED = 0, MMFFB_DG_MAXIT = 1 };

typedef struct {
    int32_t n_mols, n_conf, dim, max_atoms;
    const int32_t *conf_to_mol;      /* [n_conf] */
    const int32_t *conf_atom_starts; /* [n_conf + 1] */
    const int32_t *conf_order;       /* [n_conf] processing order (largest first), or NULL */
    const int32_t *mol_n_atoms;      /* [n_mols] */
    const int32_t *mol_atom_base;    /* [n_mols] first atom row of each molecule */
    const int32_t *dist_starts;      /* [n_mols + 1] */
    const float *dist_rec;           /* [n_dist][4] */
    const int32_t *dinc_starts;      /* [n_atom_rows + 1] */
    const float *dinc_rec;           /* [2 * n_dist][4] */
    const int32_t *chiral_starts;    /* [n_mols + 1] */
    const int32_t *chiral_quads;     /* [n_chiral][4] */
    const float *chiral_bounds;      /* [n_chiral][2] */
    const int32_t *cinc_starts;      /* [n_atom_rows + 1] */
    const int32_t *cinc_rec;         /* [4 * n_chiral][2] */
    const int32_t *fourth_count;     /* [n_atom_rows] */
} MMFFDGBatchDev;

typedef struct {
    int32_t max_iters;         /* L-BFGS iterations per conformer */
    int32_t lbfgs_m;           /* history length, 1..16 (reference default 8) */
    int32_t threads;           /* threads per conformer: 32, 64, 128 or 256; 0 = chosen from max_atoms */
    float grad_tol;            /* gradient exit (conformer_metal.py:495-503) */
    float chiral_weight;       /* weight of every chiral term */
    float fourth_dim_weight;   /* weight of every fourth-dimension term */
    int32_t hist_mode;         /* L-BFGS history: 0 or 2 = a device slot per CTA, 1 = shared memory */
} MMFFDGParams;

typedef struct {
    int32_t max_tor;                 /* most Fourier terms (torsions + impropers) of one molecule */
    const int32_t *fb_starts;        /* [n_mols + 1] */
    const float *fb_rec;             /* [n_fb][4] */
    const int32_t *fbinc_starts;     /* [n_atom_rows + 1] */
    const float *fbinc_rec;          /* [2 * n_fb][4] */
    const int32_t *tor_starts;       /* [n_mols + 1] */
    const int32_t *tor_quads;        /* [n_tor][4] */
    const float *tor_coef;           /* [n_tor][12] */
    const int32_t *tinc_starts;      /* [n_atom_rows + 1] */
    const int32_t *tinc_rec;         /* [4 * n_tor][2] */
} MMFFETKTermsDev;

/* Device scratch that mmffb_dg_minimize needs (L-BFGS histories of the resident CTAs + a work counter). */
size_t mmffb_dg_scratch_bytes(const MMFFDGBatchDev *batch, const MMFFDGParams *params);

/* Minimise every conformer in place.  energies float32[n_conf], statuses int32[n_conf]
 * (MMFFB_DG_CONVERGED or MMFFB_DG_MAXIT), iters int32[n_conf] or NULL. */
int mmffb_dg_minimize(const MMFFDGBatchDev *batch, const MMFFDGParams *params, float *pos, float *energies,
                      int32_t *statuses, int32_t *iters, void *scratch, size_t scratch_bytes, mmffb_stream_t stream);

/* DG energy and unscaled gradient of every conformer at pos (grad has pos's layout). */
int mmffb_dg_energy_grad(const MMFFDGBatchDev *batch, const MMFFDGParams *params, const float *pos,
                         float *energies, float *grad, mmffb_stream_t stream);

/* Stereo checks after DG (mlxmolkit/stereo_checks_metal.py:30-141): conformer c passes when every
 * tetrahedral quad of its molecule (tet_quads[4*t..], rows tet_starts[m]..tet_starts[m+1]:
 * neighbours n0, n1, n2 and n3 or the centre) has |V| >= vol_tol and every chiral term of the
 * batch's DG terms has V inside [lower, upper]; V = (p0-p3).((p1-p3)x(p2-p3)) on the first
 * three coordinates.  passed int32[n_conf] gets 1 or 0. */
int mmffb_stereo_check(const MMFFDGBatchDev *batch, const int32_t *tet_starts, const int32_t *tet_quads,
                       float vol_tol, const float *pos, int32_t *passed, mmffb_stream_t stream);

/* The ETK stage: scratch, minimisation in place (params: max_iters, lbfgs_m, threads, grad_tol;
 * the weights are not used), and energy + gradient.  confs->dim must be 3. */
size_t mmffb_etk_scratch_bytes(const MMFFDGBatchDev *confs, const MMFFETKTermsDev *terms, const MMFFDGParams *params);
int mmffb_etk_minimize(const MMFFDGBatchDev *confs, const MMFFETKTermsDev *terms, const MMFFDGParams *params,
                       float *pos, float *energies, int32_t *statuses, int32_t *iters, void *scratch,
                       size_t scratch_bytes, mmffb_stream_t stream);
int mmffb_etk_energy_grad(const MMFFDGBatchDev *confs, const MMFFETKTermsDev *terms, const MMFFDGParams *params,
                          const float *pos, float *energies, float *grad, mmffb_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* MMFFB200_DG_H */
