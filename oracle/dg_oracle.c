/*
 * FP64 CPU oracle for the distance-geometry (DG) minimisation stage.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker of the DG kernel: the
 * parity tests and the CPU-baseline legs of the DG benchmark call it; the
 * product path never does.
 *
 * It restates, in plain C and double precision, the reference's DG L-BFGS
 * (mlxmolkit/conformer_metal.py):
 *
 *   distance-violation energy / gradient    :37-80
 *   chiral-volume energy / gradient         :83-142
 *   fourth-dimension energy / gradient      :145-154
 *   initial energy, gradient, 0.1 scaling
 *     and halving while max|g| > 10          :239-323 (the scaling is applied to
 *                                             the first gradient only, as there)
 *   per-iteration step cap, slope, MOVETOL  :334-357
 *   cubic/quadratic backtracking search     :359-427
 *   TOLX exit, gradient exit                :429-503
 *   L-BFGS history (s.y > 1e-10 gate) and
 *     two-loop with gamma = s.y / y.y       :505-547
 *
 * Batch layout (the reference's SharedConstraintBatch as its kernel takes it,
 * conformer_metal.py:673-714): per conformer c, molecule conf_to_mol[c] and
 * coordinates pos[conf_atom_starts[c]*dim ...]; per molecule m the terms
 * [dist_term_starts[m], dist_term_starts[m+1]) of dist_pairs (t*2: i, j, local)
 * and dist_bounds (t*3: lb^2, ub^2, weight); chiral_quads (t*4) and
 * chiral_bounds (t*2: lower, upper); fourth_idx (local atom indices).
 * Statuses: 0 converged (TOLX or gradient), 1 iteration cap reached.
 *
 * The ETK stage (mlxmolkit/etk_metal.py) runs the same L-BFGS (:353-536) without the
 * first-gradient scaling, in 3-D, on
 *   torsion preferences    E = sum_k V_k (1 + s_k cos((k+1) phi)), k = 0..5  (:51-61)
 *   impropers              the same form with V = (0, w, 0...), s = (0, -1, 0...)  (:105-124)
 *   1-2 / 1-3 / 1-4 terms  flat-bottom w (d - bound)^2 outside [lb, ub], d = sqrt(d^2 + 1e-12)  (:126-150)
 * with cos(phi) from the normals of (p1-p2, p3-p2) and (p2-p3, p4-p3), 0 when their
 * product is degenerate (:35-49).  The torsion gradient here is derived independently:
 * dE/dcos through the two cross products.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define DG_TOLX 1.2e-6
#define DG_FUNCTOL 1e-4
#define DG_MOVETOL 1e-6
#define DG_MAX_STEP_FACTOR 100.0
#define DG_MAX_LS_ITERS 1000

typedef struct {
    int n_mols, n_conf, dim;
    const int32_t *conf_to_mol, *conf_atom_starts, *mol_n_atoms;
    const int32_t *dist_term_starts, *dist_pairs;
    const float *dist_bounds;
    const int32_t *chiral_term_starts, *chiral_quads;
    const float *chiral_bounds;
    const int32_t *fourth_term_starts, *fourth_idx;
} DGOBatch;

/* ETK terms in the reference kernel's layout (etk_metal.py:609-650): torsions (quads, V[6],
 * signs[6]), impropers (quads, weight), and three flat-bottom lists (pairs, {lb, ub, w}). */
typedef struct {
    const int32_t *tor_starts, *tor_quads;
    const float *tor_V, *tor_signs;
    const int32_t *imp_starts, *imp_quads;
    const float *imp_w;
    const int32_t *fb_starts[3], *fb_pairs[3];
    const float *fb_bounds[3];
} ETKOTerms;

typedef struct {
    const DGOBatch *b;
    int mol, n, dim;
    double chiral_w, fourth_w;
    const ETKOTerms *etk; /* NULL: the DG error function */
} Sys;

/* cos(phi) of the reference's torsion convention; ok = 0 where the energy treats it as 0 */
static double tors_cos(const double *x, int dim, const int *q, double t0[3], double t1[3], double r[4][3]) {
    for (int d = 0; d < 3; ++d) {
        r[0][d] = x[q[0] * dim + d] - x[q[1] * dim + d];
        r[1][d] = x[q[2] * dim + d] - x[q[1] * dim + d];
        r[2][d] = -r[1][d];
        r[3][d] = x[q[3] * dim + d] - x[q[2] * dim + d];
    }
    t0[0] = r[0][1] * r[1][2] - r[0][2] * r[1][1];
    t0[1] = r[0][2] * r[1][0] - r[0][0] * r[1][2];
    t0[2] = r[0][0] * r[1][1] - r[0][1] * r[1][0];
    t1[0] = r[2][1] * r[3][2] - r[2][2] * r[3][1];
    t1[1] = r[2][2] * r[3][0] - r[2][0] * r[3][2];
    t1[2] = r[2][0] * r[3][1] - r[2][1] * r[3][0];
    const double comb = (t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2]) * (t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    if (comb < 1e-16) return 0.0;
    double c = (t0[0] * t1[0] + t0[1] * t1[1] + t0[2] * t1[2]) / sqrt(comb);
    return c < -1.0 ? -1.0 : c > 1.0 ? 1.0 : c;
}

/* sum_k V_k (1 + s_k T_{k+1}(c)) and its derivative in c (Chebyshev T_n(cos phi) = cos(n phi)) */
static double fourier(double c, const double *V, const double *s, double *dedc) {
    double T[8], dT[8];
    T[0] = 1.0; T[1] = c; dT[0] = 0.0; dT[1] = 1.0;
    for (int n = 2; n <= 6; ++n) {
        T[n] = 2.0 * c * T[n - 1] - T[n - 2];
        dT[n] = 2.0 * T[n - 1] + 2.0 * c * dT[n - 1] - dT[n - 2];
    }
    double e = 0.0, de = 0.0;
    for (int k = 0; k < 6; ++k) {
        e += V[k] * (1.0 + s[k] * T[k + 1]);
        de += V[k] * s[k] * dT[k + 1];
    }
    if (dedc) *dedc = de;
    return e;
}

static void cross3(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

/* gradient of one Fourier torsion term added into g (the reference's degenerate cases kept) */
static void tors_grad(const double *x, int dim, const int *q, const double *V, const double *s, double *g) {
    double t0[3], t1[3], r[4][3];
    tors_cos(x, dim, q, t0, t1, r);
    const double d0 = t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2], d1 = t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2];
    if (d0 < 1e-16 || d1 < 1e-16) return;
    const double i0 = 1.0 / sqrt(d0), i1 = 1.0 / sqrt(d1);
    double n0[3], n1[3];
    for (int d = 0; d < 3; ++d) { n0[d] = t0[d] * i0; n1[d] = t1[d] * i1; }
    double c = n0[0] * n1[0] + n0[1] * n1[1] + n0[2] * n1[2];
    c = c < -1.0 ? -1.0 : c > 1.0 ? 1.0 : c;
    const double sp = sqrt(fmax(1.0 - c * c, 0.0));
    double dedc;
    fourier(c, V, s, &dedc);
    const double dedphi = -sp * dedc;
    const double st = fabs(sp) > 1e-8 ? -dedphi / sp : -dedphi / fmax(fabs(c), 1e-16) * (c + 1e-30 >= 0 ? 1.0 : -1.0);
    double dc0[3], dc1[3]; /* d cos / d t0, d cos / d t1 */
    for (int d = 0; d < 3; ++d) {
        dc0[d] = i0 * (n1[d] - c * n0[d]);
        dc1[d] = i1 * (n0[d] - c * n1[d]);
    }
    /* t0 = r1 x r2, t1 = r3 x r4: df/da = b x df/dt, df/db = df/dt x a */
    double a1[3], a2[3], a3[3], a4[3];
    cross3(r[1], dc0, a1); /* d/d r1 */
    cross3(dc0, r[0], a2); /* d/d r2 */
    cross3(r[3], dc1, a3); /* d/d r3 */
    cross3(dc1, r[2], a4); /* d/d r4 */
    for (int d = 0; d < 3; ++d) {
        g[q[0] * dim + d] += st * a1[d];                      /* r1 = p1 - p2 */
        g[q[1] * dim + d] += st * (-a1[d] - a2[d] + a3[d]);   /* r1, r2 = p3 - p2, r3 = p2 - p3 */
        g[q[2] * dim + d] += st * (a2[d] - a3[d] - a4[d]);    /* r2, r3, r4 = p4 - p3 */
        g[q[3] * dim + d] += st * a4[d];
    }
}

static const double kImpS[6] = {0, -1, 0, 0, 0, 0};

static double etk_energy(const Sys *s, const double *x) {
    const ETKOTerms *T = s->etk;
    const int m = s->mol, dim = s->dim;
    double e = 0.0, t0[3], t1[3], r[4][3], V[6], sg[6];
    for (int t = T->tor_starts[m]; t < T->tor_starts[m + 1]; ++t) {
        for (int k = 0; k < 6; ++k) { V[k] = T->tor_V[6 * t + k]; sg[k] = T->tor_signs[6 * t + k]; }
        e += fourier(tors_cos(x, dim, T->tor_quads + 4 * t, t0, t1, r), V, sg, NULL);
    }
    for (int t = T->imp_starts[m]; t < T->imp_starts[m + 1]; ++t) {
        const double Vi[6] = {0, T->imp_w[t], 0, 0, 0, 0};
        e += fourier(tors_cos(x, dim, T->imp_quads + 4 * t, t0, t1, r), Vi, kImpS, NULL);
    }
    for (int l = 0; l < 3; ++l)
        for (int t = T->fb_starts[l][m]; t < T->fb_starts[l][m + 1]; ++t) {
            const int a = T->fb_pairs[l][2 * t], b = T->fb_pairs[l][2 * t + 1];
            const double lb = T->fb_bounds[l][3 * t], ub = T->fb_bounds[l][3 * t + 1], w = T->fb_bounds[l][3 * t + 2];
            double d2 = 0.0;
            for (int d = 0; d < 3; ++d) { const double df = x[a * dim + d] - x[b * dim + d]; d2 += df * df; }
            const double dist = sqrt(d2 + 1e-12);
            if (dist < lb) e += w * (dist - lb) * (dist - lb);
            else if (dist > ub) e += w * (dist - ub) * (dist - ub);
        }
    return e;
}

static void etk_grad(const Sys *s, const double *x, double *g) {
    const ETKOTerms *T = s->etk;
    const int m = s->mol, dim = s->dim;
    memset(g, 0, sizeof(double) * (size_t)s->n * dim);
    double V[6], sg[6];
    for (int t = T->tor_starts[m]; t < T->tor_starts[m + 1]; ++t) {
        for (int k = 0; k < 6; ++k) { V[k] = T->tor_V[6 * t + k]; sg[k] = T->tor_signs[6 * t + k]; }
        tors_grad(x, dim, T->tor_quads + 4 * t, V, sg, g);
    }
    for (int t = T->imp_starts[m]; t < T->imp_starts[m + 1]; ++t) {
        const double Vi[6] = {0, T->imp_w[t], 0, 0, 0, 0};
        tors_grad(x, dim, T->imp_quads + 4 * t, Vi, kImpS, g);
    }
    for (int l = 0; l < 3; ++l)
        for (int t = T->fb_starts[l][m]; t < T->fb_starts[l][m + 1]; ++t) {
            const int a = T->fb_pairs[l][2 * t], b = T->fb_pairs[l][2 * t + 1];
            const double lb = T->fb_bounds[l][3 * t], ub = T->fb_bounds[l][3 * t + 1], w = T->fb_bounds[l][3 * t + 2];
            double df[3], d2 = 0.0;
            for (int d = 0; d < 3; ++d) { df[d] = x[a * dim + d] - x[b * dim + d]; d2 += df[d] * df[d]; }
            const double dist = sqrt(d2 + 1e-12);
            double pf = 0.0;
            if (dist < lb) pf = w * 2.0 * (dist - lb) / dist;
            else if (dist > ub) pf = w * 2.0 * (dist - ub) / dist;
            if (pf != 0.0)
                for (int d = 0; d < 3; ++d) { g[a * dim + d] += pf * df[d]; g[b * dim + d] -= pf * df[d]; }
        }
}

static double sys_energy(const Sys *s, const double *x) {
    if (s->etk) return etk_energy(s, x);
    const DGOBatch *b = s->b;
    const int dim = s->dim, m = s->mol;
    double e = 0.0;
    for (int t = b->dist_term_starts[m]; t < b->dist_term_starts[m + 1]; ++t) {
        const int i = b->dist_pairs[2 * t], j = b->dist_pairs[2 * t + 1];
        const double lb2 = b->dist_bounds[3 * t], ub2 = b->dist_bounds[3 * t + 1], w = b->dist_bounds[3 * t + 2];
        double d2 = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double df = x[i * dim + d] - x[j * dim + d];
            d2 += df * df;
        }
        if (d2 > ub2) {
            const double v = d2 / ub2 - 1.0;
            e += w * v * v;
        } else if (d2 < lb2) {
            const double v = 2.0 * lb2 / (lb2 + d2) - 1.0;
            e += w * v * v;
        }
    }
    for (int t = b->chiral_term_starts[m]; t < b->chiral_term_starts[m + 1]; ++t) {
        const int *q = b->chiral_quads + 4 * t;
        double v1[3], v2[3], v3[3];
        for (int d = 0; d < 3; ++d) {
            v1[d] = x[q[0] * dim + d] - x[q[3] * dim + d];
            v2[d] = x[q[1] * dim + d] - x[q[3] * dim + d];
            v3[d] = x[q[2] * dim + d] - x[q[3] * dim + d];
        }
        const double vol = v1[0] * (v2[1] * v3[2] - v2[2] * v3[1]) + v1[1] * (v2[2] * v3[0] - v2[0] * v3[2]) +
                           v1[2] * (v2[0] * v3[1] - v2[1] * v3[0]);
        const double lo = b->chiral_bounds[2 * t], hi = b->chiral_bounds[2 * t + 1];
        if (vol < lo) e += s->chiral_w * (vol - lo) * (vol - lo);
        else if (vol > hi) e += s->chiral_w * (vol - hi) * (vol - hi);
    }
    if (dim == 4)
        for (int t = b->fourth_term_starts[m]; t < b->fourth_term_starts[m + 1]; ++t) {
            const double w4 = x[b->fourth_idx[t] * 4 + 3];
            e += s->fourth_w * w4 * w4;
        }
    return e;
}

static void sys_grad(const Sys *s, const double *x, double *g) {
    if (s->etk) { etk_grad(s, x, g); return; }
    const DGOBatch *b = s->b;
    const int dim = s->dim, m = s->mol;
    memset(g, 0, sizeof(double) * (size_t)s->n * dim);
    for (int t = b->dist_term_starts[m]; t < b->dist_term_starts[m + 1]; ++t) {
        const int i = b->dist_pairs[2 * t], j = b->dist_pairs[2 * t + 1];
        const double lb2 = b->dist_bounds[3 * t], ub2 = b->dist_bounds[3 * t + 1], w = b->dist_bounds[3 * t + 2];
        double df[4], d2 = 0.0;
        for (int d = 0; d < dim; ++d) {
            df[d] = x[i * dim + d] - x[j * dim + d];
            d2 += df[d] * df[d];
        }
        double pf = 0.0;
        if (d2 > ub2) {
            pf = w * 4.0 * (d2 / ub2 - 1.0) / ub2;
        } else if (d2 < lb2) {
            const double l = d2 + lb2;
            pf = w * 8.0 * lb2 * (1.0 - 2.0 * lb2 / l) / (l * l);
        }
        if (pf != 0.0)
            for (int d = 0; d < dim; ++d) {
                g[i * dim + d] += pf * df[d];
                g[j * dim + d] -= pf * df[d];
            }
    }
    for (int t = b->chiral_term_starts[m]; t < b->chiral_term_starts[m + 1]; ++t) {
        const int *q = b->chiral_quads + 4 * t;
        double v1[3], v2[3], v3[3];
        for (int d = 0; d < 3; ++d) {
            v1[d] = x[q[0] * dim + d] - x[q[3] * dim + d];
            v2[d] = x[q[1] * dim + d] - x[q[3] * dim + d];
            v3[d] = x[q[2] * dim + d] - x[q[3] * dim + d];
        }
        const double c23[3] = {v2[1] * v3[2] - v2[2] * v3[1], v2[2] * v3[0] - v2[0] * v3[2], v2[0] * v3[1] - v2[1] * v3[0]};
        const double vol = v1[0] * c23[0] + v1[1] * c23[1] + v1[2] * c23[2];
        const double lo = b->chiral_bounds[2 * t], hi = b->chiral_bounds[2 * t + 1];
        double pf = 0.0;
        if (vol < lo) pf = 2.0 * s->chiral_w * (vol - lo);
        else if (vol > hi) pf = 2.0 * s->chiral_w * (vol - hi);
        if (pf == 0.0) continue;
        /* d vol / d p1 = v2 x v3, d vol / d p2 = v3 x v1, d vol / d p3 = v1 x v2, p4 takes minus the sum */
        const double c31[3] = {v3[1] * v1[2] - v3[2] * v1[1], v3[2] * v1[0] - v3[0] * v1[2], v3[0] * v1[1] - v3[1] * v1[0]};
        const double c12[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
        for (int d = 0; d < 3; ++d) {
            g[q[0] * dim + d] += pf * c23[d];
            g[q[1] * dim + d] += pf * c31[d];
            g[q[2] * dim + d] += pf * c12[d];
            g[q[3] * dim + d] -= pf * (c23[d] + c31[d] + c12[d]);
        }
    }
    if (dim == 4)
        for (int t = b->fourth_term_starts[m]; t < b->fourth_term_starts[m + 1]; ++t) {
            const int a = b->fourth_idx[t];
            g[a * 4 + 3] += 2.0 * s->fourth_w * x[a * 4 + 3];
        }
}

static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }

/* one conformer, start to exit; returns the status and writes energy / iterations */
static int minimize_one(const Sys *s, double *x, int max_iters, double grad_tol, int M, double *energy_out,
                        int *iters_out) {
    const int nv = s->n * s->dim;
    double *g = calloc((size_t)nv, sizeof(double)), *dir = calloc((size_t)nv, sizeof(double));
    double *xo = calloc((size_t)nv, sizeof(double)), *go = calloc((size_t)nv, sizeof(double));
    double *q = calloc((size_t)nv, sizeof(double));
    double *S = calloc((size_t)M * nv + 1, sizeof(double)), *Y = calloc((size_t)M * nv + 1, sizeof(double));
    double *rho = calloc((size_t)M + 1, sizeof(double)), *alpha = calloc((size_t)M + 1, sizeof(double));

    double energy = sys_energy(s, x);
    sys_grad(s, x, g);
    if (!s->etk) { /* the DG stage scales its first gradient; ETK does not (etk_metal.py:353) */
        for (int i = 0; i < nv; ++i) g[i] *= 0.1;
        for (int sc = 0; sc < 20; ++sc) {
            double mx = 0.0;
            for (int i = 0; i < nv; ++i) mx = dmax(mx, fabs(g[i]));
            if (mx <= 10.0) break;
            for (int i = 0; i < nv; ++i) g[i] *= 0.5;
        }
    }
    for (int i = 0; i < nv; ++i) dir[i] = -g[i];
    double ss = 0.0;
    for (int i = 0; i < nv; ++i) ss += x[i] * x[i];
    const double max_step = DG_MAX_STEP_FACTOR * dmax(sqrt(ss), (double)nv);

    int status = 1, hist_count = 0, hist_idx = 0, it = 0;
    for (it = 0; it < max_iters && status == 1; ++it) {
        memcpy(xo, x, sizeof(double) * (size_t)nv);
        const double old_e = energy;
        double dn = 0.0;
        for (int i = 0; i < nv; ++i) dn += dir[i] * dir[i];
        dn = sqrt(dn);
        if (dn > max_step)
            for (int i = 0; i < nv; ++i) dir[i] *= max_step / dn;
        double slope = 0.0, test = 0.0;
        for (int i = 0; i < nv; ++i) {
            slope += dir[i] * g[i];
            test = dmax(test, fabs(dir[i]) / dmax(fabs(x[i]), 1.0));
        }
        const double lam_min = DG_MOVETOL / dmax(test, 1e-30);
        double lam = 1.0, prev_lam = 1.0, prev_e = old_e;
        int done = 0;
        for (int ls = 0; ls < DG_MAX_LS_ITERS && !done; ++ls) {
            if (lam < lam_min) {
                memcpy(x, xo, sizeof(double) * (size_t)nv);
                done = 1;
                break;
            }
            for (int i = 0; i < nv; ++i) x[i] = xo[i] + lam * dir[i];
            const double te = sys_energy(s, x);
            if (te - old_e <= DG_FUNCTOL * lam * slope) {
                energy = te;
                done = 1;
            } else {
                double tl;
                if (ls == 0) {
                    tl = -slope / (2.0 * (te - old_e - slope));
                } else {
                    const double r1 = te - old_e - lam * slope, r2 = prev_e - old_e - prev_lam * slope;
                    const double l2 = lam * lam, p2 = prev_lam * prev_lam, dnm = lam - prev_lam;
                    if (fabs(dnm) < 1e-30) {
                        tl = 0.5 * lam;
                    } else {
                        const double a = (r1 / l2 - r2 / p2) / dnm, bq = (-prev_lam * r1 / l2 + lam * r2 / p2) / dnm;
                        if (fabs(a) < 1e-30) {
                            tl = fabs(bq) > 1e-30 ? -slope / (2.0 * bq) : 0.5 * lam;
                        } else {
                            const double disc = bq * bq - 3.0 * a * slope;
                            if (disc < 0.0) tl = 0.5 * lam;
                            else if (bq <= 0.0) tl = (-bq + sqrt(disc)) / (3.0 * a);
                            else tl = -slope / (bq + sqrt(disc));
                        }
                    }
                }
                /* clamp(tl, 0.1 lam, 0.5 lam); a NaN candidate becomes the lower end, as min/max do */
                tl = dmin(fmax(tl, 0.1 * lam), 0.5 * lam);
                prev_lam = lam;
                prev_e = te;
                lam = tl;
            }
        }
        if (!done) memcpy(x, xo, sizeof(double) * (size_t)nv);
        double tolx = 0.0;
        for (int i = 0; i < nv; ++i) {
            xo[i] = x[i] - xo[i]; /* s */
            tolx = dmax(tolx, fabs(xo[i]) / dmax(fabs(x[i]), 1.0));
        }
        if (tolx < DG_TOLX) {
            status = 0;
            break;
        }
        memcpy(go, g, sizeof(double) * (size_t)nv);
        energy = sys_energy(s, x);
        sys_grad(s, x, g);
        double gt = 0.0;
        for (int i = 0; i < nv; ++i) gt = dmax(gt, fabs(g[i]) * dmax(fabs(x[i]), 1.0));
        if (gt / dmax(energy, 1.0) < grad_tol) {
            status = 0;
            break;
        }
        double ys = 0.0;
        for (int i = 0; i < nv; ++i) {
            q[i] = g[i] - go[i]; /* y */
            ys += q[i] * xo[i];
        }
        if (ys > 1e-10) {
            const int slot = hist_idx % M;
            memcpy(S + (size_t)slot * nv, xo, sizeof(double) * (size_t)nv);
            memcpy(Y + (size_t)slot * nv, q, sizeof(double) * (size_t)nv);
            rho[slot] = 1.0 / ys;
            ++hist_idx;
            if (hist_count < M) ++hist_count;
        }
        memcpy(q, g, sizeof(double) * (size_t)nv);
        for (int j = hist_count - 1; j >= 0; --j) {
            int slot = (hist_idx - 1 - (hist_count - 1 - j)) % M;
            if (slot < 0) slot += M;
            double dt = 0.0;
            for (int i = 0; i < nv; ++i) dt += S[(size_t)slot * nv + i] * q[i];
            alpha[j] = rho[slot] * dt;
            for (int i = 0; i < nv; ++i) q[i] -= alpha[j] * Y[(size_t)slot * nv + i];
        }
        if (hist_count > 0) {
            int nw = (hist_idx - 1) % M;
            if (nw < 0) nw += M;
            double sy = 0.0, yy = 0.0;
            for (int i = 0; i < nv; ++i) {
                sy += S[(size_t)nw * nv + i] * Y[(size_t)nw * nv + i];
                yy += Y[(size_t)nw * nv + i] * Y[(size_t)nw * nv + i];
            }
            const double gm = sy / dmax(yy, 1e-30);
            for (int i = 0; i < nv; ++i) q[i] *= gm;
        }
        for (int j = 0; j < hist_count; ++j) {
            int slot = (hist_idx - 1 - (hist_count - 1 - j)) % M;
            if (slot < 0) slot += M;
            double dt = 0.0;
            for (int i = 0; i < nv; ++i) dt += Y[(size_t)slot * nv + i] * q[i];
            const double beta = rho[slot] * dt;
            for (int i = 0; i < nv; ++i) q[i] += (alpha[j] - beta) * S[(size_t)slot * nv + i];
        }
        for (int i = 0; i < nv; ++i) dir[i] = -q[i];
    }
    *energy_out = energy;
    *iters_out = it < max_iters ? it + 1 : max_iters;
    free(g); free(dir); free(xo); free(go); free(q); free(S); free(Y); free(rho); free(alpha);
    return status;
}

/* energy and gradient of one conformer at x (double, the conformer's n*dim coordinates) */
double dg_oracle_energy_grad(const DGOBatch *b, const ETKOTerms *etk, int conf, const double *x, double chiral_w,
                             double fourth_w, double *grad) {
    Sys s = {b, b->conf_to_mol[conf], b->mol_n_atoms[b->conf_to_mol[conf]], b->dim, chiral_w, fourth_w, etk};
    if (grad) sys_grad(&s, x, grad);
    return sys_energy(&s, x);
}

typedef struct {
    const DGOBatch *b;
    const ETKOTerms *etk;
    const float *pos_in;
    double *pos_out, *energies;
    int32_t *statuses, *iters;
    int max_iters, M;
    double grad_tol, chiral_w, fourth_w;
    int next;
    pthread_mutex_t mu;
} Job;

static void *worker(void *arg) {
    Job *J = (Job *)arg;
    for (;;) {
        pthread_mutex_lock(&J->mu);
        const int c = J->next++;
        pthread_mutex_unlock(&J->mu);
        if (c >= J->b->n_conf) break;
        const DGOBatch *b = J->b;
        const int m = b->conf_to_mol[c], n = b->mol_n_atoms[m], dim = b->dim;
        const size_t off = (size_t)b->conf_atom_starts[c] * dim;
        double *x = J->pos_out + off;
        for (int i = 0; i < n * dim; ++i) x[i] = J->pos_in[off + i];
        Sys s = {b, m, n, dim, J->chiral_w, J->fourth_w, J->etk};
        int it = 0;
        J->statuses[c] = minimize_one(&s, x, J->max_iters, J->grad_tol, J->M, &J->energies[c], &it);
        if (J->iters) J->iters[c] = it;
    }
    return NULL;
}

/* all conformers of the batch on n_threads host threads; pos_out in double */
/* etk = NULL: the DG stage; otherwise the ETK stage (dim must be 3) */
int dg_oracle_minimize(const DGOBatch *b, const ETKOTerms *etk, const float *pos_in, double *pos_out, double *energies,
                       int32_t *statuses, int32_t *iters, int max_iters, double grad_tol, double chiral_w,
                       double fourth_w, int lbfgs_m, int n_threads) {
    if (!b || !pos_in || !pos_out || !energies || !statuses || lbfgs_m < 1 || (b->dim != 3 && b->dim != 4) ||
        (etk && b->dim != 3))
        return -1;
    Job J = {b, etk, pos_in, pos_out, energies, statuses, iters, max_iters, lbfgs_m, grad_tol, chiral_w, fourth_w, 0,
             PTHREAD_MUTEX_INITIALIZER};
    if (n_threads < 1) n_threads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)n_threads);
    for (int t = 0; t < n_threads; ++t) pthread_create(&th[t], NULL, worker, &J);
    for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    free(th);
    return 0;
}
