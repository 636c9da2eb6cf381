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

typedef struct {
    const DGOBatch *b;
    int mol, n, dim;
    double chiral_w, fourth_w;
} Sys;

static double sys_energy(const Sys *s, const double *x) {
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
    for (int i = 0; i < nv; ++i) g[i] *= 0.1;
    for (int sc = 0; sc < 20; ++sc) {
        double mx = 0.0;
        for (int i = 0; i < nv; ++i) mx = dmax(mx, fabs(g[i]));
        if (mx <= 10.0) break;
        for (int i = 0; i < nv; ++i) g[i] *= 0.5;
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
double dg_oracle_energy_grad(const DGOBatch *b, int conf, const double *x, double chiral_w, double fourth_w,
                             double *grad) {
    Sys s = {b, b->conf_to_mol[conf], b->mol_n_atoms[b->conf_to_mol[conf]], b->dim, chiral_w, fourth_w};
    if (grad) sys_grad(&s, x, grad);
    return sys_energy(&s, x);
}

typedef struct {
    const DGOBatch *b;
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
        Sys s = {b, m, n, dim, J->chiral_w, J->fourth_w};
        int it = 0;
        J->statuses[c] = minimize_one(&s, x, J->max_iters, J->grad_tol, J->M, &J->energies[c], &it);
        if (J->iters) J->iters[c] = it;
    }
    return NULL;
}

/* all conformers of the batch on n_threads host threads; pos_out in double */
int dg_oracle_minimize(const DGOBatch *b, const float *pos_in, double *pos_out, double *energies, int32_t *statuses,
                       int32_t *iters, int max_iters, double grad_tol, double chiral_w, double fourth_w, int lbfgs_m,
                       int n_threads) {
    if (!b || !pos_in || !pos_out || !energies || !statuses || lbfgs_m < 1 || (b->dim != 3 && b->dim != 4))
        return -1;
    Job J = {b, pos_in, pos_out, energies, statuses, iters, max_iters, lbfgs_m, grad_tol, chiral_w, fourth_w, 0,
             PTHREAD_MUTEX_INITIALIZER};
    if (n_threads < 1) n_threads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)n_threads);
    for (int t = 0; t < n_threads; ++t) pthread_create(&th[t], NULL, worker, &J);
    for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    free(th);
    return 0;
}
