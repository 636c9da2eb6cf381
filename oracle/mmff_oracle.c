/*
 * FP64 CPU oracle for the batched MMFF94 conformer optimizer.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it; the product
 * path never does.
 *
 * It restates, in plain C and double precision, the reference's algorithm for
 * the hot path:
 *
 *   term energies / gradients  mlxmolkit/mmff_bfgs_header.metal:15-402
 *   gradient scaling           mlxmolkit/mmff_bfgs_header.metal:435-454
 *   dense BFGS driver          mlxmolkit/mmff_bfgs_source_tg.metal:115-372
 *   L-BFGS (m history) driver  mlxmolkit/mmff_lbfgs_source_tg.metal:111-298
 *
 * A four-number "mode" covers the divergences inside the reference: the angle
 * cubic constant cb (-0.4*pi/180 in the TG header, -0.007 in the mega kernel
 * and the numpy energies, mlxmolkit/mmff_energy_vectorized.py:100), the
 * angle/out-of-plane prefactor (143.9325*(pi/180)^2 in the header, the rounded
 * 0.043844 in mmff_metal_kernel.py:279 and the numpy energies), the
 * stretch-bend gradient prefactor (143.9325*pi/180 in header :154, 2.51210 in
 * numpy) and whether angle_is_linear is honoured (the TG header does, the mega
 * kernel and numpy ignore it, mlxmolkit/mmff_metal_kernel.py:350-368).
 *
 * Molecule layout ("blob"): int32 counts[8] = {n_atoms, nb, na, nsb, noop,
 * ntor, nvdw, nele}; int32 idx blob = bond i[],j[] | angle i[],j[],k[],lin[] |
 * sb i[],j[],k[] | oop i[],j[],k[],l[] | tor i[],j[],k[],l[] | vdw i[],j[] |
 * ele i[],j[],is14[]; float32 param blob = bond kb[],r0[] | angle ka[],t0[] |
 * sb kij[],kkj[],r0ij[],r0kj[],t0[] | oop koop[] | tor V1[],V2[],V3[] |
 * vdw R*[],eps[] | ele qq[].  Angles in degrees, atom indices local.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

#define DEG2RAD (3.14159265358979323846 / 180.0)
#define RAD2DEG (180.0 / 3.14159265358979323846)
#define MDYNE 143.9325
#define ELEC 332.0716

typedef struct {
    int n, nb, na, nsb, noop, ntor, nvdw, nele;
    const int32_t *bi, *bj;
    const int32_t *ai, *aj, *ak, *alin;
    const int32_t *si, *sj, *sk;
    const int32_t *oi, *oj, *ok, *ol;
    const int32_t *ti, *tj, *tk, *tl;
    const int32_t *vi, *vj;
    const int32_t *ei, *ej, *e14;
    const float *bkb, *br0;
    const float *aka, *at0;
    const float *skij, *skkj, *sr0ij, *sr0kj, *st0;
    const float *okoop;
    const float *tv1, *tv2, *tv3;
    const float *vr, *ve;
    const float *eq;
    int diel;           /* 2 = distance-dependent, anything else = constant */
    double cb;          /* angle cubic bend constant (per degree) */
    double kang;        /* angle / out-of-plane energy prefactor (143.9325*(pi/180)^2 or 0.043844) */
    double ksbg;        /* stretch-bend gradient prefactor (143.9325*pi/180 or 2.51210) */
    int use_linear;     /* honour angle_is_linear */
} Mol;

static void mol_view(Mol *m, const int32_t *counts, const int32_t *idx, const float *par,
                     int diel, const double *mode) {
    m->n = counts[0]; m->nb = counts[1]; m->na = counts[2]; m->nsb = counts[3];
    m->noop = counts[4]; m->ntor = counts[5]; m->nvdw = counts[6]; m->nele = counts[7];
    const int32_t *p = idx;
    m->bi = p; p += m->nb; m->bj = p; p += m->nb;
    m->ai = p; p += m->na; m->aj = p; p += m->na; m->ak = p; p += m->na; m->alin = p; p += m->na;
    m->si = p; p += m->nsb; m->sj = p; p += m->nsb; m->sk = p; p += m->nsb;
    m->oi = p; p += m->noop; m->oj = p; p += m->noop; m->ok = p; p += m->noop; m->ol = p; p += m->noop;
    m->ti = p; p += m->ntor; m->tj = p; p += m->ntor; m->tk = p; p += m->ntor; m->tl = p; p += m->ntor;
    m->vi = p; p += m->nvdw; m->vj = p; p += m->nvdw;
    m->ei = p; p += m->nele; m->ej = p; p += m->nele; m->e14 = p; p += m->nele;
    const float *q = par;
    m->bkb = q; q += m->nb; m->br0 = q; q += m->nb;
    m->aka = q; q += m->na; m->at0 = q; q += m->na;
    m->skij = q; q += m->nsb; m->skkj = q; q += m->nsb; m->sr0ij = q; q += m->nsb;
    m->sr0kj = q; q += m->nsb; m->st0 = q; q += m->nsb;
    m->okoop = q; q += m->noop;
    m->tv1 = q; q += m->ntor; m->tv2 = q; q += m->ntor; m->tv3 = q; q += m->ntor;
    m->vr = q; q += m->nvdw; m->ve = q; q += m->nvdw;
    m->eq = q; q += m->nele;
    m->diel = diel; m->cb = mode[0]; m->kang = mode[1]; m->ksbg = mode[2];
    m->use_linear = mode[3] != 0.0;
}

static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }
static inline double clampd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

/* ---- bond stretch: header :15-46 ---- */
static double bond_term(const double *x, double *g, int i, int j, double kb, double r0) {
    double dx = x[3*i] - x[3*j], dy = x[3*i+1] - x[3*j+1], dz = x[3*i+2] - x[3*j+2];
    double d2 = dx*dx + dy*dy + dz*dz;
    double d = sqrt(dmax(d2, 1e-16));
    double dr = d - r0;
    double e = 0.5 * MDYNE * kb * dr * dr * (1.0 - 2.0 * dr + (7.0 / 3.0) * dr * dr);
    if (g) {
        double inv = d > 1e-8 ? 1.0 / d : 0.0;
        double f = MDYNE * kb * dr * (1.0 - 3.0 * dr + (14.0 / 3.0) * dr * dr) * inv;
        g[3*i] += f*dx; g[3*i+1] += f*dy; g[3*i+2] += f*dz;
        g[3*j] -= f*dx; g[3*j+1] -= f*dy; g[3*j+2] -= f*dz;
    }
    return e;
}

/* bond vectors from the centre, inverse lengths and the clamped cosine: header :58-74 */
typedef struct { double r1[3], r2[3], id1, id2, c; } Ang;

static inline void ang_setup(const double *x, int i, int j, int k, Ang *a) {
    for (int d = 0; d < 3; ++d) { a->r1[d] = x[3*i+d] - x[3*j+d]; a->r2[d] = x[3*k+d] - x[3*j+d]; }
    double s1 = a->r1[0]*a->r1[0] + a->r1[1]*a->r1[1] + a->r1[2]*a->r1[2];
    double s2 = a->r2[0]*a->r2[0] + a->r2[1]*a->r2[1] + a->r2[2]*a->r2[2];
    a->id1 = 1.0 / sqrt(dmax(s1, 1e-16));
    a->id2 = 1.0 / sqrt(dmax(s2, 1e-16));
    double dot = a->r1[0]*a->r2[0] + a->r1[1]*a->r2[1] + a->r1[2]*a->r2[2];
    a->c = clampd(dot * a->id1 * a->id2, -1.0, 1.0);
}

/* ---- angle bend: header :76-125 ---- */
static double angle_term(const Mol *m, const double *x, double *g, int i, int j, int k,
                         double ka, double t0, int lin) {
    Ang a; ang_setup(x, i, j, k, &a);
    double theta = RAD2DEG * acos(a.c);
    int linear = lin && m->use_linear;
    double dt = theta - t0;
    double e = linear ? MDYNE * ka * (1.0 + a.c)
                      : 0.5 * m->kang * ka * dt * dt * (1.0 + m->cb * dt);
    if (g) {
        double s2 = 1.0 - a.c * a.c;
        if (s2 >= 1e-16) {
            double de = linear ? -MDYNE * ka * sqrt(dmax(s2, 0.0))
                               : m->kang * RAD2DEG * ka * dt * (1.0 + 1.5 * m->cb * dt);
            double cf = -de / sqrt(dmax(s2, 1e-16));
            for (int d = 0; d < 3; ++d) {
                double u1 = a.r1[d] * a.id1, u2 = a.r2[d] * a.id2;
                double g1 = cf * a.id1 * (u2 - a.c * u1);
                double g3 = cf * a.id2 * (u1 - a.c * u2);
                g[3*i+d] += g1; g[3*k+d] += g3; g[3*j+d] -= g1 + g3;
            }
        }
    }
    return e;
}

/* ---- stretch-bend: header :127-167 ---- */
static double strbend_term(const Mol *m, const double *x, double *g, int i, int j, int k, double r0ij,
                           double r0kj, double t0, double kij, double kkj) {
    Ang a; ang_setup(x, i, j, k, &a);
    double d1 = 1.0 / dmax(a.id1, 1e-8), d2 = 1.0 / dmax(a.id2, 1e-8);
    double dt = RAD2DEG * acos(a.c) - t0;
    double dr1 = d1 - r0ij, dr2 = d2 - r0kj;
    double e = 2.51210 * dt * (dr1 * kij + dr2 * kkj);
    if (g) {
        double s2 = 1.0 - a.c * a.c;
        if (s2 >= 1e-16) {
            double is = dmin(1.0 / sqrt(dmax(s2, 1e-16)), 1e8);
            double pf = m->ksbg;
            double beis = RAD2DEG * (kij * dr1 + kkj * dr2) * is;
            for (int d = 0; d < 3; ++d) {
                double u1 = a.r1[d] * a.id1, u2 = a.r2[d] * a.id2;
                double in1 = a.id1 * (u2 - a.c * u1), in3 = a.id2 * (u1 - a.c * u2);
                double g1 = pf * (dt * u1 * kij - in1 * beis);
                double g3 = pf * (dt * u2 * kkj - in3 * beis);
                g[3*i+d] += g1; g[3*k+d] += g3;
                g[3*j+d] += pf * (-dt * (u1 * kij + u2 * kkj) + (in1 + in3) * beis);
            }
        }
    }
    return e;
}

static inline void cross3(const double *a, const double *b, double *c) {
    c[0] = a[1]*b[2] - a[2]*b[1]; c[1] = a[2]*b[0] - a[0]*b[2]; c[2] = a[0]*b[1] - a[1]*b[0];
}

/* ---- Wilson out-of-plane: header :169-249 (i, centre j, k, l out of the i-j-k plane) ---- */
static double oop_term(const Mol *m, const double *x, double *g, int i, int j, int k, int l, double koop) {
    double rI[3], rK[3], rL[3], uI[3], uK[3], uL[3];
    for (int d = 0; d < 3; ++d) { rI[d] = x[3*i+d] - x[3*j+d]; rK[d] = x[3*k+d] - x[3*j+d]; rL[d] = x[3*l+d] - x[3*j+d]; }
    double iI = 1.0 / sqrt(dmax(rI[0]*rI[0]+rI[1]*rI[1]+rI[2]*rI[2], 1e-16));
    double iK = 1.0 / sqrt(dmax(rK[0]*rK[0]+rK[1]*rK[1]+rK[2]*rK[2], 1e-16));
    double iL = 1.0 / sqrt(dmax(rL[0]*rL[0]+rL[1]*rL[1]+rL[2]*rL[2], 1e-16));
    for (int d = 0; d < 3; ++d) { uI[d] = rI[d]*iI; uK[d] = rK[d]*iK; uL[d] = rL[d]*iL; }
    double mI[3] = {-uI[0], -uI[1], -uI[2]}, nrm[3];
    cross3(mI, uK, nrm);
    double inl = 1.0 / sqrt(dmax(nrm[0]*nrm[0]+nrm[1]*nrm[1]+nrm[2]*nrm[2], 1e-16));
    for (int d = 0; d < 3; ++d) nrm[d] *= inl;
    double s = clampd(uL[0]*nrm[0] + uL[1]*nrm[1] + uL[2]*nrm[2], -1.0, 1.0);
    double chi = RAD2DEG * asin(s);
    double e = 0.5 * m->kang * koop * chi * chi;
    if (g) {
        double c2 = 1.0 - s * s;
        double ic = c2 > 0 ? 1.0 / sqrt(dmax(c2, 1e-16)) : 1e8;
        double ct = clampd(uI[0]*uK[0] + uI[1]*uK[1] + uI[2]*uK[2], -1.0, 1.0);
        double ist = 1.0 / sqrt(dmax(1.0 - ct * ct, 1e-8));
        double dE = m->kang * RAD2DEG * koop * chi;
        double t1v = ic * ist, t2v = s * ic * ist * ist;
        double a1[3], a2[3], a3[3];
        cross3(uL, uK, a1); cross3(uI, uL, a2); cross3(uK, uI, a3);
        for (int d = 0; d < 3; ++d) {
            double g1 = dE * (a1[d] * t1v - (uI[d] - uK[d] * ct) * t2v) * iI;
            double g3 = dE * (a2[d] * t1v - (uK[d] - uI[d] * ct) * t2v) * iK;
            double g4 = dE * (a3[d] * t1v - uL[d] * s * ic) * iL;
            g[3*i+d] += g1; g[3*k+d] += g3; g[3*l+d] += g4; g[3*j+d] -= g1 + g3 + g4;
        }
    }
    return e;
}

/* ---- torsion: header :251-326 ---- */
static double torsion_term(const double *x, double *g, int i1, int i2, int i3, int i4,
                           double V1, double V2, double V3) {
    double a[3], b[3], c[3], mb[3], c1[3], c2[3];
    for (int d = 0; d < 3; ++d) { a[d] = x[3*i1+d] - x[3*i2+d]; b[d] = x[3*i3+d] - x[3*i2+d]; c[d] = x[3*i4+d] - x[3*i3+d]; mb[d] = -b[d]; }
    cross3(a, b, c1);
    cross3(mb, c, c2);
    double n1 = c1[0]*c1[0]+c1[1]*c1[1]+c1[2]*c1[2];
    double n2 = c2[0]*c2[0]+c2[1]*c2[1]+c2[2]*c2[2];
    double e = 0.0;
    if (n1 * n2 >= 1e-16) {
        double cp = clampd((c1[0]*c2[0]+c1[1]*c2[1]+c1[2]*c2[2]) / sqrt(n1 * n2), -1.0, 1.0);
        double cos2 = 2.0*cp*cp - 1.0, cos3 = cp*(4.0*cp*cp - 3.0);
        e = 0.5 * (V1*(1.0+cp) + V2*(1.0-cos2) + V3*(1.0+cos3));
    }
    if (g && n1 >= 1e-30 && n2 >= 1e-30) {
        double in1 = dmin(1.0 / sqrt(n1), 1e5), in2 = dmin(1.0 / sqrt(n2), 1e5);
        double u1[3], u2[3];
        for (int d = 0; d < 3; ++d) { u1[d] = c1[d]*in1; u2[d] = c2[d]*in2; }
        double cp = clampd(u1[0]*u2[0]+u1[1]*u2[1]+u1[2]*u2[2], -1.0, 1.0);
        double sp2 = 1.0 - cp*cp, st = 0.0;
        if (sp2 > 0.0) st = 0.5 * (V1 - 2.0*V2*(2.0*cp) + 3.0*V3*(3.0 - 4.0*sp2));
        double d0[3], d1[3];
        for (int d = 0; d < 3; ++d) { d0[d] = in1 * (u2[d] - cp*u1[d]); d1[d] = in2 * (u1[d] - cp*u2[d]); }
        g[3*i1+0] += st*(d0[2]*b[1] - d0[1]*b[2]);
        g[3*i1+1] += st*(d0[0]*b[2] - d0[2]*b[0]);
        g[3*i1+2] += st*(d0[1]*b[0] - d0[0]*b[1]);
        g[3*i4+0] += st*(d1[1]*(-b[2]) - d1[2]*(-b[1]));
        g[3*i4+1] += st*(d1[2]*(-b[0]) - d1[0]*(-b[2]));
        g[3*i4+2] += st*(d1[0]*(-b[1]) - d1[1]*(-b[0]));
        g[3*i2+0] += st*(d0[1]*(b[2]-a[2]) + d0[2]*(a[1]-b[1]) + d1[1]*(-c[2]) + d1[2]*c[1]);
        g[3*i2+1] += st*(d0[0]*(a[2]-b[2]) + d0[2]*(b[0]-a[0]) + d1[0]*c[2] + d1[2]*(-c[0]));
        g[3*i2+2] += st*(d0[0]*(b[1]-a[1]) + d0[1]*(a[0]-b[0]) + d1[0]*(-c[1]) + d1[1]*c[0]);
        g[3*i3+0] += st*(d0[1]*a[2] + d0[2]*(-a[1]) + d1[1]*(c[2]+b[2]) + d1[2]*(-c[1]-b[1]));
        g[3*i3+1] += st*(d0[0]*(-a[2]) + d0[2]*a[0] + d1[0]*(-c[2]-b[2]) + d1[2]*(c[0]+b[0]));
        g[3*i3+2] += st*(d0[0]*a[1] + d0[1]*(-a[0]) + d1[0]*(c[1]+b[1]) + d1[1]*(-c[0]-b[0]));
    }
    return e;
}

/* ---- buffered 14-7 van der Waals: header :328-365 ---- */
static double vdw_term(const double *x, double *g, int i, int j, double R, double eps) {
    double dx = x[3*i] - x[3*j], dy = x[3*i+1] - x[3*j+1], dz = x[3*i+2] - x[3*j+2];
    double d = sqrt(dmax(dx*dx + dy*dy + dz*dz, 1e-16));
    double iR = 1.0 / dmax(R, 1e-8);
    double q = d * iR;
    double q2 = q*q, q6 = q2*q2*q2, q7 = q6*q;
    double t = 1.07 / (q + 0.07);
    double t2 = t*t, t7 = t2*t2*t2*t;
    double e = eps * t7 * (1.12 / (q7 + 0.12) - 2.0);
    if (g) {
        double inv = d > 1e-8 ? 1.0 / d : 0.0;
        double iq = 1.0 / dmax(q7 + 0.12, 1e-30);
        double dE = eps * iR * t7 * (-7.84 * q6 * iq * iq + (-7.84 * iq + 14.0) / (q + 0.07));
        double f = dE * inv;
        g[3*i] += f*dx; g[3*i+1] += f*dy; g[3*i+2] += f*dz;
        g[3*j] -= f*dx; g[3*j+1] -= f*dy; g[3*j+2] -= f*dz;
    }
    return e;
}

/* ---- electrostatics: header :367-402 ---- */
static double ele_term(const Mol *m, const double *x, double *g, int i, int j, double qq, int is14) {
    double dx = x[3*i] - x[3*j], dy = x[3*i+1] - x[3*j+1], dz = x[3*i+2] - x[3*j+2];
    double d = sqrt(dmax(dx*dx + dy*dy + dz*dz, 1e-16));
    double dpd = d + 0.05;
    double sc = is14 ? 0.75 : 1.0;
    int dd = m->diel == 2;
    double e = ELEC * qq * sc / (dd ? dpd * dpd : dpd);
    if (g) {
        double inv = d > 1e-8 ? 1.0 / d : 0.0;
        double den = dd ? dpd*dpd*dpd : dpd*dpd;
        double f = -ELEC * (dd ? 2.0 : 1.0) * qq * sc / dmax(den, 1e-30) * inv;
        g[3*i] += f*dx; g[3*i+1] += f*dy; g[3*i+2] += f*dz;
        g[3*j] -= f*dx; g[3*j+1] -= f*dy; g[3*j+2] -= f*dz;
    }
    return e;
}

/* Total energy (and gradient when g != NULL; g is overwritten). */
static double eval(const Mol *m, const double *x, double *g, double *terms) {
    double e[7] = {0, 0, 0, 0, 0, 0, 0};
    if (g) memset(g, 0, sizeof(double) * 3 * (size_t)m->n);
    for (int t = 0; t < m->nb; ++t) e[0] += bond_term(x, g, m->bi[t], m->bj[t], m->bkb[t], m->br0[t]);
    for (int t = 0; t < m->na; ++t)
        e[1] += angle_term(m, x, g, m->ai[t], m->aj[t], m->ak[t], m->aka[t], m->at0[t], m->alin[t]);
    for (int t = 0; t < m->nsb; ++t)
        e[2] += strbend_term(m, x, g, m->si[t], m->sj[t], m->sk[t], m->sr0ij[t], m->sr0kj[t],
                             m->st0[t], m->skij[t], m->skkj[t]);
    for (int t = 0; t < m->noop; ++t)
        e[3] += oop_term(m, x, g, m->oi[t], m->oj[t], m->ok[t], m->ol[t], m->okoop[t]);
    for (int t = 0; t < m->ntor; ++t)
        e[4] += torsion_term(x, g, m->ti[t], m->tj[t], m->tk[t], m->tl[t], m->tv1[t], m->tv2[t], m->tv3[t]);
    for (int t = 0; t < m->nvdw; ++t) e[5] += vdw_term(x, g, m->vi[t], m->vj[t], m->vr[t], m->ve[t]);
    for (int t = 0; t < m->nele; ++t) e[6] += ele_term(m, x, g, m->ei[t], m->ej[t], m->eq[t], m->e14[t]);
    if (terms) for (int q = 0; q < 7; ++q) terms[q] = e[q];
    return e[0] + e[1] + e[2] + e[3] + e[4] + e[5] + e[6];
}

/* ---- optimizer constants (index order shared with the Python wrapper) ---- */
enum { K_TOLX, K_FUNCTOL, K_MOVETOL, K_EPS, K_MAXSTEP, K_MAXLS, K_GSCALE, K_GCAP, K_RESTARTS };

/* exit codes; 0 and the converged codes map to the reference's status 0 */
enum { ST_GRAD = 0, ST_MAXIT = 1, ST_TOLX = 2, ST_SLOPE = 3, ST_NONFINITE = 4, ST_LSFAIL = 5 };

/* scale_grad_serial (header :435-454): multiply by the sticky scale, halve while max|g| > cap */
static void scale_grad(double *g, int n, double *scale, const double *K) {
    double s = *scale, mx = 0.0;
    for (int i = 0; i < n; ++i) { g[i] *= s; mx = dmax(mx, fabs(g[i])); }
    for (int h = 0; h < 256 && mx > K[K_GCAP]; ++h) {   /* bounded: inf never ends */
        s *= 0.5; mx = 0.0;
        for (int i = 0; i < n; ++i) { g[i] *= 0.5; mx = dmax(mx, fabs(g[i])); }
    }
    *scale = s;
}

static int finite_vec(const double *v, int n) {
    for (int i = 0; i < n; ++i) if (!isfinite(v[i])) return 0;
    return 1;
}

/* Backtracking line search of the TG kernels (tg.metal:192-256).  Returns 1 when
 * the Armijo test accepted a point (x, *E updated), 0 otherwise (x restored). */
static int line_search(const Mol *m, double *x, const double *xold, const double *dir, int n,
                       double Eold, double slope, double lam_min, double *E, const double *K) {
    double lam = 1.0, plam = 1.0, pe = Eold;
    int maxls = (int)K[K_MAXLS];
    for (int ls = 0; ls < maxls; ++ls) {
        if (lam < lam_min) { memcpy(x, xold, sizeof(double) * n); return 0; }
        for (int i = 0; i < n; ++i) x[i] = xold[i] + lam * dir[i];
        double et = eval(m, x, NULL, NULL);
        if (et - Eold <= K[K_FUNCTOL] * lam * slope) { *E = et; return 1; }
        double tl;
        if (ls == 0) {
            tl = -slope / (2.0 * (et - Eold - slope));
        } else {
            double r1 = et - Eold - lam * slope, r2 = pe - Eold - plam * slope;
            double l2 = lam * lam, p2 = plam * plam, dv = lam - plam;
            if (fabs(dv) < 1e-30) tl = 0.5 * lam;
            else {
                double a = (r1 / l2 - r2 / p2) / dv, b = (-plam * r1 / l2 + lam * r2 / p2) / dv;
                if (fabs(a) < 1e-30) tl = fabs(b) > 1e-30 ? -slope / (2.0 * b) : 0.5 * lam;
                else {
                    double disc = b * b - 3.0 * a * slope;
                    if (disc < 0.0) tl = 0.5 * lam;
                    else if (b <= 0.0) tl = (-b + sqrt(disc)) / (3.0 * a);
                    else tl = -slope / (b + sqrt(disc));
                }
            }
        }
        tl = dmin(tl, 0.5 * lam);
        tl = dmax(tl, 0.1 * lam);
        plam = lam; pe = et; lam = tl;
    }
    memcpy(x, xold, sizeof(double) * n);
    return 0;
}

/*
 * One conformer.  history_m == 0: dense BFGS (tg.metal); history_m > 0: L-BFGS
 * with that many (s, y) pairs (lbfgs_tg.metal).  x is updated in place.
 */
static int minimize_one(const Mol *m, double *x, int max_iters, double grad_tol, int history_m,
                        const double *K, double *E_out, int *iters_out, double *work) {
    int n = 3 * m->n;
    double *g = work, *dir = g + n, *xold = dir + n, *dg = xold + n, *hdg = dg + n;
    double *H = hdg + n;                                  /* n*n (BFGS) or 2*m*n + 2*m (L-BFGS) */
    double gscale = K[K_GSCALE];
    double E = eval(m, x, g, NULL);
    scale_grad(g, n, &gscale, K);
    int hm = history_m;
    double *S = H, *Y = H + (size_t)hm * n, *rho = Y + (size_t)hm * n, *alpha = rho + hm;
    if (hm == 0) {
        for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) H[(size_t)i*n + j] = i == j;
    }
    for (int i = 0; i < n; ++i) dir[i] = -g[i];
    double ss = 0.0;
    for (int i = 0; i < n; ++i) ss += x[i] * x[i];
    double max_step = K[K_MAXSTEP] * dmax(sqrt(ss), (double)n);
    int status = ST_MAXIT, it = 0, hcount = 0, hidx = 0, restarts = 0, fresh = 1;
    int max_restarts = (int)K[K_RESTARTS];
    if (!isfinite(E) || !finite_vec(g, n)) { status = ST_NONFINITE; max_iters = 0; }
    for (it = 0; it < max_iters; ++it) {
        memcpy(xold, x, sizeof(double) * n);
        double Eold = E, dn = 0.0;
        for (int i = 0; i < n; ++i) dn += dir[i] * dir[i];
        dn = sqrt(dn);
        if (dn > max_step) { double sc = max_step / dn; for (int i = 0; i < n; ++i) dir[i] *= sc; }
        double slope = 0.0;
        for (int i = 0; i < n; ++i) slope += dir[i] * g[i];
        if (slope >= 0.0) {
            if (!fresh && restarts < max_restarts) {       /* restart from steepest descent */
                ++restarts; fresh = 1; hcount = 0; hidx = 0;
                if (hm == 0) for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) H[(size_t)i*n + j] = i == j;
                for (int i = 0; i < n; ++i) dir[i] = -g[i];
                continue;
            }
            status = ST_SLOPE;
            break;
        }
        double tm = 0.0;
        for (int i = 0; i < n; ++i) tm = dmax(tm, fabs(dir[i]) / dmax(fabs(x[i]), 1.0));
        double lam_min = K[K_MOVETOL] / dmax(tm, 1e-30);
        int ok = line_search(m, x, xold, dir, n, Eold, slope, lam_min, &E, K);
        if (!ok && !fresh && restarts < max_restarts) {    /* x already restored: restart */
            ++restarts; fresh = 1; hcount = 0; hidx = 0;
            if (hm == 0) for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) H[(size_t)i*n + j] = i == j;
            for (int i = 0; i < n; ++i) dir[i] = -g[i];
            continue;
        }
        fresh = 0;
        for (int i = 0; i < n; ++i) xold[i] = x[i] - xold[i];       /* xi */
        double tx = 0.0;
        for (int i = 0; i < n; ++i) tx = dmax(tx, fabs(xold[i]) / dmax(fabs(x[i]), 1.0));
        if (tx < K[K_TOLX]) { status = ok ? ST_TOLX : ST_LSFAIL; break; }
        memcpy(dg, g, sizeof(double) * n);
        eval(m, x, g, NULL);
        scale_grad(g, n, &gscale, K);
        if (!isfinite(E) || !finite_vec(g, n)) { status = ST_NONFINITE; break; }
        for (int i = 0; i < n; ++i) dg[i] = g[i] - dg[i];
        double gt = 0.0;
        for (int i = 0; i < n; ++i) gt = dmax(gt, fabs(g[i]) * dmax(fabs(x[i]), 1.0));
        if (gt / dmax(E * gscale, 1.0) < grad_tol) { status = ST_GRAD; break; }
        if (hm == 0) {
            /* dense BFGS update (tg.metal:318-366) */
            double fac = 0, fae = 0, sdg = 0, sxi = 0;
            for (int i = 0; i < n; ++i) {
                double s = 0.0;
                const double *Hi = H + (size_t)i * n;
                for (int j = 0; j < n; ++j) s += Hi[j] * dg[j];
                hdg[i] = s;
            }
            for (int i = 0; i < n; ++i) {
                fac += dg[i] * xold[i]; fae += dg[i] * hdg[i];
                sdg += dg[i] * dg[i]; sxi += xold[i] * xold[i];
            }
            if (fac * fac > K[K_EPS] * sdg * sxi && fac > 0) {
                double fi = 1.0 / fac, fei = 1.0 / fae;
                for (int i = 0; i < n; ++i) {
                    double ai = fi * xold[i] - fei * hdg[i];
                    double *Hi = H + (size_t)i * n;
                    for (int j = 0; j < n; ++j) {
                        double aj = fi * xold[j] - fei * hdg[j];
                        Hi[j] += fi * xold[i] * xold[j] - fei * hdg[i] * hdg[j] + fae * ai * aj;
                    }
                }
            }
            for (int i = 0; i < n; ++i) {
                double s = 0.0;
                const double *Hi = H + (size_t)i * n;
                for (int j = 0; j < n; ++j) s += Hi[j] * g[j];
                dir[i] = -s;
            }
        } else {
            /* L-BFGS update and two-loop recursion (lbfgs_tg.metal:247-292) */
            double ys = 0.0;
            for (int i = 0; i < n; ++i) ys += dg[i] * xold[i];
            if (ys > 1e-10) {
                int slot = hidx % hm;
                memcpy(S + (size_t)slot * n, xold, sizeof(double) * n);
                memcpy(Y + (size_t)slot * n, dg, sizeof(double) * n);
                rho[slot] = 1.0 / ys;
                hidx++;
                if (hcount < hm) hcount++;
            }
            double *q = hdg;
            memcpy(q, g, sizeof(double) * n);
            for (int jj = hcount - 1; jj >= 0; --jj) {
                int slot = ((hidx - 1 - (hcount - 1 - jj)) % hm + hm) % hm;
                double d = 0.0;
                for (int i = 0; i < n; ++i) d += S[(size_t)slot*n + i] * q[i];
                double aj = rho[slot] * d;
                alpha[jj] = aj;
                for (int i = 0; i < n; ++i) q[i] -= aj * Y[(size_t)slot*n + i];
            }
            if (hcount > 0) {
                int nw = ((hidx - 1) % hm + hm) % hm;
                double sy = 0.0, yy = 0.0;
                for (int i = 0; i < n; ++i) { sy += S[(size_t)nw*n+i] * Y[(size_t)nw*n+i]; yy += Y[(size_t)nw*n+i] * Y[(size_t)nw*n+i]; }
                double gam = sy / dmax(yy, 1e-30);
                for (int i = 0; i < n; ++i) q[i] *= gam;
            }
            for (int jj = 0; jj < hcount; ++jj) {
                int slot = ((hidx - 1 - (hcount - 1 - jj)) % hm + hm) % hm;
                double d = 0.0;
                for (int i = 0; i < n; ++i) d += Y[(size_t)slot*n + i] * q[i];
                double bj = rho[slot] * d;
                for (int i = 0; i < n; ++i) q[i] += (alpha[jj] - bj) * S[(size_t)slot*n + i];
            }
            for (int i = 0; i < n; ++i) dir[i] = -q[i];
        }
    }
    *E_out = E;
    *iters_out = it < max_iters ? it + (status == ST_SLOPE ? 0 : 1) : max_iters;
    return status;
}

static size_t work_doubles(int n_atoms, int history_m) {
    size_t n = 3 * (size_t)n_atoms;
    size_t extra = history_m == 0 ? n * n : 2 * (size_t)history_m * n + 2 * (size_t)history_m;
    return 5 * n + extra;
}

/* ------------------------------------------------------------------------- */
/* Exported C entry points (ctypes)                                           */
/* ------------------------------------------------------------------------- */

/* Energy (+ gradient if grad != NULL) of one conformer; terms[7] optional per-term split. */
/* mode[4] = {cb, kang, ksbg, use_linear}: the term-constant set (TG header or mega/numpy). */
double oracle_energy_grad(const int32_t *counts, const int32_t *idx, const float *par, int diel,
                          const double *mode, const double *x, double *grad, double *terms) {
    Mol m;
    mol_view(&m, counts, idx, par, diel, mode);
    return eval(&m, x, grad, terms);
}

/*
 * Minimise C conformers of M molecules.  Molecule b's blobs start at
 * idx_off[b] / par_off[b] with counts at counts[8*b]; conformer c belongs to
 * conf_mol[c] and its coordinates start at x[3*atom_off[c]].  Returns the
 * number of conformers processed; per-conformer status / energy / iterations.
 */
typedef struct {
    const int32_t *counts; const int64_t *idx_off, *par_off; const int32_t *idx; const float *par;
    const int32_t *diel; int C; const int32_t *conf_mol; const int64_t *atom_off; double *x;
    int max_iters; double grad_tol; int history_m; const double *K; const double *mode;
    int32_t *status; double *energy; int32_t *iters;
    int next;                       /* shared work counter (atomic) */
} BatchJob;

static void *batch_worker(void *arg) {
    BatchJob *J = (BatchJob *)arg;
    double *work = NULL;
    size_t cap = 0;
    for (;;) {
        int c = __atomic_fetch_add(&J->next, 1, __ATOMIC_RELAXED);
        if (c >= J->C) break;
        int b = J->conf_mol[c];
        Mol m;
        mol_view(&m, J->counts + 8 * (size_t)b, J->idx + J->idx_off[b], J->par + J->par_off[b],
                 J->diel[b], J->mode);
        size_t need = work_doubles(m.n, J->history_m);
        if (need > cap) { free(work); work = (double *)malloc(need * sizeof(double)); cap = need; }
        int it = 0;
        J->status[c] = minimize_one(&m, J->x + 3 * J->atom_off[c], J->max_iters, J->grad_tol,
                                    J->history_m, J->K, &J->energy[c], &it, work);
        J->iters[c] = it;
    }
    free(work);
    return NULL;
}

/*
 * Minimise C conformers of M molecules on n_threads host threads (0 = all
 * online cores).  Molecule b's blobs start at idx_off[b] / par_off[b] with
 * counts at counts[8*b]; conformer c belongs to conf_mol[c] and its
 * coordinates start at x[3*atom_off[c]].  Returns the thread count used.
 */
int oracle_minimize_batch(int M, const int32_t *counts, const int64_t *idx_off, const int64_t *par_off,
                          const int32_t *idx, const float *par, const int32_t *diel,
                          int C, const int32_t *conf_mol, const int64_t *atom_off, double *x,
                          int max_iters, double grad_tol, int history_m, const double *K,
                          const double *mode, int n_threads,
                          int32_t *status, double *energy, int32_t *iters) {
    (void)M;
    BatchJob J = {counts, idx_off, par_off, idx, par, diel, C, conf_mol, atom_off, x, max_iters,
                  grad_tol, history_m, K, mode, status, energy, iters, 0};
    if (n_threads <= 0) n_threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > C) n_threads = C > 0 ? C : 1;
    if (n_threads == 1) { batch_worker(&J); return 1; }
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)n_threads);
    for (int t = 0; t < n_threads; ++t) pthread_create(&th[t], NULL, batch_worker, &J);
    for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    free(th);
    return n_threads;
}

int oracle_max_threads(void) {
    return (int)sysconf(_SC_NPROCESSORS_ONLN);
}
