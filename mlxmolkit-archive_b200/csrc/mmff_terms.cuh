// MMFF94 term energies and gradients for one term, in registers.
//
// Semantics follow the reference's in-kernel optimizer header
// (mlxmolkit/mmff_bfgs_header.metal:15-402); the constant set is a runtime
// "mode" so that the same code also reproduces the mega / fused kernels'
// rounded constants (mlxmolkit/mmff_metal_kernel.py:274-280):
//   cb    angle cubic constant per degree        (-0.4*pi/180  |  -0.007)
//   kang  angle / out-of-plane energy prefactor  (143.9325*(pi/180)^2 | 0.043844)
//   ksbg  stretch-bend gradient prefactor        (143.9325*pi/180 | 2.51210)
//   lin   honour the linear-angle flag           (1 | 0)
//
// Every function returns the term energy and, when G is true, writes the
// gradient contribution of each participating atom into f[atom][3].
#pragma once
#include <cuda_runtime.h>

namespace mmffb {

struct TermMode {
    double cb, kang, ksbg;
    int lin;
};

template <class R> struct Num;
// FP32: hardware approximate reciprocal / reciprocal square root (about 2 ulp); the
// FP32 paths are checked against the FP64 oracle to 1e-5 relative, and the line
// search of the mixed path switches to FP64 energies near convergence.
template <> struct Num<float> {
    static __device__ __forceinline__ float sqrt_(float x) { return x * rsqrtf(x); }   // x > 0 here
    static __device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
    static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
    static __device__ __forceinline__ float acos_(float x) { return acosf(x); }
    static __device__ __forceinline__ float asin_(float x) { return asinf(x); }
};
template <> struct Num<double> {
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ double rsqrt_(double x) { return 1.0 / sqrt(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double acos_(double x) { return acos(x); }
    static __device__ __forceinline__ double asin_(double x) { return asin(x); }
};

template <class R> __device__ __forceinline__ R clampR(R x, R lo, R hi) { return x < lo ? lo : (x > hi ? hi : x); }
template <class R> __device__ __forceinline__ R maxR(R a, R b) { return a > b ? a : b; }
template <class R> __device__ __forceinline__ R minR(R a, R b) { return a < b ? a : b; }

#define MMFF_MDYNE 143.9325
#define MMFF_ELEC 332.0716
#define MMFF_RAD2DEG 57.295779513082320876798
#define MMFF_DEG2RAD 0.017453292519943295769237

// ---- bond stretch (header :15-46) ----
template <class R, bool G>
__device__ __forceinline__ R bond_term(const R* a, const R* b, R kb, R r0, R (&f)[2][3]) {
    using N = Num<R>;
    R dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    R d2 = dx * dx + dy * dy + dz * dz;
    R d = N::sqrt_(maxR(d2, R(1e-16)));
    R dr = d - r0;
    R e = R(0.5 * MMFF_MDYNE) * kb * dr * dr * (R(1) - R(2) * dr + R(7.0 / 3.0) * dr * dr);
    if (G) {
        R inv = d > R(1e-8) ? N::rcp(d) : R(0);
        R s = R(MMFF_MDYNE) * kb * dr * (R(1) - R(3) * dr + R(14.0 / 3.0) * dr * dr) * inv;
        f[0][0] = s * dx; f[0][1] = s * dy; f[0][2] = s * dz;
        f[1][0] = -f[0][0]; f[1][1] = -f[0][1]; f[1][2] = -f[0][2];
    }
    return e;
}

// ---- angle bend (header :58-125) ----
template <class R, bool G>
__device__ __forceinline__ R angle_term(const R* pi, const R* pj, const R* pk, R ka, R t0, bool lin,
                                        const TermMode& md, R (&f)[3][3]) {
    using N = Num<R>;
    R r1[3], r2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { r1[d] = pi[d] - pj[d]; r2[d] = pk[d] - pj[d]; }
    R s1 = r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2];
    R s2 = r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2];
    R id1 = N::rsqrt_(maxR(s1, R(1e-16))), id2 = N::rsqrt_(maxR(s2, R(1e-16)));
    R c = clampR((r1[0] * r2[0] + r1[1] * r2[1] + r1[2] * r2[2]) * id1 * id2, R(-1), R(1));
    bool linear = lin && md.lin;
    R dt = R(MMFF_RAD2DEG) * N::acos_(c) - t0;
    R e = linear ? R(MMFF_MDYNE) * ka * (R(1) + c)
                 : R(0.5) * R(md.kang) * ka * dt * dt * (R(1) + R(md.cb) * dt);
    if (G) {
        R sn2 = R(1) - c * c;
        R cf = R(0);
        if (sn2 >= R(1e-16)) {
            R de = linear ? -R(MMFF_MDYNE) * ka * N::sqrt_(maxR(sn2, R(0)))
                          : R(md.kang) * R(MMFF_RAD2DEG) * ka * dt * (R(1) + R(1.5) * R(md.cb) * dt);
            cf = -de * N::rsqrt_(maxR(sn2, R(1e-16)));
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            R u1 = r1[d] * id1, u2 = r2[d] * id2;
            R g1 = cf * id1 * (u2 - c * u1);
            R g3 = cf * id2 * (u1 - c * u2);
            f[0][d] = g1; f[2][d] = g3; f[1][d] = -(g1 + g3);
        }
    }
    return e;
}

// ---- stretch-bend (header :127-167) ----
template <class R, bool G>
__device__ __forceinline__ R strbend_term(const R* pi, const R* pj, const R* pk, R r0ij, R r0kj, R t0,
                                          R kij, R kkj, const TermMode& md, R (&f)[3][3]) {
    using N = Num<R>;
    R r1[3], r2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { r1[d] = pi[d] - pj[d]; r2[d] = pk[d] - pj[d]; }
    R s1 = r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2];
    R s2 = r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2];
    R id1 = N::rsqrt_(maxR(s1, R(1e-16))), id2 = N::rsqrt_(maxR(s2, R(1e-16)));
    R c = clampR((r1[0] * r2[0] + r1[1] * r2[1] + r1[2] * r2[2]) * id1 * id2, R(-1), R(1));
    R d1 = N::rcp(maxR(id1, R(1e-8))), d2 = N::rcp(maxR(id2, R(1e-8)));
    R dt = R(MMFF_RAD2DEG) * N::acos_(c) - t0;
    R dr1 = d1 - r0ij, dr2 = d2 - r0kj;
    R e = R(2.51210) * dt * (dr1 * kij + dr2 * kkj);
    if (G) {
        R sn2 = R(1) - c * c;
        if (sn2 >= R(1e-16)) {
            R is = minR(N::rsqrt_(maxR(sn2, R(1e-16))), R(1e8));
            R pf = R(md.ksbg);
            R beis = R(MMFF_RAD2DEG) * (kij * dr1 + kkj * dr2) * is;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                R u1 = r1[d] * id1, u2 = r2[d] * id2;
                R in1 = id1 * (u2 - c * u1), in3 = id2 * (u1 - c * u2);
                f[0][d] = pf * (dt * u1 * kij - in1 * beis);
                f[2][d] = pf * (dt * u2 * kkj - in3 * beis);
                f[1][d] = pf * (-dt * (u1 * kij + u2 * kkj) + (in1 + in3) * beis);
            }
        } else {
#pragma unroll
            for (int d = 0; d < 3; ++d) { f[0][d] = R(0); f[1][d] = R(0); f[2][d] = R(0); }
        }
    }
    return e;
}

template <class R>
__device__ __forceinline__ void cross3(const R* a, const R* b, R* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// ---- Wilson out-of-plane (header :169-249): centre j, l bent out of the i-j-k plane ----
template <class R, bool G>
__device__ __forceinline__ R oop_term(const R* pi, const R* pj, const R* pk, const R* pl, R koop,
                                      const TermMode& md, R (&f)[4][3]) {
    using N = Num<R>;
    R rI[3], rK[3], rL[3], uI[3], uK[3], uL[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { rI[d] = pi[d] - pj[d]; rK[d] = pk[d] - pj[d]; rL[d] = pl[d] - pj[d]; }
    R iI = N::rsqrt_(maxR(rI[0] * rI[0] + rI[1] * rI[1] + rI[2] * rI[2], R(1e-16)));
    R iK = N::rsqrt_(maxR(rK[0] * rK[0] + rK[1] * rK[1] + rK[2] * rK[2], R(1e-16)));
    R iL = N::rsqrt_(maxR(rL[0] * rL[0] + rL[1] * rL[1] + rL[2] * rL[2], R(1e-16)));
#pragma unroll
    for (int d = 0; d < 3; ++d) { uI[d] = rI[d] * iI; uK[d] = rK[d] * iK; uL[d] = rL[d] * iL; }
    R mI[3] = {-uI[0], -uI[1], -uI[2]}, nv[3];
    cross3(mI, uK, nv);
    R inl = N::rsqrt_(maxR(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2], R(1e-16)));
    R s = clampR((uL[0] * nv[0] + uL[1] * nv[1] + uL[2] * nv[2]) * inl, R(-1), R(1));
    R chi = R(MMFF_RAD2DEG) * N::asin_(s);
    R e = R(0.5) * R(md.kang) * koop * chi * chi;
    if (G) {
        R c2 = R(1) - s * s;
        R ic = c2 > R(0) ? N::rsqrt_(maxR(c2, R(1e-16))) : R(1e8);
        R ct = clampR(uI[0] * uK[0] + uI[1] * uK[1] + uI[2] * uK[2], R(-1), R(1));
        R ist = N::rsqrt_(maxR(R(1) - ct * ct, R(1e-8)));
        R dE = R(md.kang) * R(MMFF_RAD2DEG) * koop * chi;
        R t1 = ic * ist, t2 = s * ic * ist * ist;
        R a1[3], a2[3], a3[3];
        cross3(uL, uK, a1);
        cross3(uI, uL, a2);
        cross3(uK, uI, a3);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            R g1 = dE * (a1[d] * t1 - (uI[d] - uK[d] * ct) * t2) * iI;
            R g3 = dE * (a2[d] * t1 - (uK[d] - uI[d] * ct) * t2) * iK;
            R g4 = dE * (a3[d] * t1 - uL[d] * s * ic) * iL;
            f[0][d] = g1; f[2][d] = g3; f[3][d] = g4; f[1][d] = -(g1 + g3 + g4);
        }
    }
    return e;
}

// ---- torsion (header :251-326) ----
template <class R, bool G>
__device__ __forceinline__ R torsion_term(const R* p1, const R* p2, const R* p3, const R* p4, R V1, R V2,
                                          R V3, R (&f)[4][3]) {
    using N = Num<R>;
    R a[3], b[3], c[3], mb[3], c1[3], c2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { a[d] = p1[d] - p2[d]; b[d] = p3[d] - p2[d]; c[d] = p4[d] - p3[d]; mb[d] = -b[d]; }
    cross3(a, b, c1);
    cross3(mb, c, c2);
    R n1 = c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2];
    R n2 = c2[0] * c2[0] + c2[1] * c2[1] + c2[2] * c2[2];
    R e = R(0);
    R comb = n1 * n2;
    if (comb >= R(1e-16)) {
        R cp = clampR((c1[0] * c2[0] + c1[1] * c2[1] + c1[2] * c2[2]) * N::rsqrt_(comb), R(-1), R(1));
        R cos2 = R(2) * cp * cp - R(1), cos3 = cp * (R(4) * cp * cp - R(3));
        e = R(0.5) * (V1 * (R(1) + cp) + V2 * (R(1) - cos2) + V3 * (R(1) + cos3));
    }
    if (G) {
        if (n1 >= R(1e-30) && n2 >= R(1e-30)) {
            R in1 = minR(N::rsqrt_(n1), R(1e5)), in2 = minR(N::rsqrt_(n2), R(1e5));
            R u1[3], u2[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) { u1[d] = c1[d] * in1; u2[d] = c2[d] * in2; }
            R cp = clampR(u1[0] * u2[0] + u1[1] * u2[1] + u1[2] * u2[2], R(-1), R(1));
            R sp2 = R(1) - cp * cp, st = R(0);
            if (sp2 > R(0)) st = R(0.5) * (V1 - R(2) * V2 * (R(2) * cp) + R(3) * V3 * (R(3) - R(4) * sp2));
            R d0[3], d1[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) { d0[d] = in1 * (u2[d] - cp * u1[d]); d1[d] = in2 * (u1[d] - cp * u2[d]); }
            f[0][0] = st * (d0[2] * b[1] - d0[1] * b[2]);
            f[0][1] = st * (d0[0] * b[2] - d0[2] * b[0]);
            f[0][2] = st * (d0[1] * b[0] - d0[0] * b[1]);
            f[3][0] = st * (d1[1] * (-b[2]) - d1[2] * (-b[1]));
            f[3][1] = st * (d1[2] * (-b[0]) - d1[0] * (-b[2]));
            f[3][2] = st * (d1[0] * (-b[1]) - d1[1] * (-b[0]));
            f[1][0] = st * (d0[1] * (b[2] - a[2]) + d0[2] * (a[1] - b[1]) + d1[1] * (-c[2]) + d1[2] * c[1]);
            f[1][1] = st * (d0[0] * (a[2] - b[2]) + d0[2] * (b[0] - a[0]) + d1[0] * c[2] + d1[2] * (-c[0]));
            f[1][2] = st * (d0[0] * (b[1] - a[1]) + d0[1] * (a[0] - b[0]) + d1[0] * (-c[1]) + d1[1] * c[0]);
            f[2][0] = st * (d0[1] * a[2] + d0[2] * (-a[1]) + d1[1] * (c[2] + b[2]) + d1[2] * (-c[1] - b[1]));
            f[2][1] = st * (d0[0] * (-a[2]) + d0[2] * a[0] + d1[0] * (-c[2] - b[2]) + d1[2] * (c[0] + b[0]));
            f[2][2] = st * (d0[0] * a[1] + d0[1] * (-a[0]) + d1[0] * (c[1] + b[1]) + d1[1] * (-c[0] - b[0]));
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) { f[q][0] = R(0); f[q][1] = R(0); f[q][2] = R(0); }
        }
    }
    return e;
}

// ---- buffered 14-7 vdW + Coulomb of one non-bonded pair (header :328-402) ----
// Returns the vdW and electrostatic energies separately (summed by the caller
// in the same order as the reference's term loops) and the scalar radial
// force factor s such that grad_i = s * (p_i - p_j), grad_j = -grad_i.
// IRIN: Rs already holds 1/R* (staged that way for the FP32 instances)
template <class R, bool G, bool IRIN = false>
__device__ __forceinline__ void pair_term(R dx, R dy, R dz, R Rs, R eps, R qq, bool dd,
                                          R& e_vdw, R& e_ele, R& s) {
    using N = Num<R>;
    R d2 = dx * dx + dy * dy + dz * dz;
    const R x2 = maxR(d2, R(1e-16));
    R d, rd;                                   // distance and (FP32) its reciprocal
    if constexpr (sizeof(R) == 4) {
        rd = N::rsqrt_(x2);                    // one reciprocal square root gives both
        d = x2 * rd;
    } else {
        d = N::sqrt_(x2);
        rd = R(0);
    }
    R iR = IRIN ? Rs : N::rcp(maxR(Rs, R(1e-8)));
    R q = d * iR;
    R q2 = q * q, q6 = q2 * q2 * q2, q7 = q6 * q;
    R ib = N::rcp(q + R(0.07));
    R t = R(1.07) * ib;
    R t2 = t * t, t7 = t2 * t2 * t2 * t;
    R iq = N::rcp(maxR(q7 + R(0.12), R(1e-30)));
    e_vdw = eps * t7 * (R(1.12) * iq - R(2));
    R dpd = d + R(0.05);
    R idp = N::rcp(dpd);
    R cq = R(MMFF_ELEC) * qq;
    e_ele = dd ? cq * idp * idp : cq * idp;
    if (G) {
        R inv;
        if constexpr (sizeof(R) == 4) inv = d > R(1e-8) ? rd : R(0);
        else inv = d > R(1e-8) ? N::rcp(d) : R(0);
        R dv = eps * iR * t7 * (R(-7.84) * q6 * iq * iq + (R(-7.84) * iq + R(14)) * ib);
        R de = dd ? R(-2) * cq * idp * idp * idp : -cq * idp * idp;
        s = (dv + de) * inv;
    }
}

}  // namespace mmffb
