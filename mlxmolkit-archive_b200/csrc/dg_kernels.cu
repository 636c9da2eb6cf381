// Distance-geometry (DG) minimisation stage: the reference's DG L-BFGS
// (mlxmolkit/conformer_metal.py:196-547) as a persistent B200 kernel.
//
// One CTA minimises one conformer at a time, start to exit, and takes the next
// from a work counter (largest molecules first).  Per conformer:
//
//   E(x)    = sum_dist w*(d^2/ub^2 - 1)^2 above ub, w*(2lb^2/(lb^2+d^2) - 1)^2 below lb
//           + sum_chiral wc*(V - bound)^2 outside [lower, upper]  (V from the first 3 coords)
//           + sum_fourth w4 * x_4^2                                 (dim 4 only)
//   g0      = 0.1 * grad E(x0), halved while max|g0| > 10 (first gradient only, as the reference)
//   d0      = -g0, then per iteration: cap |d| at 100*max(|x|, n*dim), slope = d.g,
//             backtracking from lambda = 1 with the reference's cubic/quadratic model
//             (Armijo 1e-4, clamp [0.1, 0.5] lambda, MOVETOL 1e-6, at most 1000 trials),
//             TOLX 1.2e-6 exit, then gradient, gradient exit
//             max(|g_i| * max(|x_i|, 1)) / max(E, 1) < grad_tol,
//             history (s, y) when s.y > 1e-10 (ring of m), two-loop with gamma = s.y / y.y.
//
// B200 layout (the reference runs 32 threads per conformer with a serial thread-0
// gradient and every vector in device memory):
//   * x, g, d, s, old g and q live in shared memory as one float4 per atom (the 4th
//     component is zero in 3-D); each thread owns atoms tid, tid + NT, ... for every
//     vector operation, so elementwise steps need no barrier;
//   * the energy runs over the molecule's flat term list (16-byte records, coalesced);
//   * the gradient runs per atom over an incidence list that names each distance term
//     under both of its atoms, so every thread writes only its own atoms' gradient:
//     no atomics, and the result is bit-identical from run to run;
//   * the L-BFGS history (s, y) sits in a per-CTA slot of device memory (L2-resident),
//     read and written only by the owning thread of each atom;
//   * the energy after an accepted line-search step is the accepted trial energy: the
//     reference evaluates the same function at the same point again (same code, same
//     order), so the value is the same and the evaluation is skipped.
//
// The ETK stage (mlxmolkit/etk_metal.py:27-536) runs the same optimizer (FF = kETK) without the
// first-gradient scaling, in 3-D, on 6-term Fourier torsions (impropers are Fourier terms with
// V1 = w, s1 = -1) and flat-bottom 1-2 / 1-3 / 1-4 distance terms.  Its gradient has two
// phases: every Fourier term writes its four atoms' gradient vectors to shared memory, then
// each thread sums, for its own atoms, those rows and its flat-bottom incidences.
//
// No wait in this file spins: every loop is bounded by the iteration caps.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "mmffb200_dg.h"

namespace mmffb {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *where);

namespace dg {

constexpr float kTolx = 1.2e-6f;          // conformer_metal.py:32
constexpr float kFuncTol = 1e-4f;         // :33
constexpr float kMoveTol = 1e-6f;         // :34
constexpr float kMaxStepFactor = 100.0f;  // :35
constexpr int kMaxLs = 1000;              // :36
constexpr int kMaxHist = 16;

constexpr int kDG = 0, kETK = 1;

struct Args {
    MMFFDGBatchDev b;
    MMFFETKTermsDev e;
    MMFFDGParams p;
    float *pos;
    float *energy;
    int32_t *status;
    int32_t *iters;
    float *grad_out;
    float4 *hist;
    int *counter;
    int slot_atoms;
    int tor_slots;   // Fourier-term gradient rows in shared memory (ETK)
};

template <int NT>
__device__ __forceinline__ void bar() {
    if constexpr (NT == 32) __syncwarp();
    else __syncthreads();
}

// Block reduction of NS sums and NM maxima; every thread gets the results.  buf holds
// NW * 4 floats and alternates between two halves, so no trailing barrier is needed.
template <int NT, int NS, int NM>
__device__ __forceinline__ void breduce(float (&s)[NS > 0 ? NS : 1], float (&m)[NM > 0 ? NM : 1], float *buf) {
    static_assert(NS + NM <= 4, "at most four values per reduction");
#pragma unroll
    for (int o = 16; o; o >>= 1) {
#pragma unroll
        for (int k = 0; k < NS; ++k) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
#pragma unroll
        for (int k = 0; k < NM; ++k) m[k] = fmaxf(m[k], __shfl_xor_sync(0xffffffffu, m[k], o));
    }
    if constexpr (NT == 32) {
        __syncwarp();
    } else {
        constexpr int NW = NT / 32, K = NS + NM;
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) {
#pragma unroll
            for (int k = 0; k < NS; ++k) buf[w * K + k] = s[k];
#pragma unroll
            for (int k = 0; k < NM; ++k) buf[w * K + NS + k] = m[k];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            float v = buf[k];
            for (int i = 1; i < NW; ++i) v += buf[i * K + k];
            s[k] = v;
        }
#pragma unroll
        for (int k = 0; k < NM; ++k) {
            float v = buf[NS + k];
            for (int i = 1; i < NW; ++i) v = fmaxf(v, buf[i * K + NS + k]);
            m[k] = v;
        }
    }
}

template <int NT>
__device__ __forceinline__ float bsum(float v, float *buf) {
    float s[1] = {v}, m[1] = {0.f};
    breduce<NT, 1, 0>(s, m, buf);
    return s[0];
}

template <int NT>
__device__ __forceinline__ float bmax(float v, float *buf) {
    float s[1] = {0.f}, m[1] = {v};
    breduce<NT, 0, 1>(s, m, buf);
    return m[0];
}

__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ float amax4(float4 a) { return fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(a.z), fabsf(a.w))); }

// distance-violation energy (conformer_metal.py:37-56)
__device__ __forceinline__ float dist_e(float4 xi, float4 xj, float lb2, float ub2, float w) {
    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z, dw = xi.w - xj.w;
    const float d2 = dx * dx + dy * dy + dz * dz + dw * dw;
    if (d2 > ub2) {
        const float v = d2 / ub2 - 1.0f;
        return w * v * v;
    }
    if (d2 < lb2) {
        const float v = 2.0f * lb2 / (lb2 + d2) - 1.0f;
        return w * v * v;
    }
    return 0.0f;
}

struct Chiral {
    float3 c23, c31, c12;
    float vol;
};

__device__ __forceinline__ Chiral chiral_geom(float4 p1, float4 p2, float4 p3, float4 p4) {
    const float3 v1 = make_float3(p1.x - p4.x, p1.y - p4.y, p1.z - p4.z);
    const float3 v2 = make_float3(p2.x - p4.x, p2.y - p4.y, p2.z - p4.z);
    const float3 v3 = make_float3(p3.x - p4.x, p3.y - p4.y, p3.z - p4.z);
    Chiral r;
    r.c23 = make_float3(v2.y * v3.z - v2.z * v3.y, v2.z * v3.x - v2.x * v3.z, v2.x * v3.y - v2.y * v3.x);
    r.c31 = make_float3(v3.y * v1.z - v3.z * v1.y, v3.z * v1.x - v3.x * v1.z, v3.x * v1.y - v3.y * v1.x);
    r.c12 = make_float3(v1.y * v2.z - v1.z * v2.y, v1.z * v2.x - v1.x * v2.z, v1.x * v2.y - v1.y * v2.x);
    r.vol = v1.x * r.c23.x + v1.y * r.c23.y + v1.z * r.c23.z;
    return r;
}

// E(X) of one conformer over the flat term lists (block-reduced; every thread gets it)
template <int NT>
__device__ float dg_energy(const Args &a, const float4 *X, int mol, int N, int base, float *buf) {
    const MMFFDGBatchDev &b = a.b;
    const float4 *rec = reinterpret_cast<const float4 *>(b.dist_rec);
    float e = 0.0f;
    const int d1 = b.dist_starts[mol + 1];
    for (int t = b.dist_starts[mol] + (int)threadIdx.x; t < d1; t += NT) {
        const float4 r = __ldg(rec + t);
        const int ij = __float_as_int(r.x);
        e += dist_e(X[ij & 0xffff], X[ij >> 16], r.y, r.z, r.w);
    }
    const int c1 = b.chiral_starts[mol + 1];
    const int4 *quads = reinterpret_cast<const int4 *>(b.chiral_quads);
    const float2 *bnds = reinterpret_cast<const float2 *>(b.chiral_bounds);
    for (int t = b.chiral_starts[mol] + (int)threadIdx.x; t < c1; t += NT) {
        const int4 q = __ldg(quads + t);
        const float2 bd = __ldg(bnds + t);
        const float vol = chiral_geom(X[q.x], X[q.y], X[q.z], X[q.w]).vol;
        const float cw = a.p.chiral_weight;
        if (vol < bd.x) e += cw * (vol - bd.x) * (vol - bd.x);
        else if (vol > bd.y) e += cw * (vol - bd.y) * (vol - bd.y);
    }
    if (b.dim == 4) {
        const float fw = a.p.fourth_dim_weight;
        for (int i = threadIdx.x; i < N; i += NT) {
            const int cnt = __ldg(b.fourth_count + base + i);
            if (cnt) {
                const float w4 = X[i].w;
                e += (float)cnt * fw * w4 * w4;
            }
        }
    }
    return bsum<NT>(e, buf);
}

// unscaled gradient of one conformer into G (each thread its own atoms)
template <int NT>
__device__ void dg_gradient(const Args &a, const float4 *X, float4 *G, int mol, int N, int base) {
    const MMFFDGBatchDev &b = a.b;
    const float4 *inc = reinterpret_cast<const float4 *>(b.dinc_rec);
    const int4 *quads = reinterpret_cast<const int4 *>(b.chiral_quads);
    const float2 *bnds = reinterpret_cast<const float2 *>(b.chiral_bounds);
    const int2 *cinc = reinterpret_cast<const int2 *>(b.cinc_rec);
    const float cw = a.p.chiral_weight, fw = a.p.fourth_dim_weight;
    (void)mol;
    for (int i = threadIdx.x; i < N; i += NT) {
        const int r = base + i;
        const float4 xi = X[i];
        float gx = 0.f, gy = 0.f, gz = 0.f, gw = 0.f;
        const int e1 = __ldg(b.dinc_starts + r + 1);
#pragma unroll 2
        for (int e = __ldg(b.dinc_starts + r); e < e1; ++e) {
            const float4 q = __ldg(inc + e);
            const float4 xo = X[__float_as_int(q.x)];
            const float dx = xi.x - xo.x, dy = xi.y - xo.y, dz = xi.z - xo.z, dw = xi.w - xo.w;
            const float d2 = dx * dx + dy * dy + dz * dz + dw * dw;
            float pf = 0.0f;
            if (d2 > q.z) {
                pf = q.w * 4.0f * (d2 / q.z - 1.0f) / q.z;  // conformer_metal.py:70-71
            } else if (d2 < q.y) {
                const float l = d2 + q.y;
                pf = q.w * 8.0f * q.y * (1.0f - 2.0f * q.y / l) / (l * l);  // :72-74
            }
            gx += pf * dx;
            gy += pf * dy;
            gz += pf * dz;
            gw += pf * dw;
        }
        const int k1 = __ldg(b.cinc_starts + r + 1);
        for (int k = __ldg(b.cinc_starts + r); k < k1; ++k) {
            const int2 cr = __ldg(cinc + k);
            const int4 q = __ldg(quads + cr.x);
            const float2 bd = __ldg(bnds + cr.x);
            const Chiral c = chiral_geom(X[q.x], X[q.y], X[q.z], X[q.w]);
            float pf = 0.0f;
            if (c.vol < bd.x) pf = 2.0f * cw * (c.vol - bd.x);
            else if (c.vol > bd.y) pf = 2.0f * cw * (c.vol - bd.y);
            if (pf == 0.0f) continue;
            float3 v;
            if (cr.y == 0) v = c.c23;
            else if (cr.y == 1) v = c.c31;
            else if (cr.y == 2) v = c.c12;
            else v = make_float3(-(c.c23.x + c.c31.x + c.c12.x), -(c.c23.y + c.c31.y + c.c12.y),
                                 -(c.c23.z + c.c31.z + c.c12.z));
            gx += pf * v.x;
            gy += pf * v.y;
            gz += pf * v.z;
        }
        if (b.dim == 4) {
            const int cnt = __ldg(b.fourth_count + r);
            if (cnt) gw += (float)cnt * (2.0f * fw * xi.w);
        }
        G[i] = make_float4(gx, gy, gz, gw);
    }
}

// ---------------------------------------------------------------- ETK terms

__device__ __forceinline__ float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

struct Tors {
    float3 r1, r2, r3, r4, t0, t1;
};

// the reference's torsion convention: r1 = p1 - p2, r2 = p3 - p2, r3 = -r2, r4 = p4 - p3,
// normals t0 = r1 x r2, t1 = r3 x r4 (etk_metal.py:35-49)
__device__ __forceinline__ Tors tors_geom(float4 p1, float4 p2, float4 p3, float4 p4) {
    Tors T;
    T.r1 = sub3(xyz(p1), xyz(p2));
    T.r2 = sub3(xyz(p3), xyz(p2));
    T.r3 = make_float3(-T.r2.x, -T.r2.y, -T.r2.z);
    T.r4 = sub3(xyz(p4), xyz(p3));
    T.t0 = cross3(T.r1, T.r2);
    T.t1 = cross3(T.r3, T.r4);
    return T;
}

// cos(phi) as the energy takes it: 0 for a degenerate pair of normals, clamped to [-1, 1]
__device__ __forceinline__ float tors_cos(const Tors &T) {
    const float comb = dot3(T.t0, T.t0) * dot3(T.t1, T.t1);
    if (comb < 1e-16f) return 0.0f;
    return fminf(fmaxf(dot3(T.t0, T.t1) * rsqrtf(comb), -1.0f), 1.0f);
}

struct Coef {
    float V[6], S[6];
};

__device__ __forceinline__ Coef load_coef(const float *coef, int t) {
    const float4 *c = reinterpret_cast<const float4 *>(coef) + 3 * (size_t)t;
    const float4 a = __ldg(c), b = __ldg(c + 1), d = __ldg(c + 2);
    Coef k;
    k.V[0] = a.x; k.V[1] = a.y; k.V[2] = a.z; k.V[3] = a.w; k.V[4] = b.x; k.V[5] = b.y;
    k.S[0] = b.z; k.S[1] = b.w; k.S[2] = d.x; k.S[3] = d.y; k.S[4] = d.z; k.S[5] = d.w;
    return k;
}

// sum_k V_k (1 + s_k T_{k+1}(c)) with T_n the Chebyshev polynomials (T_n(cos phi) = cos(n phi)),
// and d/dc of it (etk_metal.py:51-61)
__device__ __forceinline__ float fourier(float c, const Coef &k, float *dedc) {
    float t0 = 1.0f, t1 = c, d0 = 0.0f, d1 = 1.0f, e = 0.0f, de = 0.0f;
#pragma unroll
    for (int n = 1; n <= 6; ++n) {
        e += k.V[n - 1] * (1.0f + k.S[n - 1] * t1);
        de += k.V[n - 1] * k.S[n - 1] * d1;
        const float t2 = 2.0f * c * t1 - t0, d2 = 2.0f * t1 + 2.0f * c * d1 - d0;
        t0 = t1; t1 = t2; d0 = d1; d1 = d2;
    }
    if (dedc) *dedc = de;
    return e;
}

// gradient of one Fourier term on its four atoms: dE/dcos through the two cross products;
// zero when a normal is degenerate (etk_metal.py:63-103 keeps the same cases)
__device__ __forceinline__ void tors_grad(const Tors &T, const Coef &k, float3 g[4]) {
    const float d0 = dot3(T.t0, T.t0), d1 = dot3(T.t1, T.t1);
    if (d0 < 1e-16f || d1 < 1e-16f) {
        g[0] = g[1] = g[2] = g[3] = make_float3(0.f, 0.f, 0.f);
        return;
    }
    const float i0 = rsqrtf(fmaxf(d0, 1e-16f)), i1 = rsqrtf(fmaxf(d1, 1e-16f));
    const float3 n0 = make_float3(T.t0.x * i0, T.t0.y * i0, T.t0.z * i0);
    const float3 n1 = make_float3(T.t1.x * i1, T.t1.y * i1, T.t1.z * i1);
    const float c = fminf(fmaxf(dot3(n0, n1), -1.0f), 1.0f);
    const float sp = sqrtf(fmaxf(1.0f - c * c, 0.0f));
    float dedc;
    fourier(c, k, &dedc);
    const float dedphi = -sp * dedc;
    const float st = fabsf(sp) > 1e-8f ? -dedphi / sp : -dedphi / fmaxf(fabsf(c), 1e-16f) * (c + 1e-30f >= 0.f ? 1.f : -1.f);
    const float3 dc0 = make_float3(i0 * (n1.x - c * n0.x), i0 * (n1.y - c * n0.y), i0 * (n1.z - c * n0.z));
    const float3 dc1 = make_float3(i1 * (n0.x - c * n1.x), i1 * (n0.y - c * n1.y), i1 * (n0.z - c * n1.z));
    const float3 a1 = cross3(T.r2, dc0), a2 = cross3(dc0, T.r1), a3 = cross3(T.r4, dc1), a4 = cross3(dc1, T.r3);
    g[0] = make_float3(st * a1.x, st * a1.y, st * a1.z);
    g[1] = make_float3(st * (a3.x - a1.x - a2.x), st * (a3.y - a1.y - a2.y), st * (a3.z - a1.z - a2.z));
    g[2] = make_float3(st * (a2.x - a3.x - a4.x), st * (a2.y - a3.y - a4.y), st * (a2.z - a3.z - a4.z));
    g[3] = make_float3(st * a4.x, st * a4.y, st * a4.z);
}

// flat-bottom term: w (d - bound)^2 outside [lb, ub], d = sqrt(d^2 + 1e-12) (etk_metal.py:126-150)
__device__ __forceinline__ float fb_e(float4 xi, float4 xj, float lb, float ub, float w) {
    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    const float dist = sqrtf(dx * dx + dy * dy + dz * dz + 1e-12f);
    if (dist < lb) return w * (dist - lb) * (dist - lb);
    if (dist > ub) return w * (dist - ub) * (dist - ub);
    return 0.0f;
}

template <int NT>
__device__ float etk_energy(const Args &a, const float4 *X, int mol, float *buf) {
    const MMFFETKTermsDev &E = a.e;
    const float4 *rec = reinterpret_cast<const float4 *>(E.fb_rec);
    float e = 0.0f;
    const int f1 = E.fb_starts[mol + 1];
    for (int t = E.fb_starts[mol] + (int)threadIdx.x; t < f1; t += NT) {
        const float4 r = __ldg(rec + t);
        const int ij = __float_as_int(r.x);
        e += fb_e(X[ij & 0xffff], X[ij >> 16], r.y, r.z, r.w);
    }
    const int4 *quads = reinterpret_cast<const int4 *>(E.tor_quads);
    const int t1 = E.tor_starts[mol + 1];
    for (int t = E.tor_starts[mol] + (int)threadIdx.x; t < t1; t += NT) {
        const int4 q = __ldg(quads + t);
        e += fourier(tors_cos(tors_geom(X[q.x], X[q.y], X[q.z], X[q.w])), load_coef(E.tor_coef, t), nullptr);
    }
    return bsum<NT>(e, buf);
}

template <int NT>
__device__ void etk_gradient(const Args &a, const float4 *X, float4 *G, int mol, int N, int base, float4 *TG) {
    const MMFFETKTermsDev &E = a.e;
    const int4 *quads = reinterpret_cast<const int4 *>(E.tor_quads);
    const int ts = E.tor_starts[mol], te = E.tor_starts[mol + 1];
    for (int t = ts + (int)threadIdx.x; t < te; t += NT) {
        const int4 q = __ldg(quads + t);
        float3 g[4];
        tors_grad(tors_geom(X[q.x], X[q.y], X[q.z], X[q.w]), load_coef(E.tor_coef, t), g);
#pragma unroll
        for (int r = 0; r < 4; ++r) TG[4 * (t - ts) + r] = make_float4(g[r].x, g[r].y, g[r].z, 0.f);
    }
    bar<NT>();
    const float4 *inc = reinterpret_cast<const float4 *>(E.fbinc_rec);
    const int2 *tinc = reinterpret_cast<const int2 *>(E.tinc_rec);
    for (int i = threadIdx.x; i < N; i += NT) {
        const int r = base + i;
        const float4 xi = X[i];
        float gx = 0.f, gy = 0.f, gz = 0.f;
        const int e1 = __ldg(E.fbinc_starts + r + 1);
        for (int k = __ldg(E.fbinc_starts + r); k < e1; ++k) {
            const float4 q = __ldg(inc + k);
            const float4 xo = X[__float_as_int(q.x)];
            const float dx = xi.x - xo.x, dy = xi.y - xo.y, dz = xi.z - xo.z;
            const float dist = sqrtf(dx * dx + dy * dy + dz * dz + 1e-12f);
            float pf = 0.0f;
            if (dist < q.y) pf = q.w * 2.0f * (dist - q.y) / dist;
            else if (dist > q.z) pf = q.w * 2.0f * (dist - q.z) / dist;
            gx += pf * dx;
            gy += pf * dy;
            gz += pf * dz;
        }
        const int k1 = __ldg(E.tinc_starts + r + 1);
        for (int k = __ldg(E.tinc_starts + r); k < k1; ++k) {
            const int2 tr = __ldg(tinc + k);
            const float4 v = TG[4 * (tr.x - ts) + tr.y];
            gx += v.x;
            gy += v.y;
            gz += v.z;
        }
        G[i] = make_float4(gx, gy, gz, 0.f);
    }
}

// ---------------------------------------------------------------- the optimizer

__device__ __forceinline__ float4 load_atom(const float *P, int i, int dim) {
    if (dim == 4) return make_float4(P[4 * i], P[4 * i + 1], P[4 * i + 2], P[4 * i + 3]);
    return make_float4(P[3 * i], P[3 * i + 1], P[3 * i + 2], 0.0f);
}

__device__ __forceinline__ void store_atom(float *P, int i, int dim, float4 v) {
    if (dim == 4) {
        P[4 * i] = v.x; P[4 * i + 1] = v.y; P[4 * i + 2] = v.z; P[4 * i + 3] = v.w;
    } else {
        P[3 * i] = v.x; P[3 * i + 1] = v.y; P[3 * i + 2] = v.z;
    }
}

__device__ __forceinline__ float4 f4(float x, float y, float z, float w) { return make_float4(x, y, z, w); }
__device__ __forceinline__ float4 axpy(float a, float4 x, float4 y) {  // y + a x
    return f4(fmaf(a, x.x, y.x), fmaf(a, x.y, y.y), fmaf(a, x.z, y.z), fmaf(a, x.w, y.w));
}
__device__ __forceinline__ float4 scale4(float a, float4 x) { return f4(a * x.x, a * x.y, a * x.z, a * x.w); }
__device__ __forceinline__ float4 sub4(float4 a, float4 b) { return f4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }

template <int NT, int FF>
__device__ __forceinline__ float ff_energy(const Args &a, const float4 *X, int mol, int N, int base, float *buf) {
    if constexpr (FF == kDG) return dg_energy<NT>(a, X, mol, N, base, buf);
    else return etk_energy<NT>(a, X, mol, buf);
}

template <int NT, int FF>
__device__ __forceinline__ void ff_gradient(const Args &a, const float4 *X, float4 *G, int mol, int N, int base,
                                            float4 *TG) {
    if constexpr (FF == kDG) dg_gradient<NT>(a, X, G, mol, N, base);
    else etk_gradient<NT>(a, X, G, mol, N, base, TG);
}

template <int NT, int FF, bool HS>
__global__ void __launch_bounds__(NT) lbfgs_kernel(const __grid_constant__ Args a) {
    constexpr int NW = NT / 32;
    extern __shared__ float4 sm[];
    __shared__ int s_next;
    const int NA = a.slot_atoms, M = a.p.lbfgs_m, tid = threadIdx.x;
    float4 *X = sm, *G = X + NA, *D = G + NA, *XO = D + NA, *GO = XO + NA, *Q = GO + NA;
    float *rbase = reinterpret_cast<float *>(Q + NA);
    float *rho = rbase + 2 * NW * 4;
    float4 *TG = reinterpret_cast<float4 *>(rho + kMaxHist);
    int rsel = 0;
    auto rb = [&]() {
        rsel ^= 1;
        return rbase + rsel * NW * 4;
    };
    // L-BFGS history: in shared memory after the Fourier-term rows (HS), else this CTA's device slot
    float4 *S = HS ? TG + 4 * a.tor_slots : a.hist + (size_t)blockIdx.x * 2 * M * NA, *Y = S + (size_t)M * NA;
    const MMFFDGBatchDev &b = a.b;
    const int dim = b.dim, max_iters = a.p.max_iters;

    for (;;) {
        if (tid == 0) s_next = atomicAdd(a.counter, 1);
        __syncthreads();
        const int k = s_next;
        if (k >= b.n_conf) break;
        const int c = b.conf_order ? b.conf_order[k] : k;
        const int mol = b.conf_to_mol[c], N = b.mol_n_atoms[mol], base = b.mol_atom_base[mol];
        const int nv = N * dim;
        float *P = a.pos + (size_t)b.conf_atom_starts[c] * dim;
        for (int i = tid; i < N; i += NT) X[i] = load_atom(P, i, dim);
        bar<NT>();

        float energy = ff_energy<NT, FF>(a, X, mol, N, base, rb());
        ff_gradient<NT, FF>(a, X, G, mol, N, base, TG);
        if constexpr (FF == kDG) {
            // 0.1 scaling, halved while max > 10 (conformer_metal.py:303-313); ETK has none
            for (int i = tid; i < N; i += NT) G[i] = scale4(0.1f, G[i]);
            for (int sc = 0; sc < 20; ++sc) {
                float mx = 0.f;
                for (int i = tid; i < N; i += NT) mx = fmaxf(mx, amax4(G[i]));
                if (bmax<NT>(mx, rb()) <= 10.0f) break;
                for (int i = tid; i < N; i += NT) G[i] = scale4(0.5f, G[i]);
            }
        }
        float ss = 0.f;
        for (int i = tid; i < N; i += NT) {
            D[i] = scale4(-1.0f, G[i]);
            ss += dot4(X[i], X[i]);
        }
        const float max_step = kMaxStepFactor * fmaxf(sqrtf(bsum<NT>(ss, rb())), (float)nv);

        int status = MMFFB_DG_MAXIT, hc = 0, hi = 0, it = 0;
        float alph[kMaxHist];
        for (it = 0; it < max_iters; ++it) {
            const float old_e = energy;
            float s2[2] = {0.f, 0.f}, m1[1] = {0.f};
            for (int i = tid; i < N; i += NT) {
                const float4 x = X[i], d = D[i];
                XO[i] = x;
                s2[0] += dot4(d, d);
                s2[1] += dot4(d, G[i]);
                m1[0] = fmaxf(m1[0], fmaxf(fmaxf(fabsf(d.x) / fmaxf(fabsf(x.x), 1.f), fabsf(d.y) / fmaxf(fabsf(x.y), 1.f)),
                                           fmaxf(fabsf(d.z) / fmaxf(fabsf(x.z), 1.f), fabsf(d.w) / fmaxf(fabsf(x.w), 1.f))));
            }
            breduce<NT, 2, 1>(s2, m1, rb());
            const float dn = sqrtf(s2[0]);
            float slope = s2[1], test = m1[0];
            if (dn > max_step) {  // conformer_metal.py:339-340
                const float sc = max_step / dn;
                for (int i = tid; i < N; i += NT) D[i] = scale4(sc, D[i]);
                slope *= sc;
                test *= sc;
            }
            const float lam_min = kMoveTol / fmaxf(test, 1e-30f);
            float lam = 1.0f, prev_lam = 1.0f, prev_e = old_e;
            bool done = false;
            for (int ls = 0; ls < kMaxLs && !done; ++ls) {
                if (lam < lam_min) {
                    for (int i = tid; i < N; i += NT) X[i] = XO[i];
                    done = true;
                    break;
                }
                for (int i = tid; i < N; i += NT) X[i] = axpy(lam, D[i], XO[i]);
                bar<NT>();
                const float te = ff_energy<NT, FF>(a, X, mol, N, base, rb());
                if (te - old_e <= kFuncTol * lam * slope) {
                    energy = te;
                    done = true;
                } else {
                    float tl;
                    if (ls == 0) {
                        tl = -slope / (2.0f * (te - old_e - slope));
                    } else {
                        const float r1 = te - old_e - lam * slope, r2 = prev_e - old_e - prev_lam * slope;
                        const float l2 = lam * lam, p2 = prev_lam * prev_lam, dnm = lam - prev_lam;
                        if (fabsf(dnm) < 1e-30f) {
                            tl = 0.5f * lam;
                        } else {
                            const float ca = (r1 / l2 - r2 / p2) / dnm, cb = (-prev_lam * r1 / l2 + lam * r2 / p2) / dnm;
                            if (fabsf(ca) < 1e-30f) {
                                tl = fabsf(cb) > 1e-30f ? -slope / (2.0f * cb) : 0.5f * lam;
                            } else {
                                const float disc = cb * cb - 3.0f * ca * slope;
                                if (disc < 0.0f) tl = 0.5f * lam;
                                else if (cb <= 0.0f) tl = (-cb + sqrtf(disc)) / (3.0f * ca);
                                else tl = -slope / (cb + sqrtf(disc));
                            }
                        }
                    }
                    tl = fminf(fmaxf(tl, 0.1f * lam), 0.5f * lam);  // a NaN candidate becomes 0.1 lam
                    prev_lam = lam;
                    prev_e = te;
                    lam = tl;
                }
            }
            if (!done)
                for (int i = tid; i < N; i += NT) X[i] = XO[i];
            float tx = 0.f;
            for (int i = tid; i < N; i += NT) {
                const float4 x = X[i], s = sub4(x, XO[i]);
                XO[i] = s;
                tx = fmaxf(tx, fmaxf(fmaxf(fabsf(s.x) / fmaxf(fabsf(x.x), 1.f), fabsf(s.y) / fmaxf(fabsf(x.y), 1.f)),
                                     fmaxf(fabsf(s.z) / fmaxf(fabsf(x.z), 1.f), fabsf(s.w) / fmaxf(fabsf(x.w), 1.f))));
            }
            if (bmax<NT>(tx, rb()) < kTolx) {  // the reduction's barrier also publishes X
                status = MMFFB_DG_CONVERGED;
                break;
            }
            for (int i = tid; i < N; i += NT) GO[i] = G[i];
            ff_gradient<NT, FF>(a, X, G, mol, N, base, TG);
            float gt = 0.f;
            for (int i = tid; i < N; i += NT) {
                const float4 g = G[i], x = X[i];
                gt = fmaxf(gt, fmaxf(fmaxf(fabsf(g.x) * fmaxf(fabsf(x.x), 1.f), fabsf(g.y) * fmaxf(fabsf(x.y), 1.f)),
                                     fmaxf(fabsf(g.z) * fmaxf(fabsf(x.z), 1.f), fabsf(g.w) * fmaxf(fabsf(x.w), 1.f))));
            }
            if (bmax<NT>(gt, rb()) / fmaxf(energy, 1.0f) < a.p.grad_tol) {
                status = MMFFB_DG_CONVERGED;
                break;
            }
            float ys = 0.f;
            for (int i = tid; i < N; i += NT) {
                const float4 y = sub4(G[i], GO[i]);
                Q[i] = y;
                ys += dot4(y, XO[i]);
            }
            ys = bsum<NT>(ys, rb());
            if (ys > 1e-10f) {
                const int slot = hi % M;
                for (int i = tid; i < N; i += NT) {
                    S[(size_t)slot * NA + i] = XO[i];
                    Y[(size_t)slot * NA + i] = Q[i];
                }
                if (tid == 0) rho[slot] = 1.0f / ys;
                ++hi;
                if (hc < M) ++hc;
            }
            // two-loop recursion (conformer_metal.py:518-545); rho is read after a reduction barrier
            for (int i = tid; i < N; i += NT) Q[i] = G[i];
            for (int j = hc - 1; j >= 0; --j) {
                int slot = (hi - 1 - (hc - 1 - j)) % M;
                if (slot < 0) slot += M;
                float t = 0.f;
                for (int i = tid; i < N; i += NT) t += dot4(S[(size_t)slot * NA + i], Q[i]);
                const float aj = rho[slot] * bsum<NT>(t, rb());
                alph[j] = aj;
                for (int i = tid; i < N; i += NT) Q[i] = axpy(-aj, Y[(size_t)slot * NA + i], Q[i]);
            }
            if (hc > 0) {
                int nw = (hi - 1) % M;
                if (nw < 0) nw += M;
                float s2b[2] = {0.f, 0.f}, mz[1] = {0.f};
                for (int i = tid; i < N; i += NT) {
                    const float4 sv = S[(size_t)nw * NA + i], yv = Y[(size_t)nw * NA + i];
                    s2b[0] += dot4(sv, yv);
                    s2b[1] += dot4(yv, yv);
                }
                breduce<NT, 2, 0>(s2b, mz, rb());
                const float gm = s2b[0] / fmaxf(s2b[1], 1e-30f);
                for (int i = tid; i < N; i += NT) Q[i] = scale4(gm, Q[i]);
            }
            for (int j = 0; j < hc; ++j) {
                int slot = (hi - 1 - (hc - 1 - j)) % M;
                if (slot < 0) slot += M;
                float t = 0.f;
                for (int i = tid; i < N; i += NT) t += dot4(Y[(size_t)slot * NA + i], Q[i]);
                const float beta = rho[slot] * bsum<NT>(t, rb());
                for (int i = tid; i < N; i += NT) Q[i] = axpy(alph[j] - beta, S[(size_t)slot * NA + i], Q[i]);
            }
            for (int i = tid; i < N; i += NT) D[i] = scale4(-1.0f, Q[i]);
        }
        for (int i = tid; i < N; i += NT) store_atom(P, i, dim, X[i]);
        if (tid == 0) {
            a.energy[c] = energy;
            a.status[c] = status;
            if (a.iters) a.iters[c] = status == MMFFB_DG_CONVERGED ? it + 1 : max_iters;
        }
        __syncthreads();
    }
}

template <int NT, int FF>
__global__ void __launch_bounds__(NT) energy_grad_kernel(const __grid_constant__ Args a) {
    constexpr int NW = NT / 32;
    extern __shared__ float4 sm[];
    const int NA = a.slot_atoms;
    float4 *X = sm, *G = X + NA;
    float *red = reinterpret_cast<float *>(G + NA);
    float4 *TG = reinterpret_cast<float4 *>(red + 2 * NW * 4 + kMaxHist);
    const MMFFDGBatchDev &b = a.b;
    const int c = blockIdx.x, dim = b.dim;
    const int mol = b.conf_to_mol[c], N = b.mol_n_atoms[mol], base = b.mol_atom_base[mol];
    const float *P = a.pos + (size_t)b.conf_atom_starts[c] * dim;
    for (int i = threadIdx.x; i < N; i += NT) X[i] = load_atom(P, i, dim);
    bar<NT>();
    const float e = ff_energy<NT, FF>(a, X, mol, N, base, red);
    ff_gradient<NT, FF>(a, X, G, mol, N, base, TG);
    float *GP = a.grad_out + (size_t)b.conf_atom_starts[c] * dim;
    for (int i = threadIdx.x; i < N; i += NT) store_atom(GP, i, dim, G[i]);
    if (threadIdx.x == 0) a.energy[c] = e;
}

// ---------------------------------------------------------------- stereo checks

struct StereoArgs {
    MMFFDGBatchDev b;
    const int32_t *tet_starts, *tet_quads;
    float vol_tol;
    const float *pos;
    int32_t *passed;
};

__device__ __forceinline__ float3 atom3(const float *P, int i, int dim) {
    return make_float3(P[dim * i], P[dim * i + 1], P[dim * i + 2]);
}

__device__ __forceinline__ float quad_volume(const float *P, int dim, int4 q) {
    const float3 p3 = atom3(P, q.w, dim);
    const float3 v1 = sub3(atom3(P, q.x, dim), p3), v2 = sub3(atom3(P, q.y, dim), p3), v3 = sub3(atom3(P, q.z, dim), p3);
    return dot3(v1, cross3(v2, v3));
}

// one warp per conformer
__global__ void __launch_bounds__(128) stereo_kernel(const __grid_constant__ StereoArgs a) {
    const int c = blockIdx.x * 4 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (c >= a.b.n_conf) return;
    const int mol = a.b.conf_to_mol[c], dim = a.b.dim;
    const float *P = a.pos + (size_t)a.b.conf_atom_starts[c] * dim;
    bool ok = true;
    const int4 *tq = reinterpret_cast<const int4 *>(a.tet_quads);
    for (int t = a.tet_starts[mol] + lane; t < a.tet_starts[mol + 1]; t += 32)
        if (fabsf(quad_volume(P, dim, __ldg(tq + t))) < a.vol_tol) ok = false;
    const int4 *cq = reinterpret_cast<const int4 *>(a.b.chiral_quads);
    const float2 *cb = reinterpret_cast<const float2 *>(a.b.chiral_bounds);
    for (int t = a.b.chiral_starts[mol] + lane; t < a.b.chiral_starts[mol + 1]; t += 32) {
        const float v = quad_volume(P, dim, __ldg(cq + t));
        const float2 bd = __ldg(cb + t);
        if (v < bd.x || v > bd.y) ok = false;
    }
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) a.passed[c] = ok ? 1 : 0;
}

int pick_threads(int max_atoms, int req) {
    if (req) return req;
    return max_atoms <= 48 ? 32 : max_atoms <= 96 ? 64 : max_atoms <= 192 ? 128 : 256;
}

// shared memory of a CTA: `vectors` float4 vectors of na atoms, the reduction halves, the
// L-BFGS rho values and (ETK) four gradient rows per Fourier term
size_t smem_bytes(int nt, int na, int vectors, int tor_slots, int hist_rows = 0) {
    return (size_t)vectors * na * sizeof(float4) + (size_t)2 * (nt / 32) * 4 * sizeof(float) +
           kMaxHist * sizeof(float) + (size_t)4 * tor_slots * sizeof(float4) + (size_t)hist_rows * na * sizeof(float4);
}

template <int FF, bool HS>
const void *minimize_kernel_ff(int nt) {
    switch (nt) {
        case 32: return reinterpret_cast<const void *>(&lbfgs_kernel<32, FF, HS>);
        case 64: return reinterpret_cast<const void *>(&lbfgs_kernel<64, FF, HS>);
        case 128: return reinterpret_cast<const void *>(&lbfgs_kernel<128, FF, HS>);
        default: return reinterpret_cast<const void *>(&lbfgs_kernel<256, FF, HS>);
    }
}

const void *minimize_kernel_for(int nt, int ff, bool hs) {
    if (ff == kDG) return hs ? minimize_kernel_ff<kDG, true>(nt) : minimize_kernel_ff<kDG, false>(nt);
    return hs ? minimize_kernel_ff<kETK, true>(nt) : minimize_kernel_ff<kETK, false>(nt);
}

template <int FF>
const void *energy_kernel_ff(int nt) {
    switch (nt) {
        case 32: return reinterpret_cast<const void *>(&energy_grad_kernel<32, FF>);
        case 64: return reinterpret_cast<const void *>(&energy_grad_kernel<64, FF>);
        case 128: return reinterpret_cast<const void *>(&energy_grad_kernel<128, FF>);
        default: return reinterpret_cast<const void *>(&energy_grad_kernel<256, FF>);
    }
}

const void *energy_kernel_for(int nt, int ff) { return ff == kDG ? energy_kernel_ff<kDG>(nt) : energy_kernel_ff<kETK>(nt); }

int check_confs(const MMFFDGBatchDev *b, const MMFFDGParams *p) {
    if (!b || !p) return fail(MMFFB_EINVAL, "null batch or parameters");
    if (b->n_conf < 0 || b->n_mols < 0) return fail(MMFFB_EINVAL, "negative count");
    if (b->dim != 3 && b->dim != 4) return fail(MMFFB_EINVAL, "dim must be 3 or 4, got %d", b->dim);
    if (b->n_conf > 0 && (b->max_atoms < 1 || b->max_atoms > 1024))
        return fail(MMFFB_ETOOBIG, "max_atoms %d outside 1..1024", b->max_atoms);
    if (p->lbfgs_m < 1 || p->lbfgs_m > kMaxHist) return fail(MMFFB_EINVAL, "lbfgs_m %d outside 1..%d", p->lbfgs_m, kMaxHist);
    if (p->max_iters < 0) return fail(MMFFB_EINVAL, "negative max_iters");
    if (p->hist_mode < 0 || p->hist_mode > 2) return fail(MMFFB_EINVAL, "hist_mode must be 0, 1 or 2");
    if (p->threads != 0 && p->threads != 32 && p->threads != 64 && p->threads != 128 && p->threads != 256)
        return fail(MMFFB_EINVAL, "threads must be 0, 32, 64, 128 or 256");
    if (b->n_conf > 0 && (!b->conf_to_mol || !b->conf_atom_starts || !b->mol_n_atoms || !b->mol_atom_base))
        return fail(MMFFB_EINVAL, "null device pointer in the conformer map");
    return 0;
}

int check(const MMFFDGBatchDev *b, const MMFFDGParams *p) {
    int r = check_confs(b, p);
    if (r) return r;
    if (b->n_conf > 0 && (!b->dist_starts || !b->dinc_starts || !b->chiral_starts || !b->cinc_starts ||
                          !b->fourth_count))
        return fail(MMFFB_EINVAL, "null device pointer in DG batch");
    return 0;
}

int check_etk(const MMFFDGBatchDev *b, const MMFFETKTermsDev *e, const MMFFDGParams *p) {
    int r = check_confs(b, p);
    if (r) return r;
    if (!e) return fail(MMFFB_EINVAL, "null ETK terms");
    if (b->dim != 3) return fail(MMFFB_EINVAL, "the ETK stage is 3-D, got dim %d", b->dim);
    if (e->max_tor < 0 || e->max_tor > 8192) return fail(MMFFB_ETOOBIG, "max_tor %d outside 0..8192", e->max_tor);
    if (b->n_conf > 0 && (!e->fb_starts || !e->fbinc_starts || !e->tor_starts || !e->tinc_starts))
        return fail(MMFFB_EINVAL, "null device pointer in ETK terms");
    return 0;
}

// resident CTAs per SM of the minimise kernel with nt threads (0 when it does not fit)
int occupancy(int nt, int ff, bool hs, int hist_m, int max_atoms, int tor_slots, int *occ, size_t *smem_out) {
    const size_t smem = smem_bytes(nt, max_atoms, 6, tor_slots, hs ? 2 * hist_m : 0);
    *occ = 0;
    *smem_out = smem;
    if (smem > 227 * 1024) return 0;
    const void *fn = minimize_kernel_for(nt, ff, hs);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(L-BFGS)");
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, fn, nt, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor(L-BFGS)");
    *smem_out = smem;
    return 0;
}

// Threads per conformer, grid and shared memory of a launch.  Unless the caller fixes the
// thread count: the largest instance whose resident CTAs hold every conformer at once (a
// batch too small to fill the GPU finishes when its slowest conformer does, so more threads
// per conformer pay), else the size-based default (measured on B200: 1000 conformers of
// <= 77 atoms 8.9k / 15.6k / 18.1k / 18.9k conformers/s at 32 / 64 / 128 / 256 threads;
// 10000 conformers of <= 87 atoms 55k / 70k / 52k / 37k).
//
// History placement: a device slot per CTA unless hist_mode = 1 asks for shared memory.  The
// slot is read back by the CTA that wrote it and stays in L1; in shared memory it only takes
// L1 capacity from the term records (measured on B200, DG stage: 20 x 50 16.1k vs 18.6k and
// 1000 x 10 54k vs 70k conformers/s, shared vs device).
int plan_grid(const MMFFDGBatchDev *b, const MMFFDGParams *p, int ff, int tor_slots, int *nt_out, size_t *smem_out,
              int *grid_out, bool *hs_out) {
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
    const int M = p->lbfgs_m;
    int nt = pick_threads(b->max_atoms, p->threads);
    size_t smem = 0;
    if (p->threads == 0)
        for (int cand = 256; cand > nt; cand /= 2) {
            int r = occupancy(cand, ff, false, M, b->max_atoms, tor_slots, &occ, &smem);
            if (r) return r;
            if (occ >= 1 && (long long)sms * occ >= b->n_conf) {
                nt = cand;
                break;
            }
        }
    int occ_g = 0, occ_s = 0;
    size_t smem_g = 0, smem_s = 0;
    int r = occupancy(nt, ff, false, M, b->max_atoms, tor_slots, &occ_g, &smem_g);
    if (r) return r;
    r = occupancy(nt, ff, true, M, b->max_atoms, tor_slots, &occ_s, &smem_s);
    if (r) return r;
    const bool hs = p->hist_mode == 1;
    if (hs && occ_s < 1) return fail(MMFFB_ETOOBIG, "the history does not fit in shared memory (%zu B)", smem_s);
    occ = hs ? occ_s : occ_g;
    smem = hs ? smem_s : smem_g;
    if (occ < 1) return fail(MMFFB_ETOOBIG, "the L-BFGS kernel does not fit an SM (%zu B shared memory)", smem);
    long long g = (long long)sms * occ;
    if (g > b->n_conf) g = b->n_conf;
    *nt_out = nt;
    *smem_out = smem;
    *grid_out = (int)g;
    *hs_out = hs;
    return 0;
}

constexpr size_t kCounterBytes = 256;

size_t scratch_for(const MMFFDGBatchDev *b, const MMFFDGParams *p, int grid, bool hs) {
    return kCounterBytes + (hs ? 0 : (size_t)grid * 2 * p->lbfgs_m * b->max_atoms * sizeof(float4));
}

int minimize(const MMFFDGBatchDev *b, const MMFFETKTermsDev *etk, const MMFFDGParams *p, int ff, float *pos,
             float *energies, int32_t *statuses, int32_t *iters, void *scratch, size_t scratch_bytes,
             mmffb_stream_t stream) {
    if (b->n_conf == 0) return 0;
    if (!pos || !energies || !statuses) return fail(MMFFB_EINVAL, "null output pointer");
    const int tor_slots = ff == kETK ? etk->max_tor : 0;
    int nt = 0, grid = 0;
    size_t smem = 0;
    bool hs = false;
    int r = plan_grid(b, p, ff, tor_slots, &nt, &smem, &grid, &hs);
    if (r) return r;
    const size_t need = scratch_for(b, p, grid, hs);
    if (!scratch || scratch_bytes < need)
        return fail(MMFFB_ESCRATCH, "scratch of %zu B given, %zu B needed", scratch_bytes, need);
    Args a;
    memset(&a, 0, sizeof a);
    a.b = *b;
    if (etk) a.e = *etk;
    a.p = *p;
    a.pos = pos;
    a.energy = energies;
    a.status = statuses;
    a.iters = iters;
    a.counter = reinterpret_cast<int *>(scratch);
    a.hist = reinterpret_cast<float4 *>(reinterpret_cast<char *>(scratch) + kCounterBytes);
    a.slot_atoms = b->max_atoms;
    a.tor_slots = tor_slots;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(a.counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(L-BFGS counter)");
    void *args[] = {&a};
    e = cudaLaunchKernel(minimize_kernel_for(nt, ff, hs), dim3(grid), dim3(nt), args, smem, st);
    if (e != cudaSuccess) return cuda_fail(e, "lbfgs_kernel launch");
    return 0;
}

int energy_grad(const MMFFDGBatchDev *b, const MMFFETKTermsDev *etk, const MMFFDGParams *p, int ff, const float *pos,
                float *energies, float *grad, mmffb_stream_t stream) {
    if (b->n_conf == 0) return 0;
    if (!pos || !energies || !grad) return fail(MMFFB_EINVAL, "null argument");
    const int nt = pick_threads(b->max_atoms, p->threads);
    const int tor_slots = ff == kETK ? etk->max_tor : 0;
    const size_t smem = smem_bytes(nt, b->max_atoms, 2, tor_slots);
    Args a;
    memset(&a, 0, sizeof a);
    a.b = *b;
    if (etk) a.e = *etk;
    a.p = *p;
    a.pos = const_cast<float *>(pos);
    a.energy = energies;
    a.grad_out = grad;
    a.slot_atoms = b->max_atoms;
    a.tor_slots = tor_slots;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const void *fn = energy_kernel_for(nt, ff);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(energy)");
    void *args[] = {&a};
    e = cudaLaunchKernel(fn, dim3(b->n_conf), dim3(nt), args, smem, st);
    if (e != cudaSuccess) return cuda_fail(e, "energy_grad_kernel launch");
    return 0;
}

size_t scratch_bytes(const MMFFDGBatchDev *b, const MMFFETKTermsDev *etk, const MMFFDGParams *p, int ff) {
    if (b->n_conf == 0) return kCounterBytes;
    int nt = 0, grid = 0;
    size_t smem = 0;
    bool hs = false;
    if (plan_grid(b, p, ff, ff == kETK ? etk->max_tor : 0, &nt, &smem, &grid, &hs)) return 0;
    return scratch_for(b, p, grid, hs);
}

}  // namespace dg
}  // namespace mmffb

using namespace mmffb;
using namespace mmffb::dg;

extern "C" {

size_t mmffb_dg_scratch_bytes(const MMFFDGBatchDev *batch, const MMFFDGParams *params) {
    if (check(batch, params)) return 0;
    return scratch_bytes(batch, nullptr, params, kDG);
}

int mmffb_dg_minimize(const MMFFDGBatchDev *batch, const MMFFDGParams *params, float *pos, float *energies,
                      int32_t *statuses, int32_t *iters, void *scratch, size_t scratch_bytes, mmffb_stream_t stream) {
    int r = check(batch, params);
    if (r) return r;
    return minimize(batch, nullptr, params, kDG, pos, energies, statuses, iters, scratch, scratch_bytes, stream);
}

int mmffb_dg_energy_grad(const MMFFDGBatchDev *batch, const MMFFDGParams *params, const float *pos, float *energies,
                         float *grad, mmffb_stream_t stream) {
    int r = check(batch, params);
    if (r) return r;
    return energy_grad(batch, nullptr, params, kDG, pos, energies, grad, stream);
}

size_t mmffb_etk_scratch_bytes(const MMFFDGBatchDev *confs, const MMFFETKTermsDev *terms, const MMFFDGParams *params) {
    if (check_etk(confs, terms, params)) return 0;
    return scratch_bytes(confs, terms, params, kETK);
}

int mmffb_etk_minimize(const MMFFDGBatchDev *confs, const MMFFETKTermsDev *terms, const MMFFDGParams *params,
                       float *pos, float *energies, int32_t *statuses, int32_t *iters, void *scratch,
                       size_t scratch_bytes, mmffb_stream_t stream) {
    int r = check_etk(confs, terms, params);
    if (r) return r;
    return minimize(confs, terms, params, kETK, pos, energies, statuses, iters, scratch, scratch_bytes, stream);
}

int mmffb_etk_energy_grad(const MMFFDGBatchDev *confs, const MMFFETKTermsDev *terms, const MMFFDGParams *params,
                          const float *pos, float *energies, float *grad, mmffb_stream_t stream) {
    int r = check_etk(confs, terms, params);
    if (r) return r;
    return energy_grad(confs, terms, params, kETK, pos, energies, grad, stream);
}

int mmffb_stereo_check(const MMFFDGBatchDev *batch, const int32_t *tet_starts, const int32_t *tet_quads,
                       float vol_tol, const float *pos, int32_t *passed, mmffb_stream_t stream) {
    if (!batch) return fail(MMFFB_EINVAL, "null batch");
    if (batch->n_conf < 0 || (batch->dim != 3 && batch->dim != 4)) return fail(MMFFB_EINVAL, "bad conformer count or dim");
    if (batch->n_conf == 0) return 0;
    if (!batch->conf_to_mol || !batch->conf_atom_starts || !batch->chiral_starts || !tet_starts || !pos || !passed)
        return fail(MMFFB_EINVAL, "null pointer");
    StereoArgs a{*batch, tet_starts, tet_quads, vol_tol, pos, passed};
    stereo_kernel<<<(batch->n_conf + 3) / 4, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "stereo_kernel launch");
    return 0;
}

}  // extern "C"
