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
// No wait in this file spins: every loop is bounded by the iteration caps.
#include <cuda_runtime.h>

#include <cstdint>

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

struct Args {
    MMFFDGBatchDev b;
    MMFFDGParams p;
    float *pos;
    float *energy;
    int32_t *status;
    int32_t *iters;
    float *grad_out;
    float4 *hist;
    int *counter;
    int slot_atoms;
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

template <int NT>
__global__ void __launch_bounds__(NT) dg_minimize_kernel(const __grid_constant__ Args a) {
    constexpr int NW = NT / 32;
    extern __shared__ float4 sm[];
    __shared__ int s_next;
    const int NA = a.slot_atoms, M = a.p.lbfgs_m, tid = threadIdx.x;
    float4 *X = sm, *G = X + NA, *D = G + NA, *XO = D + NA, *GO = XO + NA, *Q = GO + NA;
    float *rbase = reinterpret_cast<float *>(Q + NA);
    float *rho = rbase + 2 * NW * 4;
    int rsel = 0;
    auto rb = [&]() {
        rsel ^= 1;
        return rbase + rsel * NW * 4;
    };
    float4 *S = a.hist + (size_t)blockIdx.x * 2 * M * NA, *Y = S + (size_t)M * NA;
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

        float energy = dg_energy<NT>(a, X, mol, N, base, rb());
        dg_gradient<NT>(a, X, G, mol, N, base);
        // 0.1 scaling, halved while max > 10 (conformer_metal.py:303-313)
        for (int i = tid; i < N; i += NT) G[i] = scale4(0.1f, G[i]);
        for (int sc = 0; sc < 20; ++sc) {
            float mx = 0.f;
            for (int i = tid; i < N; i += NT) mx = fmaxf(mx, amax4(G[i]));
            if (bmax<NT>(mx, rb()) <= 10.0f) break;
            for (int i = tid; i < N; i += NT) G[i] = scale4(0.5f, G[i]);
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
                const float te = dg_energy<NT>(a, X, mol, N, base, rb());
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
            dg_gradient<NT>(a, X, G, mol, N, base);
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

template <int NT>
__global__ void __launch_bounds__(NT) dg_energy_grad_kernel(const __grid_constant__ Args a) {
    constexpr int NW = NT / 32;
    extern __shared__ float4 sm[];
    const int NA = a.slot_atoms;
    float4 *X = sm, *G = X + NA;
    float *red = reinterpret_cast<float *>(G + NA);
    const MMFFDGBatchDev &b = a.b;
    const int c = blockIdx.x, dim = b.dim;
    const int mol = b.conf_to_mol[c], N = b.mol_n_atoms[mol], base = b.mol_atom_base[mol];
    const float *P = a.pos + (size_t)b.conf_atom_starts[c] * dim;
    for (int i = threadIdx.x; i < N; i += NT) X[i] = load_atom(P, i, dim);
    bar<NT>();
    const float e = dg_energy<NT>(a, X, mol, N, base, red);
    (void)NW;
    dg_gradient<NT>(a, X, G, mol, N, base);
    float *GP = a.grad_out + (size_t)b.conf_atom_starts[c] * dim;
    for (int i = threadIdx.x; i < N; i += NT) store_atom(GP, i, dim, G[i]);
    if (threadIdx.x == 0) a.energy[c] = e;
}

int pick_threads(int max_atoms, int req) {
    if (req) return req;
    return max_atoms <= 48 ? 32 : max_atoms <= 96 ? 64 : max_atoms <= 192 ? 128 : 256;
}

size_t smem_bytes(int nt, int na, int vectors) {
    return (size_t)vectors * na * sizeof(float4) + (size_t)2 * (nt / 32) * 4 * sizeof(float) + kMaxHist * sizeof(float);
}

int check(const MMFFDGBatchDev *b, const MMFFDGParams *p) {
    if (!b || !p) return fail(MMFFB_EINVAL, "null DG batch or parameters");
    if (b->n_conf < 0 || b->n_mols < 0) return fail(MMFFB_EINVAL, "negative count");
    if (b->dim != 3 && b->dim != 4) return fail(MMFFB_EINVAL, "dim must be 3 or 4, got %d", b->dim);
    if (b->n_conf > 0 && (b->max_atoms < 1 || b->max_atoms > 1024))
        return fail(MMFFB_ETOOBIG, "max_atoms %d outside 1..1024", b->max_atoms);
    if (p->lbfgs_m < 1 || p->lbfgs_m > kMaxHist) return fail(MMFFB_EINVAL, "lbfgs_m %d outside 1..%d", p->lbfgs_m, kMaxHist);
    if (p->max_iters < 0) return fail(MMFFB_EINVAL, "negative max_iters");
    if (p->threads != 0 && p->threads != 32 && p->threads != 64 && p->threads != 128 && p->threads != 256)
        return fail(MMFFB_EINVAL, "threads must be 0, 32, 64, 128 or 256");
    if (b->n_conf > 0 && (!b->conf_to_mol || !b->conf_atom_starts || !b->mol_n_atoms || !b->mol_atom_base ||
                          !b->dist_starts || !b->dinc_starts || !b->chiral_starts || !b->cinc_starts ||
                          !b->fourth_count))
        return fail(MMFFB_EINVAL, "null device pointer in DG batch");
    return 0;
}

template <int NT>
const void *minimize_fn() { return reinterpret_cast<const void *>(&dg_minimize_kernel<NT>); }

const void *minimize_kernel_for(int nt) {
    switch (nt) {
        case 32: return minimize_fn<32>();
        case 64: return minimize_fn<64>();
        case 128: return minimize_fn<128>();
        default: return minimize_fn<256>();
    }
}

// resident CTAs of the minimise kernel on this device (the grid and the history slots)
int plan_grid(const MMFFDGBatchDev *b, const MMFFDGParams *p, int *nt_out, size_t *smem_out, int *grid_out) {
    const int nt = pick_threads(b->max_atoms, p->threads);
    const size_t smem = smem_bytes(nt, b->max_atoms, 6);
    const void *fn = minimize_kernel_for(nt);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(DG)");
    int dev = 0, sms = 0, occ = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, nt, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor(DG)");
    if (occ < 1) return fail(MMFFB_ETOOBIG, "DG kernel does not fit an SM (%zu B shared memory)", smem);
    long long g = (long long)sms * occ;
    if (g > b->n_conf) g = b->n_conf;
    *nt_out = nt;
    *smem_out = smem;
    *grid_out = (int)g;
    return 0;
}

constexpr size_t kCounterBytes = 256;

}  // namespace dg
}  // namespace mmffb

using namespace mmffb;
using namespace mmffb::dg;

extern "C" {

size_t mmffb_dg_scratch_bytes(const MMFFDGBatchDev *batch, const MMFFDGParams *params) {
    if (check(batch, params)) return 0;
    if (batch->n_conf == 0) return kCounterBytes;
    int nt = 0, grid = 0;
    size_t smem = 0;
    if (plan_grid(batch, params, &nt, &smem, &grid)) return 0;
    return kCounterBytes + (size_t)grid * 2 * params->lbfgs_m * batch->max_atoms * sizeof(float4);
}

int mmffb_dg_minimize(const MMFFDGBatchDev *batch, const MMFFDGParams *params, float *pos, float *energies,
                      int32_t *statuses, int32_t *iters, void *scratch, size_t scratch_bytes, mmffb_stream_t stream) {
    int r = check(batch, params);
    if (r) return r;
    if (batch->n_conf == 0) return 0;
    if (!pos || !energies || !statuses) return fail(MMFFB_EINVAL, "null output pointer");
    int nt = 0, grid = 0;
    size_t smem = 0;
    r = plan_grid(batch, params, &nt, &smem, &grid);
    if (r) return r;
    const size_t need = kCounterBytes + (size_t)grid * 2 * params->lbfgs_m * batch->max_atoms * sizeof(float4);
    if (!scratch || scratch_bytes < need)
        return fail(MMFFB_ESCRATCH, "DG scratch of %zu B given, %zu B needed", scratch_bytes, need);
    Args a;
    a.b = *batch;
    a.p = *params;
    a.pos = pos;
    a.energy = energies;
    a.status = statuses;
    a.iters = iters;
    a.grad_out = nullptr;
    a.counter = reinterpret_cast<int *>(scratch);
    a.hist = reinterpret_cast<float4 *>(reinterpret_cast<char *>(scratch) + kCounterBytes);
    a.slot_atoms = batch->max_atoms;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(a.counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(DG counter)");
    switch (nt) {
        case 32: dg_minimize_kernel<32><<<grid, 32, smem, st>>>(a); break;
        case 64: dg_minimize_kernel<64><<<grid, 64, smem, st>>>(a); break;
        case 128: dg_minimize_kernel<128><<<grid, 128, smem, st>>>(a); break;
        default: dg_minimize_kernel<256><<<grid, 256, smem, st>>>(a); break;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "dg_minimize_kernel launch");
    return 0;
}

int mmffb_dg_energy_grad(const MMFFDGBatchDev *batch, const MMFFDGParams *params, const float *pos, float *energies,
                         float *grad, mmffb_stream_t stream) {
    int r = check(batch, params);
    if (r) return r;
    if (batch->n_conf == 0) return 0;
    if (!pos || !energies || !grad) return fail(MMFFB_EINVAL, "null argument");
    const int nt = pick_threads(batch->max_atoms, params->threads);
    const size_t smem = smem_bytes(nt, batch->max_atoms, 2);
    Args a;
    a.b = *batch;
    a.p = *params;
    a.pos = const_cast<float *>(pos);
    a.energy = energies;
    a.status = nullptr;
    a.iters = nullptr;
    a.grad_out = grad;
    a.hist = nullptr;
    a.counter = nullptr;
    a.slot_atoms = batch->max_atoms;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    switch (nt) {
        case 32:
            e = cudaFuncSetAttribute(dg_energy_grad_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e == cudaSuccess) dg_energy_grad_kernel<32><<<batch->n_conf, 32, smem, st>>>(a);
            break;
        case 64:
            e = cudaFuncSetAttribute(dg_energy_grad_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e == cudaSuccess) dg_energy_grad_kernel<64><<<batch->n_conf, 64, smem, st>>>(a);
            break;
        case 128:
            e = cudaFuncSetAttribute(dg_energy_grad_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e == cudaSuccess) dg_energy_grad_kernel<128><<<batch->n_conf, 128, smem, st>>>(a);
            break;
        default:
            e = cudaFuncSetAttribute(dg_energy_grad_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e == cudaSuccess) dg_energy_grad_kernel<256><<<batch->n_conf, 256, smem, st>>>(a);
            break;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(DG energy)");
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "dg_energy_grad_kernel launch");
    return 0;
}

}  // extern "C"
