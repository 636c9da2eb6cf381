// Two non-BFGS paths behind the C ABI:
//
// * plain_kernel -- the reference's in-kernel optimizer design restated in
//   CUDA (mlxmolkit/mmff_bfgs_source_tg.metal:1-372): one 32-thread CTA per
//   conformer, the full energy + gradient computed serially by thread 0,
//   energy-only line-search evaluations 32-wide, every vector and the dense
//   inverse Hessian in global memory, FP32 throughout, one launch for the
//   whole batch.  It is kept as the measured "plain one-launch-per-batch FP32
//   GPU path" the optimized kernel is compared against.
// * fused_sd_kernel -- the reference's fused optimizer
//   (mlxmolkit/mmff_metal_kernel.py:792-1076): Barzilai-Borwein steepest
//   descent with the +1 kcal/mol energy guard and a per-atom step cap, for
//   mmff_optimize_metal_fused_multi_mol; one CTA per conformer with the
//   parallel term evaluation of the optimizer kernel.
#include <cstring>

#include "mmff_kernels.cuh"

namespace mmffb {

// ---------------------------------------------------------------------------
// plain (reference-design) kernel
// ---------------------------------------------------------------------------

struct PlainParams {
    Params P;
    float *work;       // 6 vectors of stride nvs per conformer
    float *hess;       // (3*nmax)^2 per conformer
    size_t nvs, hs;
};

// serial energy + gradient by one thread (grad zeroed first), positions in global memory
__device__ float plain_eg_serial(const Params &P, const MolV &m, const float *x, float *g) {
    const int N = m.n;
    for (int k = 0; k < 3 * N; ++k) g[k] = 0.0f;
    float E = 0.0f;
    const uint4 *BR = reinterpret_cast<const uint4 *>(P.b.bonded);
    const TermMode md = P.md;
    for (int c = 0; c < m.bnch; ++c)
        for (int l = 0; l < 32; ++l) {
            uint4 r = BR[m.boff + (size_t)c * 32 + l];
            if (r.x == 0xffffffffu) continue;
            int i = r.x & 0xffff, j = r.x >> 16;
            float f[2][3];
            E += bond_term<float, true>(x + 3 * i, x + 3 * j, u2f(r.y), u2f(r.z), f);
            add3(g + 3 * i, f[0]); add3(g + 3 * j, f[1]);
        }
    for (int c = 0; c < m.anch; ++c)
        for (int l = 0; l < 32; ++l) {
            uint4 r = BR[m.aoff + (size_t)c * 32 + l];
            if (r.x == 0xffffffffu) continue;
            int i = r.x & 0xffff, j = r.x >> 16, k = r.y & 0xffff;
            float f[3][3];
            E += angle_term<float, true>(x + 3 * i, x + 3 * j, x + 3 * k, u2f(r.z), u2f(r.w), (r.y >> 16) != 0, md, f);
            add3(g + 3 * i, f[0]); add3(g + 3 * j, f[1]); add3(g + 3 * k, f[2]);
        }
    for (int c = 0; c < m.snch; ++c)
        for (int l = 0; l < 32; ++l) {
            uint4 r0 = BR[m.soff + (size_t)c * 64 + l], r1 = BR[m.soff + (size_t)c * 64 + 32 + l];
            if (r0.x == 0xffffffffu) continue;
            int i = r0.x & 0xffff, j = r0.x >> 16, k = (int)r0.y;
            float f[3][3];
            E += strbend_term<float, true>(x + 3 * i, x + 3 * j, x + 3 * k, u2f(r0.z), u2f(r0.w), u2f(r1.x),
                                           u2f(r1.y), u2f(r1.z), md, f);
            add3(g + 3 * i, f[0]); add3(g + 3 * j, f[1]); add3(g + 3 * k, f[2]);
        }
    for (int c = 0; c < m.onch; ++c)
        for (int l = 0; l < 32; ++l) {
            uint4 r = BR[m.ooff + (size_t)c * 32 + l];
            if (r.x == 0xffffffffu) continue;
            int i = r.x & 0xffff, j = r.x >> 16, k = r.y & 0xffff, q = r.y >> 16;
            float f[4][3];
            E += oop_term<float, true>(x + 3 * i, x + 3 * j, x + 3 * k, x + 3 * q, u2f(r.z), md, f);
            add3(g + 3 * i, f[0]); add3(g + 3 * j, f[1]); add3(g + 3 * k, f[2]); add3(g + 3 * q, f[3]);
        }
    for (int c = 0; c < m.tnch; ++c)
        for (int l = 0; l < 32; ++l) {
            uint4 r0 = BR[m.toff + (size_t)c * 64 + l], r1 = BR[m.toff + (size_t)c * 64 + 32 + l];
            if (r0.x == 0xffffffffu) continue;
            int i = r0.x & 0xffff, j = r0.x >> 16, k = r0.y & 0xffff, q = r0.y >> 16;
            float f[4][3];
            E += torsion_term<float, true>(x + 3 * i, x + 3 * j, x + 3 * k, x + 3 * q, u2f(r0.z), u2f(r0.w),
                                           u2f(r1.x), f);
            add3(g + 3 * i, f[0]); add3(g + 3 * j, f[1]); add3(g + 3 * k, f[2]); add3(g + 3 * q, f[3]);
        }
    const int W = (N + 31) >> 5;
    const uint32_t *pm = P.b.pair_mask + m.mask_off, *p14 = pm + (size_t)N * W;
    const float2 *tab = reinterpret_cast<const float2 *>(P.b.cls_tab) + m.cls_off;
    const int *cls = P.b.atom_cls + m.atom_off;
    const double *qa = P.b.atom_q + m.atom_off;
    for (int i = 0; i < N - 1; ++i)
        for (int j = i + 1; j < N; ++j) {
            if (!((pm[(size_t)i * W + (j >> 5)] >> (j & 31)) & 1u)) continue;
            float2 t = tab[cls[i] * m.ncls + cls[j]];
            float qq = (float)(qa[i] * qa[j]);
            if ((p14[(size_t)i * W + (j >> 5)] >> (j & 31)) & 1u) qq *= 0.75f;
            float dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
            float ev, ee, s;
            pair_term<float, true>(dx, dy, dz, t.x, t.y, qq, m.diel == 2, ev, ee, s);
            E += ev;
            E += ee;
            g[3 * i] += s * dx; g[3 * i + 1] += s * dy; g[3 * i + 2] += s * dz;
            g[3 * j] -= s * dx; g[3 * j + 1] -= s * dy; g[3 * j + 2] -= s * dz;
        }
    return E;
}

// 32-wide energy: lanes stride over the terms, tree-free warp reduction
__device__ float plain_energy(const Params &P, const MolV &m, const float *x) {
    const int lane = threadIdx.x & 31;
    float e = 0.0f;
    const uint4 *BR = reinterpret_cast<const uint4 *>(P.b.bonded);
    const TermMode md = P.md;
    float f2[2][3], f3[3][3], f4[4][3];
    for (int c = 0; c < m.bnch; ++c) {
        uint4 r = BR[m.boff + (size_t)c * 32 + lane];
        if (r.x != 0xffffffffu)
            e += bond_term<float, false>(x + 3 * (r.x & 0xffff), x + 3 * (r.x >> 16), u2f(r.y), u2f(r.z), f2);
    }
    for (int c = 0; c < m.anch; ++c) {
        uint4 r = BR[m.aoff + (size_t)c * 32 + lane];
        if (r.x != 0xffffffffu)
            e += angle_term<float, false>(x + 3 * (r.x & 0xffff), x + 3 * (r.x >> 16), x + 3 * (r.y & 0xffff),
                                          u2f(r.z), u2f(r.w), (r.y >> 16) != 0, md, f3);
    }
    for (int c = 0; c < m.snch; ++c) {
        uint4 r0 = BR[m.soff + (size_t)c * 64 + lane], r1 = BR[m.soff + (size_t)c * 64 + 32 + lane];
        if (r0.x != 0xffffffffu)
            e += strbend_term<float, false>(x + 3 * (r0.x & 0xffff), x + 3 * (r0.x >> 16), x + 3 * (int)r0.y,
                                            u2f(r0.z), u2f(r0.w), u2f(r1.x), u2f(r1.y), u2f(r1.z), md, f3);
    }
    for (int c = 0; c < m.onch; ++c) {
        uint4 r = BR[m.ooff + (size_t)c * 32 + lane];
        if (r.x != 0xffffffffu)
            e += oop_term<float, false>(x + 3 * (r.x & 0xffff), x + 3 * (r.x >> 16), x + 3 * (r.y & 0xffff),
                                        x + 3 * (r.y >> 16), u2f(r.z), md, f4);
    }
    for (int c = 0; c < m.tnch; ++c) {
        uint4 r0 = BR[m.toff + (size_t)c * 64 + lane], r1 = BR[m.toff + (size_t)c * 64 + 32 + lane];
        if (r0.x != 0xffffffffu)
            e += torsion_term<float, false>(x + 3 * (r0.x & 0xffff), x + 3 * (r0.x >> 16), x + 3 * (r0.y & 0xffff),
                                            x + 3 * (r0.y >> 16), u2f(r0.z), u2f(r0.w), u2f(r1.x), f4);
    }
    const int N = m.n, W = (N + 31) >> 5;
    const uint32_t *pm = P.b.pair_mask + m.mask_off, *p14 = pm + (size_t)N * W;
    const float2 *tab = reinterpret_cast<const float2 *>(P.b.cls_tab) + m.cls_off;
    const int *cls = P.b.atom_cls + m.atom_off;
    const double *qa = P.b.atom_q + m.atom_off;
    for (int i = 0; i < N - 1; ++i)
        for (int jb = (i + 1) & ~31; jb < N; jb += 32) {
            const int j = jb + lane;
            if (!((pm[(size_t)i * W + (jb >> 5)] >> lane) & 1u)) continue;
            float2 t = tab[cls[i] * m.ncls + cls[j]];
            float qq = (float)(qa[i] * qa[j]);
            if ((p14[(size_t)i * W + (jb >> 5)] >> lane) & 1u) qq *= 0.75f;
            float dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
            float ev, ee, s;
            pair_term<float, false>(dx, dy, dz, t.x, t.y, qq, m.diel == 2, ev, ee, s);
            e += ev;
            e += ee;
        }
    return wsum(e);
}

__global__ void __launch_bounds__(32) plain_kernel(const PlainParams Q) {
    const Params &P = Q.P;
    const int conf = blockIdx.x, lane = threadIdx.x;
    if (conf >= P.c.n_conf) return;
    const KConst &K = P.K;
    const MolV m = load_mol(P.b.mol_desc, P.c.conf_mol[conf]);
    const int n = 3 * m.n;
    float *x = P.pos + P.c.conf_coord[conf];
    float *w = Q.work + (size_t)conf * 6 * Q.nvs;
    float *g = w, *dir = w + Q.nvs, *xo = w + 2 * Q.nvs, *dg = w + 3 * Q.nvs, *hdg = w + 4 * Q.nvs;
    float *H = Q.hess + (size_t)conf * Q.hs;
    for (size_t e = lane; e < (size_t)n * n; e += 32) H[e] = (e / n == e % n) ? 1.0f : 0.0f;
    __syncwarp();
    __shared__ float s_gs;
    if (lane == 0) {
        plain_eg_serial(P, m, x, g);
        float s = (float)K.gscale, mx = 0.0f;
        for (int k = 0; k < n; ++k) { g[k] *= s; mx = fmaxf(mx, fabsf(g[k])); }
        for (int h = 0; h < 256 && mx > (float)K.gcap; ++h) {
            s *= 0.5f; mx = 0.0f;
            for (int k = 0; k < n; ++k) { g[k] *= 0.5f; mx = fmaxf(mx, fabsf(g[k])); }
        }
        s_gs = s;
    }
    __syncwarp();
    float E = plain_energy(P, m, x);
    for (int k = lane; k < n; k += 32) dir[k] = -g[k];
    float ss = 0.0f;
    for (int k = lane; k < n; k += 32) ss += x[k] * x[k];
    const float max_step = (float)K.maxstep * fmaxf(sqrtf(wsum(ss)), (float)n);
    __syncwarp();
    int status = MMFFB_ST_MAXIT, it;
    for (it = 0; it < P.max_iters; ++it) {
        for (int k = lane; k < n; k += 32) xo[k] = x[k];
        float dn = 0.0f;
        for (int k = lane; k < n; k += 32) dn += dir[k] * dir[k];
        dn = sqrtf(wsum(dn));
        if (dn > max_step) {
            const float sc = max_step / dn;
            for (int k = lane; k < n; k += 32) dir[k] *= sc;
        }
        __syncwarp();
        float slope = 0.0f, tm = 0.0f;
        for (int k = lane; k < n; k += 32) {
            slope += dir[k] * g[k];
            tm = fmaxf(tm, fabsf(dir[k]) / fmaxf(fabsf(x[k]), 1.0f));
        }
        slope = wsum(slope);
        tm = wmax(tm);
        if (slope >= 0.0f) { status = MMFFB_ST_SLOPE; break; }
        const float lam_min = (float)K.movetol / fmaxf(tm, 1e-30f);
        float lam = 1.0f, plam = 1.0f, pe = E;
        const float Eold = E;
        bool ok = false;
        for (int ls = 0; ls < K.maxls && !ok; ++ls) {
            if (lam < lam_min) break;
            for (int k = lane; k < n; k += 32) x[k] = xo[k] + lam * dir[k];
            __syncwarp();
            const float et = plain_energy(P, m, x);
            if (et - Eold <= (float)K.functol * lam * slope) { E = et; ok = true; break; }
            float tl;
            if (ls == 0) tl = -slope / (2.0f * (et - Eold - slope));
            else {
                const float r1 = et - Eold - lam * slope, r2 = pe - Eold - plam * slope;
                const float l2 = lam * lam, p2 = plam * plam, dv = lam - plam;
                if (fabsf(dv) < 1e-30f) tl = 0.5f * lam;
                else {
                    const float a = (r1 / l2 - r2 / p2) / dv, b = (-plam * r1 / l2 + lam * r2 / p2) / dv;
                    if (fabsf(a) < 1e-30f) tl = fabsf(b) > 1e-30f ? -slope / (2.0f * b) : 0.5f * lam;
                    else {
                        const float disc = b * b - 3.0f * a * slope;
                        if (disc < 0.0f) tl = 0.5f * lam;
                        else if (b <= 0.0f) tl = (-b + sqrtf(disc)) / (3.0f * a);
                        else tl = -slope / (b + sqrtf(disc));
                    }
                }
            }
            tl = fminf(tl, 0.5f * lam);
            tl = fmaxf(tl, 0.1f * lam);
            plam = lam; pe = et; lam = tl;
        }
        if (!ok) {
            for (int k = lane; k < n; k += 32) x[k] = xo[k];
            __syncwarp();
        }
        float tx = 0.0f;
        for (int k = lane; k < n; k += 32) {
            xo[k] = x[k] - xo[k];
            tx = fmaxf(tx, fabsf(xo[k]) / fmaxf(fabsf(x[k]), 1.0f));
        }
        if (wmax(tx) < (float)K.tolx) { status = ok ? MMFFB_ST_TOLX : MMFFB_ST_LSFAIL; break; }
        for (int k = lane; k < n; k += 32) dg[k] = g[k];
        __syncwarp();
        if (lane == 0) {
            plain_eg_serial(P, m, x, g);
            float s = s_gs, mx = 0.0f;
            for (int k = 0; k < n; ++k) { g[k] *= s; mx = fmaxf(mx, fabsf(g[k])); }
            for (int h = 0; h < 256 && mx > (float)K.gcap; ++h) {
                s *= 0.5f; mx = 0.0f;
                for (int k = 0; k < n; ++k) { g[k] *= 0.5f; mx = fmaxf(mx, fabsf(g[k])); }
            }
            s_gs = s;
        }
        __syncwarp();
        float gt = 0.0f;
        for (int k = lane; k < n; k += 32) {
            dg[k] = g[k] - dg[k];
            gt = fmaxf(gt, fabsf(g[k]) * fmaxf(fabsf(x[k]), 1.0f));
        }
        if (wmax(gt) / fmaxf(E * s_gs, 1.0f) < P.grad_tol) { status = MMFFB_ST_GRAD; break; }
        __syncwarp();
        for (int i = 0; i < n; ++i) {          // H dg: one row at a time, lanes over columns
            float s = 0.0f;
            for (int j = lane; j < n; j += 32) s += H[(size_t)i * n + j] * dg[j];
            s = wsum(s);
            if (lane == 0) hdg[i] = s;
        }
        __syncwarp();
        float fac = 0, fae = 0, sdg = 0, sxi = 0;
        for (int k = lane; k < n; k += 32) {
            fac += dg[k] * xo[k]; fae += dg[k] * hdg[k]; sdg += dg[k] * dg[k]; sxi += xo[k] * xo[k];
        }
        fac = wsum(fac); fae = wsum(fae); sdg = wsum(sdg); sxi = wsum(sxi);
        if (fac * fac > (float)K.eps * sdg * sxi && fac > 0.0f) {
            const float fi = 1.0f / fac, fei = 1.0f / fae;
            for (size_t e = lane; e < (size_t)n * n; e += 32) {
                const int i = (int)(e / n), j = (int)(e % n);
                const float ai = fi * xo[i] - fei * hdg[i], aj = fi * xo[j] - fei * hdg[j];
                H[e] += fi * xo[i] * xo[j] - fei * hdg[i] * hdg[j] + fae * ai * aj;
            }
            __syncwarp();
        }
        for (int i = 0; i < n; ++i) {          // -H g, same coalesced order
            float s = 0.0f;
            for (int j = lane; j < n; j += 32) s += H[(size_t)i * n + j] * g[j];
            s = wsum(s);
            if (lane == 0) dir[i] = -s;
        }
        __syncwarp();
    }
    if (lane == 0) {
        P.energy[conf] = (double)E;
        P.status[conf] = status;
        P.iters[conf] = it < P.max_iters ? it + (status == MMFFB_ST_SLOPE ? 0 : 1) : P.max_iters;
    }
}

// ---------------------------------------------------------------------------
// fused Barzilai-Borwein steepest descent
// ---------------------------------------------------------------------------

template <int NT>
__global__ void __launch_bounds__(NT) fused_sd_kernel(const Params P, float max_step, float grad_lr) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int NW = NT / 32;
    using R = float;
    using A = double;
    const int conf = blockIdx.x, tid = threadIdx.x;
    Layout L = make_layout(P.nmax, NW, 0, false, sizeof(R), sizeof(A), P.b.max_classes);
    R *pos4 = (R *)(smem + L.pos4), *x = (R *)(smem + L.x), *g = (R *)(smem + L.g);
    R *pp = (R *)(smem + L.xo), *pg = (R *)(smem + L.dg), *gbuf = (R *)(smem + L.gbuf);
    int *cls = (int *)(smem + L.cls);
    double *qa = (double *)(smem + L.q);
    float *qf = (float *)(smem + L.qf);
    uint32_t *mask = (uint32_t *)(smem + L.mask);
    float2 *tab = (float2 *)(smem + L.tab);
    A *red = (A *)(smem + L.red);
    int rsel = 0;
    const MolV m = load_mol(P.b.mol_desc, P.c.conf_mol[conf]);
    const int N = m.n, n = 3 * N, nv = (3 * P.nmax + 3) & ~3;
    const float *gp = P.pos + P.c.conf_coord[conf];
    for (int k = tid; k < n; k += NT) {
        R v = gp[k];
        x[k] = v; pp[k] = v; pg[k] = R(0);
        pos4[4 * (k / 3) + (k % 3)] = v;
    }
    stage_molecule<NT>(P, m, cls, qa, qf, mask, tab);
    const MolSmem ms{cls, qa, qf, mask, tab};
    __syncthreads();
    R alpha = grad_lr;
    A E = A(0), Eprev = A(1e30);
    for (int it = 0; it < P.max_iters; ++it) {
        A e1[1] = {eval_terms<R, A, NW, true>(P, m, pos4, gbuf, ms, nv)}, z[1] = {A(0)};
        __syncthreads();
        for (int k = tid; k < n; k += NT) {
            R s = R(0);
#pragma unroll
            for (int w = 0; w < NW; ++w) s += gbuf[(size_t)w * nv + k];
            g[k] = s;
        }
        block_reduce<NW, 1, 1, A>(e1, z, red + rsel * NW * 8);
        rsel ^= 1;
        E = (A)(float)e1[0];
        if (it > 0 && E > Eprev + A(1)) {
            // energy guard: revert, halve the step, keep the previous energy
            for (int k = tid; k < n; k += NT) { x[k] = pp[k]; pos4[4 * (k / 3) + (k % 3)] = pp[k]; }
            alpha = fmaxf(alpha * 0.5f, 1e-7f);
            E = Eprev;
            __syncthreads();
            continue;
        }
        if (it > 0) {
            A s2[2] = {A(0), A(0)}, z2[1] = {A(0)};
            for (int k = tid; k < n; k += NT) {
                const R si = x[k] - pp[k], yi = g[k] - pg[k];
                s2[0] += (A)(si * si);
                s2[1] += (A)(si * yi);
            }
            block_reduce<NW, 2, 1, A>(s2, z2, red + rsel * NW * 8);
            rsel ^= 1;
            if (s2[1] > A(1e-20)) alpha = fminf(fmaxf((float)(s2[0] / s2[1]), 1e-6f), 0.3f);
        }
        Eprev = E;
        for (int k = tid; k < n; k += NT) { pp[k] = x[k]; pg[k] = g[k]; }
        __syncthreads();
        for (int a = tid; a < N; a += NT) {
            const R gx = g[3 * a], gy = g[3 * a + 1], gz = g[3 * a + 2];
            const R gn = sqrtf(gx * gx + gy * gy + gz * gz + 1e-30f);
            const R s = fminf(max_step / gn, alpha);
            x[3 * a] -= s * gx; x[3 * a + 1] -= s * gy; x[3 * a + 2] -= s * gz;
            pos4[4 * a] = x[3 * a]; pos4[4 * a + 1] = x[3 * a + 1]; pos4[4 * a + 2] = x[3 * a + 2];
        }
        __syncthreads();
    }
    float *op = P.pos + P.c.conf_coord[conf];
    for (int k = tid; k < n; k += NT) op[k] = x[k];
    if (tid == 0) P.energy[conf] = E;
}

static int check_common(const MMFFBatchDev *b, const MMFFConfDev *c) {
    if (!b || !c) return fail(MMFFB_EINVAL, "null batch or conformer descriptor");
    if (c->n_conf > 0 && (!b->mol_desc || !b->bonded || !b->atom_cls || !b->atom_q || !b->cls_tab ||
                          !b->pair_mask || !c->conf_mol || !c->conf_coord))
        return fail(MMFFB_EINVAL, "null device pointer in batch");
    if (c->n_conf > 0 && (c->max_atoms <= 0 || c->max_atoms > 1024))
        return fail(MMFFB_EINVAL, "max_atoms out of range");
    if (b->max_classes < 1 || b->max_classes > 64) return fail(MMFFB_EINVAL, "max_classes out of range");
    return 0;
}

}  // namespace mmffb

using namespace mmffb;

extern "C" {

size_t mmffb_plain_scratch_bytes(const MMFFBatchDev *batch, const MMFFConfDev *confs) {
    if (check_common(batch, confs)) return 0;
    const size_t n = 3 * (size_t)confs->max_atoms;
    return (size_t)confs->n_conf * (6 * n + n * n) * sizeof(float);
}

int mmffb_plain_minimize(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                         float *pos, double *energy, int32_t *status, int32_t *iters,
                         void *scratch, size_t scratch_bytes, mmffb_stream_t stream) {
    int r = check_common(batch, confs);
    if (r) return r;
    if (!opt || !pos || !energy || !status || !iters) return fail(MMFFB_EINVAL, "null argument");
    if (opt->history_m != 0) return fail(MMFFB_EINVAL, "the plain path is dense BFGS only");
    if (confs->n_conf == 0) return 0;
    const size_t need = mmffb_plain_scratch_bytes(batch, confs);
    if (!scratch || scratch_bytes < need)
        return fail(MMFFB_ESCRATCH, "scratch of %zu B given, %zu B needed", scratch_bytes, need);
    PlainParams Q;
    memset(&Q, 0, sizeof Q);
    Q.P.b = *batch;
    Q.P.c = *confs;
    Q.P.md.cb = opt->mode[0]; Q.P.md.kang = opt->mode[1]; Q.P.md.ksbg = opt->mode[2]; Q.P.md.lin = opt->mode[3] != 0.0;
    Q.P.K.tolx = opt->consts[0]; Q.P.K.functol = opt->consts[1]; Q.P.K.movetol = opt->consts[2];
    Q.P.K.eps = opt->consts[3]; Q.P.K.maxstep = opt->consts[4]; Q.P.K.maxls = (int)opt->consts[5];
    Q.P.K.gscale = opt->consts[6]; Q.P.K.gcap = opt->consts[7];
    Q.P.max_iters = opt->max_iters;
    Q.P.grad_tol = opt->grad_tol;
    Q.P.nmax = confs->max_atoms;
    Q.P.pos = pos;
    Q.P.energy = energy;
    Q.P.status = status;
    Q.P.iters = iters;
    const size_t nvec = 3 * (size_t)confs->max_atoms;
    Q.nvs = nvec;
    Q.hs = nvec * nvec;
    Q.work = reinterpret_cast<float *>(scratch);
    Q.hess = Q.work + (size_t)confs->n_conf * 6 * nvec;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    plain_kernel<<<confs->n_conf, 32, 0, st>>>(Q);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "plain_kernel launch");
    return 0;
}

int mmffb_fused_sd(const MMFFBatchDev *batch, const MMFFConfDev *confs, const MMFFOptParams *opt,
                   const float *sd, float *pos, double *energy, mmffb_stream_t stream) {
    int r = check_common(batch, confs);
    if (r) return r;
    if (!opt || !sd || !pos || !energy) return fail(MMFFB_EINVAL, "null argument");
    if (opt->max_iters < 0) return fail(MMFFB_EINVAL, "max_iters must be >= 0");
    if (confs->n_conf == 0) return 0;
    Params P;
    memset(&P, 0, sizeof P);
    P.b = *batch;
    P.c = *confs;
    P.md.cb = opt->mode[0]; P.md.kang = opt->mode[1]; P.md.ksbg = opt->mode[2]; P.md.lin = opt->mode[3] != 0.0;
    P.max_iters = opt->max_iters;
    P.nmax = confs->max_atoms;
    P.pos = pos;
    P.energy = energy;
    constexpr int NT = 128;
    Layout L = make_layout(P.nmax, NT / 32, 0, false, 4, 8, batch->max_classes);
    auto k = fused_sd_kernel<NT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k<<<confs->n_conf, NT, L.total, st>>>(P, sd[0], sd[1]);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "fused_sd_kernel launch");
    return 0;
}

}  // extern "C"
