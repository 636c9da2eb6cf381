#pragma once
// B200 (sm_100a) kernels of the batched MMFF94/94s conformer optimizer.
//
// Work unit: one conformer, owned by one CTA for its whole optimisation.
// A persistent grid pulls conformers from a global work counter (largest
// first), so a conformer that converges early frees its CTA for the next
// one instead of idling until the slowest member of a lockstep batch ends.
//
// Per conformer, shared memory holds the coordinates (float4 per atom), the
// optimizer vectors, per-warp gradient buffers, per-atom non-bonded class and
// charge, and -- when it fits -- the dense inverse Hessian (or the L-BFGS
// history); otherwise the matrix lives in a per-CTA global slot that stays
// resident in the 126 MB L2.
//
// Energy / gradient:
//  * bonded terms arrive in chunks of 32 records; inside a chunk no two terms
//    share an atom in the same role, so each role's gradient scatter is a
//    plain conflict-free read-modify-write into the warp's private buffer;
//  * non-bonded pairs are not read from a pair table: warp w walks rows i of
//    the upper triangle, lanes take j, a bit row marks the non-bonded pairs
//    (topological distance >= 3) and the 1-4 pairs, (R*, eps) comes from the
//    molecule's class x class table and q_i q_j from per-atom charges;
//  * the gradient is the fixed-order sum of the per-warp buffers and the
//    energy a fixed-order FP64 (mixed precision) reduction, so results are
//    bit-reproducible run to run.
//
// Dense BFGS: the rank-2 inverse-Hessian update of iteration k is applied
// lazily inside iteration k+1's single pass over H, which also forms both
// matrix-vector products (H g and H dg): one read and one write of H per
// iteration.  The direction -H_{k+1} g follows from H_k g and vector terms.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "mmff_terms.cuh"
#include "mmffb200.h"

namespace mmffb {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *where);

constexpr int kMaxHist = 16;       // L-BFGS history pairs supported
constexpr int kMaxAtoms = 1024;    // atom indices are packed as 16 bits; smem bounds this further

struct MolV {
    int n, atom_off, ncls, cls_off, mask_off, diel;
    int boff, bnch, aoff, anch, soff, snch, ooff, onch, toff, tnch;
};

// Data read once per conformer (descriptor, slot, coordinates, per-atom staging) is
// loaded through L2 (ld.global.cg): a serving worker reads slots that the host
// publishes while it runs, and L1 lines loaded for an earlier slot may hold the
// same lines' old contents.  The bonded records, read every evaluation, keep the
// read-only cache: each molecule's records start on a 512-byte boundary, so no
// line holds two molecules' records.
__device__ __forceinline__ MolV load_mol(const int32_t *desc, int m) {
    const int32_t *d = desc + (size_t)m * MMFFB_MOL_DESC_INTS;
    MolV v;
    v.n = __ldcg(d + MMFFB_MD_N); v.atom_off = __ldcg(d + MMFFB_MD_ATOM_OFF); v.ncls = __ldcg(d + MMFFB_MD_NCLS);
    v.cls_off = __ldcg(d + MMFFB_MD_CLS_OFF); v.mask_off = __ldcg(d + MMFFB_MD_MASK_OFF);
    v.diel = __ldcg(d + MMFFB_MD_DIEL);
    v.boff = __ldcg(d + MMFFB_MD_B_OFF); v.bnch = __ldcg(d + MMFFB_MD_B_NCH); v.aoff = __ldcg(d + MMFFB_MD_A_OFF);
    v.anch = __ldcg(d + MMFFB_MD_A_NCH); v.soff = __ldcg(d + MMFFB_MD_S_OFF); v.snch = __ldcg(d + MMFFB_MD_S_NCH);
    v.ooff = __ldcg(d + MMFFB_MD_O_OFF); v.onch = __ldcg(d + MMFFB_MD_O_NCH); v.toff = __ldcg(d + MMFFB_MD_T_OFF);
    v.tnch = __ldcg(d + MMFFB_MD_T_NCH);
    return v;
}

struct KConst {
    double tolx, functol, movetol, eps, maxstep, gscale, gcap;
    int maxls;
};

struct Params {
    MMFFBatchDev b;
    MMFFConfDev c;
    TermMode md;
    KConst K;
    int max_iters;
    int hist_m;
    float grad_tol;
    int exit_test;
    int check_every;
    float atom_grad_scale;
    int max_restarts;
    int polish64;      // mixed precision: FP64 line-search energies once the FP32 ones stall
    uint32_t wait_spins;   // tests of a ring stage's completion before its wait gives up (0: none)
    int32_t *ls_evals;
    int *err;          // set when a bounded wait gave up (never expected): the caller's word or scratch_err
    int *scratch_err;  // the scratch head's error word (byte 4), set as well
    int nmax;          // largest atom count of the launch (shared-memory layout)
    float *pos;
    double *energy;
    int32_t *status;
    int32_t *iters;
    void *gmat;        // per-CTA global matrix slots (when not in shared memory)
    size_t gslot;      // elements per slot
    int *counter;      // work counter
    // work queue of a serving worker (q_tail != nullptr): conformer slots are published by the
    // host while the launch runs (tail), claimed here (head) and flagged done in host memory
    int *q_head;
    const int *q_tail;
    const int *q_close;
    int *q_done;
    uint32_t q_idle_polls;
    uint32_t q_sleep_ns;
};

__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The next published conformer slot of a serving worker, or -1 once the queue is closed
// and drained, or after q_idle_polls empty polls (q_sleep_ns apart): bounded, never hangs.
__device__ __forceinline__ int claim_slot(const Params &P) {
    for (uint32_t polls = 0;; ++polls) {
        const int t = ld_acquire_gpu(P.q_tail);
        const int h = *(volatile int *)P.q_head;
        if (h < t) {
            if (atomicCAS(P.q_head, h, h + 1) == h) return h;
            continue;
        }
        if (ld_acquire_gpu(P.q_close)) return -1;
        if (polls >= P.q_idle_polls) return -1;
        __nanosleep(P.q_sleep_ns);
    }
}

__host__ __device__ __forceinline__ size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared-memory layout of one CTA (byte offsets).
constexpr int kStages = 4;         // rows of H in flight per warp (TMA ring)

struct Layout {
    size_t pos4, pos4d, x, g, dir, xo, dg, hp, hq, pxi, pc, pr, gbuf, cls, q, qf, mask, tab, red, rho, alpha,
        ring, mbar, mat, total;
};

// row stride of a dense inverse Hessian in global memory: 16-byte multiple for TMA rows
__host__ __device__ __forceinline__ int hld(int n) { return (n + 3) & ~3; }

__host__ __device__ inline Layout make_layout(int nmax, int nwarps, int hist_m, bool mat_in_smem,
                                              size_t rs, size_t as, int max_classes = 32) {
    Layout L;
    size_t nv = (size_t)((3 * nmax + 3) & ~3);
    size_t o = 0;
    L.pos4 = o; o = al16(o + 4 * (size_t)nmax * rs);
    L.pos4d = o; o = al16(o + (rs == 4 ? 4 * (size_t)nmax * 8 : 0));   // FP64 copy (mixed precision)
    L.x = o; o = al16(o + nv * rs);
    L.g = o; o = al16(o + nv * rs);
    L.dir = o; o = al16(o + nv * rs);
    L.xo = o; o = al16(o + nv * rs);
    L.dg = o; o = al16(o + nv * rs);
    L.hp = o; o = al16(o + nv * rs);
    L.hq = o; o = al16(o + nv * rs);
    L.pxi = o; o = al16(o + nv * rs);
    L.pc = o; o = al16(o + nv * rs);
    L.pr = o; o = al16(o + nv * rs);
    L.gbuf = o; o = al16(o + (size_t)nwarps * nv * rs);
    L.cls = o; o = al16(o + (size_t)nmax * 4);
    L.q = o; o = al16(o + (size_t)nmax * 8);
    L.qf = o; o = al16(o + (size_t)nmax * 4);
    L.mask = o; o = al16(o + 2 * (size_t)nmax * ((nmax + 31) / 32) * 4);
    L.tab = o; o = al16(o + (size_t)max_classes * max_classes * 8);
    L.red = o; o = al16(o + 2 * (size_t)nwarps * 8 * as);
    L.rho = o; o = al16(o + kMaxHist * as);
    L.alpha = o; o = al16(o + kMaxHist * as);
    L.ring = o;
    L.mbar = o;
    if (!mat_in_smem && hist_m == 0) {             // TMA row ring of the streamed H pass
        o = al16(o + (size_t)nwarps * kStages * hld(3 * nmax) * rs);
        L.mbar = o;
        o = al16(o + (size_t)nwarps * kStages * 8);
    }
    L.mat = o;
    if (mat_in_smem) {
        size_t me = hist_m > 0 ? 2 * (size_t)hist_m * nv : (size_t)(3 * nmax) * (size_t)(3 * nmax);
        o = al16(o + me * rs);
    }
    L.total = o;
    return L;
}

// Layout of the evaluation-only kernels (energy / gradient, FP64 check): coordinates,
// per-warp gradient buffers, staged molecule data and the reduction scratch -- none of
// the optimizer's vectors, so that FP64 evaluations of the largest molecules fit.
__host__ __device__ inline Layout make_eval_layout(int nmax, int nwarps, size_t rs, size_t as, int max_classes) {
    Layout L;
    memset(&L, 0, sizeof L);
    size_t nv = (size_t)((3 * nmax + 3) & ~3);
    size_t o = 0;
    L.pos4 = o; o = al16(o + 4 * (size_t)nmax * rs);
    L.gbuf = o; o = al16(o + (size_t)nwarps * nv * rs);
    L.cls = o; o = al16(o + (size_t)nmax * 4);
    L.q = o; o = al16(o + (size_t)nmax * 8);
    L.qf = o; o = al16(o + (size_t)nmax * 4);
    L.mask = o; o = al16(o + 2 * (size_t)nmax * ((nmax + 31) / 32) * 4);
    L.tab = o; o = al16(o + (size_t)max_classes * max_classes * 8);
    L.red = o; o = al16(o + 2 * (size_t)nwarps * 8 * as);
    L.total = o;
    return L;
}

__host__ __device__ inline size_t mat_elems(int nmax, int hist_m) {
    size_t nv = (size_t)((3 * nmax + 3) & ~3);
    return hist_m > 0 ? 2 * (size_t)hist_m * nv : (size_t)(3 * nmax) * (size_t)hld(3 * nmax);
}

// ---- TMA bulk copies and mbarriers (inline PTX) ----
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, uint32_t parity) {   // non-blocking
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// 1-D bulk copy global -> shared (no multicast), completion counted on the mbarrier
__device__ __forceinline__ void tma_load_row(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
constexpr uint32_t kMaxWaitSpins = 1u << 22;   // bounded waits: give up, flag, never hang (default)
constexpr uint32_t kDrainSpins = 1u << 22;     // bounded wait for copies still in flight after giving up

template <class R> __device__ __forceinline__ R qprod(double a, double b);
template <> __device__ __forceinline__ float qprod<float>(double a, double b) { return (float)(a * b); }
// the term lists carry q_i*q_j rounded to float32 (mmff_params.py:305,318); every precision uses it
template <> __device__ __forceinline__ double qprod<double>(double a, double b) { return (double)(float)(a * b); }

template <class T> __device__ __forceinline__ T wsum(T v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <class T> __device__ __forceinline__ T wmax(T v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) { T u = __shfl_xor_sync(0xffffffffu, v, o); v = u > v ? u : v; }
    return v;
}

// Block reduction of KS sums and KM maxima; every thread receives the results.
// One __syncthreads: the caller alternates between two scratch halves.
template <int NW, int KS, int KM, class A>
__device__ __forceinline__ void block_reduce(A (&s)[KS], A (&m)[KM], A *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < KS; ++k) s[k] = wsum(s[k]);
#pragma unroll
    for (int k = 0; k < KM; ++k) m[k] = wmax(m[k]);
    constexpr int K = KS + KM;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < KS; ++k) red[warp * K + k] = s[k];
#pragma unroll
        for (int k = 0; k < KM; ++k) red[warp * K + KS + k] = m[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KS; ++k) {
        A t = A(0);
#pragma unroll
        for (int w = 0; w < NW; ++w) t += red[w * K + k];
        s[k] = t;
    }
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        A t = red[KS + k];
#pragma unroll
        for (int w = 1; w < NW; ++w) { A u = red[w * K + KS + k]; t = u > t ? u : t; }
        m[k] = t;
    }
}

template <class R> __device__ __forceinline__ void add3(R *dst, const R *f) {
    dst[0] += f[0]; dst[1] += f[1]; dst[2] += f[2];
}

__device__ __forceinline__ float u2f(uint32_t u) { return __uint_as_float(u); }

// Per-conformer molecule data staged in shared memory.
struct MolSmem {
    const int *cls;        // non-bonded class per atom
    const double *qa;      // partial charge per atom (FP64)
    const float *qf;       // the same, float (FP32 pair math)
    const uint32_t *mask;  // N x W non-bonded-pair bit rows, then N x W 1-4 bit rows
    const float2 *tab;     // ncls x ncls (R*, eps)
};

template <class R> __device__ __forceinline__ void ld3(const R *p4, int a, R &x, R &y, R &z) {
    x = p4[4 * a]; y = p4[4 * a + 1]; z = p4[4 * a + 2];
}
template <> __device__ __forceinline__ void ld3<float>(const float *p4, int a, float &x, float &y, float &z) {
    const float4 v = reinterpret_cast<const float4 *>(p4)[a];
    x = v.x; y = v.y; z = v.z;
}

template <class R> __device__ __forceinline__ R pair_charge(const MolSmem &ms, int i, int j);
template <> __device__ __forceinline__ float pair_charge<float>(const MolSmem &ms, int i, int j) {
    return ms.qf[i] * ms.qf[j];
}
template <> __device__ __forceinline__ double pair_charge<double>(const MolSmem &ms, int i, int j) {
    return qprod<double>(ms.qa[i], ms.qa[j]);
}

// Copy a molecule's bit rows, class table, classes and charges into shared memory.
// IR (the FP32 instances): stage 1/R* in place of R*, the pair term's only use of R*.
template <int NT, bool IR = false>
__device__ __forceinline__ void stage_molecule(const Params &P, const MolV &m, int *cls, double *qa, float *qf,
                                               uint32_t *mask, float2 *tab) {
    const int N = m.n, W = (N + 31) >> 5;
    for (int a = threadIdx.x; a < N; a += NT) {
        cls[a] = __ldcg(P.b.atom_cls + m.atom_off + a);
        const double q = __ldcg(P.b.atom_q + m.atom_off + a);
        qa[a] = q;
        qf[a] = (float)q;
    }
    const uint32_t *gm = P.b.pair_mask + m.mask_off;
    for (int k = threadIdx.x; k < 2 * N * W; k += NT) mask[k] = __ldcg(gm + k);
    const float2 *gt = reinterpret_cast<const float2 *>(P.b.cls_tab) + m.cls_off;
    for (int k = threadIdx.x; k < m.ncls * m.ncls; k += NT) {
        float2 v = __ldcg(gt + k);
        if (IR) v.x = Num<float>::rcp(v.x > 1e-8f ? v.x : 1e-8f);
        tab[k] = v;
    }
}

// Energy (thread partial, not reduced) and -- if G -- per-warp gradient buffers.
// pos4: smem float4-strided coordinates; gbuf: NW x nv.  IRTAB: the staged class
// table holds 1/R* (see stage_molecule).
template <class R, class A, int NW, bool G, bool IRTAB = false>
__device__ __forceinline__ A eval_terms(const Params &P, const MolV &m, const R *pos4, R *gbuf,
                                        const MolSmem &ms, int nv) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int N = m.n;
    A acc = A(0);
    R *gw = gbuf + (size_t)warp * nv;
    if (G) {
        for (int k = lane; k < 3 * N; k += 32) gw[k] = R(0);
        __syncwarp();
    }
    const uint4 *BR = reinterpret_cast<const uint4 *>(P.b.bonded);
    const TermMode md = P.md;

    for (int c = warp; c < m.bnch; c += NW) {
        uint4 r = __ldg(BR + m.boff + (size_t)c * 32 + lane);
        bool v = r.x != 0xffffffffu;
        int i = r.x & 0xffff, j = r.x >> 16;
        R f[2][3];
        if (v) acc += (A)bond_term<R, G>(pos4 + 4 * i, pos4 + 4 * j, (R)u2f(r.y), (R)u2f(r.z), f);
        if (G) {
            if (v) add3(gw + 3 * i, f[0]);
            __syncwarp();
            if (v) add3(gw + 3 * j, f[1]);
            __syncwarp();
        }
    }
    for (int c = warp; c < m.anch; c += NW) {
        uint4 r = __ldg(BR + m.aoff + (size_t)c * 32 + lane);
        bool v = r.x != 0xffffffffu;
        int i = r.x & 0xffff, j = r.x >> 16, k = r.y & 0xffff;
        bool lin = (r.y >> 16) != 0;
        R f[3][3];
        if (v)
            acc += (A)angle_term<R, G>(pos4 + 4 * i, pos4 + 4 * j, pos4 + 4 * k, (R)u2f(r.z), (R)u2f(r.w),
                                       lin, md, f);
        if (G) {
            if (v) add3(gw + 3 * i, f[0]);
            __syncwarp();
            if (v) add3(gw + 3 * j, f[1]);
            __syncwarp();
            if (v) add3(gw + 3 * k, f[2]);
            __syncwarp();
        }
    }
    for (int c = warp; c < m.snch; c += NW) {
        uint4 r0 = __ldg(BR + m.soff + (size_t)c * 64 + lane);
        uint4 r1 = __ldg(BR + m.soff + (size_t)c * 64 + 32 + lane);
        bool v = r0.x != 0xffffffffu;
        int i = r0.x & 0xffff, j = r0.x >> 16, k = (int)r0.y;
        R f[3][3];
        if (v)
            acc += (A)strbend_term<R, G>(pos4 + 4 * i, pos4 + 4 * j, pos4 + 4 * k, (R)u2f(r0.z), (R)u2f(r0.w),
                                         (R)u2f(r1.x), (R)u2f(r1.y), (R)u2f(r1.z), md, f);
        if (G) {
            if (v) add3(gw + 3 * i, f[0]);
            __syncwarp();
            if (v) add3(gw + 3 * j, f[1]);
            __syncwarp();
            if (v) add3(gw + 3 * k, f[2]);
            __syncwarp();
        }
    }
    for (int c = warp; c < m.onch; c += NW) {
        uint4 r = __ldg(BR + m.ooff + (size_t)c * 32 + lane);
        bool v = r.x != 0xffffffffu;
        int i = r.x & 0xffff, j = r.x >> 16, k = r.y & 0xffff, l = r.y >> 16;
        R f[4][3];
        if (v)
            acc += (A)oop_term<R, G>(pos4 + 4 * i, pos4 + 4 * j, pos4 + 4 * k, pos4 + 4 * l, (R)u2f(r.z), md, f);
        if (G) {
            if (v) add3(gw + 3 * i, f[0]);
            __syncwarp();
            if (v) add3(gw + 3 * j, f[1]);
            __syncwarp();
            if (v) add3(gw + 3 * k, f[2]);
            __syncwarp();
            if (v) add3(gw + 3 * l, f[3]);
            __syncwarp();
        }
    }
    for (int c = warp; c < m.tnch; c += NW) {
        uint4 r0 = __ldg(BR + m.toff + (size_t)c * 64 + lane);
        uint4 r1 = __ldg(BR + m.toff + (size_t)c * 64 + 32 + lane);
        bool v = r0.x != 0xffffffffu;
        int i = r0.x & 0xffff, j = r0.x >> 16, k = r0.y & 0xffff, l = r0.y >> 16;
        R f[4][3];
        if (v)
            acc += (A)torsion_term<R, G>(pos4 + 4 * i, pos4 + 4 * j, pos4 + 4 * k, pos4 + 4 * l, (R)u2f(r0.z),
                                         (R)u2f(r0.w), (R)u2f(r1.x), f);
        if (G) {
            if (v) add3(gw + 3 * i, f[0]);
            __syncwarp();
            if (v) add3(gw + 3 * j, f[1]);
            __syncwarp();
            if (v) add3(gw + 3 * k, f[2]);
            __syncwarp();
            if (v) add3(gw + 3 * l, f[3]);
            __syncwarp();
        }
    }

    // non-bonded pairs, implicit from the staged bit rows and class table
    const int W = (N + 31) >> 5;
    const uint32_t *pm = ms.mask, *p14 = ms.mask + (size_t)N * W;
    const bool dd = m.diel == 2;
    // Rows i and i + NW per step: two independent pair chains per lane (both are
    // evaluated; a pair absent from the bit rows contributes nothing) and one
    // scatter per column.
    for (int i = warp; i < N - 1; i += 2 * NW) {
        const int i2 = i + NW;
        const bool has2 = i2 < N - 1;
        R xi, yi, zi, xk = R(0), yk = R(0), zk = R(0);
        ld3(pos4, i, xi, yi, zi);
        if (has2) ld3(pos4, i2, xk, yk, zk);
        const int ci = ms.cls[i] * m.ncls, ck = has2 ? ms.cls[i2] * m.ncls : 0;
        const int ik = has2 ? i2 : i;
        R fx = R(0), fy = R(0), fz = R(0), kx = R(0), ky = R(0), kz = R(0);
        const int jb2 = has2 ? ((i2 + 1) & ~31) : N;
        for (int jb = (i + 1) & ~31; jb < N; jb += 32) {
            const int wb = jb >> 5;
            const uint32_t wd = pm[i * W + wb];
            const uint32_t wd2 = jb >= jb2 ? pm[i2 * W + wb] : 0u;
            if ((wd | wd2) == 0u) continue;
            const bool b1 = (wd >> lane) & 1u, b2 = (wd2 >> lane) & 1u;
            if (b1 || b2) {
                const int j = jb + lane;
                const int cj = ms.cls[j];
                const float2 t1 = ms.tab[ci + cj], t2 = ms.tab[ck + cj];
                const uint32_t w14 = p14[i * W + wb], w14b = jb >= jb2 ? p14[i2 * W + wb] : 0u;
                R q1 = pair_charge<R>(ms, i, j), q2 = pair_charge<R>(ms, ik, j);
                if ((w14 >> lane) & 1u) q1 *= R(0.75);
                if ((w14b >> lane) & 1u) q2 *= R(0.75);
                R xj, yj, zj;
                ld3(pos4, j, xj, yj, zj);
                const R dx1 = xi - xj, dy1 = yi - yj, dz1 = zi - zj;
                const R dx2 = xk - xj, dy2 = yk - yj, dz2 = zk - zj;
                R ev1, ee1, s1, ev2, ee2, s2;
                pair_term<R, G, IRTAB>(dx1, dy1, dz1, (R)t1.x, (R)t1.y, q1, dd, ev1, ee1, s1);
                pair_term<R, G, IRTAB>(dx2, dy2, dz2, (R)t2.x, (R)t2.y, q2, dd, ev2, ee2, s2);
                if (b1) {
                    acc += (A)ev1;
                    acc += (A)ee1;
                }
                if (b2) {
                    acc += (A)ev2;
                    acc += (A)ee2;
                }
                if (G) {
                    const R m1 = b1 ? s1 : R(0), m2 = b2 ? s2 : R(0);
                    const R g1x = m1 * dx1, g1y = m1 * dy1, g1z = m1 * dz1;
                    const R g2x = m2 * dx2, g2y = m2 * dy2, g2z = m2 * dz2;
                    fx += g1x; fy += g1y; fz += g1z;
                    kx += g2x; ky += g2y; kz += g2z;
                    gw[3 * j] -= g1x + g2x;
                    gw[3 * j + 1] -= g1y + g2y;
                    gw[3 * j + 2] -= g1z + g2z;
                }
            }
        }
        if (G) {
            __syncwarp();
            fx = wsum(fx); fy = wsum(fy); fz = wsum(fz);
            kx = wsum(kx); ky = wsum(ky); kz = wsum(kz);
            if (lane == 0) {
                gw[3 * i] += fx; gw[3 * i + 1] += fy; gw[3 * i + 2] += fz;
                if (has2) { gw[3 * i2] += kx; gw[3 * i2 + 1] += ky; gw[3 * i2 + 2] += kz; }
            }
            __syncwarp();
        }
    }
    return acc;
}

// ---------------------------------------------------------------------------
// The persistent optimizer kernel
// ---------------------------------------------------------------------------

template <class R, class A, int NT, int NC, bool MSM, bool LB>
struct Opt {
    static constexpr int NW = NT / 32;
    const Params &P;
    R *pos4, *x, *g, *dir, *xo, *dg, *hp, *hq, *pxi, *pc, *pr, *gbuf, *mat;
    double *pos4d;     // FP64 copy of pos4 (float R only)
    R *ring;           // TMA row ring (streamed H pass)
    uint64_t *mbar;    // one mbarrier per ring stage and warp
    uint32_t phase;    // parity of each of this warp's stages
    int *abort_flag;   // CTA-wide: a bounded wait gave up (shared memory)
    int ldh;           // row stride of H
    bool use64;        // line-search energies in FP64 (escalated)
    int *cls;
    double *qa;
    float *qf;
    uint32_t *mask;
    float2 *tab;
    MolSmem ms;
    A *red, *rho_s, *alpha_s;
    int rsel;
    MolV m;
    int N, n, nv;

    __device__ Opt(const Params &p, unsigned char *sm, int *abort_ = nullptr) : P(p), abort_flag(abort_), rsel(0) {
        Layout L = make_layout(p.nmax, NW, LB ? p.hist_m : 0, MSM, sizeof(R), sizeof(A), p.b.max_classes);
        pos4 = (R *)(sm + L.pos4); x = (R *)(sm + L.x); g = (R *)(sm + L.g); dir = (R *)(sm + L.dir);
        pos4d = (double *)(sm + L.pos4d);
        use64 = false;
        ring = (R *)(sm + L.ring);
        mbar = (uint64_t *)(sm + L.mbar);
        phase = 0;
        ldh = 0;
        xo = (R *)(sm + L.xo); dg = (R *)(sm + L.dg); hp = (R *)(sm + L.hp); hq = (R *)(sm + L.hq);
        pxi = (R *)(sm + L.pxi); pc = (R *)(sm + L.pc); pr = (R *)(sm + L.pr); gbuf = (R *)(sm + L.gbuf);
        cls = (int *)(sm + L.cls); qa = (double *)(sm + L.q); red = (A *)(sm + L.red);
        qf = (float *)(sm + L.qf); mask = (uint32_t *)(sm + L.mask); tab = (float2 *)(sm + L.tab);
        ms.cls = cls; ms.qa = qa; ms.qf = qf; ms.mask = mask; ms.tab = tab;
        rho_s = (A *)(sm + L.rho); alpha_s = (A *)(sm + L.alpha);
        if (MSM) mat = (R *)(sm + L.mat);
        else mat = (R *)p.gmat + (size_t)blockIdx.x * p.gslot;
    }

    __device__ __forceinline__ A *next_red() {
        A *r = red + rsel * NW * 8;
        rsel ^= 1;
        return r;
    }

    template <int KS, int KM>
    __device__ __forceinline__ void reduce(A (&s)[KS], A (&mm)[KM]) {
        block_reduce<NW, KS, KM, A>(s, mm, next_red());
    }

    __device__ __forceinline__ A energy() {
        A e[1];
        if (sizeof(R) == 4 && use64)
            e[0] = (A)eval_terms<double, double, NW, false, sizeof(R) == 4>(P, m, pos4d, (double *)nullptr, ms, nv);
        else
            e[0] = eval_terms<R, A, NW, false, sizeof(R) == 4>(P, m, pos4, gbuf, ms, nv);
        A z[1] = {A(0)};
        reduce<1, 1>(e, z);
        return e[0];
    }

    // gradient at pos4 into dst (raw, unscaled); needs a preceding __syncthreads after pos4 writes
    __device__ __forceinline__ void gradient(R *dst) {
        eval_terms<R, A, NW, true, sizeof(R) == 4>(P, m, pos4, gbuf, ms, nv);
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += NT) {
            R s = R(0);
#pragma unroll
            for (int w = 0; w < NW; ++w) s += gbuf[(size_t)w * nv + k];
            dst[k] = s;
        }
    }

    __device__ __forceinline__ void setpos(int k, R v) {
        const int o = 4 * (k / 3) + (k % 3);
        pos4[o] = v;
        if (sizeof(R) == 4) pos4d[o] = (double)v;
    }

    // Butterfly reduce-scatter of 16 per-lane partial sums over the warp (16 shuffles):
    // afterwards lanes l and l^1 both hold the warp-wide sum of value (l >> 1).
    static __device__ __forceinline__ float reduce16(const float (&v)[16]) {
        const int lane = threadIdx.x & 31;
        const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
        float w[8], x[4], y[2];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            w[k] = (b4 ? v[k + 8] : v[k]) + __shfl_xor_sync(0xffffffffu, b4 ? v[k] : v[k + 8], 16);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            x[k] = (b3 ? w[k + 4] : w[k]) + __shfl_xor_sync(0xffffffffu, b3 ? w[k] : w[k + 4], 8);
#pragma unroll
        for (int k = 0; k < 2; ++k)
            y[k] = (b2 ? x[k + 2] : x[k]) + __shfl_xor_sync(0xffffffffu, b2 ? x[k] : x[k + 2], 4);
        float z = (b1 ? y[1] : y[0]) + __shfl_xor_sync(0xffffffffu, b1 ? y[0] : y[1], 2);
        return z + __shfl_xor_sync(0xffffffffu, z, 1);
    }

    // Warp-uniform bounded wait for ring stage st of this warp.  On giving up it
    // flags the launch (err word) and this CTA (abort flag) and returns false;
    // the stage's copy may still be in flight (drain() waits for it).
    // At most P.wait_spins tests: a non-blocking one, then potentially blocking polls
    // (none when P.wait_spins is 0: the wait gives up at once).
    __device__ __forceinline__ bool wait_stage(uint64_t *bw, int st) {
        const uint32_t par = (phase >> st) & 1u;
        bool done = P.wait_spins > 0 && mbar_test_wait(&bw[st], par);
        for (uint32_t spins = 1; !__all_sync(0xffffffffu, done); ++spins) {
            if (spins >= P.wait_spins) {
                if ((threadIdx.x & 31) == 0) {
                    atomicExch(P.err, 1);
                    atomicExch(P.scratch_err, 1);
                    atomicExch(abort_flag, 1);
                }
                return false;
            }
            done = mbar_try_wait(&bw[st], par);
        }
        phase ^= 1u << st;
        return true;
    }
    // After a wait gave up: bounded wait for this warp's copies of rows [from, to) still
    // in flight -- the row whose wait gave up included -- so none lands in shared
    // memory after the CTA has moved on or exited.
    __device__ __forceinline__ void drain(uint64_t *bw, int from, int to) {
        for (int t = from; t < to; ++t) {
            const int st = t % kStages;
            uint32_t spins = 0;
            while (!__all_sync(0xffffffffu, mbar_try_wait(&bw[st], (phase >> st) & 1u)) && ++spins < kDrainSpins) {
            }
            phase ^= 1u << st;
        }
    }

    // One pass over the dense inverse Hessian: apply the pending rank-2 update
    // H_ij += pxi_j*pr_i + pxi_i*pc_j, store, and form hp = H g, hq = H dg.
    __device__ __forceinline__ void hpass(bool pending) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        constexpr int NCR = NC > 0 ? NC : 1;   // NC == 0: columns read from shared memory
        R cx[NCR], cc[NCR], cg[NCR], cd[NCR];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int j = lane + 32 * c;
            const bool in = j < n;
            cx[c] = in ? pxi[j] : R(0);
            cc[c] = in ? pc[j] : R(0);
            cg[c] = in ? g[j] : R(0);
            cd[c] = in ? dg[j] : R(0);
        }
        for (int i = warp; i < n; i += NW) {
            R *row = mat + (size_t)i * ldh;
            const R ri = pending ? pr[i] : R(0), xi = pending ? pxi[i] : R(0);
            R ap = R(0), aq = R(0);
            if (NC == 0) {
                for (int j = lane; j < n; j += 32) {
                    R h = row[j];
                    if (pending) {
                        h = fma(pxi[j], ri, h);
                        h = fma(xi, pc[j], h);
                        row[j] = h;
                    }
                    ap = fma(h, g[j], ap);
                    aq = fma(h, dg[j], aq);
                }
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const int j = lane + 32 * c;
                if (j < n) {
                    R h = row[j];
                    if (pending) {
                        h = fma(cx[c], ri, h);
                        h = fma(xi, cc[c], h);
                        row[j] = h;
                    }
                    ap = fma(h, cg[c], ap);
                    aq = fma(h, cd[c], aq);
                }
            }
            ap = wsum(ap);
            aq = wsum(aq);
            if (lane == 0) { hp[i] = ap; hq[i] = aq; }
        }
    }

    // The same pass with H in global memory: each warp streams its rows through a
    // kStages-deep shared-memory ring with 1-D TMA bulk copies (completion on one
    // mbarrier per stage), so kStages rows per warp are in flight while the
    // previous ones are updated; updated rows go back with coalesced stores.
    __device__ __forceinline__ void hpass_stream(bool pending) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        constexpr int NCR = NC > 0 ? NC : 1;   // NC == 0: columns read from shared memory
        R cx[NCR], cc[NCR], cg[NCR], cd[NCR];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int j = lane + 32 * c;
            const bool in = j < n;
            cx[c] = in ? pxi[j] : R(0);
            cc[c] = in ? pc[j] : R(0);
            cg[c] = in ? g[j] : R(0);
            cd[c] = in ? dg[j] : R(0);
        }
        const int ldr = hld(3 * P.nmax);
        R *rw = ring + (size_t)warp * kStages * ldr;
        uint64_t *bw = mbar + warp * kStages;
        const int nrows = warp < n ? (n - warp + NW - 1) / NW : 0;
        const uint32_t bytes = (uint32_t)(ldh * sizeof(R));
        if (lane == 0) {
            for (int t = 0; t < nrows && t < kStages; ++t) {
                mbar_expect_tx(&bw[t], bytes);
                tma_load_row(rw + (size_t)t * ldr, mat + (size_t)(warp + NW * t) * ldh, bytes, &bw[t]);
            }
        }
        for (int t = 0; t < nrows; ++t) {
            const int st = t % kStages, i = warp + NW * t;
            if (!wait_stage(bw, st)) {
                drain(bw, t, nrows < t + kStages ? nrows : t + kStages);
                break;
            }
            const R *src = rw + (size_t)st * ldr;
            R *row = mat + (size_t)i * ldh;
            const R ri = pending ? pr[i] : R(0), xi = pending ? pxi[i] : R(0);
            R ap = R(0), aq = R(0);
            if (NC == 0) {
                for (int j = lane; j < n; j += 32) {
                    R h = src[j];
                    if (pending) {
                        h = fma(pxi[j], ri, h);
                        h = fma(xi, pc[j], h);
                        row[j] = h;
                    }
                    ap = fma(h, g[j], ap);
                    aq = fma(h, dg[j], aq);
                }
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const int j = lane + 32 * c;
                if (j < n) {
                    R h = src[j];
                    if (pending) {
                        h = fma(cx[c], ri, h);
                        h = fma(xi, cc[c], h);
                        row[j] = h;
                    }
                    ap = fma(h, cg[c], ap);
                    aq = fma(h, cd[c], aq);
                }
            }
            ap = wsum(ap);   // also orders every lane's reads of this stage before its reuse
            aq = wsum(aq);
            if (lane == 0) {
                hp[i] = ap;
                hq[i] = aq;
                if (t + kStages < nrows) {
                    fence_proxy_async_smem();
                    mbar_expect_tx(&bw[st], bytes);
                    tma_load_row(rw + (size_t)st * ldr, mat + (size_t)(warp + NW * (t + kStages)) * ldh, bytes,
                                 &bw[st]);
                }
            }
        }
        fence_proxy_async_global();   // this pass's row stores before the next pass's TMA reads
    }

    // The streamed pass of the register-lean FP32 instance: float4 columns (the
    // rows of H and the vectors are padded to a multiple of 4 with zeros) and two
    // rows per step, so each vector load from shared memory serves two rows and a
    // warp keeps two row copies of its TMA ring in use at once.
    __device__ __forceinline__ void hpass_stream_v4(bool pending) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int ldr = hld(3 * P.nmax);
        float *rw = (float *)ring + (size_t)warp * kStages * ldr;
        uint64_t *bw = mbar + warp * kStages;
        const int nrows = warp < n ? (n - warp + NW - 1) / NW : 0;
        const uint32_t bytes = (uint32_t)(ldh * sizeof(float));
        const int n4 = ldh >> 2;
        const float4 *X4 = (const float4 *)pxi, *C4 = (const float4 *)pc;
        const float4 *G4 = (const float4 *)g, *D4 = (const float4 *)dg;
        float *H = (float *)mat;
        if (lane == 0) {
            for (int t = 0; t < nrows && t < kStages; ++t) {
                mbar_expect_tx(&bw[t], bytes);
                tma_load_row(rw + (size_t)t * ldr, H + (size_t)(warp + NW * t) * ldh, bytes, &bw[t]);
            }
        }
        // groups of 4 row pairs: the 16 per-lane partial sums are reduced together
        for (int t0 = 0; t0 < nrows; t0 += 8) {
            float v[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] = 0.f;
            bool aborted = false;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int t = t0 + 2 * u;
                if (t >= nrows) break;
                const bool two = t + 1 < nrows;
                const int s0 = t % kStages, s1 = (t + 1) % kStages;
                const int issued = nrows < t + kStages ? nrows : t + kStages;
                if (!wait_stage(bw, s0)) {
                    drain(bw, t, issued);
                    aborted = true;
                    break;
                }
                if (two && !wait_stage(bw, s1)) {
                    drain(bw, t + 1, issued);
                    aborted = true;
                    break;
                }
                const int i0 = warp + NW * t, i1 = i0 + NW;
                const float4 *A0 = (const float4 *)(rw + (size_t)s0 * ldr), *A1 = (const float4 *)(rw + (size_t)s1 * ldr);
                float4 *W0 = (float4 *)(H + (size_t)i0 * ldh), *W1 = (float4 *)(H + (size_t)(two ? i1 : i0) * ldh);
                const float r0 = pending ? (float)pr[i0] : 0.f, x0 = pending ? (float)pxi[i0] : 0.f;
                const float r1 = (pending && two) ? (float)pr[i1] : 0.f, x1 = (pending && two) ? (float)pxi[i1] : 0.f;
                float a0 = 0.f, q0 = 0.f, a1 = 0.f, q1 = 0.f;
                for (int c = lane; c < n4; c += 32) {
                    float4 h0 = A0[c];
                    float4 h1 = two ? A1[c] : make_float4(0.f, 0.f, 0.f, 0.f);
                    if (pending) {
                        const float4 px = X4[c], pv = C4[c];
                        h0.x = fmaf(x0, pv.x, fmaf(px.x, r0, h0.x));
                        h0.y = fmaf(x0, pv.y, fmaf(px.y, r0, h0.y));
                        h0.z = fmaf(x0, pv.z, fmaf(px.z, r0, h0.z));
                        h0.w = fmaf(x0, pv.w, fmaf(px.w, r0, h0.w));
                        W0[c] = h0;
                        if (two) {
                            h1.x = fmaf(x1, pv.x, fmaf(px.x, r1, h1.x));
                            h1.y = fmaf(x1, pv.y, fmaf(px.y, r1, h1.y));
                            h1.z = fmaf(x1, pv.z, fmaf(px.z, r1, h1.z));
                            h1.w = fmaf(x1, pv.w, fmaf(px.w, r1, h1.w));
                            W1[c] = h1;
                        }
                    }
                    const float4 gg = G4[c], dd = D4[c];
                    a0 = fmaf(h0.w, gg.w, fmaf(h0.z, gg.z, fmaf(h0.y, gg.y, fmaf(h0.x, gg.x, a0))));
                    q0 = fmaf(h0.w, dd.w, fmaf(h0.z, dd.z, fmaf(h0.y, dd.y, fmaf(h0.x, dd.x, q0))));
                    a1 = fmaf(h1.w, gg.w, fmaf(h1.z, gg.z, fmaf(h1.y, gg.y, fmaf(h1.x, gg.x, a1))));
                    q1 = fmaf(h1.w, dd.w, fmaf(h1.z, dd.z, fmaf(h1.y, dd.y, fmaf(h1.x, dd.x, q1))));
                }
                v[4 * u] = a0; v[4 * u + 1] = q0; v[4 * u + 2] = a1; v[4 * u + 3] = q1;
                __syncwarp();   // every lane's reads of both stages before they are refilled
                if (lane == 0) {
                    fence_proxy_async_smem();
                    if (t + kStages < nrows) {
                        mbar_expect_tx(&bw[s0], bytes);
                        tma_load_row(rw + (size_t)s0 * ldr, H + (size_t)(warp + NW * (t + kStages)) * ldh, bytes,
                                     &bw[s0]);
                    }
                    if (t + 1 + kStages < nrows) {
                        mbar_expect_tx(&bw[s1], bytes);
                        tma_load_row(rw + (size_t)s1 * ldr, H + (size_t)(warp + NW * (t + 1 + kStages)) * ldh, bytes,
                                     &bw[s1]);
                    }
                }
            }
            if (aborted) break;
            // lanes l and l^1 now hold the sum of value l >> 1: pair u = value / 4, then a0 q0 a1 q1
            const float sum = reduce16(v);
            const int val = lane >> 1, tr = t0 + 2 * (val >> 2) + ((val >> 1) & 1);
            if (!(lane & 1) && tr < nrows) {
                const int i = warp + NW * tr;
                if (val & 1) hq[i] = sum;
                else hp[i] = sum;
            }
        }
        fence_proxy_async_global();
    }

    // L-BFGS two-loop recursion (lbfgs_tg.metal:264-292): dir = -H g from the ring history
    __device__ __forceinline__ void two_loop(int hcount, int hidx) {
        const int hm = P.hist_m;
        R *S = mat, *Y = mat + (size_t)hm * nv;
        for (int k = threadIdx.x; k < n; k += NT) hq[k] = g[k];
        for (int jj = hcount - 1; jj >= 0; --jj) {
            int slot = ((hidx - 1 - (hcount - 1 - jj)) % hm + hm) % hm;
            const R *Sj = S + (size_t)slot * nv;
            A s1[1] = {A(0)}, z[1] = {A(0)};
            for (int k = threadIdx.x; k < n; k += NT) s1[0] += (A)(Sj[k] * hq[k]);
            reduce<1, 1>(s1, z);
            A aj = rho_s[slot] * s1[0];
            if (threadIdx.x == 0) alpha_s[jj] = aj;
            const R *Yj = Y + (size_t)slot * nv;
            const R ar = (R)aj;
            for (int k = threadIdx.x; k < n; k += NT) hq[k] -= ar * Yj[k];
        }
        if (hcount > 0) {
            int nw = ((hidx - 1) % hm + hm) % hm;
            const R *Sn = S + (size_t)nw * nv, *Yn = Y + (size_t)nw * nv;
            A s2[2] = {A(0), A(0)}, z[1] = {A(0)};
            for (int k = threadIdx.x; k < n; k += NT) {
                s2[0] += (A)(Sn[k] * Yn[k]);
                s2[1] += (A)(Yn[k] * Yn[k]);
            }
            reduce<2, 1>(s2, z);
            const R gam = (R)(s2[0] / (s2[1] > A(1e-30) ? s2[1] : A(1e-30)));
            for (int k = threadIdx.x; k < n; k += NT) hq[k] *= gam;
        }
        for (int jj = 0; jj < hcount; ++jj) {
            int slot = ((hidx - 1 - (hcount - 1 - jj)) % hm + hm) % hm;
            const R *Yj = Y + (size_t)slot * nv, *Sj = S + (size_t)slot * nv;
            A s1[1] = {A(0)}, z[1] = {A(0)};
            for (int k = threadIdx.x; k < n; k += NT) s1[0] += (A)(Yj[k] * hq[k]);
            reduce<1, 1>(s1, z);
            const A bj = rho_s[slot] * s1[0];
            const R c = (R)(alpha_s[jj] - bj);
            for (int k = threadIdx.x; k < n; k += NT) hq[k] += c * Sj[k];
        }
        for (int k = threadIdx.x; k < n; k += NT) dir[k] = -hq[k];
    }

    // inverse Hessian back to the identity (dense) / history cleared (L-BFGS)
    __device__ __forceinline__ void reset_matrix() {
        if (!LB) {
            for (size_t e = threadIdx.x; e < (size_t)n * ldh; e += NT) {
                const int i = (int)(e / ldh), j = (int)(e - (size_t)i * ldh);
                mat[e] = i == j ? R(1) : R(0);
            }
            if (!MSM) fence_proxy_async_global();
        }
    }

    __device__ void run(int conf) {
        const int tid = threadIdx.x;
        const KConst &K = P.K;
        m = load_mol(P.b.mol_desc, __ldcg(P.c.conf_mol + conf));
        N = m.n;
        n = 3 * N;
        nv = (3 * P.nmax + 3) & ~3;
        use64 = false;
        const int64_t coord = __ldcg(reinterpret_cast<const long long *>(P.c.conf_coord) + conf);
        const float *gp = P.pos + coord;
        for (int k = tid; k < n; k += NT) {
            R v = (R)__ldcg(gp + k);
            x[k] = v;
            setpos(k, v);
        }
        stage_molecule<NT, sizeof(R) == 4>(P, m, cls, qa, qf, mask, tab);
        ldh = MSM ? n : hld(n);
        // zero vector pads: the float4 pass reads columns up to hld(n)
        for (int k = n + tid; k < nv; k += NT) { g[k] = R(0); dg[k] = R(0); pxi[k] = R(0); pc[k] = R(0); }
        if (!LB) reset_matrix();
        __syncthreads();

        // initial gradient and scale (header :435-454, tg.metal:115-122)
        gradient(hp);
        A gs_[2] = {A(0), A(0)}, gm_[1] = {A(0)};
        for (int k = tid; k < n; k += NT) {
            gs_[0] += (A)fabs(hp[k]);
            gs_[1] += (A)(x[k] * x[k]);
            A a = (A)fabs(hp[k]);
            gm_[0] = a > gm_[0] ? a : gm_[0];
        }
        reduce<2, 1>(gs_, gm_);
        R gsc = (R)K.gscale;
        {
            // bounded: a non-finite gradient is caught below, never halved forever
            R mx = (R)gm_[0] * gsc;
            for (int h = 0; h < 256 && mx > (R)K.gcap; ++h) { mx *= R(0.5); gsc *= R(0.5); }
        }
        for (int k = tid; k < n; k += NT) {
            R v = hp[k] * gsc;
            g[k] = v;
            dir[k] = -v;
        }
        A E = energy();
        const A max_step = (A)K.maxstep * (sqrt(gs_[1]) > (A)n ? sqrt(gs_[1]) : (A)n);
        int status = MMFFB_ST_MAXIT;
        int it = 0, done_iters = 0, nevals = 0, restarts = 0;
        bool fresh = true;     // direction is -g (start or just after a restart)
        bool pending = false;  // a rank-2 update not yet applied to H
        int hcount = 0, hidx = 0;
        if (!isfinite((double)E) || !isfinite((double)gs_[0])) {
            status = MMFFB_ST_NONFINITE;
            it = P.max_iters;
        } else {
            for (it = 0; it < P.max_iters; ++it) {
                // direction length, slope, largest relative component; xold = x
                A s3[2] = {A(0), A(0)}, m3[1] = {A(0)};
                for (int k = tid; k < n; k += NT) {
                    const R d = dir[k], xv = x[k];
                    xo[k] = xv;
                    s3[0] += (A)(d * d);
                    s3[1] += (A)(d * g[k]);
                    A t = (A)(fabs(d) / fmax(fabs(xv), R(1)));
                    m3[0] = t > m3[0] ? t : m3[0];
                }
                reduce<2, 1>(s3, m3);
                const A dn = sqrt(s3[0]);
                if (dn > max_step) {
                    const R sc = (R)(max_step / dn);
                    A s4[1] = {A(0)}, m4[1] = {A(0)};
                    for (int k = tid; k < n; k += NT) {
                        const R d = dir[k] * sc;
                        dir[k] = d;
                        s4[0] += (A)(d * g[k]);
                        A t = (A)(fabs(d) / fmax(fabs(x[k]), R(1)));
                        m4[0] = t > m4[0] ? t : m4[0];
                    }
                    reduce<1, 1>(s4, m4);
                    s3[1] = s4[0];
                    m3[0] = m4[0];
                }
                const A slope = s3[1];
                if (!(slope < A(0))) {
                    if (!fresh && restarts < P.max_restarts) {
                        // uphill quasi-Newton direction: restart from steepest descent
                        ++restarts;
                        fresh = true;
                        pending = false;
                        hcount = 0;
                        hidx = 0;
                        reset_matrix();
                        for (int k = tid; k < n; k += NT) dir[k] = -g[k];
                        __syncthreads();
                        continue;
                    }
                    status = MMFFB_ST_SLOPE;
                    break;
                }
                const A lam_min = (A)K.movetol / (m3[0] > A(1e-30) ? m3[0] : A(1e-30));

                // backtracking line search (tg.metal:192-256)
                const A Eold = E;
                A lam = A(1), plam = A(1), pe = Eold;
                bool ok = false;
                for (int ls = 0; ls < K.maxls; ++ls) {
                    if (lam < lam_min) break;
                    ++nevals;
                    const R lr = (R)lam;
                    for (int k = tid; k < n; k += NT) {
                        const R v = xo[k] + lr * dir[k];
                        x[k] = v;
                        setpos(k, v);
                    }
                    __syncthreads();
                    const A et = energy();
                    if (et - Eold <= (A)K.functol * lam * slope) { E = et; ok = true; break; }
                    A tl;
                    if (ls == 0) {
                        tl = -slope / (A(2) * (et - Eold - slope));
                    } else {
                        const A r1 = et - Eold - lam * slope, r2 = pe - Eold - plam * slope;
                        const A l2 = lam * lam, p2 = plam * plam, dv = lam - plam;
                        if (fabs(dv) < A(1e-30)) tl = A(0.5) * lam;
                        else {
                            const A a = (r1 / l2 - r2 / p2) / dv, b = (-plam * r1 / l2 + lam * r2 / p2) / dv;
                            if (fabs(a) < A(1e-30)) tl = fabs(b) > A(1e-30) ? -slope / (A(2) * b) : A(0.5) * lam;
                            else {
                                const A disc = b * b - A(3) * a * slope;
                                if (disc < A(0)) tl = A(0.5) * lam;
                                else if (b <= A(0)) tl = (-b + sqrt(disc)) / (A(3) * a);
                                else tl = -slope / (b + sqrt(disc));
                            }
                        }
                    }
                    tl = tl < A(0.5) * lam ? tl : A(0.5) * lam;
                    tl = tl > A(0.1) * lam ? tl : A(0.1) * lam;
                    plam = lam; pe = et; lam = tl;
                }
                if (!ok) {
                    for (int k = tid; k < n; k += NT) {
                        x[k] = xo[k];
                        setpos(k, xo[k]);
                    }
                    if (sizeof(R) == 4 && P.polish64 && !use64) {
                        // FP32 term energies are at their noise floor: continue with FP64
                        // line-search energies of the same FP32 coordinates
                        use64 = true;
                        __syncthreads();
                        E = energy();
                        continue;
                    }
                    if (!fresh && restarts < P.max_restarts) {
                        // no decrease along the quasi-Newton direction: restart from -g
                        ++restarts;
                        fresh = true;
                        pending = false;
                        hcount = 0;
                        hidx = 0;
                        reset_matrix();
                        for (int k = tid; k < n; k += NT) dir[k] = -g[k];
                        __syncthreads();
                        continue;
                    }
                    __syncthreads();
                }
                fresh = false;
                // xi = x - xold, TOLX (kept per thread until the next reduction)
                A tolx = A(0);
                for (int k = tid; k < n; k += NT) {
                    const R xi = x[k] - xo[k];
                    xo[k] = xi;
                    A t = (A)(fabs(xi) / fmax(fabs(x[k]), R(1)));
                    tolx = t > tolx ? t : tolx;
                }
                // gradient at the new point (computed before the TOLX verdict; one
                // wasted evaluation per conformer instead of a barrier per iteration)
                gradient(hp);
                const bool atom_test = P.exit_test == MMFFB_EXIT_ATOM_NORM &&
                                       (P.check_every <= 1 || (it + 1) % P.check_every == 0);
                A anorm = A(0);
                if (atom_test) {
                    __syncthreads();
                    for (int a = tid; a < N; a += NT) {
                        const R gx = hp[3 * a], gy = hp[3 * a + 1], gz = hp[3 * a + 2];
                        const A v = (A)sqrt(gx * gx + gy * gy + gz * gz);
                        anorm = v > anorm ? v : anorm;
                    }
                }
                A gs2[1] = {A(0)}, gm2[4] = {A(0), A(0), tolx, anorm};
                for (int k = tid; k < n; k += NT) {
                    const A a = (A)fabs(hp[k]);
                    gs2[0] += a;
                    gm2[0] = a > gm2[0] ? a : gm2[0];
                    const A b = (A)(fabs(hp[k]) * fmax(fabs(x[k]), R(1)));
                    gm2[1] = b > gm2[1] ? b : gm2[1];
                }
                reduce<1, 4>(gs2, gm2);
                if (!isfinite((double)gs2[0]) || !isfinite((double)E)) { status = MMFFB_ST_NONFINITE; break; }
                if (atom_test && gm2[3] * (A)P.atom_grad_scale <= (A)P.grad_tol) { status = MMFFB_ST_GRAD; break; }
                if (gm2[2] < (A)K.tolx) {
                    if (sizeof(R) == 4 && P.polish64 && !use64) {
                        use64 = true;
                        E = energy();
                    } else {
                        status = ok ? MMFFB_ST_TOLX : MMFFB_ST_LSFAIL;
                        break;
                    }
                }
                {
                    R mx = (R)gm2[0] * gsc;
                    for (int h = 0; h < 256 && mx > (R)K.gcap; ++h) { mx *= R(0.5); gsc *= R(0.5); }
                }
                if (P.exit_test == MMFFB_EXIT_TG) {
                    const A num = (A)((R)gm2[1] * gsc);
                    A den = E * (A)gsc;
                    den = den > A(1) ? den : A(1);
                    if (num / den < (A)P.grad_tol) { status = MMFFB_ST_GRAD; break; }
                }
                for (int k = tid; k < n; k += NT) {
                    const R gn = hp[k] * gsc;
                    dg[k] = gn - g[k];
                    g[k] = gn;
                }
                if (!LB) {
                    __syncthreads();
                    if constexpr (!MSM && NC == 0 && sizeof(R) == 4) hpass_stream_v4(pending);
                    else if (MSM) hpass(pending);
                    else hpass_stream(pending);
                    __syncthreads();
                    if (!MSM && *(volatile int *)abort_flag) { status = MMFFB_ST_TIMEOUT; break; }
                    A d6[6] = {A(0), A(0), A(0), A(0), A(0), A(0)}, z[1] = {A(0)};
                    for (int k = tid; k < n; k += NT) {
                        const R dgk = dg[k], xik = xo[k], qk = hq[k], gk = g[k];
                        d6[0] += (A)(dgk * xik);
                        d6[1] += (A)(dgk * qk);
                        d6[2] += (A)(dgk * dgk);
                        d6[3] += (A)(xik * xik);
                        d6[4] += (A)(xik * gk);
                        d6[5] += (A)(qk * gk);
                    }
                    reduce<6, 1>(d6, z);
                    const A fac = d6[0], fae = d6[1];
                    if (fac * fac > (A)K.eps * d6[2] * d6[3] && fac > A(0)) {
                        const A fi = A(1) / fac;
                        const A al = fi * (A(1) + fae * fi);
                        const R cxg = (R)(al * d6[4]), cqg = (R)(fi * d6[5]), fxg = (R)(fi * d6[4]);
                        const R rfi = (R)fi, ral = (R)al;
                        for (int k = tid; k < n; k += NT) {
                            const R xk = xo[k], qk = hq[k];
                            dir[k] = -(hp[k] + cxg * xk - cqg * xk - fxg * qk);
                            pxi[k] = xk;
                            pc[k] = -rfi * qk;
                            pr[k] = ral * xk - rfi * qk;
                        }
                        pending = true;
                    } else {
                        for (int k = tid; k < n; k += NT) dir[k] = -hp[k];
                        pending = false;
                    }
                } else {
                    // L-BFGS history update (lbfgs_tg.metal:247-262)
                    A y1[1] = {A(0)}, z[1] = {A(0)};
                    for (int k = tid; k < n; k += NT) y1[0] += (A)(dg[k] * xo[k]);
                    reduce<1, 1>(y1, z);
                    if (y1[0] > A(1e-10)) {
                        const int hm = P.hist_m;
                        const int slot = hidx % hm;
                        R *S = mat + (size_t)slot * nv, *Y = mat + (size_t)hm * nv + (size_t)slot * nv;
                        for (int k = tid; k < n; k += NT) { S[k] = xo[k]; Y[k] = dg[k]; }
                        if (tid == 0) rho_s[slot] = A(1) / y1[0];
                        hidx++;
                        if (hcount < hm) hcount++;
                    }
                    __syncthreads();
                    two_loop(hcount, hidx);
                }
            }
        }
        if (status != MMFFB_ST_NONFINITE || it < P.max_iters)
            done_iters = it < P.max_iters ? it + (status == MMFFB_ST_SLOPE ? 0 : 1) : P.max_iters;
        __syncthreads();
        float *op = P.pos + coord;
        for (int k = tid; k < n; k += NT) op[k] = (float)x[k];
        if (tid == 0) {
            P.energy[conf] = (double)E;
            P.status[conf] = status;
            P.iters[conf] = done_iters;
            if (P.ls_evals) P.ls_evals[conf] = nevals;
        }
        __syncthreads();
    }
};

// CTAs per SM a kernel instance is compiled for (its register budget): 2 for the
// register-lean 256-thread dense BFGS instances (128 registers a thread, H columns
// read from shared memory) and for the register-capped L-BFGS instances (NC = 0,
// history in shared memory or in a global slot), 1 otherwise.  For L-BFGS, NC only
// selects the budget.
template <int NT, int NC, bool MSM, bool LB>
constexpr int min_ctas() {
    return (!LB && NC == 0 && NT <= 256) || (LB && NC == 0 && NT == 256) ? 2 : 1;
}

template <class R, class A, int NT, int NC, bool MSM, bool LB>
__global__ void __launch_bounds__(NT, (min_ctas<NT, NC, MSM, LB>())) minimize_kernel(const Params P) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_item;
    __shared__ int s_abort;
    Opt<R, A, NT, NC, MSM, LB> opt(P, smem, &s_abort);
    if (threadIdx.x == 0) s_abort = 0;
    if (!MSM && !LB) {
        if (threadIdx.x == 0) {
            for (int b = 0; b < (NT / 32) * kStages; ++b) mbar_init(&opt.mbar[b], 1);
            mbar_fence_init();
        }
    }
    __syncthreads();
    const int *order = P.c.order;
    const bool queue = P.q_tail != nullptr;
    for (;;) {
        if (threadIdx.x == 0) s_item = queue ? claim_slot(P) : atomicAdd(P.counter, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item < 0 || item >= P.c.n_conf) break;
        opt.run(queue || !order ? item : order[item]);
        if (queue && threadIdx.x == 0) {
            // the slot's results are written (run() ends with a barrier): flag it for the host
            __threadfence_system();
            *(volatile int *)&P.q_done[item] = 1;
        }
        // a copy never completed: stop taking work (the conformers left keep the
        // MMFFB_ST_TIMEOUT that prepare_minimize gave them; healthy CTAs go on)
        if (*(volatile int *)&s_abort) break;
    }
}

// ---------------------------------------------------------------------------
// Energy + gradient of every conformer (one CTA each)
// ---------------------------------------------------------------------------

template <class R, class A, int NT>
__global__ void __launch_bounds__(NT) energy_grad_kernel(const Params P, float *grad) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int NW = NT / 32;
    const int conf = blockIdx.x;
    Layout L = make_eval_layout(P.nmax, NW, sizeof(R), sizeof(A), P.b.max_classes);
    R *pos4 = (R *)(smem + L.pos4), *gbuf = (R *)(smem + L.gbuf);
    int *cls = (int *)(smem + L.cls);
    double *qa = (double *)(smem + L.q);
    float *qf = (float *)(smem + L.qf);
    uint32_t *mask = (uint32_t *)(smem + L.mask);
    float2 *tab = (float2 *)(smem + L.tab);
    A *red = (A *)(smem + L.red);
    const MolV m = load_mol(P.b.mol_desc, P.c.conf_mol[conf]);
    const int n = 3 * m.n, nv = (3 * P.nmax + 3) & ~3;
    const float *gp = P.pos + P.c.conf_coord[conf];
    for (int k = threadIdx.x; k < n; k += NT) pos4[4 * (k / 3) + (k % 3)] = (R)gp[k];
    stage_molecule<NT, sizeof(R) == 4>(P, m, cls, qa, qf, mask, tab);
    const MolSmem ms{cls, qa, qf, mask, tab};
    __syncthreads();
    A e[1], z[1] = {A(0)};
    if (grad) e[0] = eval_terms<R, A, NW, true, sizeof(R) == 4>(P, m, pos4, gbuf, ms, nv);
    else e[0] = eval_terms<R, A, NW, false, sizeof(R) == 4>(P, m, pos4, gbuf, ms, nv);
    block_reduce<NW, 1, 1, A>(e, z, red);
    if (grad) {
        float *go = grad + P.c.conf_coord[conf];
        for (int k = threadIdx.x; k < n; k += NT) {
            R s = R(0);
#pragma unroll
            for (int w = 0; w < NW; ++w) s += gbuf[(size_t)w * nv + k];
            go[k] = (float)s;
        }
    }
    if (threadIdx.x == 0) P.energy[conf] = (double)e[0];
}

// ---------------------------------------------------------------------------
// FP64 check of returned conformers: energy and gradient re-evaluated in FP64
// at the returned coordinates (one CTA per conformer)
// ---------------------------------------------------------------------------

template <int NT>
__global__ void __launch_bounds__(NT) check64_kernel(const Params P, const double *e_in, double *e64,
                                                     double *derr, double *grms) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int NW = NT / 32;
    const int conf = blockIdx.x;
    Layout L = make_eval_layout(P.nmax, NW, 8, 8, P.b.max_classes);
    double *pos4 = (double *)(smem + L.pos4), *gbuf = (double *)(smem + L.gbuf);
    int *cls = (int *)(smem + L.cls);
    double *qa = (double *)(smem + L.q);
    float *qf = (float *)(smem + L.qf);
    uint32_t *mask = (uint32_t *)(smem + L.mask);
    float2 *tab = (float2 *)(smem + L.tab);
    double *red = (double *)(smem + L.red);
    const MolV m = load_mol(P.b.mol_desc, P.c.conf_mol[conf]);
    const int n = 3 * m.n, nv = (3 * P.nmax + 3) & ~3;
    const float *gp = P.pos + P.c.conf_coord[conf];
    for (int k = threadIdx.x; k < n; k += NT) pos4[4 * (k / 3) + (k % 3)] = (double)gp[k];
    stage_molecule<NT, false>(P, m, cls, qa, qf, mask, tab);
    const MolSmem ms{cls, qa, qf, mask, tab};
    __syncthreads();
    double s[2], z[1] = {0.0};
    s[0] = eval_terms<double, double, NW, true, false>(P, m, pos4, gbuf, ms, nv);
    __syncthreads();
    s[1] = 0.0;
    for (int k = threadIdx.x; k < n; k += NT) {
        double g = 0.0;
#pragma unroll
        for (int w = 0; w < NW; ++w) g += gbuf[(size_t)w * nv + k];
        s[1] += g * g;
    }
    block_reduce<NW, 2, 1, double>(s, z, red);
    if (threadIdx.x == 0) {
        e64[conf] = s[0];
        if (derr) derr[conf] = e_in[conf] - s[0];
        if (grms) grms[conf] = n > 0 ? sqrt(s[1] / n) : 0.0;
    }
}

// launch plan of a minimisation
struct Plan {
    int nt, nc;
    bool msm;
    size_t smem;
    int grid;
    size_t gslot;      // matrix elements per CTA slot when not in shared memory
    size_t rsz;
};

template <class R, class A, int NT, int NC, bool MSM, bool LB>
int launch_min(const Params &P, const Plan &pl, cudaStream_t st) {
    auto k = minimize_kernel<R, A, NT, NC, MSM, LB>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    k<<<pl.grid, NT, pl.smem, st>>>(P);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "minimize_kernel launch");
    return 0;
}

template <class R, class A, int NT>
int launch_eg(const Params &P, float *grad, cudaStream_t st) {
    Layout L = make_eval_layout(P.nmax, NT / 32, sizeof(R), sizeof(A), P.b.max_classes);
    auto k = energy_grad_kernel<R, A, NT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    k<<<P.c.n_conf, NT, L.total, st>>>(P, grad);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "energy_grad_kernel launch");
    return 0;
}

template <class R, class A, int NT, int NC, bool MSM, bool LB>
int occ_min(const Plan &pl) {
    auto k = minimize_kernel<R, A, NT, NC, MSM, LB>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, NT, pl.smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    return n;
}

struct LaunchFn {
    const Params &P;
    const Plan &pl;
    cudaStream_t st;
    template <class R, class A, int NT, int NC, bool MSM, bool LB> int run() const {
        return launch_min<R, A, NT, NC, MSM, LB>(P, pl, st);
    }
};

struct OccFn {
    const Plan &pl;
    template <class R, class A, int NT, int NC, bool MSM, bool LB> int run() const {
        return occ_min<R, A, NT, NC, MSM, LB>(pl);
    }
};

// per-precision instantiation units (mmff_inst_*.cu)
int minimize_mixed(const Params &P, const Plan &pl, cudaStream_t st);
int minimize_fp64(const Params &P, const Plan &pl, cudaStream_t st);
int minimize_fp32(const Params &P, const Plan &pl, cudaStream_t st);
int occupancy_mixed(const Plan &pl, bool lb);
int occupancy_fp64(const Plan &pl, bool lb);
int occupancy_fp32(const Plan &pl, bool lb);
int energy_grad_mixed(const Params &P, float *grad, cudaStream_t st);
int energy_grad_fp64(const Params &P, float *grad, cudaStream_t st);
int energy_grad_fp32(const Params &P, float *grad, cudaStream_t st);
int check_fp64(const Params &P, const double *e_in, double *e64, double *derr, double *grms, cudaStream_t st);

// argument checks and launch planning shared by the C ABI entry points (mmff_capi.cu)
int check_batch(const MMFFBatchDev *b, const MMFFConfDev *c);
int check_opt(const MMFFOptParams *o);
TermMode to_mode(const double *mode);
KConst to_consts(const double *k);
int plan_minimize(const MMFFBatchDev *b, const MMFFConfDev *c, const MMFFOptParams *o, Plan *pl);
// Params of a minimisation from the options and the caller's buffers (counter and
// error word in the scratch head, matrix slots from byte 256 of mats).
Params make_params(const MMFFBatchDev *b, const MMFFConfDev *c, const MMFFOptParams *o, const Plan &pl,
                   float *pos, double *energy, int32_t *status, int32_t *iters, int32_t *ls_evals,
                   unsigned char *scratch);
// Stream-ordered start of a minimisation: zero the work counter and the error word and
// mark each of the call's conformers MMFFB_ST_TIMEOUT (energy NaN, 0 iterations), so that a
// conformer no CTA reaches after a bounded wait gave up still has a defined result.
int prepare_minimize(const Params &P, cudaStream_t st);

}  // namespace mmffb
