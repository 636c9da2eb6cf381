// The reference's multi-molecule L-BFGS (mlxmolkit/mmff_metal_optimizer.py:217-535) as
// device-resident chunks.  One launch advances every conformer (one CTA each) by up to
// eval_freq iterations of:
//
//   d   = -two_loop(g)                 g = grad_scale * dE/dx, history oldest first (:47-74)
//   d_a = d_a * min(max_step / |d_a|, 1) for every atom a          per-atom step cap (:366-373)
//   x'  = x + d;  E', g' at x'          mega-kernel constants (mmff_metal_kernel.py:274-280)
//   s = x' - x, y = g' - g, rho = 1/(s.y) if s.y > 1e-10 else 0; push (s, y, rho) (:378-392)
//
// with no line search.  At the caller's check points (every eval_freq iterations) the
// kernel keeps the best-seen positions and energy and tests the largest per-atom norm
// of g against grad_tol (:394-408, :470-483).  Positions, gradient, history and the
// best-seen state stay in device memory between launches; the host only reads the count
// of conformers still over grad_tol to stop the batch, as the reference does.
#include <cstring>

#include "mmff_kernels.cuh"

namespace mmffb {
namespace {

constexpr double kEpsCurv = 1e-10;   // mmff_metal_optimizer.py:31

struct MMArgs {
    Params P;                  // batch, conformers, term mode, positions (the state's x)
    MMFFMultiMolState S;
    int hist_m;
    float grad_scale, max_step, grad_tol;
    int phase, n_iters, it_end, max_iters;
    int nv;                    // history row stride
};

template <int NW>
__device__ __forceinline__ double block_sum(double v, double *red) {
    double s[1] = {v}, z[1] = {0.0};
    block_reduce<NW, 1, 1, double>(s, z, red);
    return s[0];
}

template <int NT>
__global__ void __launch_bounds__(NT) multimol_kernel(const MMArgs a) {
    constexpr int NW = NT / 32;
    extern __shared__ __align__(16) unsigned char smem[];
    const Params &P = a.P;
    Layout L = make_layout(P.nmax, NW, 1, true, sizeof(float), sizeof(double), P.b.max_classes);
    float *pos4 = (float *)(smem + L.pos4), *gbuf = (float *)(smem + L.gbuf);
    float *xv = (float *)(smem + L.x), *gv = (float *)(smem + L.g), *dv = (float *)(smem + L.dir);
    float *qv = (float *)(smem + L.hq);
    int *cls = (int *)(smem + L.cls);
    double *qa = (double *)(smem + L.q);
    float *qf = (float *)(smem + L.qf);
    uint32_t *mask = (uint32_t *)(smem + L.mask);
    float2 *tab = (float2 *)(smem + L.tab);
    double *red0 = (double *)(smem + L.red), *red1 = red0 + NW * 8;
    double *alpha = (double *)(smem + L.alpha);
    int rsel = 0;
    auto red = [&]() { rsel ^= 1; return rsel ? red1 : red0; };

    const int conf = blockIdx.x, tid = threadIdx.x;
    const MolV m = load_mol(P.b.mol_desc, P.c.conf_mol[conf]);
    const int N = m.n, n = 3 * N, nv = (3 * P.nmax + 3) & ~3;
    const int64_t off = P.c.conf_coord[conf];
    float *X = a.S.x + off, *G = a.S.g + off, *BX = a.S.best_x + off;
    float *Sh = a.S.hist + (size_t)conf * 2 * a.hist_m * a.nv, *Yh = Sh + (size_t)a.hist_m * a.nv;
    float *rho = a.S.rho + (size_t)conf * a.hist_m;
    stage_molecule<NT, true>(P, m, cls, qa, qf, mask, tab);
    const MolSmem ms{cls, qa, qf, mask, tab};

    // energy and scaled gradient at xv (into e, gv)
    auto eval = [&](double &e) {
        for (int k = tid; k < n; k += NT) pos4[4 * (k / 3) + (k % 3)] = xv[k];
        __syncthreads();
        const double ep = eval_terms<float, double, NW, true, true>(P, m, pos4, gbuf, ms, nv);
        __syncthreads();
        for (int k = tid; k < n; k += NT) {
            float s = 0.f;
#pragma unroll
            for (int w = 0; w < NW; ++w) s += gbuf[(size_t)w * nv + k];
            gv[k] = s * a.grad_scale;
        }
        e = block_sum<NW>(ep, red());
    };

    double e = 0.0;
    int hcount = 0;
    if (a.phase == MMFFB_MM_START || a.phase == MMFFB_MM_REVERT) {
        const float *src = a.phase == MMFFB_MM_REVERT ? BX : X;
        for (int k = tid; k < n; k += NT) xv[k] = src[k];
        eval(e);
        for (int k = tid; k < n; k += NT) {
            X[k] = xv[k];
            G[k] = gv[k];
            if (a.phase == MMFFB_MM_START) BX[k] = xv[k];
        }
        if (tid == 0) {
            a.S.e[conf] = e;
            a.S.hcount[conf] = 0;
            if (a.phase == MMFFB_MM_START) {
                a.S.best_e[conf] = e;
                a.S.converged[conf] = 0;
                a.S.conv_iter[conf] = a.max_iters;
            }
        }
        return;
    }

    for (int k = tid; k < n; k += NT) { xv[k] = X[k]; gv[k] = G[k]; }
    e = a.S.e[conf];
    hcount = a.S.hcount[conf];
    __syncthreads();
    const int M = a.hist_m;
    for (int it = 0; it < a.n_iters; ++it) {
        // two-loop recursion over the pairs held, oldest first (_lbfgs_direction_batch)
        const int h = hcount < M ? hcount : M, first = hcount - h;
        for (int k = tid; k < n; k += NT) qv[k] = gv[k];
        __syncthreads();
        for (int i = h - 1; i >= 0; --i) {
            const int sl = (first + i) % M;
            const float *s_i = Sh + (size_t)sl * a.nv, *y_i = Yh + (size_t)sl * a.nv;
            double t = 0.0;
            for (int k = tid; k < n; k += NT) t += (double)s_i[k] * qv[k];
            const double ai = (double)rho[sl] * block_sum<NW>(t, red());
            if (tid == 0) alpha[i] = ai;
            const float af = (float)ai;
            for (int k = tid; k < n; k += NT) qv[k] -= af * y_i[k];
            __syncthreads();
        }
        double gamma = 1.0;
        if (h > 0) {
            const int sl = (first + h - 1) % M;
            const float *s_l = Sh + (size_t)sl * a.nv, *y_l = Yh + (size_t)sl * a.nv;
            double sy[2] = {0.0, 0.0}, z[1] = {0.0};
            for (int k = tid; k < n; k += NT) {
                sy[0] += (double)s_l[k] * y_l[k];
                sy[1] += (double)y_l[k] * y_l[k];
            }
            block_reduce<NW, 2, 1, double>(sy, z, red());
            gamma = sy[0] / (sy[1] + 1e-30);
        }
        const float gf = (float)gamma;
        for (int k = tid; k < n; k += NT) qv[k] *= gf;      // r = gamma * q
        __syncthreads();
        for (int i = 0; i < h; ++i) {
            const int sl = (first + i) % M;
            const float *s_i = Sh + (size_t)sl * a.nv, *y_i = Yh + (size_t)sl * a.nv;
            double t = 0.0;
            for (int k = tid; k < n; k += NT) t += (double)y_i[k] * qv[k];
            const double beta = (double)rho[sl] * block_sum<NW>(t, red());
            const float c = (float)(alpha[i] - beta);
            for (int k = tid; k < n; k += NT) qv[k] += s_i[k] * c;
            __syncthreads();
        }
        // per-atom step cap, x' = x + d, s = x' - x
        for (int at = tid; at < N; at += NT) {
            const float d0 = -qv[3 * at], d1 = -qv[3 * at + 1], d2 = -qv[3 * at + 2];
            const float disp = sqrtf(d0 * d0 + d1 * d1 + d2 * d2 + 1e-30f);
            const float f = fminf(a.max_step / disp, 1.0f);
            const float dd[3] = {d0 * f, d1 * f, d2 * f};
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int k = 3 * at + q;
                const float xn = xv[k] + dd[q];
                dv[k] = xn - xv[k];
                xv[k] = xn;
            }
        }
        __syncthreads();
        for (int k = tid; k < n; k += NT) qv[k] = gv[k];   // g before the step
        __syncthreads();
        eval(e);
        // history: s = x' - x, y = g' - g, rho = 1/(s.y) when s.y > EPS_CURV
        const int sl = hcount % M;
        float *s_n = Sh + (size_t)sl * a.nv, *y_n = Yh + (size_t)sl * a.nv;
        double t = 0.0;
        for (int k = tid; k < n; k += NT) {
            const float y = gv[k] - qv[k];
            s_n[k] = dv[k];
            y_n[k] = y;
            t += (double)dv[k] * y;
        }
        const double sy = block_sum<NW>(t, red());
        if (tid == 0) rho[sl] = sy > kEpsCurv ? (float)(1.0 / (sy + 1e-30)) : 0.f;
        ++hcount;
        __threadfence_block();
        __syncthreads();
    }
    // state back, then the check point (best-seen guard and convergence test)
    for (int k = tid; k < n; k += NT) { X[k] = xv[k]; G[k] = gv[k]; }
    if (tid == 0) {
        a.S.e[conf] = e;
        a.S.hcount[conf] = hcount;
    }
    if (a.phase == MMFFB_MM_MAIN_CHECK || a.phase == MMFFB_MM_POLISH_CHECK) {
        double mx[1] = {0.0}, z[1] = {0.0};
        for (int at = tid; at < N; at += NT) {
            const double g0 = gv[3 * at], g1 = gv[3 * at + 1], g2 = gv[3 * at + 2];
            const double v = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
            mx[0] = v > mx[0] ? v : mx[0];
        }
        block_reduce<NW, 1, 1, double>(z, mx, red());
        const bool improved = e < a.S.best_e[conf];
        if (improved)
            for (int k = tid; k < n; k += NT) BX[k] = xv[k];
        __syncthreads();
        if (tid == 0) {
            if (improved) a.S.best_e[conf] = e;
            const bool under = mx[0] <= (double)a.grad_tol;
            if (a.phase == MMFFB_MM_MAIN_CHECK) {
                int cv = a.S.converged[conf];
                if (!cv && under) {
                    cv = 1;
                    a.S.converged[conf] = 1;
                    a.S.conv_iter[conf] = a.it_end;
                }
                if (!cv) atomicAdd(a.S.pending, 1);
            } else if (!under) {
                atomicAdd(a.S.pending, 1);
            }
        }
    }
}

}  // namespace
}  // namespace mmffb

using namespace mmffb;

extern "C" size_t mmffb_multimol_hist_floats(const MMFFConfDev *confs, int32_t history_m) {
    if (!confs || history_m < 1 || confs->max_atoms < 1) return 0;
    return (size_t)2 * history_m * (size_t)((3 * confs->max_atoms + 3) & ~3);
}

extern "C" int mmffb_multimol_step(const MMFFBatchDev *batch, const MMFFConfDev *confs,
                                   const MMFFMultiMolParams *prm, const MMFFMultiMolState *state,
                                   int32_t phase, int32_t n_iters, int32_t it_end, int32_t max_iters,
                                   mmffb_stream_t stream) {
    int r = check_batch(batch, confs);
    if (r) return r;
    if (!prm || !state) return fail(MMFFB_EINVAL, "null parameters or state");
    if (phase < MMFFB_MM_START || phase > MMFFB_MM_POLISH_CHECK)
        return fail(MMFFB_EINVAL, "unknown multimol phase %d", phase);
    if (prm->history_m < 1 || prm->history_m > kMaxHist)
        return fail(MMFFB_EINVAL, "history_m must be in 1..%d", kMaxHist);
    if (n_iters < 0) return fail(MMFFB_EINVAL, "n_iters must be >= 0");
    if (confs->n_conf == 0) return 0;
    const MMFFMultiMolState &S = *state;
    if (!S.x || !S.g || !S.best_x || !S.e || !S.best_e || !S.hist || !S.rho || !S.hcount || !S.converged ||
        !S.conv_iter || !S.pending)
        return fail(MMFFB_EINVAL, "null pointer in the multimol state");
    MMArgs a;
    memset(&a, 0, sizeof a);
    a.P.b = *batch;
    a.P.c = *confs;
    a.P.md = to_mode(prm->mode);
    a.P.nmax = confs->max_atoms;
    a.P.pos = S.x;
    a.S = S;
    a.hist_m = prm->history_m;
    a.grad_scale = prm->grad_scale;
    a.max_step = prm->max_step_per_atom;
    a.grad_tol = prm->grad_tol;
    a.phase = phase;
    a.n_iters = n_iters;
    a.it_end = it_end;
    a.max_iters = max_iters;
    a.nv = (3 * confs->max_atoms + 3) & ~3;
    if (prm->threads != 0 && prm->threads != 64 && prm->threads != 128 && prm->threads != 256)
        return fail(MMFFB_EINVAL, "threads must be 0, 64, 128 or 256");
    int dev = 0, optin = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(smem)");
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
    // Threads per conformer: as given, else the largest instance whose resident CTAs hold every
    // conformer (one wave per launch), else 64 (the most CTAs per wave).
    int nt = prm->threads;
    size_t smem = 0;
    for (int cand = prm->threads ? prm->threads : 256; cand >= 64; cand /= 2) {
        const Layout L = make_layout(confs->max_atoms, cand / 32, 1, true, sizeof(float), sizeof(double),
                                     batch->max_classes);
        if (L.total > (size_t)optin) continue;
        const void *fn = cand == 256 ? (const void *)&multimol_kernel<256>
                         : cand == 128 ? (const void *)&multimol_kernel<128> : (const void *)&multimol_kernel<64>;
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        int occ = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, cand, L.total);
        if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        nt = cand;
        smem = L.total;
        if (prm->threads || (long long)sms * occ >= confs->n_conf) break;
    }
    if (smem == 0)
        return fail(MMFFB_ETOOBIG, "molecule of %d atoms does not fit the multimol kernel's shared memory",
                    confs->max_atoms);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (nt == 256) multimol_kernel<256><<<confs->n_conf, 256, smem, st>>>(a);
    else if (nt == 128) multimol_kernel<128><<<confs->n_conf, 128, smem, st>>>(a);
    else multimol_kernel<64><<<confs->n_conf, 64, smem, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "multimol_kernel launch");
    return 0;
}
