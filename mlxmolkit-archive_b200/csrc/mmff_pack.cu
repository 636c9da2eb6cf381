// Host-side packing helper: the chunk assignment of bonded terms (no device work).
//
// A chunk holds at most 32 terms of one type and, per role (first atom,
// second atom, ...), no atom twice, so the kernels can scatter the 32 terms'
// gradients of one role without atomics.  Terms are placed greedily, first fit
// in term order; a term that does not fit an open chunk in its given
// orientation may enter it in its equivalent reversed form.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mmffb200.h"

namespace {

constexpr int kChunk = 32;

struct Chunks {
    int roles, words;
    std::vector<uint64_t> used;   // chunk-major: roles x words bitset of atoms per chunk
    std::vector<int> fill;

    bool fits(int c, const int *atoms) const {
        const uint64_t *u = used.data() + (size_t)c * roles * words;
        for (int r = 0; r < roles; ++r) {
            const int a = atoms[r];
            if (u[(size_t)r * words + (a >> 6)] >> (a & 63) & 1u) return false;
        }
        return true;
    }
    void add(int c, const int *atoms) {
        uint64_t *u = used.data() + (size_t)c * roles * words;
        for (int r = 0; r < roles; ++r) {
            const int a = atoms[r];
            u[(size_t)r * words + (a >> 6)] |= uint64_t(1) << (a & 63);
        }
        ++fill[c];
    }
    int open_new() {
        fill.push_back(0);
        used.resize(used.size() + (size_t)roles * words, 0);
        return (int)fill.size() - 1;
    }
};

}  // namespace

extern "C" int32_t mmffb_pack_chunk(int32_t n_terms, int32_t roles, const int32_t *role_atoms,
                                    const int32_t *flip_perm, int32_t n_atoms, int64_t *chunk_out,
                                    uint8_t *flipped_out) {
    if (n_terms < 0 || roles < 1 || roles > 8 || n_atoms < 0 || (n_terms > 0 && (!role_atoms || !chunk_out)))
        return MMFFB_EINVAL;
    Chunks ch;
    ch.roles = roles;
    ch.words = (n_atoms + 63) / 64 > 0 ? (n_atoms + 63) / 64 : 1;
    int first_open = 0;
    int forms[2][8];
    for (int t = 0; t < n_terms; ++t) {
        const int32_t *a = role_atoms + (size_t)t * roles;
        for (int r = 0; r < roles; ++r) {
            if (a[r] < 0 || a[r] >= n_atoms) return MMFFB_EINVAL;
            forms[0][r] = a[r];
            if (flip_perm) forms[1][r] = a[flip_perm[r]];
        }
        const int nforms = flip_perm ? 2 : 1;
        const int nch = (int)ch.fill.size();
        int c = first_open, pick = -1;
        for (; c < nch; ++c) {
            if (ch.fill[c] >= kChunk) continue;
            for (int f = 0; f < nforms; ++f)
                if (ch.fits(c, forms[f])) { pick = f; break; }
            if (pick >= 0) break;
        }
        if (c == nch) {
            c = ch.open_new();
            pick = 0;
        }
        ch.add(c, forms[pick]);
        chunk_out[t] = c;
        if (flipped_out) flipped_out[t] = (uint8_t)(pick == 1);
        while (first_open < (int)ch.fill.size() && ch.fill[first_open] >= kChunk) ++first_open;
    }
    return (int32_t)ch.fill.size();
}

// ---------------------------------------------------------------------------
// Whole-batch packing on host threads (mmffb_pack_begin / _finish): the same
// tables, bit for bit, as mlxmolkit_b200/pack.py's pack_molecules.
// ---------------------------------------------------------------------------

#include <algorithm>
#include <atomic>
#include <string>
#include <thread>

namespace mmffb {
int fail(int code, const char *fmt, ...);
}

namespace {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kMaxPackAtoms = 1024;
constexpr int kMaxClasses = 64;

inline uint32_t f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline uint32_t pack16(int a, int b) { return ((uint32_t)a & 0xFFFFu) | ((uint32_t)b << 16); }

// One molecule's tables.
struct MolPack {
    int n = 0, ncls = 0, diel = 1;
    int64_t nch[5] = {0, 0, 0, 0, 0};
    std::vector<uint32_t> bonded;     // rows x 4, the five term types in order
    std::vector<int32_t> cls;
    std::vector<double> q;
    std::vector<float> tab;           // ncls x ncls x 2
    std::vector<uint32_t> mask;       // n x W pair words, then n x W 1-4 words
    std::string err;
};

// Greedy first-fit chunk ids (and orientation) of T terms with R roles, as mmffb_pack_chunk.
int chunk_terms(int T, int R, const int *atoms, const int *flip, int n_atoms, std::vector<int64_t> &cid,
                std::vector<uint8_t> &fl) {
    cid.resize(T);
    fl.resize(T);
    if (T == 0) return 0;
    return mmffb_pack_chunk(T, R, atoms, flip, n_atoms, cid.data(), fl.data());
}

// Scatter per-term records (h halves of 4 words) into chunks of 32 (pack.py _place):
// chunk c, half q, slot s at row (c * h + q) * 32 + s; empty slots: first word kInvalid
// in half 0, zeros elsewhere.
void place(const std::vector<int64_t> &cid, int nch, int h, const std::vector<uint32_t> &rec,
           std::vector<uint32_t> &out) {
    const size_t base = out.size();
    out.resize(base + (size_t)nch * h * 32 * 4, 0u);
    uint32_t *o = out.data() + base;
    for (int c = 0; c < nch; ++c)
        for (int s = 0; s < 32; ++s) o[((size_t)c * h * 32 + s) * 4] = kInvalid;
    std::vector<int> slot(nch, 0);
    for (size_t t = 0; t < cid.size(); ++t) {
        const int c = (int)cid[t], s = slot[c]++;
        for (int qh = 0; qh < h; ++qh)
            for (int w = 0; w < 4; ++w) o[(((size_t)c * h + qh) * 32 + s) * 4 + w] = rec[(t * h + qh) * 4 + w];
    }
}

bool pack_one(const MMFFTermsHost &T, int m, int64_t atom0, MolPack &P) {
    const int64_t *ts = T.term_start + 7 * (int64_t)m, *te = ts + 7;
    const int n = T.n_atoms[m];
    P.n = n;
    P.diel = T.diel[m] == 2 ? 2 : 1;
    if (n > kMaxPackAtoms) {
        P.err = "molecule of " + std::to_string(n) + " atoms exceeds " + std::to_string(kMaxPackAtoms);
        return false;
    }
    std::vector<int> at;
    std::vector<int64_t> cid;
    std::vector<uint8_t> fl;
    std::vector<uint32_t> rec;
    auto range_ok = [&](const int32_t *a, int64_t b, int64_t e) {
        for (int64_t k = b; k < e; ++k)
            if (a[k] < 0 || a[k] >= n) return false;
        return true;
    };
    // bonded term types: roles, reversal permutation, halves
    static const int roles[5] = {2, 3, 3, 4, 4};
    static const int flips[5][4] = {{1, 0}, {2, 1, 0}, {2, 1, 0}, {2, 1, 0, 3}, {3, 2, 1, 0}};
    static const int halves[5] = {1, 1, 2, 1, 2};
    const int32_t *idx[5][4] = {{T.bond_i, T.bond_j}, {T.angle_i, T.angle_j, T.angle_k},
                                {T.sb_i, T.sb_j, T.sb_k}, {T.oop_i, T.oop_j, T.oop_k, T.oop_l},
                                {T.tor_i, T.tor_j, T.tor_k, T.tor_l}};
    for (int ty = 0; ty < 5; ++ty) {
        const int64_t b = ts[ty], e = te[ty], cnt = e - b;
        const int R = roles[ty], h = halves[ty];
        at.resize((size_t)cnt * R);
        int amax = -1;
        for (int r = 0; r < R; ++r) {
            if (!range_ok(idx[ty][r], b, e)) {
                P.err = "atom index out of range in term type " + std::to_string(ty);
                return false;
            }
            for (int64_t k = 0; k < cnt; ++k) {
                at[(size_t)k * R + r] = idx[ty][r][b + k];
                amax = std::max(amax, (int)idx[ty][r][b + k]);
            }
        }
        const int nch = chunk_terms((int)cnt, R, at.data(), flips[ty], amax + 1, cid, fl);
        if (nch < 0) {
            P.err = "chunking failed";
            return false;
        }
        rec.assign((size_t)cnt * h * 4, 0u);
        for (int64_t k = 0; k < cnt; ++k) {
            const int64_t g = b + k;
            const bool f = fl[k] != 0;
            uint32_t *r0 = &rec[(size_t)k * h * 4], *r1 = r0 + 4;
            switch (ty) {
            case 0: {
                const int i = T.bond_i[g], j = T.bond_j[g];
                r0[0] = f ? pack16(j, i) : pack16(i, j);
                r0[1] = f2u(T.bond_kb[g]); r0[2] = f2u(T.bond_r0[g]);
                break;
            }
            case 1: {
                const int i = T.angle_i[g], j = T.angle_j[g], k3 = T.angle_k[g];
                r0[0] = pack16(f ? k3 : i, j);
                r0[1] = pack16(f ? i : k3, T.angle_linear[g] != 0 ? 1 : 0);
                r0[2] = f2u(T.angle_ka[g]); r0[3] = f2u(T.angle_theta0[g]);
                break;
            }
            case 2: {
                const int i = T.sb_i[g], j = T.sb_j[g], k3 = T.sb_k[g];
                r0[0] = pack16(f ? k3 : i, j);
                r0[1] = (uint32_t)(f ? i : k3);
                r0[2] = f2u(f ? T.sb_r0_kj[g] : T.sb_r0_ij[g]);
                r0[3] = f2u(f ? T.sb_r0_ij[g] : T.sb_r0_kj[g]);
                r1[0] = f2u(T.sb_theta0[g]);
                r1[1] = f2u(f ? T.sb_kba_kji[g] : T.sb_kba_ijk[g]);
                r1[2] = f2u(f ? T.sb_kba_ijk[g] : T.sb_kba_kji[g]);
                break;
            }
            case 3: {
                const int i = T.oop_i[g], j = T.oop_j[g], k3 = T.oop_k[g], l = T.oop_l[g];
                r0[0] = pack16(f ? k3 : i, j);
                r0[1] = pack16(f ? i : k3, l);
                r0[2] = f2u(T.oop_koop[g]);
                break;
            }
            default: {
                const int i = T.tor_i[g], j = T.tor_j[g], k3 = T.tor_k[g], l = T.tor_l[g];
                r0[0] = f ? pack16(l, k3) : pack16(i, j);
                r0[1] = f ? pack16(j, i) : pack16(k3, l);
                r0[2] = f2u(T.tor_v1[g]); r0[3] = f2u(T.tor_v2[g]);
                r1[0] = f2u(T.tor_v3[g]);
                break;
            }
            }
        }
        place(cid, nch, h, rec, P.bonded);
        P.nch[ty] = nch;
    }

    // non-bonded: classes from the sorted distinct atom types, verified class table,
    // per-atom charge, and the pair / 1-4 bit rows (pack.py _nonbonded)
    const int64_t *types = T.atom_type + atom0;
    std::vector<int64_t> uniq(types, types + n);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    const int ncls = (int)uniq.size();
    if (ncls > kMaxClasses) {
        P.err = "molecule with " + std::to_string(ncls) + " non-bonded classes exceeds 64";
        return false;
    }
    P.ncls = ncls;
    P.cls.resize(n);
    P.q.resize(n);
    for (int a = 0; a < n; ++a) {
        P.cls[a] = (int32_t)(std::lower_bound(uniq.begin(), uniq.end(), types[a]) - uniq.begin());
        const double q = T.atom_charge[atom0 + a];
        P.q[a] = std::fabs(q) <= 1e-10 ? 0.0 : q;
    }
    P.tab.assign((size_t)ncls * ncls * 2, 0.f);
    std::vector<uint8_t> seen((size_t)ncls * ncls, 0);
    for (int c = 0; c < ncls * ncls; ++c) P.tab[2 * (size_t)c] = 1.0f;
    const int64_t vb = ts[5], ve = te[5], eb = ts[6], ee = te[6];
    if (!range_ok(T.vdw_i, vb, ve) || !range_ok(T.vdw_j, vb, ve) || !range_ok(T.ele_i, eb, ee) ||
        !range_ok(T.ele_j, eb, ee)) {
        P.err = "non-bonded atom index out of range";
        return false;
    }
    for (int64_t k = vb; k < ve; ++k) {
        const int ci = P.cls[T.vdw_i[k]], cj = P.cls[T.vdw_j[k]];
        for (int s = 0; s < 2; ++s) {
            const size_t c = s == 0 ? (size_t)ci * ncls + cj : (size_t)cj * ncls + ci;
            if (!seen[c]) {
                seen[c] = 1;
                P.tab[2 * c] = T.vdw_rstar[k];
                P.tab[2 * c + 1] = T.vdw_eps[k];
            }
        }
    }
    for (int64_t k = vb; k < ve; ++k) {
        const int ci = P.cls[T.vdw_i[k]], cj = P.cls[T.vdw_j[k]];
        const size_t c1 = (size_t)ci * ncls + cj, c2 = (size_t)cj * ncls + ci;
        const uint32_t r = f2u(T.vdw_rstar[k]), e = f2u(T.vdw_eps[k]);
        if (f2u(P.tab[2 * c1]) != r || f2u(P.tab[2 * c1 + 1]) != e || f2u(P.tab[2 * c2]) != r ||
            f2u(P.tab[2 * c2 + 1]) != e) {
            P.err = "vdW pair parameters are not a symmetric function of the atom types";
            return false;
        }
    }
    const int W = (n + 31) / 32;
    P.mask.assign((size_t)2 * n * W, 0u);
    uint32_t *pm = P.mask.data(), *p14 = pm + (size_t)n * W;
    auto bit = [&](const uint32_t *rows, int i, int j) { return (rows[(size_t)i * W + (j >> 5)] >> (j & 31)) & 1u; };
    for (int64_t k = vb; k < ve; ++k) {
        const int a = T.vdw_i[k], b = T.vdw_j[k];
        if (a == b) {
            P.err = "self pair in the vdW list";
            return false;
        }
        const int lo = std::min(a, b), hi = std::max(a, b);
        pm[(size_t)lo * W + (hi >> 5)] |= 1u << (hi & 31);
    }
    std::vector<uint32_t> ele((size_t)n * W, 0u);
    for (int64_t k = eb; k < ee; ++k) {
        const int a = T.ele_i[k], b = T.ele_j[k];
        const int lo = std::min(a, b), hi = std::max(a, b);
        if (!bit(pm, lo, hi)) {
            P.err = "electrostatic pair without a vdW pair";
            return false;
        }
        if (f2u((float)(P.q[a] * P.q[b])) != f2u(T.ele_charge[k])) {
            P.err = "electrostatic charge terms are not float32(q_i * q_j)";
            return false;
        }
        ele[(size_t)lo * W + (hi >> 5)] |= 1u << (hi & 31);
    }
    for (int i = 0; i < n; ++i)
        for (int w = 0; w < W; ++w) {
            uint32_t only = pm[(size_t)i * W + w] & ~ele[(size_t)i * W + w];
            while (only) {
                const int j = w * 32 + __builtin_ctz(only);
                only &= only - 1;
                if (P.q[i] * P.q[j] != 0.0) {
                    P.err = "vdW-only pair with a non-zero charge product";
                    return false;
                }
            }
        }
    for (int64_t k = eb; k < ee; ++k) {   // in list order: a repeated pair keeps its last flag
        const int a = T.ele_i[k], b = T.ele_j[k];
        const int lo = std::min(a, b), hi = std::max(a, b);
        uint32_t &wd = p14[(size_t)lo * W + (hi >> 5)];
        if (T.ele_is14[k] != 0) wd |= 1u << (hi & 31);
        else wd &= ~(1u << (hi & 31));
    }
    return true;
}

struct PackHandle {
    std::vector<MolPack> mols;
    MMFFPackSizes sizes;
};

}  // namespace

extern "C" void *mmffb_pack_begin(const MMFFTermsHost *terms, int32_t n_threads, MMFFPackSizes *sizes) {
    if (!terms || !sizes || terms->n_mols < 0 || (terms->n_mols > 0 && (!terms->n_atoms || !terms->diel ||
                                                                        !terms->term_start || !terms->atom_type ||
                                                                        !terms->atom_charge))) {
        mmffb::fail(MMFFB_EINVAL, "null or negative argument");
        return nullptr;
    }
    const int M = terms->n_mols;
    PackHandle *h = new PackHandle();
    h->mols.resize(M);
    std::vector<int64_t> atom0(M + 1, 0);
    for (int m = 0; m < M; ++m) atom0[m + 1] = atom0[m] + terms->n_atoms[m];
    int nt = n_threads > 0 ? n_threads : (int)std::thread::hardware_concurrency();
    nt = std::max(1, std::min(nt, std::max(1, M / 8)));
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            const int m0 = next.fetch_add(16);
            if (m0 >= M) break;
            for (int m = m0; m < std::min(M, m0 + 16); ++m) pack_one(*terms, m, atom0[m], h->mols[m]);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    MMFFPackSizes s = {0, 0, 0, 0};
    for (int m = 0; m < M; ++m) {
        const MolPack &P = h->mols[m];
        if (!P.err.empty()) {
            mmffb::fail(MMFFB_EINVAL, "molecule %d: %s", m, P.err.c_str());
            delete h;
            return nullptr;
        }
        s.bonded_rows += (int64_t)P.bonded.size() / 4;
        s.atoms += P.n;
        s.cls_pairs += (int64_t)P.tab.size() / 2;
        s.mask_words += (int64_t)P.mask.size();
    }
    if (s.bonded_rows == 0) s.bonded_rows = 1;      // one invalid record
    if (M == 0) {
        s.cls_pairs = 1;
        s.mask_words = 1;
    }
    h->sizes = s;
    *sizes = s;
    return h;
}

extern "C" int mmffb_pack_finish(void *handle, int32_t *mol_desc, uint32_t *bonded, int32_t *atom_cls, double *atom_q,
                                 float *cls_tab, uint32_t *pair_mask) {
    PackHandle *h = static_cast<PackHandle *>(handle);
    if (!h) return mmffb::fail(MMFFB_EINVAL, "null pack handle");
    if (!mol_desc || !bonded || !atom_cls || !atom_q || !cls_tab || !pair_mask) {
        delete h;
        return mmffb::fail(MMFFB_EINVAL, "null output array");
    }
    const int M = (int)h->mols.size();
    int64_t rec = 0, atom = 0, tab = 0, mask = 0;
    for (int m = 0; m < M; ++m) {
        const MolPack &P = h->mols[m];
        int32_t *d = mol_desc + (size_t)m * MMFFB_MOL_DESC_INTS;
        std::memset(d, 0, MMFFB_MOL_DESC_INTS * sizeof(int32_t));
        d[MMFFB_MD_N] = P.n;
        d[MMFFB_MD_ATOM_OFF] = (int32_t)atom;
        d[MMFFB_MD_NCLS] = P.ncls;
        d[MMFFB_MD_CLS_OFF] = (int32_t)tab;
        d[MMFFB_MD_MASK_OFF] = (int32_t)mask;
        d[MMFFB_MD_DIEL] = P.diel;
        static const int halves[5] = {1, 1, 2, 1, 2};
        int64_t r = rec;
        for (int t = 0; t < 5; ++t) {
            d[MMFFB_MD_B_OFF + 2 * t] = (int32_t)r;
            d[MMFFB_MD_B_NCH + 2 * t] = (int32_t)P.nch[t];
            r += P.nch[t] * halves[t] * 32;
        }
        std::memcpy(bonded + 4 * rec, P.bonded.data(), P.bonded.size() * 4);
        std::memcpy(atom_cls + atom, P.cls.data(), P.cls.size() * 4);
        std::memcpy(atom_q + atom, P.q.data(), P.q.size() * 8);
        std::memcpy(cls_tab + 2 * tab, P.tab.data(), P.tab.size() * 4);
        std::memcpy(pair_mask + mask, P.mask.data(), P.mask.size() * 4);
        rec += (int64_t)P.bonded.size() / 4;
        atom += P.n;
        tab += (int64_t)P.tab.size() / 2;
        mask += (int64_t)P.mask.size();
    }
    if (rec == 0) bonded[0] = bonded[1] = bonded[2] = bonded[3] = kInvalid;   // one invalid record
    if (M == 0) {
        cls_tab[0] = cls_tab[1] = 0.f;
        pair_mask[0] = 0;
    }
    delete h;
    return 0;
}

extern "C" void mmffb_pack_free(void *handle) { delete static_cast<PackHandle *>(handle); }
