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
