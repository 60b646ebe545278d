// Host check of the slot and tile tables before they reach the device.
//
// The matvec kernels index through these tables without bounds checks: the
// slot permutation, the box and group offsets, the tile table (group pair,
// first slots, sizes, data offset, partial-sum slot of the transposed product)
// and the partial-sum slot bases.  check_layout verifies, once per layout,
// every property the kernels' indexing relies on, so that an inconsistent
// table becomes an error status instead of an out-of-range access.
#pragma once
#include <cstdio>
#include <string>
#include <vector>

#include "ctx.h"

struct LayoutView {
    int T, nb, ncubes, ngroups;
    const std::vector<int> *perm, *slot_of, *cube_of_slot, *cube_off, *grp_off, *grp_cube, *grp_tile;
    const std::vector<NearTile> *tiles;
    const std::vector<long long> *pslot_base;
    const std::vector<int> *pslot_cnt;
    long long tile_store;
};

// empty string when consistent, else what is wrong
inline std::string check_layout(const LayoutView &v) {
    char buf[256];
    auto bad = [&](const char *fmt, long long a, long long b) {
        snprintf(buf, sizeof buf, fmt, a, b);
        return std::string(buf);
    };
    const int T = v.T;
    const std::vector<int> &perm = *v.perm, &slot_of = *v.slot_of, &cos = *v.cube_of_slot;
    if ((int)perm.size() != T || (int)slot_of.size() != T || (int)cos.size() != T)
        return bad("slot tables hold %lld entries, T = %lld", (long long)perm.size(), T);
    for (int s = 0; s < T; ++s) {
        const int t = perm[s];
        if (t < 0 || t >= T || slot_of[t] != s) return bad("perm[%lld] = %lld is not inverted by slot_of", s, t);
    }
    const std::vector<int> &co = *v.cube_off;
    if ((int)co.size() != v.ncubes + 1 || co[0] != 0 || co[v.ncubes] != T)
        return bad("box offsets: %lld entries, last %lld", (long long)co.size(), co.empty() ? -1 : co.back());
    for (int q = 0; q < v.ncubes; ++q)
        if (co[q + 1] < co[q]) return bad("box offsets decrease at box %lld (%lld)", q, co[q + 1]);
    for (int s = 0; s < T; ++s) {
        const int q = cos[s];
        if (q < 0 || q >= v.ncubes || s < co[q] || s >= co[q + 1]) return bad("slot %lld lies outside its box %lld", s, q);
    }
    const std::vector<int> &go = *v.grp_off, &gc = *v.grp_cube;
    const int ng = v.ngroups;
    if ((int)go.size() != ng + 1 || (int)gc.size() != ng || go[0] != 0 || go[ng] != T)
        return bad("group offsets: %lld entries for %lld groups", (long long)go.size(), ng);
    for (int g = 0; g < ng; ++g) {
        const int n = go[g + 1] - go[g];
        if (n <= 0 || n > SCD_GROUP_MAX || n % v.nb) return bad("group %lld holds %lld slots", g, n);
        const int q = gc[g];
        if (q < 0 || q >= v.ncubes || go[g] < co[q] || go[g + 1] > co[q + 1])
            return bad("group %lld lies outside its box %lld", g, q);
    }
    const std::vector<NearTile> &tl = *v.tiles;
    const std::vector<long long> &pb = *v.pslot_base;
    const std::vector<int> &pc = *v.pslot_cnt;
    if ((int)pb.size() != ng + 1 || (int)pc.size() != ng) return bad("partial slots: %lld bases for %lld groups", (long long)pb.size(), ng);
    for (int g = 0; g < ng; ++g)
        if (pc[g] < 1 || pb[g + 1] - pb[g] != (long long)pc[g] * 3 * (go[g + 1] - go[g]))
            return bad("partial slots of group %lld: count %lld", g, pc[g]);
    long long off = 0, prev = -1;
    for (size_t i = 0; i < tl.size(); ++i) {
        const NearTile &t = tl[i];
        const long long key = (long long)t.g1 * ng + t.g2;
        if (t.g1 < 0 || t.g2 < t.g1 || t.g2 >= ng || key <= prev) return bad("tile %lld: groups out of order (%lld)", (long long)i, key);
        prev = key;
        if (t.s1 != go[t.g1] || t.n1 != go[t.g1 + 1] - go[t.g1] || t.s2 != go[t.g2] || t.n2 != go[t.g2 + 1] - go[t.g2])
            return bad("tile %lld: slots do not match groups (first slot %lld)", (long long)i, t.s1);
        if (t.c1 != gc[t.g1] || t.c2 != gc[t.g2]) return bad("tile %lld: boxes do not match groups (%lld)", (long long)i, t.c1);
        if (t.data_off != off) return bad("tile %lld: data offset %lld out of sequence", (long long)i, t.data_off);
        off += tile_elems(t.n1, t.n2);
        if (t.g1 == t.g2) {
            if (t.col_off != -1) return bad("diagonal tile %lld has a transposed slot %lld", (long long)i, t.col_off);
        } else if (t.col_off < pb[t.g2] + 3LL * t.n2 || t.col_off + 3LL * t.n2 > pb[t.g2 + 1]) {
            // slot 0 of every group holds the row sums
            return bad("tile %lld: transposed slot %lld outside its group's partial slots", (long long)i, t.col_off);
        }
    }
    if (off != v.tile_store) return bad("tiles hold %lld elements, storage %lld", off, v.tile_store);
    const std::vector<int> &gt = *v.grp_tile;
    if ((int)gt.size() != ng + 1 || gt[0] != 0 || gt[ng] > (int)tl.size())
        return bad("group tile ranges: %lld entries, last %lld", (long long)gt.size(), gt.empty() ? -1 : gt.back());
    for (int g = 0; g < ng; ++g) {
        if (gt[g + 1] < gt[g]) return bad("group tile ranges decrease at group %lld (%lld)", g, gt[g + 1]);
        for (int i = gt[g]; i < gt[g + 1]; ++i)
            if (tl[i].g1 != g) return bad("tile %lld listed under group %lld", i, g);
    }
    return std::string();
}
