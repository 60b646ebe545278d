// C-ABI entry points of scadyn_gpu (include/scadyn_gpu.h) and the host-side
// set-up that prepares device layouts: tet ordering by projection box,
// near-zone tiling, work buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "ctx.h"
#include "linear_basis.h"
#include "layout_check.h"

// ------------------------------------------------------------------ errors
int set_error(scd_ctx *c, int code, const char *fmt, ...) {
    if (!c) return code;
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
    return code;
}

int check_cuda(scd_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return SCD_OK;
    if (e == cudaErrorMemoryAllocation) return set_error(c, SCD_OOM, "%s: %s", what, cudaGetErrorString(e));
    return set_error(c, SCD_CUDA_ERROR, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(expr, what)                                  \
    do {                                                \
        int _rc = check_cuda(c, (expr), (what));        \
        if (_rc) return _rc;                            \
    } while (0)

static int next_pow2(int v) {
    int p = 8;
    while (p < v) p <<= 1;
    return p;
}

// FFT length of an axis with N nodes: the smallest power of two >= 2N, or
// (the default) the smallest length >= 2N among the powers of two and the
// 5-smooth lengths with register transforms (80, 96, 192)
static int fft_len(int v, bool smooth) {
    const int p2 = next_pow2(v);
    if (!smooth) return p2;
    for (int p : {80, 96, 192})
        if (p >= v && p < p2) return p;
    return p2;
}

// instruction schedule of the tensor-core near zone (near_mma.cuh) for a
// scd_grid_desc.near_kernel / scd_tuning.near_kernel value
static int nzm_sched_of(int near_kernel) {
    return near_kernel == SCD_NEAR_TENSOR_SPLIT ? 0 : near_kernel == SCD_NEAR_TENSOR_MERGED ? 1 : 2;
}

template <typename Tp>
static int dalloc(scd_ctx *c, Tp **p, size_t count, const char *what) {
    if (*p) { cudaFree(*p); *p = nullptr; }
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void **)p, sizeof(Tp) * count);
    if (e != cudaSuccess) { *p = nullptr; cudaGetLastError(); return set_error(c, SCD_OOM, "allocating %s (%zu bytes)", what, sizeof(Tp) * count); }
    return SCD_OK;
}

// -------------------------------------------------------------- work area
int ensure_work(scd_ctx *c, int nrhs) {
    if (c->nrhs_cap >= nrhs && c->d_x) return SCD_OK;
    int rc;
    const size_t r = (size_t)nrhs;
    if ((rc = dalloc(c, &c->d_bpart, r * c->ncubes * 4 * 27, "box partials"))) return rc;
    if ((rc = dalloc(c, &c->d_W, r * 4 * (size_t)c->Px * c->Py * c->Nz, "FFT work grid"))) return rc;
    if ((rc = dalloc(c, &c->d_R, r * 4 * (size_t)c->Nx * c->Ny * c->Nz, "result grid"))) return rc;
    if ((rc = dalloc(c, &c->d_nzpart, r * (size_t)std::max<long long>(c->part_len, 1), "near-zone partials"))) return rc;
    if ((rc = dalloc(c, &c->d_x, r * c->n, "x"))) return rc;
    if ((rc = dalloc(c, &c->d_y, r * c->n, "y"))) return rc;
    if ((rc = dalloc(c, &c->d_io, r * c->n, "io"))) return rc;
    if ((rc = dalloc(c, &c->d_rhs, r * c->n, "rhs"))) return rc;
    if ((rc = dalloc(c, &c->d_xT, (size_t)xt_columns(nrhs) * c->n, "interleaved x"))) return rc;
    c->nrhs_cap = nrhs;
    return SCD_OK;
}

// The buffers a solve builds on demand -- the work areas of the right-hand
// sides in flight, the complex64 operator copies and the tensor-core tile
// planes -- freed; the next solve builds them again.  A sweep releases a
// wavelength's once its last column is done.
void release_work(scd_ctx *c) {
    auto fr = [](auto *&p) { if (p) { cudaFree(p); p = nullptr; } };
    fr(c->d_bpart); fr(c->d_W); fr(c->d_R); fr(c->d_nzpart); fr(c->d_x); fr(c->d_y); fr(c->d_io); fr(c->d_rhs);
    fr(c->d_xT);
    c->nrhs_cap = 0;
    fr(c->f_bpart); fr(c->f_W); fr(c->f_R); fr(c->f_nzpart); fr(c->f_xT);
    c->f_cap = 0;
    fr(c->f_P); fr(c->f_Fo); fr(c->f_tw[0]); fr(c->f_tw[1]); fr(c->f_tw[2]); fr(c->f_Fyz);
    c->f_ready = false;
    c->fyz_ready_f = false;
    fr(c->d_t16); fr(c->d_t16_off); fr(c->d_xb); fr(c->d_xb_off); fr(c->d_xmax); fr(c->d_xinv);
    c->nzm_ready = false;
}

// error word of the near-zone kernel: a bounded wait that ran out
int near_status(scd_ctx *c) {
    if (c->near_cfg_err) {
        c->near_cfg_err = 0;
        return set_error(c, SCD_BAD_ARG, "near-zone kernel not launched: a tile with its x segment exceeds the shared-memory ring");
    }
    if (!c->d_kerr) return SCD_OK;
    int h = 0;
    CK(cudaMemcpyAsync(&h, c->d_kerr, sizeof(int), cudaMemcpyDeviceToHost, c->st), "near-zone status");
    CK(cudaStreamSynchronize(c->st), "near-zone status");
    if (!h) return SCD_OK;
    CK(cudaMemsetAsync(c->d_kerr, 0, sizeof(int), c->st), "near-zone status");
    return set_error(c, SCD_TIMEOUT, "near-zone kernel: a pipeline wait ran out");
}

// ---------------------------------------------------------------- ordering
// Slot order: tets sorted by cube, ties by original index (tetras_in_cubes,
// src/geometry.f90:330-377, lists each cube's tets in increasing order).
static int set_order(scd_ctx *c, const std::vector<int> &cube_of_tet) {
    const int T = c->T;
    std::vector<int> cnt(c->ncubes + 1, 0);
    for (int t = 0; t < T; ++t) cnt[cube_of_tet[t] + 1]++;
    for (int q = 0; q < c->ncubes; ++q) cnt[q + 1] += cnt[q];
    std::vector<int> perm(T), slot_of(T), cos(T);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int t = 0; t < T; ++t) {
        int s = fill[cube_of_tet[t]]++;
        perm[s] = t;
        slot_of[t] = s;
        cos[s] = cube_of_tet[t];
    }
    if (c->have_order) {
        if (perm != c->perm) {
            // a different binning invalidates anything stored in slot order
            c->have_proj = false;
            c->have_near = false;
            c->nzm_ready = false;
            c->mat_cols = 0;
            c->mat_Nmax = -1;
        } else {
            return SCD_OK;
        }
    }
    c->perm.swap(perm);
    c->slot_of.swap(slot_of);
    c->cube_of_slot.swap(cos);
    c->cube_off = cnt;
    c->max_per_cube = 0;
    for (int q = 0; q < c->ncubes; ++q) c->max_per_cube = std::max(c->max_per_cube, cnt[q + 1] - cnt[q]);
    // near-zone groups: each non-empty box split into ceil(n / SCD_GROUP_MAX)
    // runs whose sizes differ by at most one; with the linear basis the runs
    // hold whole tets (the blocks inside a tet are one-sided)
    c->grp_off.assign(1, 0);
    c->grp_cube.clear();
    c->grp_of_slot.assign(T, 0);
    c->max_per_group = 0;
    std::vector<int> sizes;
    for (int q = 0; q < c->ncubes; ++q) {
        const int n = cnt[q + 1] - cnt[q];
        if ((int)sizes.size() < n + 1) sizes.resize(n + 1);   // at most n runs
        const int ng = split_box(n, c->nb, SCD_GROUP_MAX, sizes.data());
        if (ng == 0) continue;
        int s = cnt[q];
        for (int g = 0; g < ng; ++g) {
            const int m = sizes[g];
            for (int k = 0; k < m; ++k) c->grp_of_slot[s + k] = (int)c->grp_cube.size();
            s += m;
            c->grp_off.push_back(s);
            c->grp_cube.push_back(q);
            c->max_per_group = std::max(c->max_per_group, m);
        }
    }
    c->ngroups = (int)c->grp_cube.size();
    int rc;
    if ((rc = dalloc(c, &c->d_perm, T, "perm"))) return rc;
    if ((rc = dalloc(c, &c->d_cube_off, c->ncubes + 1, "cube offsets"))) return rc;
    if ((rc = dalloc(c, &c->d_grp_off, c->ngroups + 1, "group offsets"))) return rc;
    if ((rc = dalloc(c, &c->d_grp_cube, std::max(c->ngroups, 1), "group boxes"))) return rc;
    CK(cudaMemcpyAsync(c->d_perm, c->perm.data(), sizeof(int) * T, cudaMemcpyHostToDevice, c->st), "perm");
    CK(cudaMemcpyAsync(c->d_cube_off, c->cube_off.data(), sizeof(int) * (c->ncubes + 1), cudaMemcpyHostToDevice, c->st), "cube offsets");
    CK(cudaMemcpyAsync(c->d_grp_off, c->grp_off.data(), sizeof(int) * (c->ngroups + 1), cudaMemcpyHostToDevice, c->st), "groups");
    if (c->ngroups)
        CK(cudaMemcpyAsync(c->d_grp_cube, c->grp_cube.data(), sizeof(int) * c->ngroups, cudaMemcpyHostToDevice, c->st), "groups");
    c->have_order = true;
    return SCD_OK;
}

// ------------------------------------------------------------ near tiles
// write / accumulate a 3x3 block (column-major src, optionally transposed)
// into its strided tile position
template <typename ST>
static void put_block(ST *tile, int n1, int i, int j, const ST *src, bool transpose, bool add) {
    for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q) {
            const ST v = transpose ? src[q + 3 * r] : src[r + 3 * q];
            ST &d = tile[tile_at(n1, i, j, r + 3 * q)];
            if (add) { d.x += v.x; d.y += v.y; }
            else d = v;
        }
}

// Tile layout for a sorted list of group pairs key = g1*ngroups + g2
// (g1 <= g2): data offsets, the partial-sum slots of every group and the
// tile range of every group.
static long long layout_tiles(scd_ctx *c, const std::vector<uint64_t> &keys, std::vector<NearTile> &tiles) {
    const int nt = (int)keys.size();
    const int ng = c->ngroups;
    tiles.assign(nt, NearTile{});
    std::vector<int> cnt(ng, 1);           // slot 0: row sums
    long long off = 0;
    c->tile_blocks = 0;
    c->max_tile_store = 0;
    c->grp_tile.assign(ng + 1, 0);
    for (int i = 0; i < nt; ++i) {
        NearTile &tl = tiles[i];
        tl.g1 = (int)(keys[i] / ng);
        tl.g2 = (int)(keys[i] % ng);
        tl.c1 = c->grp_cube[tl.g1];
        tl.c2 = c->grp_cube[tl.g2];
        tl.s1 = c->grp_off[tl.g1];
        tl.s2 = c->grp_off[tl.g2];
        tl.n1 = c->grp_off[tl.g1 + 1] - tl.s1;
        tl.n2 = c->grp_off[tl.g2 + 1] - tl.s2;
        tl.data_off = off;
        const long long te = tile_elems(tl.n1, tl.n2);
        off += te;
        c->max_tile_store = std::max(c->max_tile_store, te);
        c->tile_blocks += (long long)tl.n1 * tl.n2;
        if (tl.g2 != tl.g1) cnt[tl.g2]++;
        c->grp_tile[tl.g1 + 1] = i + 1;
    }
    for (int g = 0; g < ng; ++g) c->grp_tile[g + 1] = std::max(c->grp_tile[g + 1], c->grp_tile[g]);
    c->pslot_base.assign(ng + 1, 0);
    c->pslot_cnt = cnt;
    for (int g = 0; g < ng; ++g) {
        const int n = c->grp_off[g + 1] - c->grp_off[g];
        c->pslot_base[g + 1] = c->pslot_base[g] + (long long)cnt[g] * 3 * n;
    }
    std::vector<int> used(ng, 1);
    for (int i = 0; i < nt; ++i) {
        NearTile &tl = tiles[i];
        tl.col_off = -1;
        if (tl.g2 != tl.g1) tl.col_off = c->pslot_base[tl.g2] + (long long)(used[tl.g2]++) * 3 * tl.n2;
    }
    c->tile_store = off;
    return off;
}

static int upload_layout(scd_ctx *c, std::vector<NearTile> &tiles, long long off) {
    (void)off;
    const int nt = (int)tiles.size();
    const int ng = c->ngroups;
    const LayoutView lv{c->T, c->nb, c->ncubes, ng, &c->perm, &c->slot_of, &c->cube_of_slot, &c->cube_off,
                        &c->grp_off, &c->grp_cube, &c->grp_tile, &tiles, &c->pslot_base, &c->pslot_cnt, c->tile_store};
    const std::string why = check_layout(lv);
    if (!why.empty()) return set_error(c, SCD_BAD_ARG, "near-zone layout check: %s", why.c_str());
    int rc;
    if ((rc = dalloc(c, &c->d_tiles, nt, "tile table"))) return rc;
    if ((rc = dalloc(c, &c->d_pslot_base, ng + 1, "slot bases"))) return rc;
    if ((rc = dalloc(c, &c->d_pslot_cnt, std::max(ng, 1), "slot counts"))) return rc;
    if ((rc = dalloc(c, &c->d_grp_tile, ng + 1, "group tiles"))) return rc;
    if ((rc = dalloc(c, &c->d_kerr, 1, "error word"))) return rc;
    CK(cudaMemsetAsync(c->d_kerr, 0, sizeof(int), c->st), "error word");
    if (nt) CK(cudaMemcpyAsync(c->d_tiles, tiles.data(), sizeof(NearTile) * nt, cudaMemcpyHostToDevice, c->st), "tile table");
    CK(cudaMemcpyAsync(c->d_pslot_base, c->pslot_base.data(), sizeof(long long) * (ng + 1), cudaMemcpyHostToDevice, c->st), "slots");
    if (ng) CK(cudaMemcpyAsync(c->d_pslot_cnt, c->pslot_cnt.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, c->st), "slots");
    CK(cudaMemcpyAsync(c->d_grp_tile, c->grp_tile.data(), sizeof(int) * (ng + 1), cudaMemcpyHostToDevice, c->st), "group tiles");
    c->ntiles = nt;
    c->part_len = c->pslot_base[ng];
    c->tiles_h.swap(tiles);
    c->nrhs_cap = 0;   // partial buffer size changed
    c->f_cap = 0;
    return SCD_OK;
}

// Tiles from the geometry: every group g1 with each group g2 >= g1 whose box
// lies in the 27-neighbourhood of g1's box (find_near_cubes,
// src/geometry.f90:275-326) -- the tet pairs that
// compute_near_zone_interactions_const visits.
int build_tile_layout(scd_ctx *c) {
    std::vector<uint64_t> keys;
    // groups of each box
    std::vector<int> first(c->ncubes + 1, -1), last(c->ncubes, -1);
    for (int g = 0; g < c->ngroups; ++g) {
        if (first[c->grp_cube[g]] < 0) first[c->grp_cube[g]] = g;
        last[c->grp_cube[g]] = g;
    }
    for (int g1 = 0; g1 < c->ngroups; ++g1) {
        const int c1 = c->grp_cube[g1];
        const int x = c1 % c->ncx, y = (c1 / c->ncx) % c->ncy, z = c1 / (c->ncx * c->ncy);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int xx = x + dx, yy = y + dy, zz = z + dz;
                    if (xx < 0 || yy < 0 || zz < 0 || xx >= c->ncx || yy >= c->ncy || zz >= c->ncz) continue;
                    const int c2 = xx + c->ncx * (yy + c->ncy * zz);
                    if (first[c2] < 0) continue;
                    for (int g2 = std::max(first[c2], g1); g2 <= last[c2]; ++g2)
                        keys.push_back((uint64_t)g1 * (uint64_t)c->ngroups + (uint64_t)g2);
                }
    }
    std::sort(keys.begin(), keys.end());
    std::vector<NearTile> tiles;
    const long long off = layout_tiles(c, keys, tiles);
    return upload_layout(c, tiles, off);
}

int set_order_from_cubes(scd_ctx *c, const std::vector<int> &cube_of_tet) { return set_order(c, cube_of_tet); }

// Tile the reference's symmetric block list (tet_B >= tet_T) into dense
// group-pair tiles; see NearTile in ctx.h.  Blocks given twice are summed, as
// the reference's SpMV would sum them.  A block flagged one-sided (linear
// basis, inside a tet) is applied as given only, without its mirror.
template <typename ST>
static int build_tiles(scd_ctx *c, int64_t B, const ST *sp, const int32_t *ind, const unsigned char *one_sided = nullptr) {
    const int T = c->T;
    std::unordered_map<uint64_t, int> tid;
    tid.reserve((size_t)c->ngroups * 16);
    std::vector<uint64_t> keys;
    std::vector<int> btile((size_t)B);
    for (int64_t b = 0; b < B; ++b) {
        const int t1 = ind[2 * b] - 1, t2 = ind[2 * b + 1] - 1;
        if (t1 < 0 || t1 >= T || t2 < 0 || t2 >= T)
            return set_error(c, SCD_BAD_ARG, "sp_ind(:,%lld) = (%d,%d) outside 1..%d", (long long)b + 1, t1 + 1, t2 + 1, T);
        const int ga = c->grp_of_slot[c->slot_of[t1]], gb = c->grp_of_slot[c->slot_of[t2]];
        const uint64_t key = (uint64_t)std::min(ga, gb) * (uint64_t)c->ngroups + (uint64_t)std::max(ga, gb);
        auto it = tid.find(key);
        int id;
        if (it == tid.end()) { id = (int)keys.size(); tid.emplace(key, id); keys.push_back(key); }
        else id = it->second;
        btile[b] = id;
    }
    const int nt = (int)keys.size();
    std::vector<int> order(nt);
    for (int i = 0; i < nt; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    std::vector<int> rank(nt);
    for (int i = 0; i < nt; ++i) rank[order[i]] = i;
    std::vector<uint64_t> skeys(nt);
    for (int i = 0; i < nt; ++i) skeys[i] = keys[order[i]];
    std::vector<NearTile> tiles;
    const long long off = layout_tiles(c, skeys, tiles);
    std::vector<ST> data((size_t)off);
    std::memset(data.data(), 0, sizeof(ST) * data.size());
    std::vector<char> seen((size_t)c->tile_blocks, 0);
    std::vector<long long> block_base(nt);   // first block of each tile in `seen`
    {
        long long acc = 0;
        for (int i = 0; i < nt; ++i) { block_base[i] = acc; acc += (long long)tiles[i].n1 * tiles[i].n2; }
    }
    for (int64_t b = 0; b < B; ++b) {
        const int ti = rank[btile[b]];
        const NearTile &tl = tiles[ti];
        const int t1 = ind[2 * b] - 1, t2 = ind[2 * b + 1] - 1;
        const int s1 = c->slot_of[t1], s2 = c->slot_of[t2];
        const ST *src = sp + 9 * b;
        // position of (row tet, column tet) in the tile and whether the block
        // must be transposed (M(B,T) = M(T,B)^T)
        auto place = [&](int srow, int scol, bool tr) {
            const int i = srow - tl.s1, j = scol - tl.s2;
            const size_t e = (size_t)block_base[ti] + (size_t)i * tl.n2 + j;
            put_block(&data[(size_t)tl.data_off], tl.n1, i, j, src, tr, seen[e] != 0);
            seen[e] = 1;
        };
        if (tl.g1 == tl.g2) {
            place(s1, s2, false);
            if (s1 != s2 && !(one_sided && one_sided[b])) place(s2, s1, true);
        } else if (one_sided && one_sided[b]) {
            return set_error(c, SCD_BAD_ARG, "one-sided block between groups");
        } else if (c->grp_of_slot[s1] == tl.g1) {
            place(s1, s2, false);
        } else {
            place(s2, s1, true);
        }
    }
    int rc;
    if ((rc = dalloc(c, (ST **)&c->d_tdata, data.size(), "near-zone tiles"))) return rc;
    CK(cudaMemcpyAsync(c->d_tdata, data.data(), sizeof(ST) * data.size(), cudaMemcpyHostToDevice, c->st), "tiles");
    if ((rc = upload_layout(c, tiles, off))) return rc;
    c->B_ref = B;
    return SCD_OK;
}

// ------------------------------------------------------------------ ABI
extern "C" {

const char *scd_last_error(const scd_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int scd_create(scd_ctx **out, const scd_grid_desc *d) {
    if (!out || !d) return SCD_BAD_ARG;
    *out = nullptr;
    if ((d->order != 0 && d->order != 1) || d->M_ex != 2 || d->near_zone != 1) return SCD_BAD_ARG;
    if (d->Nx < 4 || d->Ny < 4 || d->Nz < 4 || d->T <= 0 || !(d->delta > 0)) return SCD_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return SCD_NO_DEVICE; }
    if (d->device < 0 || d->device >= ndev) return SCD_BAD_ARG;
    if (d->fft_lengths < SCD_FFT_DEFAULT || d->fft_lengths > SCD_FFT_SMOOTH) return SCD_BAD_ARG;
    if (d->near_kernel < SCD_NEAR_DEFAULT || d->near_kernel > SCD_NEAR_TENSOR_WIDE) return SCD_BAD_ARG;
    if (d->near_split < 0 || d->near_split > 2) return SCD_BAD_ARG;
    if (d->fft_passes < SCD_FFT_PASSES_DEFAULT || d->fft_passes > SCD_FFT_PASSES_THREE) return SCD_BAD_ARG;
    scd_ctx *c = new scd_ctx();
    c->d = *d;
    c->dev = d->device;
    // kernel choices: the tensor-core near zone applies to complex64 storage
    // only (checked when the near zone is set); 0 selects the defaults
    c->nzm_on = d->near_kernel != SCD_NEAR_CUDA_CORES;
    c->nzm_sched = nzm_sched_of(d->near_kernel);
    c->near_split = d->near_split == 1 ? 1 : 2;
    c->yz_on = d->fft_passes != SCD_FFT_PASSES_THREE;
    cudaSetDevice(c->dev);
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->dev);
    c->Nx = d->Nx; c->Ny = d->Ny; c->Nz = d->Nz;
    {
        const bool smooth = d->fft_lengths != SCD_FFT_POW2;
        c->Px = fft_len(2 * d->Nx, smooth); c->Py = fft_len(2 * d->Ny, smooth); c->Pz = fft_len(2 * d->Nz, smooth);
    }
    if (c->Px > 512 || c->Py > 512 || c->Pz > 512) {
        set_error(c, SCD_BAD_ARG, "grid %dx%dx%d needs an FFT longer than 512", d->Nx, d->Ny, d->Nz);
        *out = c;
        return SCD_BAD_ARG;
    }
    c->Hx = c->Px / 2 + 1; c->Hy = c->Py / 2 + 1; c->Hz = c->Pz / 2 + 1;
    c->ncx = (d->Nx - 2) / 2; c->ncy = (d->Ny - 2) / 2; c->ncz = (d->Nz - 2) / 2;
    c->ncubes = c->ncx * c->ncy * c->ncz;
    c->nb = d->order == 1 ? 4 : 1;
    c->T = c->nb * d->T;
    c->n = 3LL * c->T;
    *out = c;
    int rc;
    if ((rc = check_cuda(c, cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking), "stream"))) return rc;
    for (int i = 0; i < 8; ++i) cudaEventCreate(&c->ev[i]);
    const int Ps[3] = {c->Px, c->Py, c->Pz};
    for (int a = 0; a < 3; ++a)
        if ((rc = build_twiddles(c, Ps[a], &c->d_tw[a]))) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->st), "create");
}

int scd_destroy(scd_ctx *c) {
    if (!c) return SCD_OK;
    cudaSetDevice(c->dev);
    if (c->st) cudaStreamSynchronize(c->st);
    void *ptrs[] = {c->d_perm, c->d_cube_off, c->d_grp_off, c->d_grp_cube, c->d_grp_tile, c->d_kerr, c->d_P, c->d_Fo, c->d_tdata, c->d_tiles, c->d_pslot_base,
                    c->d_pslot_cnt, c->d_tc, c->d_tvol, c->d_eps, c->d_bpart, c->d_W, c->d_R, c->d_nzpart, c->d_x,
                    c->d_y, c->d_io, c->d_rhs,
                    c->d_bar, c->d_err, c->d_tw[0], c->d_tw[1], c->d_tw[2], c->f_P, c->f_Fo,
                    c->f_tw[0], c->f_tw[1], c->f_tw[2], c->f_bpart, c->f_W, c->f_R, c->f_nzpart, c->d_xT, c->f_xT,
                    c->d_t16, c->d_t16_off, c->d_xb, c->d_xb_off, c->d_xmax, c->d_xinv, c->d_Fyz, c->f_Fyz};
    for (void *p : ptrs) if (p) cudaFree(p);
    batch_free(c);
    if (c->d_mat) cudaFree(c->d_mat);
    for (int i = 0; i < 8; ++i) if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return SCD_OK;
}

int scd_set_wavenumber(scd_ctx *c, double k) {
    if (!c) return SCD_BAD_ARG;
    if (!(k > 0) || !std::isfinite(k)) return set_error(c, SCD_BAD_ARG, "wavenumber %g", k);
    if (c->have_k && k != c->k) c->have_green = false;   // a device-built Fg is per wavelength
    c->k = k;
    c->have_k = true;
    return SCD_OK;
}

int scd_set_green(scd_ctx *c, const scd_c128 *Fg) {
    if (!c) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    if (!Fg && !c->have_k) return set_error(c, SCD_NOT_READY, "scd_set_green(NULL) needs scd_set_wavenumber first");
    if (Fg && (c->Px != 2 * c->Nx || c->Py != 2 * c->Ny || c->Pz != 2 * c->Nz))
        return set_error(c, SCD_BAD_ARG,
                         "host Fg of size (%d,%d,%d) is not a power-of-two FFT; pass NULL to build it on the device",
                         2 * c->Nx, 2 * c->Ny, 2 * c->Nz);
    int rc = setup_green(c, Fg);
    if (rc == SCD_OK) c->have_green = true;
    c->f_ready = false;
    c->fyz_ready = c->fyz_ready_f = false;
    return rc;
}

int scd_set_projectors(scd_ctx *c, int32_t M_box, int32_t T, const scd_c128 *S, const scd_c128 *Sx,
                       const scd_c128 *Sy, const scd_c128 *Sz, const int32_t *indS) {
    if (!c) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    if (M_box != 27) return set_error(c, SCD_BAD_ARG, "M_box = %d, only 27 (M_ex = 2) is supported", M_box);
    if (T != c->T) return set_error(c, SCD_BAD_ARG, "T = %d, context has %d", T, c->T);
    if (!S || !Sx || !Sy || !Sz || !indS) return set_error(c, SCD_BAD_ARG, "null projector array");
    // the 27 nodes of every column must be the node block of one projection
    // box (src/projection.f90:160 stores etopol_box(:, cube))
    std::vector<int> cube(T);
    const int Nx = c->Nx, Ny = c->Ny;
    for (int t = 0; t < T; ++t) {
        const int32_t *id = indS + 27LL * t;
        const long long n0 = id[0] - 1;
        const int x = (int)(n0 % Nx), y = (int)((n0 / Nx) % Ny), z = (int)(n0 / ((long long)Nx * Ny));
        if (n0 < 0 || (x & 1) || (y & 1) || (z & 1) || x / 2 >= c->ncx || y / 2 >= c->ncy || z / 2 >= c->ncz)
            return set_error(c, SCD_BAD_ARG, "indS(1,%d) = %d is not the first node of a projection box", t + 1, id[0]);
        for (int j = 0; j < 27; ++j) {
            const long long want = n0 + (j % 3) + (long long)((j / 3) % 3) * Nx + (long long)(j / 9) * Nx * Ny + 1;
            if (id[j] != want) return set_error(c, SCD_BAD_ARG, "indS(%d,%d) = %d, expected %lld", j + 1, t + 1, id[j], want);
        }
        cube[t] = x / 2 + c->ncx * (y / 2 + c->ncy * (z / 2));
    }
    // linear basis: the four basis functions of a tet share its box
    for (int t = 0; t + c->nb <= T; t += c->nb)
        for (int i = 1; i < c->nb; ++i)
            if (cube[t + i] != cube[t])
                return set_error(c, SCD_BAD_ARG, "indS columns %d and %d (one tet) name different boxes", t + 1, t + i + 1);
    int rc = set_order(c, cube);
    if (rc) return rc;
    std::vector<cd> h((size_t)4 * 27 * T);
    const scd_c128 *src[4] = {S, Sx, Sy, Sz};
    for (int g = 0; g < 4; ++g)
        for (int s = 0; s < T; ++s) {
            const scd_c128 *p = src[g] + 27LL * c->perm[s];
            for (int j = 0; j < 27; ++j) h[(size_t)(g * 27 + j) * T + s] = cmk(p[j].re, p[j].im);
        }
    if ((rc = dalloc(c, &c->d_P, h.size(), "projectors"))) return rc;
    CK(cudaMemcpyAsync(c->d_P, h.data(), sizeof(cd) * h.size(), cudaMemcpyHostToDevice, c->st), "projectors");
    c->have_proj = true;
    c->f_ready = false;
    return SCD_OK;
}

int scd_set_nearzone(scd_ctx *c, int64_t B, const void *sp_mat, const int32_t *sp_ind, int32_t prec) {
    if (!c) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    if (!c->have_order) return set_error(c, SCD_NOT_READY, "set the projectors (or the mesh) before the near zone");
    if (B < 0 || (B > 0 && (!sp_mat || !sp_ind))) return set_error(c, SCD_BAD_ARG, "bad near-zone arrays");
    if (prec != SCD_STORE_C64 && prec != SCD_STORE_C128) return set_error(c, SCD_BAD_ARG, "storage_prec %d", prec);
    int rc;
    c->have_near = false;
    c->nzm_ready = false;
    c->near_prec = prec;
    c->f_cap = 0;
    if (c->nb == 4) {
        // linear basis: 12x12 blocks between tets -> 3x3 blocks between pseudo-tets
        const int ntet = c->T / 4;
        for (int64_t b = 0; b < B; ++b)
            if (sp_ind[2 * b] < 1 || sp_ind[2 * b] > ntet || sp_ind[2 * b + 1] < 1 || sp_ind[2 * b + 1] > ntet)
                return set_error(c, SCD_BAD_ARG, "sp_ind(:,%lld) = (%d,%d) outside 1..%d", (long long)b + 1,
                                 sp_ind[2 * b], sp_ind[2 * b + 1], ntet);
        std::vector<int32_t> ind3((size_t)32 * B);
        std::vector<unsigned char> one((size_t)16 * B);
        if (prec == SCD_STORE_C64) {
            std::vector<cf> sp3((size_t)144 * B);
            expand_linear_blocks<cf>(B, (const cf *)sp_mat, sp_ind, sp3.data(), ind3.data(), one.data());
            rc = build_tiles<cf>(c, 16 * B, sp3.data(), ind3.data(), one.data());
        } else {
            std::vector<cd> sp3((size_t)144 * B);
            expand_linear_blocks<cd>(B, (const cd *)sp_mat, sp_ind, sp3.data(), ind3.data(), one.data());
            rc = build_tiles<cd>(c, 16 * B, sp3.data(), ind3.data(), one.data());
        }
        if (rc == SCD_OK) c->B_ref = B;
    } else if (prec == SCD_STORE_C64) {
        rc = build_tiles<cf>(c, B, (const cf *)sp_mat, sp_ind);
    } else {
        rc = build_tiles<cd>(c, B, (const cd *)sp_mat, sp_ind);
    }
    if (rc == SCD_OK) c->have_near = true;
    return rc;
}

static int ready(scd_ctx *c) {
    if (!c->have_proj) return set_error(c, SCD_NOT_READY, "projectors not set");
    if (!c->have_green) return set_error(c, SCD_NOT_READY, "Green's function not set (or stale after a new wavenumber)");
    if (!c->have_near) return set_error(c, SCD_NOT_READY, "near zone not set");
    if (!c->have_k) return set_error(c, SCD_NOT_READY, "wavenumber not set");
    return ensure_work(c, 1);
}

int scd_matvec(scd_ctx *c, const scd_c128 *x, scd_c128 *Ax) {
    if (!c || !x || !Ax) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    int rc = ready(c);
    if (rc) return rc;
    const size_t bytes = sizeof(cd) * c->n;
    CK(cudaMemcpyAsync(c->d_io, x, bytes, cudaMemcpyHostToDevice, c->st), "x");
    launch_permute_in(c, c->d_io, c->d_x, 1, c->n);
    run_matvec(c, c->d_x, c->d_y, 1, nullptr);
    launch_permute_out(c, c->d_y, c->d_io, 1, c->n);
    CK(cudaMemcpyAsync(Ax, c->d_io, bytes, cudaMemcpyDeviceToHost, c->st), "Ax");
    CK(cudaStreamSynchronize(c->st), "matvec");
    c->n_matvec += 1;
    if ((rc = near_status(c))) return rc;
    return check_cuda(c, cudaGetLastError(), "matvec");
}

int scd_gmres(scd_ctx *c, const scd_c128 *rhs, scd_c128 *x, double tol, int32_t m, int32_t cycles, int32_t *iters,
              double *relres) {
    if (!c || !rhs || !x || m < 1 || m > SCD_M_MAX || cycles < 1 || !(tol > 0)) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    int rc = ready(c);
    if (rc) return rc;
    const size_t bytes = sizeof(cd) * c->n;
    CK(cudaMemcpyAsync(c->d_io, rhs, bytes, cudaMemcpyHostToDevice, c->st), "rhs");
    launch_permute_in(c, c->d_io, c->d_rhs, 1, c->n);
    int it = 0;
    double rr = 0;
    cudaEventRecord(c->ev[4], c->st);
    // one slot of the batched solver: the same arithmetic as that column in
    // any batch of scd_solve_columns
    const cd *col = c->d_rhs;
    rc = batch_solve(c, 1, &col, c->d_x, tol, m, cycles, 1, &it, nullptr, nullptr, &rr, SCD_PREC_FP64, 0.0, 0);
    if (rc != SCD_OK && rc != SCD_NOT_CONVERGED) return rc;
    cudaEventRecord(c->ev[5], c->st);
    launch_permute_out(c, c->d_x, c->d_io, 1, c->n);
    CK(cudaMemcpyAsync(x, c->d_io, bytes, cudaMemcpyDeviceToHost, c->st), "x");
    CK(cudaStreamSynchronize(c->st), "gmres");
    {
        const int ns = near_status(c);
        if (ns) return ns;
    }
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]);
        c->last_call_ms = ms;
        c->accum_ms += ms;
    }
    if (iters) *iters = it;
    if (relres) *relres = rr;
    return rc;
}

// the incident matrix mat (3T, nmat) on the device, slot-ordered, in c->d_mat
// (mat_Nmax = 0 marks a host-supplied matrix; scd_compute_T_matrix builds its
// own columns over it)
static int upload_rhs_matrix(scd_ctx *c, int nmat, const scd_c128 *mat) {
    const long long n = c->n;
    int rc;
    if (!c->d_mat || c->mat_cols != nmat || c->mat_Nmax != 0) {
        cudaFree(c->d_mat);
        c->d_mat = nullptr;
        c->mat_cols = 0;
        if ((rc = dalloc(c, &c->d_mat, (size_t)n * nmat, "incident matrix"))) return rc;
    }
    c->mat_Nmax = 0;
    c->mat_k = 0.0;
    for (int col = 0; col < nmat; ++col) {
        CK(cudaMemcpyAsync(c->d_io, mat + (size_t)n * col, sizeof(cd) * n, cudaMemcpyHostToDevice, c->st), "mat");
        launch_permute_in(c, c->d_io, c->d_mat + (size_t)n * col, 1, n);
    }
    c->mat_cols = nmat;
    return SCD_OK;
}

static int check_opts(scd_ctx *c, const scd_solve_opts *o) {
    if (o->m < 1 || o->m > SCD_M_MAX || o->cycles < 1 || !(o->tol > 0) || o->block < 0)
        return set_error(c, SCD_BAD_ARG, "solve options: m %d (1..%d), cycles %d, tol %g, block %d", o->m, SCD_M_MAX,
                         o->cycles, o->tol, o->block);
    if (o->precision != SCD_PREC_FP64 && o->precision != SCD_PREC_MIXED)
        return set_error(c, SCD_BAD_ARG, "precision %d", o->precision);
    if (o->gram_schmidt < SCD_GS_DEFAULT || o->gram_schmidt > SCD_GS_CLASSICAL)
        return set_error(c, SCD_BAD_ARG, "gram_schmidt %d", o->gram_schmidt);
    if (o->precision == SCD_PREC_MIXED && (!(o->inner_tol > 0) || o->max_outer < 1))
        return set_error(c, SCD_BAD_ARG, "mixed form: inner_tol %g, max_outer %d", o->inner_tol, o->max_outer);
    c->cgs_on = o->gram_schmidt != SCD_GS_MODIFIED;
    return SCD_OK;
}

int scd_set_rhs_matrix(scd_ctx *c, int32_t nmat, const scd_c128 *mat) {
    if (!c || nmat <= 0 || !mat) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    if (!c->have_order) return set_error(c, SCD_NOT_READY, "scd_set_rhs_matrix needs the projectors or the mesh first");
    int rc = ensure_work(c, 1);
    if (rc) return rc;
    if ((rc = upload_rhs_matrix(c, nmat, mat))) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->st), "incident matrix");
}

int scd_solve_columns(scd_ctx *c, int32_t nmat, const scd_c128 *mat, int32_t col0, int32_t ncol, scd_c128 *Tcols,
                      const scd_solve_opts *o, int32_t *iters, scd_c128 *X) {
    if (!c || nmat <= 0 || ncol <= 0 || !Tcols || !o) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    if (col0 < 0 || col0 + ncol > nmat)
        return set_error(c, SCD_BAD_ARG, "columns %d..%d outside 1..%d", col0 + 1, col0 + ncol, nmat);
    int rc = ready(c);
    if (rc) return rc;
    if ((rc = check_opts(c, o))) return rc;
    const long long n = c->n;
    cudaEventRecord(c->ev[4], c->st);
    if (mat) {
        if ((rc = upload_rhs_matrix(c, nmat, mat))) return rc;
    } else if (!c->d_mat || c->mat_Nmax != 0 || c->mat_cols != nmat) {
        return set_error(c, SCD_NOT_READY, "mat is NULL and no incident matrix of %d columns was set", nmat);
    }
    cd *d_X = nullptr, *d_T = nullptr;
    if ((rc = dalloc(c, &d_X, (size_t)n * ncol, "X"))) return rc;
    if ((rc = dalloc(c, &d_T, (size_t)nmat * ncol, "T"))) { cudaFree(d_X); return rc; }
    std::vector<const cd *> cols(ncol);
    for (int j = 0; j < ncol; ++j) cols[j] = c->d_mat + (size_t)n * (col0 + j);
    const int ns = o->block > 0 ? o->block : ncol;
    std::vector<int> it(ncol, 0);
    int worst = batch_solve(c, ncol, cols.data(), d_X, o->tol, o->m, o->cycles, ns, it.data(), nullptr, nullptr,
                            nullptr, o->precision, o->inner_tol, o->max_outer);
    if (worst == SCD_OK || worst == SCD_NOT_CONVERGED) {
        const int ns_ = near_status(c);
        if (ns_) worst = ns_;
    }
    if (iters) for (int j = 0; j < ncol; ++j) iters[j] = it[j];
    if (worst == SCD_OK || worst == SCD_NOT_CONVERGED) {
        // T_mat(:, col0+j) = mat^H x_j over all nmat rows (src/T_matrix.f90:260)
        launch_T_assemble(c, c->d_mat, nmat, 0, ncol, d_X, d_T);
        rc = check_cuda(c, cudaMemcpyAsync(Tcols, d_T, sizeof(cd) * (size_t)nmat * ncol, cudaMemcpyDeviceToHost, c->st), "T");
        if (!rc && X) {
            for (int col = 0; col < ncol && !rc; ++col) {
                launch_permute_out(c, d_X + (size_t)n * col, c->d_io, 1, n);
                rc = check_cuda(c, cudaMemcpyAsync(X + (size_t)n * col, c->d_io, sizeof(cd) * n, cudaMemcpyDeviceToHost, c->st), "X");
            }
        }
        cudaEventRecord(c->ev[5], c->st);
        if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "solve");
        if (rc) worst = rc;
        else {
            float ms = 0;
            cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]);
            c->last_call_ms = ms;
            c->accum_ms += ms;
        }
    }
    cudaStreamSynchronize(c->st);
    cudaFree(d_X); cudaFree(d_T);
    return worst;
}

int scd_get_timing(scd_ctx *c, scd_timing *t, int32_t reset) {
    if (!c || !t) return SCD_BAD_ARG;
    t->matvec_ms = c->t_matvec;
    t->nearzone_ms = c->t_near;
    t->fft_ms = c->t_fft;
    t->gather_ms = c->t_gather;
    t->arnoldi_ms = c->t_arn;
    t->last_call_ms = c->last_call_ms;
    t->accum_ms = c->accum_ms;
    t->launches = c->launches;
    t->matvecs = c->n_matvec;
    t->arnoldi_steps = c->n_arn;
    t->near_kernel_ms = c->t_near_k;
    if (reset) {
        c->accum_ms = 0;
        c->launches = 0;
        c->n_matvec = 0;
        c->n_arn = 0;
    }
    return SCD_OK;
}

int scd_profile_matvec(scd_ctx *c, int32_t reps, int32_t nrhs, int32_t precision) {
    if (!c || reps < 1 || nrhs < 1) return SCD_BAD_ARG;
    if (precision != SCD_PREC_FP64 && precision != SCD_PREC_MIXED)
        return set_error(c, SCD_BAD_ARG, "precision %d", precision);
    cudaSetDevice(c->dev);
    int rc = ready(c);
    if (rc) return rc;
    if ((rc = ensure_work(c, nrhs))) return rc;
    const bool mixed = precision == SCD_PREC_MIXED;
    cf *fx = nullptr, *fy = nullptr;
    if (mixed) {
        if ((rc = ensure_single(c)) || (rc = ensure_work_single(c, nrhs))) return rc;
        if ((rc = dalloc(c, &fx, (size_t)nrhs * c->n, "profile x"))) return rc;
        if ((rc = dalloc(c, &fy, (size_t)nrhs * c->n, "profile y"))) { cudaFree(fx); return rc; }
    }
    // a fixed dense vector: the memory traffic of a matvec does not depend on the values
    std::vector<cd> h((size_t)c->n);
    std::vector<cf> hf((size_t)c->n);
    for (long long i = 0; i < c->n; ++i) {
        h[i] = cmk(std::sin(0.37 * (double)i), std::cos(0.11 * (double)i));
        hf[i] = make_float2((float)h[i].x, (float)h[i].y);
    }
    // copies on the context's stream, so that the matvecs below run after them
    for (int r = 0; r < nrhs && !rc; ++r) {
        if (mixed) rc = check_cuda(c, cudaMemcpyAsync(fx + (size_t)r * c->n, hf.data(), sizeof(cf) * c->n, cudaMemcpyHostToDevice, c->st), "profile x");
        else rc = check_cuda(c, cudaMemcpyAsync(c->d_x + (size_t)r * c->n, h.data(), sizeof(cd) * c->n, cudaMemcpyHostToDevice, c->st), "profile x");
    }
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "profile x");
    double sn = 0, sf = 0, sg = 0, st = 0, sk = 0;
    c->timing = true;
    for (int r = 0; r < reps + 1 && !rc; ++r) {
        if (mixed) run_matvec(c, fx, fy, nrhs, nullptr);
        else run_matvec(c, c->d_x, c->d_y, nrhs, nullptr);
        rc = check_cuda(c, cudaStreamSynchronize(c->st), "profile");
        float a = 0, b = 0, g = 0, t = 0;
        cudaEventElapsedTime(&a, c->ev[0], c->ev[1]);
        cudaEventElapsedTime(&b, c->ev[1], c->ev[2]);
        cudaEventElapsedTime(&g, c->ev[2], c->ev[3]);
        cudaEventElapsedTime(&t, c->ev[0], c->ev[3]);
        float k = 0;
        cudaEventElapsedTime(&k, c->ev[6], c->ev[7]);
        if (r == 0) continue;   // warm-up
        sn += a; sf += b; sg += g; st += t; sk += k;
    }
    c->timing = false;
    if (fx) cudaFree(fx);
    if (fy) cudaFree(fy);
    if (rc) return rc;
    c->t_near = sn / reps;
    c->t_fft = sf / reps;
    c->t_gather = sg / reps;
    c->t_matvec = st / reps;
    c->t_near_k = sk / reps;
    if ((rc = near_status(c))) return rc;
    return check_cuda(c, cudaGetLastError(), "profile");
}

// differing 32-bit words of a and b, added to *cnt
static __global__ void k_words_differ(const unsigned *a, const unsigned *b, long long nw, unsigned long long *cnt) {
    unsigned long long d = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nw; i += (long long)gridDim.x * blockDim.x)
        d += a[i] != b[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if ((threadIdx.x & 31) == 0 && d) atomicAdd(cnt, d);
}

int scd_check_matvec_repeat(scd_ctx *c, int32_t reps, int32_t nrhs, int32_t precision, int64_t *bad_reps,
                            int64_t *bad_words) {
    if (!c || reps < 1 || nrhs < 1 || !bad_reps || !bad_words) return SCD_BAD_ARG;
    if (precision != SCD_PREC_FP64 && precision != SCD_PREC_MIXED)
        return set_error(c, SCD_BAD_ARG, "precision %d", precision);
    cudaSetDevice(c->dev);
    int rc = ready(c);
    if (rc) return rc;
    if ((rc = ensure_work(c, nrhs))) return rc;
    const bool mixed = precision == SCD_PREC_MIXED;
    if (mixed && ((rc = ensure_single(c)) || (rc = ensure_work_single(c, nrhs)))) return rc;
    const size_t es = mixed ? sizeof(cf) : sizeof(cd), col = es * (size_t)c->n;
    void *x = nullptr, *y = nullptr, *y0 = nullptr;
    unsigned long long *cnt = nullptr;
    auto release = [&]() { cudaFree(x); cudaFree(y); cudaFree(y0); cudaFree(cnt); };
    if (cudaMalloc(&x, col * nrhs) != cudaSuccess || cudaMalloc(&y, col * nrhs) != cudaSuccess ||
        cudaMalloc(&y0, col * nrhs) != cudaSuccess || cudaMalloc(&cnt, sizeof(unsigned long long) * reps) != cudaSuccess) {
        cudaGetLastError();
        release();
        return set_error(c, SCD_OOM, "matvec repeat check: %zu bytes", 3 * col * nrhs);
    }
    // column r: a dense vector with an r-dependent phase.  Each column goes up
    // on the context's stream, which orders it before the first matvec (a
    // blocking cudaMemcpy from pageable memory may return before its DMA
    // lands, and the non-blocking stream does not wait for it), and the host
    // column is refilled only after the copy is done.
    std::vector<cd> h((size_t)c->n);
    std::vector<cf> hf(mixed ? (size_t)c->n : 0);
    for (int r = 0; r < nrhs && !rc; ++r) {
        for (long long i = 0; i < c->n; ++i) {
            h[i] = cmk(std::sin(0.37 * (double)i + 0.5 * r), std::cos(0.11 * (double)i + 0.3 * r));
            if (mixed) hf[i] = make_float2((float)h[i].x, (float)h[i].y);
        }
        rc = check_cuda(c, cudaMemcpyAsync((char *)x + col * r, mixed ? (const void *)hf.data() : (const void *)h.data(),
                                           col, cudaMemcpyHostToDevice, c->st), "repeat check x");
        if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "repeat check x");
    }
    auto mv = [&](void *out) {
        if (mixed) run_matvec(c, (const cf *)x, (cf *)out, nrhs, nullptr);
        else run_matvec(c, (const cd *)x, (cd *)out, nrhs, nullptr);
    };
    if (!rc) rc = check_cuda(c, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * reps, c->st), "repeat check");
    if (!rc) mv(y0);
    const long long nw = (long long)(col * nrhs / 4);
    const int blocks = (int)std::min<long long>((nw + 255) / 256, 4 * 148);
    for (int r = 0; r < reps && !rc; ++r) {
        mv(y);
        k_words_differ<<<blocks, 256, 0, c->st>>>((const unsigned *)y0, (const unsigned *)y, nw, cnt + r);
        c->launches += 1;
        if (r % 64 == 63 || r == reps - 1) rc = check_cuda(c, cudaStreamSynchronize(c->st), "repeat check");
    }
    std::vector<unsigned long long> hc(reps, 0);
    if (!rc) rc = check_cuda(c, cudaMemcpy(hc.data(), cnt, sizeof(unsigned long long) * reps, cudaMemcpyDeviceToHost),
                             "repeat check counts");
    release();
    if (rc) return rc;
    *bad_reps = 0;
    *bad_words = 0;
    for (unsigned long long v : hc) {
        *bad_reps += v != 0;
        *bad_words += (int64_t)v;
    }
    if ((rc = near_status(c))) return rc;
    return check_cuda(c, cudaGetLastError(), "repeat check");
}

// ---------------------------------------------------------------- autotuner
static void put_tuning(scd_ctx *c, const scd_tuning &t) {
    if (t.near_kernel == SCD_NEAR_CUDA_CORES) {
        c->nzm_on = false;
    } else if (t.near_kernel >= SCD_NEAR_TENSOR_SPLIT && t.near_kernel <= SCD_NEAR_TENSOR_WIDE) {
        c->nzm_on = true;
        c->nzm_sched = nzm_sched_of(t.near_kernel);
    }
    c->yz_on = t.fft_passes != SCD_FFT_PASSES_THREE;
    c->scatter_span = std::max(0, t.scatter_span);
    c->gather_span = std::max(0, t.gather_span);
}

static scd_tuning get_tuning(const scd_ctx *c, int nrhs, int precision) {
    scd_tuning t{};
    t.nrhs = nrhs;
    t.precision = precision;
    t.near_kernel = !c->nzm_on ? SCD_NEAR_CUDA_CORES
                    : c->nzm_sched == 0 ? SCD_NEAR_TENSOR_SPLIT
                    : c->nzm_sched == 2 ? SCD_NEAR_TENSOR_WIDE : SCD_NEAR_TENSOR_MERGED;
    t.fft_passes = c->yz_on ? SCD_FFT_PASSES_FUSED_YZ : SCD_FFT_PASSES_THREE;
    t.scatter_span = c->scatter_span;
    t.gather_span = c->gather_span;
    return t;
}

int scd_apply_tuning(scd_ctx *c, const scd_tuning *t) {
    if (!c || !t) return SCD_BAD_ARG;
    if ((t->near_kernel < SCD_NEAR_DEFAULT || t->near_kernel > SCD_NEAR_TENSOR_WIDE) ||
        (t->fft_passes < SCD_FFT_PASSES_DEFAULT || t->fft_passes > SCD_FFT_PASSES_THREE) || t->scatter_span < 0 ||
        t->gather_span < 0)
        return set_error(c, SCD_BAD_ARG, "tuning out of range");
    if (t->near_kernel >= SCD_NEAR_TENSOR_SPLIT && c->have_near && c->near_prec != SCD_STORE_C64)
        return set_error(c, SCD_BAD_ARG, "the tensor-core near zone needs complex64 storage");
    put_tuning(c, *t);
    return SCD_OK;
}

int scd_tune_matvec(scd_ctx *c, int32_t nrhs, int32_t precision, int32_t reps, scd_tuning *out) {
    if (!c || !out || nrhs < 1 || reps < 1) return SCD_BAD_ARG;
    if (precision != SCD_PREC_FP64 && precision != SCD_PREC_MIXED)
        return set_error(c, SCD_BAD_ARG, "precision %d", precision);
    int rc = ready(c);
    if (rc) return rc;
    auto time_of = [&](const scd_tuning &t, double *ms) {
        put_tuning(c, t);
        const int r = scd_profile_matvec(c, reps, nrhs, precision);
        *ms = c->t_matvec;
        return r;
    };
    scd_tuning best = get_tuning(c, nrhs, precision);
    double best_ms = 0;
    if ((rc = time_of(best, &best_ms))) return rc;
    const double default_ms = best_ms;
    // one knob at a time, the others at their best so far
    auto knob = [&](int32_t scd_tuning::*field, std::initializer_list<int32_t> values) -> int {
        for (int32_t v : values) {
            if (best.*field == v) continue;
            scd_tuning t = best;
            t.*field = v;
            double ms = 0;
            const int r = time_of(t, &ms);
            if (r) return r;
            if (ms < best_ms) { best = t; best_ms = ms; }
        }
        return SCD_OK;
    };
    if (precision == SCD_PREC_MIXED && c->near_prec == SCD_STORE_C64 && c->nb == 1 &&
        (rc = knob(&scd_tuning::near_kernel,
                   {SCD_NEAR_CUDA_CORES, SCD_NEAR_TENSOR_SPLIT, SCD_NEAR_TENSOR_MERGED, SCD_NEAR_TENSOR_WIDE})))
        return rc;
    if ((rc = knob(&scd_tuning::fft_passes, {SCD_FFT_PASSES_FUSED_YZ, SCD_FFT_PASSES_THREE}))) return rc;
    if (nrhs > 8 && (rc = knob(&scd_tuning::scatter_span, {0, 8, 16}))) return rc;
    if (nrhs > 4 && (rc = knob(&scd_tuning::gather_span, {0, 4, 8, 16}))) return rc;
    put_tuning(c, best);
    best.matvec_ms = best_ms;
    best.default_ms = default_ms;
    *out = best;
    return SCD_OK;
}

int scd_column_latency(scd_ctx *c, int32_t ncol, double *ms) {
    if (!c || !ms) return SCD_BAD_ARG;
    if ((size_t)ncol != c->col_latency_ms.size())
        return set_error(c, SCD_BAD_ARG, "ncol = %d, last solve had %zu columns", ncol, c->col_latency_ms.size());
    for (int i = 0; i < ncol; ++i) ms[i] = c->col_latency_ms[i];
    return SCD_OK;
}

int64_t scd_nearzone_bytes(scd_ctx *c) {
    if (!c || !c->have_near) return -1;
    return (int64_t)c->tile_store * (c->near_prec == SCD_STORE_C64 ? 8 : 16);
}

// the device-built incident columns vswf2constant (src/T_matrix.f90:280-305)
// for Nmax at the current wavenumber, kept in c->d_mat
static int ensure_vswf(scd_ctx *c, int Nmax) {
    if (c->d_mat && c->mat_Nmax == Nmax && c->mat_k == c->k) return SCD_OK;
    const int ntot = 2 * ((Nmax + 1) * (Nmax + 1) - 1);
    cudaFree(c->d_mat);
    c->d_mat = nullptr;
    c->mat_cols = 0;
    c->mat_Nmax = -1;
    int rc;
    if ((rc = dalloc(c, &c->d_mat, (size_t)c->n * ntot, "resident VSWF columns"))) return rc;
    if ((rc = setup_vswf(c, Nmax, c->d_mat))) return rc;
    c->mat_Nmax = Nmax;
    c->mat_k = c->k;
    c->mat_cols = ntot;
    return SCD_OK;
}

// compute_T_matrix over the listed columns (0-based, any order, each once);
// T(:, j) = i k^3 mat^H x_{list[j]}
static int compute_T_list(scd_ctx *c, int32_t Nmax, const scd_solve_opts *o, int ncol, const int32_t *list,
                          scd_c128 *T, int32_t *iters, const char *who) {
    cudaSetDevice(c->dev);
    // the incident columns are constant-basis (vswf2constant); the reference
    // has no linear-basis T-matrix solve (src/T_matrix.f90:250-259)
    if (c->nb != 1) return set_error(c, SCD_BAD_ARG, "%s: constant basis only", who);
    int rc = ready(c);
    if (rc) return rc;
    if ((rc = check_opts(c, o))) return rc;
    const int nm = (Nmax + 1) * (Nmax + 1) - 1, ntot = 2 * nm;
    {
        std::vector<char> seen(ntot, 0);
        for (int j = 0; j < ncol; ++j) {
            if (list[j] < 0 || list[j] >= ntot || seen[list[j]])
                return set_error(c, SCD_BAD_ARG, "%s: column %d outside 1..%d or listed twice", who, list[j] + 1, ntot);
            seen[list[j]] = 1;
        }
    }
    const long long n = c->n;
    // the incident matrix stays resident unless it would take more than a
    // quarter of the free device memory (C5: 1350 columns of 3.6 M unknowns,
    // 78 GB): then it is built in chunks of VSWF_CHUNK columns, once for the
    // listed right-hand sides and once more for the rows of T
    constexpr int VSWF_CHUNK = 64;
    size_t dev_free = 0, dev_total = 0;
    cudaMemGetInfo(&dev_free, &dev_total);
    const bool resident = (c->d_mat && c->mat_Nmax == Nmax && c->mat_k == c->k) ||
                          sizeof(cd) * (size_t)n * ntot <= dev_free / 4;
    cd *d_X = nullptr, *d_T = nullptr, *d_B = nullptr, *d_chunk = nullptr, *d_Tc = nullptr;
    auto release = [&]() { cudaFree(d_X); cudaFree(d_T); cudaFree(d_B); cudaFree(d_chunk); cudaFree(d_Tc); };
    if (resident && (rc = ensure_vswf(c, Nmax))) return rc;
    if ((rc = dalloc(c, &d_X, (size_t)n * ncol, "X")) || (rc = dalloc(c, &d_T, (size_t)ntot * ncol, "T"))) {
        release();
        return rc;
    }
    if (!resident && ((rc = dalloc(c, &d_B, (size_t)n * ncol, "right-hand sides")) ||
                      (rc = dalloc(c, &d_chunk, (size_t)n * VSWF_CHUNK, "VSWF chunk")) ||
                      (rc = dalloc(c, &d_Tc, (size_t)VSWF_CHUNK * ncol, "T chunk")))) {
        release();
        return rc;
    }
    cudaEventRecord(c->ev[4], c->st);
    std::vector<const cd *> cols(ncol);
    if (resident) {
        for (int j = 0; j < ncol; ++j) cols[j] = c->d_mat + (size_t)n * list[j];
    } else {
        for (int c0 = 0; c0 < ntot && !rc; c0 += VSWF_CHUNK) {
            const int cw = std::min(VSWF_CHUNK, ntot - c0);
            bool any = false;
            for (int j = 0; j < ncol; ++j) any = any || (list[j] >= c0 && list[j] < c0 + cw);
            if (!any) continue;
            if ((rc = setup_vswf(c, Nmax, d_chunk, c0, cw))) break;
            for (int j = 0; j < ncol && !rc; ++j)
                if (list[j] >= c0 && list[j] < c0 + cw)
                    rc = check_cuda(c, cudaMemcpyAsync(d_B + (size_t)n * j, d_chunk + (size_t)n * (list[j] - c0),
                                                       sizeof(cd) * n, cudaMemcpyDeviceToDevice, c->st), "right-hand side");
        }
        if (rc) { release(); return rc; }
        for (int j = 0; j < ncol; ++j) cols[j] = d_B + (size_t)n * j;
    }
    const int ns = o->block > 0 ? o->block : ncol;
    std::vector<int> it(ncol, 0);
    int worst = batch_solve(c, ncol, cols.data(), d_X, o->tol, o->m, o->cycles, ns, it.data(), nullptr, nullptr,
                            nullptr, o->precision, o->inner_tol, o->max_outer);
    if (worst == SCD_OK || worst == SCD_NOT_CONVERGED) {
        const int ns_ = near_status(c);
        if (ns_) worst = ns_;
    }
    if (iters) for (int j = 0; j < ncol; ++j) iters[j] = it[j];
    if (worst == SCD_OK || worst == SCD_NOT_CONVERGED) {
        if (resident) {
            launch_T_assemble(c, c->d_mat, ntot, 0, ncol, d_X, d_T);
        } else {
            // rows c0 .. c0 + cw - 1 of T from the chunk's columns; every
            // entry is summed as in the resident path (same K split)
            for (int c0 = 0; c0 < ntot && !rc; c0 += VSWF_CHUNK) {
                const int cw = std::min(VSWF_CHUNK, ntot - c0);
                if ((rc = setup_vswf(c, Nmax, d_chunk, c0, cw))) break;
                launch_T_assemble(c, d_chunk, cw, 0, ncol, d_X, d_Tc);
                rc = check_cuda(c, cudaMemcpy2DAsync(d_T + c0, sizeof(cd) * ntot, d_Tc, sizeof(cd) * cw, sizeof(cd) * cw,
                                                     ncol, cudaMemcpyDeviceToDevice, c->st), "T rows");
            }
            if (rc) worst = rc;
        }
        cudaEventRecord(c->ev[5], c->st);
        std::vector<cd> h((size_t)ntot * ncol);
        rc = check_cuda(c, cudaMemcpyAsync(h.data(), d_T, sizeof(cd) * h.size(), cudaMemcpyDeviceToHost, c->st), "T");
        if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), who);
        if (!rc) {
            // T_mat * i k^3 (src/T_matrix.f90:270-275)
            const double k3 = std::pow(c->k, 3.0);
            for (size_t i = 0; i < h.size(); ++i) T[i] = scd_c128{-k3 * h[i].y, k3 * h[i].x};
            float ms = 0;
            cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]);
            c->last_call_ms = ms;
            c->accum_ms += ms;
        } else {
            worst = rc;
        }
    }
    cudaStreamSynchronize(c->st);
    release();
    return worst;
}

int scd_compute_T_matrix(scd_ctx *c, int32_t Nmax, const scd_solve_opts *o, int32_t col0, int32_t ncol,
                         scd_c128 *T, int32_t *iters) {
    if (!c || !o || !T || Nmax < 1) return SCD_BAD_ARG;
    const int ntot = 2 * ((Nmax + 1) * (Nmax + 1) - 1);
    if (col0 < 0 || ncol < 1 || col0 + ncol > ntot)
        return set_error(c, SCD_BAD_ARG, "columns %d..%d outside 1..%d", col0 + 1, col0 + ncol, ntot);
    std::vector<int32_t> list(ncol);
    for (int j = 0; j < ncol; ++j) list[j] = col0 + j;
    return compute_T_list(c, Nmax, o, ncol, list.data(), T, iters, "scd_compute_T_matrix");
}

int scd_compute_T_columns(scd_ctx *c, int32_t Nmax, const scd_solve_opts *o, int32_t ncol, const int32_t *cols,
                          scd_c128 *T, int32_t *iters) {
    if (!c || !o || !T || !cols || Nmax < 1 || ncol < 1) return SCD_BAD_ARG;
    return compute_T_list(c, Nmax, o, ncol, cols, T, iters, "scd_compute_T_columns");
}

}  // extern "C"

// ------------------------------------------------------------ wavelength sweep
namespace {
// every column of every wavelength, wavelength after wavelength; column j of
// wavelength w is solved with operator w
struct SweepSource final : ColumnSource {
    std::vector<scd_ctx *> ops;
    std::vector<int> ncol;
    std::vector<cd *> X;
    std::vector<int32_t *> iters;
    std::vector<std::pair<int, int>> jobs;   // tag -> (wavelength, column)
    size_t next_job = 0;
    std::vector<int> worst;
    bool next(const cd **rhs, cd **xout, int *tag) override {
        if (next_job >= jobs.size()) return false;
        const auto [w, j] = jobs[next_job];
        const long long n = ops[w]->n;
        *rhs = ops[w]->d_mat + (size_t)j * n;
        *xout = X[w] + (size_t)j * n;
        *tag = (int)next_job++;
        return true;
    }
    void finished(int tag, int it, int cv, int st, double) override {
        const auto [w, j] = jobs[tag];
        if (iters[w]) iters[w][j] = it;
        if (st != SCD_OK) worst[w] = st;
        else if (!cv && worst[w] == SCD_OK) worst[w] = SCD_NOT_CONVERGED;
    }
    int op_of(int tag) override { return jobs[tag].first; }
    // jobs are in wavelength order: w has columns left while the next job is
    // at or before its last
    std::vector<size_t> last_job;
    bool op_pending(int op) override { return next_job <= last_job[op]; }
};
}  // namespace

extern "C" {

int scd_solve_sweep(scd_ctx *const *ctxs, int32_t nw, const int32_t *Nmax, const scd_solve_opts *o, scd_c128 *const *T,
                    int32_t *const *iters, int32_t *status) {
    if (!ctxs || nw < 1 || !Nmax || !o || !T) return SCD_BAD_ARG;
    scd_ctx *c = ctxs[0];
    if (!c) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    int rc = SCD_OK;
    for (int w = 0; w < nw; ++w) {
        scd_ctx *cw = ctxs[w];
        if (!cw || Nmax[w] < 1 || !T[w]) return set_error(c, SCD_BAD_ARG, "wavelength %d: null context, Nmax or T", w);
        if (cw->dev != c->dev || cw->n != c->n)
            return set_error(c, SCD_BAD_ARG, "wavelength %d: the sweep's contexts share one device and one mesh", w);
        if (cw->nb != 1) return set_error(c, SCD_BAD_ARG, "scd_solve_sweep: constant basis only");
        for (int v = 0; v < w; ++v)
            if (ctxs[v] == cw) return set_error(c, SCD_BAD_ARG, "wavelength %d repeats the context of %d", w, v);
        if ((rc = ready(cw)) || (rc = check_opts(cw, o)) || (rc = ensure_vswf(cw, Nmax[w])))
            return set_error(c, rc, "wavelength %d: %s", w, cw->err.c_str());
    }
    if ((rc = check_opts(c, o))) return rc;
    SweepSource src;
    src.ops.assign(ctxs, ctxs + nw);
    src.worst.assign(nw, SCD_OK);
    auto release = [&]() { for (cd *p : src.X) cudaFree(p); };
    for (int w = 0; w < nw; ++w) {
        const int ncol = 2 * ((Nmax[w] + 1) * (Nmax[w] + 1) - 1);
        src.ncol.push_back(ncol);
        src.iters.push_back(iters ? iters[w] : nullptr);
        cd *X = nullptr;
        if ((rc = dalloc(c, &X, (size_t)c->n * ncol, "sweep solutions"))) { release(); return rc; }
        src.X.push_back(X);
        for (int j = 0; j < ncol; ++j) src.jobs.emplace_back(w, j);
        src.last_job.push_back(src.jobs.size() - 1);
    }
    cudaEventRecord(c->ev[4], c->st);
    const int ns = o->block > 0 ? o->block : 64;
    rc = batch_run(c, src, o->tol, o->m, o->cycles, ns, o->precision, o->inner_tol, o->max_outer, &src.ops);
    if (rc) { release(); return rc; }
    cudaEventRecord(c->ev[5], c->st);   // the solve's end: every column of every wavelength
    int worst = SCD_OK;
    for (int w = 0; w < nw && !rc; ++w) {
        scd_ctx *cw = ctxs[w];
        const int ns_ = near_status(cw);
        if (ns_) { rc = set_error(c, ns_, "wavelength %d: %s", w, cw->err.c_str()); break; }
        // T_mat = mat^H X times i k^3 (src/T_matrix.f90:260, 271-275), on the
        // wavelength's stream after the solver's stream
        const int ncol = src.ncol[w];
        cd *d_T = nullptr;
        if ((rc = dalloc(c, &d_T, (size_t)ncol * ncol, "sweep T"))) break;
        cudaStreamWaitEvent(cw->st, c->ev[5], 0);
        launch_T_assemble(cw, cw->d_mat, ncol, 0, ncol, src.X[w], d_T);
        std::vector<cd> h((size_t)ncol * ncol);
        rc = check_cuda(c, cudaMemcpyAsync(h.data(), d_T, sizeof(cd) * h.size(), cudaMemcpyDeviceToHost, cw->st), "T");
        if (!rc) rc = check_cuda(c, cudaStreamSynchronize(cw->st), "sweep T");
        cudaFree(d_T);
        if (rc) break;
        const double k3 = std::pow(cw->k, 3.0);
        for (size_t i = 0; i < h.size(); ++i) T[w][i] = scd_c128{-k3 * h[i].y, k3 * h[i].x};
        if (status) status[w] = src.worst[w];
        if (src.worst[w] != SCD_OK && src.worst[w] != SCD_NOT_CONVERGED) worst = src.worst[w];
        else if (src.worst[w] == SCD_NOT_CONVERGED && worst == SCD_OK) worst = SCD_NOT_CONVERGED;
    }
    cudaEventSynchronize(c->ev[5]);
    if (!rc) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]);
        c->last_call_ms = ms;
        c->accum_ms += ms;
    }
    release();
    return rc ? rc : worst;
}

}  // extern "C"
