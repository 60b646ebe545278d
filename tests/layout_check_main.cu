// Host run of the production slot and tile layout (set_order and
// build_tile_layout, scadyn_b200/csrc/api.cu, linked from the library's
// objects) on a binning read from stdin, and of check_layout
// (scadyn_b200/csrc/layout_check.h) on planted inconsistencies.  No GPU is
// needed: the layout tables are built on the host before the first device
// allocation, whose failure ends each call.
// stdin: int32 ncx, ncy, ncz, nb, T (basis functions), then T int32 box ids.
// Prints "production layout: ok" when build_tile_layout's check accepts the
// production layout, then "rejected: <what>" for every planted inconsistency
// and "planted: N of N rejected".  Exits non-zero on a failure.
#include <cstdint>
#include <cstdio>
#include <functional>
#include <vector>

#include "ctx.h"
#include "layout_check.h"

int set_order_from_cubes(scd_ctx *c, const std::vector<int> &cube_of_tet);
int build_tile_layout(scd_ctx *c);

int main() {
    int32_t h[5];
    if (fread(h, 4, 5, stdin) != 5) return 2;
    std::vector<int32_t> cube(h[4]);
    if (fread(cube.data(), 4, cube.size(), stdin) != cube.size()) return 2;
    scd_ctx *c = new scd_ctx();
    c->ncx = h[0]; c->ncy = h[1]; c->ncz = h[2]; c->ncubes = h[0] * h[1] * h[2];
    c->nb = h[3]; c->T = h[4]; c->n = 3LL * c->T;
    set_order_from_cubes(c, std::vector<int>(cube.begin(), cube.end()));   // tables, then a failed allocation
    c->err.clear();
    build_tile_layout(c);                          // tiles, check_layout, then a failed allocation
    if (c->err.find("layout check") != std::string::npos || c->ngroups == 0) {
        printf("production layout rejected: %s\n", c->err.c_str());
        return 1;
    }
    printf("production layout: ok (%d groups; the upload then stopped: %s)\n", c->ngroups, c->err.c_str());

    // a valid two-group layout by hand (check_layout sees only the tables):
    // group 0 = 2 tets in box 0, group 1 = 3 tets in box 1, tiles (0,0), (0,1), (1,1)
    const int nb = c->nb, n0 = 2 * nb, n1 = 3 * nb, T = n0 + n1;
    std::vector<int> perm(T), slot_of(T), cos(T), co{0, n0, T}, go{0, n0, T}, gc{0, 1}, gt{0, 2, 3}, pc{2, 1};
    for (int s = 0; s < T; ++s) { perm[s] = s; slot_of[s] = s; cos[s] = s < n0 ? 0 : 1; }
    std::vector<long long> pb{0, 2LL * 3 * n0, 2LL * 3 * n0 + 3LL * n1};
    std::vector<NearTile> tl(3);
    tl[0] = NearTile{0, 0, 0, 0, 0, 0, n0, n0, 0, -1};
    tl[1] = NearTile{0, 1, 0, 1, 0, n0, n0, n1, tile_elems(n0, n0), -1};
    tl[2] = NearTile{1, 1, 1, 1, n0, n0, n1, n1, tile_elems(n0, n0) + tile_elems(n0, n1), -1};
    // the transposed product of tile (0, 1) goes to group 1's second partial slot
    tl[1].col_off = pb[1] + 3LL * n1;
    pc[1] = 2;
    pb[2] = pb[1] + 2LL * 3 * n1;
    long long store = tl[2].data_off + tile_elems(n1, n1);
    auto V = [&]() {
        return LayoutView{T, nb, 2, 2, &perm, &slot_of, &cos, &co, &go, &gc, &gt, &tl, &pb, &pc, store};
    };
    std::string why = check_layout(V());
    if (!why.empty()) { printf("hand-built layout rejected: %s\n", why.c_str()); return 1; }
    int planted = 0, caught = 0;
    auto plant = [&](const char *what, std::function<void()> spoil, std::function<void()> undo) {
        spoil();
        const std::string w = check_layout(V());
        ++planted;
        if (!w.empty()) { ++caught; printf("rejected: %s -> %s\n", what, w.c_str()); }
        else printf("NOT rejected: %s\n", what);
        undo();
    };
    plant("perm not inverted", [&] { std::swap(perm[0], perm[1]); }, [&] { std::swap(perm[0], perm[1]); });
    plant("box offsets past T", [&] { co[2] = T + 1; }, [&] { co[2] = T; });
    plant("slot outside its box", [&] { cos[0] = 1; }, [&] { cos[0] = 0; });
    plant("group larger than the limit", [&] { go[1] = SCD_GROUP_MAX + 1; }, [&] { go[1] = n0; });
    plant("tile data offset out of sequence", [&] { tl[1].data_off += 2; }, [&] { tl[1].data_off -= 2; });
    plant("tile slots not its group's", [&] { tl[2].s1 += 1; }, [&] { tl[2].s1 -= 1; });
    plant("tiles out of order", [&] { std::swap(tl[0], tl[1]); }, [&] { std::swap(tl[0], tl[1]); });
    plant("transposed slot past the group's slots", [&] { tl[1].col_off += 3LL * n1; }, [&] { tl[1].col_off -= 3LL * n1; });
    plant("transposed slot on a row-sum slot", [&] { tl[1].col_off = pb[1]; }, [&] { tl[1].col_off = pb[1] + 3LL * n1; });
    plant("diagonal tile with a transposed slot", [&] { tl[0].col_off = 0; }, [&] { tl[0].col_off = -1; });
    plant("storage smaller than the tiles", [&] { store -= 2; }, [&] { store += 2; });
    plant("group tile range wrong", [&] { gt[1] = 1; }, [&] { gt[1] = 2; });
    if (nb == 4) plant("group not whole tets", [&] { go[1] = n0 - 1; cos[n0 - 1] = 1; co[1] = n0 - 1; },
                       [&] { go[1] = n0; cos[n0 - 1] = 0; co[1] = n0; });
    printf("planted: %d of %d rejected\n", caught, planted);
    return caught == planted ? 0 : 1;
}
