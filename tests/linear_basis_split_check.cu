// Host check of the near-zone box split (scadyn_b200/csrc/linear_basis.h,
// split_box): for one basis function per tet it reproduces the constant-basis
// split (ceil(n / 24) runs, sizes differing by at most one); for four per tet
// every run holds whole tets, at most 24 basis functions, sizes differing by
// at most one tet, and the runs cover the box.  Exits non-zero on a failure.
#include <cstdio>
#include <vector>

#include "linear_basis.h"

int main() {
    const int GMAX = 24;
    int bad = 0;
    std::vector<int> sz(4 * 400 + 1);
    for (int n = 0; n <= 400; ++n) {
        // nb = 1: the constant-basis rule
        int ng = split_box(n, 1, GMAX, sz.data());
        const int want = n == 0 ? 0 : (n + GMAX - 1) / GMAX;
        int sum = 0, lo = 1 << 30, hi = 0;
        for (int g = 0; g < ng; ++g) { sum += sz[g]; lo = sz[g] < lo ? sz[g] : lo; hi = sz[g] > hi ? sz[g] : hi; }
        if (ng != want || sum != n || (ng && (hi - lo > 1 || hi > GMAX))) { printf("nb=1 n=%d wrong\n", n); ++bad; }
        for (int g = 0; g < ng; ++g)
            if (sz[g] != n / ng + (g < n % ng ? 1 : 0)) { printf("nb=1 n=%d run %d size %d\n", n, g, sz[g]); ++bad; }
        // nb = 4: whole tets
        const int m = 4 * n;
        ng = split_box(m, 4, GMAX, sz.data());
        sum = 0; lo = 1 << 30; hi = 0;
        for (int g = 0; g < ng; ++g) {
            if (sz[g] % 4 || sz[g] > GMAX || sz[g] == 0) { printf("nb=4 n=%d run %d size %d\n", n, g, sz[g]); ++bad; }
            sum += sz[g]; lo = sz[g] < lo ? sz[g] : lo; hi = sz[g] > hi ? sz[g] : hi;
        }
        if (sum != m || (ng && hi - lo > 4) || ng != (n == 0 ? 0 : (n + 5) / 6)) { printf("nb=4 n=%d wrong (ng %d)\n", n, ng); ++bad; }
    }
    printf("box split: %d failures\n", bad);
    return bad ? 1 : 0;
}
