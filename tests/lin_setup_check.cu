// Host run of the linear-basis set-up arithmetic (scadyn_b200/csrc/lin_setup.cuh)
// that k_near_build_lin and k_projectors_lin execute on the device.
//
// Reads a binary request on stdin and writes the results on stdout:
//   int32 mode = 0, int32 npairs, then per tet pair
//     double k, eps (re, im); int32 self; double T[12], B[12]; double volT, volB;
//     cd st[432] (test projectors [node][S,Sx,Sy,Sz][27]);
//     cd gp[432] (G times the basis projectors [node][kind][27])
//   -> per pair the 12x12 block, entry e = row + 12 col (cd)
//   int32 mode = 1, int32 nsamples, then per sample
//     double tet[12], vol, r[3], k
//   -> per sample q[4] and q2[3][4] (cd): the node integrals of pfft_projection_lin
// The three phases of a block run in the kernel's item order, one item at a time.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "lin_setup.cuh"

struct HostQ {
    static const HostQuad &q() {
        static HostQuad h;
        return h;
    }
    static double t5(int i, int c) { return q().t5[i][c]; }
    static double r5(int i, int c) { return q().r5[i][c]; }
};

template <typename X>
static bool rd(X *p, size_t n) { return fread(p, sizeof(X), n, stdin) == n; }

int main() {
    int32_t mode, n;
    if (!rd(&mode, 1) || !rd(&n, 1)) return 2;
    if (mode == 0) {
        std::vector<cd> scr(LIN_POINTS * LIN_SCR), sm(LIN_SMALL), st(432), gp(432), out(144);
        for (int q = 0; q < n; ++q) {
            double k, eps[2], T[12], B[12], vT, vB;
            int32_t self;
            if (!rd(&k, 1) || !rd(eps, 2) || !rd(&self, 1) || !rd(T, 12) || !rd(B, 12) || !rd(&vT, 1) || !rd(&vB, 1) ||
                !rd((double *)st.data(), 864) || !rd((double *)gp.data(), 864))
                return 3;
            LinPair p;
            lin_pair_init(p, T, B, vT, vB, k, cmk(eps[0], eps[1]), self != 0);
            for (int it = 0; it < LIN_ITEMS; ++it) lin_point<HostQ>(p, it, scr.data());
            for (int i = 0; i < LIN_SMALL; ++i) lin_small<HostQ>(p, i, scr.data(), sm.data());
            for (int e = 0; e < 144; ++e) out[e] = lin_entry<HostQ>(p, e, scr.data(), sm.data(), st.data(), gp.data());
            fwrite(out.data(), sizeof(cd), 144, stdout);
        }
    } else if (mode == 1) {
        for (int q = 0; q < n; ++q) {
            double t[12], vol, r[3], k;
            if (!rd(t, 12) || !rd(&vol, 1) || !rd(r, 3) || !rd(&k, 1)) return 3;
            V3 v[4];
            for (int i = 0; i < 4; ++i) v[i] = V3{t[3 * i], t[3 * i + 1], t[3 * i + 2]};
            cd qq[4], q2[3][4];
            lin_proj_sample<HostQ>(v, vol, V3{r[0], r[1], r[2]}, k, qq, q2);
            fwrite(qq, sizeof(cd), 4, stdout);
            fwrite(q2, sizeof(cd), 12, stdout);
        }
    } else {
        return 4;
    }
    return 0;
}
