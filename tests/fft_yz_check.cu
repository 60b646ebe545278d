// Host check of the fused y-z FFT pass (scadyn_b200/csrc/fft_yz.cuh): runs
// the pass on one plane with the CTA's threads in turn (yz_plane_host, the
// kernel's phases in the kernel's order) and compares with a direct
// separable DFT convolution in double precision:
//   out[z][y] = sum_{ky,kz} e^{+i(ky y/PY + kz z/PZ) 2pi} G(fx,|ky|,|kz|)
//               sum_{z'<Nz,y'<Ny} e^{-i(ky y'/PY + kz z'/PZ) 2pi} in[z'][y']
// for z < Nz, y < Ny.  The shared-memory image and the plane are allocated
// to their exact sizes with NaN canaries behind them: a write past the end
// shows as a changed canary, a read past the end as NaN in the result.
// Prints the relative error per case and exits non-zero above the bound.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fft_yz.cuh"

typedef std::complex<double> Z;

template <typename C> C mk(double r, double i);
template <> cd mk<cd>(double r, double i) { return make_double2(r, i); }
template <> cf mk<cf>(double r, double i) { return make_float2((float)r, (float)i); }

static unsigned g_state = 12345u;
static double urand() {
    g_state = g_state * 1664525u + 1013904223u;
    return (g_state >> 8) / 16777216.0 - 0.5;
}

template <int PY, int PZ, typename C>
double check(int Ny, int Nz, int Px, int x, bool &canary_ok) {
    YzDims D;
    D.Nx = Px / 2; D.Ny = Ny; D.Nz = Nz; D.NzR = yz_round8(Nz); D.Px = Px;
    D.Hx = Px / 2 + 1; D.Hy = PY / 2 + 1; D.Hz = PZ / 2 + 1;
    const int CAN = 64;
    const double nan = std::nan("");
    // the plane, the transposed Green octant, the twiddles, the shared-memory image
    std::vector<C> W(Nz * Ny + CAN, mk<C>(nan, nan));
    std::vector<Z> in(Nz * Ny);
    for (int i = 0; i < Nz * Ny; ++i) {
        W[i] = mk<C>(urand(), urand());
        in[i] = Z((double)W[i].x, (double)W[i].y);
    }
    const long long no = (long long)D.Hx * D.Hy * D.Hz;
    std::vector<C> F(no);
    for (long long i = 0; i < no; ++i) F[i] = mk<C>(urand(), urand());
    std::vector<C> twy(PY), twz(PZ);
    for (int i = 0; i < PY; ++i) twy[i] = mk<C>(std::cos(-2 * M_PI * i / PY), std::sin(-2 * M_PI * i / PY));
    for (int i = 0; i < PZ; ++i) twz[i] = mk<C>(std::cos(-2 * M_PI * i / PZ), std::sin(-2 * M_PI * i / PZ));
    const long long ns = yz_smem_elems<PY, PZ>(D.NzR);
    std::vector<C> sm(ns + CAN, mk<C>(nan, nan));
    yz_plane_host<PY, PZ, C>(W.data(), F.data(), twy.data(), twz.data(), x, D, sm.data());
    for (int i = 0; i < CAN; ++i) {
        if (!std::isnan((double)W[Nz * Ny + i].x) || !std::isnan((double)sm[ns + i].x)) canary_ok = false;
    }
    // direct separable convolution
    const int fx = yz_fold(x, Px);
    std::vector<Z> U(PZ * PY);   // U[kz][ky]
    for (int kz = 0; kz < PZ; ++kz)
        for (int ky = 0; ky < PY; ++ky) {
            Z s = 0;
            for (int z = 0; z < Nz; ++z)
                for (int y = 0; y < Ny; ++y)
                    s += in[z * Ny + y] * std::polar(1.0, -2 * M_PI * (((long)ky * y % PY) / (double)PY +
                                                                       ((long)kz * z % PZ) / (double)PZ));
            const C f = F[((long long)fx * D.Hy + yz_fold(ky, PY)) * D.Hz + yz_fold(kz, PZ)];
            U[kz * PY + ky] = s * Z((double)f.x, (double)f.y);
        }
    double err = 0, nrm = 0;
    for (int z = 0; z < Nz; ++z)
        for (int y = 0; y < Ny; ++y) {
            Z s = 0;
            for (int kz = 0; kz < PZ; ++kz)
                for (int ky = 0; ky < PY; ++ky)
                    s += U[kz * PY + ky] * std::polar(1.0, 2 * M_PI * (((long)ky * y % PY) / (double)PY +
                                                                      ((long)kz * z % PZ) / (double)PZ));
            const Z got((double)W[z * Ny + y].x, (double)W[z * Ny + y].y);
            err += std::norm(got - s);
            nrm += std::norm(s);
        }
    return std::sqrt(err / nrm);
}

int main() {
    int bad = 0;
    bool can = true;
    struct R { const char *name; double e, bound; } r[] = {
        // C2's y and z lengths (Ny = 54, Nz = 40) in both precisions, x on both sides of Px/2
        {"128x80 f64 x=3", check<128, 80, cd>(54, 40, 128, 3, can), 1e-13},
        {"128x80 f32 x=100", check<128, 80, cf>(54, 40, 128, 100, can), 2e-6},
        // powers of two, Nz not a multiple of 8 (padding rows)
        {"64x64 f64", check<64, 64, cd>(30, 27, 64, 31, can), 1e-13},
        {"64x128 f32", check<64, 128, cf>(32, 61, 64, 7, can), 2e-6},
        // 5-smooth lengths with 4 and 8 threads per line, PY not a multiple of the chunk
        {"80x96 f64", check<80, 96, cd>(37, 45, 80, 41, can), 1e-13},
        {"96x192 f32", check<96, 192, cf>(48, 70, 96, 0, can), 2e-6},
        {"192x80 f64", check<192, 80, cd>(90, 33, 192, 96, can), 1e-13},
    };
    for (auto &x : r) {
        std::printf("%s %.3e\n", x.name, x.e);
        if (!(x.e < x.bound)) bad = 1;
    }
    if (!can) {
        std::printf("a canary behind the plane or the shared-memory image changed\n");
        bad = 1;
    }
    return bad;
}
