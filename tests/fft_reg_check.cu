// Host check of the register line FFT (scadyn_b200/csrc/fft_reg.cuh): runs
// the phases of the 8 threads of a line in order, as the warp does, and
// compares with a direct DFT in double precision.  Prints the largest
// relative error per (P, direction, precision) and exits non-zero above the
// stated bound.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "fft_reg.cuh"

template <typename C> C mk(double r, double i);
template <> cd mk<cd>(double r, double i) { return make_double2(r, i); }
template <> cf mk<cf>(double r, double i) { return make_float2((float)r, (float)i); }

template <int P, bool INV, typename C>
double check(unsigned seed) {
    C tw[P];
    for (int i = 0; i < P; ++i) tw[i] = mk<C>(std::cos(-2.0 * M_PI * i / P), std::sin(-2.0 * M_PI * i / P));
    const int LS = P + (P >> 4) + 1;
    C s[LS];
    double xr[P], xi[P];
    unsigned st = seed;
    for (int n = 0; n < P; ++n) {
        st = st * 1664525u + 1013904223u; xr[n] = (st >> 8) / 16777216.0 - 0.5;
        st = st * 1664525u + 1013904223u; xi[n] = (st >> 8) / 16777216.0 - 0.5;
        s[pidx(n)] = mk<C>(xr[n], xi[n]);
        xr[n] = (double)s[pidx(n)].x; xi[n] = (double)s[pidx(n)].y;
    }
    C v[8][P / 8];
    for (int t = 0; t < 8; ++t) regfft_A<P, INV>(s, tw, t, v[t]);
    for (int t = 0; t < 8; ++t) regfft_A_store<P>(s, t, v[t]);
    C u[8][RegFft<P>::PER][8];
    for (int t = 0; t < 8; ++t) regfft_B<P, INV>(s, tw, t, u[t]);
    for (int t = 0; t < 8; ++t) regfft_B_store<P>(s, t, u[t]);
    double err = 0, nrm = 0;
    for (int f = 0; f < P; ++f) {
        double re = 0, im = 0;
        for (int n = 0; n < P; ++n) {
            const double ang = (INV ? 2.0 : -2.0) * M_PI * (double)((long)n * f % P) / P;
            re += xr[n] * std::cos(ang) - xi[n] * std::sin(ang);
            im += xr[n] * std::sin(ang) + xi[n] * std::cos(ang);
        }
        const double dr = s[pidx(f)].x - re, di = s[pidx(f)].y - im;
        err += dr * dr + di * di;
        nrm += re * re + im * im;
    }
    return std::sqrt(err / nrm);
}

int main() {
    int bad = 0;
    struct R { const char *name; double e, bound; } r[] = {
        {"P64 fwd f64", check<64, false, cd>(1), 1e-14}, {"P64 inv f64", check<64, true, cd>(2), 1e-14},
        {"P128 fwd f64", check<128, false, cd>(3), 1e-14}, {"P128 inv f64", check<128, true, cd>(4), 1e-14},
        {"P64 fwd f32", check<64, false, cf>(5), 1e-6}, {"P128 inv f32", check<128, true, cf>(6), 1e-6},
    };
    for (auto &x : r) {
        std::printf("%s %.3e\n", x.name, x.e);
        if (!(x.e < x.bound)) bad = 1;
    }
    return bad;
}
