// Host check of the mixed-radix register line FFT (scadyn_b200/csrc/fft_mixed.cuh):
// runs the phases of the T threads of a line in order, as the warp does, and
// compares with a direct DFT in double precision for 5-smooth lengths.
// Prints the relative error per (P, T, direction, precision) and exits
// non-zero above the stated bound.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fft_mixed.cuh"

template <typename C> C mk(double r, double i);
template <> cd mk<cd>(double r, double i) { return make_double2(r, i); }
template <> cf mk<cf>(double r, double i) { return make_float2((float)r, (float)i); }

template <int P, int T, bool INV, typename C>
double check(unsigned seed) {
    std::vector<C> tw(P);
    for (int i = 0; i < P; ++i) tw[i] = mk<C>(std::cos(-2.0 * M_PI * i / P), std::sin(-2.0 * M_PI * i / P));
    const int LS = P + (P >> 4) + 1;
    std::vector<C> s(LS);
    std::vector<double> xr(P), xi(P);
    unsigned st = seed;
    for (int n = 0; n < P; ++n) {
        st = st * 1664525u + 1013904223u; xr[n] = (st >> 8) / 16777216.0 - 0.5;
        st = st * 1664525u + 1013904223u; xi[n] = (st >> 8) / 16777216.0 - 0.5;
        s[pidx(n)] = mk<C>(xr[n], xi[n]);
        xr[n] = (double)s[pidx(n)].x; xi[n] = (double)s[pidx(n)].y;
    }
    static C v[T][P / T];
    for (int t = 0; t < T; ++t) mixfft_A<P, T, INV>(s.data(), tw.data(), t, v[t]);
    for (int t = 0; t < T; ++t) mixfft_A_store<P, T>(s.data(), t, v[t]);
    static C u[T][MixFft<P, T>::PER][T];
    for (int t = 0; t < T; ++t) mixfft_B<P, T, INV>(s.data(), tw.data(), t, u[t]);
    for (int t = 0; t < T; ++t) mixfft_B_store<P, T>(s.data(), t, u[t]);
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
        {"P80 T4 fwd f64", check<80, 4, false, cd>(1), 1e-14},   {"P80 T4 inv f64", check<80, 4, true, cd>(2), 1e-14},
        {"P96 T4 fwd f64", check<96, 4, false, cd>(3), 1e-14},   {"P144 T4 fwd f64", check<144, 4, false, cd>(4), 1e-14},
        {"P160 T4 inv f64", check<160, 4, true, cd>(5), 1e-14},  {"P192 T8 fwd f64", check<192, 8, false, cd>(6), 1e-14},
        {"P192 T8 inv f64", check<192, 8, true, cd>(7), 1e-14},  {"P240 T4 fwd f64", check<240, 4, false, cd>(8), 1e-14},
        {"P320 T8 inv f64", check<320, 8, true, cd>(9), 1e-14},  {"P64 T8 fwd f64", check<64, 8, false, cd>(10), 1e-14},
        {"P80 T4 fwd f32", check<80, 4, false, cf>(11), 1e-6},   {"P144 T4 inv f32", check<144, 4, true, cf>(12), 1e-6},
        {"P192 T8 fwd f32", check<192, 8, false, cf>(13), 1e-6},
    };
    for (auto &x : r) {
        std::printf("%s %.3e\n", x.name, x.e);
        if (!(x.e < x.bound)) bad = 1;
    }
    return bad;
}
