// Host-side check of every register codelet against a direct DFT in double.
// Built and run by tests/test_codelets_host.py (nvcc, CPU only).
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "codelets.cuh"

using namespace sipfft;

template <int R, bool FWD>
double check()
{
    float2 a[R];
    double xr[R], xi[R];
    unsigned s = 12345u + R * 7u + (FWD ? 1u : 0u);
    for (int i = 0; i < R; i++) {
        s = s * 1664525u + 1013904223u;
        xr[i] = ((s >> 8) & 0xffff) / 32768.0 - 1.0;
        s = s * 1664525u + 1013904223u;
        xi[i] = ((s >> 8) & 0xffff) / 32768.0 - 1.0;
        a[i] = make_float2(static_cast<float>(xr[i]), static_cast<float>(xi[i]));
    }
    dft<R, FWD>(a);
    double err = 0, ref = 0;
    const double sign = FWD ? -1.0 : 1.0;
    for (int k = 0; k < R; k++) {
        double yr = 0, yi = 0;
        for (int j = 0; j < R; j++) {
            const double t = sign * 2.0 * M_PI * static_cast<double>((static_cast<long>(j) * k) % R) / R;
            yr += xr[j] * std::cos(t) - xi[j] * std::sin(t);
            yi += xr[j] * std::sin(t) + xi[j] * std::cos(t);
        }
        err += (a[k].x - yr) * (a[k].x - yr) + (a[k].y - yi) * (a[k].y - yi);
        ref += yr * yr + yi * yi;
    }
    return std::sqrt(err / ref);
}

template <int R>
int run()
{
    const double e1 = check<R, true>(), e2 = check<R, false>();
    const double bound = 4e-7 * std::log2(static_cast<double>(R) + 1.0);
    const bool ok = e1 < bound && e2 < bound;
    std::printf("radix %3d  fwd %.2e  inv %.2e  %s\n", R, e1, e2, ok ? "ok" : "FAIL");
    return ok ? 0 : 1;
}

int main()
{
    int bad = 0;
    bad += run<2>() + run<3>() + run<4>() + run<5>() + run<6>() + run<7>() + run<8>() + run<9>() + run<10>();
    bad += run<11>() + run<12>() + run<13>() + run<14>() + run<15>() + run<16>() + run<20>() + run<21>();
    bad += run<25>() + run<27>() + run<32>() + run<49>() + run<64>();
    std::printf("%s\n", bad ? "FAILED" : "ALL OK");
    return bad ? 1 : 0;
}
