// Register-resident DFT codelets and complex helpers for the sm_100a FFT kernels.
//
// Sign convention (the reference's, core/fft/fftcore/dft_core.cpp:88-97):
// FWD == true computes y[k] = sum_j a[j] * exp(-2*pi*i*j*k/R),
// FWD == false uses exp(+2*pi*i*j*k/R).  No scaling.
//
// Constants are evaluated at compile time in double from Taylor series
// (ccos/csin below) so no table or math-library call is needed in the
// butterflies; every codelet is fully unrolled into FMAs on registers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Codelets are host-callable as well so that a CPU test can check every radix
// against a direct DFT without a GPU.
#define SIPFFT_HD __host__ __device__ __forceinline__

namespace sipfft {

// ---------------------------------------------------------------- complex helpers
SIPFFT_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
SIPFFT_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
SIPFFT_HD float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
SIPFFT_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
SIPFFT_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (FWD quarter turn) or +i
template <bool FWD>
SIPFFT_HD float2 mul_quarter(float2 a)
{
    return FWD ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
// exp(sign * i * theta) with the direction's sign applied to a table entry
// that holds exp(-i * theta).
template <bool FWD>
SIPFFT_HD float2 dir(float2 w)
{
    return FWD ? w : make_float2(w.x, -w.y);
}

// ---------------------------------------------------------------- compile-time trig
constexpr double kPi = 3.141592653589793238462643383279502884;

constexpr double reduce_angle(double x)
{
    // bring x into [-pi, pi]
    while (x > kPi) x -= 2.0 * kPi;
    while (x < -kPi) x += 2.0 * kPi;
    return x;
}
constexpr double ccos(double x)
{
    x = reduce_angle(x);
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 30; k++) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}
constexpr double csin(double x)
{
    x = reduce_angle(x);
    double term = x, sum = x;
    for (int k = 1; k < 30; k++) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
// cos / sin of 2*pi*j/R
template <int R, int J>
struct Root {
    static constexpr float c = static_cast<float>(ccos(2.0 * kPi * (J % R) / R));
    static constexpr float s = static_cast<float>(csin(2.0 * kPi * (J % R) / R));
};

// multiply a by exp(-+ 2*pi*i*J/R) with the trivial angles special-cased
template <int R, int J, bool FWD>
SIPFFT_HD float2 rot(float2 a)
{
    constexpr int j = ((J % R) + R) % R;
    if constexpr (j == 0) {
        return a;
    } else if constexpr (4 * j == R) {
        return mul_quarter<FWD>(a);
    } else if constexpr (2 * j == R) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * j == 3 * R) {
        return mul_quarter<!FWD>(a);
    } else {
        constexpr float c = Root<R, j>::c;
        constexpr float s = FWD ? -Root<R, j>::s : Root<R, j>::s;  // exp(+-i theta) = c + i*s
        return make_float2(fmaf(a.x, c, -a.y * s), fmaf(a.x, s, a.y * c));
    }
}

// ---------------------------------------------------------------- power-of-two codelets
// Recursive radix-2 decimation in time on an array held in registers.
template <int R, bool FWD>
struct Pow2 {
    SIPFFT_HD static void run(float2 *a)
    {
        float2 e[R / 2], o[R / 2];
#pragma unroll
        for (int i = 0; i < R / 2; i++) {
            e[i] = a[2 * i];
            o[i] = a[2 * i + 1];
        }
        Pow2<R / 2, FWD>::run(e);
        Pow2<R / 2, FWD>::run(o);
        combine<0>(a, e, o);
    }
    template <int K>
    SIPFFT_HD static void combine(float2 *a, const float2 *e, const float2 *o)
    {
        if constexpr (K < R / 2) {
            float2 t = rot<R, K, FWD>(o[K]);
            a[K] = cadd(e[K], t);
            a[K + R / 2] = csub(e[K], t);
            combine<K + 1>(a, e, o);
        }
    }
};
template <bool FWD>
struct Pow2<1, FWD> {
    SIPFFT_HD static void run(float2 *) {}
};
template <bool FWD>
struct Pow2<2, FWD> {
    SIPFFT_HD static void run(float2 *a)
    {
        float2 t = a[1];
        a[1] = csub(a[0], t);
        a[0] = cadd(a[0], t);
    }
};
template <bool FWD>
struct Pow2<4, FWD> {
    SIPFFT_HD static void run(float2 *a)
    {
        float2 t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
        float2 t2 = cadd(a[1], a[3]), t3 = mul_quarter<FWD>(csub(a[1], a[3]));
        a[0] = cadd(t0, t2);
        a[2] = csub(t0, t2);
        a[1] = cadd(t1, t3);
        a[3] = csub(t1, t3);
    }
};

// ---------------------------------------------------------------- odd codelets
// Generic odd-length DFT using the conjugate-pair symmetry:
// for m = 1..H: y[m], y[R-m] = B_m -+ i*D_m with
// B_m = a0 + sum_k cos(2 pi k m / R) (a_k + a_{R-k}),
// D_m = sum_k sin(2 pi k m / R) (a_k - a_{R-k}).
template <int R, bool FWD>
struct Odd {
    static constexpr int H = (R - 1) / 2;
    SIPFFT_HD static void run(float2 *a)
    {
        float2 tp[H], tm[H];
#pragma unroll
        for (int k = 1; k <= H; k++) {
            tp[k - 1] = cadd(a[k], a[R - k]);
            tm[k - 1] = csub(a[k], a[R - k]);
        }
        float2 y0 = a[0];
#pragma unroll
        for (int k = 0; k < H; k++) y0 = cadd(y0, tp[k]);
        float2 out[R];
        out[0] = y0;
        terms<1>(a[0], tp, tm, out);
#pragma unroll
        for (int i = 0; i < R; i++) a[i] = out[i];
    }
    template <int M>
    SIPFFT_HD static void terms(float2 a0, const float2 *tp, const float2 *tm, float2 *out)
    {
        if constexpr (M <= H) {
            float2 b = a0, d = make_float2(0.f, 0.f);
            accum<M, 1>(b, d, tp, tm);
            // forward: y_M = b - i d ; y_{R-M} = b + i d
            float2 id = make_float2(-d.y, d.x);  // i*d
            if constexpr (FWD) {
                out[M] = csub(b, id);
                out[R - M] = cadd(b, id);
            } else {
                out[M] = cadd(b, id);
                out[R - M] = csub(b, id);
            }
            terms<M + 1>(a0, tp, tm, out);
        }
    }
    template <int M, int K>
    SIPFFT_HD static void accum(float2 &b, float2 &d, const float2 *tp, const float2 *tm)
    {
        if constexpr (K <= H) {
            constexpr float c = Root<R, (K * M) % R>::c;
            constexpr float s = Root<R, (K * M) % R>::s;
            b.x = fmaf(c, tp[K - 1].x, b.x);
            b.y = fmaf(c, tp[K - 1].y, b.y);
            d.x = fmaf(s, tm[K - 1].x, d.x);
            d.y = fmaf(s, tm[K - 1].y, d.y);
            accum<M, K + 1>(b, d, tp, tm);
        }
    }
};

template <bool FWD>
struct Odd<3, FWD> {
    SIPFFT_HD static void run(float2 *a)
    {
        constexpr float h = 0.86602540378443864676f;  // sqrt(3)/2
        float2 s = cadd(a[1], a[2]);
        float2 d = csub(a[1], a[2]);
        float2 y0 = cadd(a[0], s);
        float2 m = make_float2(fmaf(-0.5f, s.x, a[0].x), fmaf(-0.5f, s.y, a[0].y));
        // forward: y1 = m - i h d, y2 = m + i h d
        float2 ihd = make_float2(-h * d.y, h * d.x);
        a[0] = y0;
        if (FWD) {
            a[1] = csub(m, ihd);
            a[2] = cadd(m, ihd);
        } else {
            a[1] = cadd(m, ihd);
            a[2] = csub(m, ihd);
        }
    }
};

// ---------------------------------------------------------------- dispatch
template <int R>
constexpr bool is_pow2() { return R > 0 && (R & (R - 1)) == 0; }

constexpr int smallest_prime_factor(int r)
{
    for (int p = 2; p * p <= r; p++)
        if (r % p == 0) return p;
    return r;
}
// split of a composite radix R = A * B used by Comp: the power-of-two part
// first for even R, else the smallest prime factor
constexpr int comp_first(int r)
{
    if (r % 2 == 0) {
        int a = 1;
        while (r % (2 * a) == 0) a *= 2;
        return a;
    }
    return smallest_prime_factor(r);
}

template <int R, bool FWD>
SIPFFT_HD void dft(float2 *a);

// Composite radix R = A*B in registers (Cooley-Tukey, decimation in time):
// B-point DFTs over the A interleaved sub-sequences, twiddles W_R^(n1*k2),
// then A-point DFTs; output index k = k2 + B*k1.
template <int A, int B, bool FWD>
struct Comp {
    static constexpr int R = A * B;
    SIPFFT_HD static void run(float2 *a)
    {
        float2 y[A][B];
#pragma unroll
        for (int n1 = 0; n1 < A; n1++) {
#pragma unroll
            for (int n2 = 0; n2 < B; n2++) y[n1][n2] = a[n1 + A * n2];
            dft<B, FWD>(y[n1]);
        }
        twiddle<1, 1>(y);
#pragma unroll
        for (int k2 = 0; k2 < B; k2++) {
            float2 z[A];
#pragma unroll
            for (int n1 = 0; n1 < A; n1++) z[n1] = y[n1][k2];
            dft<A, FWD>(z);
#pragma unroll
            for (int k1 = 0; k1 < A; k1++) a[k2 + B * k1] = z[k1];
        }
    }
    template <int N1, int K2>
    SIPFFT_HD static void twiddle(float2 (&y)[A][B])
    {
        if constexpr (N1 < A) {
            if constexpr (K2 < B) {
                y[N1][K2] = rot<R, N1 * K2, FWD>(y[N1][K2]);
                twiddle<N1, K2 + 1>(y);
            } else {
                twiddle<N1 + 1, 1>(y);
            }
        }
    }
};

template <int R, bool FWD>
SIPFFT_HD void dft(float2 *a)
{
    if constexpr (is_pow2<R>()) {
        Pow2<R, FWD>::run(a);
    } else if constexpr (R % 2 == 0 || (smallest_prime_factor(R) != R && R > 13)) {
        Comp<comp_first(R), R / comp_first(R), FWD>::run(a);
    } else {
        Odd<R, FWD>::run(a);
    }
}

}  // namespace sipfft
