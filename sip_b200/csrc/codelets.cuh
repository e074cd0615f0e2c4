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

namespace sipfft {

// ---------------------------------------------------------------- complex helpers
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (FWD quarter turn) or +i
template <bool FWD>
__device__ __forceinline__ float2 mul_quarter(float2 a)
{
    return FWD ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
// exp(sign * i * theta) with the direction's sign applied to a table entry
// that holds exp(-i * theta).
template <bool FWD>
__device__ __forceinline__ float2 dir(float2 w)
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
__device__ __forceinline__ float2 rot(float2 a)
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
    __device__ __forceinline__ static void run(float2 *a)
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
    __device__ __forceinline__ static void combine(float2 *a, const float2 *e, const float2 *o)
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
    __device__ __forceinline__ static void run(float2 *) {}
};
template <bool FWD>
struct Pow2<2, FWD> {
    __device__ __forceinline__ static void run(float2 *a)
    {
        float2 t = a[1];
        a[1] = csub(a[0], t);
        a[0] = cadd(a[0], t);
    }
};
template <bool FWD>
struct Pow2<4, FWD> {
    __device__ __forceinline__ static void run(float2 *a)
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
    __device__ __forceinline__ static void run(float2 *a)
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
    __device__ __forceinline__ static void terms(float2 a0, const float2 *tp, const float2 *tm, float2 *out)
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
    __device__ __forceinline__ static void accum(float2 &b, float2 &d, const float2 *tp, const float2 *tm)
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
    __device__ __forceinline__ static void run(float2 *a)
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

template <int R, bool FWD>
__device__ __forceinline__ void dft(float2 *a)
{
    if constexpr (is_pow2<R>()) {
        Pow2<R, FWD>::run(a);
    } else {
        static_assert(R % 2 == 1, "composite even radices are split into stages by the planner");
        Odd<R, FWD>::run(a);
    }
}

}  // namespace sipfft
