// Test infrastructure only: the CPU checker built from the reference's own
// coefficient generator. Nothing in the shipped library links or calls this.
//
// The reference's FFT runs only on an Ascend NPU, but the matrices its
// generic core multiplies by are produced on the host by
// core/fft/utils/rotate.cpp:113-171 (rotate::OneRotateMatrix) on top of the
// wten CPU tensor library (core/utils/the_tensor.cpp, the_view.cpp,
// include/utils/operations.h).  oracle/Makefile compiles those reference
// sources unmodified, next to this driver, into oracle/_ref/libsipref.so.
// The driver applies the reference's matrices exactly as the reference's
// generic core sequences them, so its outputs carry the reference's sign,
// normalisation and packing rules:
//   * sipref_dense:       one factor (factors = {N}) — the whole transform is
//                         a single dense matrix, as in FFTCoreAny for prime N
//                         (core/fft/fftcore/fft_core_any.cpp:282-564).
//   * sipref_c2c_staged:  the multi-factor C2C stage chain of FFTCoreAny:
//                         permute, one batched matmul per merged factor,
//                         final digit permute (fft_core_any.cpp:395-500).
// C2R input mirroring follows fft_core_any.cpp:319-381: the half spectrum
// X[0..N/2] is extended with conj(X[N-k]) for k > N/2.
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <vector>
#include <cmath>
#include "utils/rotate.h"

namespace {

AsdSip::FftMode to_mode(int mode)
{
    switch (mode) {
        case 0: return AsdSip::FftMode::c2c;
        case 1: return AsdSip::FftMode::r2cOneside;
        default: return AsdSip::FftMode::c2r;
    }
}

// Restatement of Factorize + Merge (fft_core_any.cpp:64-143): prime factors
// in ascending order, merged greedily (largest first) into factors <= 32,
// at most 5 of them, and a factor >= 16 moved to the front.
std::vector<int64_t> merged_factors(int64_t n)
{
    const int64_t kFactorBound = 32, kNdimBound = 5, kFirstMin = 16;
    std::vector<int64_t> primes;
    int64_t m = n;
    int64_t bound = static_cast<int64_t>(std::sqrt(static_cast<double>(m)));
    for (int64_t f = 2; f <= bound;) {
        if (m % f == 0) {
            primes.push_back(f);
            m /= f;
            bound = static_cast<int64_t>(std::sqrt(static_cast<double>(m)));
        } else {
            f++;
        }
    }
    if (m != 1) primes.push_back(m);
    std::vector<int64_t> rev(primes.rbegin(), primes.rend());
    std::vector<bool> used(rev.size(), false);
    std::vector<int64_t> merged;
    for (size_t i = 0; i < rev.size(); i++) {
        int64_t f = 1;
        for (size_t j = i; j < rev.size(); j++) {
            if (used[j]) continue;
            if (f == 1 || rev[j] * f <= kFactorBound) {
                f *= rev[j];
                used[j] = true;
            }
        }
        if (f == 1) break;
        merged.push_back(f);
    }
    std::sort(merged.begin(), merged.end());
    if (static_cast<int64_t>(merged.size()) > kNdimBound) {
        std::vector<int64_t> top(merged.end() - kNdimBound, merged.end());
        for (size_t i = 0; i + kNdimBound < merged.size(); i++) {
            *std::min_element(top.begin(), top.end()) *= merged[i];
        }
        std::sort(top.begin(), top.end());
        merged = top;
    }
    if (merged.size() > 1 && merged[0] < kFirstMin) {
        for (size_t i = 1; i < merged.size(); i++) {
            if (merged[i] >= kFirstMin) {
                std::swap(merged[0], merged[i]);
                break;
            }
        }
    }
    return merged;
}

}  // namespace

extern "C" {

// Shape [prevN, rows, cols] of the reference matrix for one stage.
int sipref_rotate_dims(const int64_t *factors, int nf, int index, int mode, int64_t *dims3)
{
    std::vector<int64_t> f(factors, factors + nf);
    int64_t prevN = 1;
    for (int i = 0; i < index; i++) prevN *= f[i];
    auto [outN, outC, inN, inC] = rotate::computeOutShape(f, index, to_mode(mode));
    dims3[0] = prevN;
    dims3[1] = outN * outC;
    dims3[2] = inC * inN;
    return 0;
}

// Copies the reference's stage matrix (float, row-major [prevN, rows, cols]).
int sipref_rotate_matrix(const int64_t *factors, int nf, int index, int mode, int forward, float *out,
                         int64_t capacity)
{
    std::vector<int64_t> f(factors, factors + nf);
    wten::TheTensor<float> m = rotate::OneRotateMatrix(f, index, to_mode(mode), forward != 0);
    if (static_cast<int64_t>(m.size()) > capacity) return -1;
    std::memcpy(out, m.data(), m.size() * sizeof(float));
    return 0;
}

// Merged factor list of the reference's generic core for n (<= 8 entries).
int sipref_factors(int64_t n, int64_t *out8)
{
    std::vector<int64_t> f = merged_factors(n);
    for (size_t i = 0; i < f.size(); i++) out8[i] = f[i];
    return static_cast<int>(f.size());
}

// Single dense matrix transform of `batch` rows.
//   mode 0 (C2C): in [batch][n] complex64, out [batch][n] complex64
//   mode 1 (R2C): in [batch][n] float,     out [batch][n/2+1] complex64
//   mode 2 (C2R): in [batch][n/2+1] complex64, out [batch][n] float
// Accumulation is in double so that only the matrix rounding is visible.
int sipref_dense(int mode, int forward, int64_t n, int64_t batch, const float *in, float *out)
{
    std::vector<int64_t> f{n};
    wten::TheTensor<float> m = rotate::OneRotateMatrix(f, 0, to_mode(mode), forward != 0);
    const int64_t rows = m.shape()[1];
    const int64_t cols = m.shape()[2];
    const int64_t half = n / 2 + 1;
    std::vector<double> vec(cols);
    for (int64_t b = 0; b < batch; b++) {
        if (mode == 0) {
            const float *x = in + b * 2 * n;
            for (int64_t i = 0; i < n; i++) {
                vec[i] = x[2 * i];
                vec[n + i] = x[2 * i + 1];
            }
        } else if (mode == 1) {
            const float *x = in + b * n;
            for (int64_t i = 0; i < n; i++) vec[i] = x[i];
        } else {
            // Hermitian extension of the half spectrum (fft_core_any.cpp:319-381).
            const float *x = in + b * 2 * half;
            for (int64_t k = 0; k < n; k++) {
                if (k < half) {
                    vec[k] = x[2 * k];
                    vec[n + k] = x[2 * k + 1];
                } else {
                    vec[k] = x[2 * (n - k)];
                    vec[n + k] = -x[2 * (n - k) + 1];
                }
            }
        }
        float *y = (mode == 2) ? out + b * n : out + b * rows;
        for (int64_t r = 0; r < rows; r++) {
            const float *row = m.data() + r * cols;
            double acc = 0.0;
            for (int64_t c = 0; c < cols; c++) acc += static_cast<double>(row[c]) * vec[c];
            y[r] = static_cast<float>(acc);
        }
    }
    return 0;
}

// Multi-factor C2C stage chain of the reference's generic core.
// in/out: [batch][n] complex64 (interleaved float pairs).
int sipref_c2c_staged(int forward, int64_t n, int64_t batch, const float *in, float *out)
{
    std::vector<int64_t> f = merged_factors(n);
    const int s = static_cast<int>(f.size());
    const int64_t total = 2 * n * batch;
    // Initial permute [batch][n][2] -> [2][n][batch] (fft_core_any.cpp:383-392).
    std::vector<double> ping(total), pong(total);
    for (int64_t b = 0; b < batch; b++)
        for (int64_t i = 0; i < n; i++)
            for (int c = 0; c < 2; c++) ping[(c * n + i) * batch + b] = in[(b * n + i) * 2 + c];
    for (int idx = 0; idx < s; idx++) {
        wten::TheTensor<float> m = rotate::OneRotateMatrix(f, idx, AsdSip::FftMode::c2c, forward != 0);
        const int64_t P = m.shape()[0], R = m.shape()[1], K = m.shape()[2];
        const int64_t rest = total / (P * K);
        // out[p][r][j] = sum_k M[p][r][k] * in[p][k][j]
        for (int64_t p = 0; p < P; p++) {
            const float *mp = m.data() + p * R * K;
            for (int64_t r = 0; r < R; r++) {
                double *dst = pong.data() + (p * R + r) * rest;
                std::fill(dst, dst + rest, 0.0);
                for (int64_t k = 0; k < K; k++) {
                    const double w = mp[r * K + k];
                    const double *src = ping.data() + (p * K + k) * rest;
                    for (int64_t j = 0; j < rest; j++) dst[j] += w * src[j];
                }
            }
        }
        std::swap(ping, pong);
    }
    // View [f0, ..., f_{s-1}, 2, 1, batch] and permute to
    // [batch, 1, f_{s-1}, ..., f0, 2] (fft_core_any.cpp:455-500).
    std::vector<int64_t> digit(s);
    for (int64_t b = 0; b < batch; b++) {
        for (int64_t k = 0; k < n; k++) {
            // output index k = k_{s-1} * (f_{s-2}..f_0) + ... + k_0
            int64_t rem = k;
            for (int d = 0; d < s; d++) {
                digit[d] = rem % f[d];
                rem /= f[d];
            }
            int64_t src = 0;
            for (int d = 0; d < s; d++) src = src * f[d] + digit[d];
            for (int c = 0; c < 2; c++) {
                out[(b * n + k) * 2 + c] = static_cast<float>(ping[(src * 2 + c) * batch + b]);
            }
        }
    }
    return 0;
}

}  // extern "C"
