/*
 * Test infrastructure only — the CPU oracle, never part of the shipped path.
 *
 * Direct O(N^2) DFT in long double that restates the reference's FFT
 * semantics for all three transform types:
 *   - the exponent sign is set by the direction for C2C, R2C and C2R alike:
 *     FORWARD = exp(-2*pi*i*j*k/N), INVERSE = exp(+2*pi*i*j*k/N)
 *     (core/fft/fftcore/dft_core.cpp:88-97, dft_r2c_core.cpp:98-104,
 *      dft_c2r_core.cpp:98-110, core/fft/utils/rotate.cpp:80-111);
 *   - no normalisation in either direction (no 1/N anywhere on the path);
 *   - R2C returns bins 0..N/2 (N/2+1 complex values);
 *   - C2R reads N/2+1 bins and uses the Hermitian extension
 *     X[N-k] = conj(X[k]); the imaginary parts of bin 0 and, for even N,
 *     of bin N/2 do not contribute (their matrix rows are sin(0) and sin(pi)
 *     in dft_c2r_core.cpp:98-110);
 *   - angle indices are reduced mod N before the table lookup
 *     (dft_core.cpp:90-96).
 * Inputs are float (what the device path consumes), outputs double.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

static long double *twiddle_table(int64_t n, int forward)
{
    long double *t = (long double *)malloc(sizeof(long double) * 2 * (size_t)n);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    const long double sign = forward ? -1.0L : 1.0L;
    for (int64_t m = 0; m < n; m++) {
        long double a = two_pi * (long double)m / (long double)n;
        t[2 * m] = cosl(a);
        t[2 * m + 1] = sign * sinl(a);
    }
    return t;
}

/* in/out: [batch][n] interleaved complex. */
int oracle_dft_c2c(int forward, int64_t n, int64_t batch, const float *in, double *out)
{
    long double *t = twiddle_table(n, forward);
    if (!t) return -1;
    for (int64_t b = 0; b < batch; b++) {
        const float *x = in + 2 * n * b;
        double *y = out + 2 * n * b;
        for (int64_t k = 0; k < n; k++) {
            long double re = 0.0L, im = 0.0L;
            int64_t idx = 0;
            for (int64_t j = 0; j < n; j++) {
                const long double c = t[2 * idx], s = t[2 * idx + 1];
                re += (long double)x[2 * j] * c - (long double)x[2 * j + 1] * s;
                im += (long double)x[2 * j] * s + (long double)x[2 * j + 1] * c;
                idx += k;
                if (idx >= n) idx -= n;
            }
            y[2 * k] = (double)re;
            y[2 * k + 1] = (double)im;
        }
    }
    free(t);
    return 0;
}

/* in: [batch][n] real; out: [batch][n/2+1] interleaved complex. */
int oracle_dft_r2c(int forward, int64_t n, int64_t batch, const float *in, double *out)
{
    long double *t = twiddle_table(n, forward);
    if (!t) return -1;
    const int64_t half = n / 2 + 1;
    for (int64_t b = 0; b < batch; b++) {
        const float *x = in + n * b;
        double *y = out + 2 * half * b;
        for (int64_t k = 0; k < half; k++) {
            long double re = 0.0L, im = 0.0L;
            int64_t idx = 0;
            for (int64_t j = 0; j < n; j++) {
                re += (long double)x[j] * t[2 * idx];
                im += (long double)x[j] * t[2 * idx + 1];
                idx += k;
                if (idx >= n) idx -= n;
            }
            y[2 * k] = (double)re;
            y[2 * k + 1] = (double)im;
        }
    }
    free(t);
    return 0;
}

/* in: [batch][n/2+1] interleaved complex; out: [batch][n] real. */
int oracle_dft_c2r(int forward, int64_t n, int64_t batch, const float *in, double *out)
{
    long double *t = twiddle_table(n, forward);
    if (!t) return -1;
    const int64_t half = n / 2 + 1;
    long double *xr = (long double *)malloc(sizeof(long double) * (size_t)n);
    long double *xi = (long double *)malloc(sizeof(long double) * (size_t)n);
    if (!xr || !xi) {
        free(t);
        free(xr);
        free(xi);
        return -1;
    }
    for (int64_t b = 0; b < batch; b++) {
        const float *x = in + 2 * half * b;
        double *y = out + n * b;
        for (int64_t k = 0; k < n; k++) {
            if (k < half) {
                xr[k] = x[2 * k];
                xi[k] = x[2 * k + 1];
            } else {
                xr[k] = x[2 * (n - k)];
                xi[k] = -(long double)x[2 * (n - k) + 1];
            }
        }
        xi[0] = 0.0L;
        if (n % 2 == 0) xi[n / 2] = 0.0L;
        for (int64_t j = 0; j < n; j++) {
            long double acc = 0.0L;
            int64_t idx = 0;
            for (int64_t k = 0; k < n; k++) {
                acc += xr[k] * t[2 * idx] - xi[k] * t[2 * idx + 1];
                idx += j;
                if (idx >= n) idx -= n;
            }
            y[j] = (double)acc;
        }
    }
    free(xr);
    free(xi);
    free(t);
    return 0;
}
