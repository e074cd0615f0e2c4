// Stand-alone R2C post-twiddle and C2R pre-twiddle kernels, and the
// element-wise Bluestein stages.  They are used only by transforms too long
// for one CTA (the fused single-CTA kernels
// do the same arithmetic inside fft_tile.cu).  The maths follows the
// reference's even-length path (core/fft/fftcore/include/fftcore/fft_r2c_core.h:21-24,
// A/B tables in fft_core_common_func.cpp:569-673), written as the split
// X[k] = E[k] + w^k O[k] with E, O recovered from the packed spectrum Z.
#include <algorithm>

#include "async_copy.cuh"
#include "codelets.cuh"
#include "sipfft_internal.h"

namespace sipfft {

template <bool FWD>
__device__ __forceinline__ float2 tw2(const float2 *lo, const float2 *hi, int log2l, int64_t m)
{
    const int64_t mask = (int64_t(1) << log2l) - 1;
    return dir<FWD>(cmul(__ldg(lo + (m & mask)), __ldg(hi + (m >> log2l))));
}

// Z: [rows][m] packed spectrum of z[j] = x[2j] + i x[2j+1]; X: [rows][m+1]
template <bool FWD>
__global__ void r2c_post_kernel(const float2 *__restrict__ z, float2 *__restrict__ x, int64_t m, int64_t zdist,
                                int64_t xdist, const float2 *lo, const float2 *hi, int log2l)
{
    const int64_t row = blockIdx.y;
    const float2 *zr = z + row * zdist;
    float2 *xr = x + row * xdist;
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; 2 * k <= m;
         k += int64_t(gridDim.x) * blockDim.x) {
        const float2 zk = zr[k];
        const float2 zm = cconj(zr[k == 0 ? 0 : m - k]);
        const float2 e = cscale(cadd(zk, zm), 0.5f);
        const float2 t = csub(zk, zm);
        const float2 od = make_float2(0.5f * t.y, -0.5f * t.x);
        const float2 wo = cmul(tw2<FWD>(lo, hi, log2l, k), od);
        xr[k] = cadd(e, wo);
        if (2 * k != m) xr[m - k] = cconj(csub(e, wo));
    }
}

// X: [rows][m+1] half spectrum; Z: [rows][m] packed input of the m-point FFT
template <bool FWD>
__global__ void c2r_pre_kernel(const float2 *__restrict__ x, float2 *__restrict__ z, int64_t m, int64_t xdist,
                               int64_t zdist, const float2 *lo, const float2 *hi, int log2l)
{
    const int64_t row = blockIdx.y;
    const float2 *xr = x + row * xdist;
    float2 *zr = z + row * zdist;
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; 2 * k <= m;
         k += int64_t(gridDim.x) * blockDim.x) {
        float2 xk = xr[k];
        float2 xm = xr[m - k];
        if (k == 0) {
            xk.y = 0.f;
            xm.y = 0.f;
        }
        const float2 e = cadd(xk, cconj(xm));
        const float2 od = cmul(csub(xk, cconj(xm)), tw2<FWD>(lo, hi, log2l, k));
        zr[k] = make_float2(e.x - od.y, e.y + od.x);
        if (k != 0 && 2 * k != m) zr[m - k] = make_float2(e.x + od.y, -e.y + od.x);
    }
}

// ------------------------------------------------------------------------------------ Bluestein, multi-pass
// The element-wise stages of a Bluestein (chirp-z) transform whose
// convolution length m is too long for one CTA; the single-CTA form fuses the
// same arithmetic into the load / store phases of its FFT tiles (tile_io.cuh,
// IO_BLUE_PRE / IO_BLUE_POST).  One CTA row of the grid per transform row.
//   pre:  a[e] = x[e] chirp[e] for e < n, 0 for n <= e < m
//   mul:  b[e] *= bmul[e]  (bmul = FFT_m(conj chirp) / m, prepared by the planner)
//   post: y[k] = chirp[k] a[k]
template <int KIND>
__global__ void blue_pre_kernel(const void *__restrict__ in, float2 *__restrict__ a, int64_t n, int64_t m,
                                int64_t in_dist, const float2 *__restrict__ chirp)
{
    const int64_t row = blockIdx.y;
    float2 *ar = a + row * m;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < m; e += int64_t(gridDim.x) * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (e < n) {
            if (KIND == 1) {
                v = make_float2(static_cast<const float *>(in)[row * in_dist + e], 0.f);
            } else if (KIND == 2) {
                // Hermitian extension of the half spectrum (imaginary parts of bins 0 and n/2 ignored)
                const float2 *x = static_cast<const float2 *>(in) + row * in_dist;
                if (2 * e <= n) {
                    v = x[e];
                    if (e == 0 || 2 * e == n) v.y = 0.f;
                } else {
                    v = cconj(x[n - e]);
                }
            } else {
                v = static_cast<const float2 *>(in)[row * in_dist + e];
            }
            v = cmul(v, __ldg(chirp + e));
        }
        ar[e] = v;
    }
}

__global__ void point_mul_kernel(float2 *__restrict__ b, const float2 *__restrict__ bmul, int64_t m)
{
    float2 *br = b + int64_t(blockIdx.y) * m;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < m; e += int64_t(gridDim.x) * blockDim.x)
        br[e] = cmul(br[e], __ldg(bmul + e));
}

template <int KIND>
__global__ void blue_post_kernel(const float2 *__restrict__ a, void *__restrict__ out, int64_t n, int64_t m,
                                 int64_t out_dist, const float2 *__restrict__ chirp)
{
    const int64_t row = blockIdx.y;
    const float2 *ar = a + row * m;
    const int64_t count = KIND == 1 ? n / 2 + 1 : n;
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < count;
         k += int64_t(gridDim.x) * blockDim.x) {
        const float2 v = cmul(ar[k], __ldg(chirp + k));
        if (KIND == 2)
            static_cast<float *>(out)[row * out_dist + k] = v.x;
        else
            static_cast<float2 *>(out)[row * out_dist + k] = v;
    }
}

namespace {
dim3 aux_grid(int64_t rows, int64_t m)
{
    const int64_t pairs = m / 2 + 1;
    int64_t gx = (pairs + 255) / 256;
    if (gx > 1024) gx = 1024;
    return dim3(static_cast<unsigned>(gx), static_cast<unsigned>(rows), 1);
}
}  // namespace

cudaError_t launch_r2c_post(const float2 *z, float2 *x, int64_t rows, int64_t m, int64_t zdist, int64_t xdist,
                            const float2 *lo, const float2 *hi, int log2l, bool forward, cudaStream_t st)
{
    for (int64_t r0 = 0; r0 < rows; r0 += 65535) {
        const int64_t nr = rows - r0 < 65535 ? rows - r0 : 65535;
        const dim3 g = aux_grid(nr, m);
        if (forward)
            r2c_post_kernel<true><<<g, 256, 0, st>>>(z + r0 * zdist, x + r0 * xdist, m, zdist, xdist, lo, hi, log2l);
        else
            r2c_post_kernel<false><<<g, 256, 0, st>>>(z + r0 * zdist, x + r0 * xdist, m, zdist, xdist, lo, hi, log2l);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_c2r_pre(const float2 *x, float2 *z, int64_t rows, int64_t m, int64_t xdist, int64_t zdist,
                           const float2 *lo, const float2 *hi, int log2l, bool forward, cudaStream_t st)
{
    for (int64_t r0 = 0; r0 < rows; r0 += 65535) {
        const int64_t nr = rows - r0 < 65535 ? rows - r0 : 65535;
        const dim3 g = aux_grid(nr, m);
        if (forward)
            c2r_pre_kernel<true><<<g, 256, 0, st>>>(x + r0 * xdist, z + r0 * zdist, m, xdist, zdist, lo, hi, log2l);
        else
            c2r_pre_kernel<false><<<g, 256, 0, st>>>(x + r0 * xdist, z + r0 * zdist, m, xdist, zdist, lo, hi, log2l);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

namespace {
dim3 elem_grid(int64_t rows, int64_t count)
{
    int64_t gx = (count + 255) / 256;
    if (gx > 2048) gx = 2048;
    return dim3(static_cast<unsigned>(gx), static_cast<unsigned>(rows), 1);
}
}  // namespace

cudaError_t launch_blue_pre(const void *in, float2 *a, int64_t rows, int64_t n, int64_t m, int64_t in_dist, int kind,
                            const float2 *chirp, cudaStream_t st)
{
    const size_t esz = kind == 1 ? sizeof(float) : sizeof(float2);
    for (int64_t r0 = 0; r0 < rows; r0 += 65535) {
        const int64_t nr = rows - r0 < 65535 ? rows - r0 : 65535;
        const void *src = static_cast<const char *>(in) + r0 * in_dist * esz;
        float2 *dst = a + r0 * m;
        const dim3 g = elem_grid(nr, m);
        if (kind == 1)
            blue_pre_kernel<1><<<g, 256, 0, st>>>(src, dst, n, m, in_dist, chirp);
        else if (kind == 2)
            blue_pre_kernel<2><<<g, 256, 0, st>>>(src, dst, n, m, in_dist, chirp);
        else
            blue_pre_kernel<0><<<g, 256, 0, st>>>(src, dst, n, m, in_dist, chirp);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_point_mul(float2 *b, const float2 *bmul, int64_t rows, int64_t m, cudaStream_t st)
{
    for (int64_t r0 = 0; r0 < rows; r0 += 65535) {
        const int64_t nr = rows - r0 < 65535 ? rows - r0 : 65535;
        point_mul_kernel<<<elem_grid(nr, m), 256, 0, st>>>(b + r0 * m, bmul, m);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_blue_post(const float2 *a, void *out, int64_t rows, int64_t n, int64_t m, int64_t out_dist,
                             int kind, const float2 *chirp, cudaStream_t st)
{
    const size_t esz = kind == 2 ? sizeof(float) : sizeof(float2);
    for (int64_t r0 = 0; r0 < rows; r0 += 65535) {
        const int64_t nr = rows - r0 < 65535 ? rows - r0 : 65535;
        const float2 *src = a + r0 * m;
        void *dst = static_cast<char *>(out) + r0 * out_dist * esz;
        const dim3 g = elem_grid(nr, n);
        if (kind == 1)
            blue_post_kernel<1><<<g, 256, 0, st>>>(src, dst, n, m, out_dist, chirp);
        else if (kind == 2)
            blue_post_kernel<2><<<g, 256, 0, st>>>(src, dst, n, m, out_dist, chirp);
        else
            blue_post_kernel<0><<<g, 256, 0, st>>>(src, dst, n, m, out_dist, chirp);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ------------------------------------------------------------------------------------ transpose
// Out-of-place transpose of a batch of complex matrices through 32 x 32 tiles
// in shared memory: a warp reads 32 consecutive elements of one row (256
// bytes) and writes 32 consecutive elements of one output row.  The padded
// tile row (33 elements) keeps the column reads at two wavefronts per warp.
// Persistent grid; each CTA walks tiles (matrix, tile row, tile column).
__global__ void __launch_bounds__(256) transpose_kernel(const float2 *__restrict__ in, float2 *__restrict__ out,
                                                        int64_t rows, int64_t cols, int64_t tiles_r, int64_t tiles_c,
                                                        int64_t ntiles)
{
    __shared__ float2 t[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int64_t per = tiles_r * tiles_c;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t b = tile / per, rem = tile - b * per;
        const int64_t r0 = (rem / tiles_c) * 32, c0 = (rem % tiles_c) * 32;
        const float2 *src = in + b * rows * cols;
        float2 *dst = out + b * rows * cols;
#pragma unroll
        for (int i = ty; i < 32; i += 8) {
            const int64_t r = r0 + i, c = c0 + tx;
            if (r < rows && c < cols) t[i][tx] = src[r * cols + c];
        }
        __syncthreads();
#pragma unroll
        for (int i = ty; i < 32; i += 8) {
            const int64_t c = c0 + i, r = r0 + tx;
            if (c < cols && r < rows) st_stream(dst + c * rows + r, t[tx][i]);
        }
        __syncthreads();
    }
}

cudaError_t launch_transpose(const float2 *in, float2 *out, int64_t batch, int64_t rows, int64_t cols, int device,
                             cudaStream_t st)
{
    if (batch <= 0 || rows <= 0 || cols <= 0 || in == out) return cudaErrorInvalidValue;
    const int64_t tiles_r = (rows + 31) / 32, tiles_c = (cols + 31) / 32;
    const int64_t ntiles = batch * tiles_r * tiles_c;
    const int64_t grid = std::min<int64_t>(ntiles, int64_t(sm_count(device)) * 8);
    transpose_kernel<<<static_cast<int>(grid), 256, 0, st>>>(in, out, rows, cols, tiles_r, tiles_c, ntiles);
    return cudaGetLastError();
}

}  // namespace sipfft
