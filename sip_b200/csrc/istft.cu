// Overlap-add phase of the inverse STFT.
//
// The reference builds it from generic operators after its inverse C2C step
// (core/fft/fftcore/fft_core_istft_any.cpp:292-378: scale by 1/n_fft,
// multiply every frame by the window, UnfoldGrad overlap-add, the same
// overlap-add of window^2 as the envelope, divide, slice the centre).  Here
// one kernel produces each output sample directly: it sums the frames that
// cover it, weighted by the window, and divides by the window envelope at
// that sample; the centre slice is only an offset.  The frames come from the
// preceding C2C step in [channel][frame][n_fft] order, so consecutive output
// samples read consecutive frame elements.
#include "sipfft_internal.h"

namespace sipfft {

__global__ void istft_ola_kernel(const float2 *__restrict__ frames, const float *__restrict__ window,
                                 float2 *__restrict__ out, int64_t channel, int n_frames, int n_fft, int hop,
                                 int64_t out_len)
{
    const float inv_n = 1.0f / static_cast<float>(n_fft);
    const int64_t total = channel * out_len;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t c = i / out_len;
        const int64_t t = i - c * out_len + n_fft / 2;  // position in the uncropped signal
        const int64_t f_hi_t = t / hop;
        const int f_hi = static_cast<int>(f_hi_t < n_frames - 1 ? f_hi_t : n_frames - 1);
        const int f_lo = t >= n_fft ? static_cast<int>((t - n_fft) / hop + 1) : 0;
        float2 y = make_float2(0.f, 0.f);
        float env = 0.f;
        const float2 *fc = frames + c * int64_t(n_frames) * n_fft;
        for (int f = f_lo; f <= f_hi; f++) {
            const int e = static_cast<int>(t - int64_t(f) * hop);
            const float w = __ldg(window + e);
            const float2 v = fc[int64_t(f) * n_fft + e];
            y.x = fmaf(v.x, w, y.x);
            y.y = fmaf(v.y, w, y.y);
            env = fmaf(w, w, env);
        }
        out[i] = make_float2(y.x * inv_n / env, y.y * inv_n / env);
    }
}

cudaError_t launch_istft_ola(const float2 *frames, const float *window, float2 *out, int64_t channel, int n_frames,
                             int n_fft, int hop, int64_t out_len, cudaStream_t st)
{
    const int64_t total = channel * out_len;
    if (total <= 0) return cudaSuccess;
    const int64_t blocks = (total + 255) / 256;
    const int grid = static_cast<int>(blocks < int64_t(kB200Sms) * 32 ? blocks : int64_t(kB200Sms) * 32);
    istft_ola_kernel<<<grid, 256, 0, st>>>(frames, window, out, channel, n_frames, n_fft, hop, out_len);
    return cudaGetLastError();
}

}  // namespace sipfft
