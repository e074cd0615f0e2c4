// Kernel-side description of one FFT launch ("tile kernel").
//
// Every device step of a plan is one launch of the tile kernel: a CTA loads a
// tile of `tb` transforms (or of `tb` columns of one Stockham pass) from HBM
// into shared memory, runs a mixed-radix Stockham FFT of length `n` on each
// row held in shared memory (register codelets, one barrier pair per stage),
// and stores the tile back.  Pre/post-processing that the reference runs as
// separate GM passes (R2C/C2R pack twiddles: core/fft/fftcore/fft_r2c_core.cpp,
// fft_c2r_core.cpp; inter-stage twiddles of the large-N cores:
// fft_core_n.cpp, fft_core_mix_base.cpp) and the axis transposes of the
// multi-dimensional plans (fftoperation/transpose.cpp) are folded into the
// load and store phases of this kernel.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace sipfft {

constexpr int kMaxStages = 16;
// Largest radix of the compact runtime-radix engines (compiled without the
// radix 11-16 codelets so that they fit three CTAs per SM; a plan for them
// splits 16 = 4 x 4 and 12 = 4 x 3, and lengths with a factor 11 or 13 use the
// engines with every radix).
constexpr int kCompactMaxRadix = 10;

enum IoKind : int {
    IO_C2C = 0,         // complex in, complex out
    IO_R2C_PACKED = 1,  // even real length 2n read as n complex pairs; n-point FFT; post-twiddle to n+1 bins
    IO_C2R_PACKED = 2,  // n+1 bins; pre-twiddle to n complex; n-point FFT; written as 2n reals
    IO_R2C_FULL = 3,    // odd real length n, zero imaginary part; n-point FFT; bins 0..n/2
    IO_C2R_FULL = 4,    // bins 0..n/2 of odd n, Hermitian extension; n-point FFT; real part
    // Bluestein (chirp-z) for lengths with prime factors the codelets do not
    // cover: an N-point transform as a length-M circular convolution.
    IO_BLUE_PRE = 5,    // a[e] = x[e]*chirp[e] (e < N, else 0); M-point FFT; store A*Bmul
    IO_BLUE_POST = 6,   // M-point inverse FFT; store chirp[k]*y[k] for the first N (or N/2+1) outputs
};

// Address of element e of transform (outer o, column c):
//   o*dist + c*cstride + (cblock ? (c / cblock) * cjump : 0) + e*estride
// in units of the array's element type (float2 for complex and for packed
// real rows, float for the real side of the FULL kinds).
struct Addr {
    int64_t dist;
    int64_t cstride;
    int64_t estride;
    int64_t cblock;  // 0 = no block jump
    int64_t cjump;
};

// j mod ns with the precomputed reciprocal m = ceil(2^32 / ns) (ns > 1), j < 2^16
__host__ __device__ __forceinline__ int mod_ns(int j, int ns, uint32_t m)
{
#ifdef __CUDA_ARCH__
    return ns == 1 ? 0 : j - static_cast<int>(__umulhi(static_cast<uint32_t>(j), m)) * ns;
#else
    return ns == 1 ? 0 : static_cast<int>(j - ((uint64_t(uint32_t(j)) * m) >> 32) * ns);
#endif
}
__host__ __device__ constexpr uint32_t ns_reciprocal(int ns)
{
    return ns <= 1 ? 0u : static_cast<uint32_t>(((uint64_t(1) << 32) + uint64_t(ns) - 1) / uint64_t(ns));
}

struct TileDesc {
    const void *in;
    void *out;
    int n;          // FFT length held in shared memory (complex points)
    int io;         // IoKind
    int nstages;
    int radix[kMaxStages];
    int ns[kMaxStages];      // product of the radices of the earlier stages
    int tstep[kMaxStages];   // twiddle table index step: (n / (ns * radix)) * tw_mul
    // ceil(2^32 / ns) (0 when ns == 1): j mod ns = j - umulhi(j, ns_m) * ns,
    // exact for j < 2^16 and ns < 2^16 (every butterfly index of a tile)
    uint32_t ns_m[kMaxStages];
    int tb;         // transforms (columns) per tile
    int tpt;        // threads per transform
    int pitch;      // shared-memory floats2 per transform (padded)
    int xfast;      // thread mapping: 1 = transform index fastest (column tiles)
    int64_t n_outer;
    int64_t n_cols;
    int64_t tiles_per_outer;
    int64_t num_tiles;
    Addr in_a;
    Addr out_a;
    const float2 *tw;   // exp(-2 pi i m / (n * tw_mul)), m < n * tw_mul
    int tw_mul;
    // Input twiddle of a multi-pass Stockham pass over a length-F transform:
    // element r of column c is multiplied by W_F^(r * (c mod g_ns) * (F / (g_ns * n))),
    // read from a two-level table W_F^m = lo[m & (L-1)] * hi[m >> log2 L].
    int g_twiddle;
    int g_log2l;
    int64_t g_ns;
    int64_t g_step;    // F / (g_ns * n)
    // Tile column c belongs to Stockham column c / g_div (a strided axis
    // interleaves `inner` transforms per Stockham column); 0 or 1 = c itself.
    int64_t g_div;
    const float2 *g_lo;
    const float2 *g_hi;
    // Per-stage twiddle tables of the compile-time (static) kernels: stage s
    // occupies (R_s - 1) * Ns_s entries laid out [r-1][k], value
    // exp(-2 pi i r k / (Ns_s R_s)), so a warp's loads for one r are contiguous.
    const float2 *stw;
    // Bluestein: chirp[e] = exp(s*pi*i*(e^2 mod 2N)/N), bmul = FFT_M(conj chirp)/M,
    // blue_n = N, blue_kind: 0 complex, 1 real input (pre) / half spectrum
    // output (post), 2 Hermitian half-spectrum input (pre) / real output (post)
    const float2 *chirp;
    const float2 *bmul;
    int blue_n;
    int blue_kind;
    // Planar (separated) complex data: bit 0 = input, bit 1 = output.  The
    // real plane is in / out (float), the imaginary plane in_im / out_im,
    // both indexed like the interleaved layout's complex elements.
    int planar;
    const float *in_im;
    float *out_im;
    // Shared-memory buffers of a row kernel, each g_ns float2 (of a TMA column
    // kernel: each col_buf float2): 2 (double-buffered tiles; 0 reads as 2) or
    // 3 (plus a ping-pong work area).
    int row_bufs;
    // complex32 (FP16 real / imaginary pairs) user data of a C2C step: bit 0 =
    // the input, bit 1 = the output.  Loads widen to FP32, the stages run in
    // FP32, stores round to FP16 (round to nearest even).
    int half_io;
    // Shared-memory float2 count of one tile buffer of the TMA column kernel
    // (col_pipe.cu): >= tb * max(n, pitch), a multiple of 16 (128-byte aligned
    // buffers).
    int64_t col_buf;
};

// Stockham column of tile column c for the pass twiddle: (c / g_div) mod g_ns.
__host__ __device__ __forceinline__ int64_t pass_column(const TileDesc &d, int64_t c)
{
    return (d.g_div > 1 ? c / d.g_div : c) % d.g_ns;
}

// One segment of an uneven batch: a tile-kernel step whose source and
// destination are byte offsets into one of four buffers (user input, user
// output, workspace slot 0 / 1).
struct BatchSeg {
    TileDesc d;
    int64_t in_off;
    int64_t out_off;
    int in_buf;
    int out_buf;
    int dep;     // segment whose output this one reads, -1 if none
    int ntiles;
    int fwd;     // direction of this segment's FFT
};

struct BatchBufs {
    void *p[4];
};

}  // namespace sipfft
