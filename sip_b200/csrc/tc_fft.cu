// Tensor-core (tcgen05) split-precision DFT-matrix stages.
//
// The reference runs its FFT cores as DFT-matrix GEMMs on the Ascend cube
// unit (ops/fft/c2c/fft_b/fft_b/kernel/fft_b.cce: two GEMM stages with a
// twiddle pass between them, FP32).  Here a transform of length n = N1 * N2
// (N1, N2 <= 64) runs as two real GEMMs on the 5th-generation tensor cores:
//
//   stage A  Y[k1][n2] = W_n^(k1 n2) * sum_n1 F_N1[k1][n1] X[n1 N2 + n2]
//   stage B  X[k1 + N1 k2] = sum_n2 F_N2[k2][n2] Y[k1][n2]
//
// Complex values are expanded to real 2x2 blocks (K = 2*N, M = 2*N padded to
// 128).  Operands are FP16 or BF16 split into hi + lo parts, and each GEMM is
// the three products hi*hi + hi*lo + lo*hi accumulated in FP32 in tensor
// memory (TMEM); the FP16 form scales every tile by a power of two so the
// operands stay inside the half-precision range.  The DFT matrices are built
// in FP64 on the GPU and then split (tc_matrix_kernel).
//
// One elected thread issues tcgen05.mma with shared-memory descriptors
// (K-major, no swizzle: 8x16-byte core matrices); tcgen05.commit arrives on an
// mbarrier that every thread waits on with a bounded poll; the accumulator is
// read back with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = output rows).
// Each CTA owns 128 TMEM columns for its lifetime and frees them on exit,
// also on the error path.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "async_copy.cuh"
#include "tc_desc.cuh"
#include "tc_ptx.cuh"
#include "sipfft_internal.h"
#include "tile_io.cuh"

namespace sipfft {


namespace {

template <int FMT>
__device__ __forceinline__ uint16_t to_bits(float v)
{
    if constexpr (FMT == 0) return __half_as_ushort(__float2half_rn(v));
    else return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}
template <int FMT>
__device__ __forceinline__ float from_bits(uint16_t b)
{
    if constexpr (FMT == 0) return __half2float(__ushort_as_half(b));
    else return __bfloat162float(__ushort_as_bfloat16(b));
}

// hi/lo split of 8 consecutive K values into two 16-byte chunks
template <int FMT>
__device__ __forceinline__ void split8(const float *v, uint4 &hi, uint4 &lo)
{
    uint16_t h[8], l[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        h[i] = to_bits<FMT>(v[i]);
        l[i] = to_bits<FMT>(v[i] - from_bits<FMT>(h[i]));
    }
    hi = make_uint4(h[0] | (uint32_t(h[1]) << 16), h[2] | (uint32_t(h[3]) << 16), h[4] | (uint32_t(h[5]) << 16),
                    h[6] | (uint32_t(h[7]) << 16));
    lo = make_uint4(l[0] | (uint32_t(l[1]) << 16), l[2] | (uint32_t(l[3]) << 16), l[4] | (uint32_t(l[5]) << 16),
                    l[6] | (uint32_t(l[7]) << 16));
}

// power-of-two scale that brings max|v| near 2^14 (FP16 form); 1 for BF16
template <int FMT>
__device__ __forceinline__ float range_scale(float maxabs)
{
    if constexpr (FMT != 0) return 1.0f;
    if (!(maxabs > 0.0f) || !isfinite(maxabs)) return 1.0f;
    int e;
    frexpf(maxabs, &e);  // maxabs in [2^(e-1), 2^e)
    return ldexpf(1.0f, 14 - e);
}

__device__ __forceinline__ float block_max(float v, float *red)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    float m = red[0];
    for (int i = 1; i < (blockDim.x >> 5); i++) m = fmaxf(m, red[i]);
    __syncthreads();
    return m;
}

}  // namespace

// TC kernel parameters beside the tile descriptor
struct TcArgs {
    const uint16_t *a_hi;  // stage A matrix (128 x 2*N1), pre-laid-out in the operand layout
    const uint16_t *a_lo;
    const uint16_t *b_hi;  // stage B matrix (128 x 2*N2)
    const uint16_t *b_lo;
    const float2 *tw;  // W_n^m, m < n (inner twiddles between the stages)
    int *err;
};

template <int N1, int N2, int TB, int FMT, bool FWD>
struct TcShape {
    static constexpr int n = N1 * N2;
    static constexpr int KA = 2 * N1, KB = 2 * N2;
    static constexpr int CA = TB * N2, CB = TB * N1;  // GEMM N of the two stages
    static constexpr int M = 128;
    static constexpr int PITCH = ((n - 1) + ((n - 1) >> 4) + 1) | 1;
    static constexpr int A_BYTES = M * KA * 2, B_BYTES = M * KB * 2;
    static constexpr int U1 = (KA * CA * 2 * 2 > TB * n * 8) ? KA * CA * 2 * 2 : TB * n * 8;
    static constexpr int U2 = (TB * PITCH * 8 > KB * CB * 2 * 2) ? TB * PITCH * 8 : KB * CB * 2 * 2;
    // with N1 == N2 both stages use the same DFT matrix: one copy in shared
    // memory (16 KB less for 256 points, so four CTAs fit an SM)
    static constexpr bool SHARED_B = N1 == N2;
    static constexpr int OFF_AA = 128;
    static constexpr int OFF_AB = SHARED_B ? OFF_AA : OFF_AA + 2 * A_BYTES;
    static constexpr int OFF_U1 = OFF_AB + 2 * B_BYTES;
    static constexpr int OFF_U2 = OFF_U1 + ((U1 + 127) / 128) * 128;
    static constexpr int SMEM = OFF_U2 + ((U2 + 127) / 128) * 128;
    static_assert(CA % 16 == 0 && CA <= 256 && CB % 16 == 0 && CB <= 256, "GEMM N must be a multiple of 16 <= 256");
    static_assert(KA <= 128 && KB <= 128 && KA % 16 == 0 && KB % 16 == 0, "radices up to 64");
    static_assert(CA <= 128 && CB <= 128, "accumulator must fit the 128 allocated TMEM columns");
    static_assert(SMEM <= 227 * 1024, "shared memory");
};

// 256 points: at most 128 registers, so that four CTAs (shared memory 50 KB, TMEM 128 columns each) fit an SM
template <int N1, int N2, int TB, int FMT, bool FWD>
__global__ void __launch_bounds__(128, N1 * N2 <= 256 ? 4 : 1) tc_fft_kernel(const __grid_constant__ TileDesc d, TcArgs ta)
{
    using S = TcShape<N1, N2, TB, FMT, FWD>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + 8);
    float *red = reinterpret_cast<float *>(smem + 16);  // 4 floats
    unsigned char *aa = smem + S::OFF_AA;             // hi then lo
    unsigned char *ab = smem + S::OFF_AB;
    unsigned char *u1 = smem + S::OFF_U1;             // stage-A B operand (hi, lo) | Y
    unsigned char *u2 = smem + S::OFF_U2;             // X tile | stage-B B operand (hi, lo)
    float2 *xs = reinterpret_cast<float2 *>(u2);
    float *ys = reinterpret_cast<float *>(u1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // constant DFT matrices into shared memory (once per CTA)
    {
        const uint4 *src[4] = {reinterpret_cast<const uint4 *>(ta.a_hi), reinterpret_cast<const uint4 *>(ta.a_lo),
                               reinterpret_cast<const uint4 *>(ta.b_hi), reinterpret_cast<const uint4 *>(ta.b_lo)};
        uint4 *dst[4] = {reinterpret_cast<uint4 *>(aa), reinterpret_cast<uint4 *>(aa + S::A_BYTES),
                         reinterpret_cast<uint4 *>(ab), reinterpret_cast<uint4 *>(ab + S::B_BYTES)};
        const int cnt[4] = {S::A_BYTES / 16, S::A_BYTES / 16, S::B_BYTES / 16, S::B_BYTES / 16};
        for (int m = 0; m < (S::SHARED_B ? 2 : 4); m++)
            for (int i = tid; i < cnt[m]; i += blockDim.x) dst[m][i] = __ldg(src[m] + i);
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, 128);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    uint32_t phase = 0;
    bool ok = true;

    const uint32_t aa_addr = smem_u32(aa), ab_addr = smem_u32(ab), u1_addr = smem_u32(u1), u2_addr = smem_u32(u2);
    constexpr uint32_t idesc_a = umma_instr_desc(128, S::CA, FMT);
    constexpr uint32_t idesc_b = umma_instr_desc(128, S::CB, FMT);

    for (int64_t g = blockIdx.x; g < d.num_tiles; g += gridDim.x) {
        const int64_t o = g / d.tiles_per_outer;
        const int64_t c0 = (g % d.tiles_per_outer) * d.tb;
        const int64_t left = d.n_cols - c0;
        const int ntr = left < TB ? static_cast<int>(left) : TB;
        // absent transforms of a partial tile are zero, so they cannot disturb the scale
        for (int i = tid; i < (TB - ntr) * S::PITCH; i += blockDim.x) xs[ntr * S::PITCH + i] = make_float2(0.f, 0.f);
        load_tile<FWD>(d, d.in, xs, o, c0, ntr);
        __syncthreads();
        float s1 = 1.f;  // the BF16 form needs no scaling (no tile maximum)
        if constexpr (FMT == 0) {
            float mx = 0.f;
            for (int i = tid; i < TB * S::n; i += blockDim.x) {
                const float2 x = xs[(i / S::n) * S::PITCH + pad(i % S::n)];
                mx = fmaxf(mx, fmaxf(fabsf(x.x), fabsf(x.y)));
            }
            s1 = range_scale<FMT>(block_max(mx, red));
        }

        // ---- stage A operand: column j = (t, n2), K = (n1, re/im)
        for (int idx = tid; idx < S::CA * (S::KA / 8); idx += blockDim.x) {
            const int j = idx % S::CA, kg = idx / S::CA;
            const int t = j / N2, n2 = j % N2;
            float v[8];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float2 x = xs[t * S::PITCH + pad((kg * 4 + q) * N2 + n2)];
                v[2 * q] = x.x * s1;
                v[2 * q + 1] = x.y * s1;
            }
            uint4 hi, lo;
            split8<FMT>(v, hi, lo);
            const uint32_t off = umma_offset(j, kg * 8, S::KA);
            *reinterpret_cast<uint4 *>(u1 + off) = hi;
            *reinterpret_cast<uint4 *>(u1 + S::KA * S::CA * 2 + off) = lo;
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t bhi = u1_addr, blo = u1_addr + S::KA * S::CA * 2;
            const uint32_t ahi = aa_addr, alo = aa_addr + S::A_BYTES;
            const uint32_t pa[3] = {ahi, ahi, alo}, pb[3] = {bhi, blo, bhi};
#pragma unroll
            for (int p = 0; p < 3; p++)
#pragma unroll
                for (int kb = 0; kb < S::KA / 16; kb++)
                    tc_mma_f16(tmem, umma_smem_desc(pa[p] + kb * 256, 128, S::KA * 16),
                               umma_smem_desc(pb[p] + kb * 256, 128, S::KA * 16), idesc_a, (p | kb) ? 1u : 0u);
            tc_commit(bar);
        }
        ok = __syncthreads_and(mbar_wait_bounded(bar, phase) ? 1 : 0) != 0;
        phase ^= 1;
        if (!ok) {  // the tensor core did not answer: report and stop (block-uniform)
            if (tid == 0) atomicExch(ta.err, 3);
            break;
        }
        tc_fence_after();
        // ---- stage A result: row m = 2 k1 + c (warp w: lanes 32w..), twiddle, Y stored [t][n2][k1]
        float mx2 = 0.f;
        {
            const int m = warp * 32 + lane, k1 = m >> 1, c = m & 1;
            const float inv = 1.0f / s1;
            for (int c16 = 0; c16 < S::CA / 16; c16++) {
                float v[16];
                tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + c16 * 16, v);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const float own = v[i] * inv;
                    const float other = __shfl_xor_sync(0xffffffffu, own, 1);
                    const int j = c16 * 16 + i, t = j / N2, n2 = j % N2;
                    if (k1 < N1) {
                        const float2 y = c == 0 ? make_float2(own, other) : make_float2(other, own);
                        const float2 w = dir<FWD>(__ldg(ta.tw + k1 * n2));
                        const float2 z = cmul(y, w);
                        const float r = c == 0 ? z.x : z.y;
                        ys[((t * N2 + n2) * N1 + k1) * 2 + c] = r;
                        mx2 = fmaxf(mx2, fabsf(r));
                    }
                }
            }
        }
        tc_fence_before();
        __syncthreads();
        float s2 = 1.f;
        if constexpr (FMT == 0) s2 = range_scale<FMT>(block_max(mx2, red));
        // ---- stage B operand: column j' = (t, k1), K = (n2, re/im); written over the X tile
        for (int idx = tid; idx < S::CB * (S::KB / 8); idx += blockDim.x) {
            const int j = idx % S::CB, kg = idx / S::CB;
            const int t = j / N1, k1 = j % N1;
            float v[8];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int n2 = kg * 4 + q;
                v[2 * q] = ys[((t * N2 + n2) * N1 + k1) * 2] * s2;
                v[2 * q + 1] = ys[((t * N2 + n2) * N1 + k1) * 2 + 1] * s2;
            }
            uint4 hi, lo;
            split8<FMT>(v, hi, lo);
            const uint32_t off = umma_offset(j, kg * 8, S::KB);
            *reinterpret_cast<uint4 *>(u2 + off) = hi;
            *reinterpret_cast<uint4 *>(u2 + S::KB * S::CB * 2 + off) = lo;
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t bhi = u2_addr, blo = u2_addr + S::KB * S::CB * 2;
            const uint32_t ahi = ab_addr, alo = ab_addr + S::B_BYTES;
            const uint32_t pa[3] = {ahi, ahi, alo}, pb[3] = {bhi, blo, bhi};
#pragma unroll
            for (int p = 0; p < 3; p++)
#pragma unroll
                for (int kb = 0; kb < S::KB / 16; kb++)
                    tc_mma_f16(tmem, umma_smem_desc(pa[p] + kb * 256, 128, S::KB * 16),
                               umma_smem_desc(pb[p] + kb * 256, 128, S::KB * 16), idesc_b, (p | kb) ? 1u : 0u);
            tc_commit(bar);
        }
        ok = __syncthreads_and(mbar_wait_bounded(bar, phase) ? 1 : 0) != 0;
        phase ^= 1;
        if (!ok) {  // the tensor core did not answer: report and stop (block-uniform)
            if (tid == 0) atomicExch(ta.err, 3);
            break;
        }
        tc_fence_after();
        // ---- stage B result: row m = 2 k2 + c, column j' = (t, k1) -> X[t][k1 + N1 k2]
        {
            const int m = warp * 32 + lane, k2 = m >> 1, c = m & 1;
            const float inv = 1.0f / s2;
            float *xf = reinterpret_cast<float *>(xs);
            for (int c16 = 0; c16 < S::CB / 16; c16++) {
                float v[16];
                tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + c16 * 16, v);
                if (k2 < N2) {
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        const int j = c16 * 16 + i, t = j / N1, k1 = j % N1;
                        xf[(t * S::PITCH + pad(k1 + N1 * k2)) * 2 + c] = v[i] * inv;
                    }
                }
            }
        }
        tc_fence_before();
        __syncthreads();
        store_tile<FWD>(d, d.out, xs, o, c0, ntr);
        __syncthreads();
    }
    // all MMAs have completed (each was waited on) and every tcgen05.ld was waited on
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 128);
}

// Builds the 128 x 2N real DFT matrix of one stage, FP64, split into hi/lo
// parts in the K-major operand layout: row m = 2k + co, column 2n + ci,
// entries of exp(-+ 2 pi i k n / N) as [[c, -s], [s, c]]; rows >= 2N are zero.
template <int FMT>
__global__ void tc_matrix_kernel(uint16_t *hi, uint16_t *lo, int N, int fwd)
{
    const int K = 2 * N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 128 * K; i += gridDim.x * blockDim.x) {
        const int m = i / K, kk = i % K;
        double v = 0.0;
        if (m < 2 * N) {
            const int k = m >> 1, co = m & 1, n = kk >> 1, ci = kk & 1;
            double s, c;
            sincospi(2.0 * double((int64_t(k) * n) % N) / double(N), &s, &c);
            const double wi = fwd ? -s : s;  // exp(-+ i theta) = c + i wi
            v = co == 0 ? (ci == 0 ? c : -wi) : (ci == 0 ? wi : c);
        }
        const uint32_t off = umma_offset(m, kk, K) / 2;
        if (FMT == 0) {
            const __half h = __double2half(v);
            hi[off] = __half_as_ushort(h);
            lo[off] = __half_as_ushort(__double2half(v - double(__half2float(h))));
        } else {
            const __nv_bfloat16 h = __double2bfloat16(v);
            hi[off] = __bfloat16_as_ushort(h);
            lo[off] = __bfloat16_as_ushort(__double2bfloat16(v - double(__bfloat162float(h))));
        }
    }
}

// ------------------------------------------------------------------------------------ host side
namespace {

template <int N1, int N2, int TB, int FMT>
const void *tc_fn(bool fwd)
{
    return fwd ? reinterpret_cast<const void *>(tc_fft_kernel<N1, N2, TB, FMT, true>)
               : reinterpret_cast<const void *>(tc_fft_kernel<N1, N2, TB, FMT, false>);
}

}  // namespace

bool tc_config(int n, TcConfig &c)
{
    switch (n) {
        case 256: c = {16, 16, 8}; return true;
        case 1024: c = {32, 32, 4}; return true;
        case 2048: c = {64, 32, 2}; return true;
        case 4096: c = {64, 64, 1}; return true;
        default: return false;
    }
}

const void *tc_kernel(int n, int fmt, bool fwd, size_t *smem)
{
#define SIPFFT_TC(NN, A, B, T)                                                             \
    if (n == NN) {                                                                         \
        if (smem) *smem = fmt == 0 ? TcShape<A, B, T, 0, true>::SMEM : TcShape<A, B, T, 1, true>::SMEM; \
        return fmt == 0 ? tc_fn<A, B, T, 0>(fwd) : tc_fn<A, B, T, 1>(fwd);                \
    }
    SIPFFT_TC(256, 16, 16, 8)
    SIPFFT_TC(1024, 32, 32, 4)
    SIPFFT_TC(2048, 64, 32, 2)
    SIPFFT_TC(4096, 64, 64, 1)
#undef SIPFFT_TC
    return nullptr;
}

void tc_kernel_fns(std::vector<const void *> &out)
{
    for (int n : {256, 1024, 2048, 4096})
        for (int fmt = 0; fmt < 2; fmt++)
            for (int f = 0; f < 2; f++) out.push_back(tc_kernel(n, fmt, f != 0, nullptr));
}

cudaError_t fill_tc_matrix(uint16_t *hi, uint16_t *lo, int N, int fmt, bool fwd, cudaStream_t st)
{
    const int count = 128 * 2 * N;
    const int grid = (count + 255) / 256;
    if (fmt == 0)
        tc_matrix_kernel<0><<<grid, 256, 0, st>>>(hi, lo, N, fwd ? 1 : 0);
    else
        tc_matrix_kernel<1><<<grid, 256, 0, st>>>(hi, lo, N, fwd ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_tc(const TileDesc &d, int n, int fmt, bool fwd, const uint16_t *const *mats, const float2 *tw,
                      int grid, int *err, cudaStream_t st)
{
    size_t smem = 0;
    const void *fn = tc_kernel(n, fmt, fwd, &smem);
    if (!fn || grid <= 0) return cudaErrorInvalidConfiguration;
    TileDesc dd = d;
    TcArgs ta{mats[0], mats[1], mats[2], mats[3], tw, err};
    void *args[] = {&dd, &ta};
    return cudaLaunchKernel(fn, dim3(grid), dim3(128), args, smem, st);
}

}  // namespace sipfft
