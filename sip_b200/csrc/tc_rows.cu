// Tensor-core split-precision FFT of contiguous C2C rows: a warp-specialised,
// persistent tcgen05 pipeline.
//
// Same four-step split as the reference's two-GEMM core
// (ops/fft/c2c/fft_b/fft_b/kernel/fft_b.cce; host side fftcore/fft_core_b.cpp),
// n = N1 * N2, input index n1 N2 + n2, output index k1 + N1 k2:
//
//   stage A  Z[t][n2][k1] = sum_n1 X[t][n1 N2 + n2] W_N1^(n1 k1)      (rows (t, n2))
//   twiddle  Y = Z * W_n^(k1 n2)
//   stage B  X[t][k1 + N1 k2] = sum_n2 Y[t][n2][k1] W_N2^(n2 k2)        (rows (t, k1))
//
// Each stage is one real GEMM D[rows][2 bins] = A[rows][K] * F[2 bins][K]^T:
// the data is the A operand (MN-major in shared memory, K = re block then im
// block), the DFT matrix the B operand (K-major, rows = (bin, re/im)), and
// the accumulator lives in tensor memory with one row per TMEM lane, so a
// thread owns one data row and reads its bins as consecutive columns.
// Operands are FP16 or BF16 hi + lo parts; every GEMM is hi*hi + hi*lo +
// lo*hi accumulated in FP32.  The FP16 form scales each tile by a power of
// two (from the tile's max |value|) before stage A and by 2^-(log2 N1 + 1)
// before stage B, which bounds |Y| by the stage-A range, so no operand can
// overflow; the BF16 form needs no scaling.
//
// Roles (544 threads, one CTA per SM, tiles of TB transforms round-robin):
//   warps 0-7   load the tile from HBM into registers (and prefetch the next
//               tile into L2), scale, split and store operand A1
//   warps 8-15  per tile: read the stage-A accumulators, twiddle, split and
//               store operand A2; then read the previous tile's stage-B
//               accumulators and store that result to HBM (two warps per
//               TMEM lane quarter, each with half of the columns)
//   warp 16     one thread issues the MMAs and commits them to mbarriers
// Accumulators are double-buffered in TMEM (D1[2], D2[2]); operands A1 and
// A2 are single buffers.  Every wait is a bounded mbarrier poll that also
// watches a CTA-wide abort flag, so a stalled tensor core ends the kernel
// with an error code instead of a hang; TMEM is freed on every path.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "async_copy.cuh"
#include "codelets.cuh"
#include "sipfft_internal.h"
#include "tc_desc.cuh"
#include "tc_ptx.cuh"

namespace sipfft {

template <int N1, int N2, int TB>
struct TcRowShape {
    static constexpr int n = N1 * N2;
    static constexpr int KA = 2 * N1, KB = 2 * N2;  // K (and N = 2 outputs per bin) of the stages
    static constexpr int RA = TB * N2, RB = TB * N1;  // operand rows of the stages
    static constexpr int CHA = RA / 128, CHB = RB / 128;
    static constexpr int DC = CHA * KA;  // TMEM columns of one accumulator
    static constexpr int TMEM_COLS = 4 * DC;
    // 8-row group strides, padded so the loader's and the epilogue's 4- and
    // 16-byte stores of consecutive groups start in different banks
    static constexpr uint32_t SBO_A = KA * 16 + 1024 / N2;
    static constexpr uint32_t SBO_B = KB * 16 + 1024 / N1;
    static constexpr int A1_CHUNK = 16 * SBO_A, A2_CHUNK = 16 * SBO_B;  // one 128-row chunk, one part
    static constexpr int FA = KA * KA * 2, FB = KB * KB * 2;             // DFT matrix, one part
    static constexpr int OFF_FA = 1024;
    static constexpr int OFF_FB = OFF_FA + 2 * FA;
    static constexpr int OFF_A1 = OFF_FB + (N1 == N2 ? 0 : 2 * FB);
    static constexpr int OFF_A2 = OFF_A1 + 2 * CHA * A1_CHUNK;
    static constexpr int SMEM = OFF_A2 + 2 * CHB * A2_CHUNK;
    static constexpr int THREADS = kTcRowThreads;
    static_assert(n % 512 == 0, "loader: 256 threads x element pairs per transform");
    static_assert(RA % 128 == 0 && RB % 128 == 0, "tile rows must fill 128-row MMA chunks");
    static_assert(CHA * KA == CHB * KB, "both accumulators have the same width");
    static_assert(DC == 64 || DC == 128, "accumulator width");
    static_assert(KA % 16 == 0 && KB % 16 == 0 && KA <= 256 && KB <= 256, "MMA N / K");
    static_assert(N2 >= 32 && N1 >= 32, "a warp's 32 rows belong to one transform");
    static_assert(SMEM <= 227 * 1024, "shared memory");
};

namespace {

// shared-memory header: barriers, TMEM address, abort flag, FP16 tile maxima and scales
struct TcHeader {
    uint64_t a1_full, a2_full, max_bar, pad0;
    uint64_t sa_done[2], sb_done[2], d1_empty[2], d2_empty[2];
    uint32_t tmem;
    int abort;
    uint32_t smax[4];
    float scale[16];
};

// Bounded mbarrier wait that also gives up when another role has aborted.
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity, TcHeader *h, int *err)
{
    for (uint32_t it = 0; it < kMbarPollLimit; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*reinterpret_cast<volatile int *>(&h->abort)) return false;
        if (it > 64) __nanosleep(64);
    }
    *reinterpret_cast<volatile int *>(&h->abort) = 1;
    atomicExch(err, 3);
    return false;
}

template <int FMT>
__device__ __forceinline__ uint32_t pack2(float a, float b)
{
    if constexpr (FMT == 0) {
        const __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<const uint32_t *>(&h);
    } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<const uint32_t *>(&h);
    }
}
template <int FMT>
__device__ __forceinline__ float2 unpack2(uint32_t u)
{
    if constexpr (FMT == 0) return __half22float2(*reinterpret_cast<const __half2 *>(&u));
    else return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u));
}
// hi = rn(a, b); lo = rn(a - hi.a, b - hi.b)
template <int FMT>
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    hi = pack2<FMT>(a, b);
    const float2 h = unpack2<FMT>(hi);
    lo = pack2<FMT>(a - h.x, b - h.y);
}

__device__ __forceinline__ float pow2_scale_for(float maxabs)
{
    if (!(maxabs > 0.0f) || !isfinite(maxabs)) return 1.0f;
    int e;
    frexpf(maxabs, &e);  // maxabs in [2^(e-1), 2^e)
    return ldexpf(1.0f, 14 - e);
}

template <int N>
constexpr int ilog2c()
{
    int l = 0;
    while ((1 << l) < N) l++;
    return l;
}

}  // namespace

struct TcRowArgs {
    const float2 *in;
    float2 *out;
    int64_t rows;      // transforms
    int64_t in_dist;   // complex elements between consecutive input rows
    int64_t out_dist;
    const uint16_t *fa;  // stage-A DFT matrix, hi then lo (2 * FA bytes)
    const uint16_t *fb;  // stage-B DFT matrix (unused when N1 == N2)
    const float2 *tw;    // W_n^m, m < n
    int *err;
    int aligned16;       // input base and row distance allow 16-byte loads
};

namespace {
// Streaming loads of the input (read once): no L1 allocation, so the
// twiddle table the stage-A epilogue reads stays in L1.
__device__ __forceinline__ float4 load_pair(const float2 *p, bool aligned16)
{
    float4 r;
    if (aligned16) {
        asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                     : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
                     : "l"(p));
    } else {
        asm volatile("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(r.x), "=f"(r.y) : "l"(p));
        asm volatile("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(r.z), "=f"(r.w) : "l"(p + 1));
    }
    return r;
}
}  // namespace

template <int N1, int N2, int TB, int FMT, bool FWD>
__global__ void __launch_bounds__(kTcRowThreads, 1) tc_rows_kernel(const __grid_constant__ TcRowArgs a)
{
    using S = TcRowShape<N1, N2, TB>;
    extern __shared__ __align__(1024) unsigned char smem[];
    TcHeader *h = reinterpret_cast<TcHeader *>(smem);
    unsigned char *fa = smem + S::OFF_FA;
    unsigned char *fb = N1 == N2 ? fa : smem + S::OFF_FB;
    unsigned char *a1 = smem + S::OFF_A1;  // hi chunks, then lo chunks
    unsigned char *a2 = smem + S::OFF_A2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t num_tiles = (a.rows + TB - 1) / TB;

    // ---- set-up: DFT matrices into shared memory, barriers, TMEM
    {
        const int na = 2 * S::FA / 16;
        const uint4 *src = reinterpret_cast<const uint4 *>(a.fa);
        for (int i = tid; i < na; i += blockDim.x) reinterpret_cast<uint4 *>(fa)[i] = __ldg(src + i);
        if (N1 != N2) {
            const int nb = 2 * S::FB / 16;
            const uint4 *srcb = reinterpret_cast<const uint4 *>(a.fb);
            for (int i = tid; i < nb; i += blockDim.x) reinterpret_cast<uint4 *>(fb)[i] = __ldg(srcb + i);
        }
    }
    if (tid == 0) {
        mbar_init(&h->a1_full, 256);
        mbar_init(&h->a2_full, 256);
        mbar_init(&h->max_bar, 256);
        for (int b = 0; b < 2; b++) {
            mbar_init(&h->sa_done[b], 1);
            mbar_init(&h->sb_done[b], 1);
            mbar_init(&h->d1_empty[b], 256);
            mbar_init(&h->d2_empty[b], 256);
        }
        h->abort = 0;
        for (int i = 0; i < 4; i++) h->smax[i] = 0;
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(&h->tmem, S::TMEM_COLS);
        tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = h->tmem;

    if (warp < 8) {
        // ================================================================ loader: HBM -> operand A1
        // Thread tid owns element pairs (e, e+1), e = 2 tid + 512 j, of every
        // transform of the tile: the whole tile sits in registers (one pass,
        // also for the FP16 tile maximum), n2 = e mod N2 is fixed per thread.
        constexpr int JT = S::n / 512, ITER = TB * JT;
        const float2 *in = a.in;
        const int e0 = 2 * tid, n2 = e0 % N2, n1_0 = e0 / N2;
        int it = 0;
        for (int64_t g = blockIdx.x; g < num_tiles; g += gridDim.x, it++) {
            const int64_t row0 = g * TB;
            const int ntr = static_cast<int>(a.rows - row0 < TB ? a.rows - row0 : TB);
            if (tid == 0 && a.aligned16) {
                // pull this CTA's next tile into L2 while this one is processed
                const int64_t g2 = g + gridDim.x;
                for (int t = 0; g2 < num_tiles && t < TB && g2 * TB + t < a.rows; t++)
                    prefetch_l2(in + (g2 * TB + t) * a.in_dist, S::n * 8);
            }
            float4 v[ITER];
#pragma unroll
            for (int j = 0; j < ITER; j++) {
                const int t = j / JT, jj = j % JT;
                v[j] = t < ntr ? load_pair(in + (row0 + t) * a.in_dist + e0 + 512 * jj, a.aligned16 != 0)
                               : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            float s1 = 1.0f;
            if constexpr (FMT == 0) {
                if (tid == 0) h->smax[(it + 2) & 3] = 0;
                float mx = 0.f;
#pragma unroll
                for (int j = 0; j < ITER; j++)
                    mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v[j].x), fabsf(v[j].y)), fmaxf(fabsf(v[j].z), fabsf(v[j].w))));
                for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                if (lane == 0) atomicMax(&h->smax[it & 3], __float_as_uint(mx));
                mbar_arrive(&h->max_bar);
                if (!tc_wait(&h->max_bar, it & 1, h, a.err)) break;
                s1 = pow2_scale_for(__uint_as_float(*reinterpret_cast<volatile uint32_t *>(&h->smax[it & 3])));
                if (tid == 0) h->scale[it & 15] = s1;
            }
            // operand A1 is free once the previous tile's stage A has completed
            if (it >= 1 && !tc_wait(&h->sa_done[(it - 1) & 1], ((it - 1) >> 1) & 1, h, a.err)) break;
#pragma unroll
            for (int j = 0; j < ITER; j++) {
                const int t = j / JT, jj = j % JT;
                const int n1 = n1_0 + (512 / N2) * jj;
                const int r = t * N2 + n2, ch = r >> 7, m = r & 127;
                uint32_t rh, rl, ih, il;
                split2<FMT>(v[j].x * s1, v[j].z * s1, rh, rl);
                split2<FMT>(v[j].y * s1, v[j].w * s1, ih, il);
                unsigned char *base = a1 + ch * S::A1_CHUNK;
                const uint32_t o_re = umma_offset_mn(m, n1, S::SBO_A), o_im = umma_offset_mn(m, N1 + n1, S::SBO_A);
                constexpr int LO = S::CHA * S::A1_CHUNK;
                *reinterpret_cast<uint32_t *>(base + o_re) = rh;
                *reinterpret_cast<uint32_t *>(base + LO + o_re) = rl;
                *reinterpret_cast<uint32_t *>(base + o_im) = ih;
                *reinterpret_cast<uint32_t *>(base + LO + o_im) = il;
            }
            fence_proxy_async_smem();
            mbar_arrive(&h->a1_full);
        }
    } else if (warp < 16) {
        // ================================================================ epilogues (8 warps)
        // Warps w and w + 4 share TMEM lane quarter w and split the columns.
        // Per tile i: stage-A epilogue of i (D1 -> twiddle -> A2), then the
        // stage-B epilogue of tile i - 1 (D2 -> HBM), which runs while the
        // tensor core computes stage B of tile i.
        const int quarter = warp & 3, half = (warp - 8) >> 2;
        const int m = quarter * 32 + lane;
        constexpr float kScaleB = FMT == 0 ? 1.0f / float(2 << ilog2c<N1>()) : 1.0f;
        // this thread's rows all have n2 = m mod N2; twiddle W^(k1 n2) for
        // k1 = 16 c + i is W^(16 c n2) * W^(i n2), the second factor kept here
        const int n2 = m % N2;
        float2 bw[16];
#pragma unroll
        for (int i = 0; i < 16; i++) bw[i] = __ldg(a.tw + i * n2);
        const uint32_t lane_base = tmem + (uint32_t(quarter * 32) << 16);

        auto stage_b_out = [&](int j, int64_t gj) {
            const int64_t row0 = gj * TB;
            float inv = 1.0f;
            if constexpr (FMT == 0) inv = float(2 << ilog2c<N1>()) / *reinterpret_cast<volatile float *>(&h->scale[j & 15]);
            const uint32_t dcol = lane_base + (2 + (j & 1)) * S::DC;
#pragma unroll 1
            for (int cb = 0; cb < S::CHB; cb++) {
                const int r = cb * 128 + m, t = r / N1, k1 = r % N1;
                const bool valid = row0 + t < a.rows;
                float2 *dst = a.out + (row0 + t) * a.out_dist + k1;
#pragma unroll 1
                for (int c16 = half * (S::KB / 32); c16 < (half + 1) * (S::KB / 32); c16++) {
                    uint32_t v[16];
                    tmem_ld16_nowait(dcol + cb * S::KB + c16 * 16, v);
                    tmem_wait_ld();
                    if (valid) {
#pragma unroll
                        for (int i = 0; i < 8; i++) {
                            const int k2 = c16 * 8 + i;
                            dst[N1 * k2] =
                                make_float2(__uint_as_float(v[2 * i]) * inv, __uint_as_float(v[2 * i + 1]) * inv);
                        }
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&h->d2_empty[j & 1]);
        };

        int it = 0;
        int64_t gprev = 0;
        bool ok = true;
        for (int64_t g = blockIdx.x; g < num_tiles; g += gridDim.x, it++) {
            if (!tc_wait(&h->sa_done[it & 1], (it >> 1) & 1, h, a.err)) {
                ok = false;
                break;
            }
            // operand A2 (and accumulator D2 of tile it - 1) are ready once
            // the previous tile's stage B has completed
            if (it >= 1 && !tc_wait(&h->sb_done[(it - 1) & 1], ((it - 1) >> 1) & 1, h, a.err)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t dcol = lane_base + (it & 1) * S::DC;
#pragma unroll 1
            for (int ch = 0; ch < S::CHA; ch++) {
                const int t = (ch * 128 + m) / N2;
#pragma unroll 1
                for (int c32 = half * (S::KA / 64); c32 < (half + 1) * (S::KA / 64); c32++) {
                    // 16 bins: two TMEM loads in flight
                    uint32_t v[32];
                    tmem_ld16_nowait(dcol + ch * S::KA + c32 * 32, v);
                    tmem_ld16_nowait(dcol + ch * S::KA + c32 * 32 + 16, v + 16);
                    const float2 aw = __ldg(a.tw + 16 * c32 * n2);
                    tmem_wait_ld();
#pragma unroll
                    for (int hh = 0; hh < 2; hh++) {
                        float re[8], im[8];
#pragma unroll
                        for (int i = 0; i < 8; i++) {
                            const int q = hh * 8 + i;
                            const float2 w = dir<FWD>(cmul(aw, bw[q]));
                            const float2 z =
                                cmul(make_float2(__uint_as_float(v[2 * q]), __uint_as_float(v[2 * q + 1])), w);
                            re[i] = z.x * kScaleB;
                            im[i] = z.y * kScaleB;
                        }
                        uint4 rh, rl, ih, il;
                        split2<FMT>(re[0], re[1], rh.x, rl.x);
                        split2<FMT>(re[2], re[3], rh.y, rl.y);
                        split2<FMT>(re[4], re[5], rh.z, rl.z);
                        split2<FMT>(re[6], re[7], rh.w, rl.w);
                        split2<FMT>(im[0], im[1], ih.x, il.x);
                        split2<FMT>(im[2], im[3], ih.y, il.y);
                        split2<FMT>(im[4], im[5], ih.z, il.z);
                        split2<FMT>(im[6], im[7], ih.w, il.w);
                        const int r2 = t * N1 + c32 * 16 + hh * 8, cb = r2 >> 7, m2 = r2 & 127;
                        unsigned char *base = a2 + cb * S::A2_CHUNK;
                        constexpr int LO = S::CHB * S::A2_CHUNK;
                        const uint32_t o_re = umma_offset_mn(m2, n2, S::SBO_B);
                        const uint32_t o_im = umma_offset_mn(m2, N2 + n2, S::SBO_B);
                        *reinterpret_cast<uint4 *>(base + o_re) = rh;
                        *reinterpret_cast<uint4 *>(base + LO + o_re) = rl;
                        *reinterpret_cast<uint4 *>(base + o_im) = ih;
                        *reinterpret_cast<uint4 *>(base + LO + o_im) = il;
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&h->d1_empty[it & 1]);
            fence_proxy_async_smem();
            mbar_arrive(&h->a2_full);
            if (it >= 1) stage_b_out(it - 1, gprev);
            gprev = g;
        }
        if (ok && it >= 1 && tc_wait(&h->sb_done[(it - 1) & 1], ((it - 1) >> 1) & 1, h, a.err)) {
            tc_fence_after();
            stage_b_out(it - 1, gprev);
        }
    } else if (lane == 0) {
        // ================================================================ MMA issue (one thread)
        constexpr uint32_t idesc_a = umma_instr_desc(128, S::KA, FMT, 1, 0);
        constexpr uint32_t idesc_b = umma_instr_desc(128, S::KB, FMT, 1, 0);
        const uint32_t fa_hi = smem_u32(fa), fa_lo = fa_hi + S::FA;
        const uint32_t fb_hi = smem_u32(fb), fb_lo = fb_hi + S::FB;
        const uint32_t a1_hi = smem_u32(a1), a1_lo = a1_hi + S::CHA * S::A1_CHUNK;
        const uint32_t a2_hi = smem_u32(a2), a2_lo = a2_hi + S::CHB * S::A2_CHUNK;
        // Stage A of tile na and stage B of tile nb are issued as soon as each
        // is ready (never one queued behind the other's wait).
        int ntiles = 0;
        for (int64_t g = blockIdx.x; g < num_tiles; g += gridDim.x) ntiles++;
        int na = 0, nb = 0;
        uint32_t idle = 0;
        while (nb < ntiles) {
            bool progressed = false;
            if (na < ntiles && mbar_test_wait(&h->a1_full, na & 1) &&
                (na < 2 || mbar_test_wait(&h->d1_empty[na & 1], ((na - 2) >> 1) & 1))) {
                tc_fence_after();
                const uint32_t d = tmem + (na & 1) * S::DC;
                for (int ch = 0; ch < S::CHA; ch++) {
                    const uint32_t ah[3] = {a1_hi, a1_hi, a1_lo}, bh[3] = {fa_hi, fa_lo, fa_hi};
#pragma unroll
                    for (int p = 0; p < 3; p++)
#pragma unroll
                        for (int kb = 0; kb < S::KA / 16; kb++)
                            tc_mma_f16(d + ch * S::KA,
                                       umma_smem_desc(ah[p] + ch * S::A1_CHUNK + kb * 256, 128, S::SBO_A),
                                       umma_smem_desc(bh[p] + kb * 256, 128, S::KA * 16), idesc_a, (p | kb) ? 1u : 0u);
                }
                tc_commit(&h->sa_done[na & 1]);
                na++;
                progressed = true;
            }
            if (nb < na && mbar_test_wait(&h->a2_full, nb & 1) &&
                (nb < 2 || mbar_test_wait(&h->d2_empty[nb & 1], ((nb - 2) >> 1) & 1))) {
                tc_fence_after();
                const uint32_t d = tmem + (2 + (nb & 1)) * S::DC;
                for (int cb = 0; cb < S::CHB; cb++) {
                    const uint32_t ah[3] = {a2_hi, a2_hi, a2_lo}, bh[3] = {fb_hi, fb_lo, fb_hi};
#pragma unroll
                    for (int p = 0; p < 3; p++)
#pragma unroll
                        for (int kb = 0; kb < S::KB / 16; kb++)
                            tc_mma_f16(d + cb * S::KB,
                                       umma_smem_desc(ah[p] + cb * S::A2_CHUNK + kb * 256, 128, S::SBO_B),
                                       umma_smem_desc(bh[p] + kb * 256, 128, S::KB * 16), idesc_b, (p | kb) ? 1u : 0u);
                }
                tc_commit(&h->sb_done[nb & 1]);
                nb++;
                progressed = true;
            }
            if (progressed) {
                idle = 0;
                continue;
            }
            if (*reinterpret_cast<volatile int *>(&h->abort)) break;
            if (++idle >= kMbarPollLimit) {  // nothing became ready for about a second
                *reinterpret_cast<volatile int *>(&h->abort) = 1;
                atomicExch(a.err, 3);
                break;
            }
            if (idle > 64) __nanosleep(32);
        }
    }
    // every role has left its loop: on the normal path all MMAs were waited on
    // (the last stage-B commit), on an abort nothing is waited for any more
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, S::TMEM_COLS);
}

// B operand of one stage: 2N x 2N real DFT matrix, K-major.  Row j = 2 k + c
// (output bin k, c = 0 real / 1 imaginary part), column kk = ci N + n (input
// n, ci = 0 real / 1 imaginary part); built in FP64 and split into hi / lo.
template <int FMT>
__global__ void tc_bmatrix_kernel(uint16_t *hi, uint16_t *lo, int N, int fwd)
{
    const int K = 2 * N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < K * K; i += gridDim.x * blockDim.x) {
        const int j = i / K, kk = i % K;
        const int k = j >> 1, c = j & 1, ci = kk / N, nn = kk % N;
        double s, cs;
        sincospi(2.0 * double((int64_t(k) * nn) % N) / double(N), &s, &cs);
        const double wi = fwd ? -s : s;  // exp(-+ i theta) = cs + i wi
        const double v = c == 0 ? (ci == 0 ? cs : -wi) : (ci == 0 ? wi : cs);
        const uint32_t off = umma_offset(j, kk, K) / 2;
        if (FMT == 0) {
            const __half hh = __double2half(v);
            hi[off] = __half_as_ushort(hh);
            lo[off] = __half_as_ushort(__double2half(v - double(__half2float(hh))));
        } else {
            const __nv_bfloat16 hh = __double2bfloat16(v);
            hi[off] = __bfloat16_as_ushort(hh);
            lo[off] = __bfloat16_as_ushort(__double2bfloat16(v - double(__bfloat162float(hh))));
        }
    }
}

// ------------------------------------------------------------------------------------ host side
namespace {

template <int N1, int N2, int TB>
const void *rows_fn(int fmt, bool fwd, size_t *smem)
{
    if (smem) *smem = TcRowShape<N1, N2, TB>::SMEM;
    if (fmt == 0)
        return fwd ? reinterpret_cast<const void *>(tc_rows_kernel<N1, N2, TB, 0, true>)
                   : reinterpret_cast<const void *>(tc_rows_kernel<N1, N2, TB, 0, false>);
    return fwd ? reinterpret_cast<const void *>(tc_rows_kernel<N1, N2, TB, 1, true>)
               : reinterpret_cast<const void *>(tc_rows_kernel<N1, N2, TB, 1, false>);
}

}  // namespace

bool tc_rows_config(int n, TcConfig &c)
{
    switch (n) {
        case 1024: c = {32, 32, 4}; return true;
        case 2048: c = {64, 32, 4}; return true;
        case 4096: c = {64, 64, 2}; return true;
        default: return false;
    }
}

const void *tc_rows_kernel_fn(int n, int fmt, bool fwd, size_t *smem)
{
    switch (n) {
        case 1024: return rows_fn<32, 32, 4>(fmt, fwd, smem);
        case 2048: return rows_fn<64, 32, 4>(fmt, fwd, smem);
        case 4096: return rows_fn<64, 64, 2>(fmt, fwd, smem);
        default: return nullptr;
    }
}

void tc_rows_kernel_fns(std::vector<const void *> &out)
{
    for (int n : {1024, 2048, 4096})
        for (int fmt = 0; fmt < 2; fmt++)
            for (int f = 0; f < 2; f++) out.push_back(tc_rows_kernel_fn(n, fmt, f != 0, nullptr));
}

cudaError_t fill_tc_bmatrix(uint16_t *hi, uint16_t *lo, int N, int fmt, bool fwd, cudaStream_t st)
{
    const int count = 4 * N * N;
    const int grid = (count + 255) / 256;
    if (fmt == 0)
        tc_bmatrix_kernel<0><<<grid, 256, 0, st>>>(hi, lo, N, fwd ? 1 : 0);
    else
        tc_bmatrix_kernel<1><<<grid, 256, 0, st>>>(hi, lo, N, fwd ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_tc_rows(int n, int fmt, bool fwd, const float2 *in, float2 *out, int64_t rows, int64_t in_dist,
                           int64_t out_dist, const uint16_t *fa, const uint16_t *fb, const float2 *tw, int grid,
                           int *err, cudaStream_t st)
{
    size_t smem = 0;
    const void *fn = tc_rows_kernel_fn(n, fmt, fwd, &smem);
    if (!fn || grid <= 0 || rows <= 0) return cudaErrorInvalidConfiguration;
    const bool aligned16 = (reinterpret_cast<uintptr_t>(in) & 15) == 0 && (in_dist & 1) == 0;
    TcRowArgs args{in, out, rows, in_dist, out_dist, fa, fb, tw, err, aligned16 ? 1 : 0};
    void *params[] = {&args};
    return cudaLaunchKernel(fn, dim3(grid), dim3(kTcRowThreads), params, smem, st);
}

}  // namespace sipfft
