// Persistent, TMA-pipelined FFT kernel skeleton for batched contiguous rows
// (the 1D hot path: C2C, and even-length R2C / C2R through the packed
// n/2-point FFT).
//
// Each CTA walks its tiles (tb consecutive rows) with two shared-memory
// buffers: while tile i is transformed in buffer i&1, the bulk-copy engine
// (cp.async.bulk, completion on an mbarrier) streams tile i+grid into the
// other buffer, so HBM reads run continuously under the butterflies.  Stage 0
// reads the staged rows in their HBM layout (C2R: pre-twiddled pairs computed
// on the fly), the remaining stages run in the padded work layout of the same
// buffer, and the last stage writes HBM directly (C2C, C2R) or, for R2C, the
// post-twiddle pass writes the N/2+1 bins.  One HBM read and one HBM write per
// element.
//
// The butterfly engine is a template parameter: RuntimeEngine (radices read
// from the descriptor) or a compile-time StaticEngine (static_fft.cu).
#pragma once
#include "async_copy.cuh"
#include "fft_tile.cuh"
#include "stages.cuh"

namespace sipfft {

// staged row in its HBM layout (unpadded)
struct StageRow {
    const float2 *row;
    __device__ __forceinline__ float2 operator()(int e) const { return row[e]; }
};

// C2R input seen as the packed m-point sequence Z (computed from X[e], X[m-e]):
// Z[e] = E + i O, E = X[e] + conj X[m-e], O = w^e (X[e] - conj X[m-e]),
// w = exp(-+2 pi i / 2m); DC and Nyquist imaginary parts are ignored.
template <bool FWD>
struct C2RPre {
    const float2 *x;  // staged half spectrum, m+1 bins
    int m;
    const float2 *tw;  // exp(-2 pi i k / 2m)
    __device__ __forceinline__ float2 operator()(int e) const
    {
        float2 xk = x[e];
        float2 xm = x[m - e];
        if (e == 0) {
            xk.y = 0.f;
            xm.y = 0.f;
        }
        return z(xk, xm, __ldg(tw + e));
    }
    // the same for e = j + off, twiddle w^j w^off
    __device__ __forceinline__ float2 split(int j, int off) const
    {
        const int e = j + off;
        float2 xk = x[e];
        float2 xm = x[m - e];
        if (e == 0) {
            xk.y = 0.f;
            xm.y = 0.f;
        }
        const float2 wj = __ldg(tw + j);
        return z(xk, xm, off == 0 ? wj : cmul(wj, __ldg(tw + off)));
    }
    __device__ __forceinline__ static float2 z(float2 xk, float2 xm, float2 w)
    {
        const float2 ev = make_float2(xk.x + xm.x, xk.y - xm.y);
        const float2 od = cmul(make_float2(xk.x - xm.x, xk.y + xm.y), dir<FWD>(w));
        return make_float2(ev.x - od.y, ev.y + od.x);
    }
};

// R2C bins k and m-k from Z[k], Z[m-k] and w = w^k (direction applied):
// X[k] = S/2 + w U/2 and X[m-k] = conj(S/2 - w U/2), with S = Z[k] + conj Z[m-k]
// and U = -i (Z[k] - conj Z[m-k]).
__device__ __forceinline__ void r2c_pair(float2 zk, float2 zm, float2 w, float2 &xk, float2 &xm)
{
    const float sx = zk.x + zm.x, sy = zk.y - zm.y;
    const float2 u = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    const float2 wu = cmul(w, u);
    xk = make_float2(fmaf(0.5f, sx, wu.x), fmaf(0.5f, sy, wu.y));
    xm = make_float2(fmaf(0.5f, sx, -wu.x), fmaf(-0.5f, sy, wu.y));
}

struct GlobalRow {
    float2 *row;
    __device__ __forceinline__ void operator()(int e, float2 v) const { st_stream(row + e, v); }
};

// R2C post-twiddle from the padded work row to HBM, one pair (k, n-k) per
// iteration.
template <bool FWD>
__device__ __forceinline__ void r2c_post_row(const float2 *work, float2 *y, int n, int lane, int tpt,
                                             const float2 *__restrict__ tw)
{
    for (int k = lane; 2 * k <= n; k += tpt) {
        float2 a, b;
        r2c_pair(work[pad(k)], work[pad(k == 0 ? 0 : n - k)], dir<FWD>(__ldg(tw + k)), a, b);
        y[k] = a;
        if (k == 0)
            y[n] = b;
        else if (2 * k != n)
            y[n - k] = b;
    }
}

// COMPACT: radices up to kCompactMaxRadix only, CTAs of at most 256 threads,
// three per SM (80 registers); else every radix, up to 512 threads.
template <int MAXE, bool COMPACT = false>
struct RuntimeEngine {
    static constexpr bool kPingPong = false;
    static constexpr bool kSingleBuffer = false;
    static constexpr int kMaxThreads = COMPACT ? 256 : 512;
    static constexpr int kMinBlocks = COMPACT ? 3 : 1;
    template <bool FWD, class Src0, class DstL>
    __device__ __forceinline__ static void run(const TileDesc &d, float2 *work, const Src0 &src0, const DstL &dstL,
                                               bool dst_in_place, int lane, bool active, float2 * = nullptr)
    {
        run_fft<MAXE, FWD, COMPACT>(d, work, src0, true, dstL, dst_in_place, lane, active);
    }
    template <bool FWD, class DstL>
    __device__ __forceinline__ static void run_c2r(const TileDesc &d, float2 *work, const float2 *x, const DstL &dstL,
                                                   int lane, bool active, float2 * = nullptr)
    {
        run_fft<MAXE, FWD, COMPACT>(d, work, C2RPre<FWD>{x, d.n, d.tw}, true, dstL, false, lane, active);
    }
    // R2C: packed FFT into the work row, then the post-twiddle pass to HBM
    template <bool FWD, class Src0>
    __device__ __forceinline__ static void run_r2c(const TileDesc &d, float2 *work, const Src0 &src0, float2 *y,
                                                   int lane, bool active, float2 * = nullptr)
    {
        run_fft<MAXE, FWD, COMPACT>(d, work, src0, true, SmemRow{work}, true, lane, active);
        __syncthreads();
        if (active) r2c_post_row<FWD>(work, y, d.n, lane, d.tpt, d.tw);
    }
};

template <class Engine, bool FWD, int IO>
__global__ void __launch_bounds__(Engine::kMaxThreads, Engine::kMinBlocks)
    pipelined_rows_kernel(const __grid_constant__ TileDesc d, int *err)
{
    pdl_wait();
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smraw);
    const int64_t buf_f2 = d.g_ns;  // per-buffer float2 count (planner-computed, even)
    float2 *bufs = reinterpret_cast<float2 *>(smraw + 128);
    const int tid = threadIdx.x;
    const int tb = d.tb, tpt = d.tpt;
    const int l = tid / tpt, lane = tid % tpt;
    const bool thread_on = tid < tb * tpt;
    const int64_t in_dist = d.in_a.dist, out_dist = d.out_a.dist;
    const int64_t rows_total = d.n_cols;
    const float2 *in = static_cast<const float2 *>(d.in);
    float2 *out = static_cast<float2 *>(d.out);

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    __syncthreads();

    // Tile t spans elements [s, e) of the input.  The bulk engine copies whole
    // 16-byte lines from s & ~1, so with an odd s the staged rows start one
    // element in (the copy's first element is the previous row's last); an odd
    // e is rounded up (the next row's first element comes along) except at the
    // end of the input, where the last element is fetched with a plain load.
    // The input ends after the last row's own bins, not a full row distance on.
    const int64_t total = (rows_total - 1) * in_dist + d.n + (IO == IO_C2R_PACKED ? 1 : 0);
    auto tile_rows = [&](int64_t t) -> int {
        const int64_t left = rows_total - t * tb;
        return left < tb ? static_cast<int>(left) : tb;
    };
    auto issue = [&](int64_t t, int b) {
        if (tid == 0) {
            const int64_t s = t * tb * in_dist, e = min(s + tile_rows(t) * in_dist, total);
            const int64_t z = e < total ? e + (e & 1) : e & ~int64_t(1);
            const uint32_t bulk = static_cast<uint32_t>((z - (s & ~int64_t(1))) * 8);
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&bars[b], bulk);
            if (bulk) bulk_g2s(bufs + b * buf_f2, in + (s & ~int64_t(1)), bulk, &bars[b]);
        }
    };

    int64_t t = blockIdx.x;
    if (t < d.num_tiles) issue(t, 0);
    for (int i = 0; t < d.num_tiles; t += gridDim.x, i++) {
        // two buffers: the next tile streams in while this one is transformed;
        // one buffer (Engine::kSingleBuffer): the next tile is loaded after this one
        const int b = Engine::kSingleBuffer ? 0 : (i & 1);
        const int64_t tn = t + gridDim.x;
        if (!Engine::kSingleBuffer && tn < d.num_tiles) issue(tn, b ^ 1);
        // A thread whose bounded wait gave up records it and still runs the
        // tile (on whatever the buffer holds: every access stays in bounds), so
        // that every thread reaches the same barriers; the CTA leaves together
        // at the end of the iteration.
        if (tn >= d.num_tiles) pdl_launch_dependents();  // this CTA's last tile (a CTA without tiles: at exit)
        const bool timed_out = !mbar_wait_bounded(&bars[b], Engine::kSingleBuffer ? (i & 1) : ((i >> 1) & 1));
        if (timed_out) atomicExch(err, 1);
        const int rows = tile_rows(t);
        float2 *buf = bufs + b * buf_f2;
        const int64_t s = t * tb * in_dist, e = min(s + rows * in_dist, total);
        const float2 *stage = buf + (s & 1);
        if (e == total && (e & 1)) {  // last tile of an odd-length input; uniform across the CTA
            if (tid == 0) buf[(e - 1) - (s & ~int64_t(1))] = in[e - 1];
            __syncthreads();
        }
        const bool active = thread_on && l < rows;
        float2 *work = buf + l * d.pitch;
        float2 *work2 = Engine::kPingPong ? bufs + 2 * buf_f2 + l * d.pitch : nullptr;
        const int64_t row_index = t * tb + l;
        if constexpr (IO == IO_C2C) {
            Engine::template run<FWD>(d, work, StageRow{stage + l * in_dist},
                                      GlobalRow{out + row_index * out_dist}, false, lane, active, work2);
        } else if constexpr (IO == IO_C2R_PACKED) {
            Engine::template run_c2r<FWD>(d, work, stage + l * in_dist, GlobalRow{out + row_index * out_dist}, lane,
                                          active, work2);
        } else {  // IO_R2C_PACKED
            Engine::template run_r2c<FWD>(d, work, StageRow{stage + l * in_dist}, out + row_index * out_dist, lane,
                                          active, work2);
        }
        // buffer b is free for the copy issued in iteration i+1; a CTA-uniform exit after a timeout
        if (__syncthreads_or(timed_out)) return;
        if (Engine::kSingleBuffer && tn < d.num_tiles) issue(tn, 0);
    }
}

}  // namespace sipfft
