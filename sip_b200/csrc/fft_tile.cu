// sm_100a tile FFT kernel: shared-memory-resident mixed-radix Stockham.
//
// One CTA owns `tb` transforms of length n (or `tb` columns of a multi-pass
// Stockham pass).  Phases:
//   1. load  — HBM -> shared memory, coalesced along whichever axis is
//              contiguous in HBM (rows: along the transform; columns: across
//              transforms), with R2C/C2R packing and pass twiddles applied;
//   2. stages — for each radix R: every thread gathers its butterflies'
//              R inputs into registers, applies the stage twiddles, runs the
//              register codelet, barrier, scatters the outputs (Stockham
//              autosort, so no digit reversal pass);
//   3. store — shared memory -> HBM with the R2C post-twiddle or the
//              transposed (column) layout of the next axis / next pass.
// HBM traffic per launch is one read and one write of the tile.
// The shared-memory row index is padded (i + i/16) so that the strided
// scatter of the early stages and the column-tile loads are bank-conflict
// free for 8-byte elements.
#include <algorithm>
#include <vector>

#include "async_copy.cuh"
#include "codelets.cuh"
#include "fft_tile.cuh"
#include "sipfft_internal.h"
#include "tile_io.cuh"

namespace sipfft {


// Register budget of one stage: NB butterflies of radix R per thread.
template <int R, int MAXE>
constexpr int nb_for() { return (MAXE + R - 1) / R; }
template <int MAXE, bool COMPACT = false>
constexpr int maxv_for()
{
    constexpr int r[] = {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 16};
    int m = 0;
    for (int x : r)
        if (!COMPACT || x <= kCompactMaxRadix) m = m > ((MAXE + x - 1) / x) * x ? m : ((MAXE + x - 1) / x) * x;
    return m;
}

// Gather the R inputs of each of this thread's butterflies, apply the stage
// twiddles and run the codelet; results stay in v until after the barrier.
// Stage twiddles come from the stage's own table when the plan has one
// (tws[(r-1)*ns + j mod ns]: consecutive butterflies read consecutive
// entries), else from the length-n table (tw[r*(j mod ns)*tstep]).
template <int R, int MAXE, bool FWD>
__device__ __forceinline__ void stage_read(float2 *v, const float2 *row, int n, int ns, uint32_t nsm, int tstep,
                                           int lane, int tpt, bool active, const float2 *__restrict__ tw,
                                           const float2 *__restrict__ tws, const TileDesc &d, int64_t kc)
{
    constexpr int NB = nb_for<R, MAXE>();
    const int nbf = n / R;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = lane + b * tpt;
        if (active && j < nbf) {
#pragma unroll
            for (int r = 0; r < R; r++) v[b * R + r] = row[pad(j + r * nbf)];
            if (kc >= 0) {
                // inter-pass twiddle of a multi-pass step, applied on the first read
#pragma unroll
                for (int r = 0; r < R; r++) v[b * R + r] = cmul(v[b * R + r], pass_twiddle<FWD>(d, j + r * nbf, kc));
            }
            if (ns > 1) {
                const int k = mod_ns(j, ns, nsm);
                if (tws) {
#pragma unroll
                    for (int r = 1; r < R; r++)
                        v[b * R + r] = cmul(v[b * R + r], dir<FWD>(__ldg(tws + (r - 1) * ns + k)));
                } else {
                    const int step = k * tstep;
#pragma unroll
                    for (int r = 1; r < R; r++) v[b * R + r] = cmul(v[b * R + r], dir<FWD>(__ldg(tw + r * step)));
                }
            }
            dft<R, FWD>(v + b * R);
        }
    }
}

// Scatter the butterfly outputs to their Stockham positions.
template <int R, int MAXE>
__device__ __forceinline__ void stage_write(const float2 *v, float2 *row, int n, int ns, uint32_t nsm, int lane,
                                            int tpt, bool active)
{
    constexpr int NB = nb_for<R, MAXE>();
    const int nbf = n / R;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = lane + b * tpt;
        if (active && j < nbf) {
            const int k = mod_ns(j, ns, nsm);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) row[pad(base + r * ns)] = v[b * R + r];
        }
    }
}

#define SIPFFT_RADIX_CASES(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(16)
#define SIPFFT_COMPACT_RADIX_CASES(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)

// One register array is shared by all radices so that only one set of
// butterfly values is live across each stage barrier.
// kc >= 0: the tile's inter-pass twiddles (column kc) are still to be applied (first stage does it).
// COMPACT: only radices up to kCompactMaxRadix are compiled (plans built with
// Plan::max_radix = kCompactMaxRadix), which keeps the uneven-batch kernel at
// three CTAs per SM.
template <int MAXE, bool FWD, bool COMPACT = false>
__device__ __forceinline__ void run_stages(float2 *row, const TileDesc &d, int lane, bool active, int64_t kc = -1)
{
    float2 v[maxv_for<MAXE, COMPACT>()];
    int64_t toff = 0;  // offset of this stage's table in d.stw (stage 0 has none)
#pragma unroll 1
    for (int s = 0; s < d.nstages; s++) {
        const int ns = d.ns[s], ts = d.tstep[s], R = d.radix[s];
        const uint32_t nsm = d.ns_m[s];
        const float2 *tws = d.stw ? d.stw + toff : nullptr;
        if (s > 0) toff += int64_t(R - 1) * ns;
#define SIPFFT_READ(RR) \
    case RR: stage_read<RR, MAXE, FWD>(v, row, d.n, ns, nsm, ts, lane, d.tpt, active, d.tw, tws, d, s == 0 ? kc : -1); break;
#define SIPFFT_WRITE(RR) \
    case RR: stage_write<RR, MAXE>(v, row, d.n, ns, nsm, lane, d.tpt, active); break;
        if constexpr (COMPACT) {
            switch (R) {
                SIPFFT_COMPACT_RADIX_CASES(SIPFFT_READ)
                default: break;  // the planner only emits the radices above
            }
            __syncthreads();
            switch (R) {
                SIPFFT_COMPACT_RADIX_CASES(SIPFFT_WRITE)
                default: break;
            }
        } else {
            switch (R) {
                SIPFFT_RADIX_CASES(SIPFFT_READ)
                default: break;  // the planner only emits the radices above
            }
            __syncthreads();
            switch (R) {
                SIPFFT_RADIX_CASES(SIPFFT_WRITE)
                default: break;
            }
        }
#undef SIPFFT_READ
#undef SIPFFT_WRITE
        __syncthreads();
    }
}

__device__ __forceinline__ void conj_tile(const TileDesc &d, float2 *sm, int ntr)
{
    for (int i = threadIdx.x; i < ntr * d.n; i += blockDim.x) {
        float2 *p = sm + (i / d.n) * d.pitch + pad(i % d.n);
        p->y = -p->y;
    }
}

// flip: the segment's direction is the opposite of FWD (C2C / Bluestein tiles only:
// their load and store phases do not depend on the direction)
// loaded: the tile's input already sits in sm (copied by cp.async, inter-pass
// twiddles not applied yet)
template <int MAXE, bool FWD, bool COMPACT = false>
__device__ __forceinline__ void process_tile(const TileDesc &d, const void *in, void *out, int64_t g, float2 *sm,
                                             bool flip = false, bool loaded = false)
{
    const int tid = threadIdx.x;
    int l, lane;
    if (d.xfast) {
        l = tid % d.tb;
        lane = tid / d.tb;
    } else {
        l = tid / d.tpt;
        lane = tid % d.tpt;
    }
    const bool thread_on = tid < d.tb * d.tpt;
    const int64_t o = g / d.tiles_per_outer;
    const int64_t c0 = (g % d.tiles_per_outer) * d.tb;
    const int64_t left = d.n_cols - c0;
    const int ntr = left < d.tb ? static_cast<int>(left) : d.tb;
    if (!loaded) {
        load_tile<FWD>(d, in, sm, o, c0, ntr);
        __syncthreads();
    }
    const int64_t kc = loaded && d.g_twiddle ? pass_column(d, c0 + (thread_on ? l : 0)) : -1;
    if (flip) {
        conj_tile(d, sm, ntr);
        __syncthreads();
    }
    run_stages<MAXE, FWD, COMPACT>(sm + (thread_on ? l : 0) * d.pitch, d, lane, thread_on && l < ntr, kc);
    if (flip) {
        conj_tile(d, sm, ntr);
        __syncthreads();
    }
    store_tile<FWD>(d, out, sm, o, c0, ntr);
    __syncthreads();
}

template <int MAXE, bool FWD>
__global__ void __launch_bounds__(512, 1) tile_fft_kernel(const __grid_constant__ TileDesc d)
{
    pdl_enter();
    extern __shared__ float2 sm[];
    for (int64_t g = blockIdx.x; g < d.num_tiles; g += gridDim.x) process_tile<MAXE, FWD>(d, d.in, d.out, g, sm);
}

// ------------------------------------------------------------------------------------ double-buffered tiles
// Persistent variant for C2C tiles (column tiles of strided axes and of
// multi-pass steps): while a tile runs its stages, the element copies of the
// CTA's next tile are already in flight into the second buffer (cp.async,
// 8 bytes per element, no registers held), so HBM latency overlaps compute.
template <int MAXE, bool FWD>
__global__ void __launch_bounds__(512, 1) tile_db_kernel(const __grid_constant__ TileDesc d)
{
    pdl_enter();
    extern __shared__ float2 sm[];
    const int64_t span = int64_t(d.tb) * d.pitch;
    const int tid = threadIdx.x;
    int l, lane;
    if (d.xfast) {
        l = tid % d.tb;
        lane = tid / d.tb;
    } else {
        l = tid / d.tpt;
        lane = tid % d.tpt;
    }
    const bool thread_on = tid < d.tb * d.tpt;
    int64_t g = blockIdx.x;
    if (g < d.num_tiles) issue_tile_c2c(d, d.in, sm, g);
    cp_async_commit();
    for (int i = 0; g < d.num_tiles; g += gridDim.x, i++) {
        float2 *cur = sm + (i & 1) * span;
        const int64_t gn = g + gridDim.x;
        // the other buffer was released by the barrier that ended the previous tile
        if (gn < d.num_tiles) issue_tile_c2c(d, d.in, sm + ((i + 1) & 1) * span, gn);
        cp_async_commit();
        cp_async_wait<1>();  // this tile's copies (all groups but the newest) have landed
        __syncthreads();
        const int64_t o = g / d.tiles_per_outer;
        const int64_t c0 = (g % d.tiles_per_outer) * d.tb;
        const int64_t left = d.n_cols - c0;
        const int ntr = left < d.tb ? static_cast<int>(left) : d.tb;
        const int64_t kc = d.g_twiddle ? pass_column(d, c0 + (thread_on ? l : 0)) : -1;
        run_stages<MAXE, FWD>(cur + (thread_on ? l : 0) * d.pitch, d, lane, thread_on && l < ntr, kc);
        store_tile<FWD>(d, d.out, cur, o, c0, ntr);
        __syncthreads();
    }
    cp_async_wait<0>();
}

// ------------------------------------------------------------------------------------ uneven batches
// One persistent launch over many transform groups of different lengths.
// Work items (segment, tile) are dequeued in order from a global counter;
// a segment that consumes another segment's output (the next pass of a
// multi-pass transform, the second half of a Bluestein transform) waits,
// with a bounded spin, until every tile of that segment has been published.
// Items are ordered so that every producer tile is dequeued before its
// consumers and all CTAs are resident (grid = occupancy), so the waits end:
// a CTA holds at most two items (the one it computes and the next one it
// prefetches) and each waits only on items dequeued before it.
//
// Double buffering: while an item computes in one shared-memory buffer, the
// CTA dequeues its next item and, when that is a plain C2C tile whose
// producer has already finished, starts its element copies (cp.async) into
// the other buffer.  Other items (Bluestein halves, producers still running)
// load synchronously when their turn comes.
__device__ __forceinline__ bool batch_dep_done(const BatchSeg *segs, int *done, const BatchSeg &sg)
{
    if (sg.dep < 0) return true;
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(done + sg.dep) : "memory");
    return v >= segs[sg.dep].ntiles;
}

__device__ __forceinline__ bool batch_dep_wait(const BatchSeg *segs, int *done, const BatchSeg &sg, int *err)
{
    for (uint32_t poll = 0; poll < (1u << 24); poll++) {
        if (batch_dep_done(segs, done, sg)) return true;
        __nanosleep(128);
    }
    atomicExch(err, 2);
    return false;
}

// The tile descriptor of the item a CTA computes and of the one it prefetches
// sit in shared memory (copied once per item), so the stage loops read them
// with shared-memory latency instead of re-reading the segment list.
__device__ __forceinline__ void copy_desc(TileDesc *dst, const TileDesc &src)
{
    static_assert(sizeof(TileDesc) % 8 == 0, "descriptor copied as 8-byte words");
    const uint64_t *s = reinterpret_cast<const uint64_t *>(&src);
    uint64_t *d = reinterpret_cast<uint64_t *>(dst);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(TileDesc) / 8); i += blockDim.x) d[i] = __ldg(s + i);
}

// COMPACT (plans of radices <= kCompactMaxRadix): 80 registers, three CTAs per
// SM; else every radix, two CTAs per SM.
template <int MAXE, bool FWD, bool COMPACT>
__global__ void __launch_bounds__(kBatchBlock, COMPACT ? 3 : 2)
    batch_fft_kernel(const BatchSeg *__restrict__ segs, const int2 *__restrict__ items, int nitems, int *counter,
                     int *done, BatchBufs bufs, int *err, int64_t span)
{
    extern __shared__ float2 sm[];
    // [i & 1]: the item computed in iteration i (the next item's slots are
    // written while the current item's are still read)
    __shared__ int s_item[2], s_pref[2], s_ok;
    __shared__ TileDesc s_desc[2];
    const int tid = threadIdx.x;
    auto dequeue = [&](int slot) {
        const int w = atomicAdd(counter, 1);
        int pf = 0;
        if (w < nitems) {
            const BatchSeg &sg = segs[items[w].x];
            pf = sg.d.io == IO_C2C && batch_dep_done(segs, done, sg);
        }
        s_item[slot] = w;
        s_pref[slot] = pf;
    };
    // dequeue the first item; prefetch it when it is ready to read
    if (tid == 0) dequeue(0);
    __syncthreads();
    int w = s_item[0];
    bool pref = s_pref[0] != 0;
    if (w < nitems) {
        const int2 it = items[w];
        const BatchSeg &sg = segs[it.x];
        copy_desc(&s_desc[0], sg.d);
        if (pref) issue_tile_c2c(sg.d, static_cast<const char *>(bufs.p[sg.in_buf]) + sg.in_off, sm, it.y);
    }
    cp_async_commit();
    for (int i = 0; w < nitems; i++) {
        const int nx = (i + 1) & 1;
        float2 *cur = sm + (i & 1) * span;
        // dequeue the next item, copy its descriptor and prefetch it into the
        // other buffer when its producer has finished (the previous iteration's
        // item, whose slots and buffer these are, ended with a barrier)
        if (tid == 0) dequeue(nx);
        __syncthreads();
        const int wn = s_item[nx];
        const bool pref_n = s_pref[nx] != 0;
        if (wn < nitems) {
            const int2 itn = items[wn];
            const BatchSeg &nsg = segs[itn.x];
            copy_desc(&s_desc[nx], nsg.d);
            if (pref_n)
                issue_tile_c2c(nsg.d, static_cast<const char *>(bufs.p[nsg.in_buf]) + nsg.in_off, sm + nx * span,
                               itn.y);
        }
        cp_async_commit();

        const int2 it = items[w];
        const BatchSeg &sg = segs[it.x];
        const char *in = static_cast<const char *>(bufs.p[sg.in_buf]) + sg.in_off;
        char *out = static_cast<char *>(bufs.p[sg.out_buf]) + sg.out_off;
        bool ok = true;
        if (!pref) {
            if (tid == 0) s_ok = batch_dep_wait(segs, done, sg, err) ? 1 : 0;
            __syncthreads();
            ok = s_ok != 0;
        }
        cp_async_wait<1>();  // the current item's copies (if prefetched) have landed
        __syncthreads();
        if (ok) {
            // a Bluestein segment runs its convolution FFTs in both directions; the
            // other direction is conj(DFT(conj(y))) around this kernel's stages
            process_tile<MAXE, FWD, COMPACT>(s_desc[i & 1], in, out, it.y, cur, sg.fwd != (FWD ? 1 : 0), pref);
            if (tid == 0) {
                __threadfence();
                atomicAdd(done + it.x, 1);
            }
        }
        w = wn;
        pref = pref_n;
    }
    cp_async_wait<0>();
}

// ------------------------------------------------------------------------------------ twiddles
// t[m] = exp(-2 pi i * ((m * mult) mod denom) / denom), evaluated in FP64 and
// rounded once to FP32 (the reference builds its tables the same way on the
// host: core/fft/fftcore/fft_core_common_func.cpp:214-232).
__global__ void twiddle_kernel(float2 *t, int64_t count, int64_t denom, int64_t mult)
{
    for (int64_t m = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; m < count;
         m += int64_t(gridDim.x) * blockDim.x) {
        const int64_t idx = (m * mult) % denom;
        double s, c;
        sincospi(2.0 * static_cast<double>(idx) / static_cast<double>(denom), &s, &c);
        t[m] = make_float2(static_cast<float>(c), static_cast<float>(-s));
    }
}

// Bluestein tables.  chirp[n] = exp(s*pi*i*(n^2 mod 2N)/N) (s = -1 forward),
// with n^2 reduced exactly in 64-bit integers before the FP64 evaluation.
__global__ void chirp_kernel(float2 *t, int64_t n_len, int sign)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_len;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t q = (i * i) % (2 * n_len);
        double s, c;
        sincospi(static_cast<double>(q) / static_cast<double>(n_len), &s, &c);
        t[i] = make_float2(static_cast<float>(c), static_cast<float>(sign * s));
    }
}

// b[m] = conj(chirp[m]) for m < N, b[M-m] = conj(chirp[m]) for 0 < m < N, else 0
__global__ void bluestein_b_kernel(float2 *b, const float2 *chirp, int64_t n_len, int64_t m_len)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m_len;
         i += int64_t(gridDim.x) * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (i < n_len)
            v = cconj(chirp[i]);
        else if (m_len - i < n_len)
            v = cconj(chirp[m_len - i]);
        b[i] = v;
    }
}

__global__ void scale_kernel(float2 *b, int64_t count, float s)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
         i += int64_t(gridDim.x) * blockDim.x)
        b[i] = cscale(b[i], s);
}

cudaError_t fill_chirp(float2 *t, int64_t n_len, bool forward, cudaStream_t st)
{
    const int grid = static_cast<int>(std::min<int64_t>((n_len + 255) / 256, 1024));
    chirp_kernel<<<grid, 256, 0, st>>>(t, n_len, forward ? -1 : 1);
    return cudaGetLastError();
}

cudaError_t fill_bluestein_b(float2 *b, const float2 *chirp, int64_t n_len, int64_t m_len, cudaStream_t st)
{
    const int grid = static_cast<int>(std::min<int64_t>((m_len + 255) / 256, 1024));
    bluestein_b_kernel<<<grid, 256, 0, st>>>(b, chirp, n_len, m_len);
    return cudaGetLastError();
}

cudaError_t scale_table(float2 *b, int64_t count, float s, cudaStream_t st)
{
    const int grid = static_cast<int>(std::min<int64_t>((count + 255) / 256, 1024));
    scale_kernel<<<grid, 256, 0, st>>>(b, count, s);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------ host side
namespace {
template <int MAXE, bool FWD>
cudaError_t launch_one(const TileDesc &d, int grid, int block, size_t smem, cudaStream_t st)
{
    TileDesc dd = d;
    void *args[] = {&dd};
    return launch_pdl(reinterpret_cast<const void *>(tile_fft_kernel<MAXE, FWD>), dim3(grid), dim3(block), smem, st,
                      args);
}
}  // namespace

// Kernels of this file whose dynamic shared-memory limit must be raised
// before their first launch (configure_kernels() in runtime.cpp).
void tile_kernel_fns(std::vector<const void *> &out)
{
    out.push_back(reinterpret_cast<const void *>(tile_fft_kernel<8, true>));
    out.push_back(reinterpret_cast<const void *>(tile_fft_kernel<8, false>));
    out.push_back(reinterpret_cast<const void *>(tile_fft_kernel<16, true>));
    out.push_back(reinterpret_cast<const void *>(tile_fft_kernel<16, false>));
    out.push_back(reinterpret_cast<const void *>(tile_fft_kernel<32, true>));
    out.push_back(reinterpret_cast<const void *>(tile_fft_kernel<32, false>));
    for (int c = 0; c < 2; c++) {
        out.push_back(batch_kernel_fn(true, c != 0));
        out.push_back(batch_kernel_fn(false, c != 0));
    }
    for (int maxe : {8, 16, 32})
        for (int f = 0; f < 2; f++) out.push_back(tile_db_kernel_fn(maxe, f != 0));
}

const void *tile_db_kernel_fn(int maxe, bool forward)
{
    if (maxe <= 8) return forward ? reinterpret_cast<const void *>(tile_db_kernel<8, true>)
                                  : reinterpret_cast<const void *>(tile_db_kernel<8, false>);
    if (maxe <= 16) return forward ? reinterpret_cast<const void *>(tile_db_kernel<16, true>)
                                   : reinterpret_cast<const void *>(tile_db_kernel<16, false>);
    return forward ? reinterpret_cast<const void *>(tile_db_kernel<32, true>)
                   : reinterpret_cast<const void *>(tile_db_kernel<32, false>);
}

cudaError_t launch_tile_db(const TileDesc &d, int maxe, bool forward, int grid, cudaStream_t st)
{
    const int block = d.tb * d.tpt;
    const size_t smem = 2 * static_cast<size_t>(d.tb) * d.pitch * sizeof(float2);
    if (block <= 0 || block > 512 || smem > static_cast<size_t>(kMaxSmemBytes) || grid <= 0 || d.io != IO_C2C)
        return cudaErrorInvalidConfiguration;
    TileDesc dd = d;
    void *args[] = {&dd};
    return launch_pdl(tile_db_kernel_fn(maxe, forward), dim3(grid), dim3(block), smem, st, args);
}

cudaError_t launch_tile(const TileDesc &d, int maxe, bool forward, int grid, cudaStream_t st)
{
    const int block = d.tb * d.tpt;
    const size_t smem = static_cast<size_t>(d.tb) * d.pitch * sizeof(float2);
    if (block <= 0 || block > 512 || smem > static_cast<size_t>(kMaxSmemBytes) || grid <= 0)
        return cudaErrorInvalidConfiguration;
    if (maxe <= 8) return forward ? launch_one<8, true>(d, grid, block, smem, st)
                                  : launch_one<8, false>(d, grid, block, smem, st);
    if (maxe <= 16) return forward ? launch_one<16, true>(d, grid, block, smem, st)
                                   : launch_one<16, false>(d, grid, block, smem, st);
    return forward ? launch_one<32, true>(d, grid, block, smem, st) : launch_one<32, false>(d, grid, block, smem, st);
}

const void *batch_kernel_fn(bool forward, bool compact)
{
    if (compact)
        return forward ? reinterpret_cast<const void *>(batch_fft_kernel<kBatchMaxe, true, true>)
                       : reinterpret_cast<const void *>(batch_fft_kernel<kBatchMaxe, false, true>);
    return forward ? reinterpret_cast<const void *>(batch_fft_kernel<kBatchMaxe, true, false>)
                   : reinterpret_cast<const void *>(batch_fft_kernel<kBatchMaxe, false, false>);
}

cudaError_t launch_batch(int grid, int block, size_t smem, const BatchSeg *segs, const int2 *items, int nitems,
                         int *counter, int *done, const BatchBufs &bufs, int *err, bool forward, bool compact,
                         cudaStream_t st)
{
    const void *fn = batch_kernel_fn(forward, compact);
    BatchBufs b = bufs;
    int64_t span = static_cast<int64_t>(smem / 2 / sizeof(float2));  // float2 per buffer
    void *args[] = {&segs, &items, &nitems, &counter, &done, &b, &err, &span};
    return cudaLaunchKernel(fn, dim3(grid), dim3(block), args, smem, st);
}

cudaError_t fill_twiddles(float2 *t, int64_t count, int64_t denom, int64_t mult, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    const int block = 256;
    int64_t grid = (count + block - 1) / block;
    if (grid > 4096) grid = 4096;
    twiddle_kernel<<<static_cast<int>(grid), block, 0, st>>>(t, count, denom, mult);
    return cudaGetLastError();
}

}  // namespace sipfft
