// Compile-time specialised FFT engines for the hot lengths: their row
// kernels (TMA-pipelined, pipelined_rows.cuh), their double-buffered tile
// kernels (strided axes and multi-pass steps), the registry the planner
// looks engines up in, and the per-stage twiddle tables.  The engines
// themselves are in static_engine.cuh.  Lengths without a specialisation use
// the runtime-radix engine.
#include "sipfft_internal.h"
#include "static_engine.cuh"

namespace sipfft {

// ------------------------------------------------------------------------------------ double-buffered tiles
// The engines in the double-buffered tile skeleton (strided axes and
// multi-pass steps): the next tile's element copies are in flight (cp.async)
// while the engine runs the current tile in place; the first stage applies the
// inter-pass twiddles of a multi-pass step on read.
template <bool FWD>
struct PassRow {
    const float2 *row;
    const TileDesc *d;
    int64_t kc;
    __device__ __forceinline__ float2 operator()(int e) const
    {
        return cmul(row[pad(e)], pass_twiddle<FWD>(*d, e, kc));
    }
};

template <class E, bool FWD>
__global__ void __launch_bounds__(512, 1) static_db_kernel(const __grid_constant__ TileDesc d, int *)
{
    pdl_enter();
    extern __shared__ float2 sm[];
    const int64_t span = int64_t(d.tb) * d.pitch;
    const int tid = threadIdx.x;
    const int l = d.xfast ? tid % d.tb : tid / d.tpt;
    const int lane = d.xfast ? tid / d.tb : tid % d.tpt;
    const bool thread_on = tid < d.tb * d.tpt;
    int64_t g = blockIdx.x;
    if (g < d.num_tiles) issue_tile_c2c(d, d.in, sm, g);
    cp_async_commit();
    for (int i = 0; g < d.num_tiles; g += gridDim.x, i++) {
        float2 *cur = sm + (i & 1) * span;
        const int64_t gn = g + gridDim.x;
        if (gn < d.num_tiles) issue_tile_c2c(d, d.in, sm + ((i + 1) & 1) * span, gn);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int64_t o = g / d.tiles_per_outer;
        const int64_t c0 = (g % d.tiles_per_outer) * d.tb;
        const int64_t left = d.n_cols - c0;
        const int ntr = left < d.tb ? static_cast<int>(left) : d.tb;
        float2 *row = cur + (thread_on ? l : 0) * d.pitch;
        const bool act = thread_on && l < ntr;
        if (d.g_twiddle) {
            const int64_t kc = pass_column(d, c0 + (thread_on ? l : 0));
            E::template run<FWD>(d, row, PassRow<FWD>{row, &d, kc}, SmemRow{row}, true, lane, act);
        } else {
            E::template run<FWD>(d, row, SmemRow{row}, SmemRow{row}, true, lane, act);
        }
        __syncthreads();
        store_tile<FWD>(d, d.out, cur, o, c0, ntr);
        __syncthreads();
    }
    cp_async_wait<0>();
}

// ------------------------------------------------------------------------------------ registry
namespace {

// every boundary layout fits in the work row the planner sizes for i + i/16
template <class Q, class PD>
constexpr bool pads_fit()
{
    for (int b = 0; b + 1 < Q::S; b++) {
        const int i = Q::N - 1;
        const int at = PD::p(b) == 0 ? i : i + PD::q(b) * (i / PD::p(b));
        if (at > i + i / 16) return false;
    }
    return true;
}

// SH: the row kernels run a last radix-2 stage as warp-shuffle butterflies
// (StaticEngine WL = 2) where the engine's shape allows it
template <class Q, int T, class PD = Pads<>, bool PP = false, bool SH = false>
StaticKernel make_entry(int io_mask = 7)
{
    static_assert(pads_fit<Q, PD>(), "padded work row exceeds the planner's pitch");
    StaticKernel e{};
    e.io_mask = io_mask;
    e.n = Q::N;
    e.nstages = Q::S;
    for (int s = 0; s < Q::S; s++) e.radix[s] = Q::r[s];
    e.tpt = T;
    // row kernels: a transform of T <= 32 threads lives in one warp
    using E = StaticEngine<Q, T, PD, PP, (T <= 32 ? (SH ? 2 : 1) : 0)>;
    static_assert(!SH || ShflLast<Q, T, 2>::ok, "no warp-shuffle last stage for this engine");
    using EDb = StaticEngine<Q, T, PD, PP>;
    e.row_bufs = PP ? 3 : (E::kSingleBuffer ? 1 : 2);
    e.fn[1][0] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, true, IO_C2C>);
    e.fn[1][1] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, true, IO_R2C_PACKED>);
    e.fn[1][2] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, true, IO_C2R_PACKED>);
    e.fn[0][0] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, false, IO_C2C>);
    e.fn[0][1] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, false, IO_R2C_PACKED>);
    e.fn[0][2] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, false, IO_C2R_PACKED>);
    if constexpr (!PP && Q::N <= 8192) {  // the double-buffered tile kernel: no ping-pong area, two tiles in smem
        e.db[1] = reinterpret_cast<const void *>(static_db_kernel<EDb, true>);
        e.db[0] = reinterpret_cast<const void *>(static_db_kernel<EDb, false>);
    }
    return e;
}

const std::vector<StaticKernel> &registry()
{
    static const std::vector<StaticKernel> r = {
        make_entry<Seq<16, 4>, 4>(),            // 64
        make_entry<Seq<16, 8>, 8>(),            // 128
        make_entry<Seq<16, 16>, 16>(),          // 256
        // 512: C2C with a shared-memory last stage; the packed halves of the
        // 1024-point real transforms with warp-shuffle butterflies in the last
        // radix-2 stage (measured: C2R 1024 7 % and R2C 1024 3 % faster, C2C
        // 512 3 % slower than the shared-memory stage)
        make_entry<Seq<16, 16, 2>, 32>(1),
        make_entry<Seq<16, 16, 2>, 32, Pads<>, false, true>(6),
        make_entry<Seq<16, 16, 4>, 64>(),       // 1024
        // 2048, C2R: pre-twiddle fused into the radix-8 first stage, ping-pong
        // work rows (4 CTAs per SM instead of 6, measured 3 % faster; the R2C
        // engine measured the same either way and keeps 6)
        make_entry<Seq<8, 16, 16>, 128, Pads<>, true>(2),
        make_entry<Seq<16, 16, 8>, 128, Pads<1, 16, 1, 128>>(),  // 2048
        make_entry<Seq<16, 16, 16>, 256>(),     // 4096
        make_entry<Seq<16, 16, 16, 2>, 512>(),  // 8192
        // 16384, single pass: 32 points per thread, one row per CTA, the row loaded
        // once per tile into a single 139 KB buffer
        make_entry<Seq<16, 16, 16, 4>, 512>(),
        // 1500, the packed half of the 3000-point real transform: R2C on a
        // radix-5 last stage of 300 butterflies, two per thread, so that the
        // post-twiddle fuses into it; C2C and C2R on 10 x 10 x 15, one
        // butterfly per thread in the radix-10 stages; both with per-boundary
        // work-row layouts that halve the bank-conflicting shared-memory words
        make_entry<Seq<12, 5, 5, 5>, 150, Pads<1, 48, 1, 0, 1, 0>, true>(4),
        make_entry<Seq<10, 10, 15>, 150, Pads<1, 80, 3, 50>, true>(2),
        make_entry<Seq<10, 10, 15>, 150, Pads<1, 80, 3, 50>>(1),
    };
    return r;
}

}  // namespace

void static_kernel_fns(std::vector<const void *> &out)
{
    for (const StaticKernel &e : registry())
        for (int f = 0; f < 2; f++) {
            for (int io = 0; io < 3; io++) out.push_back(e.fn[f][io]);
            if (e.db[f]) out.push_back(e.db[f]);
        }
}

const StaticKernel *find_static_kernel(int n, int io)
{
    const int bit = io == IO_C2C ? 1 : (io == IO_C2R_PACKED ? 2 : (io == IO_R2C_PACKED ? 4 : 0));
    for (const StaticKernel &e : registry())
        if (e.n == n && (e.io_mask & bit)) return &e;
    return nullptr;
}

// t[off_s + (r-1)*Ns + k] = exp(-2 pi i r k / (Ns R)) for every stage s >= 1, in FP64 rounded to FP32
__global__ void stage_twiddle_kernel(float2 *t, int64_t count, int ns, int radix)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = i / ns + 1, k = i % ns;
        const int64_t den = int64_t(ns) * radix;
        const int64_t m = (r * k) % den;
        double s, c;
        sincospi(2.0 * static_cast<double>(m) / static_cast<double>(den), &s, &c);
        t[i] = make_float2(static_cast<float>(c), static_cast<float>(-s));
    }
}

cudaError_t fill_stage_twiddles(float2 *t, const int *radix, int nstages, cudaStream_t st)
{
    int64_t off = 0, ns = radix[0];
    for (int s = 1; s < nstages; s++) {
        const int64_t count = (radix[s] - 1) * ns;
        const int grid = static_cast<int>(std::min<int64_t>((count + 255) / 256, 1024));
        stage_twiddle_kernel<<<grid, 256, 0, st>>>(t + off, count, static_cast<int>(ns), radix[s]);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        off += count;
        ns *= radix[s];
    }
    return cudaSuccess;
}

int64_t stage_twiddle_count(const int *radix, int nstages)
{
    int64_t off = 0, ns = radix[0];
    for (int s = 1; s < nstages; s++) {
        off += (radix[s] - 1) * ns;
        ns *= radix[s];
    }
    return off;
}

}  // namespace sipfft
