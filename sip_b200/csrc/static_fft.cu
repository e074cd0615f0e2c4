// Compile-time specialised FFT engines for the hot lengths.
//
// For a length whose radix sequence and threads per transform are fixed at
// compile time, every stage's butterfly count, Ns, (j mod Ns), padded
// shared-memory address and twiddle-table offset folds into constants, loops
// unroll completely, and the stage twiddles come from per-stage tables laid
// out [r-1][k] so that the 32 lanes of a warp read consecutive entries.  The
// engines plug into the TMA-pipelined row skeleton (pipelined_rows.cuh).
// Lengths without a specialisation use the runtime-radix engine.
#include "pipelined_rows.cuh"
#include "tile_io.cuh"

namespace sipfft {

template <int... Rs>
struct Seq {
    static constexpr int S = sizeof...(Rs);
    static constexpr int r[S] = {Rs...};
    static constexpr int N = (Rs * ... * 1);
    static constexpr int ns(int s)
    {
        int p = 1;
        for (int i = 0; i < s; i++) p *= r[i];
        return p;
    }
    // offset of stage s's twiddle table (stage 0 needs none)
    static constexpr int tw_off(int s)
    {
        int o = 0;
        for (int i = 1; i < s; i++) o += (r[i] - 1) * ns(i);
        return o;
    }
};

template <class Q, int T>
constexpr int static_maxv()
{
    int m = 0;
    for (int s = 0; s < Q::S; s++) {
        const int nbf = Q::N / Q::r[s];
        const int nb = (nbf + T - 1) / T;
        m = m > nb * Q::r[s] ? m : nb * Q::r[s];
    }
    return m;
}

template <class Q, int S, int T, bool FWD, class Src>
__device__ __forceinline__ void sgather(float2 *v, const Src &src, int lane, bool active,
                                        const float2 *__restrict__ stw)
{
    constexpr int R = Q::r[S], N = Q::N, NS = Q::ns(S), NBF = N / R, NB = (NBF + T - 1) / T;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = lane + b * T;
        if (active && (NBF % T == 0 || j < NBF)) {
#pragma unroll
            for (int r = 0; r < R; r++) v[b * R + r] = src(j + r * NBF);
        }
    }
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = lane + b * T;
        if (active && (NBF % T == 0 || j < NBF)) {
            if constexpr (S > 0) {
                const float2 *t = stw + Q::tw_off(S) + (j % NS);
#pragma unroll
                for (int r = 1; r < R; r++) v[b * R + r] = cmul(v[b * R + r], dir<FWD>(__ldg(t + (r - 1) * NS)));
            }
            dft<R, FWD>(v + b * R);
        }
    }
}

template <class Q, int S, int T, class Dst>
__device__ __forceinline__ void sscatter(const float2 *v, const Dst &dst, int lane, bool active)
{
    constexpr int R = Q::r[S], N = Q::N, NS = Q::ns(S), NBF = N / R, NB = (NBF + T - 1) / T;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = lane + b * T;
        if (active && (NBF % T == 0 || j < NBF)) {
            const int k = j % NS;
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) dst(base + r * NS, v[b * R + r]);
        }
    }
}

// Stage S of the static FFT; stage 0 reads src0 (the staging rows, which
// alias the work buffer), the last stage writes dstL.
template <class Q, int T, bool FWD, int S, class Src0, class DstL>
__device__ __forceinline__ void srun(float2 *v, float2 *work, const Src0 &src0, const DstL &dstL, bool dst_in_place,
                                     int lane, bool active, const float2 *stw)
{
    constexpr bool last = S == Q::S - 1;
    const SmemRow w{work};
    if constexpr (S == 0)
        sgather<Q, 0, T, FWD>(v, src0, lane, active, stw);
    else
        sgather<Q, S, T, FWD>(v, w, lane, active, stw);
    if (!last || dst_in_place) __syncthreads();
    if constexpr (last) {
        sscatter<Q, S, T>(v, dstL, lane, active);
    } else {
        sscatter<Q, S, T>(v, w, lane, active);
        __syncthreads();
        srun<Q, T, FWD, S + 1>(v, work, src0, dstL, dst_in_place, lane, active, stw);
    }
}

// Up to 256 threads per CTA the engines are compiled for three resident CTAs
// per SM (at most 85 registers per thread: the codelets fit without
// spilling), which doubles the warps available to hide shared-memory and
// twiddle-load latency compared with an unconstrained build.
template <class Q, int T, bool FWD>
struct FusedR2C {
    static constexpr int S = Q::S - 1;
    static constexpr int R = Q::r[S], N = Q::N, NS = Q::ns(S), NBF = N / R;
    static constexpr bool ok = Q::S >= 2 && NBF % 2 == 0 && T == NBF / 2;

    __device__ __forceinline__ static void run(float2 *v, const float2 *work, float2 *y, int lane, bool active,
                                               const float2 *__restrict__ stw, const float2 *__restrict__ tw)
    {
        const int j0 = lane, j1 = lane == 0 ? NBF / 2 : NBF - lane;
        if (active) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                v[r] = work[pad(j0 + r * NBF)];
                v[R + r] = work[pad(j1 + r * NBF)];
            }
            const float2 *t0 = stw + Q::tw_off(S) + j0;
            const float2 *t1 = stw + Q::tw_off(S) + j1;
#pragma unroll
            for (int r = 1; r < R; r++) {
                v[r] = cmul(v[r], dir<FWD>(__ldg(t0 + (r - 1) * NS)));
                v[R + r] = cmul(v[R + r], dir<FWD>(__ldg(t1 + (r - 1) * NS)));
            }
            dft<R, FWD>(v);
            dft<R, FWD>(v + R);
            float2 a, b;
            if (lane != 0) {
                // bin j0 + r NBF pairs with its mirror j1 + (R-1-r) NBF
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const int k0 = j0 + r * NBF;
                    r2c_pair(v[r], v[2 * R - 1 - r], dir<FWD>(__ldg(tw + k0)), a, b);
                    y[k0] = a;
                    y[j1 + (R - 1 - r) * NBF] = b;
                }
            } else {
                // bins r NBF pair with (R-r) NBF (r = 0: with the Nyquist bin N),
                // bins NBF/2 + r NBF with NBF/2 + (R-1-r) NBF
#pragma unroll
                for (int r = 0; 2 * r <= R; r++) {
                    r2c_pair(v[r], v[(R - r) % R], dir<FWD>(__ldg(tw + r * NBF)), a, b);
                    y[r * NBF] = a;
                    if (2 * r != R) y[N - r * NBF] = b;
                }
#pragma unroll
                for (int r = 0; 2 * r < R; r++) {
                    const int k = NBF / 2 + r * NBF;
                    r2c_pair(v[R + r], v[2 * R - 1 - r], dir<FWD>(__ldg(tw + k)), a, b);
                    y[k] = a;
                    if (2 * r != R - 1) y[N - k] = b;
                }
            }
        }
    }
};

template <class Q, int T>
struct StaticEngine {
    static constexpr int kMaxThreads = T <= 256 ? 256 : T;
    // 3 CTAs per SM (<= 80 registers) unless a thread holds more than 16 points
    static constexpr int kMinBlocks = T <= 256 ? (Q::N / T > 16 ? 2 : 3) : 1;
    template <bool FWD, class Src0, class DstL>
    __device__ __forceinline__ static void run(const TileDesc &d, float2 *work, const Src0 &src0, const DstL &dstL,
                                               bool dst_in_place, int lane, bool active)
    {
        float2 v[static_maxv<Q, T>()];
        srun<Q, T, FWD, 0>(v, work, src0, dstL, dst_in_place, lane, active, d.stw);
    }

    template <bool FWD, class Src0>
    __device__ __forceinline__ static void run_r2c(const TileDesc &d, float2 *work, const Src0 &src0, float2 *y,
                                                   int lane, bool active)
    {
        using F = FusedR2C<Q, T, FWD>;
        if constexpr (F::ok) {
            constexpr int V = static_maxv<Q, T>() > 2 * F::R ? static_maxv<Q, T>() : 2 * F::R;
            float2 v[V];
            srun_prefix<FWD>(v, work, src0, lane, active, d.stw);
            __syncthreads();
            F::run(v, work, y, lane, active, d.stw, d.tw);
        } else {
            run<FWD>(d, work, src0, SmemRow{work}, true, lane, active);
            __syncthreads();
            if (active) r2c_post_row<FWD>(work, y, d.n, lane, d.tpt, d.tw);
        }
    }

    // every stage but the last, leaving the data in the padded work row
    template <bool FWD, class Src0>
    __device__ __forceinline__ static void srun_prefix(float2 *v, float2 *work, const Src0 &src0, int lane,
                                                       bool active, const float2 *stw)
    {
        prefix<FWD, 0>(v, work, src0, lane, active, stw);
    }
    template <bool FWD, int S, class Src0>
    __device__ __forceinline__ static void prefix(float2 *v, float2 *work, const Src0 &src0, int lane, bool active,
                                                  const float2 *stw)
    {
        if constexpr (S < Q::S - 1) {
            const SmemRow w{work};
            if constexpr (S == 0)
                sgather<Q, 0, T, FWD>(v, src0, lane, active, stw);
            else
                sgather<Q, S, T, FWD>(v, w, lane, active, stw);
            __syncthreads();
            sscatter<Q, S, T>(v, w, lane, active);
            if constexpr (S + 1 < Q::S - 1) __syncthreads();
            prefix<FWD, S + 1>(v, work, src0, lane, active, stw);
        }
    }
};

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
            const int64_t kc = (c0 + (thread_on ? l : 0)) % d.g_ns;
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

template <class Q, int T>
StaticKernel make_entry(int io_mask = 7)
{
    StaticKernel e{};
    e.io_mask = io_mask;
    e.n = Q::N;
    e.nstages = Q::S;
    for (int s = 0; s < Q::S; s++) e.radix[s] = Q::r[s];
    e.tpt = T;
    using E = StaticEngine<Q, T>;
    e.fn[1][0] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, true, IO_C2C>);
    e.fn[1][1] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, true, IO_R2C_PACKED>);
    e.fn[1][2] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, true, IO_C2R_PACKED>);
    e.fn[0][0] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, false, IO_C2C>);
    e.fn[0][1] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, false, IO_R2C_PACKED>);
    e.fn[0][2] = reinterpret_cast<const void *>(pipelined_rows_kernel<E, false, IO_C2R_PACKED>);
    e.db[1] = reinterpret_cast<const void *>(static_db_kernel<E, true>);
    e.db[0] = reinterpret_cast<const void *>(static_db_kernel<E, false>);
    return e;
}

const std::vector<StaticKernel> &registry()
{
    static const std::vector<StaticKernel> r = {
        make_entry<Seq<16, 4>, 4>(),            // 64
        make_entry<Seq<16, 8>, 8>(),            // 128
        make_entry<Seq<16, 16>, 16>(),          // 256
        make_entry<Seq<16, 16, 2>, 32>(),       // 512
        make_entry<Seq<16, 16, 4>, 64>(),       // 1024
        make_entry<Seq<16, 16, 8>, 128>(),      // 2048
        make_entry<Seq<16, 16, 16>, 256>(),     // 4096
        make_entry<Seq<16, 16, 16, 2>, 512>(),  // 8192
        // 1500, the packed half of the 3000-point real transform: R2C on a
        // radix-5 last stage of 300 butterflies, two per thread, so that the
        // post-twiddle fuses into it; C2C and C2R on 10 x 10 x 15, one
        // butterfly per thread in the radix-10 stages
        make_entry<Seq<12, 5, 5, 5>, 150>(4),
        make_entry<Seq<10, 10, 15>, 150>(3),
    };
    return r;
}

}  // namespace

void static_kernel_fns(std::vector<const void *> &out)
{
    for (const StaticKernel &e : registry())
        for (int f = 0; f < 2; f++) {
            for (int io = 0; io < 3; io++) out.push_back(e.fn[f][io]);
            out.push_back(e.db[f]);
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
