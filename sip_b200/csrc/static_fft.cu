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
template <class Q, int T>
struct StaticEngine {
    static constexpr int kMaxThreads = T <= 256 ? 256 : T;
    static constexpr int kMinBlocks = T <= 256 ? 3 : 1;
    template <bool FWD, class Src0, class DstL>
    __device__ __forceinline__ static void run(const TileDesc &d, float2 *work, const Src0 &src0, const DstL &dstL,
                                               bool dst_in_place, int lane, bool active)
    {
        float2 v[static_maxv<Q, T>()];
        srun<Q, T, FWD, 0>(v, work, src0, dstL, dst_in_place, lane, active, d.stw);
    }
};

// ------------------------------------------------------------------------------------ registry
namespace {

template <class Q, int T>
StaticKernel make_entry()
{
    StaticKernel e{};
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
        make_entry<Seq<10, 10, 15>, 100>(),     // 1500 (packed half of the 3000-point real transform)
    };
    return r;
}

}  // namespace

const StaticKernel *find_static_kernel(int n)
{
    for (const StaticKernel &e : registry())
        if (e.n == n) return &e;
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
