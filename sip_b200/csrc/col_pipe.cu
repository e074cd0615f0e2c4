// TMA-pipelined persistent kernel for strided axes: the column pass of 2D /
// 3D plans, vertical 1D, and every pass of a multi-pass (long) transform.
//
// A tile is TB adjacent transforms of a strided axis, i.e. TB adjacent
// columns of an [outer][n][cols] array.  The tensor-memory-access engine
// copies it into shared memory as 3D boxes of TB columns x up to 256 rows
// (one rectangular copy per 256 rows, issued by one thread and completed on
// an mbarrier), double-buffered so that the next tile streams in while the
// current one is transformed.  The first Stockham stage reads the staged rows
// column by column (applying a multi-pass step's inter-pass twiddles), the
// stages run in the padded work rows that overwrite the staging buffer, and
// the last stage stores straight from registers to HBM (TB consecutive threads
// write TB consecutive columns of one row).  The reference runs this axis as
// a transpose plus a DFT-matrix GEMM (core/fft/fftcore/fft_core_stride.cpp:36-188,
// ops/fft/c2c/fft_stride/fft_stride/kernel/fft_stride.cce) or as explicit
// Transpose steps around the row cores (core/fft/fft_api.cpp:527-697).
//
// Launch preconditions (the planner checks them, the exec path re-checks the
// pointer): source 16-byte aligned, column stride 1, element and outer
// strides multiples of 2 complex values (16 bytes), TB even.
#include <cuda.h>

#include "sipfft_internal.h"
#include "static_engine.cuh"

namespace sipfft {

namespace {

// 3D tiled bulk-tensor load of box {x: columns, y: rows, z: outer} into shared memory
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// element e of column l of the staged tile ([row][TB] dense), with the
// inter-pass twiddle of a multi-pass step applied on read
template <int TB, bool FWD>
struct ColStage {
    const float2 *tile;
    int l;
    const TileDesc *d;
    int64_t kc;  // Stockham column of the pass twiddle, < 0 for none
    __device__ __forceinline__ float2 operator()(int e) const
    {
        const float2 v = tile[e * TB + l];
        return kc >= 0 ? cmul(v, pass_twiddle<FWD>(*d, e, kc)) : v;
    }
};

struct ColOut {
    float2 *col;
    int64_t es;
    __device__ __forceinline__ void operator()(int e, float2 v) const { st_stream(col + e * es, v); }
};

}  // namespace

// PP: a third shared-memory buffer holds the even stage boundaries (ping-pong
// work rows), so stage 0 scatters outside the staged tile and no stage needs a
// barrier between its gather and its scatter.
// COUT: each column's N outputs are contiguous (output element stride 1, the
// first pass of a multi-pass transform): the last stage writes the work rows and
// the CTA then stores whole column runs, a warp 32 consecutive elements instead
// of 16 columns x 2.
template <class Q, int T, int TB, bool PP, bool COUT, bool FWD>
__global__ void __launch_bounds__(TB *T, (TB * T <= 256) ? 3 : 1)
    col_pipe_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ TileDesc d, int *err)
{
    pdl_enter();
    using E = StaticEngine<Q, T, Pads<>, PP>;
    constexpr int N = Q::N;
    constexpr int BOX = N < 256 ? N : 256;
    constexpr int NBOX = N / BOX;
    constexpr uint32_t kTileBytes = uint32_t(TB) * N * sizeof(float2);
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smraw);
    float2 *bufs = reinterpret_cast<float2 *>(smraw + 128);
    const int64_t buf_f2 = d.col_buf;  // per-buffer float2 count (planner-computed)
    const int tid = threadIdx.x;
    const int l = tid % TB, lane = tid / TB;
    float2 *out = static_cast<float2 *>(d.out);
    __shared__ int64_t s_base[COUT ? TB : 1];  // output offsets of the tile's columns (COUT)

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](int64_t t, int b) {
        if (tid == 0) {
            const int o = static_cast<int>(t / d.tiles_per_outer);
            const int c0 = static_cast<int>((t % d.tiles_per_outer) * TB);
            float2 *dst = bufs + b * buf_f2;
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&bars[b], kTileBytes);
#pragma unroll
            for (int k = 0; k < NBOX; k++) tma_load_3d(dst + k * BOX * TB, &tmap, c0, k * BOX, o, &bars[b]);
        }
    };

    int64_t t = blockIdx.x;
    if (t < d.num_tiles) issue(t, 0);
    for (int i = 0; t < d.num_tiles; t += gridDim.x, i++) {
        const int b = i & 1;
        const int64_t tn = t + gridDim.x;
        if (tn < d.num_tiles) issue(tn, b ^ 1);
        // a thread whose bounded wait gave up still runs the tile (every access
        // stays in bounds) and the CTA leaves together at the end of the iteration
        const bool timed_out = !mbar_wait_bounded(&bars[b], (i >> 1) & 1);
        if (timed_out) atomicExch(err, 1);
        const int64_t o = t / d.tiles_per_outer;
        const int64_t c0 = (t % d.tiles_per_outer) * TB;
        const int64_t left = d.n_cols - c0;
        const bool active = l < left;
        float2 *buf = bufs + b * buf_f2;
        float2 *work2 = PP ? bufs + 2 * buf_f2 + l * d.pitch : nullptr;
        const int64_t kc = d.g_twiddle ? pass_column(d, c0 + l) : -1;
        if constexpr (COUT) {
            if (tid < TB) s_base[tid] = col_base(d.out_a, o, c0 + tid);
            E::template run<FWD>(d, buf + l * d.pitch, ColStage<TB, FWD>{buf, l, &d, kc}, SmemRow{buf + l * d.pitch},
                                 true, lane, active, work2);
            __syncthreads();
            const int cols = left < TB ? static_cast<int>(left) : TB;
            for (int c = 0; c < cols; c++) {
                float2 *dst = out + s_base[c];
                const float2 *src = buf + c * d.pitch;
                for (int e = tid; e < N; e += TB * T) st_stream(dst + e, src[pad(e)]);
            }
        } else {
            E::template run<FWD>(d, buf + l * d.pitch, ColStage<TB, FWD>{buf, l, &d, kc},
                                 ColOut{out + col_base(d.out_a, o, c0 + l), d.out_a.estride}, false, lane, active,
                                 work2);
        }
        // buffer b is free for the copy issued in iteration i+1; a CTA-uniform exit after a timeout
        if (__syncthreads_or(timed_out)) return;
    }
}

// ------------------------------------------------------------------------------------ host side
namespace {

struct ColPipeEntry {
    int n, tpt, tb, bufs;  // bufs: shared-memory buffers of col_buf float2 each (3: ping-pong work rows)
    const void *fn[2][2];  // [contiguous column outputs][forward]
};

template <class Q, int T, int TB, bool PP = false>
ColPipeEntry col_entry()
{
    static_assert(TB % 2 == 0 && TB * T <= 512, "column tile shape");
    ColPipeEntry e{Q::N, T, TB, PP ? 3 : 2,
                   {{reinterpret_cast<const void *>(col_pipe_kernel<Q, T, TB, PP, false, false>),
                     reinterpret_cast<const void *>(col_pipe_kernel<Q, T, TB, PP, false, true>)},
                    {nullptr, nullptr}}};
    // staged contiguous-column stores pay off where a warp's direct stores would
    // cover less than a 32-byte sector of each column (TB >= 16: two lanes, 16 bytes)
    if constexpr (TB >= 16) {
        e.fn[1][0] = reinterpret_cast<const void *>(col_pipe_kernel<Q, T, TB, PP, true, false>);
        e.fn[1][1] = reinterpret_cast<const void *>(col_pipe_kernel<Q, T, TB, PP, true, true>);
    }
    return e;
}

// Engines with 16 points per thread (the same radix sequences as the
// power-of-two row engines); TB columns per tile as the planner chooses them
// (CTAs of at most 256 threads, three per SM, while TB stays >= 4, i.e. rows
// of at least one 32-byte sector; 512 threads for 2048 points, one CTA per SM,
// whose shared memory also holds the ping-pong work rows).
const std::vector<ColPipeEntry> &col_registry()
{
    static const std::vector<ColPipeEntry> r = {
        col_entry<Seq<16, 4>, 4, 16>(),     col_entry<Seq<16, 8>, 8, 16>(),   col_entry<Seq<16, 16>, 16, 16>(),
        col_entry<Seq<16, 16, 2>, 32, 8>(), col_entry<Seq<16, 16, 4>, 64, 4>(), col_entry<Seq<16, 16, 8>, 128, 4, true>(),
    };
    return r;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<EncodeTiledFn>(nullptr);
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

}  // namespace

const void *col_pipe_kernel_fn(int n, int tpt, int tb, bool forward, bool contiguous_out)
{
    for (const ColPipeEntry &e : col_registry())
        if (e.n == n && e.tpt == tpt && e.tb == tb) {
            const int f = forward ? 1 : 0;
            return contiguous_out && e.fn[1][f] ? e.fn[1][f] : e.fn[0][f];
        }
    return nullptr;
}

int col_pipe_bufs(int n, int tpt, int tb)
{
    for (const ColPipeEntry &e : col_registry())
        if (e.n == n && e.tpt == tpt && e.tb == tb) return e.bufs;
    return 2;
}

bool col_pipe_has_engine(int n)
{
    for (const ColPipeEntry &e : col_registry())
        if (e.n == n) return true;
    return false;
}

void col_pipe_kernel_fns(std::vector<const void *> &out)
{
    for (const ColPipeEntry &e : col_registry())
        for (int c = 0; c < 2; c++)
            for (int f = 0; f < 2; f++)
                if (e.fn[c][f]) out.push_back(e.fn[c][f]);
}

size_t col_pipe_smem(const TileDesc &d)
{
    return 128 + (d.row_bufs == 3 ? 3 : 2) * static_cast<size_t>(d.col_buf) * sizeof(float2);
}

bool col_pipe_layout_ok(const TileDesc &d)
{
    const Addr &a = d.in_a;
    return d.tb % 2 == 0 && d.n_cols >= d.tb && a.cstride == 1 && a.cblock == 0 && a.estride % 2 == 0 && a.estride > 0 &&
           (d.n_outer == 1 || a.dist % 2 == 0) && d.n_outer < (int64_t(1) << 31) &&
           d.tiles_per_outer * d.tb < (int64_t(1) << 31) && encode_fn() != nullptr;
}

cudaError_t launch_col_pipe(const void *fn, const TileDesc &d, int grid, int *err, cudaStream_t st)
{
    if (!fn || grid <= 0 || (reinterpret_cast<uintptr_t>(d.in) & 15)) return cudaErrorInvalidConfiguration;
    EncodeTiledFn enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const int n = d.n;
    const int box_rows = n < 256 ? n : 256;
    CUtensorMap map;
    // complex64 elements moved as opaque 8-byte words
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(d.n_cols), static_cast<cuuint64_t>(n),
                                static_cast<cuuint64_t>(d.n_outer)};
    const int64_t outer_stride = d.n_outer > 1 ? d.in_a.dist : d.in_a.estride * n + (d.in_a.estride * n) % 2;
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(d.in_a.estride) * 8,
                                   static_cast<cuuint64_t>(outer_stride) * 8};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(d.tb), static_cast<cuuint32_t>(box_rows), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(d.in), dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    TileDesc dd = d;
    void *args[] = {&map, &dd, &err};
    return launch_pdl(fn, dim3(grid), dim3(d.tb * d.tpt), col_pipe_smem(d), st, args);
}

}  // namespace sipfft
