// Compile-time specialised FFT engines (static radix sequences), shared by
// the row kernels (static_fft.cu) and the TMA column kernels (col_pipe.cu).
//
// For a length whose radix sequence and threads per transform are fixed at
// compile time, every stage's butterfly count, Ns, (j mod Ns), padded
// shared-memory address and twiddle-table offset folds into constants, loops
// unroll completely, and the stage twiddles come from per-stage tables laid
// out [r-1][k] so that the 32 lanes of a warp read consecutive entries.
#pragma once
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

// Shared-memory layout of the work row between stage b and stage b+1 of a
// static engine: element i at i + Q_b * (i / P_b), P_b = 0 for unpadded.
// Chosen per engine (and per boundary) so that the scatter of stage b and the
// gather of stage b+1 touch few bank-conflicting words; the default is the
// i + i/16 layout of the runtime engine and of the tile IO, which the first
// read and the last write of every engine keep.
template <int... QP>
struct Pads {
    static constexpr int n = sizeof...(QP) / 2;
    static constexpr int q(int b)
    {
        constexpr int a[] = {QP..., 0};
        return b < n ? a[2 * b] : 1;
    }
    static constexpr int p(int b)
    {
        constexpr int a[] = {QP..., 0};
        return b < n ? a[2 * b + 1] : 16;
    }
};

template <int QQ, int PP>
struct PadRow {
    float2 *row;
    __device__ __forceinline__ static int at(int i)
    {
        if constexpr (PP == 0)
            return i;
        else
            return i + QQ * static_cast<int>(static_cast<unsigned>(i) / PP);
    }
    __device__ __forceinline__ float2 operator()(int e) const { return row[at(e)]; }
    __device__ __forceinline__ void operator()(int e, float2 v) const { row[at(e)] = v; }
};

template <class PD, int B>
using BoundaryRow = PadRow<PD::q(B), PD::p(B)>;

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

// Stage-0 element e = j + off of a butterfly's source: plain sources take
// e; the C2R pre-twiddle splits its twiddle as tw[j] * tw[off] (one entry per
// butterfly and one shared by every lane) so that the lines of the
// half-length table a CTA keeps in L1 shrink to NBF entries (used from 2048
// points, where the whole table no longer fits next to the stage tables).
template <class Src>
__device__ __forceinline__ float2 fetch(const Src &src, int j, int off)
{
    return src(j + off);
}
template <bool FWD>
__device__ __forceinline__ float2 fetch(const C2RPre<FWD> &src, int j, int off)
{
    return src.split(j, off);
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
            for (int r = 0; r < R; r++) {
                if constexpr (N >= 2048)
                    v[b * R + r] = fetch(src, j, r * NBF);
                else
                    v[b * R + r] = src(j + r * NBF);
            }
        }
    }
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = lane + b * T;
        if (active && (NBF % T == 0 || j < NBF)) {
            if constexpr (S > 0) {
                const float2 *t = stw + Q::tw_off(S) + (j % NS);
                if constexpr ((R == 8 || R == 16) && NS >= 128) {
                    // long stage tables: rows 1, 2, 4 (8) of w^r are read and the
                    // other powers formed as products (at most three deep), so
                    // that log2 R rows rather than R-1 stay resident in L1
                    float2 w[R];
                    w[1] = __ldg(t);
                    w[2] = __ldg(t + NS);
                    w[4] = __ldg(t + 3 * NS);
                    w[3] = cmul(w[1], w[2]);
                    w[5] = cmul(w[1], w[4]);
                    w[6] = cmul(w[2], w[4]);
                    w[7] = cmul(w[3], w[4]);
                    if constexpr (R == 16) {
                        w[8] = __ldg(t + 7 * NS);
#pragma unroll
                        for (int r = 1; r < 8; r++) w[8 + r] = cmul(w[r], w[8]);
                    }
#pragma unroll
                    for (int r = 1; r < R; r++) v[b * R + r] = cmul(v[b * R + r], dir<FWD>(w[r]));
                } else {
#pragma unroll
                    for (int r = 1; r < R; r++)
                        v[b * R + r] = cmul(v[b * R + r], dir<FWD>(__ldg(t + (r - 1) * NS)));
                }
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

// Work row of boundary b (the layout stage b writes and stage b+1 reads).
// With a ping-pong area (PP) even boundaries live in work2 and odd ones in
// work, so that no stage scatters over the row it gathers from and the
// barrier between a stage's gather and its scatter goes away.
template <bool PP, int B>
__device__ __forceinline__ float2 *bbuf(float2 *work, float2 *work2)
{
    return (PP && B % 2 == 0) ? work2 : work;
}

// Barrier between two steps that touch only the work rows of the CTA's own
// transforms.  With warp-local lanes (WL: the T <= 32 threads of a transform
// are consecutive lanes of one warp, as in the row kernels) a transform's
// work row is written and read by its own warp only, so the warp's barrier
// suffices; stage 0's gather still ends with a CTA barrier, because the
// staged input rows alias the work rows of other warps' transforms.
template <int WL>
__device__ __forceinline__ void row_sync()
{
    if constexpr (WL > 0)
        __syncwarp();
    else
        __syncthreads();
}

// Last stage of radix 2 as warp-shuffle butterflies.  When stage S-2 has one
// butterfly per thread and T = 2 Ns(S-2) <= 32 (warp-local lanes), element
// j < N/2 of the last boundary sits in register j / H of lane j mod H and
// element j + N/2 in the same register of lane H + j mod H (H = T/2), so the
// butterfly X[j] = a + w^j b, X[j + N/2] = a - w^j b pairs lanes (lane,
// lane ^ H) register by register.  Every lane multiplies its operand by a
// stage-table entry (w^j in the upper lane, entry 0 = 1 in the lower one, so
// both run the same instructions), swaps the product with its partner and
// keeps one output: lower a + w^j b, upper a - w^j b.  The stage needs no
// shared memory and no barrier; stores of one register cover two runs of H
// consecutive bins.
template <class Q, int T, int WL>
struct ShflLast {
    static constexpr bool ok =
        WL == 2 && Q::S >= 2 && Q::r[Q::S - 1] == 2 && T == 2 * Q::ns(Q::S - 2) && Q::N / Q::r[Q::S - 2] == T;
};

template <class Q, int T, bool FWD, class DstL>
__device__ __forceinline__ void shfl_last(const float2 *v, const DstL &dst, int lane, bool active,
                                          const float2 *__restrict__ stw)
{
    constexpr int S = Q::S - 1, RP = Q::r[S - 1], H = T / 2, HALF = Q::N / 2;
    const bool up = (lane & H) != 0;
    const int lo = lane & (H - 1);
    const int sel = up ? -1 : 0;
    const float sg = up ? -1.f : 1.f;
    const float2 *t = stw + Q::tw_off(S);
#pragma unroll
    for (int r = 0; r < RP; r++) {
        const int j = lo + r * H;
        const float2 q = cmul(v[r], dir<FWD>(__ldg(t + (j & sel))));
        const float px = __shfl_xor_sync(0xffffffffu, q.x, H);
        const float py = __shfl_xor_sync(0xffffffffu, q.y, H);
        if (active) dst(j + (up ? HALF : 0), make_float2(fmaf(sg, q.x, px), fmaf(sg, q.y, py)));
    }
}

// Stage S of the static FFT; stage 0 reads src0 (the staging rows, which
// alias the work buffer), the last stage writes dstL.
template <class Q, int T, class PD, bool PP, int WL, bool FWD, int S, class Src0, class DstL>
__device__ __forceinline__ void srun(float2 *v, float2 *work, float2 *work2, const Src0 &src0, const DstL &dstL,
                                     bool dst_in_place, int lane, bool active, const float2 *stw)
{
    constexpr bool shfl = ShflLast<Q, T, WL>::ok && S == Q::S - 2;
    constexpr bool last = S == Q::S - 1 || shfl;
    if constexpr (S == 0)
        sgather<Q, 0, T, FWD>(v, src0, lane, active, stw);
    else
        sgather<Q, S, T, FWD>(v, BoundaryRow<PD, S - 1>{bbuf<PP, S - 1>(work, work2)}, lane, active, stw);
    if constexpr (last) {
        // an in-place destination is the work row: wait while it is still gathered from
        constexpr bool src_is_work = S == 0 || !(PP && (S - 1) % 2 == 0);
        if (dst_in_place && src_is_work) {
            if constexpr (S == 0)
                __syncthreads();
            else
                row_sync<WL>();
        }
        if constexpr (shfl)
            shfl_last<Q, T, FWD>(v, dstL, lane, active, stw);
        else
            sscatter<Q, S, T>(v, dstL, lane, active);
    } else {
        if constexpr (!PP) {
            if constexpr (S == 0)
                __syncthreads();
            else
                row_sync<WL>();
        }
        sscatter<Q, S, T>(v, BoundaryRow<PD, S>{bbuf<PP, S>(work, work2)}, lane, active);
        row_sync<WL>();
        srun<Q, T, PD, PP, WL, FWD, S + 1>(v, work, work2, src0, dstL, dst_in_place, lane, active, stw);
    }
}

// Up to 256 threads per CTA the engines are compiled for three resident CTAs
// per SM (at most 85 registers per thread: the codelets fit without
// spilling), which doubles the warps available to hide shared-memory and
// twiddle-load latency compared with an unconstrained build.
template <class Q, int T, class PD, bool FWD>
struct FusedR2C {
    static constexpr int S = Q::S - 1;
    static constexpr int R = Q::r[S], N = Q::N, NS = Q::ns(S), NBF = N / R;
    static constexpr bool ok = Q::S >= 2 && NBF % 2 == 0 && T == NBF / 2;

    __device__ __forceinline__ static void run(float2 *v, const float2 *work, float2 *y, int lane, bool active,
                                               const float2 *__restrict__ stw, const float2 *__restrict__ tw)
    {
        const int j0 = lane, j1 = lane == 0 ? NBF / 2 : NBF - lane;
        if (active) {
            const BoundaryRow<PD, S - 1> w{const_cast<float2 *>(work)};
#pragma unroll
            for (int r = 0; r < R; r++) {
                v[r] = w(j0 + r * NBF);
                v[R + r] = w(j1 + r * NBF);
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
            // Post twiddles w^(j + r NBF) = w^j w^(r NBF): one table entry per
            // butterfly and R entries shared by every lane.  Lane 0 owns the
            // self-mirrored butterflies 0 and NBF/2, whose bins pair within each
            // butterfly.
            if constexpr (R % 2 == 0)
                post_selected(v, y, lane, j0, j1, tw);
            else
                post_branched(v, y, lane, j0, j1, tw);
        }
    }

    // Lane 0 moves its values into the slots where the common loop over pairs
    // (u[r], u[2R-1-r]) meets its pairs and selects its bins and twiddles
    // (no branch of its own, which would put extra work on one warp
    // scheduler): iterations r < G pair bins NBF/2 + r NBF and
    // NBF/2 + (R-1-r) NBF, iterations r >= G pair p NBF and (R-p) NBF
    // (p = r - G + 1), and bins 0 and N follow from Z[0] alone.
    __device__ __forceinline__ static void post_selected(const float2 *v, float2 *y, int lane, int j0, int j1,
                                                         const float2 *__restrict__ tw)
    {
        constexpr int G = (R + 1) / 2;
        const bool z = lane == 0;
        float2 u[2 * R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            if (r < G) {
                u[r] = z ? v[R + r] : v[r];
                u[2 * R - 1 - r] = v[2 * R - 1 - r];
            } else {
                const int p = r - G + 1;
                u[r] = z ? v[p] : v[r];
                u[2 * R - 1 - r] = z ? v[R - p] : v[2 * R - 1 - r];
            }
        }
        const int a0 = z ? NBF / 2 : j0;
        const float2 wa = __ldg(tw + a0);
        const float2 wb = z ? make_float2(1.f, 0.f) : wa;
        float2 a, b;
#pragma unroll
        for (int r = 0; r < R; r++) {
            int o1, o2;
            float2 w;
            if (r < G) {
                o1 = a0 + r * NBF;
                o2 = j1 + (R - 1 - r) * NBF;
                w = r == 0 ? wa : cmul(wa, __ldg(tw + r * NBF));
            } else {
                const int p = r - G + 1;
                o1 = z ? p * NBF : j0 + r * NBF;
                o2 = z ? (R - p) * NBF : j1 + (R - 1 - r) * NBF;
                w = cmul(wb, __ldg(tw + (z ? p : r) * NBF));
            }
            r2c_pair(u[r], u[2 * R - 1 - r], dir<FWD>(w), a, b);
            st_stream(y + o1, a);
            st_stream(y + o2, b);
        }
        if (z) {
            r2c_pair(v[0], v[0], make_float2(1.f, 0.f), a, b);
            st_stream(y, a);
            st_stream(y + N, b);
        }
    }

    // Lane 0 in a branch of its own (odd radices, where the selected form
    // spills registers).
    __device__ __forceinline__ static void post_branched(const float2 *v, float2 *y, int lane, int j0, int j1,
                                                         const float2 *__restrict__ tw)
    {
        float2 a, b;
        if (lane != 0) {
            // bin j0 + r NBF pairs with its mirror j1 + (R-1-r) NBF
            const float2 w0 = __ldg(tw + j0);
#pragma unroll
            for (int r = 0; r < R; r++) {
                const float2 w = r == 0 ? w0 : cmul(w0, __ldg(tw + r * NBF));
                r2c_pair(v[r], v[2 * R - 1 - r], dir<FWD>(w), a, b);
                st_stream(y + j0 + r * NBF, a);
                st_stream(y + j1 + (R - 1 - r) * NBF, b);
            }
        } else {
            // bins r NBF pair with (R-r) NBF (r = 0: with the Nyquist bin N),
            // bins NBF/2 + r NBF with NBF/2 + (R-1-r) NBF
#pragma unroll
            for (int r = 0; 2 * r <= R; r++) {
                r2c_pair(v[r], v[(R - r) % R], dir<FWD>(__ldg(tw + r * NBF)), a, b);
                st_stream(y + r * NBF, a);
                if (2 * r != R) st_stream(y + N - r * NBF, b);
            }
            const float2 wh = __ldg(tw + NBF / 2);
#pragma unroll
            for (int r = 0; 2 * r < R; r++) {
                const int k = NBF / 2 + r * NBF;
                const float2 w = r == 0 ? wh : cmul(wh, __ldg(tw + r * NBF));
                r2c_pair(v[R + r], v[2 * R - 1 - r], dir<FWD>(w), a, b);
                st_stream(y + k, a);
                if (2 * r != R - 1) st_stream(y + N - k, b);
            }
        }
    }
};

// First stage of a C2R transform with the pre-twiddle fused: the thread owns
// butterflies j0 = lane and j1 = NBF - lane, so the inputs X[e], X[m-e] it
// reads give two of its own packed inputs, Z[e] = E + i O and
// Z[m-e] = conj(E) + i conj(O) (E = X[e] + conj X[m-e],
// O = w^e (X[e] - conj X[m-e])), one twiddle per pair.  Lane 0 owns the
// self-mirrored butterflies 0 and NBF/2 and, as in FusedR2C, runs the common
// loop with its inputs and twiddles selected, then moves the results into
// butterfly order; Z[0] (DC and Nyquist, imaginary parts ignored) follows alone.
template <class Q, int T, bool FWD>
struct FusedC2R {
    static constexpr int R = Q::r[0], N = Q::N, NBF = N / R, G = (R + 1) / 2;
    static constexpr bool ok = Q::S >= 2 && NBF % 2 == 0 && T == NBF / 2;

    __device__ __forceinline__ static void pair(float2 xk, float2 xm, float2 w, float2 &ze, float2 &zm)
    {
        const float2 ev = make_float2(xk.x + xm.x, xk.y - xm.y);
        const float2 od = cmul(make_float2(xk.x - xm.x, xk.y + xm.y), w);
        ze = make_float2(ev.x - od.y, ev.y + od.x);
        zm = make_float2(ev.x + od.y, od.x - ev.y);
    }

    // slot of the loop's results that lane 0 keeps in register k (k > 0)
    static constexpr int lane0_slot(int k)
    {
        if (k >= R) return k - R < G ? k - R : k;
        return k <= R - G ? G - 1 + k : R - G + k;
    }

    // x: staged half spectrum (N+1 bins); v[0..R) = butterfly j0, v[R..2R) = j1
    __device__ __forceinline__ static void gather(float2 *v, const float2 *x, int lane,
                                                  const float2 *__restrict__ tw)
    {
        const bool z = lane == 0;
        const int j0 = lane;
        const int a0 = z ? NBF / 2 : j0;
        const float2 wa = __ldg(tw + a0);
        const float2 wb = z ? make_float2(1.f, 0.f) : wa;
        float2 u[2 * R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            int e;
            float2 w;
            if (r < G) {
                e = a0 + r * NBF;
                w = r == 0 ? wa : cmul(wa, __ldg(tw + r * NBF));
            } else {
                const int p = r - G + 1;
                e = z ? p * NBF : j0 + r * NBF;
                w = cmul(wb, __ldg(tw + (z ? p : r) * NBF));
            }
            pair(x[e], x[N - e], dir<FWD>(w), u[r], u[2 * R - 1 - r]);
        }
#pragma unroll
        for (int k = 1; k < 2 * R; k++) v[k] = z ? u[lane0_slot(k)] : u[k];
        float2 x0 = x[0], xn = x[N], unused;
        x0.y = 0.f;
        xn.y = 0.f;
        float2 z0;
        pair(x0, xn, make_float2(1.f, 0.f), z0, unused);
        v[0] = z ? z0 : u[0];
    }
};

// WL = 1: the T threads of a transform are consecutive lanes of one warp (row
// kernels with T <= 32), so barriers that guard only a transform's own work
// row are warp barriers; WL = 2 also runs a last radix-2 stage as
// warp-shuffle butterflies where ShflLast applies.  WL = 0 (the column and
// double-buffered tile kernels, which spread a transform's threads over the
// CTA) keeps CTA barriers.
template <class Q, int T, class PD = Pads<>, bool PP = false, int WL = 0>
struct StaticEngine {
    static_assert(WL == 0 || (T <= 32 && 32 % T == 0), "warp-local lanes need T dividing 32");
    static constexpr bool kPingPong = PP;  // a third shared-memory buffer holds the even boundaries
    // a 16384-point row (139 KB padded) fits shared memory once: the row kernel
    // loads the next tile into the same buffer after the current one is done
    static constexpr bool kSingleBuffer = Q::N >= 16384;
    static constexpr int kMaxThreads = T <= 256 ? 256 : T;
    // 3 CTAs per SM (<= 80 registers) unless a thread holds more than 16 points
    static constexpr int kMinBlocks = T <= 256 ? (Q::N / T > 16 ? 2 : 3) : 1;
    template <bool FWD, class Src0, class DstL>
    __device__ __forceinline__ static void run(const TileDesc &d, float2 *work, const Src0 &src0, const DstL &dstL,
                                               bool dst_in_place, int lane, bool active, float2 *work2 = nullptr)
    {
        float2 v[static_maxv<Q, T>()];
        srun<Q, T, PD, PP, WL, FWD, 0>(v, work, work2, src0, dstL, dst_in_place, lane, active, d.stw);
    }

    template <bool FWD, class Src0>
    __device__ __forceinline__ static void run_r2c(const TileDesc &d, float2 *work, const Src0 &src0, float2 *y,
                                                   int lane, bool active, float2 *work2 = nullptr)
    {
        using F = FusedR2C<Q, T, PD, FWD>;
        if constexpr (F::ok) {
            constexpr int V = static_maxv<Q, T>() > 2 * F::R ? static_maxv<Q, T>() : 2 * F::R;
            float2 v[V];
            prefix<FWD, 0>(v, work, work2, src0, lane, active, d.stw);
            row_sync<WL>();
            F::run(v, bbuf<PP, Q::S - 2>(work, work2), y, lane, active, d.stw, d.tw);
        } else {
            run<FWD>(d, work, src0, SmemRow{work}, true, lane, active, work2);
            row_sync<WL>();
            if (active) r2c_post_row<FWD>(work, y, d.n, lane, d.tpt, d.tw);
        }
    }

    // C2R from the staged half spectrum x: with FusedC2R the first stage builds
    // the packed inputs pairwise, else every element goes through C2RPre.
    template <bool FWD, class DstL>
    __device__ __forceinline__ static void run_c2r(const TileDesc &d, float2 *work, const float2 *x, const DstL &dstL,
                                                   int lane, bool active, float2 *work2 = nullptr)
    {
        using F = FusedC2R<Q, T, FWD>;
        if constexpr (F::ok) {
            constexpr int R = F::R;
            constexpr int V = static_maxv<Q, T>() > 2 * R ? static_maxv<Q, T>() : 2 * R;
            float2 v[V];
            const int j0 = lane, j1 = lane == 0 ? F::NBF / 2 : F::NBF - lane;
            if (active) {
                F::gather(v, x, lane, d.tw);
                dft<R, FWD>(v);
                dft<R, FWD>(v + R);
            }
            if constexpr (!PP) __syncthreads();  // the staged spectrum is read before the work row overwrites it
            if (active) {
                const BoundaryRow<PD, 0> w{bbuf<PP, 0>(work, work2)};
#pragma unroll
                for (int r = 0; r < R; r++) {
                    w(j0 * R + r, v[r]);
                    w(j1 * R + r, v[R + r]);
                }
            }
            row_sync<WL>();
            srun<Q, T, PD, PP, WL, FWD, 1>(v, work, work2, SmemRow{work}, dstL, false, lane, active, d.stw);
        } else {
            run<FWD>(d, work, C2RPre<FWD>{x, d.n, d.tw}, dstL, false, lane, active, work2);
        }
    }

    // every stage but the last, leaving the data in the work row of boundary S-2
    template <bool FWD, int S, class Src0>
    __device__ __forceinline__ static void prefix(float2 *v, float2 *work, float2 *work2, const Src0 &src0, int lane,
                                                  bool active, const float2 *stw)
    {
        if constexpr (S < Q::S - 1) {
            if constexpr (S == 0)
                sgather<Q, 0, T, FWD>(v, src0, lane, active, stw);
            else
                sgather<Q, S, T, FWD>(v, BoundaryRow<PD, S - 1>{bbuf<PP, S - 1>(work, work2)}, lane, active, stw);
            if constexpr (!PP) {
                if constexpr (S == 0)
                    __syncthreads();
                else
                    row_sync<WL>();
            }
            sscatter<Q, S, T>(v, BoundaryRow<PD, S>{bbuf<PP, S>(work, work2)}, lane, active);
            if constexpr (S + 1 < Q::S - 1) row_sync<WL>();
            prefix<FWD, S + 1>(v, work, work2, src0, lane, active, stw);
        }
    }
};


}  // namespace sipfft
