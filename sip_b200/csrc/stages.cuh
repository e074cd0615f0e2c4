// Stockham stage machinery shared by the FFT kernels.
//
// A transform of length n is processed as stages of radix R with
// Ns = product of the earlier radices.  In every stage each of the n/R
// butterflies j reads x[j + r*n/R] (r < R), multiplies input r by
// w^(r*(j mod Ns)) with w = exp(-+2 pi i / (Ns*R)), runs the R-point codelet,
// and writes output r to position (j - j mod Ns)*R + j mod Ns + r*Ns
// (Stockham autosort: after the last stage the data is in natural order).
// A thread owns butterflies j = lane + b*tpt, b < NB; all of its butterfly
// values sit in one register array `v` shared by every radix, so only one set
// is live across a stage barrier.
//
// Sources and destinations are functors so that the first stage can read the
// raw input (from a bulk-copied staging buffer or HBM, with R2C/C2R packing
// applied on the fly) and the last stage can write HBM directly.
#pragma once
#include "codelets.cuh"
#include "fft_tile.cuh"

namespace sipfft {

#ifndef SIPFFT_PAD_DEFINED
#define SIPFFT_PAD_DEFINED
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
#endif

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

// padded shared-memory row
struct SmemRow {
    float2 *row;
    __device__ __forceinline__ float2 operator()(int e) const { return row[pad(e)]; }
    __device__ __forceinline__ void operator()(int e, float2 v) const { row[pad(e)] = v; }
};

template <int R, int MAXE, bool FWD, class Src>
__device__ __forceinline__ void stage_gather(float2 *v, const Src &src, int n, int ns, uint32_t nsm, int tstep,
                                             int lane, int tpt, bool active, const float2 *__restrict__ tw,
                                             const float2 *__restrict__ tws = nullptr)
{
    constexpr int NB = nb_for<R, MAXE>();
    const int nbf = n / R;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = lane + b * tpt;
        if (active && j < nbf) {
#pragma unroll
            for (int r = 0; r < R; r++) v[b * R + r] = src(j + r * nbf);
        }
    }
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = lane + b * tpt;
        if (active && j < nbf) {
            if (ns > 1) {
                // the stage's own table when present: consecutive butterflies, consecutive entries
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

template <int R, int MAXE, class Dst>
__device__ __forceinline__ void stage_scatter(const float2 *v, const Dst &dst, int n, int ns, uint32_t nsm, int lane,
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
            for (int r = 0; r < R; r++) dst(base + r * ns, v[b * R + r]);
        }
    }
}

#define SIPFFT_RADIX_CASES(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(16)
#define SIPFFT_COMPACT_RADIX_CASES(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)

template <int MAXE, bool FWD, bool COMPACT, class Src>
__device__ __forceinline__ void gather_any(int R, float2 *v, const Src &src, int n, int ns, uint32_t nsm, int ts,
                                           int lane, int tpt, bool active, const float2 *tw, const float2 *tws)
{
#define SIPFFT_G(RR) \
    case RR: stage_gather<RR, MAXE, FWD>(v, src, n, ns, nsm, ts, lane, tpt, active, tw, tws); break;
    if constexpr (COMPACT) {
        switch (R) {
            SIPFFT_COMPACT_RADIX_CASES(SIPFFT_G)
            default: break;
        }
    } else {
        switch (R) {
            SIPFFT_RADIX_CASES(SIPFFT_G)
            default: break;
        }
    }
#undef SIPFFT_G
}

template <int MAXE, bool COMPACT, class Dst>
__device__ __forceinline__ void scatter_any(int R, const float2 *v, const Dst &dst, int n, int ns, uint32_t nsm,
                                            int lane, int tpt, bool active)
{
#define SIPFFT_S(RR) \
    case RR: stage_scatter<RR, MAXE>(v, dst, n, ns, nsm, lane, tpt, active); break;
    if constexpr (COMPACT) {
        switch (R) {
            SIPFFT_COMPACT_RADIX_CASES(SIPFFT_S)
            default: break;
        }
    } else {
        switch (R) {
            SIPFFT_RADIX_CASES(SIPFFT_S)
            default: break;
        }
    }
#undef SIPFFT_S
}

// Full FFT of one transform per thread group.
//   src0     — where stage 0 reads (may be the padded work row itself: src0_in_place)
//   dstL     — where the last stage writes (may be the work row: dstL_in_place)
// Every other stage runs in place in the padded work row.  On return the
// caller must barrier before reusing `work` if dstL wrote into it.
template <int MAXE, bool FWD, bool COMPACT = false, class Src0, class DstL>
__device__ __forceinline__ void run_fft(const TileDesc &d, float2 *work, const Src0 &src0, bool src0_in_place,
                                        const DstL &dstL, bool dstL_in_place, int lane, bool active)
{
    float2 v[maxv_for<MAXE, COMPACT>()];
    const int S = d.nstages;
    const int n = d.n;
    const SmemRow w{work};
    if (S == 0) {
        // length-1 transform: copy (the same thread reads and writes)
        if (active && lane == 0) dstL(0, src0(0));
        return;
    }
    // stage 0 (no twiddles); stage s >= 1 reads d.stw + toff when the plan has stage tables
    int64_t toff = 0;
    auto tws = [&](int s) -> const float2 * { return d.stw ? d.stw + toff : nullptr; };
    gather_any<MAXE, FWD, COMPACT>(d.radix[0], v, src0, n, d.ns[0], d.ns_m[0], d.tstep[0], lane, d.tpt, active, d.tw, nullptr);
    if (src0_in_place || (S == 1 && dstL_in_place)) __syncthreads();
    if (S == 1) {
        scatter_any<MAXE, COMPACT>(d.radix[0], v, dstL, n, d.ns[0], d.ns_m[0], lane, d.tpt, active);
        return;
    }
    scatter_any<MAXE, COMPACT>(d.radix[0], v, w, n, d.ns[0], d.ns_m[0], lane, d.tpt, active);
    __syncthreads();
#pragma unroll 1
    for (int s = 1; s < S - 1; s++) {
        gather_any<MAXE, FWD, COMPACT>(d.radix[s], v, w, n, d.ns[s], d.ns_m[s], d.tstep[s], lane, d.tpt, active, d.tw, tws(s));
        toff += int64_t(d.radix[s] - 1) * d.ns[s];
        __syncthreads();
        scatter_any<MAXE, COMPACT>(d.radix[s], v, w, n, d.ns[s], d.ns_m[s], lane, d.tpt, active);
        __syncthreads();
    }
    gather_any<MAXE, FWD, COMPACT>(d.radix[S - 1], v, w, n, d.ns[S - 1], d.ns_m[S - 1], d.tstep[S - 1], lane, d.tpt, active, d.tw,
                          tws(S - 1));
    if (dstL_in_place) __syncthreads();
    scatter_any<MAXE, COMPACT>(d.radix[S - 1], v, dstL, n, d.ns[S - 1], d.ns_m[S - 1], lane, d.tpt, active);
}

}  // namespace sipfft
