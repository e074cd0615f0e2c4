// Load / store phases of the tile kernels: HBM <-> shared-memory tile with
// the layout, packing and pass-twiddle handling of every TileDesc kind.
// Shared by the SIMT tile kernel (fft_tile.cu) and the tensor-core kernel
// (tc_fft.cu).  The shared-memory row index is padded (pad(i) = i + i/16).
#pragma once
#include <cuda_fp16.h>

#include "async_copy.cuh"
#include "codelets.cuh"
#include "fft_tile.cuh"

namespace sipfft {

#ifndef SIPFFT_PAD_DEFINED
#define SIPFFT_PAD_DEFINED
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
#endif

__device__ __forceinline__ int64_t col_base(const Addr &a, int64_t o, int64_t c)
{
    int64_t x = o * a.dist + c * a.cstride;
    if (a.cblock) x += (c / a.cblock) * a.cjump;
    return x;
}

// W_F^(e kc step) from the two-level table.  The exponent is below F (e < n,
// kc < Ns, step = F / (Ns n)), and every multi-pass length F is at most 2^28
// (transforms up to 2^27 points, Bluestein convolutions up to 2^28), so the
// index arithmetic is exact in 32 bits.
template <bool FWD>
__device__ __forceinline__ float2 pass_twiddle(const TileDesc &d, int64_t e, int64_t kc)
{
    const uint32_t m = static_cast<uint32_t>(e) * static_cast<uint32_t>(kc) * static_cast<uint32_t>(d.g_step);
    const uint32_t mask = (1u << d.g_log2l) - 1u;
    const float2 w = cmul(__ldg(d.g_lo + (m & mask)), __ldg(d.g_hi + (m >> d.g_log2l)));
    return dir<FWD>(w);
}

// ------------------------------------------------------------------------------------ load
template <bool FWD>
__device__ __forceinline__ void load_tile(const TileDesc &d, const void *in, float2 *sm, int64_t o, int64_t c0,
                                          int ntr)
{
    const int tid = threadIdx.x, bd = blockDim.x;
    const int n = d.n, P = d.pitch;
    const int io = d.io;
    if (io == IO_C2R_PACKED) {
        // pairs (k, n-k) of the half spectrum -> packed n-point input
        const int l = tid / d.tpt, lane = tid % d.tpt;
        if (l >= ntr) return;
        const float2 *x = static_cast<const float2 *>(in) + col_base(d.in_a, o, c0 + l);
        float2 *row = sm + l * P;
        for (int k = lane; 2 * k <= n; k += d.tpt) {
            float2 xk = x[k];
            float2 xm = x[n - k];
            if (k == 0) {
                xk.y = 0.f;
                xm.y = 0.f;
            }
            const float2 e = cadd(xk, cconj(xm));
            const float2 w = dir<FWD>(__ldg(d.tw + k));
            const float2 od = cmul(csub(xk, cconj(xm)), w);
            // Z[k] = e + i*od ; Z[n-k] = conj(e) + i*conj(od)
            row[pad(k)] = make_float2(e.x - od.y, e.y + od.x);
            if (k != 0 && 2 * k != n) row[pad(n - k)] = make_float2(e.x + od.y, -e.y + od.x);
        }
        return;
    }
    if (io == IO_BLUE_PRE) {
        const int l = tid / d.tpt, lane = tid % d.tpt;
        if (l >= ntr) return;
        const int64_t base = col_base(d.in_a, o, c0 + l);
        float2 *row = sm + l * P;
        const int nb = d.blue_n;
        for (int e = lane; e < n; e += d.tpt) {
            float2 v = make_float2(0.f, 0.f);
            if (e < nb) {
                if (d.blue_kind == 1) {
                    v = make_float2(static_cast<const float *>(in)[base + e], 0.f);
                } else if (d.blue_kind == 2) {
                    const float2 *x = static_cast<const float2 *>(in) + base;
                    if (2 * e <= nb) {
                        v = x[e];
                        if (e == 0 || 2 * e == nb) v.y = 0.f;
                    } else {
                        v = cconj(x[nb - e]);
                    }
                } else if (d.planar & 1) {
                    v = make_float2(static_cast<const float *>(in)[base + e], d.in_im[base + e]);
                } else {
                    v = static_cast<const float2 *>(in)[base + e];
                }
                v = cmul(v, __ldg(d.chirp + e));
            }
            row[pad(e)] = v;
        }
        return;
    }
    if (io == IO_C2R_FULL) {
        const int l = tid / d.tpt, lane = tid % d.tpt;
        if (l >= ntr) return;
        const float2 *x = static_cast<const float2 *>(in) + col_base(d.in_a, o, c0 + l);
        float2 *row = sm + l * P;
        for (int k = lane; 2 * k <= n; k += d.tpt) {
            float2 xk = x[k];
            if (k == 0) xk.y = 0.f;
            row[pad(k)] = xk;
            if (k != 0) row[pad(n - k)] = cconj(xk);
        }
        return;
    }
    // element-wise kinds: C2C, R2C_PACKED (float pairs), R2C_FULL (floats)
    const bool contiguous = d.in_a.estride == 1;
    int l, e0, estep;
    if (contiguous) {
        l = tid / d.tpt;
        e0 = tid % d.tpt;
        estep = d.tpt;
    } else {
        l = tid % d.tb;
        e0 = tid / d.tb;
        estep = bd / d.tb;
    }
    if (l >= ntr) return;
    const int64_t base = col_base(d.in_a, o, c0 + l);
    const int64_t es = d.in_a.estride;
    float2 *row = sm + l * P;
    if (d.planar & 1) {
        // separated real / imaginary planes (C2C)
        const float *xr = static_cast<const float *>(in) + base;
        const float *xi = d.in_im + base;
        if (d.g_twiddle) {
            const int64_t kc = pass_column(d, c0 + l);
            for (int e = e0; e < n; e += estep)
                row[pad(e)] = cmul(make_float2(xr[e * es], xi[e * es]), pass_twiddle<FWD>(d, e, kc));
        } else {
            for (int e = e0; e < n; e += estep) row[pad(e)] = make_float2(xr[e * es], xi[e * es]);
        }
        return;
    }
    if (io == IO_R2C_FULL) {
        const float *x = static_cast<const float *>(in) + base;
        for (int e = e0; e < n; e += estep) row[pad(e)] = make_float2(x[e * es], 0.f);
        return;
    }
    if (d.half_io & 1) {
        // complex32 input (first step of a C2C plan, no pass twiddle)
        const __half2 *xh = static_cast<const __half2 *>(in) + base;
        for (int e = e0; e < n; e += estep) row[pad(e)] = __half22float2(xh[e * es]);
        return;
    }
    const float2 *x = static_cast<const float2 *>(in) + base;
    if (d.g_twiddle) {
        const int64_t kc = pass_column(d, c0 + l);
        for (int e = e0; e < n; e += estep) row[pad(e)] = cmul(x[e * es], pass_twiddle<FWD>(d, e, kc));
    } else {
        for (int e = e0; e < n; e += estep) row[pad(e)] = x[e * es];
    }
}

// ------------------------------------------------------------------------------------ store
template <bool FWD>
__device__ __forceinline__ void store_tile(const TileDesc &d, void *out, const float2 *sm, int64_t o, int64_t c0,
                                           int ntr)
{
    const int tid = threadIdx.x, bd = blockDim.x;
    const int n = d.n, P = d.pitch;
    const int io = d.io;
    if (io == IO_R2C_PACKED) {
        const int l = tid / d.tpt, lane = tid % d.tpt;
        if (l >= ntr) return;
        float2 *y = static_cast<float2 *>(out) + col_base(d.out_a, o, c0 + l);
        const float2 *row = sm + l * P;
        for (int k = lane; 2 * k <= n; k += d.tpt) {
            const float2 zk = row[pad(k)];
            const float2 zm = cconj(row[pad(k == 0 ? 0 : n - k)]);
            const float2 e = cscale(cadd(zk, zm), 0.5f);
            const float2 t = csub(zk, zm);
            const float2 od = make_float2(0.5f * t.y, -0.5f * t.x);  // -i/2 * t
            const float2 wo = cmul(dir<FWD>(__ldg(d.tw + k)), od);
            y[k] = cadd(e, wo);
            if (2 * k != n) y[n - k] = cconj(csub(e, wo));
        }
        return;
    }
    if (io == IO_BLUE_PRE || io == IO_BLUE_POST) {
        const int l = tid / d.tpt, lane = tid % d.tpt;
        if (l >= ntr) return;
        const int64_t base = col_base(d.out_a, o, c0 + l);
        const float2 *row = sm + l * P;
        if (io == IO_BLUE_PRE) {
            float2 *y = static_cast<float2 *>(out) + base;
            for (int e = lane; e < n; e += d.tpt) y[e] = cmul(row[pad(e)], __ldg(d.bmul + e));
        } else if (d.blue_kind == 2) {
            float *y = static_cast<float *>(out) + base;
            for (int e = lane; e < d.blue_n; e += d.tpt) y[e] = cmul(row[pad(e)], __ldg(d.chirp + e)).x;
        } else if (d.planar & 2) {
            float *yr = static_cast<float *>(out) + base;
            float *yi = d.out_im + base;
            for (int e = lane; e < d.blue_n; e += d.tpt) {
                const float2 v = cmul(row[pad(e)], __ldg(d.chirp + e));
                yr[e] = v.x;
                yi[e] = v.y;
            }
        } else {
            const int count = d.blue_kind == 1 ? d.blue_n / 2 + 1 : d.blue_n;
            float2 *y = static_cast<float2 *>(out) + base;
            for (int e = lane; e < count; e += d.tpt) y[e] = cmul(row[pad(e)], __ldg(d.chirp + e));
        }
        return;
    }
    const bool contiguous = d.out_a.estride == 1;
    int l, e0, estep;
    if (contiguous) {
        l = tid / d.tpt;
        e0 = tid % d.tpt;
        estep = d.tpt;
    } else {
        l = tid % d.tb;
        e0 = tid / d.tb;
        estep = bd / d.tb;
    }
    if (l >= ntr) return;
    const int64_t base = col_base(d.out_a, o, c0 + l);
    const int64_t es = d.out_a.estride;
    const float2 *row = sm + l * P;
    if (d.planar & 2) {
        float *yr = static_cast<float *>(out) + base;
        float *yi = d.out_im + base;
        for (int e = e0; e < n; e += estep) {
            const float2 v = row[pad(e)];
            yr[e * es] = v.x;
            yi[e * es] = v.y;
        }
        return;
    }
    if (io == IO_C2R_FULL) {
        float *y = static_cast<float *>(out) + base;
        for (int e = e0; e < n; e += estep) y[e * es] = row[pad(e)].x;
        return;
    }
    if (d.half_io & 2) {
        // complex32 output (last step of a C2C plan)
        __half2 *yh = static_cast<__half2 *>(out) + base;
        for (int e = e0; e < n; e += estep) yh[e * es] = __float22half2_rn(row[pad(e)]);
        return;
    }
    const int count = (io == IO_R2C_FULL) ? n / 2 + 1 : n;
    float2 *y = static_cast<float2 *>(out) + base;
    for (int e = e0; e < count; e += estep) st_stream(y + e * es, row[pad(e)]);
}

// ------------------------------------------------------------------------------------ async tile loads
// Element copies of one C2C tile issued with cp.async (8 bytes per element, no
// registers held); a double-buffered kernel issues the next tile's copies
// before it runs the current one.  Inter-pass twiddles are left to the first
// stage.
__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void issue_tile_c2c(const TileDesc &d, const void *in, float2 *sm, int64_t g)
{
    const int tid = threadIdx.x, bd = blockDim.x;
    const int64_t o = g / d.tiles_per_outer;
    const int64_t c0 = (g % d.tiles_per_outer) * d.tb;
    const int64_t left = d.n_cols - c0;
    const int ntr = left < d.tb ? static_cast<int>(left) : d.tb;
    int l, e0, estep;
    if (d.in_a.estride == 1) {
        l = tid / d.tpt;
        e0 = tid % d.tpt;
        estep = d.tpt;
    } else {
        l = tid % d.tb;
        e0 = tid / d.tb;
        estep = bd / d.tb;
    }
    if (l >= ntr) return;
    const float2 *x = static_cast<const float2 *>(in) + col_base(d.in_a, o, c0 + l);
    const int64_t es = d.in_a.estride;
    float2 *row = sm + l * d.pitch;
    for (int e = e0; e < d.n; e += estep) cp_async8(row + pad(e), x + e * es);
}


// One tile: load, Stockham stages, store.  Threads beyond tb*tpt (a launch
// shared by tiles of different shapes) only take part in the barriers.

}  // namespace sipfft
