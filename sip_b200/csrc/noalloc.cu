// C2C FFT entry point that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they need an FFT:
// real-time loops that forbid allocator calls once they are running, or
// hosts that hand the library raw buffers and own every allocation
// themselves.  The
// ordinary exec path for long transforms needs a caller-provided workspace
// and a plan whose twiddle tables are allocated with cudaMalloc.  This entry
// point instead keeps its scratch (the twiddle tables and the intermediate
// between its two Stockham passes) in one file-scope __device__ array of
// fixed size, so it never calls cudaMalloc, cudaFree or any other allocating
// routine.
//
// Scope: 1D C2C, lengths 16385..2^20 that split into two shared-memory passes
// of at most 2048 points with radices 2..16 / 3 / 5 / 7 / 11 / 13, and
// length * batch <= 2^20 complex values (8 MiB of intermediate).
//
// The array lives on every GPU that loads the library until the process
// exits (8.5 MiB).  Every call writes the tables and the intermediate before
// reading them, so nothing has to start at zero and no state carries over
// from the previous call; but calls that overlap on the GPU (two streams, or
// two host threads) share the one array and race.  The first call on a device
// looks up the array's device address (cudaGetSymbolAddress) and sets the
// kernels' shared-memory limits; make that first call before any stream
// capture.
#include <algorithm>
#include <mutex>

#include "../../include/asdsip_fft_ext.h"
#include "sipfft_internal.h"

namespace sipfft {

namespace {

constexpr int64_t kNoAllocTableElems = 1 << 16;  // twiddle tables (512 KiB)
constexpr int64_t kNoAllocDataElems = 1 << 20;   // intermediate between the passes (8 MiB)
constexpr int kNoAllocMaxDevices = 64;

}  // namespace

// The scratch.  In host code this name is only a stand-in for the symbol, not
// a device address: kernels receive the address looked up by scratch_for().
static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocTableElems + kNoAllocDataElems];

namespace {

std::mutex g_noalloc_mu;
float2 *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on `device` (current), looked up once per device.
float2 *scratch_for(int device)
{
    if (device < 0 || device >= kNoAllocMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        if (configure_kernels(device) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return nullptr;
        }
        g_noalloc_ptr[device] = static_cast<float2 *>(p);
    }
    return g_noalloc_ptr[device];
}

// Radices of one pass (same rules as the planner), fixed-size output.
bool pass_radices(int n, int *r, int &count)
{
    count = 0;
    int m = n, twos = 0;
    while (m % 2 == 0) {
        m /= 2;
        twos++;
    }
    if (twos > 0) {
        const int s = (twos + 3) / 4, base = twos / s, extra = twos % s;
        for (int i = 0; i < s; i++) {
            if (count >= kMaxStages) return false;
            r[count++] = 1 << (base + (i < extra ? 1 : 0));
        }
    }
    for (int p : {13, 11, 7, 5, 3}) {
        while (m % p == 0) {
            if (count >= kMaxStages) return false;
            r[count++] = p;
            m /= p;
        }
    }
    return m == 1;
}

// Two balanced pass lengths p0 >= p1, p0 * p1 = n, both <= 2048.
bool split_two(int64_t n, int &p0, int &p1)
{
    int64_t g[2] = {1, 1};
    int64_t m = n;
    int64_t primes[64];
    int np = 0;
    for (int64_t f = 2; f * f <= m; f++)
        while (m % f == 0 && np < 64) {
            primes[np++] = f;
            m /= f;
        }
    if (m > 1 && np < 64) primes[np++] = m;
    for (int i = np - 1; i >= 0; i--) {  // ascending list: largest factors first
        const int k = g[0] <= g[1] ? 0 : 1;
        g[k] *= primes[i];
    }
    if (g[0] > 2048 || g[1] > 2048) return false;
    p0 = static_cast<int>(g[0] >= g[1] ? g[0] : g[1]);
    p1 = static_cast<int>(g[0] >= g[1] ? g[1] : g[0]);
    return true;
}

int log2_ceil(int64_t x)
{
    int l = 0;
    while ((int64_t(1) << l) < x) l++;
    return l;
}

// Column-tile descriptor of one Stockham pass (the addressing of planner.cpp's multi-pass steps).
bool make_pass(TileDesc &d, int &maxe, int &grid, int rp, int64_t F, int64_t rows, int64_t ns, const float2 *tw,
               const float2 *lo, const float2 *hi, int log2l)
{
    int radix[kMaxStages];
    int cnt = 0;
    if (!pass_radices(rp, radix, cnt)) return false;
    d = TileDesc{};
    d.n = rp;
    d.io = IO_C2C;
    d.nstages = cnt;
    int nsr = 1;
    for (int s = 0; s < cnt; s++) {
        d.radix[s] = radix[s];
        d.ns[s] = nsr;
        d.ns_m[s] = ns_reciprocal(nsr);
        d.tstep[s] = rp / (nsr * radix[s]);
        nsr *= radix[s];
    }
    maxe = rp <= 4096 ? 16 : 32;
    d.tpt = (rp + maxe - 1) / maxe;
    int pitch = (rp - 1) + ((rp - 1) >> 4) + 1;
    if ((pitch & 1) == 0) pitch += 1;
    d.pitch = pitch;
    d.tb = 0;
    for (int tb = 16; tb >= 1; tb /= 2) {
        if (tb * d.tpt <= 512 && int64_t(tb) * pitch * 8 <= kMaxSmemBytes) {
            d.tb = tb;
            break;
        }
    }
    if (d.tb == 0) return false;
    if (d.tb >= 2) {
        // column tiles: a pitch with P mod (32/tb) = 16/tb puts a half warp's
        // tb transforms x 16/tb elements on 16 distinct 8-byte bank pairs
        const int m = 32 / d.tb, want = 16 / d.tb;
        int p = pitch;
        while (p % m != want) p++;
        if (int64_t(d.tb) * p * 8 <= kMaxSmemBytes) d.pitch = p;
    }
    d.xfast = 1;
    d.n_outer = rows;
    d.n_cols = F / rp;
    d.tiles_per_outer = (d.n_cols + d.tb - 1) / d.tb;
    d.num_tiles = d.tiles_per_outer * rows;
    d.in_a = Addr{F, 1, F / rp, 0, 0};
    d.out_a = Addr{F, 1, ns, ns, ns * (rp - 1)};
    d.tw = tw;
    d.tw_mul = 1;
    d.g_twiddle = ns > 1 ? 1 : 0;
    d.g_ns = ns;
    d.g_step = F / (ns * rp);
    d.g_lo = lo;
    d.g_hi = hi;
    d.g_log2l = log2l;
    const int64_t cap = int64_t(kB200Sms) * 64;
    grid = static_cast<int>(d.num_tiles < cap ? d.num_tiles : cap);
    return true;
}

}  // namespace

}  // namespace sipfft

extern "C" int32_t asdFftExecC2CNoAlloc(const void *input, void *output, int64_t fftSize, int64_t batchSize,
                                        int32_t direction, void *stream)
{
    using namespace sipfft;
    if (!input || !output || fftSize <= 16384 || fftSize > (int64_t(1) << 20) || batchSize <= 0) {
        set_last_error("asdFftExecC2CNoAlloc: length must be in 16385..1048576 and batch >= 1");
        return AsdSip::ACL_ERROR_INVALID_PARAM;
    }
    if (direction != AsdSip::ASCEND_FFT_FORWARD && direction != AsdSip::ASCEND_FFT_INVERSE) {
        set_last_error("asdFftExecC2CNoAlloc: invalid direction");
        return AsdSip::ACL_ERROR_INVALID_PARAM;
    }
    if (batchSize > kNoAllocDataElems / fftSize) {  // fftSize * batchSize > kNoAllocDataElems, without overflow
        set_last_error("asdFftExecC2CNoAlloc: fftSize * batchSize exceeds the 1048576-element scratch array");
        return AsdSip::ACL_ERROR_INVALID_PARAM;
    }
    if ((reinterpret_cast<uintptr_t>(input) & 7) || (reinterpret_cast<uintptr_t>(output) & 7)) {
        set_last_error("asdFftExecC2CNoAlloc: buffers must be 8-byte aligned");
        return AsdSip::ACL_ERROR_INVALID_PARAM;
    }
    int p0 = 0, p1 = 0;
    if (!split_two(fftSize, p0, p1)) {
        set_last_error("asdFftExecC2CNoAlloc: length does not split into two passes of <= 2048 points");
        return AsdSip::ACL_ERROR_API_NOT_SUPPORT;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    }
    float2 *base = scratch_for(dev);
    if (!base) {
        set_last_error("asdFftExecC2CNoAlloc: scratch array set-up failed");
        return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool fwd = direction == AsdSip::ASCEND_FFT_FORWARD;
    const int64_t F = fftSize;

    // Front of the array: pass-0 stage table, pass-1 stage table, then the
    // two-level table of W_F (lo: L entries, hi: ceil(F/L) entries), then each
    // pass's per-stage tables ([r-1][k] per stage, < 2048 entries a pass); at
    // most 2048 + 2048 + 1024 + 1024 + 2 x 2048 entries.  The intermediate follows.
    const int log2l = (log2_ceil(F) + 1) / 2;
    const int64_t L = int64_t(1) << log2l;
    float2 *tw0 = base;
    float2 *tw1 = tw0 + p0;
    float2 *lo = tw1 + p1;
    float2 *hi = lo + L;
    float2 *data = base + kNoAllocTableElems;

    TileDesc d0{}, d1{};
    int maxe0 = 16, maxe1 = 16, grid0 = 1, grid1 = 1;
    if (!make_pass(d0, maxe0, grid0, p0, F, batchSize, 1, tw0, lo, hi, log2l) ||
        !make_pass(d1, maxe1, grid1, p1, F, batchSize, p0, tw1, lo, hi, log2l)) {
        set_last_error("asdFftExecC2CNoAlloc: pass does not fit a tile");
        return AsdSip::ACL_ERROR_API_NOT_SUPPORT;
    }
    float2 *stw0 = hi + (F + L - 1) / L;
    float2 *stw1 = stw0 + stage_twiddle_count(d0.radix, d0.nstages);
    if (stw1 + stage_twiddle_count(d1.radix, d1.nstages) > base + kNoAllocTableElems) {
        set_last_error("asdFftExecC2CNoAlloc: twiddle tables exceed the scratch table area");
        return AsdSip::ACL_ERROR_API_NOT_SUPPORT;
    }
    d0.stw = stw0;
    d1.stw = stw1;
    cudaError_t e = fill_twiddles(tw0, p0, p0, 1, st);
    if (e == cudaSuccess) e = fill_twiddles(tw1, p1, p1, 1, st);
    if (e == cudaSuccess) e = fill_twiddles(lo, L, F, 1, st);
    if (e == cudaSuccess) e = fill_twiddles(hi, (F + L - 1) / L, F, L, st);
    if (e == cudaSuccess) e = fill_stage_twiddles(stw0, d0.radix, d0.nstages, st);
    if (e == cudaSuccess) e = fill_stage_twiddles(stw1, d1.radix, d1.nstages, st);
    // each pass on the double-buffered tile kernel when two tiles fit shared
    // memory (the next tile's copies overlap this tile's stages), else one tile at a time
    auto run_pass = [&](TileDesc &d, int maxe, int grid) -> cudaError_t {
        const size_t smem2 = 2 * static_cast<size_t>(d.tb) * d.pitch * sizeof(float2);
        if (smem2 <= static_cast<size_t>(kMaxSmemBytes)) {
            const int per_sm = kernel_blocks_per_sm(tile_db_kernel_fn(maxe, fwd), d.tb * d.tpt, smem2);
            if (per_sm > 0) {
                const int64_t g = std::min<int64_t>(d.num_tiles, int64_t(per_sm) * sm_count(dev));
                return launch_tile_db(d, maxe, fwd, static_cast<int>(g), st);
            }
        }
        return launch_tile(d, maxe, fwd, grid, st);
    };
    if (e == cudaSuccess) {
        d0.in = input;
        d0.out = data;
        e = run_pass(d0, maxe0, grid0);
    }
    if (e == cudaSuccess) {
        d1.in = data;
        d1.out = output;
        e = run_pass(d1, maxe1, grid1);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("asdFftExecC2CNoAlloc: ") + cudaGetErrorString(e));
        cudaGetLastError();
        return AsdSip::ACL_ERROR_INTERNAL_ERROR;
    }
    return AsdSip::ACL_SUCCESS;
}
