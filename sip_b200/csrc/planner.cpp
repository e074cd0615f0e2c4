// FFT planner: turns a reference-style plan (type, direction, sizes, batch,
// vertical/horizontal) into a list of tile-kernel launches.
//
// Reference counterpart: core/fft/fft_api.cpp — addFFTSteps (485-499),
// getCore (383-432), init2DSteps (527-602), init3DSteps (604-697) and the
// per-core radix tables (fft_core_b.cpp:126-168, fft_core_n.cpp:206-265,
// fft_core_common_func.cpp:675-826).  The reference chooses one of ~16 core
// families and inserts explicit Transpose steps between axes; here every axis
// is one launch of the same tile kernel whose load/store addressing walks the
// axis in place (no transpose steps), and transforms longer than one CTA's
// shared memory become a short sequence of Stockham passes whose butterflies
// are shared-memory FFTs (2 passes up to 2^18 complex points, 3 up to 2^27).
#include <algorithm>
#include <cmath>
#include <map>
#include <sstream>

#include "sipfft_internal.h"

namespace sipfft {

bool valid_radices(const std::vector<int> &r, int64_t n);

namespace {

constexpr int64_t kMaxRowN = 16384;        // longest single-CTA transform: 512 threads x 32 points
constexpr int64_t kMaxSingleTileC2C = 8192;  // longest C2C row planned as one tile
constexpr int kMaxPassRadix = 2048;        // longest sub-FFT of one multi-pass Stockham pass
constexpr int64_t kMaxStridedTile = 8192;  // longest strided axis planned as one column tile
constexpr int64_t kMaxBluesteinM = int64_t(1) << 28;  // Bluestein for every N <= 2^27
constexpr int kRowThreadsTarget = 256;     // threads per CTA for batched rows
constexpr int kStaticRowThreads = 128;     // threads per CTA for rows on a compile-time engine
constexpr int kRowSmemTarget = 64 * 1024;  // keep >= 3 CTAs per SM for short rows
constexpr int kColTile = 16;               // columns per tile: 16 x 8 B = one 128-byte line
constexpr int kMaxThreads = 512;           // launch bound of the tile kernel (keeps 128 registers/thread)
const int kRadices[] = {16, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};

int padded(int i) { return i + (i >> 4); }

int pitch_for(int n)
{
    int p = (n > 0 ? padded(n - 1) + 1 : 1);
    if ((p & 1) == 0) p += 1;  // odd pitch: column-tile accesses hit distinct banks
    return p;
}

int ilog2_ceil(int64_t x)
{
    int l = 0;
    while ((int64_t(1) << l) < x) l++;
    return l;
}

struct TileCfg {
    int maxe = 16, tpt = 1, tb = 1, pitch = 1;
};

// Threads, transforms per CTA and shared-memory pitch for one tile launch.
bool choose_cfg(int n, bool column, int64_t ncols, TileCfg &c, std::string &err, int maxe_override = 0,
                int row_threads = kRowThreadsTarget, int row_smem = kRowSmemTarget, int max_maxe = 32,
                int max_threads = 512)
{
    if (n < 1 || n > 32768) {
        err = "transform length out of the single-CTA range";
        return false;
    }
    c.maxe = n <= 4096 ? 16 : 32;
    if (c.maxe > max_maxe) c.maxe = max_maxe;
    if (maxe_override == 8 || maxe_override == 16 || maxe_override == 32) {
        if ((n + maxe_override - 1) / maxe_override <= max_threads) c.maxe = maxe_override;
    }
    c.tpt = std::max(1, (n + c.maxe - 1) / c.maxe);
    if (c.tpt > max_threads) {
        err = "too many threads per transform";
        return false;
    }
    c.pitch = pitch_for(n);
    const int64_t bytes_per = int64_t(c.pitch) * 8;
    if (column) {
        // column tiles: at most 256 threads while that keeps >= 4 columns (32-byte
        // row runs), so that several CTAs share an SM; else up to max_threads
        const int col_threads = (4 * c.tpt <= 256) ? 256 : max_threads;
        c.tb = 0;
        for (int tb = kColTile; tb >= 1; tb /= 2) {
            if (tb * c.tpt <= col_threads && tb * bytes_per <= kMaxSmemBytes) {
                c.tb = tb;
                break;
            }
        }
    } else {
        int tb = std::max(1, row_threads / c.tpt);
        while (tb > 1 && tb * bytes_per > row_smem) tb /= 2;
        if (tb > ncols) tb = static_cast<int>(std::max<int64_t>(1, ncols));
        while (tb > 1 && tb * c.tpt > max_threads) tb /= 2;
        c.tb = (bytes_per <= kMaxSmemBytes) ? tb : 0;
    }
    if (c.tb == 0) {
        err = "transform does not fit in shared memory";
        return false;
    }
    if (column && c.tb >= 2) {
        // column tiles: lane l = tid mod tb works on transform l, so a half warp
        // touches tb transforms x 16/tb consecutive elements; a pitch with
        // P mod (32/tb) = 16/tb puts them on 16 distinct 8-byte bank pairs
        const int m = 32 / c.tb, want = 16 / c.tb;
        int p = padded(n - 1) + 1;
        while (p % m != want) p++;
        if (int64_t(c.tb) * p * 8 <= kMaxSmemBytes) c.pitch = p;
    }
    return true;
}

// Resident CTAs per SM of the single-tile tensor-core kernel (128 threads):
// limited by its registers, its shared memory and its 128 of the SM's 512
// TMEM columns.  (The occupancy query reports one CTA for this kernel.)
int tc_tile_blocks_per_sm(const void *fn, size_t smem)
{
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, fn) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    const int regs = std::max(1, a.numRegs);
    const int by_regs = 65536 / (128 * ((regs + 7) / 8 * 8));
    const int by_smem = static_cast<int>((228 * 1024) / (smem + a.sharedSizeBytes + 1024));
    return std::max(1, std::min({4, by_regs, by_smem}));
}

int grid_for(int64_t tiles)
{
    const int64_t cap = int64_t(kB200Sms) * 64;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(tiles, cap)));
}

void set_stages(TileDesc &d, const std::vector<int> &radices, int n, int tw_mul)
{
    d.nstages = static_cast<int>(radices.size());
    int ns = 1;
    for (size_t s = 0; s < radices.size(); s++) {
        d.radix[s] = radices[s];
        d.ns[s] = ns;
        d.ns_m[s] = ns_reciprocal(ns);
        d.tstep[s] = (n / (ns * radices[s])) * tw_mul;
        ns *= radices[s];
    }
}

// Split the prime factors of n into `parts` groups with balanced products.
bool split_passes(int64_t n, int parts, std::vector<int> &out)
{
    std::vector<int64_t> primes;
    int64_t m = n;
    for (int64_t f = 2; f * f <= m; f++)
        while (m % f == 0) {
            primes.push_back(f);
            m /= f;
        }
    if (m > 1) primes.push_back(m);
    std::sort(primes.rbegin(), primes.rend());
    std::vector<int64_t> g(parts, 1);
    for (int64_t p : primes) {
        auto it = std::min_element(g.begin(), g.end());
        *it *= p;
    }
    out.clear();
    for (int64_t v : g) {
        if (v > kMaxPassRadix) return false;
        out.push_back(static_cast<int>(v));
    }
    std::sort(out.rbegin(), out.rend());
    return true;
}

// Splits radices above max_r into supported pairs (16 = 4 x 4, 12 = 4 x 3);
// false when a prime radix (11, 13) is above it.
bool limit_radices(std::vector<int> &radices, int max_r)
{
    if (max_r >= 16) return true;
    std::vector<int> out;
    for (int r : radices) {
        if (r <= max_r) {
            out.push_back(r);
        } else if (r == 16 && max_r >= 4) {
            out.push_back(4);
            out.push_back(4);
        } else if (r == 12 && max_r >= 4) {
            out.push_back(4);
            out.push_back(3);
        } else {
            return false;
        }
    }
    radices = out;
    return static_cast<int>(radices.size()) <= kMaxStages;
}

struct Builder {
    Plan &p;
    bool fwd;
    int device;
    explicit Builder(Plan &plan) : p(plan), fwd(plan.forward()), device(plan.device) {}

    std::string err;
    bool in_multipass = false;  // planning the passes of a multi-pass transform

    const float2 *table(int64_t count, int64_t denom, int64_t mult = 1)
    {
        TablePtr t = get_table(count, denom, mult, device, &err);
        if (!t) return nullptr;
        p.tables.push_back(t);
        return t->ptr;
    }

    // two-level table for W_F^m, m < F: lo[m & (L-1)] * hi[m >> log2 L]
    bool table2(int64_t F, const float2 *&lo, const float2 *&hi, int &log2l)
    {
        log2l = std::max(1, (ilog2_ceil(F) + 1) / 2);
        const int64_t L = int64_t(1) << log2l;
        lo = table(L, F, 1);
        hi = table((F + L - 1) / L, F, L);
        return lo && hi;
    }

    void need_ws(Buf b, size_t bytes)
    {
        const int i = static_cast<int>(b) - static_cast<int>(Buf::kWs0);
        if (i >= 0 && i < kWsSlots) p.ws_buf_bytes[i] = std::max(p.ws_buf_bytes[i], bytes);
    }

    // ASCEND_FFT_C2C_SEP: the C2C steps with separated real / imaginary user
    // planes.  The first step reads the planes, the last writes them; any
    // intermediate that the interleaved plan keeps in the user output (which
    // holds only the real plane here) moves to workspace slot 3.
    bool make_planar()
    {
        const size_t S = p.steps.size();
        if (S == 0) return false;
        int64_t elems = p.batch;
        for (int64_t v : p.sizes) elems *= v;
        bool redirect = false;
        for (size_t i = 0; i < S; i++) {
            Step &s = p.steps[i];
            const bool ok_io = s.d.io == IO_C2C || (i == 0 && s.d.io == IO_BLUE_PRE && s.d.blue_kind == 0) ||
                               (i + 1 == S && s.d.io == IO_BLUE_POST && s.d.blue_kind == 0);
            if (s.kind != StepKind::kTile || !ok_io) {
                err = "separated layout supports C2C steps only";
                return false;
            }
            if (i + 1 < S && s.dst == Buf::kUserOut) {
                s.dst = Buf::kWs3;
                redirect = true;
            }
            if (i > 0 && s.src == Buf::kUserOut) s.src = Buf::kWs3;
            if (i > 0 && s.src == Buf::kUserIn) {
                err = "separated layout: a later step reads the user input";
                return false;
            }
        }
        p.steps.front().d.planar |= 1;
        if (p.steps.back().dst == Buf::kUserOut) p.steps.back().d.planar |= 2;
        for (Step &s : p.steps) {
            if (!s.d.planar) continue;
            // the planar load / store phases live in the tile kernel only
            s.has_row = false;
            s.row_fn = nullptr;
            s.db = false;
            s.db_fn = nullptr;
            s.cp_fn = nullptr;
            s.tc_fmt = -1;
            s.what += " [separated re/im]";
        }
        if (redirect) need_ws(Buf::kWs3, size_t(elems) * sizeof(float2));
        return true;
    }

    // One single-CTA launch over a set of transforms.
    bool add_tile(int io, int n, int tw_mul, const float2 *tw, bool column, int64_t n_outer, int64_t n_cols,
                  const Addr &ia, const Addr &oa, Buf src, Buf dst, const std::string &what)
    {
        Step s;
        if (!make_tile(s, io, n, tw_mul, tw, column, n_outer, n_cols, ia, oa, src, dst, what)) return false;
        p.steps.push_back(s);
        return true;
    }

    bool make_tile(Step &s, int io, int n, int tw_mul, const float2 *tw, bool column, int64_t n_outer,
                   int64_t n_cols, const Addr &ia, const Addr &oa, Buf src, Buf dst, const std::string &what)
    {
        std::vector<int> radices;
        if (!factor_radices(n, radices)) {
            err = "length " + std::to_string(n) + " has a prime factor above 13";
            return false;
        }
        int maxe_override = 0;
        int row_threads = p.row_threads;
        TuneChoice tc;
        if (p.use_tuned && tuned_choice(n, tc) && valid_radices(tc.radices, n) && tc.maxe <= p.max_maxe) {
            radices = tc.radices;
            maxe_override = tc.maxe;
            if (tc.row_threads > 0 && tc.row_threads <= p.row_threads) row_threads = tc.row_threads;
        }
        if (!limit_radices(radices, p.max_radix)) {
            err = "length " + std::to_string(n) + " needs a radix above " + std::to_string(p.max_radix);
            return false;
        }
        TileCfg c;
        if (!choose_cfg(n, column, n_cols, c, err, maxe_override, row_threads, p.row_smem, p.max_maxe,
                        p.max_maxe < 32 ? p.row_threads : kMaxThreads))
            return false;
        s = Step();
        s.kind = StepKind::kTile;
        s.forward = fwd;
        s.src = src;
        s.dst = dst;
        s.maxe = c.maxe;
        s.what = what;
        TileDesc &d = s.d;
        d.n = n;
        d.io = io;
        set_stages(d, radices, n, tw_mul);
        d.tb = c.tb;
        d.tpt = c.tpt;
        d.pitch = c.pitch;
        d.xfast = column ? 1 : 0;
        d.n_outer = n_outer;
        d.n_cols = n_cols;
        d.tiles_per_outer = (n_cols + c.tb - 1) / c.tb;
        d.num_tiles = d.tiles_per_outer * n_outer;
        d.in_a = ia;
        d.out_a = oa;
        d.tw = tw;
        d.tw_mul = tw_mul;
        if (d.nstages > 1) {
            // contiguous per-stage twiddles: coalesced reads in every stage
            TablePtr st = get_stage_table(d.radix, d.nstages, device, &err);
            if (!st) return false;
            p.tables.push_back(st);
            d.stw = st->ptr;
        }
        s.grid = grid_for(d.num_tiles);
        if (!column && n_outer == 1 && ia.estride == 1 && oa.estride == 1 &&
            (io == IO_C2C || io == IO_R2C_PACKED || io == IO_C2R_PACKED))
            add_row_variant(s, c, ia.cstride, oa.cstride);
        if (column && io == IO_C2C && 2 * int64_t(d.tb) * d.pitch * 8 <= kMaxSmemBytes) {
            // strided C2C axis or multi-pass step: double-buffered persistent tiles,
            // with the compile-time engine of the length when one matches the tile shape
            const size_t smem = 2 * size_t(d.tb) * d.pitch * 8;
            const void *fn = tile_db_kernel_fn(s.maxe, s.forward);
            const StaticKernel *sk = find_static_kernel(n, IO_C2C);
            const float2 *stw = d.stw;
            if (sk && sk->tpt == d.tpt && sk->db[s.forward ? 1 : 0]) {
                TablePtr t = get_stage_table(*sk, device, &err);
                if (!t) return false;
                p.tables.push_back(t);
                fn = sk->db[s.forward ? 1 : 0];
                stw = t->ptr;
            }
            const int per_sm = kernel_blocks_per_sm(fn, d.tb * d.tpt, smem);
            if (per_sm > 0) {
                s.db = true;
                if (fn != tile_db_kernel_fn(s.maxe, s.forward)) {
                    // d keeps the runtime radices' tables; the engine's own go in db_stw
                    s.db_fn = fn;
                    s.db_stw = stw;
                }
                s.grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(d.num_tiles, int64_t(per_sm) * sm_count(device))));
            }
            // TMA column tiles of the same engine: box copies instead of per-element
            // copies, last stage stored from registers
            const void *cfn =
                s.db_fn ? col_pipe_kernel_fn(n, d.tpt, d.tb, s.forward, d.out_a.estride == 1) : nullptr;
            if (cfn && col_pipe_layout_ok(d)) {
                const int64_t need = int64_t(d.tb) * std::max(n, d.pitch);
                d.col_buf = (need + 15) / 16 * 16;
                d.row_bufs = col_pipe_bufs(static_cast<int>(n), d.tpt, d.tb);
                const int cps = kernel_blocks_per_sm(cfn, d.tb * d.tpt, col_pipe_smem(d));
                if (cps > 0) {
                    s.cp_fn = cfn;
                    s.cp_grid = static_cast<int>(
                        std::max<int64_t>(1, std::min<int64_t>(d.num_tiles, int64_t(cps) * sm_count(device))));
                }
            }
        }
        // passes of a multi-pass transform keep the FP32 kernels: their tiles would run on the
        // single-tile tensor-core kernel, several times slower than the double-buffered FP32 passes
        if (in_multipass || p.fft_type == 0x30 || !(io == IO_C2C || io == IO_R2C_PACKED || io == IO_C2R_PACKED))
            return true;
        const int form = tc_form(n);
        return form == 1 || form == 2 ? add_tc_variant(s, form) : true;
    }

    // Stage arithmetic of a length-n step: 0 FP32, 1 FP16 x3, 2 BF16 x3 (in
    // precision mode 3, per length, what the autotuner measured fastest).
    int tc_form(int64_t n) const
    {
        int form = p.precision;
        if (form == 3) {
            TuneChoice t;
            form = tuned_choice(n, t) ? t.precision : 0;
        }
        return form;
    }

    // Out-of-place transpose of `batch` matrices rows x cols -> cols x rows.
    void add_transpose(int64_t batch, int64_t rows, int64_t cols, Buf src, Buf dst, const std::string &what)
    {
        Step s;
        s.kind = StepKind::kTranspose;
        s.src = src;
        s.dst = dst;
        s.t_batch = batch;
        s.t_rows = rows;
        s.t_cols = cols;
        s.what = what;
        p.steps.push_back(s);
    }

    // A strided C2C axis [outer][n][inner] through transposes: transpose the axis
    // into contiguous rows in workspace, run them on the row kernels (the
    // tensor-core row pipeline in the split-precision forms), transpose back.
    // Three HBM round trips instead of one, for axes whose column kernel is the
    // slower (the single-tile tensor-core kernel is latency-bound; FP32 column
    // tiles of long axes keep only 2-4 columns).  The reference runs its strided
    // axes through explicit Transpose steps as well (core/fft/fft_api.cpp:527-697).
    bool add_transposed_axis(int64_t n, int64_t outer, int64_t inner, Buf src, Buf dst)
    {
        const Buf a = free_ws({src, dst}), b = free_ws({src, dst, a});
        const size_t bytes = size_t(outer) * size_t(n) * size_t(inner) * sizeof(float2);
        need_ws(a, bytes);
        need_ws(b, bytes);
        std::ostringstream w;
        w << "C2C axis n=" << n << " outer=" << outer << " inner=" << inner;
        add_transpose(outer, n, inner, src, a, w.str() + ": transpose to rows");
        const float2 *tw = table(n, n);
        if (!tw) return false;
        Addr ra{0, n, 1, 0, 0};
        if (!add_tile(IO_C2C, static_cast<int>(n), 1, tw, false, 1, outer * inner, ra, ra, a, b,
                      w.str() + ": rows"))
            return false;
        add_transpose(outer, inner, n, b, dst, w.str() + ": transpose back");
        return true;
    }

    // Tensor-core split-precision form of a tile step (lengths with a
    // tcgen05 kernel); replaces the FP32 kernels of the step.
    bool add_tc_variant(Step &s, int form)
    {
        TcConfig tc;
        const int n = s.d.n;
        const int fmt_rows = form == 1 ? 0 : 1;
        if (s.d.io == IO_C2C && !s.d.xfast && s.d.n_outer == 1 && s.d.in_a.estride == 1 && s.d.out_a.estride == 1 &&
            tc_rows_config(n, tc)) {
            // contiguous C2C rows: the warp-specialised row pipeline
            size_t smem = 0;
            const void *fn = tc_rows_kernel_fn(n, fmt_rows, s.forward, &smem);
            if (fn) {
                TablePtr fa = get_tc_matrix(tc.n1, fmt_rows, fwd, device, &err, 1);
                if (!fa) return false;
                TablePtr fb = tc.n2 == tc.n1 ? fa : get_tc_matrix(tc.n2, fmt_rows, fwd, device, &err, 1);
                if (!fb) return false;
                const float2 *tw = table(n, n);
                if (!tw) return false;
                p.tables.push_back(fa);
                p.tables.push_back(fb);
                const int64_t tiles = (s.d.n_cols + tc.tb - 1) / tc.tb;
                const int per_sm = std::max(1, kernel_blocks_per_sm(fn, kTcRowThreads, smem));
                s.grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(tiles, int64_t(per_sm) * sm_count(device))));
                s.d.tb = tc.tb;
                s.has_row = false;
                s.row_fn = nullptr;
                s.tc_fmt = fmt_rows;
                s.tc_kind = 1;
                s.tc_mat[0] = reinterpret_cast<const uint16_t *>(fa->ptr);
                s.tc_mat[1] = reinterpret_cast<const uint16_t *>(fb->ptr);
                s.tc_tw = tw;
                return true;
            }
        }
        if (!tc_config(n, tc)) return true;
        const int fmt = form == 1 ? 0 : 1;
        size_t smem = 0;
        const void *fn = tc_kernel(n, fmt, s.forward, &smem);
        if (!fn) return true;
        TablePtr m1 = get_tc_matrix(tc.n1, fmt, fwd, device, &err);
        if (!m1) return false;
        TablePtr m2 = tc.n2 == tc.n1 ? m1 : get_tc_matrix(tc.n2, fmt, fwd, device, &err);
        if (!m2) return false;
        const float2 *tw = table(n, n);
        if (!tw) return false;
        p.tables.push_back(m1);
        p.tables.push_back(m2);
        TileDesc &d = s.d;
        d.tb = tc.tb;
        d.tpt = 128 / tc.tb;
        d.pitch = ((n - 1) + ((n - 1) >> 4) + 1) | 1;
        d.tiles_per_outer = (d.n_cols + d.tb - 1) / d.tb;
        d.num_tiles = d.tiles_per_outer * d.n_outer;
        const int per_sm = tc_tile_blocks_per_sm(fn, smem);
        s.grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(d.num_tiles, int64_t(per_sm) * sm_count(device))));
        s.has_row = false;
        s.row_fn = nullptr;
        s.tc_fmt = fmt;
        s.tc_mat[0] = reinterpret_cast<const uint16_t *>(m1->ptr);
        s.tc_mat[1] = reinterpret_cast<const uint16_t *>(m1->ptr + int64_t(64) * tc.n1);
        s.tc_mat[2] = reinterpret_cast<const uint16_t *>(m2->ptr);
        s.tc_mat[3] = reinterpret_cast<const uint16_t *>(m2->ptr + int64_t(64) * tc.n2);
        s.tc_tw = tw;
        return true;
    }

    // TMA-pipelined persistent variant for contiguous rows: two staging
    // buffers per CTA, each large enough for a tile in its HBM layout and in
    // the padded work layout.
    void add_row_variant(Step &s, const TileCfg &c0, int64_t in_dist, int64_t out_dist)
    {
        const int64_t rows = s.d.n_cols;
        TileCfg c = c0;
        const StaticKernel *sk = find_static_kernel(s.d.n, s.d.io);
        const float2 *stw = nullptr;
        if (sk) {
            TablePtr t = get_stage_table(*sk, device, &err);
            if (t) {
                p.tables.push_back(t);
                stw = t->ptr;
                c.tpt = sk->tpt;
                // 128-thread CTAs: the barriers between stages span 4 warps (about 6 CTAs per SM
                // rather than 3 of 8 warps), measured 5-8 % faster on 1500- to 2048-point rows
                c.tb = std::max(1, std::min(kStaticRowThreads / sk->tpt, static_cast<int>(std::min<int64_t>(rows, 64))));
                // static engines are built for 256-thread CTAs (512 only when one transform needs them)
                const int cap = sk->tpt <= 256 ? 256 : kMaxThreads;
                while (c.tb > 1 && c.tb * c.tpt > cap) c.tb /= 2;
            } else {
                sk = nullptr;
                err.clear();
            }
        }
        for (int tb = c.tb; tb >= 1; tb /= 2) {
            // staged tile (one element more when tiles may start at an odd element) or padded work rows
            int64_t buf = std::max<int64_t>(tb * in_dist + (tb * in_dist) % 2, int64_t(tb) * c.pitch);
            buf = (buf + 1) / 2 * 2;
            TileDesc d = s.d;
            d.tb = tb;
            d.num_tiles = (rows + tb - 1) / tb;
            d.tiles_per_outer = d.num_tiles;
            d.in_a = Addr{in_dist, 0, 1, 0, 0};
            d.out_a = Addr{out_dist, 0, 1, 0, 0};
            d.g_ns = buf;
            d.tpt = c.tpt;
            if (sk) d.row_bufs = sk->row_bufs;
            if (row_kernel_smem(d) > static_cast<size_t>(kMaxSmemBytes)) continue;
            const void *fn = nullptr;
            if (sk) {
                const int io = d.io == IO_C2C ? 0 : (d.io == IO_R2C_PACKED ? 1 : 2);
                fn = sk->fn[s.forward ? 1 : 0][io];
                d.stw = stw;
            }
            const int per_sm = fn ? kernel_blocks_per_sm(fn, tb * c.tpt, row_kernel_smem(d))
                                  : row_kernel_blocks_per_sm(d, s.maxe, s.forward);
            if (per_sm <= 0) continue;
            s.has_row = true;
            s.row_fn = fn;
            s.rd = d;
            s.row_grid = static_cast<int>(std::min<int64_t>(d.num_tiles, int64_t(per_sm) * sm_count(device)));
            return;
        }
    }

    // The first workspace slot that is none of `used` (slot 3 is kept for the
    // planar redirect and only handed out when 0-2 are all taken).
    Buf free_ws(std::initializer_list<Buf> used)
    {
        for (Buf c : {Buf::kWs0, Buf::kWs1, Buf::kWs2, Buf::kWs3}) {
            bool taken = false;
            for (Buf u : used) taken = taken || u == c;
            if (!taken) return c;
        }
        return Buf::kWs3;
    }
    Buf other_ws(Buf a, Buf b) { return free_ws({a, b}); }

    // Multi-pass Stockham C2C of length F along one axis of [outer][F][inner]
    // (inner = 1: contiguous rows; src rows at in_dist, dst rows at out_dist
    // complex elements).  Pass i is a column-tile launch over the F / R_i
    // Stockham columns of every transform: tile column C = c * inner + j is
    // Stockham column c of transform j, so a tile of consecutive C reads
    // consecutive addresses whenever inner > 1.  The pass twiddle W_F^(r c ns)
    // comes from the two-level table; intermediates go to workspace slots that
    // are neither src nor dst.
    bool add_multipass(int64_t F, int64_t outer, int64_t in_dist, int64_t out_dist, Buf src, Buf dst,
                       int64_t inner = 1)
    {
        std::vector<int> passes;
        int parts = 2;
        while (!split_passes(F, parts, passes)) {
            if (++parts > 6) {
                err = "length " + std::to_string(F) + " cannot be split into shared-memory passes";
                return false;
            }
        }
        const float2 *lo = nullptr, *hi = nullptr;
        int log2l = 0;
        if (!table2(F, lo, hi, log2l)) return false;
        Buf cur = src;
        int64_t cur_dist = in_dist;
        int64_t ns = 1;
        struct Flag {
            bool &f;
            explicit Flag(bool &x) : f(x) { f = true; }
            ~Flag() { f = false; }
        } flag(in_multipass);
        for (size_t i = 0; i < passes.size(); i++) {
            const int rp = passes[i];
            const bool last = i + 1 == passes.size();
            Buf nxt = last ? dst : other_ws(cur, dst);
            const int64_t nxt_dist = last ? out_dist : F * inner;
            if (!last) need_ws(nxt, size_t(outer) * F * inner * sizeof(float2));
            const float2 *tw = table(rp, rp);
            if (!tw) return false;
            Addr ia{cur_dist, 1, (F / rp) * inner, 0, 0};
            Addr oa{nxt_dist, 1, ns * inner, ns * inner, ns * inner * (rp - 1)};
            std::ostringstream w;
            w << "pass " << i << " radix " << rp << " of " << F << " (Ns=" << ns << ")";
            if (inner > 1) w << " strided x" << inner;
            if (!add_tile(IO_C2C, rp, 1, tw, true, outer, (F / rp) * inner, ia, oa, cur, nxt, w.str())) return false;
            TileDesc &d = p.steps.back().d;
            d.g_twiddle = ns > 1 ? 1 : 0;
            d.g_ns = ns;
            d.g_div = inner;
            d.g_step = F / (ns * rp);
            d.g_lo = lo;
            d.g_hi = hi;
            d.g_log2l = log2l;
            ns *= rp;
            cur = nxt;
            cur_dist = nxt_dist;
        }
        return true;
    }

    // Bluestein (chirp-z) N-point transform of contiguous rows for lengths
    // whose prime factors the codelets do not cover: a length-M circular
    // convolution (M = 2^k >= 2N-1) done as two M-point FFT launches with the
    // chirp pre/post multiplies and the precomputed FFT of the chirp fused in.
    // kind: 0 C2C, 1 R2C (real in, N/2+1 out), 2 C2R (N/2+1 in, real out).
    bool add_bluestein(int kind, int64_t n, int64_t rows, int64_t in_dist, int64_t out_dist, Buf src, Buf dst)
    {
        int64_t m = 1;
        while (m < 2 * n - 1) m *= 2;
        if (m > kMaxBluesteinM) {
            err = "length " + std::to_string(n) + " needs Bluestein with M > " + std::to_string(kMaxBluesteinM);
            return false;
        }
        const bool multipass = m > kMaxRowN;
        auto chirp = std::make_shared<DeviceTable>();
        auto bmul = std::make_shared<DeviceTable>();
        chirp->device = bmul->device = device;
        chirp->count = n;
        bmul->count = m;
        cudaError_t e = cudaMalloc(&chirp->ptr, sizeof(float2) * n);
        if (e == cudaSuccess) e = cudaMalloc(&bmul->ptr, sizeof(float2) * m);
        if (e == cudaSuccess) e = fill_chirp(chirp->ptr, n, fwd, 0);
        if (e == cudaSuccess) e = fill_bluestein_b(bmul->ptr, chirp->ptr, n, m, 0);
        const float2 *twm = multipass ? nullptr : table(m, m);
        if (!multipass && !twm) return false;
        if (e == cudaSuccess && multipass) {
            e = fft_in_place_once(bmul->ptr, m);
        } else if (e == cudaSuccess) {
            // FFT_M of b in place (one row, forward), then fold in the 1/M of the inverse
            Step tmp;
            if (!make_tile(tmp, IO_C2C, static_cast<int>(m), 1, twm, false, 1, 1, Addr{0, m, 1, 0, 0},
                           Addr{0, m, 1, 0, 0}, Buf::kUserIn, Buf::kUserOut, "bluestein table"))
                return false;
            tmp.d.in = bmul->ptr;
            tmp.d.out = bmul->ptr;
            e = launch_tile(tmp.d, tmp.maxe, true, tmp.grid, 0);
        }
        if (e == cudaSuccess) e = scale_table(bmul->ptr, m, 1.0f / static_cast<float>(m), 0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
        if (e != cudaSuccess) {
            err = std::string("twiddle table: ") + cudaGetErrorString(e);
            cudaGetLastError();
            return false;
        }
        p.tables.push_back(chirp);
        p.tables.push_back(bmul);
        if (multipass) return add_bluestein_steps(kind, n, m, rows, in_dist, out_dist, src, dst, chirp->ptr, bmul->ptr);
        Buf ws = other_ws(src, dst);
        need_ws(ws, size_t(rows) * m * sizeof(float2));
        std::ostringstream w;
        w << "Bluestein n=" << n << " via M=" << m << " rows=" << rows;
        Step s1, s2;
        if (!make_tile(s1, IO_BLUE_PRE, static_cast<int>(m), 1, twm, false, 1, rows, Addr{0, in_dist, 1, 0, 0},
                       Addr{0, m, 1, 0, 0}, src, ws, w.str() + " (chirp, FFT, multiply)"))
            return false;
        if (!make_tile(s2, IO_BLUE_POST, static_cast<int>(m), 1, twm, false, 1, rows, Addr{0, m, 1, 0, 0},
                       Addr{0, out_dist, 1, 0, 0}, ws, dst, w.str() + " (inverse FFT, chirp)"))
            return false;
        for (Step *st : {&s1, &s2}) {
            st->d.chirp = chirp->ptr;
            st->d.bmul = bmul->ptr;
            st->d.blue_n = static_cast<int>(n);
            st->d.blue_kind = kind;
        }
        s1.forward = true;
        s2.forward = false;
        p.steps.push_back(s1);
        p.steps.push_back(s2);
        return true;
    }

    // Forward FFT of one length-m row in place at plan time (the Bluestein
    // filter of a multi-pass convolution): a one-row plan of this planner run
    // with a temporary workspace.
    cudaError_t fft_in_place_once(float2 *row, int64_t m)
    {
        Plan tmp;
        tmp.device = device;
        tmp.fft_type = 0x10;
        tmp.direction = 0x10;
        tmp.sizes = {m};
        tmp.batch = 1;
        const std::string why = build_plan_1d(tmp);
        if (!why.empty()) return cudaErrorInvalidValue;
        void *ws = nullptr;
        cudaError_t e = tmp.ws_bytes ? cudaMalloc(&ws, tmp.ws_bytes) : cudaSuccess;
        if (e == cudaSuccess) e = execute_steps(tmp, tmp.steps, row, row, ws, 0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
        if (ws) cudaFree(ws);
        return e;
    }

    // Bluestein with a convolution length m too long for one CTA: chirp
    // multiply into workspace A, forward multi-pass FFT A -> B, pointwise
    // product with the transformed filter, inverse multi-pass FFT B -> A, chirp
    // multiply into the destination.
    bool add_bluestein_steps(int kind, int64_t n, int64_t m, int64_t rows, int64_t in_dist, int64_t out_dist, Buf src,
                             Buf dst, const float2 *chirp, const float2 *bmul)
    {
        const Buf A = free_ws({src, dst}), B = free_ws({src, dst, A});
        need_ws(A, size_t(rows) * m * sizeof(float2));
        need_ws(B, size_t(rows) * m * sizeof(float2));
        std::ostringstream w;
        w << "Bluestein n=" << n << " via M=" << m << " rows=" << rows << " (multi-pass)";
        Step pre;
        pre.kind = StepKind::kBluePre;
        pre.src = src;
        pre.dst = A;
        pre.rows = rows;
        pre.m = m;
        pre.src_dist = in_dist;
        pre.d.blue_n = static_cast<int>(n);
        pre.d.blue_kind = kind;
        pre.d.chirp = chirp;
        pre.what = w.str() + ": chirp multiply";
        p.steps.push_back(pre);
        const bool plan_fwd = fwd;
        fwd = true;
        bool ok = add_multipass(m, rows, m, m, A, B);
        if (ok) {
            Step mul = pre;
            mul.kind = StepKind::kPointMul;
            mul.src = mul.dst = B;
            mul.d.bmul = bmul;
            mul.what = w.str() + ": filter product";
            p.steps.push_back(mul);
            fwd = false;
            ok = add_multipass(m, rows, m, m, B, A);
        }
        fwd = plan_fwd;
        if (!ok) return false;
        Step post = pre;
        post.kind = StepKind::kBluePost;
        post.src = A;
        post.dst = dst;
        post.dst_dist = out_dist;
        post.what = w.str() + ": chirp multiply";
        p.steps.push_back(post);
        return true;
    }

    // C2C along one axis of a contiguous tensor viewed as [outer][n][inner].
    bool axis_c2c(int64_t n, int64_t outer, int64_t inner, Buf src, Buf dst)
    {
        if (n == 1) {
            // identity along this axis; still move the data when src != dst
            if (src == dst) return true;
            return add_copy(outer * inner, src, dst);
        }
        std::ostringstream w;
        w << "C2C axis n=" << n << " outer=" << outer << " inner=" << inner;
        std::vector<int> probe;
        const bool smooth = factor_radices(n, probe);
        if (inner == 1 && !smooth) return add_bluestein(0, n, outer, n, n, src, dst);
        if (inner == 1) {
            // rows up to 8192 points run as one tile; longer rows as two double-buffered
            // passes, which keep ~16 columns per tile and overlap loads with compute
            // (up to 16384 points where a compile-time engine exists: one row per CTA)
            if (n <= std::min<int64_t>(kMaxSingleTileC2C, p.max_row_n) ||
                (n <= std::min<int64_t>(kMaxRowN, p.max_row_n) && find_static_kernel(n, IO_C2C))) {
                const float2 *tw = table(n, n);
                if (!tw) return false;
                Addr a{0, n, 1, 0, 0};
                return add_tile(IO_C2C, static_cast<int>(n), 1, tw, false, 1, outer, a, a, src, dst, w.str());
            }
            return add_multipass(n, outer, n, n, src, dst);
        }
        if (!smooth) {
            err = "strided axis of length " + std::to_string(n) + " has a prime factor above 13";
            return false;
        }
        // Through transposes: the tensor-core form of lengths with the row pipeline,
        // and FP32 axes above 1024 points without a TMA column engine, whose column
        // tiles shrink to 2-4 columns (16-32-byte row runs).  Measured, 2D C2C
        // (column axis strided; us, column kernel -> transposes): 4096^2 x 2
        // 539 -> 391, 8192 x 1024 x 4 690 -> 419, 3000 x 1024 x 8 605 -> 454,
        // 6561 x 512 x 8 548 -> 459, 1500^2 x 12 446 -> 345; 1000^2 x 64 1146 -> 1330
        // and 2048^2 x 8 244 -> 374 (TMA column engine) stay on column tiles.
        // Vertical 1D plans keep their column tiles (complex32 data converts in
        // the first and last tile steps).
        if (!in_multipass && p.fft_type != 0x30) {
            TcConfig tcc;
            const int form = tc_form(n);
            const bool tc = (form == 1 || form == 2) && tc_rows_config(static_cast<int>(n), tcc);
            const bool slow_columns =
                form == 0 && !p.vertical && n > 1024 && n <= kMaxStridedTile &&
                !(col_pipe_has_engine(static_cast<int>(n)) && inner % 2 == 0);
            if (tc || slow_columns) return add_transposed_axis(n, outer, inner, src, dst);
        }
        TileCfg c;
        if (n > kMaxStridedTile || !choose_cfg(static_cast<int>(n), true, inner, c, err)) {
            // longer strided axes: multi-pass Stockham with 16-column tiles along the
            // contiguous inner dimension (the reference's stride core plans powers of
            // two up to 262144, core/fft/fftcore/fft_core_stride.cpp:119-161)
            err.clear();
            return add_multipass(n, outer, n * inner, n * inner, src, dst, inner);
        }
        const float2 *tw = table(n, n);
        if (!tw) return false;
        Addr a{n * inner, 1, inner, 0, 0};
        return add_tile(IO_C2C, static_cast<int>(n), 1, tw, true, outer, inner, a, a, src, dst, w.str());
    }

    // Plain copy expressed as a length-1 transform (keeps one kernel family).
    bool add_copy(int64_t count, Buf src, Buf dst)
    {
        const float2 *tw = table(1, 1);
        if (!tw) return false;
        Addr a{0, 1, 1, 0, 0};
        return add_tile(IO_C2C, 1, 1, tw, false, 1, count, a, a, src, dst, "copy");
    }

    // R2C along contiguous rows of real length n (output rows of n/2+1 bins).
    bool rows_r2c(int64_t n, int64_t rows, Buf src, Buf dst)
    {
        const int64_t h = n / 2 + 1;
        std::vector<int> probe;
        if (!factor_radices(n % 2 == 0 ? n / 2 : n, probe)) return add_bluestein(1, n, rows, n, h, src, dst);
        std::ostringstream w;
        w << "R2C rows n=" << n << " rows=" << rows;
        if (n % 2 == 0 && n / 2 <= kMaxRowN) {
            const int m = static_cast<int>(n / 2);
            const float2 *tw = table(n, n);
            if (!tw) return false;
            Addr ia{0, m, 1, 0, 0};  // real row viewed as m float pairs
            Addr oa{0, h, 1, 0, 0};
            return add_tile(IO_R2C_PACKED, m, 2, tw, false, 1, rows, ia, oa, src, dst, w.str());
        }
        if (n % 2 == 1 && n <= kMaxRowN) {
            const float2 *tw = table(n, n);
            if (!tw) return false;
            Addr ia{0, n, 1, 0, 0};
            Addr oa{0, h, 1, 0, 0};
            return add_tile(IO_R2C_FULL, static_cast<int>(n), 1, tw, false, 1, rows, ia, oa, src, dst, w.str());
        }
        if (n % 2 == 0) {
            // packed multi-pass FFT of n/2 points into a workspace, then the post-twiddle
            const int64_t m = n / 2;
            Buf z = other_ws(src, dst);
            need_ws(z, size_t(rows) * m * sizeof(float2));
            if (!add_multipass(m, rows, m, m, src, z)) return false;
            Step s;
            s.kind = StepKind::kR2CPost;
            s.forward = fwd;
            s.src = z;
            s.dst = dst;
            s.rows = rows;
            s.m = m;
            s.src_dist = m;
            s.dst_dist = h;
            s.what = "R2C post-twiddle n=" + std::to_string(n);
            if (!table2(n, s.lo, s.hi, s.log2l)) return false;
            p.steps.push_back(s);
            return true;
        }
        err = "odd real length above " + std::to_string(kMaxRowN) + " is not supported";
        return false;
    }

    // C2R along contiguous rows (input rows of n/2+1 bins, output n reals).
    bool rows_c2r(int64_t n, int64_t rows, Buf src, Buf dst)
    {
        const int64_t h = n / 2 + 1;
        std::vector<int> probe;
        if (!factor_radices(n % 2 == 0 ? n / 2 : n, probe)) return add_bluestein(2, n, rows, h, n, src, dst);
        std::ostringstream w;
        w << "C2R rows n=" << n << " rows=" << rows;
        if (n % 2 == 0 && n / 2 <= kMaxRowN) {
            const int m = static_cast<int>(n / 2);
            const float2 *tw = table(n, n);
            if (!tw) return false;
            Addr ia{0, h, 1, 0, 0};
            Addr oa{0, m, 1, 0, 0};
            return add_tile(IO_C2R_PACKED, m, 2, tw, false, 1, rows, ia, oa, src, dst, w.str());
        }
        if (n % 2 == 1 && n <= kMaxRowN) {
            const float2 *tw = table(n, n);
            if (!tw) return false;
            Addr ia{0, h, 1, 0, 0};
            Addr oa{0, n, 1, 0, 0};
            return add_tile(IO_C2R_FULL, static_cast<int>(n), 1, tw, false, 1, rows, ia, oa, src, dst, w.str());
        }
        if (n % 2 == 0) {
            const int64_t m = n / 2;
            Buf z = other_ws(src, dst);
            need_ws(z, size_t(rows) * m * sizeof(float2));
            Step s;
            s.kind = StepKind::kC2RPre;
            s.forward = fwd;
            s.src = src;
            s.dst = z;
            s.rows = rows;
            s.m = m;
            s.src_dist = h;
            s.dst_dist = m;
            s.what = "C2R pre-twiddle n=" + std::to_string(n);
            if (!table2(n, s.lo, s.hi, s.log2l)) return false;
            p.steps.push_back(s);
            return add_multipass(m, rows, m, m, z, dst);
        }
        err = "odd real length above " + std::to_string(kMaxRowN) + " is not supported";
        return false;
    }
};

std::string finish(Plan &p, Builder &b, bool ok)
{
    if (!ok) {
        p.steps.clear();
        return b.err.empty() ? std::string("planning failed") : b.err;
    }
    if (p.fft_type == 0x30 && !b.make_planar()) {
        p.steps.clear();
        return b.err;
    }
    p.ws_bytes = 0;
    for (size_t b : p.ws_buf_bytes) p.ws_bytes += (b + 255) / 256 * 256;
    return std::string();
}

}  // namespace

// Pass lengths of a multi-pass transform of length F (the split add_multipass
// makes), empty if F cannot be split.
std::vector<int> multipass_split(int64_t F)
{
    std::vector<int> passes;
    for (int parts = 2; parts <= 6; parts++)
        if (split_passes(F, parts, passes)) return passes;
    return {};
}

bool valid_radices(const std::vector<int> &r, int64_t n)
{
    int64_t prod = 1;
    for (int x : r) {
        if (x < 2 || x > 16 || x == 14 || x == 15) return false;
        prod *= x;
    }
    return prod == n && r.size() <= static_cast<size_t>(kMaxStages);
}

bool factor_radices(int64_t n, std::vector<int> &radices)
{
    radices.clear();
    if (n < 1) return false;
    int64_t m = n;
    int twos = 0;
    while (m % 2 == 0) {
        m /= 2;
        twos++;
    }
    if (twos > 0) {
        const int s = (twos + 3) / 4;
        const int base = twos / s, extra = twos % s;
        for (int i = 0; i < s; i++) radices.push_back(1 << (base + (i < extra ? 1 : 0)));
    }
    // odd part: pairs of 3 as radix 9, then the primes
    std::vector<int> odd;
    for (int p : {13, 11, 7, 5}) {
        while (m % p == 0) {
            odd.push_back(p);
            m /= p;
        }
    }
    while (m % 9 == 0) {
        odd.push_back(9);
        m /= 9;
    }
    if (m % 3 == 0) {
        // a single 3 (or a 5 below) joins a power-of-two radix when that keeps it <= 16: 4*3, 2*3, 2*5
        m /= 3;
        auto it = std::find(radices.begin(), radices.end(), 4);
        if (it == radices.end()) it = std::find(radices.begin(), radices.end(), 2);
        if (it != radices.end()) *it *= 3;
        else odd.push_back(3);
    }
    for (int &r : odd) {
        if (r != 5) continue;
        auto it = std::find(radices.begin(), radices.end(), 2);
        if (it != radices.end()) {
            *it = 10;
            r = 1;
        }
    }
    for (int r : odd)
        if (r > 1) radices.push_back(r);
    return m == 1;
}

bool Plan::forward() const { return direction == 0x10; }

std::string build_plan_1d(Plan &p)
{
    Builder b(p);
    const int64_t n = p.sizes[0];
    bool ok = false;
    switch (p.fft_type) {
        case 0x30:  // C2C on separated planes (converted after planning)
        case 0x10:  // C2C
            ok = p.vertical ? b.axis_c2c(n, 1, p.batch, Buf::kUserIn, Buf::kUserOut)
                            : b.axis_c2c(n, p.batch, 1, Buf::kUserIn, Buf::kUserOut);
            break;
        case 0x12:  // R2C
            ok = b.rows_r2c(n, p.batch, Buf::kUserIn, Buf::kUserOut);
            break;
        case 0x11:  // C2R
            ok = b.rows_c2r(n, p.batch, Buf::kUserIn, Buf::kUserOut);
            break;
        default:
            b.err = "unsupported transform type";
    }
    return finish(p, b, ok);
}

std::string build_plan_2d(Plan &p)
{
    Builder b(p);
    const int64_t B = p.batch, X = p.sizes[0], Y = p.sizes[1];
    const int64_t Yh = Y / 2 + 1;
    bool ok = false;
    switch (p.fft_type) {
        case 0x30:
        case 0x10:
            ok = b.axis_c2c(Y, B * X, 1, Buf::kUserIn, Buf::kUserOut) &&
                 b.axis_c2c(X, B, Y, Buf::kUserOut, Buf::kUserOut);
            break;
        case 0x12:
            ok = b.rows_r2c(Y, B * X, Buf::kUserIn, Buf::kUserOut) &&
                 b.axis_c2c(X, B, Yh, Buf::kUserOut, Buf::kUserOut);
            break;
        case 0x11:
            b.need_ws(Buf::kWs0, size_t(B) * X * Yh * sizeof(float2));
            ok = b.axis_c2c(X, B, Yh, Buf::kUserIn, Buf::kWs0) && b.rows_c2r(Y, B * X, Buf::kWs0, Buf::kUserOut);
            break;
        default:
            b.err = "unsupported transform type";
    }
    return finish(p, b, ok);
}

std::string build_plan_3d(Plan &p)
{
    Builder b(p);
    const int64_t B = p.batch, X = p.sizes[0], Y = p.sizes[1], Z = p.sizes[2];
    const int64_t Zh = Z / 2 + 1;
    bool ok = false;
    switch (p.fft_type) {
        case 0x30:
        case 0x10:
            ok = b.axis_c2c(Z, B * X * Y, 1, Buf::kUserIn, Buf::kUserOut) &&
                 b.axis_c2c(Y, B * X, Z, Buf::kUserOut, Buf::kUserOut) &&
                 b.axis_c2c(X, B, Y * Z, Buf::kUserOut, Buf::kUserOut);
            break;
        case 0x12:
            ok = b.rows_r2c(Z, B * X * Y, Buf::kUserIn, Buf::kUserOut) &&
                 b.axis_c2c(Y, B * X, Zh, Buf::kUserOut, Buf::kUserOut) &&
                 b.axis_c2c(X, B, Y * Zh, Buf::kUserOut, Buf::kUserOut);
            break;
        case 0x11:
            b.need_ws(Buf::kWs0, size_t(B) * X * Y * Zh * sizeof(float2));
            ok = b.axis_c2c(X, B, Y * Zh, Buf::kUserIn, Buf::kWs0) &&
                 b.axis_c2c(Y, B * X, Zh, Buf::kWs0, Buf::kWs0) &&
                 b.rows_c2r(Z, B * X * Y, Buf::kWs0, Buf::kUserOut);
            break;
        default:
            b.err = "unsupported transform type";
    }
    return finish(p, b, ok);
}

// Inverse STFT (core/fft/istft.cpp:495-575): the reference transposes
// [channel, n_fft, frames] to [channel, frames, n_fft] and runs an INVERSE C2C
// plan over the frames; here one column-tile step reads the frequency-major
// input in place and writes the frames in [channel][frame][n_fft] order into
// workspace slot 0, where the overlap-add kernel reads them.
std::string build_plan_istft(Plan &p)
{
    Builder b(p);
    const int64_t n = p.istft_nfft, F = p.istft_frames, C = p.istft_channel;
    std::vector<int> probe;
    if (!factor_radices(n, probe)) return "ISTFT length " + std::to_string(n) + " has a prime factor above 13";
    const float2 *tw = b.table(n, n);
    if (!tw) return b.err;
    std::ostringstream w;
    w << "ISTFT frames: inverse C2C n=" << n << " channels=" << C << " frames=" << F;
    b.need_ws(Buf::kWs0, size_t(C) * F * n * sizeof(float2));
    const Addr ia{n * F, 1, F, 0, 0};  // element e of frame f of channel c at c n F + f + e F
    const Addr oa{F * n, n, 1, 0, 0};  // written at c F n + f n + e
    const bool ok = b.add_tile(IO_C2C, static_cast<int>(n), 1, tw, true, C, F, ia, oa, Buf::kUserIn, Buf::kWs0, w.str());
    return finish(p, b, ok);
}

std::string describe_plan(const Plan &p)
{
    std::ostringstream o;
    o << "steps=" << p.steps.size() << " workspace=" << p.ws_bytes << "\n";
    for (const Step &s : p.steps) {
        o << "  [" << static_cast<int>(s.src) << "->" << static_cast<int>(s.dst) << "] " << s.what;
        if (s.kind == StepKind::kTile) {
            o << (s.cp_fn ? " [TMA column tiles, static engine]"
                          : (s.db ? (s.db_fn ? " [double-buffered, static engine]" : " [double-buffered]") : ""))
              << " n=" << s.d.n
              << " radices=";
            for (int i = 0; i < s.d.nstages; i++) o << (i ? "x" : "") << s.d.radix[i];
            o << " tb=" << s.d.tb << " tpt=" << s.d.tpt << " tiles=" << s.d.num_tiles << " grid=" << s.grid
              << " smem=" << s.d.tb * s.d.pitch * 8;
            if (s.tc_fmt >= 0)
                o << " | tensor-core " << (s.tc_fmt == 0 ? "fp16x3" : "bf16x3") << (s.tc_kind == 1 ? " rows" : " tile")
                  << " tb=" << s.d.tb << " grid=" << s.grid;
            if (s.has_row)
                o << " | row-pipelined" << (s.row_fn ? " static" : "") << " tb=" << s.rd.tb << " tpt=" << s.rd.tpt
                  << " grid=" << s.row_grid << " smem=" << row_kernel_smem(s.rd);
        }
        o << "\n";
    }
    return o.str();
}

}  // namespace sipfft
