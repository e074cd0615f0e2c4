// Device-side runtime of the planner: the process-wide twiddle-table cache
// and the step executor.
//
// Reference counterparts: FFTensorCache (core/fft/utils/fftensor_cache.cpp:20-92,
// coefficient tensors shared across plans through weak pointers, built on the
// host and copied to the device at plan time) and asdFftExecV2
// (core/fft/fft_api.cpp:1001-1045, ping-pong of intermediate caches carved
// from the caller's workspace).  Here the tables are generated directly on the
// GPU in FP64 and rounded to FP32, and intermediate buffers are two fixed
// slots of the caller's workspace.
#include <algorithm>
#include <map>
#include <tuple>

#include "sipfft_internal.h"

namespace sipfft {

DeviceTable::~DeviceTable()
{
    if (ptr) {
        int cur = 0;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != device) cudaSetDevice(device);
        cudaFree(ptr);
        if (cur != device) cudaSetDevice(cur);
        cudaGetLastError();  // a torn-down context at exit is not an error worth reporting
    }
}

namespace {
std::mutex g_table_mu;
std::map<std::tuple<int, int64_t, int64_t, int64_t>, std::weak_ptr<DeviceTable>> g_tables;
}  // namespace

TablePtr get_table(int64_t count, int64_t denom, int64_t mult, int device, std::string *err)
{
    std::lock_guard<std::mutex> lock(g_table_mu);
    auto key = std::make_tuple(device, count, denom, mult);
    auto it = g_tables.find(key);
    if (it != g_tables.end()) {
        if (TablePtr t = it->second.lock()) return t;
    }
    auto t = std::make_shared<DeviceTable>();
    t->count = count;
    t->device = device;
    cudaError_t e = cudaMalloc(&t->ptr, sizeof(float2) * static_cast<size_t>(count));
    if (e == cudaSuccess) e = fill_twiddles(t->ptr, count, denom, mult, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        if (err) *err = std::string("twiddle table: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return nullptr;
    }
    g_tables[key] = t;
    return t;
}

TablePtr get_stage_table(const StaticKernel &k, int device, std::string *err)
{
    return get_stage_table(k.radix, k.nstages, device, err);
}

TablePtr get_stage_table(const int *radix, int nstages, int device, std::string *err)
{
    static std::mutex mu;
    static std::map<std::pair<int, std::string>, std::weak_ptr<DeviceTable>> cache;  // (device, radix sequence)
    std::lock_guard<std::mutex> lock(mu);
    std::string seq;
    for (int s = 0; s < nstages; s++) seq += std::to_string(radix[s]) + ",";
    auto key = std::make_pair(device, seq);
    auto it = cache.find(key);
    if (it != cache.end()) {
        if (TablePtr t = it->second.lock()) return t;
    }
    auto t = std::make_shared<DeviceTable>();
    t->count = std::max<int64_t>(1, stage_twiddle_count(radix, nstages));
    t->device = device;
    cudaError_t e = cudaMalloc(&t->ptr, sizeof(float2) * static_cast<size_t>(t->count));
    if (e == cudaSuccess) e = fill_stage_twiddles(t->ptr, radix, nstages, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        if (err) *err = std::string("twiddle table: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return nullptr;
    }
    cache[key] = t;
    return t;
}

TablePtr get_tc_matrix(int N, int fmt, bool fwd, int device, std::string *err, int layout)
{
    static std::mutex mu;
    // (device, N, fmt, fwd, layout)
    static std::map<std::tuple<int, int, int, int, int>, std::weak_ptr<DeviceTable>> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_tuple(device, N, fmt, fwd ? 1 : 0, layout);
    auto it = cache.find(key);
    if (it != cache.end()) {
        if (TablePtr t = it->second.lock()) return t;
    }
    auto t = std::make_shared<DeviceTable>();
    // hi + lo 16-bit parts: 2 x (128 x 2N) (layout 0) or 2 x (2N x 2N) (layout 1)
    const int64_t half = layout == 0 ? int64_t(64) * N : int64_t(N) * N;  // float2 units: 8 N^2 bytes per part
    t->count = 2 * half;
    t->device = device;
    cudaError_t e = cudaMalloc(&t->ptr, sizeof(float2) * static_cast<size_t>(t->count));
    if (e == cudaSuccess) {
        uint16_t *hi = reinterpret_cast<uint16_t *>(t->ptr);
        uint16_t *lo = reinterpret_cast<uint16_t *>(t->ptr + half);
        e = layout == 0 ? fill_tc_matrix(hi, lo, N, fmt, fwd, 0) : fill_tc_bmatrix(hi, lo, N, fmt, fwd, 0);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        if (err) *err = std::string("twiddle table: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return nullptr;
    }
    cache[key] = t;
    return t;
}

namespace {
thread_local std::string t_last_error;
}  // namespace

void set_last_error(const std::string &msg) { t_last_error = msg; }
const std::string &last_error() { return t_last_error; }

namespace {
std::mutex g_dev_mu;
std::map<int, int *> g_err_words;
std::map<int, int> g_sms;
}  // namespace

int *device_error_word(int device)
{
    std::lock_guard<std::mutex> lock(g_dev_mu);
    auto it = g_err_words.find(device);
    if (it != g_err_words.end()) return it->second;
    int *w = nullptr;
    if (cudaMalloc(&w, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    cudaMemset(w, 0, sizeof(int));
    g_err_words[device] = w;
    return w;
}

cudaError_t configure_kernels(int device)
{
    static std::mutex mu;
    static std::map<int, bool> done;
    std::lock_guard<std::mutex> lock(mu);
    if (done[device]) return cudaSuccess;
    std::vector<const void *> fns;
    tile_kernel_fns(fns);
    row_kernel_fns(fns);
    static_kernel_fns(fns);
    tc_kernel_fns(fns);
    tc_rows_kernel_fns(fns);
    col_pipe_kernel_fns(fns);
    for (const void *fn : fns) {
        cudaError_t e = allow_max_dynamic_smem(fn);
        if (e != cudaSuccess) return e;
    }
    // the error word is allocated here, at set-up, never inside a capture
    if (!device_error_word(device)) return cudaErrorMemoryAllocation;
    done[device] = true;
    return cudaSuccess;
}

int sm_count(int device)
{
    std::lock_guard<std::mutex> lock(g_dev_mu);
    auto it = g_sms.find(device);
    if (it != g_sms.end()) return it->second;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        n = kB200Sms;
    }
    g_sms[device] = n;
    return n;
}

std::string complex32_steps(const Plan &p, std::vector<Step> &out)
{
    if (p.fft_type != 0x10 || p.sizes.size() != 1) return "complex32 data is supported for 1D C2C plans";
    if (p.precision != 0) return "complex32 data runs with FP32 stages only (precision mode 0)";
    out = p.steps;
    if (out.empty()) return "empty plan";
    for (size_t i = 0; i < out.size(); i++) {
        Step &s = out[i];
        if (s.kind != StepKind::kTile || s.d.io != IO_C2C || s.d.planar)
            return "complex32 data needs a plan of C2C tile steps (no Bluestein lengths)";
        if ((i == 0) != (s.src == Buf::kUserIn) || (i + 1 == out.size()) != (s.dst == Buf::kUserOut) ||
            s.src == Buf::kUserOut)
            return "complex32 data needs the user buffers to be read first and written last only";
    }
    for (Step *s : {&out.front(), &out.back()}) {
        // the first / last step run on the generic tile kernel, whose load and
        // store phases convert
        s->has_row = false;
        s->row_fn = nullptr;
        s->db = false;
        s->db_fn = nullptr;
        s->cp_fn = nullptr;
    }
    out.front().d.half_io |= 1;
    out.back().d.half_io |= 2;
    return std::string();
}

// Copy of a 1D row plan's steps re-targeted to `rows` (<= the planned
// batch) transforms, so one resident plan serves batches of any size.
bool scale_steps_to_rows(const Plan &p, int64_t rows, std::vector<Step> &out)
{
    if (p.sizes.size() != 1 || p.vertical || rows <= 0 || rows > p.batch) return false;
    out = p.steps;
    for (Step &s : out) {
        if (s.kind != StepKind::kTile) {
            s.rows = rows;
            continue;
        }
        TileDesc &d = s.d;
        if (d.n_outer == 1 && !d.xfast) {
            d.n_cols = rows;  // batched rows
            d.tiles_per_outer = (rows + d.tb - 1) / d.tb;
            d.num_tiles = d.tiles_per_outer;
        } else if (d.n_outer == p.batch) {
            d.n_outer = rows;  // multi-pass: one outer group per transform
            d.num_tiles = d.tiles_per_outer * rows;
        } else {
            return false;
        }
        s.grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(d.num_tiles, s.grid)));
        if (s.has_row) {
            TileDesc &r = s.rd;
            r.n_cols = rows;
            r.num_tiles = (rows + r.tb - 1) / r.tb;
            r.tiles_per_outer = r.num_tiles;
            s.row_grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(r.num_tiles, s.row_grid)));
        }
    }
    return true;
}

cudaError_t execute_plan(Plan &p, const void *in, void *out, cudaStream_t st, const float *in_im, float *out_im)
{
    return execute_steps(p, p.steps, in, out, p.workspace, st, in_im, out_im);
}

cudaError_t execute_steps(const Plan &p, const std::vector<Step> &steps, const void *in, void *out, void *workspace,
                          cudaStream_t st, const float *in_im, float *out_im)
{
    char *ws = static_cast<char *>(workspace);
    void *bufs[2 + kWsSlots] = {const_cast<void *>(in), out};
    size_t off = 0;
    for (int i = 0; i < kWsSlots; i++) {
        bufs[2 + i] = ws ? ws + off : nullptr;
        off += (p.ws_buf_bytes[i] + 255) / 256 * 256;
    }
    for (const Step &s : steps) {
        const void *src = bufs[static_cast<int>(s.src)];
        void *dst = bufs[static_cast<int>(s.dst)];
        if (src == nullptr || dst == nullptr) return cudaErrorInvalidDevicePointer;
        cudaError_t e = cudaSuccess;
        switch (s.kind) {
            case StepKind::kTile: {
                if (s.tc_fmt >= 0 && s.tc_kind == 1) {
                    e = launch_tc_rows(s.d.n, s.tc_fmt, s.forward, static_cast<const float2 *>(src),
                                       static_cast<float2 *>(dst), s.d.n_cols, s.d.in_a.cstride, s.d.out_a.cstride,
                                       s.tc_mat[0], s.tc_mat[1], s.tc_tw, s.grid, device_error_word(p.device), st);
                } else if (s.tc_fmt >= 0) {
                    TileDesc d = s.d;
                    d.in = src;
                    d.out = dst;
                    e = launch_tc(d, d.n, s.tc_fmt, s.forward, s.tc_mat, s.tc_tw, s.grid, device_error_word(p.device),
                                  st);
                } else if (s.has_row && (reinterpret_cast<uintptr_t>(src) & 15) == 0 && src != dst) {
                    TileDesc d = s.rd;
                    d.in = src;
                    d.out = dst;
                    if (s.row_fn)
                        e = launch_kernel_fn(s.row_fn, d, s.row_grid, row_kernel_smem(d), device_error_word(p.device),
                                             st);
                    else
                        e = launch_row_tiles(d, s.maxe, s.forward, s.row_grid, device_error_word(p.device), st);
                } else if (s.cp_fn && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
                    TileDesc d = s.d;
                    d.in = src;
                    d.out = dst;
                    d.stw = s.db_stw;
                    e = launch_col_pipe(s.cp_fn, d, s.cp_grid, device_error_word(p.device), st);
                } else if (s.db) {
                    TileDesc d = s.d;
                    d.in = src;
                    d.out = dst;
                    if (s.db_fn) {
                        d.stw = s.db_stw;
                        e = launch_kernel_fn(s.db_fn, d, s.grid, 2 * size_t(d.tb) * d.pitch * sizeof(float2),
                                             device_error_word(p.device), st);
                    } else {
                        e = launch_tile_db(d, s.maxe, s.forward, s.grid, st);
                    }
                } else {
                    TileDesc d = s.d;
                    d.in = src;
                    d.out = dst;
                    d.in_im = in_im;
                    d.out_im = out_im;
                    if ((d.planar & 1 && !in_im) || (d.planar & 2 && !out_im)) return cudaErrorInvalidDevicePointer;
                    e = launch_tile(d, s.maxe, s.forward, s.grid, st);
                }
                break;
            }
            case StepKind::kR2CPost:
                e = launch_r2c_post(static_cast<const float2 *>(src), static_cast<float2 *>(dst), s.rows, s.m,
                                    s.src_dist, s.dst_dist, s.lo, s.hi, s.log2l, s.forward, st);
                break;
            case StepKind::kC2RPre:
                e = launch_c2r_pre(static_cast<const float2 *>(src), static_cast<float2 *>(dst), s.rows, s.m,
                                   s.src_dist, s.dst_dist, s.lo, s.hi, s.log2l, s.forward, st);
                break;
            case StepKind::kBluePre:
                e = launch_blue_pre(src, static_cast<float2 *>(dst), s.rows, s.d.blue_n, s.m, s.src_dist,
                                    s.d.blue_kind, s.d.chirp, st);
                break;
            case StepKind::kPointMul:
                e = launch_point_mul(static_cast<float2 *>(dst), s.d.bmul, s.rows, s.m, st);
                break;
            case StepKind::kBluePost:
                e = launch_blue_post(static_cast<const float2 *>(src), dst, s.rows, s.d.blue_n, s.m, s.dst_dist,
                                     s.d.blue_kind, s.d.chirp, st);
                break;
            case StepKind::kTranspose:
                e = launch_transpose(static_cast<const float2 *>(src), static_cast<float2 *>(dst), s.t_batch, s.t_rows,
                                     s.t_cols, p.device, st);
                break;
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace sipfft
