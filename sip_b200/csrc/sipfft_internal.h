// Internal declarations shared by the planner, the C-ABI layer and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "fft_tile.cuh"

namespace sipfft {

// Largest dynamic shared memory a CTA may use on sm_100 (227 KiB).
constexpr int kMaxSmemBytes = 227 * 1024;
// Number of SMs of a B200; the planner sizes persistent grids with the
// queried count and falls back to this.
constexpr int kB200Sms = 148;

cudaError_t launch_tile(const TileDesc &d, int maxe, bool forward, int grid, cudaStream_t st);
// Persistent double-buffered C2C tile kernel (cp.async prefetch of the next tile).
const void *tile_db_kernel_fn(int maxe, bool forward);
cudaError_t launch_tile_db(const TileDesc &d, int maxe, bool forward, int grid, cudaStream_t st);
cudaError_t fill_twiddles(float2 *t, int64_t count, int64_t denom, int64_t mult, cudaStream_t st);
cudaError_t fill_chirp(float2 *t, int64_t n_len, bool forward, cudaStream_t st);
cudaError_t fill_bluestein_b(float2 *b, const float2 *chirp, int64_t n_len, int64_t m_len, cudaStream_t st);
cudaError_t scale_table(float2 *b, int64_t count, float s, cudaStream_t st);
// TMA-pipelined persistent kernel for contiguous rows (row_fft.cu).  The row
// descriptor keeps the row distance in in_a.dist / out_a.dist and the
// per-buffer float2 count in g_ns.
cudaError_t launch_row_tiles(const TileDesc &d, int maxe, bool forward, int grid, int *err, cudaStream_t st);
size_t row_kernel_smem(const TileDesc &d);
int row_kernel_blocks_per_sm(const TileDesc &d, int maxe, bool forward);
int kernel_blocks_per_sm(const void *fn, int threads, size_t smem);
cudaError_t allow_max_dynamic_smem(const void *fn);
// Raises the dynamic shared-memory limit of every kernel of the library on
// `device` (once).  Called by every set-up entry point (plan creation, batch
// plans, servers, the first allocation-free call) so that nothing is
// configured lazily inside a stream capture.
cudaError_t configure_kernels(int device);
void tile_kernel_fns(std::vector<const void *> &out);
void row_kernel_fns(std::vector<const void *> &out);
void static_kernel_fns(std::vector<const void *> &out);
// persistent uneven-batch kernel (fft_tile.cu): CTAs of kBatchBlock threads, at
// most kBatchMaxe points per thread; batch plans keep single-tile rows at or
// below kBatchMaxRowN (longer rows are multi-pass) so several CTAs fit per SM
constexpr int kBatchBlock = 256;
constexpr int kBatchMaxe = 16;
constexpr int64_t kBatchMaxRowN = 4096;
const void *batch_kernel_fn(bool forward, bool compact);
cudaError_t launch_batch(int grid, int block, size_t smem, const BatchSeg *segs, const int2 *items, int nitems,
                         int *counter, int *done, const BatchBufs &bufs, int *err, bool forward, bool compact,
                         cudaStream_t st);
cudaError_t launch_kernel_fn(const void *fn, const TileDesc &d, int grid, size_t smem, int *err, cudaStream_t st);
// Launch with programmatic stream serialization (the kernel calls pdl_enter()
// before its first global access).
cudaError_t launch_pdl(const void *fn, dim3 grid, dim3 block, size_t smem, cudaStream_t st, void **args);

// Compile-time specialised pipelined row kernels (static_fft.cu).
struct StaticKernel {
    int io_mask = 7;  // bit 0: C2C, bit 1: C2R (packed), bit 2: R2C (packed)
    int n = 0;
    int nstages = 0;
    int radix[8] = {};
    int tpt = 0;
    const void *fn[2][3] = {};  // [forward][C2C, R2C packed, C2R packed]
    const void *db[2] = {};     // [forward] double-buffered C2C tiles (strided axes, multi-pass steps)
    int row_bufs = 2;           // shared-memory buffers of its row kernel (3: ping-pong work area)
};
const StaticKernel *find_static_kernel(int n, int io);
// TMA-pipelined column kernels (col_pipe.cu) for the power-of-two static
// engines with 16 points per thread: n, threads per transform and columns per
// tile must match an instantiation.  contiguous_out: each column's outputs are
// contiguous (output element stride 1); the variant that stages them through
// shared memory is returned where one exists.
const void *col_pipe_kernel_fn(int n, int tpt, int tb, bool forward, bool contiguous_out);
bool col_pipe_has_engine(int n);  // a TMA column engine exists for this length
int col_pipe_bufs(int n, int tpt, int tb);  // its shared-memory tile buffers (TileDesc::row_bufs)
void col_pipe_kernel_fns(std::vector<const void *> &out);
size_t col_pipe_smem(const TileDesc &d);
// the step's input addressing and sizes fit the tensor map of the column kernel
bool col_pipe_layout_ok(const TileDesc &d);
cudaError_t launch_col_pipe(const void *fn, const TileDesc &d, int grid, int *err, cudaStream_t st);
cudaError_t fill_stage_twiddles(float2 *t, const int *radix, int nstages, cudaStream_t st);
int64_t stage_twiddle_count(const int *radix, int nstages);
// Tensor-core split-precision stages (tc_fft.cu): n = n1 * n2 as two DFT-matrix
// GEMMs on tcgen05 with hi/lo FP16 or BF16 operands and FP32 accumulation.
// fmt 0 = FP16 x3 (per-tile power-of-two scaling), 1 = BF16 x3.
struct TcConfig {
    int n1 = 0, n2 = 0, tb = 0;  // tb transforms per CTA (128 threads)
};
bool tc_config(int n, TcConfig &c);
const void *tc_kernel(int n, int fmt, bool fwd, size_t *smem);
void tc_kernel_fns(std::vector<const void *> &out);
// 128 x 2N real DFT matrix of one stage in the operand layout, hi and lo parts
cudaError_t fill_tc_matrix(uint16_t *hi, uint16_t *lo, int N, int fmt, bool fwd, cudaStream_t st);
cudaError_t launch_tc(const TileDesc &d, int n, int fmt, bool fwd, const uint16_t *const *mats, const float2 *tw,
                      int grid, int *err, cudaStream_t st);
// Warp-specialised tensor-core kernel for contiguous C2C rows (tc_rows.cu):
// 8 loader warps, 4 + 4 epilogue warps and one MMA warp.
constexpr int kTcRowThreads = 544;
bool tc_rows_config(int n, TcConfig &c);
const void *tc_rows_kernel_fn(int n, int fmt, bool fwd, size_t *smem);
void tc_rows_kernel_fns(std::vector<const void *> &out);
// 2N x 2N B-operand DFT matrix of one stage (hi at hi, lo at lo)
cudaError_t fill_tc_bmatrix(uint16_t *hi, uint16_t *lo, int N, int fmt, bool fwd, cudaStream_t st);
cudaError_t launch_tc_rows(int n, int fmt, bool fwd, const float2 *in, float2 *out, int64_t rows, int64_t in_dist,
                           int64_t out_dist, const uint16_t *fa, const uint16_t *fb, const float2 *tw, int grid,
                           int *err, cudaStream_t st);
// Overlap-add, window envelope and centre slice of the inverse STFT (istft.cu).
cudaError_t launch_istft_ola(const float2 *frames, const float *window, float2 *out, int64_t channel, int n_frames,
                             int n_fft, int hop, int64_t out_len, cudaStream_t st);
// Process-wide device error word of the current device (bounded waits that
// gave up set it); read and cleared by asdFftSynchronize.
int *device_error_word(int device);
// Message of the last failing call on this thread (asdFftGetErrorMessage).
void set_last_error(const std::string &msg);
const std::string &last_error();
int sm_count(int device);
// R2C post-twiddle / C2R pre-twiddle of the multi-pass (large-N) plans.
cudaError_t launch_r2c_post(const float2 *z, float2 *x, int64_t rows, int64_t m, int64_t zdist, int64_t xdist,
                            const float2 *tw_lo, const float2 *tw_hi, int log2l, bool forward, cudaStream_t st);
cudaError_t launch_c2r_pre(const float2 *x, float2 *z, int64_t rows, int64_t m, int64_t xdist, int64_t zdist,
                           const float2 *tw_lo, const float2 *tw_hi, int log2l, bool forward, cudaStream_t st);
// Element-wise Bluestein stages for multi-pass convolution lengths (fft_aux.cu):
// a[r][e] = x_r[e] chirp[e] (e < n, else 0) over rows of m; b[r][e] *= bmul[e];
// y_r[k] = chirp[k] a[r][k] for the first n (kind 1: n/2+1; kind 2: real part of n).
// kind: 0 complex, 1 real input / half-spectrum output, 2 Hermitian half-spectrum
// input / real output.
cudaError_t launch_blue_pre(const void *in, float2 *a, int64_t rows, int64_t n, int64_t m, int64_t in_dist, int kind,
                            const float2 *chirp, cudaStream_t st);
cudaError_t launch_point_mul(float2 *b, const float2 *bmul, int64_t rows, int64_t m, cudaStream_t st);
cudaError_t launch_blue_post(const float2 *a, void *out, int64_t rows, int64_t n, int64_t m, int64_t out_dist,
                             int kind, const float2 *chirp, cudaStream_t st);
// out[b][c][r] = in[b][r][c] for `batch` matrices of rows x cols complex values
cudaError_t launch_transpose(const float2 *in, float2 *out, int64_t batch, int64_t rows, int64_t cols, int device,
                             cudaStream_t st);

// A device twiddle table shared between plans (the reference's FFTensorCache,
// core/fft/utils/fftensor_cache.cpp:55-92, keeps coefficient tensors alive
// through weak pointers in the same way).
struct DeviceTable {
    float2 *ptr = nullptr;
    int64_t count = 0;
    int device = 0;
    ~DeviceTable();
};
using TablePtr = std::shared_ptr<DeviceTable>;
// t[m] = exp(-2 pi i (m*mult mod denom) / denom), m < count
TablePtr get_table(int64_t count, int64_t denom, int64_t mult, int device, std::string *err);
// per-stage twiddle tables of a static kernel's radix sequence
TablePtr get_stage_table(const StaticKernel &k, int device, std::string *err);
// per-stage twiddle tables of any radix sequence: stage s >= 1 holds
// W_{ns R}^{r k} at [(r-1) ns + k], stages back to back (stage 0 has none)
TablePtr get_stage_table(const int *radix, int nstages, int device, std::string *err);
// hi/lo operand matrices of one tensor-core stage (N points, fmt, direction).
// layout 0 (A operand of tc_fft_kernel): hi at ptr, lo at ptr + 64 N float2,
// each 128 x 2N 16-bit values; layout 1 (B operand of tc_rows_kernel): hi at
// ptr, lo at ptr + N^2 float2, each 2N x 2N 16-bit values.
TablePtr get_tc_matrix(int N, int fmt, bool fwd, int device, std::string *err, int layout = 0);

// Buffers a step reads or writes: the caller's input and output, and four
// slots of the caller's workspace (kWs3 holds the intermediates that a planar
// plan moves out of the caller's output).
enum class Buf : int { kUserIn = 0, kUserOut = 1, kWs0 = 2, kWs1 = 3, kWs2 = 4, kWs3 = 5 };
constexpr int kWsSlots = 4;

// kBluePre / kPointMul / kBluePost: the element-wise stages of a Bluestein
// transform whose convolution length M is too long for one CTA (the M-point
// FFTs between them are multi-pass tile steps).
enum class StepKind : int {
    kTile = 0, kR2CPost = 1, kC2RPre = 2, kBluePre = 3, kPointMul = 4, kBluePost = 5, kTranspose = 6
};

struct Step {
    StepKind kind = StepKind::kTile;
    TileDesc d{};
    int maxe = 16;
    int grid = 1;
    bool forward = true;
    Buf src = Buf::kUserIn;
    Buf dst = Buf::kUserOut;
    // optional TMA-pipelined row variant of the same step (used when the
    // source pointer is 16-byte aligned); row_fn != nullptr selects a
    // compile-time specialised kernel instead of the runtime-radix one
    bool db = false;  // run d on the double-buffered tile kernel (grid is then persistent)
    const void *db_fn = nullptr;  // compile-time engine for it (else the runtime-radix kernel)
    const float2 *db_stw = nullptr;  // that engine's per-stage twiddle tables
    // TMA column kernel of the same engine (used when the source is 16-byte aligned)
    const void *cp_fn = nullptr;
    int cp_grid = 1;
    bool has_row = false;
    TileDesc rd{};
    int row_grid = 1;
    const void *row_fn = nullptr;
    // tensor-core variant (tc_fmt >= 0): d is launched by launch_tc with these matrices
    int tc_fmt = -1;
    int tc_kind = 0;  // 0: tile kernel (any IO / layout), 1: row pipeline (contiguous C2C rows)
    const uint16_t *tc_mat[4] = {};  // stage-1 hi, lo, stage-2 hi, lo
    const float2 *tc_tw = nullptr;
    // kR2CPost / kC2RPre
    int64_t rows = 0, m = 0, src_dist = 0, dst_dist = 0;
    // kTranspose: t_batch matrices of t_rows x t_cols complex values -> t_cols x t_rows
    int64_t t_batch = 0, t_rows = 0, t_cols = 0;
    const float2 *lo = nullptr, *hi = nullptr;
    int log2l = 0;
    std::string what;  // human-readable description (plan dump)
};

// Autotuned choice for one length: radix order, elements per thread and
// tile shape (threads per CTA that the tile kernels aim for, 0 = planner
// default) of the SIMT tile kernels, and the stage arithmetic that ran the
// whole plan fastest (0 FP32 SIMT, 1 tensor-core FP16 x3, 2 BF16 x3).
struct TuneChoice {
    std::vector<int> radices;
    int maxe = 0;
    int row_threads = 0;
    double us = 0.0;
    int precision = 0;
    double plan_us = 0.0;  // time of the whole plan in the chosen arithmetic
};

struct Plan {
    // reference FFTPlan fields (core/fft/fftplan/include/fftplan/fft_plan.h:49-70)
    int fft_type = 0;
    int direction = 0;
    std::vector<int64_t> sizes;
    std::vector<int64_t> strides;
    int64_t batch = 0;
    bool vertical = false;
    void *stream = nullptr;
    void *workspace = nullptr;
    bool initialized = false;
    bool failed = false;
    // build-specific
    int device = 0;
    std::vector<Step> steps;
    size_t ws_buf_bytes[kWsSlots] = {0, 0, 0, 0};
    size_t ws_bytes = 0;
    std::vector<TablePtr> tables;
    std::mutex mu;
    bool use_tuned = false;  // consult the autotuner's choices (uneven-batch plans)
    int row_threads = 256;   // threads per CTA the row tiles aim for
    int row_smem = 64 * 1024;  // shared memory per CTA the row tiles stay under
    int64_t max_row_n = 1 << 30;  // C2C rows longer than this take the multi-pass path
    int max_maxe = 32;            // largest points per thread a tile may use (tuned choices above are ignored)
    int max_radix = 16;           // largest radix a tile may use (16 and 12 split below it)
    // inverse STFT plan (asdFftIstftMakePlan): one column C2C step into workspace
    // slot 0 ([channel][frame][n_fft]), then the overlap-add kernel
    bool istft = false;
    int64_t istft_channel = 0, istft_frames = 0, istft_nfft = 0, istft_hop = 0, istft_out_len = 0;
    // 0: FP32 kernels; 1: tensor-core FP16 hi/lo x3; 2: tensor-core BF16 hi/lo x3
    // (lengths without a tensor-core stage keep the FP32 kernels); 3: per length,
    // the arithmetic the autotuner measured fastest (FP32 when untuned)
    int precision = 0;
    // complex32 (FP16 pairs) variant of a 1D C2C plan's steps, built at the
    // first complex32 exec (c32_state: 0 not built, 1 built, -1 unsupported)
    std::vector<Step> c32_steps;
    int c32_state = 0;
    bool forward() const;
};

// Process-wide autotuner choices keyed by (transform length); see tuner.cpp.
bool tuned_choice(int64_t n, TuneChoice &out);
void set_tuned_choice(int64_t n, const TuneChoice &c);
int load_tune_cache(const std::string &path, int device);
bool save_tune_cache(const std::string &path, int device);

// Planner entry points (planner.cpp).  They fill plan.steps / ws sizes and
// return an empty string on success, else the reason.
std::string build_plan_1d(Plan &p);
std::string build_plan_2d(Plan &p);
std::string build_plan_3d(Plan &p);
std::string build_plan_istft(Plan &p);
// Launch every step of an initialised plan.
cudaError_t execute_plan(Plan &p, const void *in, void *out, cudaStream_t st, const float *in_im = nullptr,
                         float *out_im = nullptr);
// Same for an explicit step list (e.g. re-targeted to fewer rows) and workspace.
// in_im / out_im: imaginary planes of a planar (ASCEND_FFT_C2C_SEP) plan's user buffers.
cudaError_t execute_steps(const Plan &p, const std::vector<Step> &steps, const void *in, void *out, void *workspace,
                          cudaStream_t st, const float *in_im = nullptr, float *out_im = nullptr);
bool scale_steps_to_rows(const Plan &p, int64_t rows, std::vector<Step> &out);
// Copy of a 1D C2C plan's steps that reads and writes complex32 user data
// (the first step widens on load, the last rounds on store, FP32 in between).
// Empty string on success, else why the plan has no complex32 form.
std::string complex32_steps(const Plan &p, std::vector<Step> &out);
std::string describe_plan(const Plan &p);

// Radix decomposition used by the tile kernel (largest radices first).
bool factor_radices(int64_t n, std::vector<int> &radices);
// true when every radix has a codelet in the runtime engine and they multiply to n
bool valid_radices(const std::vector<int> &r, int64_t n);
std::vector<int> multipass_split(int64_t F);  // pass lengths of a multi-pass transform

}  // namespace sipfft
