// C ABI of libasdsip_fft.so: the reference's asdFft* surface
// (include/fft_api.h, core/fft/fft_api.cpp) plus the aclTensor descriptor shim.
//
// Behaviour kept from the reference:
//   * handles live in a process-wide registry (FFTPlanCache,
//     core/fft/fftplan/fft_plan_cache.cpp:15-42); every entry point validates
//     the handle first;
//   * parameter checks and their status codes follow fft_api.cpp:737-1233
//     (sizes in (0, 2^27], batch > 0, stream != NULL, dtype/trailing-shape
//     matching of the exec tensors, missing workspace -> 500000,
//     Synchronize/GetType on an unknown handle -> 500000);
//   * execution is asynchronous on the handle's stream.
// Differences, all on the safe side: plan-time failures return a status
// instead of throwing across the C boundary; exec also rejects tensors whose
// element count is smaller than the plan's batch (the reference would read
// or write past them); a transform the kernels cannot plan returns
// ACL_ERROR_API_NOT_SUPPORT.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>

#include "../../include/asdsip_fft.h"
#include "../../include/asdsip_fft_ext.h"
#include "sipfft_internal.h"

struct aclTensor {
    std::vector<int64_t> view;
    std::vector<int64_t> strides;
    std::vector<int64_t> storage;
    aclDataType dtype = ACL_DT_UNDEFINED;
    aclFormat format = ACL_FORMAT_ND;
    int64_t offset = 0;
    void *data = nullptr;
};

namespace {

size_t dtype_size(aclDataType t)
{
    switch (t) {
        case ACL_FLOAT: case ACL_INT32: case ACL_UINT32: return 4;
        case ACL_FLOAT16: case ACL_BF16: case ACL_INT16: case ACL_UINT16: return 2;
        case ACL_INT8: case ACL_UINT8: case ACL_BOOL: return 1;
        case ACL_INT64: case ACL_UINT64: case ACL_DOUBLE: case ACL_COMPLEX64: return 8;
        case ACL_COMPLEX128: return 16;
        case ACL_COMPLEX32: return 4;
        default: return 0;
    }
}

bool log_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *v = std::getenv("ASDSIP_FFT_LOG");
        on = (v && *v && *v != '0') ? 1 : 0;
    }
    return on == 1;
}

void log_error(const char *where, const std::string &msg)
{
    sipfft::set_last_error(std::string(where) + ": " + msg);
    if (log_enabled()) std::fprintf(stderr, "[asdsip_fft] %s: %s\n", where, msg.c_str());
}

std::mutex g_fft_mtx;  // guards the registry (the reference's fft_mtx, core/utils/sip_lock.cpp:13)
std::unordered_map<void *, std::unique_ptr<sipfft::Plan>> g_plans;

sipfft::Plan *find_plan(void *h)
{
    std::lock_guard<std::mutex> lock(g_fft_mtx);
    auto it = g_plans.find(h);
    return it == g_plans.end() ? nullptr : it->second.get();
}

constexpr int64_t kMaxFftSize = int64_t(1) << 27;  // fft_api.cpp:61

using namespace AsdSip;

bool valid_type(int t)
{
    return t == ASCEND_FFT_C2C || t == ASCEND_FFT_C2R || t == ASCEND_FFT_R2C || t == ASCEND_FFT_C2C_SEP;
}
bool valid_dir(int d) { return d == ASCEND_FFT_FORWARD || d == ASCEND_FFT_INVERSE; }

int64_t prod(const std::vector<int64_t> &v)
{
    int64_t p = 1;
    for (int64_t x : v) p *= x;
    return p;
}

// Runs the planner under the plan's lock; maps failures to status codes.
AspbStatus finish_plan(sipfft::Plan &p, std::string (*builder)(sipfft::Plan &), const char *where)
{
    p.steps.clear();
    p.tables.clear();
    p.c32_steps.clear();
    p.c32_state = 0;
    for (size_t &b : p.ws_buf_bytes) b = 0;
    if (builder != sipfft::build_plan_istft) p.istft = false;
    p.ws_bytes = 0;
    p.initialized = false;
    p.failed = false;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        p.failed = true;
        log_error(where, "no CUDA device");
        return ACL_ERROR_INTERNAL_ERROR;
    }
    p.device = dev;
    if (sipfft::configure_kernels(dev) != cudaSuccess) {
        cudaGetLastError();
        p.failed = true;
        log_error(where, "kernel configuration failed");
        return ACL_ERROR_INTERNAL_ERROR;
    }
    std::string err;
    try {
        err = builder(p);
    } catch (const std::exception &e) {
        err = std::string("exception: ") + e.what();
    } catch (...) {
        err = "unknown exception";
    }
    if (!err.empty()) {
        p.failed = true;
        log_error(where, err);
        if (err.rfind("twiddle table", 0) == 0) return ACL_ERROR_INTERNAL_ERROR;
        return ACL_ERROR_API_NOT_SUPPORT;
    }
    p.initialized = true;
    return ACL_SUCCESS;
}

// Trailing-shape / dtype matching (fft_api.cpp:1047-1167) plus an element-count
// check against the plan's batch.  kind: 0 complex full, 1 complex half, 2 real full.
bool match_tensor(const sipfft::Plan &p, const aclTensor *t, int kind, bool complex32 = false)
{
    if (t == nullptr || t->data == nullptr) return false;
    const aclDataType want = kind == 2 ? ACL_FLOAT : (complex32 ? ACL_COMPLEX32 : ACL_COMPLEX64);
    if (t->dtype != want) return false;
    const auto &dims = t->view;
    int64_t expect = p.batch;
    if (p.vertical) {
        expect *= p.sizes[0];
    } else {
        if (dims.size() < p.sizes.size()) return false;
        for (size_t i = 0; i < p.sizes.size(); i++) {
            const int64_t want_dim = (kind == 1 && i + 1 == p.sizes.size()) ? p.sizes[i] / 2 + 1 : p.sizes[i];
            if (dims[dims.size() - p.sizes.size() + i] != want_dim) return false;
            expect *= want_dim;
        }
    }
    return prod(dims) >= expect;
}

void *tensor_addr(const aclTensor *t)
{
    return static_cast<char *>(t->data) + t->offset * static_cast<int64_t>(dtype_size(t->dtype));
}

AspbStatus run(sipfft::Plan &p, const void *in, void *out, const char *where, const float *in_im = nullptr,
               float *out_im = nullptr, bool complex32 = false)
{
    std::lock_guard<std::mutex> lock(p.mu);
    if (!p.initialized) {
        log_error(where, "plan is not initialised");
        return ACL_ERROR_INVALID_PARAM;
    }
    if (complex32 && p.c32_state == 0) {
        const std::string why = sipfft::complex32_steps(p, p.c32_steps);
        p.c32_state = why.empty() ? 1 : -1;
        if (!why.empty()) log_error(where, why.c_str());
    }
    if (complex32 && p.c32_state < 0) return ACL_ERROR_API_NOT_SUPPORT;
    if (p.ws_bytes > 0 && p.workspace == nullptr) {
        log_error(where, "workspace has not been set");
        return ACL_ERROR_INTERNAL_ERROR;
    }
    if (in == nullptr || out == nullptr) {
        log_error(where, "tensor data is null");
        return ACL_ERROR_INTERNAL_ERROR;
    }
    if (p.fft_type != ASCEND_FFT_C2C && p.fft_type != ASCEND_FFT_C2C_SEP && in == out) {
        log_error(where, "in-place execution is supported for C2C plans only");
        return ACL_ERROR_INVALID_PARAM;
    }
    if (p.fft_type == ASCEND_FFT_C2C_SEP) {
        if (!in_im || !out_im || (in == out) != (static_cast<const void *>(in_im) == out_im)) {
            log_error(where, "separated plans need both planes, in place for both or for neither");
            return ACL_ERROR_INVALID_PARAM;
        }
        if ((reinterpret_cast<uintptr_t>(in_im) & 3) || (reinterpret_cast<uintptr_t>(out_im) & 3)) {
            log_error(where, "imaginary planes must be 4-byte aligned");
            return ACL_ERROR_INVALID_PARAM;
        }
    }
    const uintptr_t align_mask = (p.fft_type == ASCEND_FFT_C2C_SEP || complex32) ? 3 : 7;
    if ((reinterpret_cast<uintptr_t>(in) & align_mask) || (reinterpret_cast<uintptr_t>(out) & align_mask)) {
        log_error(where, complex32 ? "device buffers must be 4-byte aligned" : "device buffers must be 8-byte aligned");
        return ACL_ERROR_INVALID_PARAM;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p.device) cudaSetDevice(p.device);
    cudaError_t e = complex32 ? sipfft::execute_steps(p, p.c32_steps, in, out, p.workspace,
                                                      static_cast<cudaStream_t>(p.stream))
                              : sipfft::execute_plan(p, in, out, static_cast<cudaStream_t>(p.stream), in_im, out_im);
    if (cur != p.device) cudaSetDevice(cur);
    if (e != cudaSuccess) {
        log_error(where, cudaGetErrorString(e));
        cudaGetLastError();
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------------------------------ aclTensor
aclTensor *aclCreateTensor(const int64_t *viewDims, uint64_t viewDimsNum, aclDataType dataType, const int64_t *stride,
                           int64_t offset, aclFormat format, const int64_t *storageDims, uint64_t storageDimsNum,
                           void *tensorData)
{
    if ((viewDimsNum > 0 && viewDims == nullptr) || viewDimsNum > 64 || offset < 0) return nullptr;
    try {
        auto *t = new aclTensor;
        t->view.assign(viewDims, viewDims + viewDimsNum);
        if (stride) t->strides.assign(stride, stride + viewDimsNum);
        if (storageDims) t->storage.assign(storageDims, storageDims + storageDimsNum);
        t->dtype = dataType;
        t->format = format;
        t->offset = offset;
        t->data = tensorData;
        for (int64_t d : t->view) {
            if (d < 0) {
                delete t;
                return nullptr;
            }
        }
        return t;
    } catch (...) {
        return nullptr;
    }
}

int32_t aclDestroyTensor(const aclTensor *tensor)
{
    delete tensor;
    return 0;
}

int32_t aclGetDataType(const aclTensor *tensor, aclDataType *dataType)
{
    if (!tensor || !dataType) return AsdSip::ACL_ERROR_INVALID_PARAM;
    *dataType = tensor->dtype;
    return 0;
}

int32_t aclGetViewShape(const aclTensor *tensor, int64_t **viewDims, uint64_t *viewDimsNum)
{
    if (!tensor || !viewDims || !viewDimsNum) return AsdSip::ACL_ERROR_INVALID_PARAM;
    *viewDimsNum = tensor->view.size();
    *viewDims = new int64_t[tensor->view.size() + 1];
    for (size_t i = 0; i < tensor->view.size(); i++) (*viewDims)[i] = tensor->view[i];
    return 0;
}

void *aclGetTensorAddr(const aclTensor *tensor) { return tensor ? tensor_addr(tensor) : nullptr; }

}  // extern "C"

// ------------------------------------------------------------------------------------------ FFT API
// Defined inside AsdSip with the header's C++ signatures; the declarations in
// asdsip_fft.h give them C linkage (unmangled names), as in the reference.
namespace AsdSip {

AspbStatus asdFftCreate(asdFftHandle &handle)
{
    try {
        auto p = std::make_unique<sipfft::Plan>();
        void *h = p.get();
        std::lock_guard<std::mutex> lock(g_fft_mtx);
        g_plans.emplace(h, std::move(p));
        handle = h;
        return ACL_SUCCESS;
    } catch (...) {
        return ACL_ERROR_INTERNAL_ERROR;
    }
}

AspbStatus asdFftSetStream(asdFftHandle handle, void *stream)
{
    if (stream == nullptr) {
        log_error("asdFftSetStream", "stream is nullptr");
        return ACL_ERROR_INVALID_PARAM;
    }
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    std::lock_guard<std::mutex> lock(p->mu);
    p->stream = stream;
    return ACL_SUCCESS;
}

AspbStatus asdFftMakePlan1D(asdFftHandle handle, int64_t fftSize, enum asdFftType fftType,
                            enum asdFftDirection direction, int64_t batchSize, enum asdFft1dDimType dimType)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    if (fftSize <= 0 || fftSize > kMaxFftSize || batchSize <= 0) return ACL_ERROR_INVALID_PARAM;
    if (fftType == ASCEND_STFT_C2C || fftType == ASCEND_STFT_C2R || fftType == ASCEND_STFT_R2C)
        return ACL_ERROR_API_NOT_SUPPORT;
    if (!valid_type(fftType) || !valid_dir(direction)) return ACL_ERROR_INVALID_PARAM;
    const bool vertical = dimType == ASCEND_FFT_VERTICAL;
    if (!vertical && dimType != ASCEND_FFT_HORIZONTAL) return ACL_ERROR_INVALID_PARAM;
    if (vertical && fftType != ASCEND_FFT_C2C) return ACL_ERROR_API_NOT_SUPPORT;
    std::lock_guard<std::mutex> lock(p->mu);
    p->fft_type = fftType;
    p->direction = direction;
    p->sizes = {fftSize};
    p->vertical = vertical;
    // fft_api.cpp:785-791: a vertical plan is one transform per column
    p->batch = batchSize;
    p->strides = {vertical ? batchSize : 1};
    return finish_plan(*p, sipfft::build_plan_1d, "asdFftMakePlan1D");
}

AspbStatus asdFftMakePlan2D(asdFftHandle handle, int64_t fftSizeX, int64_t fftSizeY, enum asdFftType fftType,
                            enum asdFftDirection direction, int32_t batchSize)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    if (fftSizeX <= 0 || fftSizeX > kMaxFftSize || fftSizeY <= 0 || fftSizeY > kMaxFftSize || batchSize <= 0)
        return ACL_ERROR_INVALID_PARAM;
    if (fftType == ASCEND_STFT_C2C || fftType == ASCEND_STFT_C2R || fftType == ASCEND_STFT_R2C)
        return ACL_ERROR_API_NOT_SUPPORT;
    if (!valid_type(fftType) || !valid_dir(direction)) return ACL_ERROR_INVALID_PARAM;
    std::lock_guard<std::mutex> lock(p->mu);
    p->fft_type = fftType;
    p->direction = direction;
    p->sizes = {fftSizeX, fftSizeY};
    p->strides = {1, 1};
    p->vertical = false;
    p->batch = batchSize;
    return finish_plan(*p, sipfft::build_plan_2d, "asdFftMakePlan2D");
}

AspbStatus asdFftMakePlan3D(asdFftHandle handle, int64_t fftSizeX, int64_t fftSizeY, int64_t fftSizeZ,
                            enum asdFftType fftType, enum asdFftDirection direction, int32_t batchSize)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    if (fftSizeX <= 0 || fftSizeX > kMaxFftSize || fftSizeY <= 0 || fftSizeY > kMaxFftSize || fftSizeZ <= 0 ||
        fftSizeZ > kMaxFftSize || batchSize <= 0)
        return ACL_ERROR_INVALID_PARAM;
    if (fftType == ASCEND_STFT_C2C || fftType == ASCEND_STFT_C2R || fftType == ASCEND_STFT_R2C)
        return ACL_ERROR_API_NOT_SUPPORT;
    if (!valid_type(fftType) || !valid_dir(direction)) return ACL_ERROR_INVALID_PARAM;
    std::lock_guard<std::mutex> lock(p->mu);
    p->fft_type = fftType;
    p->direction = direction;
    p->sizes = {fftSizeX, fftSizeY, fftSizeZ};
    p->strides = {1, 1, 1};
    p->vertical = false;
    p->batch = batchSize;
    return finish_plan(*p, sipfft::build_plan_3d, "asdFftMakePlan3D");
}

// core/fft/istft.cpp:300-390 (IstftParamsCheck) and 530-552: options the
// reference does not support are forced to center = true, normalized = false,
// onesided = false, length = 0, return_complex = true with a warning; the
// input is complex64 [channel, n_fft, frames] with frames > 1; 0 < hop <= win
// length == n_fft; n_fft and hop below 1500.  The plan is an INVERSE C2C plan
// (GetType reports C2C) whose workspace holds the transformed frames.
AspbStatus asdFftIstftMakePlan(asdFftHandle handle, const aclTensor *input, const int64_t nFft,
                               const int64_t hopLengthOpt, const int64_t winLengthOpt, const bool center,
                               const bool normalized, const bool onesidedOpt, int64_t lengthOpt, const bool returnComplex)
{
    constexpr int64_t kMaxIstft = 1500;  // istft.cpp:32-33
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    const char *where = "asdFftIstftMakePlan";
    if (!input || input->dtype != ACL_COMPLEX64 || input->view.size() != 3) {
        log_error(where, "input must be a 3-dimensional complex64 tensor [channel, n_fft, frames]");
        return ACL_ERROR_INVALID_PARAM;
    }
    if (!center) log_error(where, "warning: only center = true is supported; using it");
    if (normalized) log_error(where, "warning: only normalized = false is supported; using it");
    if (onesidedOpt) log_error(where, "warning: only onesided = false is supported; using it");
    if (!returnComplex) log_error(where, "warning: only return_complex = true is supported; using it");
    if (lengthOpt != 0) log_error(where, "warning: only length = 0 is supported; using it");
    const int64_t channel = input->view[0], fft_size = input->view[1], frames = input->view[2];
    if (channel <= 0 || frames <= 1 || nFft != fft_size || !(0 < hopLengthOpt && hopLengthOpt <= winLengthOpt) ||
        !(winLengthOpt > 0 && winLengthOpt == nFft) || nFft >= kMaxIstft || hopLengthOpt >= kMaxIstft) {
        log_error(where, "parameters outside the supported ISTFT range");
        return ACL_ERROR_INVALID_PARAM;
    }
    std::lock_guard<std::mutex> lock(p->mu);
    p->fft_type = ASCEND_FFT_C2C;
    p->direction = ASCEND_FFT_INVERSE;
    p->sizes = {nFft};
    p->strides = {frames};
    p->vertical = false;
    p->batch = channel * frames;
    p->istft = true;
    p->istft_channel = channel;
    p->istft_frames = frames;
    p->istft_nfft = nFft;
    p->istft_hop = hopLengthOpt;
    p->istft_out_len = nFft + hopLengthOpt * (frames - 1) - 2 * (nFft / 2);  // istft.cpp:245-260
    return finish_plan(*p, sipfft::build_plan_istft, where);
}

// core/fft/istft.cpp:554-575 and the checks it calls: input as recorded at
// plan time, window float32 [n_fft], output complex64 [channel, out_len].
AspbStatus asdFftExecIstft(asdFftHandle handle, const aclTensor *input, const aclTensor *windowOpt,
                           const aclTensor *output)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    const char *where = "asdFftExecIstft";
    std::lock_guard<std::mutex> lock(p->mu);
    if (!p->istft || !p->initialized) {
        log_error(where, "the handle holds no initialised ISTFT plan");
        return ACL_ERROR_INVALID_PARAM;
    }
    if (!input || input->dtype != ACL_COMPLEX64 || input->view.size() != 3 || input->view[0] != p->istft_channel ||
        input->view[1] != p->istft_nfft || input->view[2] != p->istft_frames) {
        log_error(where, "input does not match the ISTFT plan");
        return ACL_ERROR_INVALID_PARAM;
    }
    if (!output || output->dtype != ACL_COMPLEX64 || output->view.size() != 2 ||
        output->view[0] != p->istft_channel || output->view[1] != p->istft_out_len) {
        log_error(where, "output must be complex64 [channel, n_fft + hop (frames - 1) - 2 (n_fft / 2)]");
        return ACL_ERROR_INVALID_PARAM;
    }
    if (!windowOpt || windowOpt->dtype != ACL_FLOAT || windowOpt->view.size() != 1 ||
        windowOpt->view[0] != p->istft_nfft) {
        log_error(where, "window must be float32 [n_fft]");
        return ACL_ERROR_INVALID_PARAM;
    }
    if (p->ws_bytes > 0 && p->workspace == nullptr) {
        log_error(where, "workspace has not been set");
        return ACL_ERROR_INTERNAL_ERROR;
    }
    const void *in = input->data ? tensor_addr(input) : nullptr;
    const void *win = windowOpt->data ? tensor_addr(windowOpt) : nullptr;
    void *out = output->data ? tensor_addr(output) : nullptr;
    if (!in || !win || !out) {
        log_error(where, "tensor data is null");
        return ACL_ERROR_INTERNAL_ERROR;
    }
    if ((reinterpret_cast<uintptr_t>(in) & 7) || (reinterpret_cast<uintptr_t>(out) & 7) ||
        (reinterpret_cast<uintptr_t>(win) & 3)) {
        log_error(where, "misaligned device buffer");
        return ACL_ERROR_INVALID_PARAM;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p->device) cudaSetDevice(p->device);
    cudaStream_t st = static_cast<cudaStream_t>(p->stream);
    cudaError_t e = sipfft::execute_plan(*p, in, out, st);
    if (e == cudaSuccess)
        e = sipfft::launch_istft_ola(static_cast<const float2 *>(p->workspace), static_cast<const float *>(win),
                                     static_cast<float2 *>(out), p->istft_channel, static_cast<int>(p->istft_frames),
                                     static_cast<int>(p->istft_nfft), static_cast<int>(p->istft_hop),
                                     p->istft_out_len, st);
    if (cur != p->device) cudaSetDevice(cur);
    if (e != cudaSuccess) {
        log_error(where, cudaGetErrorString(e));
        cudaGetLastError();
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

// fft_api.cpp:1281-1342: the four planes must have the same rank and shape
// (else 500000); the plan must be an ASCEND_FFT_C2C_SEP plan.
AspbStatus asdFftExecC2CSeparated(asdFftHandle handle, const aclTensor *inputReal, const aclTensor *inputImag,
                                  const aclTensor *outputReal, const aclTensor *outputImag)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    const aclTensor *t[4] = {inputReal, inputImag, outputReal, outputImag};
    for (const aclTensor *x : t)
        if (!x || !x->data) {
            log_error("asdFftExecC2CSeparated", "tensor data is null");
            return ACL_ERROR_INTERNAL_ERROR;
        }
    for (int i = 1; i < 4; i++)
        if (t[i]->view != t[0]->view) {
            log_error("asdFftExecC2CSeparated", "input/output planes differ in shape");
            return ACL_ERROR_INTERNAL_ERROR;
        }
    if (p->initialized && p->fft_type != ASCEND_FFT_C2C_SEP) return ACL_ERROR_INVALID_PARAM;
    for (const aclTensor *x : t)
        if (!match_tensor(*p, x, 2)) {
            log_error("asdFftExecC2CSeparated", "planes do not match plan (float32, trailing dims = sizes)");
            return ACL_ERROR_INVALID_PARAM;
        }
    return run(*p, tensor_addr(inputReal), tensor_addr(outputReal), "asdFftExecC2CSeparated",
               static_cast<const float *>(tensor_addr(inputImag)), static_cast<float *>(tensor_addr(outputImag)));
}

AspbStatus asdFftExecC2C(asdFftHandle handle, const aclTensor *input, const aclTensor *output)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    if (p->istft) return ACL_ERROR_INVALID_PARAM;  // an ISTFT plan runs through asdFftExecIstft
    if (p->initialized && p->fft_type != ASCEND_FFT_C2C) return ACL_ERROR_INVALID_PARAM;
    // complex32 in and out: the reference's FP16-complex DFT variant
    // (ops/fft/c2c/dft/dft/kernel/dft_complex32.cpp:33, DftC32Kernel): FP16
    // data, FP32 arithmetic
    const bool c32 = input && output && input->dtype == ACL_COMPLEX32 && output->dtype == ACL_COMPLEX32;
    if (!match_tensor(*p, input, 0, c32) || !match_tensor(*p, output, 0, c32)) {
        log_error("asdFftExecC2C", "input/output does not match plan");
        return ACL_ERROR_INVALID_PARAM;
    }
    return run(*p, tensor_addr(input), tensor_addr(output), "asdFftExecC2C", nullptr, nullptr, c32);
}

AspbStatus asdFftExecC2R(asdFftHandle handle, const aclTensor *input, const aclTensor *output)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    if (p->istft) return ACL_ERROR_INVALID_PARAM;  // an ISTFT plan runs through asdFftExecIstft
    if (p->initialized && p->fft_type != ASCEND_FFT_C2R) return ACL_ERROR_INVALID_PARAM;
    if (!match_tensor(*p, input, 1) || !match_tensor(*p, output, 2)) {
        log_error("asdFftExecC2R", "input/output does not match plan");
        return ACL_ERROR_INVALID_PARAM;
    }
    return run(*p, tensor_addr(input), tensor_addr(output), "asdFftExecC2R");
}

AspbStatus asdFftExecR2C(asdFftHandle handle, const aclTensor *input, const aclTensor *output)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    if (p->istft) return ACL_ERROR_INVALID_PARAM;  // an ISTFT plan runs through asdFftExecIstft
    if (p->initialized && p->fft_type != ASCEND_FFT_R2C) return ACL_ERROR_INVALID_PARAM;
    if (!match_tensor(*p, input, 2) || !match_tensor(*p, output, 1)) {
        log_error("asdFftExecR2C", "input/output does not match plan");
        return ACL_ERROR_INVALID_PARAM;
    }
    return run(*p, tensor_addr(input), tensor_addr(output), "asdFftExecR2C");
}

AspbStatus asdFftDestroy(asdFftHandle handle)
{
    std::unique_ptr<sipfft::Plan> victim;
    {
        std::lock_guard<std::mutex> lock(g_fft_mtx);
        auto it = g_plans.find(handle);
        if (it == g_plans.end()) return ACL_ERROR_INVALID_PARAM;
        victim = std::move(it->second);
        g_plans.erase(it);
    }
    std::lock_guard<std::mutex> lock(victim->mu);  // wait for an exec in flight on another thread
    return ACL_SUCCESS;
}

AspbStatus asdFftGetWorkspaceSize(asdFftHandle handle, size_t &workspaceSize)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    std::lock_guard<std::mutex> lock(p->mu);
    workspaceSize = p->ws_bytes;
    return ACL_SUCCESS;
}

AspbStatus asdFftSetWorkspace(asdFftHandle handle, void *workspace)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INVALID_PARAM;
    std::lock_guard<std::mutex> lock(p->mu);
    p->workspace = workspace;
    return ACL_SUCCESS;
}

AspbStatus asdFftSynchronize(asdFftHandle handle)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INTERNAL_ERROR;
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(p->stream));
    if (e != cudaSuccess) {
        log_error("asdFftSynchronize", cudaGetErrorString(e));
        cudaGetLastError();
        return ACL_ERROR_INTERNAL_ERROR;
    }
    // a bounded wait inside a kernel that gave up leaves a non-zero error word
    if (int *w = sipfft::device_error_word(p->device)) {
        int flag = 0;
        if (cudaMemcpy(&flag, w, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && flag != 0) {
            cudaMemset(w, 0, sizeof(int));
            log_error("asdFftSynchronize", "a kernel wait timed out; results are incomplete");
            return ACL_ERROR_INTERNAL_ERROR;
        }
        cudaGetLastError();
    }
    return ACL_SUCCESS;
}

AspbStatus asdFftGetType(asdFftHandle handle, asdFftType &fftType)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return ACL_ERROR_INTERNAL_ERROR;
    fftType = static_cast<asdFftType>(p->fft_type);
    return ACL_SUCCESS;
}

}  // namespace AsdSip

extern "C" {

// ------------------------------------------------------------------------------------------ extensions
int32_t asdFftExecRaw(void *handle, const void *input, void *output)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return AsdSip::ACL_ERROR_INVALID_PARAM;
    return run(*p, input, output, "asdFftExecRaw");
}

int64_t asdFftDescribePlan(void *handle, char *buf, int64_t len)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return -1;
    std::string s;
    {
        std::lock_guard<std::mutex> lock(p->mu);
        s = sipfft::describe_plan(*p);
    }
    if (buf && len > 0) {
        const int64_t n = std::min<int64_t>(len - 1, static_cast<int64_t>(s.size()));
        std::memcpy(buf, s.data(), static_cast<size_t>(n));
        buf[n] = '\0';
    }
    return static_cast<int64_t>(s.size()) + 1;
}

int64_t asdFftGetErrorMessage(char *buf, int64_t len)
{
    const std::string &s = sipfft::last_error();
    if (buf && len > 0) {
        const int64_t n = std::min<int64_t>(len - 1, static_cast<int64_t>(s.size()));
        std::memcpy(buf, s.data(), static_cast<size_t>(n));
        buf[n] = '\0';
    }
    return static_cast<int64_t>(s.size()) + 1;
}

int32_t asdFftSetPrecision(void *handle, int32_t mode)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p || mode < 0 || mode > 3) {
        log_error("asdFftSetPrecision", "unknown handle or precision mode");
        return AsdSip::ACL_ERROR_INVALID_PARAM;
    }
    std::lock_guard<std::mutex> lock(p->mu);
    if (p->precision == mode) return AsdSip::ACL_SUCCESS;
    p->precision = mode;
    if (!p->initialized) return AsdSip::ACL_SUCCESS;
    const size_t ws = p->ws_bytes;
    std::string (*builder)(sipfft::Plan &) = p->sizes.size() == 1   ? sipfft::build_plan_1d
                                             : p->sizes.size() == 2 ? sipfft::build_plan_2d
                                                                    : sipfft::build_plan_3d;
    const AspbStatus st = finish_plan(*p, builder, "asdFftSetPrecision");
    if (st == AsdSip::ACL_SUCCESS && p->ws_bytes > ws) {
        // the rebuilt plan needs more workspace (a strided axis through transposes):
        // the old buffer is too small, so it is dropped and exec refuses to run
        // (missing workspace) until the caller sets one of the new size
        p->workspace = nullptr;
        log_error("asdFftSetPrecision", "rebuilt plan needs a larger workspace: query and set it again");
    }
    return st;
}

int32_t asdFftPlanLaunchCount(void *handle)
{
    sipfft::Plan *p = find_plan(handle);
    if (!p) return -1;
    std::lock_guard<std::mutex> lock(p->mu);
    int32_t n = 0;
    for (const auto &s : p->steps) {
        if (s.kind == sipfft::StepKind::kTile || s.kind == sipfft::StepKind::kTranspose)
            n += 1;
        else
            n += static_cast<int32_t>((s.rows + 65534) / 65535);
    }
    return n;
}

}  // extern "C"
