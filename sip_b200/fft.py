"""Python binding of libasdsip_fft.so (ctypes), mirroring the reference's FFT API.

The functions keep the reference's names, argument meaning and status codes
(AscendSiPBoost include/fft_api.h:46-99): ``asdFftCreate`` returns the handle
instead of filling a reference argument, everything else returns the
``AspbStatus`` integer.  Tensors are described with ``AclTensor`` (the
library's aclTensor shim) built from CUDA torch tensors; PyTorch is only the
device-memory and stream plumbing here, every transform runs in the library's
own sm_100a kernels.

``FftPlan`` is a convenience wrapper used by the tests and the benchmark: it
creates a handle, plans, allocates the workspace the plan asks for and runs
the exec entry point that matches the plan type.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libasdsip_fft.so")

# --- status codes (core/utils/include/utils/aspb_status.h:18-27) ---------------------------------
ACL_SUCCESS = 0
ACL_ERROR_INVALID_PARAM = 100000
ACL_ERROR_OP_INPUT_NOT_MATCH = 100021
ACL_ERROR_OP_OUTPUT_NOT_MATCH = 100022
ACL_ERROR_UNSUPPORTED_DATA_TYPE = 100026
ACL_ERROR_FORMAT_NOT_MATCH = 100027
ACL_ERROR_API_NOT_SUPPORT = 200001
ACL_ERROR_INTERNAL_ERROR = 500000

# --- enums (include/fft_api.h:24-44) -------------------------------------------------------------
ASCEND_FFT_C2C = 0x10
ASCEND_FFT_C2R = 0x11
ASCEND_FFT_R2C = 0x12
ASCEND_STFT_C2C = 0x20
ASCEND_STFT_C2R = 0x21
ASCEND_STFT_R2C = 0x22
ASCEND_FFT_C2C_SEP = 0x30
ASCEND_FFT_FORWARD = 0x10
ASCEND_FFT_INVERSE = 0x11
ASCEND_FFT_HORIZONTAL = 0x10
ASCEND_FFT_VERTICAL = 0x11

# asdFftSetPrecision modes (arithmetic of the transform stages)
PRECISION_FP32 = 0       # CUDA-core FP32 kernels
PRECISION_FP16X3 = 1     # tensor-core DFT-matrix stages, FP16 hi/lo split, 3 products, FP32 accumulate
PRECISION_BF16X3 = 2     # the same with BF16 hi/lo parts
PRECISION_AUTO = 3       # per length, the arithmetic the autotuner measured fastest

ACL_FLOAT = 0
ACL_COMPLEX64 = 16
ACL_COMPLEX32 = 33  # FP16 real / imaginary pairs (CANN aclDataType)
ACL_FORMAT_ND = 2

# every exported symbol the public headers declare
EXPORTED_SYMBOLS = (
    "aclCreateTensor", "aclDestroyTensor", "aclGetDataType", "aclGetViewShape", "aclGetTensorAddr",
    "asdFftCreate", "asdFftSetStream", "asdFftMakePlan1D", "asdFftIstftMakePlan", "asdFftExecC2C",
    "asdFftExecC2CSeparated", "asdFftExecC2R", "asdFftExecR2C", "asdFftExecIstft", "asdFftDestroy",
    "asdFftMakePlan2D", "asdFftMakePlan3D", "asdFftGetWorkspaceSize", "asdFftSetWorkspace",
    "asdFftSynchronize", "asdFftGetType",
    "asdFftExecRaw", "asdFftDescribePlan", "asdFftPlanLaunchCount",
    "asdFftBatchPlanCreate", "asdFftBatchGetWorkspaceSize", "asdFftBatchExec", "asdFftBatchPlanDestroy",
    "asdFftBatchDescribe", "asdFftAutotune", "asdFftTuneCacheLoad",
    "asdFftServerCreate", "asdFftServerWarm", "asdFftServerSubmit", "asdFftServerDrain", "asdFftServerBatches",
    "asdFftServerDestroy", "asdFftServeRun", "asdFftServerHold", "asdFftGetErrorMessage",
    "asdFftExecC2CNoAlloc", "asdFftSetPrecision", "asdFftServerSetPrecision",
)


class FftError(RuntimeError):
    def __init__(self, where: str, status: int):
        msg = ""
        try:
            msg = last_error_message()
        except Exception:
            pass
        super().__init__(f"{where} returned {status}" + (f" ({msg})" if msg else ""))
        self.status = status


def last_error_message() -> str:
    lib = load_library()
    n = lib.asdFftGetErrorMessage(None, 0)
    buf = ctypes.create_string_buffer(int(max(1, n)))
    lib.asdFftGetErrorMessage(buf, n)
    return buf.value.decode(errors="replace")


_lib: Optional[ctypes.CDLL] = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -m sip_b200.build`")
    lib = ctypes.CDLL(path)
    vp, i32, i64, u64, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_size_t
    P64 = ctypes.POINTER(ctypes.c_int64)
    sig = {
        "aclCreateTensor": (vp, [P64, u64, ctypes.c_int, P64, i64, ctypes.c_int, P64, u64, vp]),
        "aclDestroyTensor": (i32, [vp]),
        "aclGetDataType": (i32, [vp, ctypes.POINTER(ctypes.c_int)]),
        "aclGetViewShape": (i32, [vp, ctypes.POINTER(P64), ctypes.POINTER(u64)]),
        "aclGetTensorAddr": (vp, [vp]),
        "asdFftCreate": (i32, [ctypes.POINTER(vp)]),
        "asdFftSetStream": (i32, [vp, vp]),
        "asdFftMakePlan1D": (i32, [vp, i64, ctypes.c_int, ctypes.c_int, i64, ctypes.c_int]),
        "asdFftMakePlan2D": (i32, [vp, i64, i64, ctypes.c_int, ctypes.c_int, i32]),
        "asdFftMakePlan3D": (i32, [vp, i64, i64, i64, ctypes.c_int, ctypes.c_int, i32]),
        "asdFftIstftMakePlan": (i32, [vp, vp, i64, i64, i64, ctypes.c_bool, ctypes.c_bool, ctypes.c_bool, i64,
                                      ctypes.c_bool]),
        "asdFftExecC2C": (i32, [vp, vp, vp]),
        "asdFftExecC2R": (i32, [vp, vp, vp]),
        "asdFftExecR2C": (i32, [vp, vp, vp]),
        "asdFftExecC2CSeparated": (i32, [vp, vp, vp, vp, vp]),
        "asdFftExecIstft": (i32, [vp, vp, vp, vp]),
        "asdFftDestroy": (i32, [vp]),
        "asdFftGetWorkspaceSize": (i32, [vp, ctypes.POINTER(sz)]),
        "asdFftSetWorkspace": (i32, [vp, vp]),
        "asdFftSynchronize": (i32, [vp]),
        "asdFftGetType": (i32, [vp, ctypes.POINTER(ctypes.c_int)]),
        "asdFftExecRaw": (i32, [vp, vp, vp]),
        "asdFftDescribePlan": (i64, [vp, ctypes.c_char_p, i64]),
        "asdFftPlanLaunchCount": (i32, [vp]),
        "asdFftSetPrecision": (i32, [vp, i32]),
        "asdFftServerSetPrecision": (i32, [vp, i32]),
        "asdFftBatchPlanCreate": (i32, [ctypes.POINTER(vp), P64, P64, i32, i32, ctypes.c_char_p]),
        "asdFftBatchGetWorkspaceSize": (i32, [vp, ctypes.POINTER(sz)]),
        "asdFftBatchExec": (i32, [vp, vp, vp, vp, vp, i32]),
        "asdFftBatchPlanDestroy": (i32, [vp]),
        "asdFftBatchDescribe": (i64, [vp, ctypes.c_char_p, i64]),
        "asdFftAutotune": (i32, [P64, P64, i32, i32, ctypes.c_char_p]),
        "asdFftTuneCacheLoad": (i32, [ctypes.c_char_p]),
        "asdFftServerCreate": (i32, [ctypes.POINTER(vp), i64, i32, i64, i32]),
        "asdFftServerWarm": (i32, [vp, i32, i32, i64]),
        "asdFftServerSubmit": (i64, [vp, i32, i32, i64, i64, vp, vp]),
        "asdFftServerDrain": (i64, [vp, P64, ctypes.POINTER(ctypes.c_double), i64]),
        "asdFftServerBatches": (i64, [vp]),
        "asdFftServerHold": (i32, [vp, i32]),
        "asdFftGetErrorMessage": (i64, [ctypes.c_char_p, i64]),
        "asdFftServerDestroy": (i32, [vp]),
        "asdFftServeRun": (ctypes.c_double, [vp, ctypes.c_double, i64, ctypes.c_uint64, i32,
                                             ctypes.POINTER(ctypes.c_int32), P64, ctypes.POINTER(vp),
                                             ctypes.POINTER(vp), i64, i64, i32, ctypes.POINTER(ctypes.c_double),
                                             P64, ctypes.POINTER(ctypes.c_int32)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


# --- reference-named entry points ----------------------------------------------------------------
def asdFftCreate() -> int:
    h = ctypes.c_void_p()
    st = load_library().asdFftCreate(ctypes.byref(h))
    if st != ACL_SUCCESS:
        raise FftError("asdFftCreate", st)
    return h.value


def asdFftSetStream(handle, stream) -> int:
    return load_library().asdFftSetStream(handle, stream)


def asdFftMakePlan1D(handle, fft_size, fft_type, direction, batch, dim_type=ASCEND_FFT_HORIZONTAL) -> int:
    return load_library().asdFftMakePlan1D(handle, fft_size, fft_type, direction, batch, dim_type)


def asdFftMakePlan2D(handle, x, y, fft_type, direction, batch) -> int:
    return load_library().asdFftMakePlan2D(handle, x, y, fft_type, direction, batch)


def asdFftMakePlan3D(handle, x, y, z, fft_type, direction, batch) -> int:
    return load_library().asdFftMakePlan3D(handle, x, y, z, fft_type, direction, batch)


def asdFftGetWorkspaceSize(handle) -> tuple[int, int]:
    n = ctypes.c_size_t(0)
    st = load_library().asdFftGetWorkspaceSize(handle, ctypes.byref(n))
    return st, n.value


def asdFftSetWorkspace(handle, ptr) -> int:
    return load_library().asdFftSetWorkspace(handle, ptr)


def asdFftExecC2C(handle, inp, out) -> int:
    return load_library().asdFftExecC2C(handle, _t(inp), _t(out))


def asdFftExecR2C(handle, inp, out) -> int:
    return load_library().asdFftExecR2C(handle, _t(inp), _t(out))


def asdFftExecC2R(handle, inp, out) -> int:
    return load_library().asdFftExecC2R(handle, _t(inp), _t(out))


def asdFftSynchronize(handle) -> int:
    return load_library().asdFftSynchronize(handle)


def asdFftGetType(handle) -> tuple[int, int]:
    t = ctypes.c_int(0)
    st = load_library().asdFftGetType(handle, ctypes.byref(t))
    return st, t.value


def asdFftDestroy(handle) -> int:
    return load_library().asdFftDestroy(handle)


def describe_plan(handle) -> str:
    lib = load_library()
    n = lib.asdFftDescribePlan(handle, None, 0)
    if n < 0:
        return ""
    buf = ctypes.create_string_buffer(int(n))
    lib.asdFftDescribePlan(handle, buf, n)
    return buf.value.decode()


def launch_count(handle) -> int:
    return load_library().asdFftPlanLaunchCount(handle)


# --- aclTensor -----------------------------------------------------------------------------------
class AclTensor:
    """aclTensor descriptor over a device buffer (shape, dtype, data pointer)."""

    def __init__(self, shape: Sequence[int], dtype: int, data_ptr: int, owner=None):
        lib = load_library()
        self.shape = [int(s) for s in shape]
        nd = len(self.shape)
        dims = (ctypes.c_int64 * max(1, nd))(*self.shape)
        strides = [1] * nd
        for i in range(nd - 2, -1, -1):
            strides[i] = strides[i + 1] * self.shape[i + 1]
        st = (ctypes.c_int64 * max(1, nd))(*strides)
        self.ptr = lib.aclCreateTensor(dims, nd, dtype, st, 0, ACL_FORMAT_ND, dims, nd, ctypes.c_void_p(data_ptr))
        if not self.ptr:
            raise ValueError("aclCreateTensor failed")
        self._owner = owner  # keeps the torch storage alive

    @classmethod
    def from_torch(cls, t):
        import torch

        if t.dtype == torch.complex64:
            dt = ACL_COMPLEX64
        elif t.dtype == torch.float32:
            dt = ACL_FLOAT
        else:
            raise TypeError(f"unsupported dtype {t.dtype}")
        if not t.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return cls(list(t.shape), dt, t.data_ptr(), owner=t)

    def close(self):
        if self.ptr:
            load_library().aclDestroyTensor(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _t(x):
    if isinstance(x, AclTensor):
        return x.ptr
    return x


# --- convenience plan --------------------------------------------------------------------------
class FftPlan:
    """Handle + plan + workspace; executes on torch CUDA tensors through the aclTensor entry points."""

    def __init__(self, sizes: Sequence[int], fft_type: int, direction: int, batch: int,
                 dim_type: int = ASCEND_FFT_HORIZONTAL, stream=None, precision: int = PRECISION_FP32):
        import torch

        self.sizes = [int(s) for s in sizes]
        self.fft_type = fft_type
        self.direction = direction
        self.batch = int(batch)
        self.precision = int(precision)
        self.handle = asdFftCreate()
        if self.precision != PRECISION_FP32:
            st = load_library().asdFftSetPrecision(self.handle, self.precision)
            if st != ACL_SUCCESS:
                asdFftDestroy(self.handle)
                self.handle = None
                raise FftError("asdFftSetPrecision", st)
        if len(sizes) == 1:
            st = asdFftMakePlan1D(self.handle, self.sizes[0], fft_type, direction, self.batch, dim_type)
        elif len(sizes) == 2:
            st = asdFftMakePlan2D(self.handle, self.sizes[0], self.sizes[1], fft_type, direction, self.batch)
        else:
            st = asdFftMakePlan3D(self.handle, *self.sizes, fft_type, direction, self.batch)
        if st != ACL_SUCCESS:
            asdFftDestroy(self.handle)
            self.handle = None
            raise FftError("asdFftMakePlan", st)
        st, ws = asdFftGetWorkspaceSize(self.handle)
        self.workspace_bytes = ws
        self.workspace = None
        if ws > 0:
            self.workspace = torch.empty(ws, dtype=torch.uint8, device="cuda")
            asdFftSetWorkspace(self.handle, self.workspace.data_ptr())
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        asdFftSetStream(self.handle, ctypes.c_void_p(self.stream.cuda_stream))

    def set_stream(self, stream):
        self.stream = stream
        return asdFftSetStream(self.handle, ctypes.c_void_p(stream.cuda_stream))

    def __call__(self, inp, out):
        a, b = AclTensor.from_torch(inp), AclTensor.from_torch(out)
        try:
            if self.fft_type == ASCEND_FFT_C2C:
                st = asdFftExecC2C(self.handle, a, b)
            elif self.fft_type == ASCEND_FFT_R2C:
                st = asdFftExecR2C(self.handle, a, b)
            else:
                st = asdFftExecC2R(self.handle, a, b)
        finally:
            a.close()
            b.close()
        if st != ACL_SUCCESS:
            raise FftError("asdFftExec", st)
        return out

    def exec_raw(self, inp_ptr: int, out_ptr: int) -> int:
        return load_library().asdFftExecRaw(self.handle, inp_ptr, out_ptr)

    def describe(self) -> str:
        return describe_plan(self.handle)

    def launches(self) -> int:
        return launch_count(self.handle)

    def close(self):
        if self.handle:
            asdFftDestroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --- uneven batches (one persistent launch) and the autotuner ------------------------------------
class BatchPlan:
    """Groups (length, count) of 1D C2C transforms stored back to back, run by one persistent launch."""

    def __init__(self, groups, direction=ASCEND_FFT_FORWARD, tune_cache: Optional[str] = None):
        import torch

        lib = load_library()
        self.groups = [(int(n), int(b)) for n, b in groups]
        sizes = (ctypes.c_int64 * len(self.groups))(*[n for n, _ in self.groups])
        batches = (ctypes.c_int64 * len(self.groups))(*[b for _, b in self.groups])
        h = ctypes.c_void_p()
        st = lib.asdFftBatchPlanCreate(ctypes.byref(h), sizes, batches, len(self.groups), direction,
                                       tune_cache.encode() if tune_cache else None)
        if st != ACL_SUCCESS:
            raise FftError("asdFftBatchPlanCreate", st)
        self.handle = h.value
        n = ctypes.c_size_t(0)
        lib.asdFftBatchGetWorkspaceSize(self.handle, ctypes.byref(n))
        self.workspace_bytes = n.value
        self.workspace = torch.empty(max(1, n.value), dtype=torch.uint8, device="cuda")
        self.total = sum(n * b for n, b in self.groups)
        self.offsets = []
        off = 0
        for n_, b in self.groups:
            self.offsets.append(off)
            off += n_ * b

    def __call__(self, inp, out, stream=None, use_graph=True):
        import torch

        s = stream if stream is not None else torch.cuda.current_stream()
        st = load_library().asdFftBatchExec(self.handle, inp.data_ptr(), out.data_ptr(), self.workspace.data_ptr(),
                                            ctypes.c_void_p(s.cuda_stream), 1 if use_graph else 0)
        if st != ACL_SUCCESS:
            raise FftError("asdFftBatchExec", st)
        return out

    def describe(self) -> str:
        lib = load_library()
        n = lib.asdFftBatchDescribe(self.handle, None, 0)
        buf = ctypes.create_string_buffer(int(n))
        lib.asdFftBatchDescribe(self.handle, buf, n)
        return buf.value.decode()

    def close(self):
        if self.handle:
            load_library().asdFftBatchPlanDestroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(groups, direction=ASCEND_FFT_FORWARD, cache_path: Optional[str] = None) -> int:
    lib = load_library()
    sizes = (ctypes.c_int64 * len(groups))(*[int(n) for n, _ in groups])
    rows = (ctypes.c_int64 * len(groups))(*[int(b) for _, b in groups])
    return lib.asdFftAutotune(sizes, rows, len(groups), direction, cache_path.encode() if cache_path else None)


def tune_cache_load(cache_path: str) -> int:
    return load_library().asdFftTuneCacheLoad(cache_path.encode())


# --- continuous-batching server --------------------------------------------------------------------
class Server:
    """The library's C++ continuous-batching FFT server (see include/asdsip_fft_ext.h)."""

    def __init__(self, budget_bytes=32 << 30, lanes=4, max_rows=1024, device_io=False,
                 precision: int = PRECISION_FP32):
        h = ctypes.c_void_p()
        st = load_library().asdFftServerCreate(ctypes.byref(h), int(budget_bytes), int(lanes), int(max_rows),
                                               1 if device_io else 0)
        if st != ACL_SUCCESS:
            raise FftError("asdFftServerCreate", st)
        self.handle = h.value
        if precision != PRECISION_FP32:
            st = load_library().asdFftServerSetPrecision(self.handle, int(precision))
            if st != ACL_SUCCESS:
                raise FftError("asdFftServerSetPrecision", st)

    def warm(self, fft_type, direction, n):
        return load_library().asdFftServerWarm(self.handle, fft_type, direction, n)

    def submit(self, fft_type, direction, n, rows, in_ptr, out_ptr) -> int:
        return load_library().asdFftServerSubmit(self.handle, fft_type, direction, n, rows, in_ptr, out_ptr)

    def drain(self, cap=1 << 20):
        import numpy as np

        ids = np.zeros(cap, np.int64)
        lat = np.zeros(cap, np.float64)
        n = load_library().asdFftServerDrain(self.handle, ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                             lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap)
        n = min(n, cap)
        return ids[:n], lat[:n]

    def batches(self) -> int:
        return load_library().asdFftServerBatches(self.handle)

    def hold(self, on: bool = True):
        return load_library().asdFftServerHold(self.handle, 1 if on else 0)

    def run_poisson(self, rate, count, seed, classes, pool_in, pool_out, rows_min, rows_max,
                    direction=ASCEND_FFT_FORWARD):
        import numpy as np

        k = len(classes)
        types = (ctypes.c_int32 * k)(*[int(t) for t, _ in classes])
        sizes = (ctypes.c_int64 * k)(*[int(n) for _, n in classes])
        pin = (ctypes.c_void_p * k)(*pool_in)
        pout = (ctypes.c_void_p * k)(*pool_out)
        lat = np.zeros(count, np.float64)
        rows = np.zeros(count, np.int64)
        cls = np.zeros(count, np.int32)
        wall = load_library().asdFftServeRun(
            self.handle, float(rate), int(count), int(seed), k, types, sizes, pin, pout, int(rows_min),
            int(rows_max), direction, lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            rows.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), cls.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        return wall, lat, rows, cls

    def close(self):
        if self.handle:
            load_library().asdFftServerDestroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
