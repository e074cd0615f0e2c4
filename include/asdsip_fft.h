/*
 * asdsip_fft.h — C ABI of the B200 (sm_100a) FFT library libasdsip_fft.so.
 *
 * Drop-in for the FFT surface of AscendSiPBoost: every entry point below has
 * the same unmangled name, argument meaning, enum values and status codes as
 * the reference declaration it replaces (include/fft_api.h:17-99 of the
 * reference).  C++ callers get the reference's namespace AsdSip and its
 * reference parameters; C callers see plain pointers (same ABI).
 *
 * Streams are cudaStream_t passed as void*; tensors are described with the
 * aclTensor shim below (the CANN descriptor the reference reads with
 * aclGetDataType / aclGetViewShape, core/fft/fft_api.cpp:1047-1167);
 * their data pointers are CUDA device pointers.
 */
#ifndef ASDSIP_FFT_B200_H
#define ASDSIP_FFT_B200_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#if defined(__GNUC__)
#define ASDSIP_API __attribute__((visibility("default")))
#else
#define ASDSIP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------------
 * aclTensor descriptor shim (subset of CANN aclnn/acl_meta.h that the reference's FFT path uses).
 * ---------------------------------------------------------------------------------------------- */
typedef struct aclTensor aclTensor;

enum aclDataType {
    ACL_DT_UNDEFINED = -1,
    ACL_FLOAT = 0,
    ACL_FLOAT16 = 1,
    ACL_INT8 = 2,
    ACL_INT32 = 3,
    ACL_UINT8 = 4,
    ACL_INT16 = 6,
    ACL_UINT16 = 7,
    ACL_UINT32 = 8,
    ACL_INT64 = 9,
    ACL_UINT64 = 10,
    ACL_DOUBLE = 11,
    ACL_BOOL = 12,
    ACL_COMPLEX64 = 16,
    ACL_COMPLEX128 = 17,
    ACL_BF16 = 27,
    ACL_COMPLEX32 = 33
};
typedef enum aclDataType aclDataType;

enum aclFormat { ACL_FORMAT_UNDEFINED = -1, ACL_FORMAT_NCHW = 0, ACL_FORMAT_NHWC = 1, ACL_FORMAT_ND = 2 };
typedef enum aclFormat aclFormat;

/* Same signature as CANN's aclCreateTensor; tensorData is a CUDA device pointer,
 * offset is in elements.  Returns NULL on invalid arguments. */
ASDSIP_API aclTensor *aclCreateTensor(const int64_t *viewDims, uint64_t viewDimsNum, aclDataType dataType,
                           const int64_t *stride, int64_t offset, aclFormat format, const int64_t *storageDims,
                           uint64_t storageDimsNum, void *tensorData);
ASDSIP_API int32_t aclDestroyTensor(const aclTensor *tensor);
ASDSIP_API int32_t aclGetDataType(const aclTensor *tensor, aclDataType *dataType);
/* *viewDims is allocated with new[]; the caller releases it with delete[] (as the reference does). */
ASDSIP_API int32_t aclGetViewShape(const aclTensor *tensor, int64_t **viewDims, uint64_t *viewDimsNum);
/* Device address of element 0 of the view (storage base + offset). */
ASDSIP_API void *aclGetTensorAddr(const aclTensor *tensor);

/* ------------------------------------------------------------------------------------------------
 * FFT API (reference include/fft_api.h, core/utils/include/utils/aspb_status.h)
 * ---------------------------------------------------------------------------------------------- */
#ifdef __cplusplus
namespace AsdSip {
#endif

typedef int32_t AspbStatus;

/* core/utils/include/utils/aspb_status.h:18-27 */
enum ErrorType {
    ACL_SUCCESS = 0,
    ACL_ERROR_INVALID_PARAM = 100000,
    ACL_ERROR_OP_INPUT_NOT_MATCH = 100021,
    ACL_ERROR_OP_OUTPUT_NOT_MATCH = 100022,
    ACL_ERROR_UNSUPPORTED_DATA_TYPE = 100026,
    ACL_ERROR_FORMAT_NOT_MATCH = 100027,
    ACL_ERROR_API_NOT_SUPPORT = 200001,
    ACL_ERROR_INTERNAL_ERROR = 500000
};

typedef void *asdFftHandle;

enum asdFftStatus { SUCCESS = 0, FAILED = 1 };

/* include/fft_api.h:24-44 */
enum asdFftType {
    ASCEND_FFT_C2C = 0x10,
    ASCEND_FFT_C2R = 0x11,
    ASCEND_FFT_R2C = 0x12,
    ASCEND_STFT_C2C = 0x20,
    ASCEND_STFT_C2R = 0x21,
    ASCEND_STFT_R2C = 0x22,
    ASCEND_FFT_C2C_SEP = 0x30
};

enum asdFftDirection {
    ASCEND_FFT_FORWARD = 0x10,
    ASCEND_FFT_INVERSE = 0x11,
};

enum asdFft1dDimType {
    ASCEND_FFT_HORIZONTAL = 0x10,
    ASCEND_FFT_VERTICAL = 0x11,
};

#ifndef __cplusplus
typedef enum asdFftType asdFftType;
typedef enum asdFftDirection asdFftDirection;
typedef enum asdFft1dDimType asdFft1dDimType;
#endif

#ifdef __cplusplus
#define ASDSIP_OUT_REF(T, name) T &name
#define ASDSIP_DEFAULT(v) = v
#else
#define ASDSIP_OUT_REF(T, name) T *name
#define ASDSIP_DEFAULT(v)
#endif

/* Creates an empty plan handle.  (fft_api.h:46-48; fft_api.cpp:737-742) */
ASDSIP_API AspbStatus asdFftCreate(ASDSIP_OUT_REF(asdFftHandle, handle));

/* Binds a cudaStream_t to the handle; NULL -> ACL_ERROR_INVALID_PARAM.  (fft_api.h:50-51; fft_api.cpp:744-759) */
ASDSIP_API AspbStatus asdFftSetStream(asdFftHandle handle, void *stream);

/* 1D plan: 0 < fftSize <= 2^27, batchSize > 0.  HORIZONTAL: [batch, N];
 * VERTICAL (C2C): [N, batch].  (fft_api.h:53-57; fft_api.cpp:761-795) */
ASDSIP_API AspbStatus asdFftMakePlan1D(asdFftHandle handle, int64_t fftSize, enum asdFftType fftType,
                            enum asdFftDirection direction, int64_t batchSize,
                            enum asdFft1dDimType dimType ASDSIP_DEFAULT(ASCEND_FFT_HORIZONTAL));

/* ISTFT plan for input complex64 [channel, nFft, frames] (frames > 1, 0 < hop <= winLength == nFft < 1500,
 * hop < 1500); center / normalized / onesided / length / returnComplex are forced to true / false / false / 0 /
 * true as in the reference.  Builds an INVERSE C2C plan (GetType reports C2C) that needs a workspace.
 * (fft_api.h:59-62; core/fft/istft.cpp:300-390, 530-552) */
ASDSIP_API AspbStatus asdFftIstftMakePlan(asdFftHandle handle, const aclTensor *input, const int64_t nFft,
                               const int64_t hopLengthOpt, const int64_t winLengthOpt,
                               const bool center ASDSIP_DEFAULT(true), const bool normalized ASDSIP_DEFAULT(false),
                               const bool onesidedOpt ASDSIP_DEFAULT(false), int64_t lengthOpt ASDSIP_DEFAULT(0),
                               const bool returnComplex ASDSIP_DEFAULT(true));

/* C2C on complex64 tensors whose trailing dims equal the plan sizes.  (fft_api.h:65; fft_api.cpp:1169-1189) */
ASDSIP_API AspbStatus asdFftExecC2C(asdFftHandle handle, const aclTensor *input, const aclTensor *output);

/* C2C on planar float32 real/imag tensors of a plan made with type ASCEND_FFT_C2C_SEP (1D, 2D or 3D); the four
 * tensors must have the same shape (else ACL_ERROR_INTERNAL_ERROR, as in the reference); in place when both
 * planes are.  (fft_api.h:68-69; fft_api.cpp:1236-1342) */
ASDSIP_API AspbStatus asdFftExecC2CSeparated(asdFftHandle handle, const aclTensor *inputReal, const aclTensor *inputImag,
                                  const aclTensor *outputReal, const aclTensor *outputImag);

/* C2R: complex64 [.., N/2+1] -> float32 [.., N].  (fft_api.h:73; fft_api.cpp:1191-1211) */
ASDSIP_API AspbStatus asdFftExecC2R(asdFftHandle handle, const aclTensor *input, const aclTensor *output);

/* R2C: float32 [.., N] -> complex64 [.., N/2+1].  (fft_api.h:76; fft_api.cpp:1213-1233) */
ASDSIP_API AspbStatus asdFftExecR2C(asdFftHandle handle, const aclTensor *input, const aclTensor *output);

/* ISTFT execution: window float32 [nFft], output complex64 [channel, nFft + hop (frames - 1) - 2 (nFft / 2)].
 * (fft_api.h:78-79; core/fft/istft.cpp:554-575; fftcore/fft_core_istft_any.cpp:292-378) */
ASDSIP_API AspbStatus asdFftExecIstft(asdFftHandle handle, const aclTensor *input, const aclTensor *windowOpt,
                           const aclTensor *output);

/* Destroys the handle and releases its plan.  (fft_api.h:82; fft_api.cpp:872-881) */
ASDSIP_API AspbStatus asdFftDestroy(asdFftHandle handle);

/* 2D plan over [batch, X, Y].  (fft_api.h:84-85; fft_api.cpp:883-903) */
ASDSIP_API AspbStatus asdFftMakePlan2D(asdFftHandle handle, int64_t fftSizeX, int64_t fftSizeY, enum asdFftType fftType,
                            enum asdFftDirection direction, int32_t batchSize);

/* 3D plan over [batch, X, Y, Z].  (fft_api.h:87-88; fft_api.cpp:905-931) */
ASDSIP_API AspbStatus asdFftMakePlan3D(asdFftHandle handle, int64_t fftSizeX, int64_t fftSizeY, int64_t fftSizeZ,
                            enum asdFftType fftType, enum asdFftDirection direction, int32_t batchSize);

/* Bytes of caller-owned device workspace the plan needs (may be 0).  (fft_api.h:90; fft_api.cpp:933-947) */
ASDSIP_API AspbStatus asdFftGetWorkspaceSize(asdFftHandle handle, ASDSIP_OUT_REF(size_t, workspaceSize));

/* Binds the caller's workspace (device memory, >= GetWorkspaceSize bytes).  (fft_api.h:92; fft_api.cpp:949-961) */
ASDSIP_API AspbStatus asdFftSetWorkspace(asdFftHandle handle, void *workspace);

/* Waits for the handle's stream; invalid handle -> ACL_ERROR_INTERNAL_ERROR.  (fft_api.h:94; fft_api.cpp:963-973) */
ASDSIP_API AspbStatus asdFftSynchronize(asdFftHandle handle);

/* Plan type; invalid handle -> ACL_ERROR_INTERNAL_ERROR.  (fft_api.h:96; fft_api.cpp:975-987) */
ASDSIP_API AspbStatus asdFftGetType(asdFftHandle handle, ASDSIP_OUT_REF(enum asdFftType, fftType));

#ifdef __cplusplus
}  /* namespace AsdSip */
#endif

#ifdef __cplusplus
}
#endif

#endif /* ASDSIP_FFT_B200_H */
