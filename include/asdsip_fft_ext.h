/*
 * asdsip_fft_ext.h — entry points of libasdsip_fft.so that have no
 * counterpart in the reference's fft_api.h.  They serve the additions of
 * this library (raw-pointer execution for callers that do not build
 * aclTensor descriptors, plan inspection, uneven batching, serving).
 */
#ifndef ASDSIP_FFT_B200_EXT_H
#define ASDSIP_FFT_B200_EXT_H

#include "asdsip_fft.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Executes an initialised plan on raw device pointers (layouts as for the
 * aclTensor entry points; in == out is accepted for C2C plans).  No
 * counterpart in the reference. */
ASDSIP_API int32_t asdFftExecRaw(void *handle, const void *input, void *output);

/* Writes a one-line-per-launch description of the plan into buf
 * (NUL-terminated, truncated to len).  Returns the full length needed. */
ASDSIP_API int64_t asdFftDescribePlan(void *handle, char *buf, int64_t len);

/* Message of the last failing call on the calling thread (NUL-terminated); returns the length needed. */
ASDSIP_API int64_t asdFftGetErrorMessage(char *buf, int64_t len);

/* Number of kernel launches one execution of the plan issues. */
ASDSIP_API int32_t asdFftPlanLaunchCount(void *handle);

/* ---- arithmetic of the transform stages.  No counterpart in the reference (its cores are FP32 only).
 * mode 0: FP32 CUDA-core kernels (default).
 * mode 1: tensor-core (tcgen05) DFT-matrix stages, operands split into FP16 hi + lo parts with a
 *         power-of-two scale per tile, three products hi*hi + hi*lo + lo*hi accumulated in FP32.
 * mode 2: the same with BF16 hi + lo parts (no scaling; about 16 significant bits per operand).
 * mode 3: per transform length, the arithmetic that the autotuner (asdFftAutotune, or a cache loaded
 *         with asdFftTuneCacheLoad) measured fastest on this GPU; FP32 for lengths it has not timed.
 * Tensor-core stages exist for transform lengths 256, 1024, 2048 and 4096 of a C2C axis (and 512, 2048,
 * 4096 and 8192 for R2C / C2R, whose packed inner transform has half the length); every other step keeps the FP32
 * kernels, which asdFftDescribePlan shows.  Strided axes of 1024, 2048 and 4096 points run their
 * tensor-core stages as rows between two transposes, which needs workspace for two copies of the data.
 * May be called before or after MakePlan*: an initialised plan is rebuilt; when the rebuilt plan needs
 * more workspace than before, the workspace set earlier is dropped (exec then returns the missing-
 * workspace error) and asdFftGetWorkspaceSize reports the new size for asdFftSetWorkspace.  Returns
 * ACL_ERROR_INVALID_PARAM for an unknown handle or mode. */
ASDSIP_API int32_t asdFftSetPrecision(void *handle, int32_t mode);

/* ---- uneven batches: many 1D C2C groups (length sizes[i], count batches[i]) stored back to back,
 * executed by ONE persistent kernel launch (optionally replayed from a captured CUDA graph).
 * tune_cache: optional path of the autotuner's cache (choices for this GPU are loaded). */
ASDSIP_API int32_t asdFftBatchPlanCreate(void **plan, const int64_t *sizes, const int64_t *batches, int32_t ngroups,
                                         int32_t direction, const char *tune_cache);
ASDSIP_API int32_t asdFftBatchGetWorkspaceSize(void *plan, size_t *bytes);
/* in != out; workspace of GetWorkspaceSize bytes; stream = cudaStream_t; use_graph != 0 captures once and
 * replays while (in, out, workspace, stream) stay the same. */
ASDSIP_API int32_t asdFftBatchExec(void *plan, const void *input, void *output, void *workspace, void *stream,
                                   int32_t use_graph);
ASDSIP_API int32_t asdFftBatchPlanDestroy(void *plan);
ASDSIP_API int64_t asdFftBatchDescribe(void *plan, char *buf, int64_t len);

/* ---- autotuner: for each length (rows[i] transforms, capped at 256) times the radix orders, elements per
 * thread and tile shapes (threads per CTA) of the SIMT tile kernels and keeps the fastest (uneven-batch
 * plans use it), and for lengths with a tensor-core stage times the whole plan in FP32 and in the FP16 x3
 * and BF16 x3 forms and keeps the fastest (plans in precision mode 3 use it).  cache_path (optional)
 * receives one JSON object per line keyed by GPU name, type and length.  TuneCacheLoad returns the number
 * of entries loaded for this GPU. */
ASDSIP_API int32_t asdFftAutotune(const int64_t *sizes, const int64_t *rows, int32_t n, int32_t direction,
                                  const char *cache_path);
ASDSIP_API int32_t asdFftTuneCacheLoad(const char *cache_path);

/* ---- continuous-batching server: requests (type C2C 0x10 or R2C 0x12, direction, length n, rows) are
 * admitted by a byte budget onto `lanes` CUDA streams with resident plans (one per class, sized for
 * max_rows) and resident staging buffers; same-class requests that are pending when a lane frees up are
 * batched into one launch.  device_io != 0: request buffers are device pointers, else host (pinned). */
ASDSIP_API int32_t asdFftServerCreate(void **server, int64_t budget_bytes, int32_t lanes, int64_t max_rows,
                                      int32_t device_io);
/* Stage arithmetic of the server's resident plans (modes of asdFftSetPrecision); call before the first
 * Warm / Submit (ACL_ERROR_INVALID_PARAM afterwards). */
ASDSIP_API int32_t asdFftServerSetPrecision(void *server, int32_t mode);
ASDSIP_API int32_t asdFftServerWarm(void *server, int32_t type, int32_t direction, int64_t n);
/* Returns the request id (>= 0) or -1. */
ASDSIP_API int64_t asdFftServerSubmit(void *server, int32_t type, int32_t direction, int64_t n, int64_t rows,
                                      const void *input, void *output);
/* Waits for every submitted request; writes up to cap (id, latency in seconds; < 0 = failed). */
ASDSIP_API int64_t asdFftServerDrain(void *server, int64_t *ids, double *latency_s, int64_t cap);
ASDSIP_API int64_t asdFftServerBatches(void *server);
/* hold != 0: keep admitting nothing (requests queue); 0: resume. */
ASDSIP_API int32_t asdFftServerHold(void *server, int32_t hold);
ASDSIP_API int32_t asdFftServerDestroy(void *server);
/* Poisson load generator over per-class input/output pools; returns wall seconds (< 0 on error). */
ASDSIP_API double asdFftServeRun(void *server, double rate, int64_t count, uint64_t seed, int32_t nclasses,
                                 const int32_t *types, const int64_t *sizes, const void *const *pool_in,
                                 void *const *pool_out, int64_t rows_min, int64_t rows_max, int32_t direction,
                                 double *latency_s, int64_t *rows_out, int32_t *class_out);

/* ---- 1D C2C that allocates nothing.  No counterpart in the reference.
 * For callers that cannot allocate device memory when they need the transform (allocation-free
 * real-time loops, hosts that own every allocation): the long-transform path normally needs a plan
 * (cudaMalloc'd twiddle tables) and a caller workspace; this entry point keeps both in a fixed 8.5 MiB
 * __device__ array of the library instead, held on every GPU that loads the library until exit.
 * Limits: fftSize in 16385..2^20 splitting into two passes of <= 2048 points (radices 2-16/3/5/7/11/13),
 * fftSize * batchSize <= 2^20 complex values; larger sizes return ACL_ERROR_INVALID_PARAM.  Same layout
 * and semantics as a HORIZONTAL C2C plan ([batch, N] complex64, unnormalised, in == out allowed).
 * Calls that overlap on the GPU share the array and race.  The first call on a device looks up the
 * array's address; make it before any stream capture. */
ASDSIP_API int32_t asdFftExecC2CNoAlloc(const void *input, void *output, int64_t fftSize, int64_t batchSize,
                                        int32_t direction, void *stream);

#ifdef __cplusplus
}
#endif

#endif
