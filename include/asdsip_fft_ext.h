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

/* Number of kernel launches one execution of the plan issues. */
ASDSIP_API int32_t asdFftPlanLaunchCount(void *handle);

#ifdef __cplusplus
}
#endif

#endif
