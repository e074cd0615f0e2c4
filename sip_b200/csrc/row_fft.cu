// Runtime-radix TMA-pipelined row kernels (pipelined_rows.cuh, instantiated in
// row_inst_*.cu) and their host-side launch helpers.
#include <vector>

#include "row_fft_inst.cuh"
#include "sipfft_internal.h"

namespace sipfft {

namespace {

const void *row_fn_io8(bool forward, int io)
{
    return forward ? runtime_row_kernel_8_fwd(io) : runtime_row_kernel_8_inv(io);
}
const void *row_fn_io16(bool forward, int io)
{
    return forward ? runtime_row_kernel_16_fwd(io) : runtime_row_kernel_16_inv(io);
}
const void *row_fn_io32(bool forward, int io)
{
    return forward ? runtime_row_kernel_32_fwd(io) : runtime_row_kernel_32_inv(io);
}

// the compact engine when the tile's radices are all <= kCompactMaxRadix and its
// CTA has at most 256 threads
bool compact_ok(const TileDesc &d)
{
    if (d.tb * d.tpt > 256) return false;
    for (int s = 0; s < d.nstages; s++)
        if (d.radix[s] > kCompactMaxRadix) return false;
    return true;
}

const void *pick(const TileDesc &d, int maxe, bool forward)
{
    if (maxe <= 8) return row_fn_io8(forward, d.io);
    if (maxe <= 16) {
        if (compact_ok(d)) return forward ? runtime_row_kernel_16c_fwd(d.io) : runtime_row_kernel_16c_inv(d.io);
        return row_fn_io16(forward, d.io);
    }
    return row_fn_io32(forward, d.io);
}

}  // namespace

size_t row_kernel_smem(const TileDesc &d)
{
    // row_bufs: 1 (single-buffered engines), 2, or 3 (ping-pong work area); 0 reads as 2
    return 128 + (d.row_bufs >= 1 ? d.row_bufs : 2) * static_cast<size_t>(d.g_ns) * sizeof(float2);
}

// Raises a kernel's dynamic shared-memory limit to what the SM allows next
// to the kernel's static shared memory.
cudaError_t allow_max_dynamic_smem(const void *fn)
{
    cudaFuncAttributes attr{};
    cudaError_t e = cudaFuncGetAttributes(&attr, fn);
    if (e != cudaSuccess) return e;
    const int limit = kMaxSmemBytes - static_cast<int>(attr.sharedSizeBytes);
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
}

int kernel_blocks_per_sm(const void *fn, int threads, size_t smem)
{
    int nb = 0;
    if (!fn) return 0;
    if (allow_max_dynamic_smem(fn) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nb;
}

cudaError_t launch_pdl(const void *fn, dim3 grid, dim3 block, size_t smem, cudaStream_t st, void **args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

cudaError_t launch_kernel_fn(const void *fn, const TileDesc &d, int grid, size_t smem, int *err, cudaStream_t st)
{
    if (!fn || d.tb * d.tpt > 512 || smem > static_cast<size_t>(kMaxSmemBytes) || grid <= 0)
        return cudaErrorInvalidConfiguration;
    TileDesc dd = d;
    void *args[] = {&dd, &err};
    return launch_pdl(fn, dim3(grid), dim3(d.tb * d.tpt), smem, st, args);
}

void row_kernel_fns(std::vector<const void *> &out)
{
    for (int io : {IO_C2C, IO_R2C_PACKED, IO_C2R_PACKED}) {
        for (bool f : {true, false}) {
            out.push_back(row_fn_io8(f, io));
            out.push_back(row_fn_io16(f, io));
            out.push_back(row_fn_io32(f, io));
            out.push_back(f ? runtime_row_kernel_16c_fwd(io) : runtime_row_kernel_16c_inv(io));
        }
    }
}

int row_kernel_blocks_per_sm(const TileDesc &d, int maxe, bool forward)
{
    return kernel_blocks_per_sm(pick(d, maxe, forward), d.tb * d.tpt, row_kernel_smem(d));
}

cudaError_t launch_row_tiles(const TileDesc &d, int maxe, bool forward, int grid, int *err, cudaStream_t st)
{
    return launch_kernel_fn(pick(d, maxe, forward), d, grid, row_kernel_smem(d), err, st);
}

}  // namespace sipfft
