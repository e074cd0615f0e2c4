// Explicit instantiation of the runtime-radix row kernel for one points-per-
// thread bound and direction.  Each combination lives in its own translation
// unit (row_inst_*.cu) so that the slow device compiles run in parallel.
#pragma once
#include "pipelined_rows.cuh"

namespace sipfft {

template <int MAXE, bool FWD, bool COMPACT = false>
const void *runtime_row_kernel(int io)
{
    using E = RuntimeEngine<MAXE, COMPACT>;
    switch (io) {
        case IO_C2C: return reinterpret_cast<const void *>(pipelined_rows_kernel<E, FWD, IO_C2C>);
        case IO_R2C_PACKED: return reinterpret_cast<const void *>(pipelined_rows_kernel<E, FWD, IO_R2C_PACKED>);
        case IO_C2R_PACKED: return reinterpret_cast<const void *>(pipelined_rows_kernel<E, FWD, IO_C2R_PACKED>);
        default: return nullptr;
    }
}

// defined in row_inst_<maxe>_<fwd|inv>.cu
const void *runtime_row_kernel_8_fwd(int io);
const void *runtime_row_kernel_8_inv(int io);
const void *runtime_row_kernel_16_fwd(int io);
const void *runtime_row_kernel_16_inv(int io);
const void *runtime_row_kernel_32_fwd(int io);
const void *runtime_row_kernel_32_inv(int io);
// compact radix set (2..10), at most 16 points per thread, three CTAs per SM
const void *runtime_row_kernel_16c_fwd(int io);
const void *runtime_row_kernel_16c_inv(int io);

}  // namespace sipfft
