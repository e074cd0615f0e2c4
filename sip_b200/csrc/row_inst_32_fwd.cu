// Runtime-radix row kernels, at most 32 points per thread, FORWARD direction.
#include "row_fft_inst.cuh"

namespace sipfft {

const void *runtime_row_kernel_32_fwd(int io) { return runtime_row_kernel<32, true>(io); }

}  // namespace sipfft
