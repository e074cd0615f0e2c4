// Runtime-radix row kernels, at most 16 points per thread, FORWARD direction.
#include "row_fft_inst.cuh"

namespace sipfft {

const void *runtime_row_kernel_16_fwd(int io) { return runtime_row_kernel<16, true>(io); }

}  // namespace sipfft
