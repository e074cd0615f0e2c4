// Runtime-radix row kernels, at most 16 points per thread, INVERSE direction.
#include "row_fft_inst.cuh"

namespace sipfft {

const void *runtime_row_kernel_16_inv(int io) { return runtime_row_kernel<16, false>(io); }

}  // namespace sipfft
