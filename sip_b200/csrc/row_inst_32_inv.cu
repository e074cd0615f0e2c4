// Runtime-radix row kernels, at most 32 points per thread, INVERSE direction.
#include "row_fft_inst.cuh"

namespace sipfft {

const void *runtime_row_kernel_32_inv(int io) { return runtime_row_kernel<32, false>(io); }

}  // namespace sipfft
