// Runtime-radix row kernels of the compact radix set (2..10), at most 16 points
// per thread, FORWARD direction.
#include "row_fft_inst.cuh"

namespace sipfft {

const void *runtime_row_kernel_16c_fwd(int io) { return runtime_row_kernel<16, true, true>(io); }

}  // namespace sipfft
