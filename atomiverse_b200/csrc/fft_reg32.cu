// fft_reg32.cu -- the FP32 (mixed-precision) register forms of the PME line
// transforms (fft_reg.cuh); a separate unit so the two precisions compile
// in parallel.
#include "fft_reg.cuh"

namespace atvb {

void launch_fft_reg32(int pass, int idx, const ItemList& il, const SysParams* sp,
                      cudaStream_t s) {
    fftr::launch_any<true>(pass, idx, il, sp, s);
}

} // namespace atvb
