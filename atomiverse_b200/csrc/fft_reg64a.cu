// fft_reg64a.cu -- the FP64 register forms of the PME line transforms
// (fft_reg.cuh), first half of the size table; the table lookups and the
// dispatch over the four units (two precisions x two halves, compiled in
// parallel).
#include "fft_reg.cuh"

namespace atvb {

bool fftr_launch_64b(int pass, int idx, const ItemList& il, const SysParams* sp, cudaStream_t s);
bool fftr_launch_32a(int pass, int idx, const ItemList& il, const SysParams* sp, cudaStream_t s);
bool fftr_launch_32b(int pass, int idx, const ItemList& il, const SysParams* sp, cudaStream_t s);

int fft_reg_index(int n) {
    switch (n) {
#define ATVB_FFTR_IDX(i, len, a, b)                                                     \
    case len: return i;
        ATVB_FFTR_SIZES(ATVB_FFTR_IDX)
#undef ATVB_FFTR_IDX
    default: return -1;
    }
}

int fft_reg_lines(int idx, bool mixed) {
    switch (idx) {
#define ATVB_FFTR_LINES(i, len, a, b)                                                   \
    case i: return mixed ? fftr::Shape<a, b>::zlines<true>() : fftr::Shape<a, b>::zlines<false>();
        ATVB_FFTR_SIZES(ATVB_FFTR_LINES)
#undef ATVB_FFTR_LINES
    default: return 1;
    }
}

int fft_reg_cols(bool mixed) { return mixed ? fftr::cols<true>() : fftr::cols<false>(); }

void launch_fft_reg(int pass, int idx, bool mixed, const ItemList& il, const SysParams* sp,
                    cudaStream_t s) {
    if (il.n == 0)
        return;
    if (mixed) {
        if (!fftr_launch_32a(pass, idx, il, sp, s))
            fftr_launch_32b(pass, idx, il, sp, s);
    } else if (!fftr::launch_half_a<false>(pass, idx, il, sp, s)) {
        fftr_launch_64b(pass, idx, il, sp, s);
    }
}

} // namespace atvb
