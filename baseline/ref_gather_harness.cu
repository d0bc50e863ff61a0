// Launch harness for the reference's own CUDA gather, compiled from the
// reference's source for sm_100a (the Makefile beside this file includes
// src/integration/cuda/kernels.cu from a reference checkout; nothing of it is
// copied here). It launches the reference's compensated-FP32 CSR kernels
// with the reference engine's launch rule (src/integration/cuda/device.rs):
// the layout by entries per bin (block above 5000, warp above 256 for 2D
// tables, sub-warp below; device.rs:2355-2363), 128 threads, a grid of
// (bin groups, frames / 4) and at most 256 frames per launch (device.rs:41,
// :816-845). Inputs are the reference's upload formats: u32 row pointers and
// columns, f32 weights, f64 denominators; results are [I, sigma] interleaved
// per bin (kernels.cu:75-108). Used by bench.py only, as a measured baseline
// on the same GPU.
#include <cstdint>

#include "kernels.cu"

namespace {

using Kern = void (*)(const unsigned *, const unsigned *, const float *, const double *,
                      const void *, double *, unsigned, unsigned, unsigned, unsigned);

template <typename P>
Kern pick(const char *layout, bool variance);

#define REF_PICK(P, PREFIX)                                                                \
    template <>                                                                            \
    Kern pick<P>(const char *layout, bool variance) {                                      \
        if (layout[0] == 'b') return Kern(variance ? PREFIX##_block_iv : PREFIX##_block_i); \
        if (layout[0] == 'w') return Kern(variance ? PREFIX##_warp_iv : PREFIX##_warp_i);   \
        return Kern(variance ? PREFIX##_subwarp_iv : PREFIX##_subwarp_i);                  \
    }
REF_PICK(unsigned short, u16_compensated)
REF_PICK(unsigned, u32_compensated)
REF_PICK(int, i32_compensated)
REF_PICK(float, compensated)

}  // namespace

extern "C" {

// The layout the reference engine picks for a table (device.rs:2355-2363).
const char *ref_gather_layout(int64_t entries, int64_t bins, int allow_subwarp) {
    if (allow_subwarp && entries <= bins * 256) return "subwarp";
    if (entries <= bins * 5000) return "warp";
    return "block";
}

// dtype: 0 u16, 1 u32, 2 i32, 3 f32. Launches every 256 frames as the
// reference's engine does; returns a cudaError_t.
int ref_gather_launch(int dtype, const char *layout, int variance, const unsigned *rows,
                      const unsigned *columns, const float *weights, const double *den,
                      const void *frames, double *out, unsigned pixels, unsigned bins,
                      unsigned n_frames, void *stream) {
    Kern k = nullptr;
    size_t px = 4;
    switch (dtype) {
    case 0: k = pick<unsigned short>(layout, variance); px = 2; break;
    case 1: k = pick<unsigned>(layout, variance); break;
    case 2: k = pick<int>(layout, variance); break;
    case 3: k = pick<float>(layout, variance); break;
    default: return int(cudaErrorInvalidValue);
    }
    const unsigned bpb = layout[0] == 'b' ? 1 : layout[0] == 'w' ? 4 : 16;
    const unsigned groups = (bins + bpb - 1) / bpb;
    const unsigned out_per_frame = bins * (variance ? 2 : 1);
    for (unsigned first = 0; first < n_frames; first += 256) {
        const unsigned count = n_frames - first < 256 ? n_frames - first : 256;
        const void *in = static_cast<const unsigned char *>(frames) + size_t(first) * pixels * px;
        k<<<dim3(groups, (count + 3) / 4), 128, 0, static_cast<cudaStream_t>(stream)>>>(
            rows, columns, weights, den, in, out + size_t(first) * out_per_frame, pixels, bins, 1,
            count);
    }
    return int(cudaGetLastError());
}

}  // extern "C"
