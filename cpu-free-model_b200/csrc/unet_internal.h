// Internal interface of the tensor-core convolutions used by the learned
// preconditioner (unet.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace cfm {

// out = act(conv3x3(x, w) + bias) [* (mask > 0)], NHWC BF16, padding 1.
// w is [9][Cout][Cin] (tap = 3 dy + dx), bias FP32 [Cout] or null.
struct ConvArgs {
    const __nv_bfloat16 *x;
    const __nv_bfloat16 *w;
    const float *bias;
    const __nv_bfloat16 *mask;  // [B][H][W][Cout] or null
    __nv_bfloat16 *out;
    int *err;  // device word, nonzero after a timed-out pipeline wait
    int B, H, W, Cin, Cout;
    int relu;
    // optional split-K workspace (FP32); layers with fewer pixel tiles than
    // SMs then split their K steps over several CTAs
    float *ws = nullptr;
    long long ws_floats = 0;
};
int tc_conv_fwd(const ConvArgs &a, cudaStream_t s);
// Split-K workspace a net keeps for its convolutions (floats).
constexpr long long TC_WS_FLOATS = 4LL << 20;

// dw[tap][co][ci] += sum over pixels of dz[p][co] * x[p + shift(tap)][ci],
// x and dz NHWC BF16 (zero outside the image).  The K (pixel) range is
// split over CTAs; the splits' partial tiles go to the workspace `ws` and
// are added in split order (deterministic).
struct WgradArgs {
    const __nv_bfloat16 *x;
    const __nv_bfloat16 *dz;
    float *dw;
    int *err;
    int B, H, W, Cin, Cout;
    float *ws = nullptr;  // at least 9 * Cin * Cout floats; more lets K split wider
    long long ws_floats = 0;
};
int tc_conv_wgrad(const WgradArgs &a, cudaStream_t s);
// Workspace (floats) the widest K split of that weight gradient uses on a
// device with `num_sms` SMs.
long long tc_wgrad_ws_floats(int B, int H, int W, int Cin, int Cout, int num_sms);

}  // namespace cfm
