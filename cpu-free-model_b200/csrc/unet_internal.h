// Internal interface of the tensor-core convolutions used by the learned
// preconditioner (unet.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "cfm_internal.h"
#include "learned_internal.h"

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

// Grid barrier state of the persistent forward (uf_grid_sync).
struct UfBarrier {
    unsigned long long count;  // arrivals, a multiple of the grid between passes
    int error;                 // set by a wait that ran out of budget (or a pipeline timeout)
    int where;                 // barrier index of the first timeout
    unsigned long long timeout_ns;
};

// The whole U-Net forward as one persistent cooperative kernel
// (unet_fused.cuh): conv[0..6] are the tensor-core layers e1 e2 e3 d3 d2 d1
// d0 as tc_conv_fwd would run them (their outputs h1 h2 h3 g3 g2 g1 g0);
// skip[l] / uout[l], when set, fold the following upsample-and-add into
// layer l (uout = up(out) + skip at twice the resolution).  The output and
// every activation are bit-identical to the per-layer kernels.
// CFM_UNSUPPORTED when a layer's staging does not fit the shared ring.
struct FusedForwardArgs {
    int B, H, W;
    const float *x;
    float *out;
    UNetInputScale in_scale;
    const float *cin_w, *cin_b, *cout_w, *cout_b;
    __nv_bfloat16 *h0, *p1, *h1, *p2, *h2, *p3;
    ConvArgs conv[7];
    const __nv_bfloat16 *skip[7];
    __nv_bfloat16 *uout[7];
    UfBarrier *bar;  // zeroed before the first pass
};
int unet_forward_fused(const FusedForwardArgs &f, cudaStream_t s);

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
