// Internal interface of the learned preconditioner (learned.cu, fpcg.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace cfm {

constexpr int UNET_NLAYERS = 9;

struct UNetLayer {
    const char *name;
    int ci, co;
    int level;  // 0..3 (resolution H / 2^level)
    bool tc;    // tensor-core convolution (else CUDA cores)
};
extern const UNetLayer UNET_LAYERS[UNET_NLAYERS];
size_t unet_num_params();

struct UNetImpl;
int unet_create(int H, int W, int max_batch, UNetImpl **out);
void unet_destroy(UNetImpl *u);
size_t unet_params(const UNetImpl *u);
void unet_shape(const UNetImpl *u, int *H, int *W);
float *unet_theta(UNetImpl *u);
float *unet_grad(UNetImpl *u);
int *unet_err(UNetImpl *u);
int unet_refresh_weights(UNetImpl *u, cudaStream_t s);
// Optional scaling of input channel 0 by sqrt(cells / sum(part[0 .. nparts))),
// the partial sums of |r|^2 a solver left on the device (1 / rms(r)).
struct UNetInputScale {
    const double *part;
    int nparts;
    double cells;
    // a batch: image z reads part + z part_stride and, when cells_img is
    // given, takes cells_img[z] cells
    long long part_stride = 0;
    const double *cells_img = nullptr;
};
// x FP32 [B][H][W][2] -> out FP32 [B][H][W] (device pointers).
int unet_forward(UNetImpl *u, int B, const float *x, float *out, cudaStream_t s,
                 const UNetInputScale *in_scale = nullptr);
// Accumulates the gradient of sum(out * dout) into unet_grad (after unet_forward).
int unet_backward(UNetImpl *u, int B, const float *x, const float *dout, cudaStream_t s);
int unet_adam(UNetImpl *u, float lr, float grad_scale, cudaStream_t s);
int unet_check_err(UNetImpl *u);

}  // namespace cfm

// The C-ABI handle of a network: the net and its host-call staging buffers.
struct cfm_unet {
    cfm::UNetImpl *u = nullptr;
    float *xin = nullptr, *out = nullptr, *dout = nullptr;
    int maxB = 0;
    int smooth = 0;   // Jacobi sweeps around the network it was trained for
    int coarsen = 1;  // the systems' grid is the network's times this factor
    // checkpoint selection during training (cfm_unet_set_validation)
    unsigned long long val_seed = 0;
    int val_every = 0;           // 0: off
    int val_best_epoch = -1;     // epochs of the kept parameters
    double val_best_ms = 0.0;    // their FPCG time on the validation system
};
