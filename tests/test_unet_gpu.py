"""U-Net forward and parameter gradient on the GPU (tensor-core convolutions,
BF16 activations, FP32 accumulation) against the NumPy oracle evaluated in
float64 on the same BF16-rounded weights and activations.  The GPU rounds
each activation once after FP32 accumulation and the oracle after float64
accumulation, so single BF16 roundings can differ; the bar is a relative
L2 error of 2e-2 on the output and 5e-2 per layer on the gradient."""
import numpy as np
import pytest

import cfm
import unet_oracle as U

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)


@pytest.fixture(scope="module")
def case():
    rng = np.random.default_rng(1)
    net = cfm.UNet(32, 256, max_batch=2, seed=3)
    theta = net.params()
    x = rng.normal(size=(2, 32, 256, 2)).astype(np.float32)
    dout = rng.normal(size=(2, 32, 256)).astype(np.float32)
    return net, theta, x, dout


def test_unet_forward_matches_oracle(case):
    net, theta, x, _ = case
    got = net.forward(x)
    want, _ = U.forward(theta.astype(np.float64), x.astype(np.float64))
    assert rel(got, want) < 2e-2, rel(got, want)


def test_unet_backward_matches_oracle_on_gpu_activations(case):
    """The backward kernels alone: the oracle's backward runs on the GPU's
    own forward activations (same ReLU masks), rounding the gradient tensors
    to BF16 where the GPU stores them.  Per-layer relative error < 2e-2."""
    net, theta, x, dout = case
    got = net.gradient(x, dout).astype(np.float64)
    acts = net.activations(x.shape[0])
    _, cache = U.forward(theta.astype(np.float64), x.astype(np.float64))
    cache.update({k: v.astype(np.float64) for k, v in acts.items()})
    want = U.backward(cache, dout.astype(np.float64), round_bf16=True)
    o, errs = 0, {}
    for name, ci, co in U.LAYERS:
        nw = 9 * ci * co
        errs[name + ".w"] = rel(got[o:o + nw], want[o:o + nw])
        errs[name + ".b"] = rel(got[o + nw:o + nw + co], want[o + nw:o + nw + co])
        o += nw + co
    print("relative gradient errors:", errs)
    assert all(e < 2e-2 for e in errs.values()), errs


def test_unet_gradient_end_to_end_close_to_float64(case):
    """End to end against the float64 oracle: the GPU's BF16 activations and
    tensor-core accumulation differ from float64 by ~0.2% (the forward
    test), which flips a few ReLU masks near zero; each flip changes the
    backpropagated gradient by a full term, so the bar here is direction
    (cosine > 0.99) and 15% relative error per layer."""
    net, theta, x, dout = case
    got = net.gradient(x, dout).astype(np.float64)
    _, cache = U.forward(theta.astype(np.float64), x.astype(np.float64))
    want = U.backward(cache, dout.astype(np.float64))
    o = 0
    for name, ci, co in U.LAYERS:
        sl = slice(o, o + 9 * ci * co + co)
        a, b = got[sl], want[sl]
        assert rel(a, b) < 0.15 and a @ b / (np.linalg.norm(a) * np.linalg.norm(b)) > 0.99, name
        o += 9 * ci * co + co


def test_unet_params_roundtrip(case):
    net, theta, _, _ = case
    t2 = theta * 0.5
    net.set_params(t2)
    np.testing.assert_array_equal(net.params(), t2)
    net.set_params(theta)


def test_training_step_timer():
    """cfm_unet_time_train_step runs forward, backward and Adam on device
    buffers; the network stays finite and usable afterwards."""
    net = cfm.UNet(32, 256, max_batch=2, seed=4)
    ms = net.time_train_step(2, 3)
    assert ms > 0
    y = net.forward(np.zeros((1, 32, 256, 2), np.float32))
    assert np.isfinite(y).all()
