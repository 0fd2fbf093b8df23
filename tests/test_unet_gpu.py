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


def test_unet_gradient_matches_oracle_per_layer(case):
    net, theta, x, dout = case
    got = net.gradient(x, dout).astype(np.float64)
    _, cache = U.forward(theta.astype(np.float64), x.astype(np.float64))
    want = U.backward(cache, dout.astype(np.float64))
    o = 0
    for name, ci, co in U.LAYERS:
        nw = 9 * ci * co
        for part, sl in (("w", slice(o, o + nw)), ("b", slice(o + nw, o + nw + co))):
            e = rel(got[sl], want[sl])
            assert e < 5e-2, (name, part, e)
        o += nw + co


def test_unet_params_roundtrip(case):
    net, theta, _, _ = case
    t2 = theta * 0.5
    net.set_params(t2)
    np.testing.assert_array_equal(net.params(), t2)
    net.set_params(theta)
