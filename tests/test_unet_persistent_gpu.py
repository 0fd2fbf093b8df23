"""The persistent U-Net forward (one cooperative kernel over all layers)
against the per-layer kernels: the output and all fourteen activations
bit for bit, at the preconditioner's shape and at uneven ones, and a learned
FPCG solve that takes the same iterations and returns the same x with
either forward inside its graph."""
import numpy as np
import pytest

import cfm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("H,W,B", [(256, 256, 1), (32, 256, 2), (64, 512, 3), (128, 256, 4)])
def test_persistent_forward_bit_identical(H, W, B):
    rng = np.random.default_rng(H + W + B)
    net = cfm.UNet(H, W, max_batch=B, seed=H + B)
    x = rng.normal(size=(B, H, W, 2)).astype(np.float32)
    net.set_forward_mode(cfm.UNET_FORWARD_LAYERS)
    want = net.forward(x)
    acts = net.activations(B)
    net.set_forward_mode(cfm.UNET_FORWARD_PERSISTENT)
    for _ in range(2):  # the barrier and ring state carry over between calls
        got = net.forward(x)
        np.testing.assert_array_equal(got, want)
    for name, a in net.activations(B).items():
        np.testing.assert_array_equal(a, acts[name], err_msg=name)
    net.close()


def test_fpcg_same_with_either_forward():
    k, f = cfm.varcoef_problem((256, 256), 5)
    S = cfm.Stencil(k)
    out = []
    for mode in (cfm.UNET_FORWARD_LAYERS, cfm.UNET_FORWARD_PERSISTENT):
        net = cfm.UNet(256, 256, max_batch=1, seed=4)
        net.set_training_info(2, 1)
        net.set_forward_mode(mode)
        fp = cfm.FPCG(S, k, net, maxiter=60, tol=1e-8)
        x, st = fp.solve(f)
        out.append((x, st.iterations))
        fp.close()
        net.close()
    assert out[0][1] == out[1][1]
    np.testing.assert_array_equal(out[0][0], out[1][0])
