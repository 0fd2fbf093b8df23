"""Tensor-core (tcgen05) 3x3 convolutions against a NumPy convolution of the
same BF16 values: forward with bias / ReLU (output rounded to BF16, so a
tolerance of a few BF16 ulps) and the FP32 weight gradient (FP32
accumulation of exact products), over every channel width the network uses,
odd batch sizes and both operand swizzles (32- and 64-channel K chunks)."""
import numpy as np
import pytest

import cfm

pytestmark = pytest.mark.gpu


def bf16_round(a):
    return cfm.from_bf16_bits(cfm.to_bf16_bits(a))


def conv_ref(x, w, bias=None, relu=False):
    """x [B,H,W,Ci], w [9,Co,Ci] float64 -> [B,H,W,Co]; zero padding 1."""
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((B, H, W, w.shape[1]))
    for t in range(9):
        dy, dx = divmod(t, 3)
        out += xp[:, dy:dy + H, dx:dx + W, :] @ w[t].T
    if bias is not None:
        out += bias
    return np.maximum(out, 0) if relu else out


def wgrad_ref(x, dz):
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dw = np.zeros((9, dz.shape[3], x.shape[3]))
    for t in range(9):
        dy, dx = divmod(t, 3)
        dw[t] = np.einsum("byxo,byxi->oi", dz, xp[:, dy:dy + H, dx:dx + W, :])
    return dw


@pytest.mark.parametrize("B,H,W,Cin,Cout", [
    (1, 8, 16, 32, 32), (2, 16, 64, 64, 64), (1, 4, 128, 128, 128), (1, 2, 256, 256, 256),
    (3, 64, 64, 32, 256), (1, 16, 32, 256, 32), (2, 8, 512, 32, 32), (1, 6, 128, 96, 64)])
@pytest.mark.parametrize("act", ["plain", "bias_relu"])
def test_tc_conv_forward(B, H, W, Cin, Cout, act):
    rng = np.random.default_rng(B * 1000 + H + W + Cin + Cout)
    x = bf16_round(rng.normal(size=(B, H, W, Cin)).astype(np.float32))
    w = bf16_round((rng.normal(size=(9, Cout, Cin)) / np.sqrt(9 * Cin)).astype(np.float32))
    bias = rng.normal(size=Cout).astype(np.float32) * 0.1 if act == "bias_relu" else None
    got = cfm.from_bf16_bits(cfm.tc_conv3x3(cfm.to_bf16_bits(x), cfm.to_bf16_bits(w), bias,
                                            relu=act == "bias_relu")).astype(np.float64)
    ref = conv_ref(x.astype(np.float64), w.astype(np.float64), bias, act == "bias_relu")
    scale = np.sqrt(np.mean(ref ** 2)) + 1e-30
    err = np.abs(got - ref)
    # BF16 output rounding (2^-8 relative) plus FP32 accumulation
    assert np.all(err <= 2 ** -8 * np.abs(ref) + 1e-4 * scale), err.max() / scale


@pytest.mark.parametrize("B,H,W,Cin,Cout", [
    (1, 8, 64, 32, 32), (2, 16, 64, 64, 128), (1, 4, 128, 128, 64), (1, 4, 64, 256, 256),
    (1, 2, 32, 32, 64), (2, 32, 256, 64, 32), (1, 8, 64, 128, 256), (2, 4, 96, 64, 64),
    (1, 4, 64, 96, 32), (1, 4, 32, 160, 64)])
def test_tc_conv_weight_gradient(B, H, W, Cin, Cout):
    rng = np.random.default_rng(B + H + W + Cin + 7 * Cout)
    x = bf16_round(rng.normal(size=(B, H, W, Cin)).astype(np.float32))
    dz = bf16_round(rng.normal(size=(B, H, W, Cout)).astype(np.float32))
    got = cfm.tc_conv3x3_wgrad(cfm.to_bf16_bits(x), cfm.to_bf16_bits(dz)).astype(np.float64)
    ref = wgrad_ref(x.astype(np.float64), dz.astype(np.float64))
    scale = np.sqrt(B * H * W)
    assert np.max(np.abs(got - ref)) <= 1e-4 * scale, np.max(np.abs(got - ref)) / scale
    # the K splits are added in split order: a second call gives the same bits
    again = cfm.tc_conv3x3_wgrad(cfm.to_bf16_bits(x), cfm.to_bf16_bits(dz)).astype(np.float64)
    np.testing.assert_array_equal(again, got)
