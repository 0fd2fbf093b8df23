"""The NumPy U-Net oracle (oracle/unet_oracle.py) is itself right: its
backward pass matches central finite differences in float64, and its
parameter count is the library's."""
import numpy as np

import cfm
import unet_oracle as U


def test_param_count_matches_library():
    assert U.num_params() == cfm.lib.cfm_unet_num_params()


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    n = U.num_params()
    theta = rng.normal(size=n) * 0.1
    x = rng.normal(size=(2, 16, 16, 2))
    dout = rng.normal(size=(2, 16, 16))
    out, cache = U.forward(theta, x, round_bf16=False)
    g = U.backward(cache, dout)
    # one entry of every layer's weight and bias, plus random ones
    idx, o = [], 0
    for _, ci, co in U.LAYERS:
        idx += [o + 5, o + 9 * ci * co]
        o += 9 * ci * co + co
    idx += list(rng.choice(n, 8, replace=False))
    for i in idx:
        e = np.zeros(n)
        e[i] = 1e-6
        fd = ((U.forward(theta + e, x, False)[0] - U.forward(theta - e, x, False)[0]) * dout).sum() / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])
