"""The single-system FPCG device loop (the iterations between network
applications in one persistent cooperative launch) against one kernel per
phase: the same iterations and the same x bit for bit, in FP64 and in mixed
precision, with Jacobi smoothing alone and with a network."""
import numpy as np
import pytest

import cfm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("with_net", [False, True])
def test_device_loop_matches_kernels(precision, with_net):
    k, f = cfm.varcoef_problem((256, 256), 3)
    S = cfm.Stencil(k)
    net = None
    if with_net:
        net = cfm.UNet(256, 256, max_batch=1, seed=5)
        net.set_training_info(2, 1)
    prec = cfm.FP64 if precision == "fp64" else cfm.FP32
    out = []
    for loop in (0, 1):
        fp = cfm.FPCG(S, k, net, maxiter=3000, tol=1e-8, smooth=2, precision=prec)
        fp.set_device_loop(loop)
        for _ in range(2):  # the second solve replays the captured graph
            x, st = fp.solve(f)
        out.append((x, st.iterations, st.refinements))
        fp.close()
    if net is not None:
        net.close()
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]
    np.testing.assert_array_equal(out[0][0], out[1][0])
