"""The TMA-fed 3D sweep under concurrent device-memory traffic.

Each consumer warp of j3d_tma_kernel reads a ring slot of shared memory and
then releases it to the producer, whose next tensor load refills the slot.
Without a proxy fence between those reads and the release, runs made while
other streams copied device memory gave wrong cells (values of the plane
STAGES further on) from the second sweep on, in about a third of the runs.
Here two host threads keep 1 GiB device-to-device copies going on their own
streams while the grid is swept; every run must equal the quiet run bit for
bit, for one sweep per pass and for two (temporal blocking)."""
import os
import threading

import numpy as np
import pytest
import torch

import cfm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant,niter", [(None, 2), (None, 3), ("12", 2)])
def test_tma_sweeps_equal_under_copy_traffic(variant, niter, monkeypatch):
    if variant is not None:
        monkeypatch.setenv("CFM_J3D_TMA_VARIANT", variant)
    N = 512
    h = cfm.Jacobi(3, N, N, N, cfm.FP64, 1, cfm.JACOBI_PERSISTENT)
    try:
        a = h.problem_host(cfm.PROBLEM_CONFIG)
        h.upload(a)
        h.run(niter)
        quiet = h.download().copy()

        n = 1 << 27  # 1 GiB of FP64 per tensor
        src = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
        dst = [torch.empty_like(t) for t in src]
        streams = [torch.cuda.Stream() for _ in range(2)]
        stop = threading.Event()

        def traffic(k):
            while not stop.is_set():
                with torch.cuda.stream(streams[k]):
                    dst[k].copy_(src[k], non_blocking=True)
                streams[k].synchronize()

        threads = [threading.Thread(target=traffic, args=(k,)) for k in range(2)]
        for t in threads:
            t.start()
        wrong = []
        try:
            for rep in range(24):
                h.upload(a)
                h.run(niter)
                got = h.download()
                if not np.array_equal(got, quiet):
                    wrong.append((rep, int(np.count_nonzero(got != quiet))))
        finally:
            stop.set()
            for t in threads:
                t.join()
        assert not wrong, f"runs differing from the quiet run (rep, cells): {wrong}"
    finally:
        h.close()
