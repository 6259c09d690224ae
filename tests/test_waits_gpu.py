"""GPU: the bounded device waits give up, report, and leave the context usable.

Every spin of the kernels here (the batched ALS kernel's work-queue
dependencies, the mbarrier waits for bulk copies) has a bound, after which the
kernel sets an error bit that the host turns into PTIERR_CUDA_ERROR.  These
tests make such waits run out on purpose, without a fault or a hang: a queue
whose one task depends on a task that is not in it, and an mbarrier armed for
bytes that no copy sends.
"""
import time

import numpy as np
import pytest

from hiparti_b200 import ffi, synth

pytestmark = pytest.mark.gpu
PTIERR_CUDA_ERROR = 0x20000


def test_mbarrier_wait_gives_up(lib, cuda):
    gave_up, completed = ffi.new("int *", -1), ffi.new("int *", -1)
    assert lib.ptiB200MbarrierWaitProbe(1 << 16, gave_up, completed) == 0
    assert gave_up[0] == 1      # the withheld bytes never arrive: the bounded wait returns
    assert completed[0] == 1    # a barrier whose phase completes is still seen complete


def test_batched_queue_wait_gives_up_and_the_batch_still_runs(lib, cuda, orc):
    import torch
    from hiparti_b200.batched import Batch, stride_for
    dims = [(60, 50, 40), (30, 20, 10)]
    tensors = []
    for k, d in enumerate(dims):
        inds, vals = synth.uniform_tensor(d, 1500, seed=40 + k)
        tensors.append((d, inds, vals))
    ranks = [8, 4]
    bt = Batch(tensors, ranks, tune=False)
    lib.ptiClearLastError()
    t0 = time.perf_counter()
    rc = lib.ptiB200BatchWaitProbe(bt._h, 0.05)
    took = time.perf_counter() - t0
    assert rc == PTIERR_CUDA_ERROR
    assert took < 5.0  # gave up after its 50 ms bound, not after the 2 s default
    # the same handle runs a normal ALS iteration afterwards
    inits = [[np.abs(np.random.default_rng(50 + m).standard_normal((d, r))).astype(np.float32) for m, d in
              enumerate(t[0])] for t, r in zip(tensors, ranks)]
    facs = []
    for fs, r in zip(inits, ranks):
        row = []
        for a in fs:
            x = torch.zeros((a.shape[0], stride_for(r)), dtype=torch.float32)
            x[:, :r] = torch.from_numpy(a)
            row.append(x.cuda())
        facs.append(row)
    _, fits, _ = bt.cpd_als(facs, 2, precision="fp32", fp32_sweeps=0)
    for b, (t, r) in enumerate(zip(tensors, ranks)):
        o = orc.cpd_als(list(t[0]), t[1], t[2], r, 2, inits[b])
        assert abs(fits[b][-1] - o["fit"]) < 1e-4
    bt.free()


def test_probe_rejects_unbounded_waits(lib, cuda):
    from hiparti_b200.batched import Batch
    inds, vals = synth.uniform_tensor((20, 20, 20), 300, seed=3)
    bt = Batch([((20, 20, 20), inds, vals)], [4], tune=False)
    assert lib.ptiB200BatchWaitProbe(bt._h, 10.0) == 3  # PTIERR_VALUE_ERROR: bound above 2 s
    bt.free()
