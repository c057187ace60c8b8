"""The tensor-core kernel's bounded waits, made to run out on purpose (GPU).

Every mbarrier wait of tc_sum_kernel is bounded; a wait that runs out sets a
device error word, the CTAs leave their loops, wait for their bulk copies,
release tensor memory and return, and the next synchronising call reports
VIS_ERROR_CUDA.  vis_tensor_wait_test_hook makes the next tensor launch bound
its waits by 1 ms and withhold one arrival on its first pipeline stage, so the
MMA thread's first wait runs out before any MMA is issued (error code 2).
Nothing faults, traps or hangs: the test then checks that the next compute on
the same device and config matches the FP64 oracle.  Both the one-CTA tile
(64x64x48: 24 tensor planes) and the CTA-pair tile (32^3: 16 planes, pairs of
256 rows) are covered.
"""
import re

import numpy as np
import pytest

import oracle as O
from libmeshlessvis_b200 import meshless as M
from libmeshlessvis_b200.workloads import constraints

from util import to_dataset

pytestmark = pytest.mark.gpu

VIS_ERROR_CUDA = 3
CODE_MMA_FULL_WAIT = 2  # the MMA thread's wait for a filled stage


@pytest.mark.parametrize("grid", [(64, 64, 48), (32, 32, 32)])
def test_a_wait_that_runs_out_is_reported_and_the_device_stays_usable(grid):
    lib = M.lib()
    rng = np.random.default_rng(71)
    n = 3000
    pos = rng.random((n, 3), dtype=np.float32)
    w = rng.standard_normal(n).astype(np.float32)
    h = np.exp(rng.uniform(np.log(0.01), np.log(0.05), n)).astype(np.float32)
    groups = [(constraints(pos, w), h, M.GAUSSIAN_DECAYING)]
    cfg = M.Config(cutoff=(16, 16), samples=(32, 32), block_length=64)
    ds = to_dataset(groups)
    cfg.register(ds)
    sp = M.Spectrum(grid, 1.0)
    try:
        assert lib.vis_tensor_wait_test_hook(10) == 1  # below the accepted range
        lib.vis_clear_last_error()
        assert lib.vis_tensor_wait_test_hook(1_000_000) == 0
        sp.compute(cfg, ds, M.FORM_TENSOR)
        rc = lib.vis_config_synchronize(cfg.ptr)
        assert rc == VIS_ERROR_CUDA
        msg = lib.vis_get_last_error_message().decode()
        assert "timed out in a bounded wait" in msg, msg
        code = int(re.search(r"code (\d+)", msg).group(1))
        assert code & CODE_MMA_FULL_WAIT, msg
        lib.vis_clear_last_error()
        # the word was cleared when reported; the hook was one shot
        assert lib.vis_config_synchronize(cfg.ptr) == 0
        sp.compute(cfg, ds, M.FORM_TENSOR)
        spec = sp.to_host(cfg)
        ref = O.spectrum_grid(groups, 1.0, grid)
        assert O.rel_l2(spec, ref) < 1e-5
    finally:
        sp.close()
        cfg.unregister(ds)
        cfg.close()
