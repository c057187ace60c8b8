"""GPU test of the autotuner (vis_autotune_spectrum): it times launch
parameter candidates on the caller's data, keeps the fastest set for the
spectrum's shape, and later computes of that shape use it -- with results
still within the parity tolerance against the FP64 oracle."""
import ctypes

import numpy as np
import pytest

import oracle as O
from libmeshlessvis_b200 import _lib as L
from libmeshlessvis_b200 import meshless as M
from libmeshlessvis_b200.workloads import constraints

from util import to_dataset

pytestmark = pytest.mark.gpu

SPEC_TOL = 1e-5


def test_autotune_records_a_candidate_set_and_keeps_results_exact():
    rng = np.random.default_rng(51)
    n = 3000
    pos = rng.random((n, 3), dtype=np.float32)
    w = rng.standard_normal(n).astype(np.float32)
    h = np.exp(rng.uniform(np.log(0.01), np.log(0.05), n)).astype(np.float32)
    # one tensor-form group (decaying Gaussian) and one plain-form group (SPH, per-particle h)
    groups = [(constraints(pos[: n // 2], w[: n // 2]), h[: n // 2], M.GAUSSIAN_DECAYING),
              (constraints(pos[n // 2:], w[n // 2:]), h[n // 2:], M.SPH)]
    grid = (32, 32, 64)
    lib = M.lib()
    lib.vis_autotune_clear()
    cfg = M.Config(cutoff=(16, 16), samples=(32, 32), block_length=64)
    ds = to_dataset(groups)
    cfg.register(ds)
    sp = M.Spectrum(grid, 1.0)
    best = sp.autotune(cfg, ds, M.FORM_AUTO)
    assert best > 0.0
    vals = [ctypes.c_int(), ctypes.c_int(), ctypes.c_int()]
    tuned = lib.vis_autotune_lookup(L.int3(*grid), n, 2, M.FORM_AUTO, *[ctypes.byref(v) for v in vals])
    assert tuned == 1
    plain_waves, tc_waves, flush = (v.value for v in vals)
    assert plain_waves in (2, 4, 6, 8) and tc_waves in (2, 4, 8) and flush in (8, 16)
    # a compute of the same shape now runs with the tuned parameters
    sp.compute(cfg, ds, M.FORM_AUTO)
    spec = sp.to_host(cfg)
    ref = O.spectrum_grid(groups, 1.0, grid)
    assert O.rel_l2(spec, ref) < SPEC_TOL
    sp.close()
    cfg.unregister(ds)
    cfg.close()
    lib.vis_autotune_clear()
    assert lib.vis_autotune_lookup(L.int3(*grid), n, 2, M.FORM_AUTO, None, None, None) == 0
