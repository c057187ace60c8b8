"""GPU test of the autotuner (vis_autotune_spectrum): it times launch
parameter candidates on the caller's data, keeps the fastest set for the
spectrum's shape, and later computes of that shape use it -- with results
still within the parity tolerance against the FP64 oracle.  Every tile-shape
set it may try (vis_autotune_store) matches the plain form and FP64."""
import ctypes

import numpy as np
import pytest

import oracle as O
from libmeshlessvis_b200 import _lib as L
from libmeshlessvis_b200 import meshless as M
from libmeshlessvis_b200.workloads import constraints

from util import spectrum_and_views, to_dataset

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
    shapes = [ctypes.c_int(), ctypes.c_int()]
    assert lib.vis_autotune_lookup_shapes(L.int3(*grid), n, 2, M.FORM_AUTO, *[ctypes.byref(v) for v in shapes]) == 1
    assert 0 <= shapes[0].value <= L.TILE_ALL and shapes[1].value in (256, 1024, 4096)
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


_ALL = L.TILE_ALL


@pytest.mark.parametrize("shapes", [_ALL, _ALL & ~L.TILE_ROW_FOLD, _ALL & ~L.TILE_AXIS_EXCHANGE,
                                    _ALL & ~L.TILE_DOUBLE_BUFFER, _ALL & ~L.TILE_CTA_PAIRS, 0])
def test_every_tile_shape_set_matches_the_plain_form_and_fp64(shapes):
    """The tile-shape sets the autotuner tries (each VIS_TILE_* shape turned
    off, and all of them), recorded for the shape by vis_autotune_store, on a
    32x128x192 lattice that uses every shape by default: a pure-phase SPH
    group (row fold 4: 96 planes x 4 fill three 128-c n-tiles), a decaying
    Gaussian with radii (axis exchange: 128 b columns instead of 96 planes), a
    Wendland group with per-particle radii (h-bins, row-folded), 2000
    particles each (items of at most 8 chains: double-buffered CTA pairs),
    4096 rows (CTA pairs).  Against the plain form over the whole spectrum
    and the FP64 oracle at 600 points."""
    rng = np.random.default_rng(57)
    n = 2000
    pos = rng.random((3, n, 3), dtype=np.float32)
    w = rng.standard_normal((3, n)).astype(np.float32)
    h = np.exp(rng.uniform(np.log(0.01), np.log(0.05), (2, n))).astype(np.float32)
    groups = [(constraints(pos[0] * 0.05, w[0]), None, M.SPH),
              (constraints(pos[1], w[1]), h[0], M.GAUSSIAN_DECAYING),
              (constraints(pos[2], w[2]), h[1], M.WENDLAND_D3_C2)]
    grid = (32, 128, 192)
    lib = M.lib()
    lib.vis_autotune_clear()
    try:
        assert lib.vis_autotune_store(L.int3(*grid), 3 * n, 3, M.FORM_TENSOR, 6, 4, 16, shapes, 1024) == 0
        spec_tc, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
    finally:
        lib.vis_autotune_clear()
    spec_pl, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_PLAIN)
    assert O.rel_l2(spec_tc, spec_pl) < SPEC_TOL
    kx, ky, kz = grid
    ijk = np.stack([rng.integers(-kx // 2, kx // 2, 600), rng.integers(-ky // 2, ky // 2, 600),
                    rng.integers(0, kz // 2 + 1, 600)], 1)
    ref = sum(O.spectrum_points(g[0], g[1], g[2], 1.0, ijk) for g in groups)
    got = spec_tc[ijk[:, 0] + kx // 2, ijk[:, 1] + ky // 2, ijk[:, 2]]
    assert O.rel_l2(got, ref) < SPEC_TOL
