"""GPU parity of the h-binned tensor-core form (SPH and Wendland groups with
per-particle radii), against the FP64 oracle.

The reference evaluates Phi^(|k| h_j) per term (fourier_transform.cu:111-118;
fourier_transform_cpu.cpp:107-118).  The tensor form bins particles by h and
replaces Phi^(|k| h) within a bin by its Chebyshev interpolant in h, so each
Chebyshev order is a separable sum on the tensor cores and the per-|k|
coefficients are applied in the dump; the sum must still match FP64 within
1e-5 rel-L2 (spectra) and 1e-4 (images).  Cases cover every tile kind the
columns (order x planes) can land on, the Nyquist plane as transposed jobs,
B operands computed per tile and copied from images, groups sharing an
accumulator with a decaying-Gaussian group, and the automatic form choice.
"""
import numpy as np
import pytest

import oracle as O
from libmeshlessvis_b200 import meshless as M
from libmeshlessvis_b200.workloads import constraints, knn_radius, plummer_positions, rotating_views

from util import spectrum_and_views

pytestmark = pytest.mark.gpu

SPEC_TOL = 1e-5
IMAGE_TOL = 1e-4


def _group(rng, n, basis, lo=0.01, hi=0.05, plummer=False):
    pos = plummer_positions(rng, n) if plummer else rng.random((n, 3), dtype=np.float32)
    w = rng.standard_normal(n).astype(np.float32)
    h = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.float32)
    return (constraints(pos, w), h, basis)


@pytest.mark.parametrize("basis", [M.WENDLAND_D3_C2, M.SPH])
@pytest.mark.parametrize("grid", [(32, 32, 32), (64, 64, 48), (64, 64, 64), (48, 64, 80), (128, 128, 32)])
def test_binned_tensor_form_matches_fp64(basis, grid):
    rng = np.random.default_rng(81)
    groups = [_group(rng, 6007, basis)]
    views = rotating_views(3)
    spec, imgs = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), views, M.FORM_TENSOR)
    ref = O.spectrum_grid(groups, 1.0, grid)
    assert O.rel_l2(spec, ref) < SPEC_TOL
    assert O.rel_l2(spec[:, :, -1], ref[:, :, -1]) < SPEC_TOL  # Nyquist plane
    ref_imgs = O.render_from_spectrum(ref, grid, 1.0, (1.0, 1.0), (16, 16), views, (32, 32))
    assert O.rel_l2(imgs, ref_imgs) < IMAGE_TOL


def test_binned_tensor_form_wide_h_range_and_operand_images():
    """A Plummer set with 32-NN radii (about a 50x range of h, as the SPH-like
    configuration) on 64^3, with B operands copied from images and computed
    per tile: both match FP64 and each other."""
    rng = np.random.default_rng(83)
    n = 20000
    pos = plummer_positions(rng, n)
    h = knn_radius(pos, 32)
    w = (4.0 / 3.0 * np.pi * h.astype(np.float64) ** 3 / 32.0).astype(np.float32)
    groups = [(constraints(pos, w), h, M.WENDLAND_D3_C2)]
    grid = (64, 64, 64)
    lib = M.lib()
    try:
        lib.vis_set_operand_cache_limit(0)
        spec_tile, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
        lib.vis_set_operand_cache_limit(-1)
        spec_img, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
    finally:
        lib.vis_set_operand_cache_limit(-1)
    ref = O.spectrum_grid(groups, 1.0, grid)
    assert O.rel_l2(spec_img, ref) < SPEC_TOL
    assert O.rel_l2(spec_tile, ref) < SPEC_TOL
    assert O.rel_l2(spec_img, spec_tile) < 1e-6


def test_binned_and_gaussian_groups_share_one_spectrum():
    """A Wendland group with radii (h-binned), a decaying-Gaussian group with
    radii and an SPH group with one radius, summed into one spectrum by one
    persistent launch; the binned and Gaussian jobs share an accumulator."""
    rng = np.random.default_rng(85)
    g1 = _group(rng, 3000, M.WENDLAND_D3_C2)
    g2 = _group(rng, 2500, M.GAUSSIAN_DECAYING)
    pos = rng.random((1500, 3), dtype=np.float32)
    g3 = (constraints(pos, rng.standard_normal(1500).astype(np.float32)), np.full(1500, 0.03, np.float32), M.SPH)
    groups = [g1, g2, g3]
    grid = (64, 64, 64)
    spec, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
    ref = O.spectrum_grid(groups, 1.0, grid)
    assert O.rel_l2(spec, ref) < SPEC_TOL


def test_automatic_form_takes_binned_groups_to_the_tensor_cores():
    """FORM_AUTO sends an h-binned group to the tensor kernel (launch counted
    by the tensor stage timer) and matches FP64."""
    rng = np.random.default_rng(87)
    groups = [_group(rng, 8000, M.WENDLAND_D3_C2)]
    cfg = M.Config(cutoff=(16, 16), samples=(32, 32), block_length=64)
    from util import to_dataset

    ds = to_dataset(groups)
    cfg.register(ds)
    sp = M.Spectrum((64, 64, 64), 1.0)
    try:
        cfg.enable_timing(True)
        cfg.kernel_time(M.STAGE_TENSOR_SUM)
        sp.compute(cfg, ds, M.FORM_AUTO)
        spec = sp.to_host(cfg)
        _, launches = cfg.kernel_time(M.STAGE_TENSOR_SUM)
        cfg.enable_timing(False)
    finally:
        sp.close()
        cfg.unregister(ds)
        cfg.close()
    assert launches >= 1
    ref = O.spectrum_grid(groups, 1.0, (64, 64, 64))
    assert O.rel_l2(spec, ref) < SPEC_TOL


def test_binned_and_gaussian_spectra_are_bitwise_reproducible():
    """Repeated computes of the same registered data give the same bits: the
    h-binned group's particles go into their bins in ascending radius (a
    stable sort, not an atomic scatter) and every item's totals are reduced
    in a fixed order."""
    rng = np.random.default_rng(7)
    groups = [_group(rng, 20011, M.WENDLAND_D3_C2, plummer=True),
              (constraints(rng.random((9001, 3), dtype=np.float32), rng.random(9001, dtype=np.float32)),
               np.exp(rng.uniform(np.log(0.01), np.log(0.05), 9001)).astype(np.float32), M.GAUSSIAN_DECAYING)]
    cfg = M.Config(step=(1.0, 1.0), cutoff=(32, 32), samples=(64, 64), block_length=64)
    ds = M.Dataset(groups)
    cfg.register(ds)
    sp = M.Spectrum((64, 64, 64), 1.0)
    try:
        sp.compute(cfg, ds, M.FORM_TENSOR)
        first = sp.to_host(cfg).copy()
        for _ in range(2):
            sp.compute(cfg, ds, M.FORM_TENSOR)
            assert np.array_equal(sp.to_host(cfg).view(np.uint32), first.view(np.uint32))
        ref = O.spectrum_grid(groups, 1.0, (64, 64, 64))
        assert O.rel_l2(first, ref) < SPEC_TOL
    finally:
        sp.close()
        cfg.unregister(ds)
        cfg.close()
