"""GPU parity at the benchmark configurations' full sizes (the shapes the bench
measures), against the FP64 oracle (the reference's per-term sum restated in
FP64, meshless_vis/fourier_transform_cpu.cpp:73-134, on the 3D half-spectrum):

  C2  N=262,144 Plummer particles with 32-NN weights and radii, Wendland,
      128^3 lattice, the plain form, the h-binned tensor form and the
      automatic choice; 1024 points.
  C3  N=2^20 uniform particles, decaying Gaussian with log-uniform h in 16
      h-bins, 256^3 lattice (CTA-pair tensor tiles, B-operand images, the
      Nyquist plane as tensor jobs, 16-stage accumulation chains); the
      workload's own 4096 check points.
  C5  one frame's shapes at N=2^20: Plummer particles, 8 h-bins of the
      decaying Gaussian, 384^3 lattice (CTA pairs with n-tiles of 96 + 96 c
      values); 1024 points; 4 of its 360 views against FP64 slicing of the
      same spectrum.
  C4  four of the 64 batch sets at their real sizes (the largest, the
      smallest and two in between) as one batch with all their views.

Tolerances: 1e-5 rel-L2 for spectra, 1e-4 for images.
"""
import numpy as np
import pytest

import oracle as O
from libmeshlessvis_b200 import meshless as M
from libmeshlessvis_b200 import workloads as W

from util import spectrum_and_views, to_dataset

pytestmark = pytest.mark.gpu

SPEC_TOL = 1e-5
IMAGE_TOL = 1e-4


def _points(grid, count, seed):
    kx, ky, kz = grid
    prng = np.random.default_rng(seed)
    return np.stack([prng.integers(-kx // 2, kx // 2, count), prng.integers(-ky // 2, ky // 2, count),
                     prng.integers(0, kz // 2 + 1, count)], 1).astype(np.int32)


def _at(spec, grid, ijk):
    kx, ky, _ = grid
    return spec[ijk[:, 0] + kx // 2, ijk[:, 1] + ky // 2, ijk[:, 2]]


def _fp64(groups, step3, ijk):
    return sum(O.spectrum_points(c, r, b, step3, ijk) for c, r, b in groups)


@pytest.mark.parametrize("form", [M.FORM_PLAIN, M.FORM_AUTO, M.FORM_TENSOR])
def test_c2_full_size(form):
    w = W.c2()
    spec, _ = spectrum_and_views(w["groups"], w["grid"], w["step3"], w["step"], w["cutoff"], w["samples"], None,
                                 form)
    ijk = _points(w["grid"], 1024, 1)
    assert O.rel_l2(_at(spec, w["grid"], ijk), _fp64(w["groups"], w["step3"], ijk)) < SPEC_TOL


def test_c3_full_size_tensor_form():
    w = W.c3()
    spec, _ = spectrum_and_views(w["groups"], w["grid"], w["step3"], w["step"], w["cutoff"], w["samples"], None,
                                 M.FORM_TENSOR)
    ijk = w["check_points"]
    ref = _fp64(w["groups"], w["step3"], ijk)
    got = _at(spec, w["grid"], ijk)
    assert O.rel_l2(got, ref) < SPEC_TOL
    # the Nyquist plane (two transposed tensor jobs) on its own
    nyq = _points(w["grid"], 512, 7)
    nyq[:, 2] = w["grid"][2] // 2
    assert O.rel_l2(_at(spec, w["grid"], nyq), _fp64(w["groups"], w["step3"], nyq)) < SPEC_TOL


def test_c5_lattice_and_tiles_at_2e20_particles():
    w = next(W.c5_frames(n=1 << 20, frames=1))
    views = w["views"][::90]
    spec, imgs = spectrum_and_views(w["groups"], w["grid"], w["step3"], w["step"], w["cutoff"], w["samples"], views,
                                    M.FORM_TENSOR)
    ijk = _points(w["grid"], 1024, 2)
    assert O.rel_l2(_at(spec, w["grid"], ijk), _fp64(w["groups"], w["step3"], ijk)) < SPEC_TOL
    ref_imgs = O.render_from_spectrum(spec.astype(np.complex128), w["grid"], w["step3"], w["step"], w["cutoff"],
                                      views, w["samples"])
    assert O.rel_l2(imgs, ref_imgs) < IMAGE_TOL


def test_c4_sets_at_real_sizes_as_one_batch():
    sets = W.c4()
    sizes = [sum(len(c) for c, _, _ in w["groups"]) for w in sets]
    order = np.argsort(sizes)
    picks = [int(order[-1]), int(order[0]), int(order[len(order) // 2]), int(order[3 * len(order) // 4])]
    cfg = M.Config(block_length=64)
    batch = M.Batch(cfg)
    datasets = []
    try:
        for j in picks:
            w = sets[j]
            ds = to_dataset(w["groups"])
            cfg.register(ds)
            datasets.append(ds)
            batch.add(ds, w["grid"], w["step3"], w["step"], w["cutoff"], w["samples"], [v[0] for v in w["views"]],
                      [v[1] for v in w["views"]])
        batch.execute(M.FORM_AUTO)
        batch.execute(M.FORM_AUTO)  # the replayed graph
        for b, j in enumerate(picks):
            w = sets[j]
            spec = batch.spectrum(b)
            ijk = _points(w["grid"], 512, 10 + b)
            assert O.rel_l2(_at(spec, w["grid"], ijk), _fp64(w["groups"], w["step3"], ijk)) < SPEC_TOL
            imgs = batch.images(b)
            views = w["views"][:4]
            ref_imgs = O.render_from_spectrum(spec.astype(np.complex128), w["grid"], w["step3"], w["step"],
                                              w["cutoff"], views, w["samples"])
            assert O.rel_l2(imgs[:4], ref_imgs) < IMAGE_TOL
    finally:
        batch.close()
        for ds in datasets:
            cfg.unregister(ds)
        cfg.close()
