"""GPU parity: the CUDA path, called through the C ABI, against the golden
vectors of the reference's own CPU renderer and against the FP64 oracle.

Tolerances (relative L2 over the whole output):
  spectra and direct slices vs FP64 ..... 1e-5
  images cut from the 3D spectrum ....... 1e-4
  anything vs the reference's FP32 CPU .. 5e-5 (the reference itself is up to
                                           2.8e-5 off FP64 for Wendland)
"""
import numpy as np
import pytest

import oracle as O
from libmeshlessvis_b200 import meshless as M
from libmeshlessvis_b200.workloads import c1, constraints, plummer_positions, knn_radius, rotating_views

from util import render_direct, spectrum_and_views, to_dataset

pytestmark = pytest.mark.gpu

SPEC_TOL = 1e-5
IMAGE_TOL = 1e-4
REF_TOL = 5e-5

DIRECT = ["b0_xy", "b0_rot", "b0_noradii", "b1_xy", "b1_rot", "b1_noradii", "b2_xy", "b2_rot", "b2_noradii",
          "two_groups_step01", "timing_test_radii", "timing_test_factor1", "single_particle"]
SPECTRA = ["spec_b0", "spec_b1", "spec_b2", "spec_b3", "spec_noradii_step05"]


@pytest.mark.parametrize("name", DIRECT)
def test_direct_render_matches_reference_and_fp64(golden, name):
    c = golden[name]
    img = render_direct(c["groups"], c["step"], c["cutoff"], c["u"], c["v"], c["samples"])
    assert O.rel_l2(img, c["fp64_image"]) < SPEC_TOL
    assert O.rel_l2(img, c["ref_image"]) < REF_TOL


@pytest.mark.parametrize("name", SPECTRA)
@pytest.mark.parametrize("form", [M.FORM_PLAIN, M.FORM_AUTO])
def test_spectrum_and_views_match_fp64(golden, name, form):
    c = golden[name]
    spec, imgs = spectrum_and_views(c["groups"], c["grid"], float(c["step3"]), c["step"], c["cutoff"], c["samples"],
                                    [tuple(map(tuple, v)) for v in c["views"]], form)
    assert O.rel_l2(spec, c["fp64_spectrum"]) < SPEC_TOL
    assert O.rel_l2(imgs, c["fp64_images"]) < IMAGE_TOL


def test_c1_full_spectrum_view_and_kat5():
    """Config C1 in full (N=4096, 64x64x33 half-spectrum, one z-normal view):
    spectrum vs FP64; the view cut from the spectrum equals the direct render
    (KAT-5: the z-normal slice lands on lattice points)."""
    w = c1()
    spec, imgs = spectrum_and_views(w["groups"], w["grid"], w["step3"], w["step"], w["cutoff"], w["samples"],
                                    w["views"], M.FORM_PLAIN)
    ref = O.spectrum_grid(w["groups"], w["step3"], w["grid"])
    assert O.rel_l2(spec, ref) < SPEC_TOL
    u, v = w["views"][0]
    direct = render_direct(w["groups"], w["step"], w["cutoff"], u, v, w["samples"])
    fp64 = O.render_direct(w["groups"], w["step"], w["cutoff"], u, v, w["samples"])
    assert O.rel_l2(direct, fp64) < SPEC_TOL
    assert O.rel_l2(imgs[0], fp64) < SPEC_TOL
    assert O.rel_l2(imgs[0], direct) < SPEC_TOL


def test_c2_shape_wendland_per_particle_h_on_random_points():
    """C2's particle set (Plummer, 32-NN h and weights, Wendland) at N=65,536
    on the 128^3 half-spectrum; FP64 check on 1024 random lattice points."""
    rng = np.random.default_rng(0)
    n = 65536
    pos = plummer_positions(rng, n)
    r32 = knn_radius(pos, 32)
    wgt = (4.0 / 3.0 * np.pi * r32.astype(np.float64) ** 3 / 32.0).astype(np.float32)  # m / rho, m = 1/N
    groups = [(constraints(pos, wgt), r32, M.WENDLAND_D3_C2)]
    spec, _ = spectrum_and_views(groups, (128, 128, 128), 1.0, (1.0, 1.0), (64, 64), (128, 128), None, M.FORM_PLAIN)
    prng = np.random.default_rng(1)
    ijk = np.stack([prng.integers(-64, 64, 1024), prng.integers(-64, 64, 1024), prng.integers(0, 65, 1024)], 1)
    ref = O.spectrum_points(groups[0][0], r32, M.WENDLAND_D3_C2, 1.0, ijk)
    got = spec[ijk[:, 0] + 64, ijk[:, 1] + 64, ijk[:, 2]]
    assert O.rel_l2(got, ref) < SPEC_TOL


def test_decaying_gaussian_many_groups_large_n_random_points():
    """16 groups (h-bins) of a log-uniform-h decaying Gaussian set, N=2^18,
    64^3 lattice; FP64 check on 2048 random points."""
    rng = np.random.default_rng(2)
    n = 1 << 18
    pos = rng.random((n, 3), dtype=np.float32)
    w = rng.random(n, dtype=np.float32)
    h = np.exp(rng.uniform(np.log(0.005), np.log(0.05), n)).astype(np.float32)
    edges = np.exp(np.linspace(np.log(0.005), np.log(0.05), 17))
    b = np.clip(np.searchsorted(edges, h, side="right") - 1, 0, 15)
    groups = [(constraints(pos[b == k], w[b == k]), h[b == k], M.GAUSSIAN_DECAYING) for k in range(16)]
    spec, _ = spectrum_and_views(groups, (64, 64, 64), 1.0, (1.0, 1.0), (32, 32), (64, 64), None, M.FORM_PLAIN)
    prng = np.random.default_rng(3)
    ijk = np.stack([prng.integers(-32, 32, 2048), prng.integers(-32, 32, 2048), prng.integers(0, 33, 2048)], 1)
    ref = sum(O.spectrum_points(g[0], g[1], g[2], 1.0, ijk) for g in groups)
    got = spec[ijk[:, 0] + 32, ijk[:, 1] + 32, ijk[:, 2]]
    assert O.rel_l2(got, ref) < SPEC_TOL


@pytest.mark.parametrize("grid,basis", [((32, 32, 32), M.WENDLAND_D3_C2), ((32, 32, 32), M.GAUSSIAN_DECAYING),
                                        ((48, 32, 16), M.SPH), ((32, 48, 24), M.GAUSSIAN_DECAYING),
                                        ((64, 64, 8), M.SPH)])
def test_plain_form_whole_spectra_on_square_and_oblong_lattices(grid, basis):
    """The plain (folded) form over whole half-spectra with per-particle radii
    (Phi^ table and Gaussian exp2 amplitudes), on lattices whose x and y
    extents agree and on oblong ones, against the FP64 sum at every point (the
    reference's per-term sum, meshless_vis/fourier_transform.cu:100-130)."""
    rng = np.random.default_rng(sum(grid) + basis)
    n = 3001
    h = np.exp(rng.uniform(np.log(0.01), np.log(0.06), n)).astype(np.float32)
    groups = [(constraints(rng.random((n, 3)), rng.standard_normal(n)), h, basis)]
    spec, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (grid[0] // 2, grid[1] // 2), grid[:2], None,
                                 M.FORM_PLAIN)
    ref = O.spectrum_grid(groups, 1.0, grid)
    assert O.rel_l2(spec, ref) < SPEC_TOL


def test_spectrum_l0_plane_is_hermitian():
    rng = np.random.default_rng(4)
    groups = [(constraints(rng.random((999, 3)), rng.standard_normal(999)), np.full(999, 0.03, np.float32), M.SPH)]
    spec, _ = spectrum_and_views(groups, (32, 32, 32), 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_PLAIN)
    p = spec[:, :, 0]
    # F(-i,-j,0) = conj F(i,j,0) for i, j in (-16, 16)
    a = p[1:, 1:]
    b = np.conj(p[1:, 1:][::-1, ::-1])
    assert O.rel_l2(a, b) < 1e-6


def test_rotated_views_match_fp64_interpolation():
    rng = np.random.default_rng(6)
    groups = [(constraints(rng.random((2000, 3)), rng.standard_normal(2000)),
               np.exp(rng.uniform(np.log(0.01), np.log(0.04), 2000)).astype(np.float32), M.WENDLAND_D3_C2)]
    views = rotating_views(12) + [((0.6, 0.8, 0.0), (0.0, 0.0, 1.0)), ((0.0, 0.0, -1.0), (0.0, 1.0, 0.0))]
    spec, imgs = spectrum_and_views(groups, (32, 32, 32), 1.0, (1.0, 1.0), (16, 16), (32, 32), views, M.FORM_PLAIN)
    ref_spec = O.spectrum_grid(groups, 1.0, (32, 32, 32))
    assert O.rel_l2(spec, ref_spec) < SPEC_TOL
    ref_imgs = O.render_from_spectrum(ref_spec, (32, 32, 32), 1.0, (1.0, 1.0), (16, 16), views, (32, 32))
    assert O.rel_l2(imgs, ref_imgs) < IMAGE_TOL


@pytest.mark.parametrize("n", [0, 1, 255, 257, 4097])
def test_ragged_and_empty_particle_counts(n):
    rng = np.random.default_rng(n)
    groups = [(constraints(rng.random((n, 3)), rng.standard_normal(n)), np.full(n, 0.05, np.float32), M.SPH)]
    img = render_direct(groups, (1.0, 1.0), (8, 8), (1, 0, 0), (0, 1, 0), (16, 16))
    ref = O.render_direct(groups, (1.0, 1.0), (8, 8), (1, 0, 0), (0, 1, 0), (16, 16))
    if n == 0:
        assert np.all(img == 0)
    else:
        assert O.rel_l2(img, ref) < SPEC_TOL
    spec, _ = spectrum_and_views(groups, (8, 8, 8), 1.0, (1.0, 1.0), (4, 4), (8, 8), None, M.FORM_PLAIN)
    ref_s = O.spectrum_grid(groups, 1.0, (8, 8, 8))
    if n == 0:
        assert np.all(spec == 0)
    else:
        assert O.rel_l2(spec, ref_s) < SPEC_TOL


def test_dataset_without_groups_renders_zero():
    img = render_direct([], (1.0, 1.0), (8, 8), (1, 0, 0), (0, 1, 0), (16, 16))
    assert np.all(img == 0)


@pytest.mark.parametrize("cutoff,samples,bl,ps", [((1, 32), (2, 64), 64, 1), ((32, 32), (64, 64), 512, 4),
                                                   ((24, 8), (48, 16), 128, 3)])
def test_config_edges_nyquist_and_partial_sums(cutoff, samples, bl, ps):
    """2cx == Nx (the u-Nyquist column is dropped), tiny cutoffs, several
    block lengths and partial-sum counts (they change only the padding)."""
    rng = np.random.default_rng(9)
    groups = [(constraints(rng.random((700, 3)), rng.standard_normal(700)),
               np.full(700, 0.02, np.float32), M.GAUSSIAN)]
    img = render_direct(groups, (1.0, 1.0), cutoff, (1, 0, 0), (0, 1, 0), samples, block_length=bl,
                        partial_sums=ps)
    ref = O.render_direct(groups, (1.0, 1.0), cutoff, (1, 0, 0), (0, 1, 0), samples)
    assert O.rel_l2(img, ref) < SPEC_TOL


def test_register_pads_like_the_reference():
    rng = np.random.default_rng(10)
    ds = to_dataset([(constraints(rng.random((300, 3)), rng.random(300)), None, M.SPH)])
    cfg = M.Config(cutoff=(8, 8), samples=(16, 16), block_length=128, partial_sums=3)
    cfg.register(ds)
    g = ds.group(0)
    assert g.d_number_of_terms == 384 and g.d_constraints and not g.d_radii
    cfg.unregister(ds)
    cfg.close()


def test_invalid_config_and_unregistered_dataset_report_errors():
    lib = M.lib()
    cfg = M.Config(cutoff=(40, 8), samples=(64, 16), block_length=64)  # 2*40*8 % 64 != 0
    assert not cfg.check()
    ds = to_dataset([(constraints(np.zeros((4, 3)), np.ones(4)), None, M.SPH)])
    lib.vis_fourier_volume_rendering(ds.ref, cfg.ptr)
    assert lib.vis_get_last_error() == 2
    lib.vis_clear_last_error()
    cfg.close()
    cfg = M.Config(cutoff=(8, 8), samples=(16, 16), block_length=64)
    lib.vis_fourier_volume_rendering(ds.ref, cfg.ptr)
    assert lib.vis_get_last_error() == 6
    lib.vis_clear_last_error()
    cfg.close()


def test_repeat_render_is_deterministic():
    rng = np.random.default_rng(12)
    groups = [(constraints(rng.random((5000, 3)), rng.standard_normal(5000)),
               np.full(5000, 0.02, np.float32), M.WENDLAND_D3_C2)]
    cfg = M.Config(cutoff=(16, 16), samples=(32, 32), block_length=64)
    ds = to_dataset(groups)
    cfg.register(ds)
    cfg.render(ds)
    a = cfg.image()
    cfg.render(ds)
    b = cfg.image()
    cfg.unregister(ds)
    cfg.close()
    np.testing.assert_array_equal(a, b)


def test_manual_d_image_stream_and_timing():
    """A caller-owned device image (the headless stand-in for the reference's
    GL pixel buffer) on a caller-owned stream, with per-stage timing."""
    import torch

    lib = M.lib()
    rng = np.random.default_rng(13)
    groups = [(constraints(rng.random((1000, 3)), rng.standard_normal(1000)), np.full(1000, 0.03, np.float32),
               M.SPH)]
    cfg = M.Config(cutoff=(8, 8), samples=(16, 16), block_length=64, automatic_d_image=False)
    buf = torch.zeros((16, 16), dtype=torch.float32, device="cuda")
    lib.vis_config_manual_d_image(cfg.ptr, buf.data_ptr())
    stream = torch.cuda.Stream()
    cfg.set_stream(stream.cuda_stream)
    ds = to_dataset(groups)
    cfg.register(ds)
    cfg.enable_timing(True)
    cfg.render(ds)
    cfg.synchronize()
    img = buf.cpu().numpy()
    ms, launches = cfg.kernel_time(M.STAGE_SUM)
    assert launches == 1 and ms > 0
    ms_fft, launches_fft = cfg.kernel_time(M.STAGE_FFT)
    assert launches_fft == 1
    cfg.unregister(ds)
    cfg.close()
    ref = O.render_direct(groups, (1.0, 1.0), (8, 8), (1, 0, 0), (0, 1, 0), (16, 16))
    assert O.rel_l2(img, ref) < SPEC_TOL


# ---------------------------------------------------------------- tensor form
def _tc_groups(rng, n):
    pos = rng.random((n, 3), dtype=np.float32)
    w = rng.standard_normal(n).astype(np.float32)
    h = np.exp(rng.uniform(np.log(0.01), np.log(0.06), n)).astype(np.float32)
    return {
        "gauss_decaying_radii": [(constraints(pos, w), h, M.GAUSSIAN_DECAYING)],
        "sph_no_radii": [(constraints(pos * 0.05, w), None, M.SPH)],
        "wendland_uniform_radius": [(constraints(pos, w), np.full(n, 0.03, np.float32), M.WENDLAND_D3_C2)],
        "two_groups": [(constraints(pos[: n // 2], w[: n // 2]), h[: n // 2], M.GAUSSIAN_DECAYING),
                       (constraints(pos[n // 2:], w[n // 2:]), np.full(n - n // 2, 0.02, np.float32), M.SPH)],
    }


@pytest.mark.parametrize("case", ["gauss_decaying_radii", "sph_no_radii", "wendland_uniform_radius", "two_groups"])
def test_tensor_form_matches_fp64(case):
    """Separable groups on a 32x32x17 half-spectrum through the tcgen05 path
    (FORM_TENSOR), including the Nyquist plane and ragged particle counts."""
    rng = np.random.default_rng(21)
    groups = _tc_groups(rng, 3001)[case]
    grid = (32, 32, 32)
    spec, imgs = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), rotating_views(3),
                                    M.FORM_TENSOR)
    ref = O.spectrum_grid(groups, 1.0, grid)
    assert O.rel_l2(spec, ref) < SPEC_TOL
    assert O.rel_l2(spec[:, :, -1], ref[:, :, -1]) < SPEC_TOL  # Nyquist plane (plain form)
    ref_imgs = O.render_from_spectrum(ref, grid, 1.0, (1.0, 1.0), (16, 16), rotating_views(3), (32, 32))
    assert O.rel_l2(imgs, ref_imgs) < IMAGE_TOL


@pytest.mark.parametrize("case", ["gauss_decaying_radii", "wendland_uniform_radius"])
@pytest.mark.parametrize("grid", [(32, 32, 272), (32, 32, 288), (32, 32, 16)])
def test_tensor_form_uneven_and_narrowest_n_tiles(case, grid):
    """32x32x272: the tensor planes c < 136 split into n-tiles of 72 and 64 c
    values (one CTA, MMA N = 144 and 128); 32x32x288: 144 planes, a multiple
    of 16, go to CTA pairs with n-tiles of 80 and 64 c values (40 and 32 per
    CTA); 32x32x16: one tile of 8 (N = 16, the smallest MMA width)."""
    rng = np.random.default_rng(23)
    groups = _tc_groups(rng, 2001)[case]
    spec, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
    ref = O.spectrum_grid(groups, 1.0, grid)
    assert O.rel_l2(spec, ref) < SPEC_TOL
    lz = grid[2] // 2
    assert O.rel_l2(spec[:, :, lz - 8:lz], ref[:, :, lz - 8:lz]) < SPEC_TOL  # the last tile's planes


@pytest.mark.parametrize("case", ["gauss_decaying_radii", "wendland_uniform_radius"])
@pytest.mark.parametrize("grid", [(128, 128, 16), (128, 128, 144), (256, 256, 160), (128, 128, 160),
                                  (64, 384, 160)])
def test_tensor_form_nyquist_plane(case, grid):
    """The Nyquist plane l = Kz/2 as two transposed tensor-core jobs (rows b,
    columns a >= 0; and by conjugate symmetry columns -a > 0 at -Kz/2 with b
    reversed): 128x128x16 with 128x128 tiles, 128x128x144 (72 planes, not a
    multiple of 16) with 128x256 tiles, 256x256x160 with CTA pairs.
    128x128x160 and 64x384x160 take CTA pairs, whose 256-row m-tiles their 128
    and 384 b rows fill partly: the rows past Ky are computed but not dumped.
    The whole plane against FP64 (both signs of a and b, a = -Kx/2 and b =
    -Ky/2 included), and the spectrum against the plain form."""
    rng = np.random.default_rng(29)
    groups = _tc_groups(rng, 1001)[case]
    kx, ky, kz = grid
    spec_tc, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
    spec_pl, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_PLAIN)
    a, b = np.meshgrid(np.arange(kx) - kx // 2, np.arange(ky) - ky // 2, indexing="ij")
    ijk = np.stack([a.ravel(), b.ravel(), np.full(a.size, kz // 2)], 1)
    ref = sum(O.spectrum_points(g[0], g[1], g[2], 1.0, ijk) for g in groups)
    assert O.rel_l2(spec_tc[:, :, kz // 2].ravel(), ref) < SPEC_TOL
    assert O.rel_l2(spec_tc, spec_pl) < SPEC_TOL


@pytest.mark.parametrize("grid", [(64, 64, 48), (64, 64, 64), (64, 64, 144), (256, 256, 160)])
def test_tensor_form_operand_images_match_per_tile_operands(grid):
    """B operands copied from images made once per compute (the default)
    against B operands computed per tile (vis_set_operand_cache_limit(0)), in
    128x128 tiles (24 planes), narrow CTA pairs (64^3: 32 planes), 128x256
    tiles (72 planes) and CTA pairs (256x256x160); a Gaussian and a factored
    group.  Both paths run the same arithmetic, and both match FP64."""
    rng = np.random.default_rng(31)
    groups = _tc_groups(rng, 2001)["two_groups"]
    lib = M.lib()
    try:
        lib.vis_set_operand_cache_limit(0)
        spec_tile, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
        lib.vis_set_operand_cache_limit(-1)
        spec_img, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
    finally:
        lib.vis_set_operand_cache_limit(-1)
    assert O.rel_l2(spec_img, spec_tile) < 1e-7
    kx, ky, kz = grid
    prng = np.random.default_rng(5)
    ijk = np.stack([prng.integers(-kx // 2, kx // 2, 2048), prng.integers(-ky // 2, ky // 2, 2048),
                    prng.integers(0, kz // 2 + 1, 2048)], 1)
    ref = sum(O.spectrum_points(g[0], g[1], g[2], 1.0, ijk) for g in groups)
    got = spec_img[ijk[:, 0] + kx // 2, ijk[:, 1] + ky // 2, ijk[:, 2]]
    assert O.rel_l2(got, ref) < SPEC_TOL


def test_tensor_form_operand_cache_limit_covers_some_jobs():
    """A limit that holds the first group's B-operand images but not the
    second's: one launch mixes image jobs and per-tile jobs (and the Nyquist
    jobs, which never use images).  Same spectrum as with the images off."""
    rng = np.random.default_rng(37)
    n = 1000
    groups = []
    for k in range(2):
        pos = rng.random((n, 3), dtype=np.float32)
        w = rng.standard_normal(n).astype(np.float32)
        h = np.exp(rng.uniform(np.log(0.01), np.log(0.05), n)).astype(np.float32)
        groups.append((constraints(pos, w), h, M.GAUSSIAN_DECAYING))
    grid = (64, 64, 64)
    # images of one group: 32 blocks x 1 n-tile x 32 c values x 512 B = 512 KiB
    lib = M.lib()
    try:
        lib.vis_set_operand_cache_limit(0)
        spec_tile, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
        lib.vis_set_operand_cache_limit(600 * 1024)
        spec_mix, _ = spectrum_and_views(groups, grid, 1.0, (1.0, 1.0), (16, 16), (32, 32), None, M.FORM_TENSOR)
    finally:
        lib.vis_set_operand_cache_limit(-1)
    assert O.rel_l2(spec_mix, spec_tile) < 1e-7
    ref = O.spectrum_grid(groups, 1.0, grid)
    assert O.rel_l2(spec_mix, ref) < SPEC_TOL


def test_tensor_form_long_accumulation_random_points():
    """N = 2^18 decaying-Gaussian particles in 16 h-bins on a 64^3 lattice
    (8192 particles ... per item, long TMEM accumulation with flushes);
    FP64 check on 2048 random points, and agreement with the plain form."""
    rng = np.random.default_rng(22)
    n = 1 << 18
    pos = rng.random((n, 3), dtype=np.float32)
    w = rng.random(n, dtype=np.float32)
    h = np.exp(rng.uniform(np.log(0.005), np.log(0.05), n)).astype(np.float32)
    edges = np.exp(np.linspace(np.log(0.005), np.log(0.05), 17))
    b = np.clip(np.searchsorted(edges, h, side="right") - 1, 0, 15)
    groups = [(constraints(pos[b == k], w[b == k]), h[b == k], M.GAUSSIAN_DECAYING) for k in range(16)]
    spec_tc, _ = spectrum_and_views(groups, (64, 64, 64), 1.0, (1.0, 1.0), (32, 32), (64, 64), None, M.FORM_TENSOR)
    spec_pl, _ = spectrum_and_views(groups, (64, 64, 64), 1.0, (1.0, 1.0), (32, 32), (64, 64), None, M.FORM_PLAIN)
    prng = np.random.default_rng(3)
    ijk = np.stack([prng.integers(-32, 32, 2048), prng.integers(-32, 32, 2048), prng.integers(0, 33, 2048)], 1)
    ref = sum(O.spectrum_points(g[0], g[1], g[2], 1.0, ijk) for g in groups)
    got = spec_tc[ijk[:, 0] + 32, ijk[:, 1] + 32, ijk[:, 2]]
    assert O.rel_l2(got, ref) < SPEC_TOL
    assert O.rel_l2(spec_tc, spec_pl) < SPEC_TOL


# ---------------------------------------------------------------- batching
def test_batch_of_uneven_jobs_matches_fp64_and_replays_as_a_graph():
    """Three jobs of different particle counts, bases, lattices and image sizes
    (tensor-form and plain-form groups mixed) executed as one batch; each job's
    spectrum and views match the FP64 oracle, and a second execute replaying
    the captured CUDA graph gives the same images, also after the datasets are
    unregistered and registered again."""
    rng = np.random.default_rng(41)
    cfg = M.Config(cutoff=(8, 8), samples=(16, 16), block_length=64)
    specs = [
        # (n, basis, radii kind, grid, cutoff, samples, views)
        (1500, M.WENDLAND_D3_C2, "uniform", (32, 32, 32), (16, 16), (32, 32), rotating_views(4)),
        (777, M.GAUSSIAN_DECAYING, "per_particle", (48, 48, 32), (20, 24), (48, 48), rotating_views(3)),
        (2048, M.SPH, "per_particle", (16, 16, 16), (8, 8), (16, 16), rotating_views(2)),  # plain form
    ]
    datasets, groups_of = [], []
    for n, basis, kind, *_ in specs:
        pos = rng.random((n, 3), dtype=np.float32)
        w = rng.standard_normal(n).astype(np.float32)
        radii = (np.full(n, 0.03, np.float32) if kind == "uniform"
                 else np.exp(rng.uniform(np.log(0.01), np.log(0.05), n)).astype(np.float32))
        groups = [(constraints(pos, w), radii, basis)]
        groups_of.append(groups)
        ds = to_dataset(groups)
        cfg.register(ds)
        datasets.append(ds)
    batch = M.Batch(cfg)
    for ds, (n, basis, kind, grid, cutoff, samples, views) in zip(datasets, specs):
        batch.add(ds, grid, 1.0, (1.0, 1.0), cutoff, samples, [v[0] for v in views], [v[1] for v in views])
    batch.execute(M.FORM_AUTO)
    first = [batch.images(j) for j in range(len(specs))]
    batch.execute(M.FORM_AUTO)
    assert batch.uses_graph() == 1
    for j, (groups, (n, basis, kind, grid, cutoff, samples, views)) in enumerate(zip(groups_of, specs)):
        spec = batch.spectrum(j)
        ref = O.spectrum_grid(groups, 1.0, grid)
        assert O.rel_l2(spec, ref) < SPEC_TOL
        imgs = batch.images(j)
        ref_imgs = O.render_from_spectrum(ref, grid, 1.0, (1.0, 1.0), cutoff, views, samples)
        assert O.rel_l2(imgs, ref_imgs) < IMAGE_TOL
        np.testing.assert_array_equal(imgs, first[j])
    # a frame loop that registers the same datasets again gets the same device
    # blocks back (the config keeps unregistered blocks for the next
    # registration of the same size), so the batch replays its graph: no
    # launch passes through the library's host code
    addrs = [(ds.group(0).d_constraints, ds.group(0).d_radii) for ds in datasets]
    lib = M.lib()
    for _ in range(2):
        for ds in datasets:
            cfg.unregister(ds)
        for ds in datasets:
            cfg.register(ds)
        assert [(ds.group(0).d_constraints, ds.group(0).d_radii) for ds in datasets] == addrs
        c0 = lib.vis_kernel_launch_count()
        batch.execute(M.FORM_AUTO)
        assert lib.vis_kernel_launch_count() == c0 and batch.uses_graph() == 1
        for j in range(len(specs)):
            np.testing.assert_array_equal(batch.images(j), first[j])
    # new weights at the same addresses change the registration statistics
    # the plan reads (the weight scale), so the batch is planned and captured
    # again; the sum is linear in the weights
    cons0 = datasets[0]._keep[0]
    cons0["weight"] *= 2.0
    cfg.unregister(datasets[0])
    cfg.register(datasets[0])
    assert (datasets[0].group(0).d_constraints, datasets[0].group(0).d_radii) == addrs[0]
    c0 = lib.vis_kernel_launch_count()
    batch.execute(M.FORM_AUTO)
    assert lib.vis_kernel_launch_count() > c0 and batch.uses_graph() == 1
    assert O.rel_l2(batch.images(0), 2.0 * first[0]) < 1e-5
    for j in range(1, len(specs)):
        np.testing.assert_array_equal(batch.images(j), first[j])
    batch.close()
    for ds in datasets:
        cfg.unregister(ds)
    cfg.close()


# --------------------------------------------------------- post-processing
@pytest.mark.parametrize("color_map,log_scale", [(1, 1), (2, 0), (3, 1)])
def test_image_postprocessing_matches_restatement(color_map, log_scale):
    import torch

    rng = np.random.default_rng(51)
    imgs = (rng.standard_normal((3, 24, 20)) * 5 + 2).astype(np.float32)
    cfg = M.Config(cutoff=(8, 8), samples=(24, 20), block_length=64)
    d_img = torch.from_numpy(imgs).cuda()
    d_rgb = torch.empty((3, 24, 20, 3), dtype=torch.float32, device="cuda")
    lib = M.lib()
    from libmeshlessvis_b200 import _lib as L

    rc = lib.vis_images_normalize_to_rgb(cfg.ptr, d_img.data_ptr(), 3, L.int2(24, 20), d_rgb.data_ptr())
    assert rc == 0
    cfg.synchronize()
    np.testing.assert_allclose(d_rgb.cpu().numpy(), O.normalize_to_rgb(imgs), rtol=1e-6, atol=1e-7)
    rc = lib.vis_images_colormap(cfg.ptr, d_img.data_ptr(), 3, L.int2(24, 20), -1.0, 9.0, log_scale, color_map,
                                 d_rgb.data_ptr())
    assert rc == 0
    cfg.synchronize()
    np.testing.assert_allclose(d_rgb.cpu().numpy(), O.colormap(imgs, -1.0, 9.0, log_scale, color_map),
                               rtol=1e-5, atol=1e-6)
    cfg.close()


def test_device_shift_matches_host_shift():
    """vis_noninteractive shifts every dataset by -5 before rendering
    (vis_noninteractive/main.cpp:46); shifting the registered device copy gives
    the same image as shifting on the host."""
    rng = np.random.default_rng(61)
    n = 900
    pos = rng.random((n, 3), dtype=np.float32) * 10
    cons = constraints(pos, rng.random(n, dtype=np.float32))
    radii = np.full(n, 0.4, np.float32)
    cfg = M.Config(step=(0.1, 0.1), cutoff=(16, 16), samples=(64, 64), block_length=64)
    ds = to_dataset([(cons, radii, M.SPH)])
    cfg.register(ds)
    lib = M.lib()
    assert lib.vis_shift_registered_dataset(cfg.ptr, ds.ref, -5.0, -5.0, -5.0) == 0
    cfg.render(ds)
    img = cfg.image()
    cfg.unregister(ds)
    cfg.close()
    shifted = constraints(pos - np.float32(5.0), cons["weight"])
    ref = O.render_direct([(shifted, radii, M.SPH)], (0.1, 0.1), (16, 16), (1, 0, 0), (0, 1, 0), (64, 64))
    assert O.rel_l2(img, ref) < SPEC_TOL


# ------------------------------------------------------------ aliasing cull
@pytest.mark.parametrize("with_radii", [True, False])
def test_aliasing_cull_sums_only_the_kept_particles(with_radii):
    """cull_fully_aliased_terms (meshless_vis.cu:39-127, disabled in the
    reference): with the flag set, the direct render equals the FP64 render of
    the particles the oracle's mask keeps (about half of them here, in two
    groups); the registered arrays are untouched, so clearing the flag renders
    the full set again."""
    rng = np.random.default_rng(91)
    step, cutoff, samples = (0.1, 0.1), (16, 16), (64, 64)
    u, v = (0.8, 0.0, -0.6), (0.0, 1.0, 0.0)
    groups = []
    for basis, n in ((M.SPH, 3001), (M.WENDLAND_D3_C2, 2500)):
        pos = (rng.random((n, 3), dtype=np.float32) * 8.0 - 1.0).astype(np.float32)
        radii = np.exp(rng.uniform(np.log(0.1), np.log(0.6), n)).astype(np.float32) if with_radii else None
        groups.append((constraints(pos, rng.standard_normal(n).astype(np.float32)), radii, basis))
    kept = []
    for cons, radii, basis in groups:
        m = O.cull_mask(cons, radii, u, v, step)
        assert 0.2 < m.mean() < 0.8
        kept.append((cons[m], None if radii is None else radii[m], basis))
    cfg = M.Config(step=step, cutoff=cutoff, u=u, v=v, samples=samples, block_length=64)
    ds = to_dataset(groups)
    cfg.register(ds)
    cfg.c.cull_fully_aliased_terms = True
    cfg.render(ds)
    culled = cfg.image()
    cfg.c.cull_fully_aliased_terms = False
    cfg.render(ds)
    full = cfg.image()
    cfg.unregister(ds)
    cfg.close()
    assert O.rel_l2(culled, O.render_direct(kept, step, cutoff, u, v, samples)) < SPEC_TOL
    assert O.rel_l2(full, O.render_direct(groups, step, cutoff, u, v, samples)) < SPEC_TOL
