"""CPU tests of the checker itself: the FP64 oracle against the golden vectors
that the reference's own CPU code produced, and against known answers."""
import numpy as np
import pytest

import oracle as O


def test_phi_known_values():
    # Phi^(0): SPH pi, Gaussian 1, Wendland 0.2992 (fourier_transform_cpu.cpp:37-66)
    v = O.phi(O.SPH, [0.0])[0]
    assert v == pytest.approx(np.pi, rel=1e-15)
    assert O.phi(O.GAUSSIAN, [0.0])[0] == 1.0
    assert O.phi(O.WENDLAND_D3_C2, [0.0])[0] == pytest.approx(0.299199300341890, rel=1e-15)
    assert O.phi(O.GAUSSIAN_DECAYING, [1.0])[0] == pytest.approx(np.exp(-np.pi), rel=1e-15)
    # closed forms are continuous with the quadratic fits at the branch points
    for b, s0 in [(O.SPH, 0.06), (O.WENDLAND_D3_C2, 0.24)]:
        lo, hi = O.phi(b, [np.float32(s0) - 1e-9, np.float32(s0) + 1e-9])
        assert abs(lo - hi) / abs(O.phi(b, [0.0])[0]) < 2e-4


@pytest.mark.parametrize("name", ["b0_xy", "b0_rot", "b0_noradii", "b1_xy", "b1_rot", "b1_noradii", "b2_xy",
                                  "b2_rot", "b2_noradii", "two_groups_step01", "timing_test_radii",
                                  "timing_test_factor1", "single_particle"])
def test_oracle_matches_reference_golden(golden, name):
    """The FP64 restatement reproduces the reference CPU renderer's output to
    within the reference's own FP32 rounding (it is 1.7e-5..2.8e-5 rel-L2 off
    FP64 for Wendland, a few 1e-6 elsewhere)."""
    c = golden[name]
    cx, cy = (int(x) for x in c["cutoff"])
    sl = np.zeros(2 * cx * cy, dtype=np.complex128)
    for xyzw, radii, basis in c["groups"]:
        O.slice_sum(xyzw, radii, basis, tuple(c["step"]), (cx, cy), c["u"], c["v"], out=sl)
    np.testing.assert_allclose(sl, c["fp64_slice"], rtol=1e-12, atol=1e-12 * np.abs(sl).max())
    assert O.rel_l2(c["ref_slice"], sl) < 5e-5
    img = O.c2r(O.arrange(sl, (cx, cy), tuple(int(s) for s in c["samples"])), tuple(int(s) for s in c["samples"]))
    assert O.rel_l2(c["ref_image"], img) < 5e-5


def test_kat1_particles_at_origin_give_real_spectrum(golden):
    c = golden["timing_test_radii"]
    assert np.abs(c["fp64_slice"].imag).max() == 0.0
    # F = sum w Phi^(r h) scale = 1024 * Phi^(r * 1e-5) ~ 1024 * pi near k = 0
    assert c["fp64_slice"][0].real == pytest.approx(1024 * np.pi, rel=1e-6)


def test_kat2_single_particle_phase():
    cons = np.array([[0.3, 0.6, 0.2, 2.0]], np.float32)
    ijk = np.array([[3, -2, 5], [0, 0, 0], [-7, 1, 2]], np.int32)
    h = np.array([0.05], np.float32)
    got = O.spectrum_points(cons, h, O.WENDLAND_D3_C2, 1.0, ijk)
    k = ijk.astype(np.float64)
    r = np.linalg.norm(k, axis=1)
    x = cons[0, :3].astype(np.float64)
    want = 2.0 * O.phi(O.WENDLAND_D3_C2, r * np.float64(h[0])) * np.exp(-2j * np.pi * (k @ x))
    np.testing.assert_allclose(got, want, rtol=1e-13)


def test_kat3_and_kat4_hermitian_symmetry():
    rng = np.random.default_rng(3)
    cons = np.concatenate([rng.random((50, 3)), rng.standard_normal((50, 1))], axis=1).astype(np.float32)
    h = rng.uniform(0.01, 0.05, 50).astype(np.float32)
    ijk = np.array([[2, 3, 1], [-2, -3, -1], [0, 0, 0]], np.int32)
    f = O.spectrum_points(cons, h, O.SPH, 1.0, ijk)
    np.testing.assert_allclose(f[0], np.conj(f[1]), rtol=1e-12)
    assert f[2].real == pytest.approx(float(np.sum(cons[:, 3].astype(np.float64))) * np.pi, rel=1e-12)


def test_kat5_z_normal_slice_from_spectrum_equals_direct(golden):
    """A z-normal view at the lattice step lands on lattice points, so the
    interpolated slice equals the reference's direct slice."""
    rng = np.random.default_rng(5)
    cons = np.concatenate([rng.random((200, 3)), rng.standard_normal((200, 1))], axis=1).astype(np.float32)
    h = np.full(200, 0.03, np.float32)
    groups = [(cons, h, O.GAUSSIAN)]
    spec = O.spectrum_grid(groups, 1.0, (16, 16, 16))
    img_s = O.render_from_spectrum(spec, (16, 16, 16), 1.0, (1.0, 1.0), (8, 8), [((1, 0, 0), (0, 1, 0))], (16, 16))[0]
    img_d = O.render_direct(groups, (1.0, 1.0), (8, 8), (1, 0, 0), (0, 1, 0), (16, 16))
    np.testing.assert_allclose(img_s, img_d, rtol=1e-12, atol=1e-12 * np.abs(img_d).max())


def test_c2r_matches_numpy_irfft2():
    rng = np.random.default_rng(7)
    for nx, ny in [(16, 12), (12, 10), (32, 32)]:
        real = rng.standard_normal((nx, ny))
        spec = np.fft.rfft2(real)  # Hermitian-consistent input
        got = O.c2r(spec, (nx, ny))
        np.testing.assert_allclose(got, real * nx * ny, rtol=1e-10, atol=1e-9)


def test_spectrum_grid_matches_points(golden):
    c = golden["spec_b2"]
    grid = tuple(int(g) for g in c["grid"])
    kx, ky, kz = grid
    xyzw, radii, basis = c["groups"][0]
    ijk = np.array([[i, j, l] for i in (-kx // 2, 0, kx // 2 - 1) for j in (-ky // 2, 1) for l in (0, kz // 2)])
    pts = O.spectrum_points(xyzw, radii, basis, float(c["step3"]), ijk)
    spec = c["fp64_spectrum"]
    got = np.array([spec[i + kx // 2, j + ky // 2, l] for i, j, l in ijk])
    np.testing.assert_allclose(got, pts, rtol=1e-12, atol=1e-14)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_reference_build_runs_and_matches_oracle_live():
    rng = np.random.default_rng(11)
    cons = np.concatenate([rng.random((300, 3)), rng.standard_normal((300, 1))], axis=1).astype(np.float32)
    h = np.full(300, 0.04, np.float32)
    groups = [(cons, h, O.SPH)]
    R = O.RefRenderer(groups, (1.0, 1.0), (8, 8), (1, 0, 0), (0, 1, 0), (16, 16))
    img = R.render()
    R.close()
    assert O.rel_l2(img, O.render_direct(groups, (1.0, 1.0), (8, 8), (1, 0, 0), (0, 1, 0), (16, 16))) < 2e-5


def test_cull_mask_known_answers():
    """meshless_vis.cu:39-57: kept when the footprint square lies in
    [0, 1/(2 step.x)] x [0, 1/(2 step.y)] (step 0.1: the box is [0, 5]^2)."""
    from libmeshlessvis_b200.workloads import constraints

    pos = np.array([[1, 1, 9], [4.9, 2, 0], [4.9, 2, 0], [-0.1, 1, 0], [2, 5.2, 0], [0.3, 0.3, 0]], np.float32)
    radii = np.array([0.5, 0.2, 0.05, 0.01, 0.1, 0.3], np.float32)
    cons = constraints(pos, np.ones(len(pos), np.float32))
    keep = O.cull_mask(cons, radii, (1, 0, 0), (0, 1, 0), (0.1, 0.1))
    assert keep.tolist() == [True, False, True, False, False, True]
    # without radii the footprint is the centre
    assert O.cull_mask(cons, None, (1, 0, 0), (0, 1, 0), (0.1, 0.1)).tolist() == [True, True, True, False, False, True]
    # a rotated view projects z onto u
    keep = O.cull_mask(cons, None, (0, 0, 1), (0, 1, 0), (0.1, 0.1))
    assert keep.tolist() == [False, True, True, True, False, True]
