"""Seeded synthetic particle sets for the five benchmark configurations.

No dataset ships with the reference (vis_noninteractive/main.cpp:322 names a
missing ../data/cartwheel.sph), so inputs are generated with the shapes, sizes
and value distributions each configuration specifies:

  C1  N=4096 uniform in [0,1)^3, w ~ N(0,1), GAUSSIAN h=0.02, 64x64x64 grid,
      one z-normal view, cutoff 32, 64^2 image.
  C2  N=262,144 Plummer (scale 0.1, centred at 0.5, resampled into the unit
      cube), mass m = 1/N, mass density rho_j = 32 m / (4/3 pi r32_j^3) from the
      distance r32_j to the 32nd nearest neighbour, w_j = m / rho_j (the
      particle's volume), h_j = r32_j,
      WENDLAND_D3_C2, 128^3 grid, 64 views rotating about y, cutoff 64, 128^2.
  C3  N=2^20 uniform, w ~ U(0,1), GAUSSIAN_DECAYING with h log-uniform in
      [0.005, 0.05] (16 log-spaced h-bins), 256^3 grid; error on 4096 random
      half-spectrum wavenumbers (seed 1).
  C4  64 sets, N_s log-uniform in [1k, 512k], alternating uniform / Plummer,
      WENDLAND_D3_C2 with one h per set in U[0.01, 0.04], grid per set from
      {64,96,128,192}^3, 16 views per set.
  C5  8 frames of N=2^24 Plummer drifting by N(0, 0.002) per frame,
      w ~ N(1, 0.1), GAUSSIAN_DECAYING with 8 h-bins in [0.002, 0.02],
      384^3 grid, 360 views per frame at 384^2.
Step is 1 everywhere, so wavenumbers are integers (as in
vis_timing_test/main.cpp:63).
"""
import numpy as np

from ._lib import CONSTRAINT_DTYPE, GAUSSIAN, GAUSSIAN_DECAYING, WENDLAND_D3_C2


def constraints(pos, w):
    c = np.zeros(len(w), dtype=CONSTRAINT_DTYPE)
    c["position"] = pos
    c["weight"] = w
    return c


def uniform_positions(rng, n):
    return rng.random((n, 3), dtype=np.float32)


def plummer_positions(rng, n, scale=0.1, centre=0.5):
    """Plummer sphere of scale radius `scale`: r = a / sqrt(u^(-2/3) - 1),
    isotropic direction; points outside [0,1)^3 are redrawn."""
    out = np.empty((0, 3), dtype=np.float64)
    while len(out) < n:
        m = 2 * (n - len(out)) + 1024
        u = rng.random(m)
        u = np.clip(u, 1e-12, 1 - 1e-12)
        r = scale / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        d = rng.standard_normal((m, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        p = centre + r[:, None] * d
        ok = np.all((p >= 0.0) & (p < 1.0), axis=1)
        out = np.concatenate([out, p[ok]])
    return out[:n].astype(np.float32)


def knn_radius(pos, k=32):
    """Distance from each point to its k-th nearest other point."""
    from scipy.spatial import cKDTree

    tree = cKDTree(pos.astype(np.float64))
    d, _ = tree.query(pos.astype(np.float64), k=k + 1, workers=-1)
    return d[:, k].astype(np.float32)


def c1(seed=0):
    rng = np.random.default_rng(seed)
    n = 4096
    pos = uniform_positions(rng, n)
    w = rng.standard_normal(n).astype(np.float32)
    h = np.full(n, 0.02, dtype=np.float32)
    return dict(name="C1", groups=[(constraints(pos, w), h, GAUSSIAN)], grid=(64, 64, 64), step3=1.0,
                cutoff=(32, 32), samples=(64, 64), views=[((1, 0, 0), (0, 1, 0))], step=(1.0, 1.0))


def rotating_views(count):
    """Views rotating about y (vis_wx/main.cpp:60-80 basis with phi = 0):
    u = (cos t, 0, -sin t), v = (0, 1, 0), t = 2 pi i / count."""
    out = []
    for i in range(count):
        t = 2.0 * np.pi * i / count
        out.append(((np.cos(t), 0.0, -np.sin(t)), (0.0, 1.0, 0.0)))
    return out


def c2(seed=0, n=262144, grid=128, views=64):
    rng = np.random.default_rng(seed)
    pos = plummer_positions(rng, n)
    r32 = knn_radius(pos, 32)
    mass = 1.0 / n
    rho = 32.0 * mass / (4.0 / 3.0 * np.pi * r32.astype(np.float64) ** 3)
    w = (mass / rho).astype(np.float32)
    return dict(name="C2", groups=[(constraints(pos, w), r32, WENDLAND_D3_C2)], grid=(grid, grid, grid), step3=1.0,
                cutoff=(grid // 2, grid // 2), samples=(grid, grid), views=rotating_views(views), step=(1.0, 1.0))


def c3(seed=0, n=1 << 20, grid=256, bins=16):
    rng = np.random.default_rng(seed)
    pos = uniform_positions(rng, n)
    w = rng.random(n, dtype=np.float32)
    lo, hi = np.log(0.005), np.log(0.05)
    h = np.exp(rng.uniform(lo, hi, n)).astype(np.float32)
    # 16 log-spaced bins: the group order is by bin, one group per bin
    edges = np.exp(np.linspace(lo, hi, bins + 1))
    b = np.clip(np.searchsorted(edges, h, side="right") - 1, 0, bins - 1)
    groups = []
    for k in range(bins):
        sel = b == k
        groups.append((constraints(pos[sel], w[sel]), h[sel], GAUSSIAN_DECAYING))
    prng = np.random.default_rng(1)
    ijk = np.stack([prng.integers(-grid // 2, grid // 2, 4096), prng.integers(-grid // 2, grid // 2, 4096),
                    prng.integers(0, grid // 2 + 1, 4096)], axis=1).astype(np.int32)
    return dict(name="C3", groups=groups, grid=(grid, grid, grid), step3=1.0, check_points=ijk,
                cutoff=(grid // 2, grid // 2), samples=(grid, grid), views=[((1, 0, 0), (0, 1, 0))], step=(1.0, 1.0))


def c4(seed=0, sets=64, max_n=512 * 1024):
    rng = np.random.default_rng(seed)
    out = []
    for s in range(sets):
        n = int(np.exp(rng.uniform(np.log(1024), np.log(max_n))))
        pos = uniform_positions(rng, n) if s % 2 == 0 else plummer_positions(rng, n)
        w = rng.standard_normal(n).astype(np.float32) / np.sqrt(n)
        h = float(rng.uniform(0.01, 0.04))
        g = int(rng.choice([64, 96, 128, 192]))
        # one h per set, given as a constant radii array: Phi^(|k| h) then
        # factors out of the sum (the tensor-core form applies it per frequency)
        out.append(dict(groups=[(constraints(pos, w), np.full(n, h, np.float32), WENDLAND_D3_C2)], grid=(g, g, g),
                        step3=1.0, cutoff=(g // 2, g // 2), samples=(g, g), views=rotating_views(16), step=(1.0, 1.0)))
    return out


def c5_frames(seed=0, n=1 << 24, frames=8, bins=8):
    """Generator of frames (positions drift by N(0, 0.002) per frame)."""
    rng = np.random.default_rng(seed)
    pos = plummer_positions(rng, n)
    w = rng.normal(1.0, 0.1, n).astype(np.float32)
    edges = np.exp(np.linspace(np.log(0.002), np.log(0.02), bins + 1))
    h = np.exp(rng.uniform(np.log(0.002), np.log(0.02), n)).astype(np.float32)
    b = np.clip(np.searchsorted(edges, h, side="right") - 1, 0, bins - 1)
    for f in range(frames):
        if f:
            pos = np.clip(pos + rng.normal(0.0, 0.002, pos.shape).astype(np.float32), 0.0, np.nextafter(1, 0))
        groups = [(constraints(pos[b == k], w[b == k]), h[b == k], GAUSSIAN_DECAYING) for k in range(bins)]
        yield dict(name="C5", groups=groups, grid=(384, 384, 384), step3=1.0, cutoff=(192, 192), samples=(384, 384),
                   views=rotating_views(360), step=(1.0, 1.0))
