"""Checker for the libMeshlessVis hot path.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg (and its
`--impl reference` arm) may import this package.  The product library neither
links nor calls anything here.

Two checkers:
  * the FP64 restatement (oracle.c -> liboracle.so), each function citing the
    reference lines it restates;
  * the reference's own CPU path (meshless_vis/fourier_transform_cpu.cpp,
    meshless.cpp, meshless_vis_cpu.cpp compiled verbatim by oracle/Makefile into
    _ref/libmeshless_vis_ref.so), which pins the restatement and serves as the
    timed CPU baseline.
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, c_bool, c_double, c_float, c_int, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libmeshless_vis_ref.so"

SPH, GAUSSIAN, WENDLAND_D3_C2, GAUSSIAN_DECAYING = 0, 1, 2, 3

_dp = POINTER(c_double)
_fp = POINTER(c_float)


def build(quiet=True):
    """Builds liboracle.so (and _ref/ when the reference sources are present)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


_olib = None


def olib():
    global _olib
    if _olib is None:
        if not ORACLE_SO.exists():
            build()
        lib = ctypes.CDLL(str(ORACLE_SO), mode=ctypes.RTLD_LOCAL)
        lib.mvo_phi.restype = c_double
        lib.mvo_phi.argtypes = [c_int, c_double]
        lib.mvo_phi_array.argtypes = [c_int, _dp, c_int, _dp]
        lib.mvo_slice_sum.argtypes = [_fp, _fp, c_int, c_int, c_float, c_float, c_int, c_int, _fp, _fp, c_int, _dp]
        lib.mvo_arrange.argtypes = [_dp, c_int, c_int, c_int, c_int, _dp]
        lib.mvo_c2r.argtypes = [_dp, c_int, c_int, _dp]
        lib.mvo_spectrum_points.argtypes = [_fp, _fp, c_int, c_int, c_double, POINTER(c_int), c_int, _dp]
        lib.mvo_spectrum_grid.argtypes = [_fp, _fp, c_int, c_int, c_double, c_int, c_int, c_int, c_int, _dp]
        lib.mvo_extract_slice.argtypes = [_dp, c_int, c_int, c_int, c_double, c_float, c_float, c_int, c_int,
                                          _fp, _fp, c_int, c_int, _dp]
        _olib = lib
    return _olib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _xyzw(cons):
    """Constraint records (or an (n,4) array) -> contiguous (n,4) float32."""
    if cons.dtype.names:
        out = np.empty((len(cons), 4), dtype=np.float32)
        out[:, :3] = cons["position"]
        out[:, 3] = cons["weight"]
        return out
    return _f32(cons).reshape(-1, 4)


def phi(basis, r):
    r = np.ascontiguousarray(r, dtype=np.float64).ravel()
    out = np.empty_like(r)
    olib().mvo_phi_array(basis, _ptr(r, _dp), len(r), _ptr(out, _dp))
    return out


def slice_sum(cons, radii, basis, step, cutoff, u, v, out=None):
    """Direct slice sum of one group in the reference's index order
    (fourier_transform_cpu.cpp:73-134); accumulates into `out` if given."""
    xyzw = _xyzw(cons)
    r = None if radii is None else _f32(radii)
    cx, cy = cutoff
    acc = out is not None
    res = np.zeros(2 * 2 * cx * cy, dtype=np.float64) if out is None else out.view(np.float64)
    olib().mvo_slice_sum(_ptr(xyzw, _fp), _ptr(r, _fp), len(xyzw), basis, step[0], step[1], cx, cy,
                         _ptr(_f32(u), _fp), _ptr(_f32(v), _fp), int(acc), res.ctypes.data_as(_dp))
    return res.view(np.complex128)


def arrange(slice_values, cutoff, samples):
    s = np.ascontiguousarray(slice_values, dtype=np.complex128)
    nx, ny = samples
    out = np.empty((nx, ny // 2 + 1), dtype=np.complex128)
    olib().mvo_arrange(s.view(np.float64).ctypes.data_as(_dp), cutoff[0], cutoff[1], nx, ny,
                       out.view(np.float64).ctypes.data_as(_dp))
    return out


def c2r(arranged, samples):
    a = np.ascontiguousarray(arranged, dtype=np.complex128)
    nx, ny = samples
    out = np.empty((nx, ny), dtype=np.float64)
    olib().mvo_c2r(a.view(np.float64).ctypes.data_as(_dp), nx, ny, out.ctypes.data_as(_dp))
    return out


def render_direct(groups, step, cutoff, u, v, samples):
    """The reference's vis_fourier_volume_rendering in FP64: slice sum of every
    group, arrange_samples, unnormalised C2R.  groups: [(cons, radii, basis)]."""
    cx, cy = cutoff
    sl = np.zeros(2 * cx * cy, dtype=np.complex128)
    for cons, radii, basis in groups:
        slice_sum(cons, radii, basis, step, cutoff, u, v, out=sl)
    return c2r(arrange(sl, cutoff, samples), samples)


def spectrum_points(cons, radii, basis, step3, ijk):
    xyzw = _xyzw(cons)
    r = None if radii is None else _f32(radii)
    ijk = np.ascontiguousarray(ijk, dtype=np.int32).reshape(-1, 3)
    out = np.empty(len(ijk), dtype=np.complex128)
    olib().mvo_spectrum_points(_ptr(xyzw, _fp), _ptr(r, _fp), len(xyzw), basis, step3,
                               ijk.ctypes.data_as(POINTER(c_int)), len(ijk), out.view(np.float64).ctypes.data_as(_dp))
    return out


def spectrum_grid(groups, step3, grid):
    """3D half-spectrum [Kx][Ky][Kz/2+1] of all groups (first assigns)."""
    kx, ky, kz = grid
    out = np.zeros((kx, ky, kz // 2 + 1), dtype=np.complex128)
    for gi, (cons, radii, basis) in enumerate(groups):
        xyzw = _xyzw(cons)
        r = None if radii is None else _f32(radii)
        olib().mvo_spectrum_grid(_ptr(xyzw, _fp), _ptr(r, _fp), len(xyzw), basis, step3, kx, ky, kz, int(gi > 0),
                                 out.view(np.float64).ctypes.data_as(_dp))
    return out


def extract_slice(spec, grid, step3, step, cutoff, u, v, samples):
    s = np.ascontiguousarray(spec, dtype=np.complex128)
    nx, ny = samples
    out = np.empty((nx, ny // 2 + 1), dtype=np.complex128)
    olib().mvo_extract_slice(s.view(np.float64).ctypes.data_as(_dp), grid[0], grid[1], grid[2], step3, step[0],
                             step[1], cutoff[0], cutoff[1], _ptr(_f32(u), _fp), _ptr(_f32(v), _fp), nx, ny,
                             out.view(np.float64).ctypes.data_as(_dp))
    return out


def render_from_spectrum(spec, grid, step3, step, cutoff, views, samples):
    """FP64 images of views [(u, v)] cut from a half-spectrum."""
    return np.stack([c2r(extract_slice(spec, grid, step3, step, cutoff, u, v, samples), samples) for u, v in views])


def cull_mask(cons, radii, u, v, step):
    """The aliasing cull's keep mask, as meshless_vis/meshless_vis.cu:39-57
    (compute_mask, point_in_box) with the box of :88-89: a particle is kept
    when its footprint square, centre (p.u, p.v) and half-side h (0 without
    radii), lies inside [0, 1/(2 step.x)] x [0, 1/(2 step.y)].  Computed in
    FP32 as the reference does."""
    xyzw = _xyzw(cons)
    p = xyzw[:, :3].astype(np.float32)
    u = np.asarray(u, np.float32)
    v = np.asarray(v, np.float32)
    cx = (p[:, 0] * u[0] + p[:, 1] * u[1] + p[:, 2] * u[2]).astype(np.float32)
    cy = (p[:, 0] * v[0] + p[:, 1] * v[1] + p[:, 2] * v[2]).astype(np.float32)
    r = np.zeros(len(p), np.float32) if radii is None else _f32(radii)
    bx = np.float32(0.5) / np.float32(step[0])
    by = np.float32(0.5) / np.float32(step[1])
    keep = np.ones(len(p), bool)
    for xs in (cx + r, cx - r):
        for ys in (cy + r, cy - r):
            keep &= (xs >= 0) & (ys >= 0) & (xs <= bx) & (ys <= by)
    return keep


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / den) if den > 0 else float(np.linalg.norm(a.ravel()))


def max_abs(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if np.size(a) else 0.0


# ---------------------------------------------------------------------------
# The reference's own CPU path (oracle/_ref)
# ---------------------------------------------------------------------------
class _f2(ctypes.Structure):
    _fields_ = [("x", c_float), ("y", c_float)]


class _i2(ctypes.Structure):
    _fields_ = [("x", c_int), ("y", c_int)]


class _f3(ctypes.Structure):
    _fields_ = [("x", c_float), ("y", c_float), ("z", c_float)]


class RefGroup(ctypes.Structure):
    _fields_ = [("number_of_terms", c_int), ("d_number_of_terms", c_int), ("basis_function_id", c_int),
                ("h_constraints", c_void_p), ("d_constraints", c_void_p),
                ("h_radii", c_void_p), ("d_radii", c_void_p)]


class RefDataset(ctypes.Structure):
    _fields_ = [("groups", POINTER(RefGroup)), ("number_of_groups", c_int)]


class RefVisConfig(ctypes.Structure):
    """include/meshless_vis.h:39-79 with _LIBMESHLESSVIS_USE_CPU (FFTW types)."""
    _fields_ = [("step_size", _f2), ("_cutoff_frequency", _i2), ("u_axis", _f3), ("v_axis", _f3),
                ("cull_fully_aliased_terms", c_bool), ("_automatic_d_image", c_bool), ("_plan", c_void_p),
                ("_number_of_samples", _i2), ("block_length", c_int), ("_scale", c_float),
                ("_d_image", c_void_p), ("_d_freq_image", c_void_p), ("_number_of_partial_sums", c_int),
                ("_d_freq_image_arranged", c_void_p)]


_rlib = None


def ref_available():
    return REF_SO.exists()


def rlib():
    global _rlib
    if _rlib is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference sources: make -C oracle ref)")
        lib = ctypes.CDLL(str(REF_SO), mode=ctypes.RTLD_LOCAL)
        P = POINTER(RefVisConfig)
        lib.vis_config_create.restype = P
        lib.vis_config_create.argtypes = [c_bool, _f2, _i2, _f3, _f3, _i2, c_int, c_int]
        lib.vis_config_destroy.argtypes = [P]
        lib.vis_config_check.restype = c_bool
        lib.vis_config_check.argtypes = [P]
        lib.vis_register_meshless_dataset.argtypes = [P, POINTER(RefDataset)]
        lib.vis_unregister_meshless_dataset.argtypes = [P, POINTER(RefDataset)]
        lib.vis_fourier_volume_rendering.argtypes = [POINTER(RefDataset), P]
        lib.vis_copy_to_host.argtypes = [P, c_void_p]
        ft = getattr(lib, "_Z17fourier_transformP15MeshlessDatasetP9VisConfig")
        ft.argtypes = [POINTER(RefDataset), P]
        lib.fourier_transform = ft
        _rlib = lib
    return _rlib


class RefRenderer:
    """The reference CPU renderer driven through its public C API
    (vis_config_create / vis_register_meshless_dataset /
    vis_fourier_volume_rendering / vis_copy_to_host)."""

    def __init__(self, groups, step, cutoff, u, v, samples, block_length=256):
        self.lib = rlib()
        self._keep = []
        self._groups = (RefGroup * max(1, len(groups)))()
        for i, (cons, radii, basis) in enumerate(groups):
            xyzw = _xyzw(cons)
            self._keep.append(xyzw)
            g = self._groups[i]
            g.number_of_terms = len(xyzw)
            g.basis_function_id = basis
            g.h_constraints = xyzw.ctypes.data
            if radii is not None:
                r = _f32(radii)
                self._keep.append(r)
                g.h_radii = r.ctypes.data
            else:
                g.h_radii = None
        self.ds = RefDataset(self._groups, len(groups))
        self.samples = tuple(samples)
        self.cutoff = tuple(cutoff)
        self.cfg = self.lib.vis_config_create(True, _f2(*step), _i2(*cutoff), _f3(*u), _f3(*v), _i2(*samples),
                                              block_length, 1)
        self.lib.vis_register_meshless_dataset(self.cfg, ctypes.byref(self.ds))
        self.registered = True

    def set_axes(self, u, v):
        self.cfg.contents.u_axis = _f3(*u)
        self.cfg.contents.v_axis = _f3(*v)

    def fourier_transform(self):
        """The hot path alone: the reference's fourier_transform() (OpenMP)."""
        self.lib.fourier_transform(ctypes.byref(self.ds), self.cfg)

    def slice(self):
        """Slice values after fourier_transform(), reference index order."""
        cx, cy = self.cutoff
        buf = (ctypes.c_float * (2 * 2 * cx * cy)).from_address(self.cfg.contents._d_freq_image)
        return np.frombuffer(buf, dtype=np.float32).copy().view(np.complex64)

    def render(self):
        self.lib.vis_fourier_volume_rendering(ctypes.byref(self.ds), self.cfg)
        out = np.empty(self.samples, dtype=np.float32)
        self.lib.vis_copy_to_host(self.cfg, out.ctypes.data)
        return out

    def close(self):
        if self.cfg:
            # the reference CPU build frees the padded copies with free()
            self.lib.vis_unregister_meshless_dataset(self.cfg, ctypes.byref(self.ds))
            self.lib.vis_config_destroy(self.cfg)
            self.cfg = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Image post-processing (numpy restatements)
# ---------------------------------------------------------------------------
def normalize_to_rgb(images):
    """vis_noninteractive/main.cpp:70-84: m = max over the raw samples (from
    sample 0), negatives clamped to 0, grey RGB = sample / m."""
    images = np.asarray(images, dtype=np.float64)
    out = []
    for img in images.reshape(images.shape[0], -1):
        m = img.max()
        g = np.maximum(img, 0.0) / m
        out.append(np.repeat(g[:, None], 3, axis=1))
    return np.stack(out).reshape(images.shape + (3,))


_KNOTS = {
    1: ([0.0, 0.475, 0.694, 0.745, 1.0], [(0, 0, 0), (0.686, 0.004, 0.0), (1.0, 0.42, 0.0), (1.0, 0.518, 0.0),
                                          (1, 1, 1)]),
    2: ([0.0, 0.25, 0.5, 0.75, 1.0], [(0, 0, 1), (0, 1, 1), (0, 1, 0), (1, 1, 0), (1, 0, 0)]),
    3: ([0.0, 0.475, 0.694, 0.745, 1.0], [(0, 0, 0), (0.0, 0.004, 0.686), (0.0, 0.42, 1.0), (0.0, 0.518, 1.0),
                                          (1, 1, 1)]),
}


def colormap(images, imin, imax, log_scale, color_map):
    """vis_wx/local_glsl.h:28-87: a = max(0, (a-min)/(max-min)); log scale
    (eps 1e-3, alpha 0.01); piecewise-linear map over 5 knots, the last colour
    above the last knot."""
    a = np.maximum(0.0, (np.asarray(images, dtype=np.float64) - imin) / (imax - imin))
    if log_scale:
        eps, alpha = 1e-3, 0.01
        a = (-np.log(eps) + np.log(alpha * a + eps)) / (np.log(alpha + eps) - np.log(eps))
    xs, cs = _KNOTS[color_map]
    cs = np.asarray(cs, dtype=np.float64)
    out = np.empty(a.shape + (3,))
    flat = a.ravel()
    res = out.reshape(-1, 3)
    for idx, v in enumerate(flat):
        col = cs[-1]
        for i in range(1, 5):
            if v <= xs[i]:
                d = xs[i] - xs[i - 1]
                col = ((v - xs[i - 1]) * cs[i] + (xs[i] - v) * cs[i - 1]) / d
                break
        res[idx] = col
    return out
