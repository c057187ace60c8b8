"""Python binding of the drop-in library, mirroring the reference's
python/meshless_vis/meshless.py (whose argtypes are `None #todo` and which
calls a function that does not exist) with working ctypes declarations, plus a
thin object layer used by the tests and the benchmark.

Everything here calls the C ABI of libmeshless_vis.so; no computation happens
in Python.
"""
import ctypes

import numpy as np

from . import _lib as L
from ._lib import (CONSTRAINT_DTYPE, FORM_AUTO, FORM_PLAIN, FORM_TENSOR, GAUSSIAN, GAUSSIAN_DECAYING, SPH,
                   STAGE_FFT, STAGE_SLICE, STAGE_SUM, STAGE_TENSOR_SUM, WENDLAND_D3_C2, Group, MeshlessDataset, VisError, float2,
                   float3, int2, int3)

__all__ = ["get_simple_meshless_dataset", "delete_meshless_dataset", "delete_meshless_datasets",
           "get_number_of_terms", "load_meshless_datasets_from_file", "save_meshless_datasets_to_file",
           "shift_meshless_dataset", "Dataset", "Config", "Spectrum", "constraints_from_arrays", "VisError",
           "SPH", "GAUSSIAN", "WENDLAND_D3_C2", "GAUSSIAN_DECAYING", "FORM_AUTO", "FORM_PLAIN", "FORM_TENSOR",
           "STAGE_SUM", "STAGE_SLICE", "STAGE_FFT", "STAGE_TENSOR_SUM", "Batch", "set_operand_cache_limit"]


def lib():
    return L.load()


def set_operand_cache_limit(nbytes):
    """Device memory the tensor form may keep as precomputed B operands
    (vis_set_operand_cache_limit): None restores the default (an eighth of
    device memory, or MV_TC_OPERAND_CACHE_MB), 0 turns them off.  Applies to
    later computes in this process."""
    lib().vis_set_operand_cache_limit(-1 if nbytes is None else max(0, int(nbytes)))


def constraints_from_arrays(positions, weights):
    """(n,3) positions + (n,) weights -> contiguous Constraint records."""
    positions = np.asarray(positions, dtype=np.float32).reshape(-1, 3)
    weights = np.asarray(weights, dtype=np.float32).reshape(-1)
    c = np.zeros(len(weights), dtype=CONSTRAINT_DTYPE)
    c["position"] = positions
    c["weight"] = weights
    return c


# ---------------------------------------------------------------------------
# Reference-named functions (python/meshless_vis/meshless.py)
# ---------------------------------------------------------------------------
def get_simple_meshless_dataset(number_of_terms, h_constraints, h_radii, basis_function_id):
    """Copies the arrays into library-owned new[] buffers and returns the
    MeshlessDataset that adopts them (release with delete_meshless_dataset)."""
    lb = lib()
    n = int(number_of_terms)
    c = np.ascontiguousarray(h_constraints, dtype=CONSTRAINT_DTYPE)
    pc = lb.meshless_new_constraints(n)
    ctypes.memmove(pc, c.ctypes.data, 16 * n)
    pr = None
    if h_radii is not None:
        r = np.ascontiguousarray(h_radii, dtype=np.float32)
        pr = lb.meshless_new_radii(n)
        ctypes.memmove(pr, r.ctypes.data, 4 * n)
    return lb.get_simple_meshless_dataset(n, pc, pr, int(basis_function_id))


def delete_meshless_dataset(meshless_dataset):
    lib().delete_meshless_dataset(meshless_dataset)


def delete_meshless_datasets(meshless_datasets, number_of_datasets):
    lib().delete_meshless_datasets(meshless_datasets, int(number_of_datasets))


def get_number_of_terms(meshless_dataset):
    return lib().get_number_of_terms(ctypes.byref(meshless_dataset))


def shift_meshless_dataset(meshless_dataset, x, y, z):
    lib().shift_meshless_dataset(ctypes.byref(meshless_dataset), x, y, z)


def load_meshless_datasets_from_file(filename):
    """Returns (pointer to MeshlessDataset array, count)."""
    out = L.PDataset()
    n = ctypes.c_int(0)
    lib().load_meshless_datasets_from_file(str(filename).encode(), ctypes.byref(out), ctypes.byref(n))
    return out, n.value


def save_meshless_datasets_to_file(filename, meshless_datasets, number_of_datasets):
    lib().save_meshless_datasets_to_file(str(filename).encode(), meshless_datasets, int(number_of_datasets))


# ---------------------------------------------------------------------------
# Object layer
# ---------------------------------------------------------------------------
class Dataset:
    """A MeshlessDataset whose host arrays are owned by numpy (kept alive here).
    groups: list of (constraints[CONSTRAINT_DTYPE], radii or None, basis)."""

    def __init__(self, groups):
        self._keep = []
        self._groups = (Group * max(1, len(groups)))()
        for i, (cons, radii, basis) in enumerate(groups):
            cons = np.ascontiguousarray(cons, dtype=CONSTRAINT_DTYPE)
            self._keep.append(cons)
            g = self._groups[i]
            g.number_of_terms = len(cons)
            g.basis_function_id = int(basis)
            g.h_constraints = cons.ctypes.data if len(cons) else None
            if radii is not None:
                r = np.ascontiguousarray(radii, dtype=np.float32)
                self._keep.append(r)
                g.h_radii = r.ctypes.data if len(r) else None
            else:
                g.h_radii = None
        self.ds = MeshlessDataset(self._groups, len(groups))

    @property
    def ref(self):
        return ctypes.byref(self.ds)

    def group(self, i):
        return self._groups[i]


class Config:
    """Owns a VisConfig* (vis_config_create .. vis_config_destroy)."""

    def __init__(self, step=(1.0, 1.0), cutoff=(32, 32), u=(1, 0, 0), v=(0, 1, 0), samples=(64, 64),
                 block_length=256, partial_sums=1, automatic_d_image=True):
        self.lib = lib()
        self.ptr = self.lib.vis_config_create(bool(automatic_d_image), float2(*step), int2(*cutoff), float3(*u),
                                              float3(*v), int2(*samples), int(block_length), int(partial_sums))
        if not self.ptr:
            L.check(self.lib)
            raise VisError(-1, "vis_config_create returned NULL")

    @property
    def c(self):
        return self.ptr.contents

    def check(self):
        return bool(self.lib.vis_config_check(self.ptr))

    def set_axes(self, u, v):
        self.c.u_axis = float3(*u)
        self.c.v_axis = float3(*v)

    def register(self, dataset):
        self.lib.vis_register_meshless_dataset(self.ptr, dataset.ref)
        L.check(self.lib)

    def unregister(self, dataset):
        self.lib.vis_unregister_meshless_dataset(self.ptr, dataset.ref)
        L.check(self.lib)

    def render(self, dataset):
        self.lib.vis_fourier_volume_rendering(dataset.ref, self.ptr)
        L.check(self.lib)

    def image(self):
        nx, ny = self.c._number_of_samples.x, self.c._number_of_samples.y
        out = np.empty((nx, ny), dtype=np.float32)
        self.lib.vis_copy_to_host(self.ptr, out.ctypes.data)
        L.check(self.lib)
        return out

    def set_stream(self, stream_handle):
        L.check(self.lib, self.lib.vis_config_set_stream(self.ptr, stream_handle))

    def synchronize(self):
        L.check(self.lib, self.lib.vis_config_synchronize(self.ptr))

    def enable_timing(self, on=True):
        L.check(self.lib, self.lib.vis_config_enable_kernel_timing(self.ptr, int(bool(on))))

    def kernel_time(self, stage):
        ms = ctypes.c_float(0)
        n = ctypes.c_int(0)
        L.check(self.lib, self.lib.vis_config_kernel_timing(self.ptr, int(stage), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def close(self):
        if self.ptr:
            self.lib.vis_config_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Spectrum:
    """Owns a VisSpectrum* (3D half-spectrum on the device)."""

    def __init__(self, grid, step=1.0):
        self.lib = lib()
        self.grid = tuple(int(g) for g in grid)
        self.ptr = self.lib.vis_spectrum_create(int3(*self.grid), float(step))
        if not self.ptr:
            L.check(self.lib)
            raise VisError(-1, "vis_spectrum_create returned NULL")

    @property
    def shape(self):
        kx, ky, kz = self.grid
        return (kx, ky, kz // 2 + 1)

    def compute(self, config, dataset, form=FORM_AUTO):
        L.check(self.lib, self.lib.vis_spectrum_compute(self.ptr, config.ptr, dataset.ref, int(form)))

    def autotune(self, config, dataset, form=FORM_AUTO):
        """Times the launch-parameter candidates for this shape on `dataset`
        (vis_autotune_spectrum) and returns the best time in ms; later
        computes of the same shape use the chosen parameters."""
        ms = ctypes.c_float(0.0)
        L.check(self.lib, self.lib.vis_autotune_spectrum(self.ptr, config.ptr, dataset.ref, int(form),
                                                         ctypes.byref(ms)))
        return ms.value

    def to_host(self, config):
        out = np.empty(self.shape, dtype=np.complex64)
        L.check(self.lib, self.lib.vis_spectrum_copy_to_host(self.ptr, config.ptr, out.ctypes.data))
        return out

    def render_views(self, config, u_axes, v_axes, d_images=None, to_host=True):
        u = np.ascontiguousarray(u_axes, dtype=np.float32).reshape(-1, 3)
        v = np.ascontiguousarray(v_axes, dtype=np.float32).reshape(-1, 3)
        nv = len(u)
        nx, ny = config.c._number_of_samples.x, config.c._number_of_samples.y
        host = np.empty((nv, nx, ny), dtype=np.float32) if to_host else None
        rc = self.lib.vis_spectrum_render_views(self.ptr, config.ptr, nv, u.ctypes.data, v.ctypes.data,
                                                d_images, host.ctypes.data if to_host else None)
        L.check(self.lib, rc)
        return host

    def close(self):
        if self.ptr:
            self.lib.vis_spectrum_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Owns a VisBatch*: jobs of (registered dataset, lattice, views), executed
    as one CUDA graph (vis_batch_*)."""

    def __init__(self, config):
        self.lib = lib()
        self.config = config
        self.ptr = self.lib.vis_batch_create(config.ptr)
        if not self.ptr:
            L.check(self.lib)
        self.jobs = []

    def add(self, dataset, grid, spectrum_step, view_step, cutoff, samples, u_axes, v_axes):
        u = np.ascontiguousarray(u_axes, dtype=np.float32).reshape(-1, 3)
        v = np.ascontiguousarray(v_axes, dtype=np.float32).reshape(-1, 3)
        j = self.lib.vis_batch_add(self.ptr, dataset.ref, int3(*grid), float(spectrum_step), float2(*view_step),
                                   int2(*cutoff), int2(*samples), len(u), u.ctypes.data, v.ctypes.data)
        if j < 0:
            L.check(self.lib, -j)
        self.jobs.append((tuple(grid), tuple(samples), len(u)))
        return j

    def execute(self, form=FORM_AUTO):
        L.check(self.lib, self.lib.vis_batch_execute(self.ptr, int(form)))

    def uses_graph(self):
        return self.lib.vis_batch_uses_graph(self.ptr)

    def images(self, job):
        _, (nx, ny), nv = self.jobs[job]
        out = np.empty((nv, nx, ny), dtype=np.float32)
        L.check(self.lib, self.lib.vis_batch_copy_images_to_host(self.ptr, job, out.ctypes.data))
        return out

    def spectrum(self, job):
        import ctypes as ct

        (kx, ky, kz), _, _ = self.jobs[job]
        out = np.empty((kx, ky, kz // 2 + 1), dtype=np.complex64)
        d = self.lib.vis_batch_spectrum(self.ptr, job)
        self.config.synchronize()
        rt = _cudart()
        assert rt.cudaMemcpy(out.ctypes.data, ct.c_void_p(d), out.nbytes, 2) == 0
        return out

    def close(self):
        if self.ptr:
            self.lib.vis_batch_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _cudart():
    """The CUDA runtime already loaded in this process (for plain device->host
    copies of library-owned buffers)."""
    import ctypes as ct

    for name in ("libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so"):
        try:
            rt = ct.CDLL(name)
            rt.cudaMemcpy.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_size_t, ct.c_int]
            rt.cudaMemcpy.restype = ct.c_int
            return rt
        except OSError:
            continue
    raise RuntimeError("CUDA runtime library not found")
