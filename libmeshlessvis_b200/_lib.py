"""ctypes declarations of libmeshless_vis.so (include/meshless.h,
include/meshless_vis.h, include/meshless_vis_b200.h).

The library is the product: this module only describes its C ABI.  It raises
at import time when the shared library has not been built, so no caller can
silently run without the CUDA code.
"""
import ctypes
from ctypes import POINTER, c_bool, c_char_p, c_float, c_int, c_longlong, c_void_p
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libmeshless_vis.so"


class float2(ctypes.Structure):
    _fields_ = [("x", c_float), ("y", c_float)]


class int2(ctypes.Structure):
    _fields_ = [("x", c_int), ("y", c_int)]


class float3(ctypes.Structure):
    _fields_ = [("x", c_float), ("y", c_float), ("z", c_float)]


class int3(ctypes.Structure):
    _fields_ = [("x", c_int), ("y", c_int), ("z", c_int)]


# include/meshless.h: enum BasisFunctionId
SPH, GAUSSIAN, WENDLAND_D3_C2, GAUSSIAN_DECAYING = 0, 1, 2, 3
BASIS_NAMES = {"sph": SPH, "gaussian": GAUSSIAN, "wendland_d3_c2": WENDLAND_D3_C2,
               "gaussian_decaying": GAUSSIAN_DECAYING}

# include/meshless_vis_b200.h: enum VisSumForm / VisTimingStage / VisError
FORM_AUTO, FORM_PLAIN, FORM_TENSOR = 0, 1, 2
# include/meshless_vis_b200.h: VIS_TILE_* (tensor-form tile shapes, bits)
TILE_ROW_FOLD, TILE_AXIS_EXCHANGE, TILE_DOUBLE_BUFFER, TILE_CTA_PAIRS, TILE_ALL = 1, 2, 4, 8, 15
STAGE_SUM, STAGE_SLICE, STAGE_FFT, STAGE_TENSOR_SUM = 0, 1, 2, 3
VIS_SUCCESS = 0

# Constraint: __align__(16) { float3 position; float weight; }
CONSTRAINT_DTYPE = np.dtype({"names": ["position", "weight"], "formats": [(np.float32, 3), np.float32],
                             "offsets": [0, 12], "itemsize": 16})


class Group(ctypes.Structure):
    _fields_ = [("number_of_terms", c_int), ("d_number_of_terms", c_int), ("basis_function_id", c_int),
                ("h_constraints", c_void_p), ("d_constraints", c_void_p),
                ("h_radii", c_void_p), ("d_radii", c_void_p)]


class MeshlessDataset(ctypes.Structure):
    _fields_ = [("groups", POINTER(Group)), ("number_of_groups", c_int)]


class VisConfig(ctypes.Structure):
    _fields_ = [("step_size", float2), ("_cutoff_frequency", int2), ("u_axis", float3), ("v_axis", float3),
                ("cull_fully_aliased_terms", c_bool), ("_automatic_d_image", c_bool), ("_plan", c_int),
                ("_number_of_samples", int2), ("block_length", c_int), ("_scale", c_float),
                ("_d_image", c_void_p), ("_d_freq_image", c_void_p), ("_number_of_partial_sums", c_int),
                ("_d_freq_image_arranged", c_void_p)]


PDataset = POINTER(MeshlessDataset)
PConfig = POINTER(VisConfig)

# name -> (restype, argtypes)
SIGNATURES = {
    # include/meshless.h
    "get_simple_meshless_dataset": (MeshlessDataset, [c_int, c_void_p, c_void_p, c_int]),
    "delete_meshless_dataset": (None, [MeshlessDataset]),
    "delete_meshless_datasets": (None, [PDataset, c_int]),
    "get_number_of_terms": (c_int, [PDataset]),
    "shift_meshless_dataset": (None, [PDataset, c_float, c_float, c_float]),
    "shift_meshless_datasets": (None, [PDataset, c_int, c_float, c_float, c_float]),
    "load_meshless_datasets_from_file": (None, [c_char_p, POINTER(PDataset), POINTER(c_int)]),
    "save_meshless_datasets_to_file": (None, [c_char_p, PDataset, c_int]),
    "meshless_new_constraints": (c_void_p, [c_int]),
    "meshless_new_radii": (c_void_p, [c_int]),
    # include/meshless_vis.h
    "vis_config_create": (PConfig, [c_bool, float2, int2, float3, float3, int2, c_int, c_int]),
    "vis_config_get_default": (PConfig, []),
    "vis_config_check": (c_bool, [PConfig]),
    "vis_config_manual_d_image": (None, [PConfig, c_void_p]),
    "vis_config_change_number_of_samples": (None, [PConfig, int2]),
    "vis_config_change_cutoff_frequency": (None, [PConfig, int2]),
    "vis_config_change_number_of_partial_sums": (None, [PConfig, c_int]),
    "vis_config_destroy": (None, [PConfig]),
    "vis_config_compute_scale": (None, [PConfig]),
    "vis_register_meshless_dataset": (None, [PConfig, PDataset]),
    "vis_unregister_meshless_dataset": (None, [PConfig, PDataset]),
    "vis_opengl_fourier_volume_rendering": (None, [PDataset, PConfig, ctypes.c_uint]),
    "vis_fourier_volume_rendering": (None, [PDataset, PConfig]),
    "vis_copy_to_host": (None, [PConfig, c_void_p]),
    # include/meshless_vis_b200.h
    "vis_get_last_error": (c_int, []),
    "vis_get_last_error_message": (c_char_p, []),
    "vis_get_error_string": (c_char_p, [c_int]),
    "vis_clear_last_error": (None, []),
    "vis_config_set_stream": (c_int, [PConfig, c_void_p]),
    "vis_config_get_stream": (c_void_p, [PConfig]),
    "vis_config_synchronize": (c_int, [PConfig]),
    "vis_spectrum_create": (c_void_p, [int3, c_float]),
    "vis_spectrum_destroy": (None, [c_void_p]),
    "vis_spectrum_grid_size": (int3, [c_void_p]),
    "vis_spectrum_device_data": (c_void_p, [c_void_p]),
    "vis_spectrum_compute": (c_int, [c_void_p, PConfig, PDataset, c_int]),
    "vis_autotune_spectrum": (c_int, [c_void_p, PConfig, PDataset, c_int, POINTER(c_float)]),
    "vis_autotune_lookup": (c_int, [int3, c_longlong, c_int, c_int, POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "vis_autotune_lookup_shapes": (c_int, [int3, c_longlong, c_int, c_int, POINTER(c_int), POINTER(c_int)]),
    "vis_autotune_store": (c_int, [int3, c_longlong, c_int, c_int, c_int, c_int, c_int, c_int, c_int]),
    "vis_autotune_clear": (None, []),
    "vis_set_operand_cache_limit": (None, [ctypes.c_longlong]),
    "vis_tensor_wait_test_hook": (c_int, [ctypes.c_longlong]),
    "vis_spectrum_copy_to_host": (c_int, [c_void_p, PConfig, c_void_p]),
    "vis_spectrum_render_views": (c_int, [c_void_p, PConfig, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "vis_config_enable_kernel_timing": (c_int, [PConfig, c_int]),
    "vis_config_kernel_timing": (c_int, [PConfig, c_int, POINTER(c_float), POINTER(c_int)]),
    "vis_kernel_launch_count": (ctypes.c_ulonglong, []),
    "vis_batch_create": (c_void_p, [PConfig]),
    "vis_batch_add": (c_int, [c_void_p, PDataset, int3, c_float, float2, int2, int2, c_int, c_void_p, c_void_p]),
    "vis_batch_execute": (c_int, [c_void_p, c_int]),
    "vis_batch_uses_graph": (c_int, [c_void_p]),
    "vis_batch_images": (c_void_p, [c_void_p, c_int]),
    "vis_batch_spectrum": (c_void_p, [c_void_p, c_int]),
    "vis_batch_copy_images_to_host": (c_int, [c_void_p, c_int, c_void_p]),
    "vis_batch_destroy": (None, [c_void_p]),
    "vis_images_normalize_to_rgb": (c_int, [PConfig, c_void_p, c_int, int2, c_void_p]),
    "vis_images_colormap": (c_int, [PConfig, c_void_p, c_int, int2, c_float, c_float, c_int, c_int, c_void_p]),
    "vis_write_ppm": (c_int, [c_char_p, c_void_p, int2]),
    "vis_shift_registered_dataset": (c_int, [PConfig, PDataset, c_float, c_float, c_float]),
    "vis_fourier_slice_sum_noalloc": (c_int, [c_void_p, c_void_p, c_int, c_int, float2, int2, float3, float3, int2,
                                              c_void_p, c_int, c_void_p]),
}

_lib = None


def load():
    """Loads libmeshless_vis.so once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m libmeshlessvis_b200.build` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH), mode=ctypes.RTLD_LOCAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class VisError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"libmeshless_vis error {code}: {message}")
        self.code = code


def check(lib, rc=None):
    """Raises VisError if the last call failed (rc != 0, or a recorded error)."""
    code = lib.vis_get_last_error() if rc is None else rc
    if code != 0:
        msg = lib.vis_get_last_error_message() or b""
        lib.vis_clear_last_error()
        raise VisError(code, msg.decode(errors="replace"))
