"""CPU tests of the C-ABI boundary: the library loads, exports every function
include/*.h declares, its struct layouts match what a C compiler computes from
the headers, and its host-only entry points (data model, .sph I/O, errors)
behave like the reference's.  No GPU compute runs here."""
import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from libmeshlessvis_b200 import _lib as L
from libmeshlessvis_b200 import meshless as M
from libmeshlessvis_b200.workloads import constraints

ROOT = Path(__file__).resolve().parents[1]
HEADERS = sorted((ROOT / "include").glob("*.h"))
DECL = re.compile(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for line in text.splitlines():
            s = line.strip()
            if s.startswith(("#", "typedef", "enum", "struct", "}", "{")) or "(" not in s:
                continue
            m = DECL.match(s)
            if m:
                names.add(m.group(1))
    return names


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_library_loads_and_exports_every_declared_function():
    lib = L.load()
    decl = declared_functions()
    assert len(decl) >= 40, decl
    missing = decl - exported_symbols()
    assert not missing, f"declared in include/*.h but not exported: {sorted(missing)}"
    for name in decl:
        assert hasattr(lib, name)
    # the ctypes table covers the whole ABI
    assert decl == set(L.SIGNATURES), (decl ^ set(L.SIGNATURES))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_struct_layouts_match_c_compiler(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stddef.h>
#include <stdio.h>
#include "meshless_vis_b200.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m))
int main(void) {
  printf("Constraint %zu\nGroup %zu\nMeshlessDataset %zu\nVisConfig %zu\n", sizeof(Constraint), sizeof(Group),
         sizeof(MeshlessDataset), sizeof(VisConfig));
  F(Group, basis_function_id); F(Group, h_constraints); F(Group, d_radii);
  F(VisConfig, u_axis); F(VisConfig, cull_fully_aliased_terms); F(VisConfig, _plan);
  F(VisConfig, _number_of_samples); F(VisConfig, block_length); F(VisConfig, _d_image);
  F(VisConfig, _number_of_partial_sums); F(VisConfig, _d_freq_image_arranged);
  return 0;
}''')
    exe = tmp_path / "layout"
    subprocess.run(["/usr/bin/gcc", "-std=c11", "-I", str(ROOT / "include"), "-I", "/usr/local/cuda/include",
                    str(src), "-o", str(exe)], check=True)
    got = dict(ln.rsplit(" ", 1) for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    assert int(got["Constraint"]) == 16 == L.CONSTRAINT_DTYPE.itemsize
    assert int(got["Group"]) == ctypes.sizeof(L.Group)
    assert int(got["MeshlessDataset"]) == ctypes.sizeof(L.MeshlessDataset)
    assert int(got["VisConfig"]) == ctypes.sizeof(L.VisConfig)
    for key, val in got.items():
        if "." in key:
            t, m = key.split(".")
            assert getattr(getattr(L, t), m).offset == int(val), key


def test_simple_dataset_ownership_and_counts():
    rng = np.random.default_rng(0)
    c = constraints(rng.random((10, 3)), rng.random(10))
    ds = M.get_simple_meshless_dataset(10, c, np.full(10, 0.1, np.float32), M.WENDLAND_D3_C2)
    assert ds.number_of_groups == 1
    g = ds.groups[0]
    assert g.number_of_terms == 10 and g.basis_function_id == M.WENDLAND_D3_C2
    assert M.get_number_of_terms(ds) == 10
    M.shift_meshless_dataset(ds, -5.0, 1.0, 0.5)
    got = np.ctypeslib.as_array(ctypes.cast(g.h_constraints, ctypes.POINTER(ctypes.c_float)), (10, 4))
    np.testing.assert_allclose(got[:, 0], c["position"][:, 0] - 5.0, rtol=1e-6)
    np.testing.assert_allclose(got[:, 2], c["position"][:, 2] + 0.5, rtol=1e-6)
    M.delete_meshless_dataset(ds)


def test_sph_file_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    c1 = constraints(rng.random((7, 3)) * 10 - 5, rng.standard_normal(7))
    c2 = constraints(rng.random((3, 3)), rng.random(3))
    d = M.Dataset([(c1, np.linspace(0.1, 0.7, 7).astype(np.float32), M.SPH),
                   (c2, np.full(3, 0.2, np.float32), M.GAUSSIAN_DECAYING)])
    f = tmp_path / "set.sph"
    M.save_meshless_datasets_to_file(f, ctypes.byref(d.ds), 1)
    text = f.read_text().split()
    assert text[:3] == ["1", "2", "7"] and text[3] == "sph"
    sets, n = M.load_meshless_datasets_from_file(f)
    assert n == 1
    ds = sets[0]
    assert ds.number_of_groups == 2
    g0, g1 = ds.groups[0], ds.groups[1]
    assert (g0.number_of_terms, g0.basis_function_id) == (7, M.SPH)
    assert (g1.number_of_terms, g1.basis_function_id) == (3, M.GAUSSIAN_DECAYING)
    pos = np.ctypeslib.as_array(ctypes.cast(g0.h_constraints, ctypes.POINTER(ctypes.c_float)), (7, 4))
    np.testing.assert_array_equal(pos[:, :3], c1["position"])
    np.testing.assert_array_equal(pos[:, 3], c1["weight"])
    rad = np.ctypeslib.as_array(ctypes.cast(g1.h_radii, ctypes.POINTER(ctypes.c_float)), (3,))
    np.testing.assert_array_equal(rad, np.full(3, 0.2, np.float32))
    M.delete_meshless_datasets(sets, n)


def test_load_of_missing_file_gives_no_datasets(tmp_path):
    sets, n = M.load_meshless_datasets_from_file(tmp_path / "nope.sph")
    assert n == 0 and not sets


def test_error_strings_and_null_arguments_do_not_crash():
    lib = L.load()
    lib.vis_clear_last_error()
    assert lib.vis_get_last_error() == 0
    assert lib.vis_get_error_string(0) == b"success"
    assert b"invalid" in lib.vis_get_error_string(1)
    # NULL config: recorded as invalid value, no exception, no exit()
    assert lib.vis_config_check(None) is False
    assert lib.vis_get_last_error() == 1
    lib.vis_clear_last_error()
    lib.vis_fourier_volume_rendering(None, None)
    assert lib.vis_get_last_error() == 1
    lib.vis_clear_last_error()
    assert lib.vis_spectrum_compute(None, None, None, 0) == 1
    assert lib.vis_spectrum_create(L.int3(3, 4, 4), 1.0) is None  # odd extent
    assert lib.vis_get_last_error() == 1
    lib.vis_clear_last_error()


def test_opengl_entry_point_reports_unsupported():
    lib = L.load()
    lib.vis_clear_last_error()
    lib.vis_opengl_fourier_volume_rendering(None, None, 1)
    assert lib.vis_get_last_error() == 7
    lib.vis_clear_last_error()


def test_write_ppm_layout_and_flip(tmp_path):
    lib = L.load()
    w, h = 4, 3
    rgb = np.zeros((h, w, 3), np.float32)
    rgb[0, :, 0] = 1.0    # first row red
    rgb[2, 1, 2] = 0.5    # last row, second pixel half blue
    f = tmp_path / "img.ppm"
    assert lib.vis_write_ppm(str(f).encode(), rgb.ctypes.data, L.int2(w, h)) == 0
    data = f.read_bytes()
    header = b"P6\n4 3\n255\n"
    assert data.startswith(header)
    px = np.frombuffer(data[len(header):], np.uint8).reshape(h, w, 3)
    # vertical flip, as the reference's JPEG writer (vis_noninteractive/main.cpp:31)
    assert (px[2, :, 0] == 255).all() and px[0, 1, 2] == 128


def test_autotune_table_starts_with_the_defaults():
    """Without a tuning run, every shape reports the default launch parameters
    (plain split-K 6 blocks per SM, tensor splits 4 waves, 16-stage chains
    in the single-accumulator tiles)."""
    lib = L.load()
    lib.vis_autotune_clear()
    vals = [ctypes.c_int(), ctypes.c_int(), ctypes.c_int()]
    tuned = lib.vis_autotune_lookup(L.int3(64, 64, 64), 4096, 2, 0, *[ctypes.byref(v) for v in vals])
    assert tuned == 0
    assert [v.value for v in vals] == [6, 4, 16]
    shapes = [ctypes.c_int(), ctypes.c_int()]
    assert lib.vis_autotune_lookup_shapes(L.int3(64, 64, 64), 4096, 2, 0, *[ctypes.byref(v) for v in shapes]) == 0
    assert [v.value for v in shapes] == [L.TILE_ALL, 1024]


def test_autotune_store_records_a_set_and_refuses_values_outside_the_candidates():
    """vis_autotune_store puts a parameter set in the table (host only, no
    GPU): both lookups return it; a value outside its candidate set is refused
    with VIS_ERROR_INVALID_VALUE and leaves the entry as it was."""
    lib = L.load()
    lib.vis_autotune_clear()
    shape = (L.int3(96, 64, 32), 12345, 3, 2)
    shapes_off = L.TILE_ALL & ~L.TILE_AXIS_EXCHANGE
    assert lib.vis_autotune_store(*shape, 4, 8, 8, shapes_off, 256) == 0
    vals = [ctypes.c_int() for _ in range(5)]
    assert lib.vis_autotune_lookup(*shape, *[ctypes.byref(v) for v in vals[:3]]) == 1
    assert lib.vis_autotune_lookup_shapes(*shape, *[ctypes.byref(v) for v in vals[3:]]) == 1
    assert [v.value for v in vals] == [4, 8, 8, shapes_off, 256]
    for bad in [(3, 8, 8, 0, 256), (4, 16, 8, 0, 256), (4, 8, 32, 0, 256), (4, 8, 8, 16, 256), (4, 8, 8, -1, 256),
                (4, 8, 8, 0, 0)]:
        assert lib.vis_autotune_store(*shape, *bad) == 1
    assert lib.vis_autotune_store(shape[0], 12345, 3, 7, 4, 8, 8, 0, 256) == 1  # unknown form
    assert lib.vis_autotune_lookup_shapes(*shape, *[ctypes.byref(v) for v in vals[3:]]) == 1
    assert [v.value for v in vals[3:]] == [shapes_off, 256]
    lib.vis_autotune_clear()
    assert lib.vis_autotune_lookup_shapes(*shape, None, None) == 0


def test_operand_cache_limit_setter_takes_every_form():
    """The operand-cache limit is a process-wide setting that needs no GPU to
    set: a byte count, 0 (off), and None / negative (the default)."""
    M.set_operand_cache_limit(0)
    M.set_operand_cache_limit(3 << 30)
    M.set_operand_cache_limit(None)
    L.load().vis_set_operand_cache_limit(-5)
    M.set_operand_cache_limit(None)
