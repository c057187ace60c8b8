"""The reference's own application, compiled unchanged against this library.

vis_timing_test/main.cpp (reference) includes only meshless_vis.h and drives
vis_config_create, vis_config_check, get_simple_meshless_dataset,
vis_register_meshless_dataset, vis_fourier_volume_rendering (number_of_runs
times), vis_unregister_meshless_dataset, vis_config_destroy and
delete_meshless_dataset (main.cpp:63-88).  tests/apps/Makefile compiles it from
the reference's sources with include/ and links libmeshless_vis.so, plus a
probe that prints vis_get_last_error() at exit.

CPU: the binary exists, links this library, and its usage path runs.
GPU: it runs the reference's call sequence with radii (factor 0) and without
(factor 1), exits 0 and leaves no library error.
"""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
APP = ROOT / "tests" / "apps" / "_bin" / "vis_timing_test"
LIB = ROOT / "libmeshlessvis_b200" / "libmeshless_vis.so"


def _need_app():
    if not APP.exists():
        pytest.skip("tests/apps/_bin/vis_timing_test not built (the reference sources were absent at build time)")


def test_reference_timing_app_links_this_library_and_runs_its_usage_path():
    _need_app()
    ldd = subprocess.run(["ldd", str(APP)], capture_output=True, text=True, timeout=60).stdout
    line = [ln for ln in ldd.splitlines() if "libmeshless_vis.so" in ln]
    assert line and Path(line[0].split("=>")[1].split("(")[0].strip()).resolve() == LIB.resolve()
    r = subprocess.run([str(APP)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    assert "vis_timing_test number_of_runs number_of_terms" in r.stdout
    assert "vis_get_last_error=0" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("factor", [0, 1])
def test_reference_timing_app_runs_on_the_gpu(factor):
    _need_app()
    args = ["2", "4096", "32", "256", "64", str(factor), "1"]
    r = subprocess.run([str(APP), *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Valid Configuration" in r.stdout
    assert "finished running tests" in r.stdout
    assert "vis_get_last_error=0" in r.stdout, r.stdout
