"""CPU tests of bench.py's output contract that need no GPU: the reference
arm (the reference's own CPU path, single process) reports the same metric
and workload keys as the GPU arm, with its CPU baseline and end-to-end
figures; and the split of a step's terms between the tensor-core launch and
the plain form follows the library's planning rule."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _reference_line(workload):
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", workload, "--steps", "1",
           "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=str(ROOT), env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    return json.loads(lines[0])


def test_reference_arm_reports_the_gpu_arms_metric_and_workload():
    d = _reference_line("c1")
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC_SPECTRUM and d["unit"] == "GTerms/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"] == "C1" and d["config"]["grid"] == [64, 64, 64]
    assert d["config"]["half_spectrum"] == 64 * 64 * 33
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == "GTerms/s" and cb["cores"] >= 1
    assert cb["kind"] in ("reference", "port") and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GTerms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_for_the_batch_uses_the_batch_metric():
    d = _reference_line("c4")
    assert d["metric"] == bench.METRIC_BATCH
    assert d["config"]["workload"].startswith("C4")
    assert d["value"] > 0


def _w(grid, n=10):
    cons = np.zeros((n, 4), np.float32)
    return {"grid": grid, "groups": [(cons, None, 0)]}


def test_term_split_follows_the_tensor_plan():
    # 256^3: CTA pairs, Kx/2 = 128 splits into 16-c units -> the Nyquist plane is on the tensor cores
    tc, plain = bench.sum_terms_split(_w((256, 256, 256)))
    assert tc == 10 * 256 * 256 * 129 and plain == 0
    # 384^3 (C5): also
    tc, plain = bench.sum_terms_split(_w((384, 384, 384)))
    assert tc == 10 * 384 * 384 * 193 and plain == 0
    # Kx/2 = 20 is no multiple of 16 on CTA pairs: the Nyquist plane stays plain
    tc, plain = bench.sum_terms_split(_w((40, 256, 160)))
    assert tc == 10 * 40 * 256 * 80 and plain == 10 * 40 * 256


def test_reference_sample_gives_every_thread_four_chunks():
    """The reference's loop hands out block_length frequencies at a time
    (schedule(dynamic, block_length), fourier_transform_cpu.cpp:85); the timed
    slice gives every host thread at least four such chunks, so no core idles
    and the reference arm and the GPU arm's cpu_baseline time the same sample."""
    for cores in (1, 2, 8, 16, 64, 192):
        for n in (4096, 262144, 1 << 20, 1 << 24):
            c, bl = bench.reference_sample(n, cores)
            assert bl == bench.REF_BLOCK_LENGTH == 32
            assert (2 * c * c) // bl >= 4 * cores
            assert c >= 4
    # C3 on a 16-thread host: one 64x32 slice (2048 frequencies, 64 chunks)
    assert bench.reference_sample(1 << 20, 16) == (32, 32)
