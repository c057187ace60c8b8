#!/usr/bin/env python
"""Benchmark of the libMeshlessVis hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c3|c1|c2|c4|c5|...] [--form auto|plain|tensor]
                    [--no-compare-forms]

One step = one pass of the hot path over one particle set resident in HBM:
the 3D half-spectrum Fourier sum of every group, then slice extraction and
batched 2D C2R of all the workload's views.  Default workload: C3, the
precision-form configuration (N=2^20 uniform particles, w ~ U(0,1),
GAUSSIAN_DECAYING with h log-uniform in [0.005, 0.05] in 16 h-bins, 256x256x129
half-spectrum, one z-normal view at 256^2), with the spectrum sum also timed
alone in the tensor-core form and in the plain FP32 form (tc_vs_plain).

Prints one JSON line (rank 0).  value = particle x frequency terms per second
over the whole step (GTerms/s), device time by CUDA events on the library's
stream, max over ranks.  e2e = the same metric through the public C API with
host buffers: registration (H2D of the particles from pinned memory),
spectrum, views and D2H of the images, every step.

Multi-GPU: the path does not shard on one particle set here, so N GPUs run N
independent replicas (weak scaling); value sums all ranks' terms.
--impl reference times the reference's own CPU implementation
(oracle/_ref, built from the reference sources; the FP64 oracle's C code if
that is absent) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FP32_LANES_PER_SM = 128


STAGE_NAMES = {0: "plain_sum", 3: "tensor_sum", 1: "slice", 2: "fft"}
STAGES = tuple(STAGE_NAMES)


METRIC_SPECTRUM = "GTerms/s (particle x frequency terms per second; 3D half-spectrum sum + all views)"
METRIC_BATCH = "GTerms/s (particle x frequency terms per second; batch of 64 uneven sets + all views)"


def sum_terms_split(w):
    """Terms per step done by the tensor-core kernel if every group takes it,
    and by the plain form.  The planes l < Kz/2 go to the tensor cores, and so
    does the Nyquist plane l = Kz/2 (two transposed jobs in the same launch)
    when Kx/2 fills whole n-tile units (16 c for CTA pairs, else 8); otherwise
    the plain form sums it.  The rule is the library's tensor_plan."""
    kx, ky, kz = w["grid"]
    n = sum(len(c) for c, _, _ in w["groups"])
    lz_tc = kz // 2
    pairs = os.environ.get("MV_TC_PAIRS", "1")[:1] != "0"
    pair = pairs and lz_tc > 64 and lz_tc % 16 == 0 and (kx * ky) % 256 == 0
    nyq_tc = ky % 16 == 0 and (kx // 2) % (16 if pair else 8) == 0 and kx % 2 == 0
    plane = n * kx * ky
    return plane * (lz_tc + (1 if nyq_tc else 0)), (0 if nyq_tc else plane)


# DRAM bytes (read + write) per launch of the dominant kernel, from ncu
# captures of dram__bytes_read.sum + dram__bytes_write.sum of the full-size
# launch (profiles/tc_sum_kernel_c3_dram.md names the capture and its
# command); None where no capture exists.
DRAM_TRAFFIC_PER_LAUNCH = {("C3", "tc_sum_kernel"): 21.89e9 + 4.44e9}


def sum_roofline(stage_t, w, steps, peaks, peak_src, clk, sm_count):
    """Roofline of the dominant Fourier-sum kernel: 8 algorithmic flops per
    particle x frequency term over the kernel's own event-timed duration.  The
    tensor kernel runs back to back inside a long step, so its denominator is
    the sustained dense bf16 figure (the FP16 dense rate is the same)."""
    terms, n, g = terms_per_step(w)
    (p_ms, p_n), (t_ms, t_n) = stage_t[0], stage_t[3]
    max_mhz = clk.get("sm_max_mhz") or peaks.get("sm_max_mhz", 1965.0)
    if t_ms > p_ms and t_n > 0:
        tc_terms, _ = sum_terms_split(w)
        per_launch_terms = tc_terms * steps / t_n
        launch_s = t_ms / t_n / 1000.0
        alg = 8.0 * per_launch_terms / launch_s / 1e12
        issued = 24.0 * per_launch_terms / launch_s / 1e12
        peak = peaks.get("bf16_tflops_sustained", 1400.0)
        burst = peaks.get("bf16_tflops", 1590.0)
        return {"bound": "tensor", "achieved": alg, "peak": peak, "unit": "TFLOP/s", "frac": alg / peak,
                "traffic": DRAM_TRAFFIC_PER_LAUNCH.get((w["name"], "tc_sum_kernel")), "kernel": "tc_sum_kernel",
                "flops_per_term": 8,
                "issued_tflops": issued, "issued_frac": issued / peak, "issued_frac_of_burst": issued / burst,
                "issued_note": "3 FP16 products per term (hi*hi, hi*lo, lo*hi): 24 issued flops per term",
                "terms_per_launch": per_launch_terms, "launch_ms": t_ms / t_n, "launches": t_n,
                "peak_source": f"{peak_src} dense bf16 cuBLAS, sustained (the kernel runs back to back inside a "
                               f"long step; burst {burst})"}
    per_launch_terms = terms * steps / max(1, p_n)
    launch_s = p_ms / max(1, p_n) / 1000.0
    alg = 8.0 * per_launch_terms / launch_s / 1e12 if launch_s > 0 else 0.0
    peak = sm_count * FP32_LANES_PER_SM * 2 * max_mhz * 1e6 / 1e12
    r = {"bound": "fp32", "achieved": alg, "peak": peak, "unit": "TFLOP/s", "frac": alg / peak,
         "traffic": DRAM_TRAFFIC_PER_LAUNCH.get((w["name"], "fold_sum_kernel")),
         "kernel": "fold_sum_kernel", "flops_per_term": 8, "terms_per_launch": per_launch_terms,
         "launch_ms": p_ms / max(1, p_n), "launches": p_n,
         "peak_source": f"nominal FP32: {sm_count} SMs x {FP32_LANES_PER_SM} lanes x 2 flop x {max_mhz:.0f} MHz "
                        "(MEASURED_PEAKS.json has no FP32 figure)"}
    if clk.get("sm_mhz"):
        r["frac_at_sampled_clock"] = alg / (peak * clk["sm_mhz"] / max_mhz)
    return r


def max_over_ranks(x, dist, device):
    """Largest value of x over all ranks (the job's time is its slowest
    rank's); x itself when there is no process group."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank_step, steps, t_max_ms, world):
    """Whole-job throughput of `world` independent replicas, each processing
    units_per_rank_step per step, timed by the slowest rank."""
    return world * units_per_rank_step * steps / (t_max_ms / 1000.0)


def compare_forms(M, cfg, sp, ds, w, stream, flush, args, steps=2):
    """The spectrum sum alone, tensor form vs plain form, same inputs."""
    import torch

    terms, _, _ = terms_per_step(w)
    out = {}
    for name, form in (("tensor", M.FORM_TENSOR), ("plain", M.FORM_PLAIN)):
        sp.compute(cfg, ds, form)
        cfg.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        with torch.cuda.stream(stream):
            for k in range(steps):
                flush.zero_()
                ev[k][0].record(stream)
                sp.compute(cfg, ds, form)
                ev[k][1].record(stream)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        out[name] = {"ms_per_sum": ms, "gterms_per_s": terms / (ms / 1000.0) / 1e9}
    out["ratio"] = out["tensor"]["gterms_per_s"] / out["plain"]["gterms_per_s"]
    out["workload"] = w["name"]
    return out


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["c1", "c2", "c2s", "c3", "c3s", "c3w", "c4", "c5", "c5s"], default="c3",
                   help="c2s: C2's particle model at N=65,536 on a 64^3 lattice, 16 views; c3s: C3's model at "
                        "N=2^17, 128^3, 4 h-bins; c3w: the same on 256^3; c5s: C5's model at N=2^17 on its 384^3 "
                        "lattice, 8 views (profiling cases)")
    p.add_argument("--form", choices=["auto", "plain", "tensor"], default="auto")
    p.add_argument("--autotune", action="store_true",
                   help="run the library's autotuner (vis_autotune_spectrum) on the workload before the warm-up")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-compare-forms", dest="compare_forms", action="store_false",
                   help="skip timing the spectrum sum alone in the tensor and the plain form (tc_vs_plain; on by "
                        "default)")
    return p.parse_args()


def workload(name):
    from libmeshlessvis_b200 import workloads as W

    if name == "c1":
        return W.c1()
    if name == "c3":
        return W.c3()
    if name == "c5":
        # the first frame of the 8-frame series (every frame has the same shapes)
        return next(W.c5_frames())
    if name == "c3w":
        w = W.c3(n=1 << 17, grid=256, bins=4)
        w["name"] = "C3-wide-small"
        return w
    if name == "c3s":
        w = W.c3(n=1 << 17, grid=128, bins=4)
        w["name"] = "C3-small"
        return w
    if name == "c2s":
        w = W.c2(n=65536, grid=64, views=16)
        w["name"] = "C2-small"
        return w
    if name == "c5s":
        # C5's lattice and tile (384^3: CTA pairs with n-tiles of 96 + 96 c
        # values) and its particle model at N=2^17, for profiling
        w = next(W.c5_frames(n=1 << 17, frames=1))
        w["name"] = "C5-small"
        w["views"] = w["views"][:8]
        return w
    return W.c2()


def terms_per_step(w):
    kx, ky, kz = w["grid"]
    g = kx * ky * (kz // 2 + 1)
    n = sum(len(c) for c, _, _ in w["groups"])
    return n * g, n, g


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = [ln.split(", ") for ln in Path(self.f.name).read_text().splitlines() if ln.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) >= 9:
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower().startswith("active"):
                        reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text()), "measured"
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def reference_groups(groups):
    """The groups as the reference's fourier_transform can take them: it has
    no GAUSSIAN_DECAYING (an appended basis id it skips without work), so its
    own GAUSSIAN, with the same per-term work (one exponential), stands in."""
    from libmeshlessvis_b200 import meshless as M

    out, note = [], ""
    for cons, radii, basis in groups:
        if basis == M.GAUSSIAN_DECAYING:
            basis = M.GAUSSIAN
            note = " (GAUSSIAN_DECAYING groups timed with the reference's GAUSSIAN, the same per-term work)"
        out.append((cons, radii, basis))
    return out, note


# The reference's CPU loop hands out block_length frequencies at a time to its
# OpenMP threads (schedule(dynamic, block_length),
# meshless_vis/fourier_transform_cpu.cpp:85); 32 is its smallest supported
# block length (fourier_transform_cpu.cpp:159-163).
REF_BLOCK_LENGTH = 32
REF_MIN_CHUNKS_PER_THREAD = 4


def reference_sample(n, cores, target_terms=2e9):
    """The slice the reference's CPU path is timed on: all n particles over one
    z-normal slice of 2*c*c frequencies, c chosen so the sample holds about
    target_terms terms (at most c = 64) but never fewer than
    REF_MIN_CHUNKS_PER_THREAD chunks of REF_BLOCK_LENGTH frequencies for every
    host thread.  Returns (c, block_length)."""
    c_min = int(np.ceil((REF_MIN_CHUNKS_PER_THREAD * REF_BLOCK_LENGTH * max(1, cores) / 2.0) ** 0.5))
    c = int(max(4, min(64, (target_terms / (2.0 * max(1, n))) ** 0.5)))
    return max(c, c_min), REF_BLOCK_LENGTH


def reference_timer(groups, cores, target_terms=2e9):
    """(fn, terms, kind, sample text, close): one call of fn runs the
    reference's own fourier_transform (OpenMP, all host threads) over the
    sample of reference_sample; without oracle/_ref the FP64 oracle's C slice
    sum (kind "port") stands in."""
    import oracle as O

    n = sum(len(c) for c, _, _ in groups)
    c, bl = reference_sample(n, cores, target_terms)
    terms = n * 2 * c * c
    note = ""
    if O.ref_available():
        ref_groups, note = reference_groups(groups)
        R = O.RefRenderer(ref_groups, (1.0, 1.0), (c, c), (1, 0, 0), (0, 1, 0), (2 * c, 2 * c), block_length=bl)
        fn, close, kind = R.fourier_transform, R.close, "reference"
    else:
        def fn():
            for cons, radii, basis in groups:
                O.slice_sum(cons, radii, basis, (1.0, 1.0), (c, c), (1, 0, 0), (0, 1, 0))

        close, kind = (lambda: None), "port"
    chunks = 2 * c * c // bl
    sample = (f"the reference's fourier_transform (OpenMP, {cores} threads, block_length {bl}: {chunks} chunks, "
              f"{chunks / max(1, cores):.1f} per thread) over all {n} particles and one z-normal slice of "
              f"2*{c}*{c}={2 * c * c} frequencies ({terms:.3e} terms){note}")
    return fn, terms, kind, sample, close


def cpu_baseline(w, target_terms=2e9):
    """The reference's own fourier_transform on the workload's particles, one
    call over the reference_sample slice, timed on the host."""
    cores = len(os.sched_getaffinity(0))
    fn, terms, kind, sample, close = reference_timer(w["groups"], cores, target_terms)
    t0 = time.perf_counter()
    fn()
    dt = time.perf_counter() - t0
    close()
    return {"value": terms / dt / 1e9, "unit": "GTerms/s", "cores": cores, "kind": kind,
            "sample": f"{sample}, {dt:.2f} s"}


def accuracy_check(w, spec, images, n_points=1024, n_views=2):
    """Part of the CPU-baseline leg, with the oracle as the checker: the FP64
    direct sum at seeded half-spectrum points (the workload's own check points
    when it has them) against the spectrum of the timed run, and FP64 slice
    extraction + C2R of that spectrum against the first views' images."""
    import oracle as O

    kx, ky, kz = w["grid"]
    ijk = w.get("check_points")
    if ijk is None:
        prng = np.random.default_rng(1)
        ijk = np.stack([prng.integers(-kx // 2, kx // 2, n_points), prng.integers(-ky // 2, ky // 2, n_points),
                        prng.integers(0, kz // 2 + 1, n_points)], axis=1).astype(np.int32)
    t0 = time.perf_counter()
    ref = sum(O.spectrum_points(c, r, b, w["step3"], ijk) for c, r, b in w["groups"])
    got = spec[ijk[:, 0] + kx // 2, ijk[:, 1] + ky // 2, ijk[:, 2]]
    t_spec = time.perf_counter() - t0
    scale = float(np.max(np.abs(ref))) or 1.0
    out = {"spectrum": {"rel_l2": O.rel_l2(got, ref), "max_abs_over_max": O.max_abs(got, ref) / scale,
                        "points": int(len(ijk)), "tolerance": 1e-5, "oracle": "FP64 direct sum",
                        "seconds": round(t_spec, 2)}}
    nv = min(n_views, len(w["views"]))
    ref_img = O.render_from_spectrum(spec.astype(np.complex128), w["grid"], w["step3"], w["step"], w["cutoff"],
                                     w["views"][:nv], w["samples"])
    out["images"] = {"rel_l2": O.rel_l2(images[:nv], ref_img), "views": nv, "tolerance": 1e-4,
                     "oracle": "FP64 slice interpolation + C2R of the same spectrum"}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle as O
    from libmeshlessvis_b200 import workloads as W

    # the batch (C4): its largest set's particles stand in for the batch
    if args.workload == "c4":
        w = dict(max(W.c4(), key=lambda x: sum(len(c) for c, _, _ in x["groups"])), name="C4 (largest set)")
    else:
        w = workload(args.workload)
    groups = w["groups"]
    n = sum(len(c) for c, _, _ in groups)
    cores = len(os.sched_getaffinity(0))
    fn, terms, kind, sample, close = reference_timer(groups, cores)
    for _ in range(args.warmup):
        fn()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fn()
    dt = time.perf_counter() - t0
    close()
    value = terms * args.steps / dt / 1e9
    sample = f"per step, workload {w['name']}: {sample}"
    n_freq = terms // max(1, n)
    kx, ky, kz = w["grid"]
    # our arm's metric and workload keys; the reference's rate per term is
    # timed on one slice of the same particles (it cannot offset k_z)
    line = {"impl": "reference", "metric": METRIC_BATCH if args.workload == "c4" else METRIC_SPECTRUM, "value": value,
            "unit": "GTerms/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1000 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w["name"], "particles": n, "grid": [kx, ky, kz],
                       "half_spectrum": kx * ky * (kz // 2 + 1), "sample_frequencies": int(n_freq)},
            "cpu_baseline": {"value": value, "unit": "GTerms/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "GTerms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist:
            dist.barrier()

    def allmax(x):
        return max_over_ranks(x, dist, "cuda")

    from libmeshlessvis_b200 import meshless as M

    form = {"auto": M.FORM_AUTO, "plain": M.FORM_PLAIN, "tensor": M.FORM_TENSOR}[args.form]
    w = workload(args.workload)
    terms, n, g = terms_per_step(w)
    views = w["views"]
    nv = len(views)
    u = np.array([v[0] for v in views], np.float32)
    v = np.array([v[1] for v in views], np.float32)
    nx, ny = w["samples"]

    lib = M.lib()
    cfg = M.Config(step=w["step"], cutoff=w["cutoff"], samples=w["samples"], block_length=64)
    stream = torch.cuda.Stream()
    cfg.set_stream(stream.cuda_stream)
    ds = M.Dataset(w["groups"])
    cfg.register(ds)
    sp = M.Spectrum(w["grid"], w["step3"])
    d_images = torch.empty((nv, nx, ny), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def step():
        sp.compute(cfg, ds, form)
        sp.render_views(cfg, u, v, d_images=d_images.data_ptr(), to_host=False)

    tuned = None
    if args.autotune:
        # outside the timed region: times the candidates, keeps the best for this shape
        import ctypes

        best_ms = sp.autotune(cfg, ds, form)
        vals = [ctypes.c_int(), ctypes.c_int(), ctypes.c_int()]
        lib.vis_autotune_lookup(M.int3(*w["grid"]), n, len(w["groups"]), form, *[ctypes.byref(x) for x in vals])
        shapes = [ctypes.c_int(), ctypes.c_int()]
        lib.vis_autotune_lookup_shapes(M.int3(*w["grid"]), n, len(w["groups"]), form,
                                       *[ctypes.byref(x) for x in shapes])
        tuned = {"plain_waves": vals[0].value, "tensor_waves": vals[1].value, "tensor_flush_stages": vals[2].value,
                 "tile_shapes": shapes[0].value, "hbin_price": shapes[1].value, "best_sum_ms": best_ms}
    for _ in range(max(3, args.warmup)):
        step()
    cfg.synchronize()
    cfg.enable_timing(True)
    for st in STAGES:
        cfg.kernel_time(st)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = Clocks(torch.cuda.current_device())
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = lib.vis_kernel_launch_count()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = lib.vis_kernel_launch_count() - launches0
    clk = clocks.stop()
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    stage_t = {st: cfg.kernel_time(st) for st in STAGES}
    cfg.enable_timing(False)
    t_max = allmax(t_ms)
    value = replica_throughput(terms, args.steps, t_max, world) / 1e9
    check_inputs = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the timed run's outputs, for the oracle check below (outside the timed region)
        check_inputs = (sp.to_host(cfg), d_images[:2].cpu().numpy())
    views_per_s = replica_throughput(nv, args.steps, t_max, world)

    peaks, peak_src = measured_peaks()
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    roofline = sum_roofline(stage_t, w, args.steps, peaks, peak_src, clk, sm_count)
    comparison = None
    if args.compare_forms:
        comparison = compare_forms(M, cfg, sp, ds, w, stream, flush, args)
    # end to end through the public C API with host buffers
    e2e = None
    if not args.no_e2e:
        pinned = []
        groups = []
        h2d = 0
        for cons, radii, basis in w["groups"]:
            tc = torch.empty(len(cons) * 16, dtype=torch.uint8, pin_memory=True)
            pc = tc.numpy().view(cons.dtype)
            pc[:] = cons
            pinned.append(tc)
            h2d += pc.nbytes
            pr = None
            if radii is not None:
                tr = torch.empty(len(radii), dtype=torch.float32, pin_memory=True)
                pr = tr.numpy()
                pr[:] = radii
                pinned.append(tr)
                h2d += pr.nbytes
            groups.append((pc, pr, basis))
        ds2 = M.Dataset(groups)
        h_images = torch.empty((nv, nx, ny), dtype=torch.float32, pin_memory=True)
        d2h = h_images.numel() * 4

        def e2e_step():
            cfg.register(ds2)
            sp.compute(cfg, ds2, form)
            lib.vis_spectrum_render_views(sp.ptr, cfg.ptr, nv, u.ctypes.data, v.ctypes.data, None,
                                          h_images.data_ptr())
            cfg.unregister(ds2)

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(args.steps)]
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                e_ev[k][0].record(stream)
                e2e_step()
                e_ev[k][1].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        e_ms = allmax(sum(a.elapsed_time(b) for a, b in e_ev))
        e2e = {"value": world * terms * args.steps / (e_ms / 1000.0) / 1e9, "unit": "GTerms/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e_ms / args.steps,
               "wall_ms_per_step": wall * 1000 / args.steps}

    cpu = None
    accuracy = None
    if check_inputs is not None:
        cpu = cpu_baseline(w)
        accuracy = accuracy_check(w, *check_inputs)

    sp.close()
    cfg.unregister(ds)
    cfg.close()
    if rank == 0:
        line = {"metric": METRIC_SPECTRUM,
                "value": value, "unit": "GTerms/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, BASELINE config shapes)",
                "config": {"workload": w["name"], "particles": n, "grid": list(w["grid"]),
                           "half_spectrum": g, "views": nv, "image": [nx, ny], "form": args.form,
                           "l2": "flushed between timed steps (256 MB write outside the event pair)",
                           "parallelism": f"replicas x{world}", "autotune": tuned},
                "views_per_s": views_per_s,
                "stages_ms_per_step": {name: stage_t[st][0] / args.steps for st, name in STAGE_NAMES.items()},
                "roofline": roofline, "clocks": clk, "gpu_launches": int(launches),
                "peaks_source": peak_src}
        if e2e:
            line["e2e"] = e2e
        if cpu:
            line["cpu_baseline"] = cpu
        if accuracy:
            line["accuracy"] = accuracy
        if comparison:
            line["tc_vs_plain"] = comparison
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def batch_accuracy(sets, batch, picks, n_points=256, n_views=1):
    """The oracle as the checker of a batch run: for the picked jobs, the FP64
    direct sum at seeded half-spectrum points against the job's spectrum, and
    FP64 slice extraction + C2R of that spectrum against its first views."""
    import oracle as O

    prng = np.random.default_rng(1)
    got_all, ref_all, img_err = [], [], []
    t0 = time.perf_counter()
    for j in picks:
        w = sets[j]
        kx, ky, kz = w["grid"]
        ijk = np.stack([prng.integers(-kx // 2, kx // 2, n_points), prng.integers(-ky // 2, ky // 2, n_points),
                        prng.integers(0, kz // 2 + 1, n_points)], axis=1).astype(np.int32)
        spec = batch.spectrum(j)
        ref = sum(O.spectrum_points(c, r, b, w["step3"], ijk) for c, r, b in w["groups"])
        got_all.append(spec[ijk[:, 0] + kx // 2, ijk[:, 1] + ky // 2, ijk[:, 2]])
        ref_all.append(ref)
        imgs = batch.images(j)[:n_views]
        ref_img = O.render_from_spectrum(spec.astype(np.complex128), w["grid"], w["step3"], w["step"], w["cutoff"],
                                         w["views"][:n_views], w["samples"])
        img_err.append(O.rel_l2(imgs, ref_img))
    got, ref = np.concatenate(got_all), np.concatenate(ref_all)
    return {"spectrum": {"rel_l2": O.rel_l2(got, ref), "max_abs_over_max": O.max_abs(got, ref) / np.max(np.abs(ref)),
                         "points": int(len(got)), "jobs": [int(j) for j in picks], "tolerance": 1e-5,
                         "oracle": "FP64 direct sum", "seconds": round(time.perf_counter() - t0, 2)},
            "images": {"rel_l2": max(img_err), "views_per_job": n_views, "tolerance": 1e-4,
                       "oracle": "FP64 slice interpolation + C2R of the same spectrum (worst job)"}}


def run_batch(args):
    """C4: 64 particle sets of uneven size and lattice, 16 views each, as one
    batch (one CUDA graph per execute)."""
    import torch

    from libmeshlessvis_b200 import _lib as L
    from libmeshlessvis_b200 import meshless as M
    from libmeshlessvis_b200 import workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    form = {"auto": M.FORM_AUTO, "plain": M.FORM_PLAIN, "tensor": M.FORM_TENSOR}[args.form]
    sets = W.c4()
    lib = M.lib()
    cfg = M.Config(block_length=64)
    stream = torch.cuda.Stream()
    cfg.set_stream(stream.cuda_stream)
    terms = 0
    tc_terms = 0
    n_total = 0
    n_views = 0
    datasets = []
    batch = M.Batch(cfg)

    def add_all(b, dss):
        for ds, w in zip(dss, sets):
            b.add(ds, w["grid"], w["step3"], w["step"], w["cutoff"], w["samples"], [v[0] for v in w["views"]],
                  [v[1] for v in w["views"]])

    for w in sets:
        w["name"] = "C4-set"
        ds = M.Dataset(w["groups"])
        cfg.register(ds)
        datasets.append(ds)
        t, n, g = terms_per_step(w)
        terms += t
        tc_terms += sum_terms_split(w)[0]
        n_total += n
        n_views += len(w["views"])
    add_all(batch, datasets)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(max(3, args.warmup)):
        batch.execute(form)
    cfg.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = Clocks(torch.cuda.current_device())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = lib.vis_kernel_launch_count()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            batch.execute(form)
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches_host = lib.vis_kernel_launch_count() - launches0
    clk = clocks.stop()
    t_max = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), dist, "cuda")
    value = replica_throughput(terms, args.steps, t_max, world) / 1e9
    uses_graph = batch.uses_graph()
    # kernels per execute, counted on a direct (non-graph) run: graph replays
    # launch the same nodes without passing through the library's host code
    per_exec = launches_host / max(1, args.steps)
    if uses_graph == 1:
        probe = M.Batch(cfg)
        add_all(probe, datasets)
        c0 = lib.vis_kernel_launch_count()
        probe.execute(form)  # builds: one direct run + one capture of the same sequence
        per_exec = (lib.vis_kernel_launch_count() - c0) / 2
        probe.close()
    accuracy = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the largest, the smallest and two middle sets (outside the timed region)
        order = np.argsort([sum(len(c) for c, _, _ in w["groups"]) for w in sets])
        picks = sorted({int(order[-1]), int(order[0]), int(order[len(order) // 2]), int(order[len(order) // 4])})
        accuracy = batch_accuracy(sets, batch, picks)
    # end to end: every step registers all sets from pinned host memory,
    # executes the batch, copies every job's images to the host and unregisters
    e2e = None
    if not args.no_e2e:
        groups_h, pinned, h2d = [], [], 0
        for w in sets:
            gs = []
            for cons, radii, basis in w["groups"]:
                tc = torch.empty(len(cons) * 16, dtype=torch.uint8, pin_memory=True)
                pc = tc.numpy().view(cons.dtype)
                pc[:] = cons
                tr = torch.empty(len(radii), dtype=torch.float32, pin_memory=True)
                pr = tr.numpy()
                pr[:] = radii
                pinned += [tc, tr]
                h2d += pc.nbytes + pr.nbytes
                gs.append((pc, pr, basis))
            groups_h.append(gs)
        h_imgs = [torch.empty((len(w["views"]),) + tuple(w["samples"]), dtype=torch.float32, pin_memory=True)
                  for w in sets]
        d2h = sum(t.numel() * 4 for t in h_imgs)
        ds2 = [M.Dataset(gs) for gs in groups_h]
        b2 = M.Batch(cfg)
        add_all(b2, ds2)

        def e2e_step():
            for d in ds2:
                cfg.register(d)
            b2.execute(form)
            for j, t in enumerate(h_imgs):
                L.check(lib, lib.vis_batch_copy_images_to_host(b2.ptr, j, t.data_ptr()))
            for d in ds2:
                cfg.unregister(d)

        e2e_step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(args.steps)]
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                e_ev[k][0].record(stream)
                e2e_step()
                e_ev[k][1].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        e_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in e_ev), dist, "cuda")
        e2e = {"value": world * terms * args.steps / (e_ms / 1000.0) / 1e9, "unit": "GTerms/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e_ms / args.steps,
               "wall_ms_per_step": wall * 1000 / args.steps, "cuda_graph": b2.uses_graph()}
        b2.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        big = max(sets, key=lambda x: sum(len(c) for c, _, _ in x["groups"]))
        cpu = cpu_baseline(big)
        cpu["sample"] = "largest set of the batch: " + cpu["sample"]
    batch.close()
    for ds in datasets:
        cfg.unregister(ds)
    cfg.close()
    if rank == 0:
        peaks, peak_src = measured_peaks()
        # the batch runs as one CUDA graph, whose launches the library's stage
        # timer cannot see: the step time bounds the tensor kernel's time
        alg = 8.0 * tc_terms * args.steps / (t_max / 1000.0) / 1e12
        peak = peaks.get("bf16_tflops_sustained", 1400.0)
        roofline = {"bound": "tensor", "achieved": alg, "peak": peak, "unit": "TFLOP/s", "frac": alg / peak,
                    "traffic": None, "kernel": "tc_sum_kernel", "flops_per_term": 8,
                    "issued_tflops": 3 * alg, "issued_frac": 3 * alg / peak,
                    "timing": "whole-step CUDA-event time (graph replay: every kernel of the step included), so "
                              "achieved is a lower bound for the tensor kernel",
                    "peak_source": f"{peak_src} dense bf16 cuBLAS, sustained"}
        line = {"metric": METRIC_BATCH,
                "value": value, "unit": "GTerms/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, BASELINE config shapes)",
                "config": {"workload": "C4", "sets": len(sets), "particles": n_total, "views": n_views,
                           "form": args.form, "cuda_graph": uses_graph,
                           "l2": "flushed between timed steps (256 MB write outside the event pair)",
                           "parallelism": f"replicas x{world}"},
                "views_per_s": replica_throughput(n_views, args.steps, t_max, world),
                "roofline": roofline, "clocks": clk, "gpu_launches": int(round(per_exec * args.steps)),
                "peaks_source": peak_src}
        if e2e:
            line["e2e"] = e2e
        if cpu:
            line["cpu_baseline"] = cpu
        if accuracy:
            line["accuracy"] = accuracy
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c4":
        run_batch(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
