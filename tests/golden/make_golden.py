"""Generates tests/golden/golden.npz.

Run here (where the reference sources and oracle/_ref exist):
    make -C oracle && python tests/golden/make_golden.py

Each case stores its seeded inputs and
  * ref_slice / ref_image: outputs of the reference's own CPU renderer
    (meshless_vis/fourier_transform_cpu.cpp + meshless_vis_cpu.cpp, compiled
    verbatim into oracle/_ref; C2R by the project's FP64 FFTW shim) driven
    through its C API: vis_config_create, vis_register_meshless_dataset,
    fourier_transform / vis_fourier_volume_rendering, vis_copy_to_host;
  * fp64_slice / fp64_image: the FP64 oracle (oracle/oracle.c) on the same
    inputs.
Spectrum cases (no reference twin) store the FP64 oracle's 3D half-spectrum
and view images only.
The GPU tests read this file; nothing at test time needs the reference.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle as O  # noqa: E402
from libmeshlessvis_b200.workloads import constraints, rotating_views  # noqa: E402

OUT = Path(__file__).resolve().parent / "golden.npz"


def direct_cases():
    rng = np.random.default_rng(20081)
    cases = []

    def add(name, groups, step, cutoff, u, v, samples):
        cases.append(dict(name=name, groups=groups, step=step, cutoff=cutoff, u=u, v=v, samples=samples))

    n = 600  # not a multiple of any tile size (ragged)
    for basis, h in [(O.SPH, 0.05), (O.GAUSSIAN, 0.02), (O.WENDLAND_D3_C2, 0.03)]:
        pos = rng.random((n, 3), dtype=np.float32)
        w = rng.standard_normal(n).astype(np.float32)
        r = np.exp(rng.uniform(np.log(h / 2), np.log(2 * h), n)).astype(np.float32)
        add(f"b{basis}_xy", [(constraints(pos, w), r, basis)], (1.0, 1.0), (16, 16), (1, 0, 0), (0, 1, 0), (32, 32))
        u, v = rotating_views(7)[3]
        add(f"b{basis}_rot", [(constraints(pos, w), r, basis)], (1.0, 1.0), (16, 8), u, v, (48, 32))
        # no radii: Phi^ at |f| itself; step 0.05 keeps the reference's growing
        # Gaussian finite, positions in [0, 20) keep the phases large
        add(f"b{basis}_noradii", [(constraints(pos * 20, w), None, basis)], (0.05, 0.05), (16, 16), (1, 0, 0),
            (0, 1, 0), (32, 32))
    # two groups, different bases, step 0.1 on shifted positions (the headless
    # renderer shifts by -5, vis_noninteractive/main.cpp:46)
    p1 = rng.random((300, 3), dtype=np.float32) * 10 - 5
    p2 = rng.random((200, 3), dtype=np.float32) * 10 - 5
    g1 = (constraints(p1, rng.random(300, dtype=np.float32)), np.full(300, 0.4, np.float32), O.SPH)
    g2 = (constraints(p2, rng.random(200, dtype=np.float32)), np.full(200, 0.6, np.float32), O.WENDLAND_D3_C2)
    add("two_groups_step01", [g1, g2], (0.1, 0.1), (16, 16), (1, 0, 0), (0, 1, 0), (64, 64))
    # vis_timing_test workload (vis_timing_test/main.cpp:72-78): all particles
    # at the origin, weight 1, radius 1e-5, SPH; factor=1 drops the radii.
    z = constraints(np.zeros((1024, 3), np.float32), np.ones(1024, np.float32))
    add("timing_test_radii", [(z, np.full(1024, 1e-5, np.float32), O.SPH)], (1.0, 1.0), (16, 16), (1, 0, 0),
        (0, 1, 0), (32, 32))
    add("timing_test_factor1", [(z, None, O.SPH)], (1.0, 1.0), (16, 16), (1, 0, 0), (0, 1, 0), (32, 32))
    # single particle (KAT-2)
    one = constraints(np.array([[0.3, 0.6, 0.2]], np.float32), np.array([2.0], np.float32))
    add("single_particle", [(one, np.array([0.05], np.float32), O.WENDLAND_D3_C2)], (1.0, 1.0), (16, 16),
        (1, 0, 0), (0, 1, 0), (32, 32))
    return cases


def spectrum_cases():
    rng = np.random.default_rng(20082)
    cases = []
    n = 700
    for basis in (O.SPH, O.GAUSSIAN, O.WENDLAND_D3_C2, O.GAUSSIAN_DECAYING):
        pos = rng.random((n, 3), dtype=np.float32)
        w = rng.standard_normal(n).astype(np.float32)
        r = np.exp(rng.uniform(np.log(0.01), np.log(0.05), n)).astype(np.float32)
        cases.append(dict(name=f"spec_b{basis}", groups=[(constraints(pos, w), r, basis)], grid=(16, 12, 10),
                          step3=1.0, step=(1.0, 1.0), cutoff=(8, 6), samples=(16, 12),
                          views=[((1, 0, 0), (0, 1, 0))] + rotating_views(5)))
    pos = rng.random((n, 3), dtype=np.float32)
    cases.append(dict(name="spec_noradii_step05", groups=[(constraints(pos, rng.random(n, dtype=np.float32)), None,
                                                           O.GAUSSIAN_DECAYING)],
                      grid=(16, 16, 16), step3=0.5, step=(0.5, 0.5), cutoff=(8, 8), samples=(16, 16),
                      views=rotating_views(4)))
    return cases


def pack_groups(prefix, groups, store):
    store[prefix + "ngroups"] = np.array(len(groups))
    for gi, (cons, radii, basis) in enumerate(groups):
        store[f"{prefix}g{gi}_xyzw"] = O._xyzw(cons)
        store[f"{prefix}g{gi}_basis"] = np.array(basis)
        if radii is not None:
            store[f"{prefix}g{gi}_radii"] = np.asarray(radii, np.float32)


def main():
    store = {}
    names = []
    for c in direct_cases():
        p = c["name"] + "/"
        names.append(c["name"])
        pack_groups(p, c["groups"], store)
        for k in ("step", "cutoff", "u", "v", "samples"):
            store[p + k] = np.array(c[k])
        store[p + "kind"] = np.array("direct")
        R = O.RefRenderer(c["groups"], c["step"], c["cutoff"], c["u"], c["v"], c["samples"])
        R.fourier_transform()
        store[p + "ref_slice"] = R.slice()
        store[p + "ref_image"] = R.render()
        R.close()
        cx, cy = c["cutoff"]
        sl = np.zeros(2 * cx * cy, dtype=np.complex128)
        for cons, radii, basis in c["groups"]:
            O.slice_sum(cons, radii, basis, c["step"], c["cutoff"], c["u"], c["v"], out=sl)
        store[p + "fp64_slice"] = sl
        store[p + "fp64_image"] = O.c2r(O.arrange(sl, c["cutoff"], c["samples"]), c["samples"])
        print(c["name"], "ref vs fp64 slice rel-L2 %.2e" % O.rel_l2(store[p + "ref_slice"], sl))
    for c in spectrum_cases():
        p = c["name"] + "/"
        names.append(c["name"])
        pack_groups(p, c["groups"], store)
        for k in ("grid", "step3", "step", "cutoff", "samples"):
            store[p + k] = np.array(c[k])
        store[p + "views"] = np.array(c["views"], dtype=np.float64)
        store[p + "kind"] = np.array("spectrum")
        spec = O.spectrum_grid(c["groups"], c["step3"], c["grid"])
        store[p + "fp64_spectrum"] = spec
        store[p + "fp64_images"] = O.render_from_spectrum(spec, c["grid"], c["step3"], c["step"], c["cutoff"],
                                                          c["views"], c["samples"])
        print(c["name"], "spectrum", spec.shape)
    store["cases"] = np.array(names)
    np.savez_compressed(OUT, **store)
    print("wrote", OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
