"""Helpers shared by the tests: convert (xyzw, radii, basis) groups into the
library's Dataset, and run the product through its C API."""
import numpy as np

from libmeshlessvis_b200.meshless import Config, Dataset, Spectrum
from libmeshlessvis_b200.workloads import constraints


def to_dataset(groups):
    gs = []
    for cons, radii, basis in groups:
        if getattr(cons, "dtype", None) is None or cons.dtype.names is None:
            a = np.asarray(cons, np.float32).reshape(-1, 4)
            cons = constraints(a[:, :3], a[:, 3])
        gs.append((cons, radii, basis))
    return Dataset(gs)


def render_direct(groups, step, cutoff, u, v, samples, block_length=64, partial_sums=1):
    cfg = Config(step=tuple(step), cutoff=tuple(int(c) for c in cutoff), u=tuple(u), v=tuple(v),
                 samples=tuple(int(s) for s in samples), block_length=block_length, partial_sums=partial_sums)
    ds = to_dataset(groups)
    cfg.register(ds)
    cfg.render(ds)
    img = cfg.image()
    cfg.unregister(ds)
    cfg.close()
    return img


def spectrum_and_views(groups, grid, step3, step, cutoff, samples, views, form=0):
    cfg = Config(step=tuple(step), cutoff=tuple(int(c) for c in cutoff), samples=tuple(int(s) for s in samples),
                 block_length=64)
    ds = to_dataset(groups)
    cfg.register(ds)
    sp = Spectrum(tuple(int(g) for g in grid), float(step3))
    sp.compute(cfg, ds, form)
    spec = sp.to_host(cfg)
    imgs = None
    if views is not None and len(views):
        u = np.array([vv[0] for vv in views], np.float32)
        v = np.array([vv[1] for vv in views], np.float32)
        imgs = sp.render_views(cfg, u, v)
    sp.close()
    cfg.unregister(ds)
    cfg.close()
    return spec, imgs
