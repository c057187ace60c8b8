"""CPU check of csrc/phi_series.h, the power series of the reference's
closed-form SPH and Wendland transforms (meshless_vis/fourier_transform.cu:
31-60) that the h-binned tensor form evaluates below each branch point: the
series equals the closed form (the oracle's FP64 formula) above the branch
point, where the closed form is accurate, and reproduces the known value at
r = 0 (the reference's quadratic fits start from the same constant)."""
import re
from pathlib import Path

import numpy as np

import oracle as O

HDR = Path(__file__).resolve().parents[1] / "libmeshlessvis_b200" / "csrc" / "phi_series.h"


def _coef(name):
    text = HDR.read_text()
    body = re.search(name + r"\[\d+\] = \{([^}]*)\}", text).group(1)
    return [float(x) for x in body.split(",")]


def _series(name, scale, r):
    c = _coef(name)
    m2 = (np.pi * np.asarray(r, np.float64)) ** 2
    acc = np.zeros_like(m2)
    for v in reversed(c):
        acc = acc * m2 + v
    return scale * acc


def test_series_match_the_closed_forms_above_the_branch_points():
    for name, scale, basis, r0 in (("MV_WENDLAND_SERIES", np.pi * 7.5, O.WENDLAND_D3_C2, 0.24),
                                   ("MV_SPH_SERIES", 2.3561944901923448, O.SPH, 0.06)):
        r = np.linspace(r0, 0.6, 200)
        closed = O.phi(basis, r)
        assert np.max(np.abs(_series(name, scale, r) - closed)) < 1e-12 * abs(closed[0])


def test_series_start_from_the_transform_at_zero():
    assert abs(_series("MV_WENDLAND_SERIES", np.pi * 7.5, [0.0])[0] - 0.299199300341890) < 1e-12
    assert abs(_series("MV_SPH_SERIES", 2.3561944901923448, [0.0])[0] - np.pi) < 1e-12
