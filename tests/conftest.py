import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a) and the built library")


def load_golden():
    z = np.load(GOLDEN)
    cases = {}
    for name in z["cases"]:
        name = str(name)
        p = name + "/"
        d = {k[len(p):]: z[k] for k in z.files if k.startswith(p)}
        groups = []
        for gi in range(int(d["ngroups"])):
            xyzw = d[f"g{gi}_xyzw"]
            radii = d.get(f"g{gi}_radii")
            groups.append((xyzw, radii, int(d[f"g{gi}_basis"])))
        d["groups"] = groups
        d["kind"] = str(d["kind"])
        cases[name] = d
    return cases


@pytest.fixture(scope="session")
def golden():
    return load_golden()
