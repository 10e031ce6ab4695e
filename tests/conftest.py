import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


INT_KEYS = ("nz", "ny", "nx", "n_z_bed", "n_per_cell", "n_max", "n_alloc", "n_sub",
            "n_substeps", "drying_mode", "n_soil", "lambda_x", "n_iters")


class Vectors:
    """Access to the reference's golden kernel vectors (tests/golden/kernel_vectors.npz)."""

    def __init__(self, path):
        self.d = np.load(path)
        self.keys = self.d.files

    def cases(self, section):
        names = sorted({k.split("/")[1] for k in self.keys
                        if k.startswith(section + "/") and not k.split("/")[1].startswith("_")})
        return names

    def case(self, section, name):
        pre = f"{section}/{name}/"
        out = {}
        for k in self.keys:
            if k.startswith(pre):
                v = self.d[k]
                out[k[len(pre):]] = v.item() if v.ndim == 0 else v
        for k in INT_KEYS:
            if k in out:
                out[k] = int(out[k])
        return out


@pytest.fixture(scope="session")
def vectors():
    return Vectors(GOLDEN / "kernel_vectors.npz")


def load_ref(name):
    d = np.load(GOLDEN / name)
    out = {}
    for k in d.files:
        grp, key = k.split("/", 1)
        out.setdefault(grp, {})[key] = d[k]
    return out


@pytest.fixture(scope="session")
def ref_tiny():
    return load_ref("ref_tiny.npz")


@pytest.fixture(scope="session")
def ref_smoke():
    return load_ref("ref_smoke.npz")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    if den == 0.0:
        return num
    return num / den


def dom_s8_cases():
    """Cases of tests/golden/dom_s8.npz (reference DOM solves at S8, made by
    tests/golden/make_dom_s8.py): {case: (inputs, [outputs of solve 0, solve 1])}."""
    d = np.load(GOLDEN / "dom_s8.npz")
    out = {}
    for k in d.files:
        parts = k.split("/")
        case = out.setdefault(parts[0], ({}, [{}, {}]))
        v = d[k]
        v = v.item() if v.ndim == 0 else v
        if len(parts) == 2:
            case[0][parts[1]] = v
        else:
            case[1][int(parts[1][4:])][parts[2]] = v
    for inp, _ in out.values():
        for key in ("nz", "ny", "nx"):
            inp[key] = int(inp[key])
    return out

