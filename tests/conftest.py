import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


class Golden:
    """Fixtures written by tests/golden/make_golden.py from the reference implementation."""

    def __init__(self):
        self.small = np.load(os.path.join(GOLDEN, "tables_small.npz"))
        self.hashes = json.load(open(os.path.join(GOLDEN, "tables_hash.json")))
        self.sponge = np.load(os.path.join(GOLDEN, "sponge.npz"))
        self.units = json.load(open(os.path.join(GOLDEN, "units.json")))
        self.vessels = np.load(os.path.join(GOLDEN, "vessels.npz"))

    def small_names(self):
        return sorted({k.split("/")[0] for k in self.small.files})

    def small_case(self, name):
        meta = json.loads(str(self.small[name + "/meta"]))
        arrays = {k: self.small[f"{name}/{k}"] for k in ("phi", "nbr", "q", "uin", "coords")}
        return meta, arrays

    def vessel(self, case):
        """The reference's packed centrelines of `case` (vessel._packed), its bounds and its openings."""
        v = {k: self.vessels[f"{case}/{k}"] for k in ("pts", "rad", "start", "count", "cap_p", "cap_n", "cap_r",
                                                       "lo", "hi")}
        v["meta"] = json.loads(str(self.vessels[f"{case}/meta"]))
        return v


@pytest.fixture(scope="session")
def golden():
    return Golden()
