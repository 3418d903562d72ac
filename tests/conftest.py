import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the device path")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def load_golden(name):
    """A golden fixture (tests/golden/make_golden.py) as (System, dict)."""
    from agbnp3_b200.system import System
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    s = System(x=d["x"], y=d["y"], z=d["z"], r=d["r"], charge=d["charge"], igamma=d["igamma"],
               sgamma=d["sgamma"], ialpha=d["ialpha"], salpha=d["salpha"], hbtype=d["hbtype"].astype(np.int32),
               hbcorr=d["hbcorr"], ihydrogen=d["ihydrogen"].astype(np.int32), bonds=d["bonds"].astype(np.int32),
               eps_in=float(d["eps"][0]), eps_out=float(d["eps"][1]))
    return s, d


GOLDEN_CASES = ["globule50", "globule300_shuffled", "globule2000_hbmix"]
ENERGY_KEYS = ("egb", "evdw", "ecorr_vdw", "ecav", "ecorr_cav", "ehb", "mol_volume")


def rms_rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    den = np.sqrt((b ** 2).sum())
    return float(np.sqrt(((a - b) ** 2).sum()) / den) if den > 0 else float(np.abs(a - b).max())
