"""Helpers shared by the tests (paths are set up by conftest.py)."""
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def relerr(a, b):
    dt = np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64
    a = np.asarray(a, dt).ravel()
    b = np.asarray(b, dt).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))
