"""Shared helpers for the tests (loading golden fixtures, error statistics)."""
import os

import numpy as np

from sysmat_b200.params import Params

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_pe_golden(name: str):
    z = np.load(os.path.join(GOLDEN, "pe_%s.npz" % name))
    col = np.zeros(max(80000, z["collimator"].size), np.float32)
    col[:z["collimator"].size] = z["collimator"]
    det = np.zeros(max(80000, z["detector"].size), np.float32)
    det[:z["detector"].size] = z["detector"]
    p = Params(col, det, z["image"].astype(np.float32), z["physics"].astype(np.float32),
               tuple(int(v) for v in z["sv"]), tuple(int(v) for v in z["sc"]), name)
    return p, z


def rel_err(a, b, floor=0.0):
    """|a - b| / |b| on entries where b != 0 (b is the reference)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nz = np.abs(b) > floor
    if not nz.any():
        return np.zeros(0)
    return np.abs(a[nz] - b[nz]) / np.abs(b[nz])


def load_scatter_golden(name: str):
    """Params and arrays of tests/golden/scatter_<name>.npz."""
    z = np.load(os.path.join(GOLDEN, "scatter_%s.npz" % name))
    col = np.zeros(max(80000, z["collimator"].size), np.float32)
    col[:z["collimator"].size] = z["collimator"]
    det = np.zeros(max(80000, z["detector"].size), np.float32)
    det[:z["detector"].size] = z["detector"]
    p = Params(col, det, z["image"].astype(np.float32), z["physics"].astype(np.float32), (1, 1, 1), (2, 4, 2),
               "scatter_" + name)
    return p, z
