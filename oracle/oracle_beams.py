"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the reference's beam
post-processing, the checker of sm_beam_metrics and sysmat_b200.beams.

* ``beam_rows`` follows PEGen_RayTracing_CircularHole/extract_beam_prop_masks.py:52-87:
  per (rotation, crystal) row of a float32 sysmat, mx = max, threshold =
  0.05 * mx in single precision (numpy keeps a float32 scalar times a Python
  float in float32), 1.0 for mx <= 0; mask = row > threshold (int8); the beam
  properties row [r, d, 1.0, r * 2 pi / n_rot, 8.0, mask size, 1.0, row sum,
  0, 0, 0] for rows whose mask is not empty.
* ``mpxi`` follows compute_mpxi_3d.py:45-52: the rotation's masks summed over
  crystals (uint32), one count per voxel.
* ``summarize`` and ``summary_text`` follow compute_mpxi_3d.py:55-98.

Pinned by tests/golden/beams_reference.npz (the reference's own scripts run
on a synthetic sysmat) and tests/golden/mpxi_shipped_rot000.npz (the MPXI
volume and summary the reference ships).
"""
from __future__ import annotations

import numpy as np


def beam_rows(block: np.ndarray, frac: float = 0.05):
    """(row max, row sum (float32, numpy's), mask int8) of a [rows][voxels] float32 block."""
    block = np.asarray(block, dtype=np.float32)
    mx = block.max(axis=1)
    thr = np.where(mx > 0, np.float32(frac) * mx, np.float32(1.0)).astype(np.float32)
    mask = (block > thr[:, None]).astype(np.int8)
    sums = np.array([np.sum(row) for row in block], dtype=np.float32)
    return mx, sums, mask


def properties(rotation: int, n_rotations: int, sums: np.ndarray, counts: np.ndarray, first_row: int = 0):
    """Beam property rows (float32, 11 columns) of the active rows, in row order."""
    out = []
    angle = rotation * (2 * np.pi / n_rotations)
    for i in range(len(counts)):
        if counts[i] > 0:
            out.append([float(rotation), float(first_row + i), 1.0, angle, 8.0, float(counts[i]), 1.0,
                        float(sums[i]), 0.0, 0.0, 0.0])
    return np.asarray(out, dtype=np.float32).reshape(-1, 11)


def mpxi(mask: np.ndarray) -> np.ndarray:
    return np.sum(mask, axis=0, dtype=np.uint32)


def summarize(mpxi_3d: np.ndarray) -> dict:
    vals = mpxi_3d.ravel()
    nonzero = vals[vals > 0]
    s = {
        "shape": tuple(mpxi_3d.shape),
        "num_voxels_total": int(vals.size),
        "num_voxels_sampled": int(np.sum(vals > 0)),
        "num_voxels_unsampled": int(np.sum(vals == 0)),
        "num_voxels_nonmultiplexed": int(np.sum(vals == 1)),
        "num_voxels_multiplexed": int(np.sum(vals > 1)),
        "max_mpxi": int(np.max(vals)),
        "mean_mpxi_all_voxels": float(np.mean(vals)),
        "mean_mpxi_sampled_voxels": float(np.mean(nonzero)) if nonzero.size > 0 else 0.0,
        "median_mpxi_sampled_voxels": float(np.median(nonzero)) if nonzero.size > 0 else 0.0,
    }
    u, c = np.unique(vals, return_counts=True)
    s["histogram"] = list(zip(u.tolist(), c.tolist()))
    return s
