"""Beam masks, beam properties and multiplexing (MPXI) of a photoelectric sysmat.

The reference derives these after generation, on the CPU, from the .sysmat
file (PEGen_RayTracing_CircularHole/extract_beam_prop_masks.py:52-87,
compute_mpxi_3d.py:45-98).  Here the per-entry work runs on the GPU where the
sysmat lives (``sm_beam_metrics``, csrc/beam_kernel.cu); what is left on the
host is per row or per voxel:

* ``beam_metrics``: one rotation's block of rows on the device -> row max,
  row sum, mask size, the int8 beam masks (``entry > frac * row max``) and the
  MPXI counts;
* ``beam_properties``: the reference's 11-column beam property records of the
  active rows;
* ``mpxi_summary`` / ``mpxi_summary_text``: the reference's MPXI summary and
  its text file;
* ``sysmat_file_metrics`` (and ``python -m sysmat_b200.beams``): the whole
  pipeline for a .sysmat file, streamed through the GPU in row chunks, writing
  the masks, properties, MPXI volumes and summaries as .npy / .txt files (the
  reference writes HDF5 and PNGs; the arrays are the same).
"""
from __future__ import annotations

import argparse
import os
from typing import Optional, Sequence

import numpy as np

from . import _check, lib

DEFAULT_FRAC = 0.05


def beam_metrics(block, frac: float = DEFAULT_FRAC, keep_mask: bool = True, mpxi: bool = True, stream=None):
    """``block``: a CUDA float32 torch tensor [rows][voxels] (row stride may
    exceed voxels).  Returns a dict of CUDA tensors: ``row_max`` (float32),
    ``row_sum`` (float64), ``row_count`` (int32), ``mask`` (int8 [rows][voxels]
    or None) and ``mpxi`` (int32 [voxels], the uint32 counts, or None)."""
    import torch
    if block.dtype != torch.float32 or not block.is_cuda or block.dim() != 2 or block.stride(1) != 1:
        raise ValueError("block must be a 2-D CUDA float32 tensor with unit column stride")
    rows, vox = block.shape
    dev = block.device
    row_max = torch.empty(rows, dtype=torch.float32, device=dev)
    row_sum = torch.empty(rows, dtype=torch.float64, device=dev)
    row_count = torch.empty(rows, dtype=torch.int32, device=dev)
    mask = torch.empty((rows, vox), dtype=torch.int8, device=dev) if keep_mask else None
    counts = torch.empty(vox, dtype=torch.int32, device=dev) if mpxi else None
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    with torch.cuda.device(dev):
        _check(lib().sm_beam_metrics(block.data_ptr(), rows, vox, block.stride(0), float(frac), row_max.data_ptr(),
                                     row_sum.data_ptr(), row_count.data_ptr(),
                                     mask.data_ptr() if mask is not None else None, vox,
                                     counts.data_ptr() if counts is not None else None, s.cuda_stream))
    return {"row_max": row_max, "row_sum": row_sum, "row_count": row_count, "mask": mask, "mpxi": counts}


def beam_properties(rotation: int, n_rotations: int, row_sum: np.ndarray, row_count: np.ndarray,
                    first_row: int = 0) -> np.ndarray:
    """Property records (float32, 11 columns) of the rows whose mask is not
    empty, in row order: rotation, crystal, 1, rotation * 2 pi / n_rotations,
    8, mask size, 1, row sum, 0, 0, 0 (the record extract_beam_prop_masks.py
    writes; its constant columns are kept as it writes them)."""
    row_sum = np.asarray(row_sum)
    row_count = np.asarray(row_count)
    active = np.flatnonzero(row_count > 0)
    out = np.zeros((active.size, 11), dtype=np.float32)
    out[:, 0] = rotation
    out[:, 1] = first_row + active
    out[:, 2] = 1.0
    out[:, 3] = rotation * (2 * np.pi / n_rotations)
    out[:, 4] = 8.0
    out[:, 5] = row_count[active]
    out[:, 6] = 1.0
    out[:, 7] = row_sum[active].astype(np.float32)
    return out


def mpxi_summary(mpxi_3d: np.ndarray) -> dict:
    """Counts and moments of an MPXI volume, keyed as compute_mpxi_3d.py keys them."""
    vals = np.asarray(mpxi_3d).ravel()
    sampled = vals[vals > 0]
    levels, counts = np.unique(vals, return_counts=True)
    return {
        "shape": tuple(np.asarray(mpxi_3d).shape),
        "num_voxels_total": int(vals.size),
        "num_voxels_sampled": int(sampled.size),
        "num_voxels_unsampled": int(vals.size - sampled.size),
        "num_voxels_nonmultiplexed": int(np.count_nonzero(vals == 1)),
        "num_voxels_multiplexed": int(np.count_nonzero(vals > 1)),
        "max_mpxi": int(vals.max()) if vals.size else 0,
        "mean_mpxi_all_voxels": float(vals.mean()) if vals.size else 0.0,
        "mean_mpxi_sampled_voxels": float(sampled.mean()) if sampled.size else 0.0,
        "median_mpxi_sampled_voxels": float(np.median(sampled)) if sampled.size else 0.0,
        "histogram": list(zip(levels.tolist(), counts.tolist())),
    }


def mpxi_summary_text(summary: dict, rotation: int) -> str:
    """The summary file compute_mpxi_3d.py writes (same lines, same formats)."""
    lines = ["3D MPXI Summary | Rotation %d" % rotation, "=" * 60, "",
             "Volume shape: %s" % (summary["shape"],),
             "Total voxels: %d" % summary["num_voxels_total"],
             "Sampled voxels (MPXI > 0): %d" % summary["num_voxels_sampled"],
             "Unsampled voxels (MPXI = 0): %d" % summary["num_voxels_unsampled"],
             "Non-multiplexed voxels (MPXI = 1): %d" % summary["num_voxels_nonmultiplexed"],
             "Multiplexed voxels (MPXI > 1): %d" % summary["num_voxels_multiplexed"],
             "Max MPXI: %d" % summary["max_mpxi"],
             "Mean MPXI (all voxels): %.4f" % summary["mean_mpxi_all_voxels"],
             "Mean MPXI (sampled voxels): %.4f" % summary["mean_mpxi_sampled_voxels"],
             "Median MPXI (sampled voxels): %.4f" % summary["median_mpxi_sampled_voxels"], "",
             "Histogram (MPXI value -> voxel count)", "-" * 60]
    lines += ["%6d -> %d" % (v, c) for v, c in summary["histogram"]]
    return "\n".join(lines) + "\n"


def sysmat_file_metrics(path: str, n_rotations: int, n_crystals: int, grid: Sequence[int], out_dir: str,
                        frac: float = DEFAULT_FRAC, device: int = 0, chunk_bytes: int = 1 << 30,
                        write_masks: bool = True) -> dict:
    """Beam masks, properties and MPXI of a .sysmat file ([rotation][crystal][voxel]
    float32), streamed through the GPU in chunks of rows.  Writes into out_dir:
    beam_masks.npy (int8 [rotation * crystal][voxel], when write_masks),
    beam_properties.npy (float32 [active beams][11]), and per rotation
    mpxi_3d_rot_RRR.npy (uint32, shape (nz, ny, nx)) with
    mpxi_3d_rot_RRR_summary.txt."""
    import torch
    nx, ny, nz = (int(v) for v in grid)
    vox = nx * ny * nz
    data = np.memmap(path, dtype=np.float32, mode="r", shape=(n_rotations * n_crystals, vox))
    os.makedirs(out_dir, exist_ok=True)
    masks = (np.lib.format.open_memmap(os.path.join(out_dir, "beam_masks.npy"), mode="w+", dtype=np.int8,
                                       shape=(n_rotations * n_crystals, vox)) if write_masks else None)
    dev = torch.device("cuda", device)
    rows_per_chunk = max(1, min(n_crystals, chunk_bytes // (4 * vox)))
    staging = torch.empty((rows_per_chunk, vox), dtype=torch.float32, pin_memory=True)
    props, summaries = [], []
    for rot in range(n_rotations):
        total = torch.zeros(vox, dtype=torch.int64, device=dev)
        for r0 in range(0, n_crystals, rows_per_chunk):
            r1 = min(n_crystals, r0 + rows_per_chunk)
            g0 = rot * n_crystals
            staging[:r1 - r0].numpy()[:] = data[g0 + r0:g0 + r1]
            block = staging[:r1 - r0].to(dev)
            m = beam_metrics(block, frac=frac, keep_mask=write_masks)
            total += m["mpxi"].to(torch.int64)
            props.append(beam_properties(rot, n_rotations, m["row_sum"].cpu().numpy(), m["row_count"].cpu().numpy(),
                                         first_row=r0))
            if masks is not None:
                masks[g0 + r0:g0 + r1] = m["mask"].cpu().numpy()
        vol = total.cpu().numpy().astype(np.uint32).reshape(nz, ny, nx)
        s = mpxi_summary(vol)
        summaries.append(s)
        np.save(os.path.join(out_dir, "mpxi_3d_rot_%03d.npy" % rot), vol)
        with open(os.path.join(out_dir, "mpxi_3d_rot_%03d_summary.txt" % rot), "w") as f:
            f.write(mpxi_summary_text(s, rot))
    allprops = np.concatenate(props) if props else np.zeros((0, 11), np.float32)
    np.save(os.path.join(out_dir, "beam_properties.npy"), allprops)
    if masks is not None:
        masks.flush()
    return {"active_beams": int(allprops.shape[0]), "summaries": summaries}


def main(argv: Optional[Sequence[str]] = None) -> int:
    ap = argparse.ArgumentParser(description="Beam masks, properties and MPXI of a PE .sysmat file on the GPU.")
    ap.add_argument("sysmat")
    ap.add_argument("--rotations", type=int, required=True)
    ap.add_argument("--crystals", type=int, required=True)
    ap.add_argument("--grid", type=int, nargs=3, required=True, metavar=("NX", "NY", "NZ"))
    ap.add_argument("--frac", type=float, default=DEFAULT_FRAC)
    ap.add_argument("--outdir", default="beam_metrics")
    ap.add_argument("--cuda", type=int, default=0)
    ap.add_argument("--no-masks", action="store_true")
    a = ap.parse_args(argv)
    r = sysmat_file_metrics(a.sysmat, a.rotations, a.crystals, a.grid, a.outdir, a.frac, a.cuda,
                            write_masks=not a.no_masks)
    print("active beams: %d; MPXI max per rotation: %s" % (r["active_beams"], [s["max_mpxi"] for s in r["summaries"]]))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
