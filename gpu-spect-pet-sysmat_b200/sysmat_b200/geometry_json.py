"""Geometry front-end: JSON -> Params_*.dat tables, read-back verification,
and the geometry sanity report, as library calls and as a command line.

Replaces the reference's stand-alone scripts
``PEGen_RayTracing_CircularHole/json_to_dat.py:166-313`` (the annotated JSON
schema of ``geometry.annotated.json``, the four float32 tables, ``--verify``
read-back) and ``check_geometry_sanity.py:13-165`` (FOV / plate / hole /
detector statistics and warnings).  Differences:

* the tables also pass the library's own validation (``sm_tables_check``:
  counts against lengths, sizes > 0, capacities), which the reference tools
  never run;
* ``params_to_json`` writes the schema from a :class:`Params`, so the seeded
  workloads of :mod:`sysmat_b200.configs` round-trip through JSON.

Schema and table layout are the reference's (a file format, kept as it is):
collimator ``layers[]`` with ``hole_count``, ``width_mm``, ``thickness_mm``,
``height_mm``, ``offset_from_layer0_mm``, ``mu_total``, ``mu_pe``,
``mu_compton`` and ``holes[]`` (``cx``, ``cy1``, ``cy2``, ``cz``, ``radius``,
``mu_total``, ``mu_pe``, ``mu_compton``, ``flag``); detector ``bins[]``
(``cx``, ``cy``, ``cz``, ``width_mm``, ``thickness_mm``, ``height_mm``,
``mu_total``, ``mu_pe``, ``mu_compton``, ``energy_resolution_at_target``,
``rotation_about_y_rad``, ``flag``); image and physics scalars.  Keys starting
with ``_comment`` are ignored.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np

from .params import Params

F32 = np.dtype("<f4")

IMAGE_KEYS = ("num_voxel_x", "num_voxel_y", "num_voxel_z", "voxel_size_x_mm", "voxel_size_y_mm", "voxel_size_z_mm",
              "num_rotation", "angle_per_rotation_rad", "shift_fov_x_mm", "shift_fov_y_mm", "shift_fov_z_mm",
              "fov_to_collimator0_mm")
IMAGE_INT = {0, 1, 2, 6}
PHYSICS_KEYS = ("use_compton", "save_pe_sysmat", "save_compton_sysmat", "save_pecompton_sysmat",
                "use_same_energy_window", "energy_window_lower", "energy_window_upper", "target_pe_energy",
                "calc_crystal_geometry_relationship", "calc_collimator_geometry_relationship")
LAYER_KEYS = ("hole_count", "width_mm", "thickness_mm", "height_mm", "offset_from_layer0_mm", "mu_total", "mu_pe",
              "mu_compton")
HOLE_KEYS = ("cx", "cy1", "cy2", "cz", "radius", "mu_total", "mu_pe", "mu_compton", "flag")
BIN_KEYS = ("cx", "cy", "cz", "width_mm", "thickness_mm", "height_mm", "mu_total", "mu_pe", "mu_compton",
            "energy_resolution_at_target", "rotation_about_y_rad", "flag")


class GeometryJsonError(ValueError):
    """A JSON geometry that cannot be converted; the message names the field."""


def _field(d: Dict[str, Any], key: str, where: str) -> Any:
    if key not in d:
        raise GeometryJsonError("Missing key '%s' in %s" % (key, where))
    return d[key]


def _number(x: Any, where: str, integer: bool = False) -> float:
    try:
        return float(int(x)) if integer else float(x)
    except Exception:
        raise GeometryJsonError("Expected %s at %s, got: %r" % ("an int" if integer else "a number", where, x))


def _record(d: Dict[str, Any], keys: Sequence[str], where: str, ints=()) -> List[float]:
    if not isinstance(d, dict):
        raise GeometryJsonError("%s must be an object" % where)
    return [_number(_field(d, k, where), "%s.%s" % (where, k), integer=i in ints) for i, k in enumerate(keys)]


def _collimator_table(col: Dict[str, Any], layer_base: int, holes_base: int) -> np.ndarray:
    layers = _field(col, "layers", "collimator")
    if not isinstance(layers, list) or not layers:
        raise GeometryJsonError("collimator.layers must be a non-empty list")
    if layer_base < 0 or holes_base < 0 or holes_base < layer_base:
        raise GeometryJsonError("need 0 <= layer_base <= holes_base")
    # hole lists first (counts, list types), then the layer records, then the holes
    flat = []
    for li, layer in enumerate(layers):
        where = "collimator.layers[%d]" % li
        count = int(_number(_field(layer, "hole_count", where), where + ".hole_count", integer=True))
        holes = _field(layer, "holes", where)
        if not isinstance(holes, list):
            raise GeometryJsonError("%s.holes must be a list" % where)
        if len(holes) != count:
            raise GeometryJsonError("%s: hole_count=%d but holes has %d entries" % (where, count, len(holes)))
        for hi, h in enumerate(holes):
            if not isinstance(h, dict):
                raise GeometryJsonError("%s.holes[%d] must be an object" % (where, hi))
        flat += holes
    records = [_record(layer, LAYER_KEYS, "collimator.layers[%d]" % li, ints=(0,)) for li, layer in enumerate(layers)]
    holes = [_record(h, HOLE_KEYS, "collimator.holes_flat[%d]" % i) for i, h in enumerate(flat)]
    out = np.zeros(max(layer_base + 10 * len(layers), holes_base + 9 * len(holes), 1), dtype=F32)
    out[0] = len(layers)
    for li, rec in enumerate(records):
        out[layer_base + 10 * li: layer_base + 10 * li + 8] = rec
    if holes:
        out[holes_base: holes_base + 9 * len(holes)] = np.asarray(holes, dtype=F32).ravel()
    return out


def _detector_table(det: Dict[str, Any]) -> np.ndarray:
    bins = _field(det, "bins", "detector")
    if not isinstance(bins, list) or not bins:
        raise GeometryJsonError("detector.bins must be a non-empty list")
    out = np.zeros(1 + 12 * len(bins), dtype=F32)
    out[0] = len(bins)
    out[1:] = np.asarray([_record(b, BIN_KEYS, "detector.bins[%d]" % i) for i, b in enumerate(bins)], dtype=F32).ravel()
    return out


def tables_from_json(cfg: Dict[str, Any], layer_base: int = 10,
                     holes_base: int = 100) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(collimator, detector, image, physics) float32 tables of a JSON geometry,
    sized as json_to_dat.py sizes them (image 12, physics 10, detector 1 + 12 N,
    collimator up to its last layer or hole record).  Fields are checked in the
    order json_to_dat.py checks them, so the first fault reported is the same."""
    col, det = _field(cfg, "collimator", "root"), _field(cfg, "detector", "root")
    img, phy = _field(cfg, "image", "root"), _field(cfg, "physics", "root")
    collimator = _collimator_table(col, layer_base, holes_base)
    detector = _detector_table(det)
    image = np.asarray(_record(img, IMAGE_KEYS, "image", IMAGE_INT), dtype=F32)
    physics = np.asarray(_record(phy, PHYSICS_KEYS, "physics"), dtype=F32)
    return collimator, detector, image, physics


def load_json(path: str) -> Dict[str, Any]:
    with open(path, "r", encoding="utf-8") as f:
        return json.load(f)


def params_from_json(cfg_or_path, sv=(1, 1, 1), sc=(8, 16, 8)) -> Params:
    """A :class:`Params` (tables padded to the reference's 80000 / 100 floats)."""
    cfg = load_json(cfg_or_path) if isinstance(cfg_or_path, str) else cfg_or_path
    col, det, img, phy = tables_from_json(cfg)
    pad = lambda a, n: np.concatenate([a, np.zeros(max(0, n - a.size), F32)]).astype(np.float32)  # noqa: E731
    return Params(pad(col, 80000), pad(det, 80000), pad(img, 100), pad(phy, 100), tuple(sv), tuple(sc), "json")


def params_to_json(p: Params) -> Dict[str, Any]:
    """The JSON schema of a Params (inverse of tables_from_json up to float32 rounding)."""
    col, det, img, phy = p.collimator, p.detector, p.image, p.physics
    layers, hole = [], 0
    for l in range(p.n_plates):
        rec = col[(l + 1) * 10:(l + 1) * 10 + 8]
        nh = int(rec[0])
        holes = [dict(zip(HOLE_KEYS, (float(v) for v in col[100 + 9 * h:109 + 9 * h]))) for h in range(hole, hole + nh)]
        hole += nh
        layer = {k: float(v) for k, v in zip(LAYER_KEYS, rec)}
        layer["hole_count"] = nh
        layer["holes"] = holes
        layers.append(layer)
    bins = [dict(zip(BIN_KEYS, (float(v) for v in det[1 + 12 * d:13 + 12 * d]))) for d in range(p.n_crystals)]
    image = {k: (int(img[i]) if i in IMAGE_INT else float(img[i])) for i, k in enumerate(IMAGE_KEYS)}
    physics = {k: float(phy[i]) for i, k in enumerate(PHYSICS_KEYS)}
    return {"collimator": {"layers": layers}, "detector": {"bins": bins}, "image": image, "physics": physics}


def write_dat_files(cfg: Dict[str, Any], outdir: str, prefix: str = "Param", layer_base: int = 10,
                    holes_base: int = 100) -> Dict[str, np.ndarray]:
    """Writes <prefix>_{Collimator,Detector,Image,Physics}.dat.  The reference's
    converter writes the prefix "Param"; its generators read "Params"."""
    tables = dict(zip(("Collimator", "Detector", "Image", "Physics"), tables_from_json(cfg, layer_base, holes_base)))
    os.makedirs(outdir, exist_ok=True)
    for name, arr in tables.items():
        arr.astype(F32).tofile(os.path.join(outdir, "%s_%s.dat" % (prefix, name)))
    return tables


def read_dat_files(outdir: str, prefix: str = "Param") -> Dict[str, np.ndarray]:
    return {name: np.fromfile(os.path.join(outdir, "%s_%s.dat" % (prefix, name)), dtype=F32)
            for name in ("Collimator", "Detector", "Image", "Physics")}


def verify_dat_files(outdir: str, prefix: str = "Param", layer_base: int = 10, holes_base: int = 100) -> Dict[str, Any]:
    """Reads the four files back and validates them with the library
    (sm_tables_check).  Returns what --verify prints."""
    from . import SysmatError, tables_check
    t = read_dat_files(outdir, prefix)
    col = t["Collimator"]
    out = {"image": t["Image"][:12].tolist(), "physics": t["Physics"][:10].tolist(),
           "detector_floats": int(t["Detector"].size), "crystals": float(t["Detector"][0]),
           "collimator_floats": int(col.size), "layers": float(col[0]) if col.size else 0.0,
           "layer0": col[layer_base:layer_base + 8].tolist() if col.size >= layer_base + 8 else None,
           "first_hole": col[holes_base:holes_base + 9].tolist() if col.size >= holes_base + 9 else None}
    try:
        out["check"] = tables_check(col, t["Detector"], t["Image"], t["Physics"])
        out["valid"] = True
    except SysmatError as e:
        out["check"] = str(e)
        out["valid"] = False
    return out


# ---------------------------------------------------------------------------
# Geometry sanity report (check_geometry_sanity.py:13-165)
# ---------------------------------------------------------------------------

def sanity_report(collimator, detector, image, max_holes: int = 5) -> Dict[str, Any]:
    """The statistics check_geometry_sanity.py prints, as a dict.  Its
    conventions are kept: plate 0 assumed at y in [0, thickness], FOV centre at
    y = -FOV2Collimator0 + shift_y, layer-0 holes only."""
    col = np.asarray(collimator, dtype=np.float32)
    det = np.asarray(detector, dtype=np.float32)
    img = np.asarray(image, dtype=np.float32)
    r: Dict[str, Any] = {"warnings": []}
    nx, ny, nz = (int(v) for v in img[0:3])
    vx, vy, vz = img[3:6]
    size = np.array([nx * vx, ny * vy, nz * vz], dtype=float)
    centre = np.array([img[8], -img[11] + img[9], img[10]], dtype=float)
    r["image"] = {"grid": (nx, ny, nz), "voxel": (vx, vy, vz), "fov_size": size, "shift": tuple(img[8:11]),
                  "fov2collimator0": img[11], "fov_center": centre, "fov_min": centre - 0.5 * size,
                  "fov_max": centre + 0.5 * size, "rotations": int(img[6]), "angle_per_rotation": img[7]}
    layers = int(round(float(col[0])))
    if layers < 1:
        raise GeometryJsonError("No collimator layers found.")
    l0 = col[10:15]
    n_holes = int(round(float(l0[0])))
    plate_th = float(l0[2])
    r["layer0"] = {"layers": layers, "holes": n_holes, "width_x": float(l0[1]), "thickness_y": plate_th,
                   "height_z": float(l0[3]), "distance": float(l0[4])}
    holes = []
    for h in range(n_holes):
        off = 100 + 9 * h
        if off + 8 >= col.size:
            r["warnings"].append("col file too short for hole %d (off=%d)." % (h, off))
            break
        holes.append([float(v) for v in col[off:off + 5]])
    holes = np.array(holes, dtype=float).reshape(-1, 5)
    r["holes"] = holes
    n_det = int(round(float(det[0])))
    if 1 + 12 * n_det > det.size:
        raise GeometryJsonError("Detector file length mismatch: det_len=%d floats but expects >= %d"
                                % (det.size, 1 + 12 * n_det))
    D = det[1:1 + 12 * n_det].reshape(n_det, 12)
    xyz = D[:, 0:3]
    y = xyz[:, 1]
    uy, cy = np.unique(np.round(y, 2), return_counts=True)
    top = np.argsort(cy)[::-1][:10]
    r["detector"] = {"count": n_det, "center_min": xyz.min(axis=0), "center_max": xyz.max(axis=0),
                     "sizes": np.unique(np.round(D[:, 3:6], 6), axis=0), "y": y,
                     "y_planes": [(float(uy[i]), int(cy[i])) for i in top],
                     "in_plate": int(np.logical_and(y >= 0.0 - 1e-6, y <= plate_th + 1e-6).sum()),
                     "in_front": int((y < 0.0).sum())}
    fmin, fmax = r["image"]["fov_min"][1], r["image"]["fov_max"][1]
    if fmax > 0:
        r["warnings"].append("FOV extends into +Y (behind/into plate region). That is usually wrong.")
    if fmax > 0 and fmin < 0:
        r["warnings"].append("FOV straddles y=0 (overlaps plate). Likely wrong.")
    r["fov_in_front"] = bool(fmax <= 0)
    return r


def sanity_text(r: Dict[str, Any], max_holes: int = 5) -> str:
    """The report as check_geometry_sanity.py prints it, line for line up to
    its closing hints about the paper's dataset (not repeated here).  Scalars
    read from the float32 tables are formatted as Python formats a numpy
    float32 ("{}".format), which is not str()."""
    im, l0, d, holes = r["image"], r["layer0"], r["detector"], r["holes"]
    nx, ny, nz = im["grid"]
    vx, vy, vz = im["voxel"]
    sx, sy, sz = im["shift"]
    out = ["=== Param_Image ===",
           "voxels (nx,ny,nz)=({},{},{})  voxel_size=({},{},{}) mm".format(nx, ny, nz, vx, vy, vz),
           "FOV size (mm) = %s" % im["fov_size"].tolist(), "shift = ({},{},{}) mm".format(sx, sy, sz),
           "FOV2Collimator0 = {} mm".format(im["fov2collimator0"]), "FOV center (x,y,z) = %s" % im["fov_center"].tolist(),
           "FOV bbox min = %s" % im["fov_min"].tolist(), "FOV bbox max = %s" % im["fov_max"].tolist(),
           "numRotation={}  anglePerRotation={}".format(im["rotations"], im["angle_per_rotation"]),
           "", "=== Param_Collimator ===", "numLayers = %d" % l0["layers"],
           "Layer0: numHoles=%d  widthX=%smm  thickY=%smm  heightZ=%smm  dist=%smm"
           % (l0["holes"], l0["width_x"], l0["thickness_y"], l0["height_z"], l0["distance"])]
    out += ["WARNING: %s" % w for w in r["warnings"] if w.startswith("col file")]
    if holes.size > 0:
        xz = holes[:, [0, 3]]
        out += ["Holes parsed = %d" % holes.shape[0],
                "Hole radius stats (mm): min=%.4f max=%.4f mean=%.4f" % (holes[:, 4].min(), holes[:, 4].max(),
                                                                          holes[:, 4].mean()),
                "Hole y1/y2 unique-ish: y1(min,max)=(%.3f,%.3f)  y2(min,max)=(%.3f,%.3f)"
                % (holes[:, 1].min(), holes[:, 1].max(), holes[:, 2].min(), holes[:, 2].max()),
                "Hole center bbox X: [%.3f, %.3f]  Z: [%.3f, %.3f]" % (xz[:, 0].min(), xz[:, 0].max(), xz[:, 1].min(),
                                                                      xz[:, 1].max()),
                "", "Sample holes (x,y1,y2,z,r):"]
        out += ["  %d: %s" % (i, holes[i].tolist()) for i in range(min(max_holes, holes.shape[0]))]
    out += ["", "=== Param_Detector ===", "numDet = %d" % d["count"],
            "Detector center bbox min = %s" % d["center_min"].tolist(),
            "Detector center bbox max = %s" % d["center_max"].tolist(),
            "Detector center span     = %s" % (d["center_max"] - d["center_min"]).tolist(),
            "Unique detector sizes (widthX,thickY,heightZ) count=%d:" % len(d["sizes"])]
    out += ["  %s" % s.tolist() for s in d["sizes"]]
    y = d["y"]
    out += ["Detector Y stats: min=%.3f max=%.3f mean=%.3f" % (y.min(), y.max(), y.mean()), "",
            "Top Y-planes (rounded to 0.01mm):"]
    out += ["  y=%.2f  count=%d" % (v, c) for v, c in d["y_planes"]]
    th = l0["thickness_y"]
    fmin, fmax = im["fov_min"][1], im["fov_max"][1]
    out += ["", "Detectors with center y in plate thickness [0, %s]: %d" % (th, d["in_plate"]),
            "Detectors with center y < 0 (in front of plate): %d" % d["in_front"], "", "=== FOV vs Plate sanity ===",
            "Plate assumed at y in [0, %s]" % th, "FOV bbox y-range = [%.3f, %.3f]" % (fmin, fmax)]
    out += ["WARNING: %s" % w for w in r["warnings"] if w.startswith("FOV")]
    if r["fov_in_front"]:
        out.append("OK: FOV entirely in front of plate (y<=0).")
    return "\n".join(out) + "\n"


def main(argv: Optional[Sequence[str]] = None) -> int:
    ap = argparse.ArgumentParser(description="Convert an annotated geometry JSON into float32 <prefix>_*.dat tables.")
    ap.add_argument("json_path")
    ap.add_argument("--outdir", default=".")
    ap.add_argument("--collimator-layer-base", type=int, default=10)
    ap.add_argument("--collimator-holes-base", type=int, default=100)
    ap.add_argument("--prefix", default="Param", help="file prefix (the generators read 'Params')")
    ap.add_argument("--print-summary", action="store_true")
    ap.add_argument("--verify", action="store_true", help="read back, validate with the library, print key fields")
    ap.add_argument("--sanity", action="store_true", help="print the geometry sanity report")
    a = ap.parse_args(argv)
    try:
        cfg = load_json(a.json_path)
        t = write_dat_files(cfg, a.outdir, a.prefix, a.collimator_layer_base, a.collimator_holes_base)
    except GeometryJsonError as e:
        print("ERROR: %s" % e, file=sys.stderr)
        return 1
    if a.print_summary:
        for name, arr in t.items():
            print("  %s_%s.dat : %d float32 (%d bytes)" % (a.prefix, name, arr.size, arr.nbytes))
    rc = 0
    if a.verify:
        v = verify_dat_files(a.outdir, a.prefix, a.collimator_layer_base, a.collimator_holes_base)
        print("=== VERIFY (read-back) ===")
        for k in ("image", "physics", "detector_floats", "crystals", "collimator_floats", "layers", "layer0",
                  "first_hole", "check"):
            print("%s: %s" % (k, v[k]))
        rc = 0 if v["valid"] else 2
    if a.sanity:
        print(sanity_text(sanity_report(t["Collimator"], t["Detector"], t["Image"])), end="")
    return rc


if __name__ == "__main__":
    raise SystemExit(main())
