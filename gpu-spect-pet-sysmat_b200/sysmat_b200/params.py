"""Params_{Collimator,Detector,Image,Physics}.dat tables: layout, reader, writer.

The four tables are raw little-endian float32 arrays with positional fields.
The layout is the one the reference's CLI hosts read and its kernels index:

Collimator (``PEGen_RayTracing_CircularHole/ReadMe.txt:2-20``,
``PESysMatGen.cu:382-385,494-500,559-563,647-654``):
    [0]                          number of plates (collimator layers) P
    [(l+1)*10 + 0..7]            plate l: n_holes, width X, thickness Y, height Z,
                                 distance to plate 0 along Y, mu_total, mu_pe, mu_compton
    [100 + 9*h + 0..8]           hole h (global index, plates in order):
                                 x, y1, y2, z, R, mu_total, mu_pe, mu_compton, flag
Detector (``ReadMe.txt:22-35``, ``PESysMatGen.cu:452-458,477-478``):
    [0]                          number of crystals N
    [12*d + 1..12]               crystal d: x, y, z, width X, thickness Y, height Z,
                                 mu_total, mu_pe, mu_compton, energy resolution,
                                 rotation about Y, flag
Image (``ReadMe.txt:37-49``; side channel ``PEGen_CircularHole.cpp:165,177,189-190``):
    [0..11]                      nx, ny, nz, vx, vy, vz, n_rotations, angle per rotation,
                                 shift x, shift y, shift z, FOV centre to plate 0 (Y)
    [20] rotation index, [30] full nz, [31] slab z0 (written by the host per call)
Physics (``ReadMe.txt:51-61``):
    [0] use Compton, [1..3] save PE / Compton / PE+Compton, [4] same energy window,
    [5] window low keV, [6] window high keV, [7] photopeak keV,
    [8] compute crystal bitmap, [9] compute collimator bitmap

Y is the depth axis (image -> plates -> crystals).  Plate, hole and crystal Y
values are stored relative to plate 0 and shifted by Image[11] in the kernels.

The reference reads exactly 80000 / 80000 / 100 / 100 floats
(``PEGen_CircularHole.cpp:39-62``); :data:`LEGACY_TABLE_FLOATS` keeps that size
for files and for the legacy entry points.  Geometries with more than 6666
crystals need a longer detector table and use the length-explicit API.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

LEGACY_TABLE_FLOATS = 80000
SMALL_TABLE_FLOATS = 100

COL_LAYER_STRIDE = 10
COL_HOLE_BASE = 100
COL_HOLE_STRIDE = 9
DET_STRIDE = 12

FILE_NAMES = {
    "collimator": "Params_Collimator.dat",
    "detector": "Params_Detector.dat",
    "image": "Params_Image.dat",
    "physics": "Params_Physics.dat",
}


@dataclasses.dataclass
class Plate:
    """One tungsten plate (collimator layer) and its holes."""
    width: float          # X extent (mm)
    thickness: float      # Y extent (mm)
    height: float         # Z extent (mm)
    distance: float       # Y offset of this plate's centre from plate 0 (mm)
    mu_total: float
    mu_pe: float
    mu_compton: float
    holes: np.ndarray     # (n, 9) float32 rows: x, y1, y2, z, R, mu_t, mu_pe, mu_c, flag


@dataclasses.dataclass
class Crystal:
    x: float
    y: float
    z: float
    width: float          # X
    thickness: float      # Y (depth)
    height: float         # Z
    mu_total: float
    mu_pe: float
    mu_compton: float
    energy_resolution: float = 0.1
    rotation: float = 0.0
    flag: float = 1.0


@dataclasses.dataclass
class Params:
    """The four float32 tables plus the sub-sampling chosen for a run.

    ``sv`` is the voxel sub-sample grid (kx, ky, kz); ``sc`` the crystal
    sub-cell grid (cx, cy_depth, cz).  The reference kernel hard-codes
    sv = (1, 1, 1) and sc = (8, 16, 8) (``PESysMatGen.cu:435-440``).
    """
    collimator: np.ndarray
    detector: np.ndarray
    image: np.ndarray
    physics: np.ndarray
    sv: Tuple[int, int, int] = (1, 1, 1)
    sc: Tuple[int, int, int] = (8, 16, 8)
    name: str = ""

    # ---- derived sizes -------------------------------------------------
    @property
    def n_crystals(self) -> int:
        return int(np.floor(self.detector[0] + 0.001))

    @property
    def n_plates(self) -> int:
        return int(np.floor(self.collimator[0] + 0.001))

    @property
    def n_holes(self) -> int:
        return sum(int(np.floor(self.collimator[(l + 1) * COL_LAYER_STRIDE] + 0.001))
                   for l in range(self.n_plates))

    @property
    def grid(self) -> Tuple[int, int, int]:
        return tuple(int(np.floor(self.image[i] + 0.001)) for i in range(3))

    @property
    def n_voxels(self) -> int:
        nx, ny, nz = self.grid
        return nx * ny * nz

    @property
    def n_rotations(self) -> int:
        return max(1, int(np.floor(self.image[6] + 0.001)))

    @property
    def rays_per_entry(self) -> int:
        return int(np.prod(self.sv)) * int(np.prod(self.sc))

    def copy(self) -> "Params":
        return Params(self.collimator.copy(), self.detector.copy(), self.image.copy(),
                      self.physics.copy(), tuple(self.sv), tuple(self.sc), self.name)

    # ---- file IO ---------------------------------------------------------
    def write_dat(self, directory: str) -> None:
        """Write the four ``Params_*.dat`` files the CLI hosts read."""
        os.makedirs(directory, exist_ok=True)
        for key, fname in FILE_NAMES.items():
            arr = np.ascontiguousarray(getattr(self, key), dtype="<f4")
            arr.tofile(os.path.join(directory, fname))

    @staticmethod
    def read_dat(directory: str, sv=(1, 1, 1), sc=(8, 16, 8)) -> "Params":
        """Read ``Params_*.dat``; short files are zero-padded like ``fread`` into a zeroed buffer."""
        out = {}
        for key, fname in FILE_NAMES.items():
            raw = np.fromfile(os.path.join(directory, fname), dtype="<f4")
            n = LEGACY_TABLE_FLOATS if key in ("collimator", "detector") else SMALL_TABLE_FLOATS
            n = max(n, raw.size) if key == "detector" else n
            buf = np.zeros(n, dtype=np.float32)
            buf[:min(n, raw.size)] = raw[:n]
            out[key] = buf
        return Params(out["collimator"], out["detector"], out["image"], out["physics"], sv, sc,
                      os.path.basename(os.path.abspath(directory)))


def build_collimator(plates: Sequence[Plate]) -> np.ndarray:
    n_holes = sum(len(p.holes) for p in plates)
    need = COL_HOLE_BASE + COL_HOLE_STRIDE * n_holes
    if len(plates) > 9:
        raise ValueError("at most 9 plates: plate records (l+1)*10 collide with the hole table at 100")
    col = np.zeros(max(LEGACY_TABLE_FLOATS, need), dtype=np.float32)
    col[0] = len(plates)
    h = 0
    for l, p in enumerate(plates):
        b = (l + 1) * COL_LAYER_STRIDE
        col[b:b + 8] = [len(p.holes), p.width, p.thickness, p.height, p.distance,
                        p.mu_total, p.mu_pe, p.mu_compton]
        for row in np.asarray(p.holes, dtype=np.float32).reshape(-1, 9):
            col[COL_HOLE_BASE + COL_HOLE_STRIDE * h: COL_HOLE_BASE + COL_HOLE_STRIDE * (h + 1)] = row
            h += 1
    return col


def build_detector(crystals: Sequence[Crystal]) -> np.ndarray:
    need = 1 + DET_STRIDE * len(crystals)
    det = np.zeros(max(LEGACY_TABLE_FLOATS, need), dtype=np.float32)
    det[0] = len(crystals)
    for d, c in enumerate(crystals):
        det[DET_STRIDE * d + 1: DET_STRIDE * d + 13] = [
            c.x, c.y, c.z, c.width, c.thickness, c.height, c.mu_total, c.mu_pe,
            c.mu_compton, c.energy_resolution, c.rotation, c.flag]
    return det


def build_image(grid, voxel, n_rotations=1, angle_per_rotation=0.0, shift=(0.0, 0.0, 0.0),
                fov_to_plate0=30.0) -> np.ndarray:
    img = np.zeros(SMALL_TABLE_FLOATS, dtype=np.float32)
    img[0:3] = grid
    img[3:6] = voxel
    img[6] = n_rotations
    img[7] = angle_per_rotation
    img[8:11] = shift
    img[11] = fov_to_plate0
    img[2] = grid[2]
    img[30] = grid[2]
    img[31] = 0.0
    return img


def build_physics(use_compton=1, save_pe=1, save_compton=1, save_total=1, same_window=1,
                  window=(126.45, 154.55), energy_kev=140.5, calc_crystal_bitmap=1,
                  calc_collimator_bitmap=1) -> np.ndarray:
    phy = np.zeros(SMALL_TABLE_FLOATS, dtype=np.float32)
    phy[0:10] = [use_compton, save_pe, save_compton, save_total, same_window, window[0], window[1],
                 energy_kev, calc_crystal_bitmap, calc_collimator_bitmap]
    return phy


def grid_holes(nx: int, nz: int, pitch: float, radius, thickness: float, distance: float,
               jitter: float = 0.0, rng: Optional[np.random.Generator] = None) -> np.ndarray:
    """Holes on an nx x nz grid centred on the plate axis.

    Hole y1/y2 span the plate's own thickness about its centre, so that the
    hole and plate boxes coincide after the kernels add Image[11]
    (``PESysMatGen.cu:650-651`` vs ``:560-561``).
    """
    xs = (np.arange(nx) - (nx - 1) / 2.0) * pitch
    zs = (np.arange(nz) - (nz - 1) / 2.0) * pitch
    rows = []
    for z in zs:
        for x in xs:
            r = radius() if callable(radius) else radius
            jx = jz = 0.0
            if jitter > 0.0 and rng is not None:
                jx, jz = rng.uniform(-jitter, jitter, size=2)
            rows.append([x + jx, distance - thickness / 2.0, distance + thickness / 2.0, z + jz, r,
                         0.0, 0.0, 0.0, 1.0])
    return np.asarray(rows, dtype=np.float32).reshape(-1, 9)


def crystal_layer(nx: int, nz: int, pitch: float, size, y: float, mu=(0.35, 0.28, 0.07),
                  energy_resolution: float = 0.1) -> List[Crystal]:
    """An nx x nz layer of identical crystals at depth ``y`` (relative to plate 0)."""
    w, t, h = size
    out = []
    for iz in range(nz):
        for ix in range(nx):
            out.append(Crystal((ix - (nx - 1) / 2.0) * pitch, y, (iz - (nz - 1) / 2.0) * pitch,
                               w, t, h, mu[0], mu[1], mu[2], energy_resolution, 0.0, 1.0))
    return out
