"""Seeded synthetic geometries for the photoelectric / scatter sysmat workloads.

There is no public dataset for this path; every workload is generated here
from a seed, in the reference's units (mm, 1/mm, keV) and its axis
convention: Y is depth, and plate/crystal Y values are relative to plate 0,
which sits ``fov_to_plate0`` mm from the FOV centre (``Image[11]``).

Named workloads
---------------
``pe_small``   16^3 voxels of 1 mm; one 100x100x5 mm plate at 30 mm (mu 3.5/mm)
               with a 7x7 grid of 1.0 mm holes at 10 mm pitch; 32x32 crystals of
               1.6x1.6x6 mm at 60 mm; voxel sub-samples 4x4x4, crystal sub-cells
               2x4x2 (x, depth, z) -> [1024 x 4096], 1024 rays per entry.
``pe_large``   64x64x32 voxels of 0.5 mm; plates 5 mm at 30 mm and 3 mm at 40 mm,
               400 holes each (seeded jittered 20x20 grid at 5 mm pitch, diameters
               U(0.6, 1.2) mm); 4 layers of 40x40 crystals 1.6x1.6x3 mm at
               60/64/68/72 mm -> [6400 x 131072].  Sub-sampling as ``pe_small``.
``sweep``      64 seeded geometries: grids 16^3..48^3, 1-3 plates, 16-400 holes per
               plate, 16^2..48^2 crystals x 1-4 layers.
``sweep_small`` 64 small seeded geometries (grids 8^3..20^3, 8^2..24^2 crystals).
``scatter_small``  32x32x16 voxels of 1 mm, the ``pe_small`` collimator, 2 layers of
               32x32 crystals (60 and 66 mm) -> [2048 x 16384].
``scatter_large``  the same geometry with 64x64x32 voxels -> [2048 x 131072].

The attenuation values that the workload descriptions leave open
(plate mu_pe / mu_compton) are fixed here: tungsten 3.5 / 3.2 / 0.3 per mm,
CZT 0.35 / 0.28 / 0.07 per mm.  Only mu_total enters the photoelectric tracer
through the plates.
"""
from __future__ import annotations

from typing import List

import numpy as np

from .params import (Params, Plate, build_collimator, build_detector, build_image,
                     build_physics, crystal_layer, grid_holes)

TUNGSTEN = (3.5, 3.2, 0.3)
CZT = (0.35, 0.28, 0.07)


def _plate(width, thickness, height, distance, holes, mu=TUNGSTEN) -> Plate:
    return Plate(width, thickness, height, distance, mu[0], mu[1], mu[2], holes)


def pe_small() -> Params:
    holes = grid_holes(7, 7, 10.0, 0.5, 5.0, 0.0)
    col = build_collimator([_plate(100.0, 5.0, 100.0, 0.0, holes)])
    det = build_detector(crystal_layer(32, 32, 1.6, (1.6, 6.0, 1.6), 30.0, CZT))
    img = build_image((16, 16, 16), (1.0, 1.0, 1.0), fov_to_plate0=30.0)
    return Params(col, det, img, build_physics(), sv=(4, 4, 4), sc=(2, 4, 2), name="pe_small")


def pe_large(seed: int = 1) -> Params:
    rng = np.random.default_rng(seed)
    radius = lambda: float(rng.uniform(0.6, 1.2)) / 2.0  # noqa: E731
    h0 = grid_holes(20, 20, 5.0, radius, 5.0, 0.0, jitter=1.0, rng=rng)
    h1 = grid_holes(20, 20, 5.0, radius, 3.0, 10.0, jitter=1.0, rng=rng)
    col = build_collimator([_plate(100.0, 5.0, 100.0, 0.0, h0), _plate(100.0, 3.0, 100.0, 10.0, h1)])
    crystals = []
    for y in (30.0, 34.0, 38.0, 42.0):
        crystals += crystal_layer(40, 40, 1.6, (1.6, 3.0, 1.6), y, CZT)
    det = build_detector(crystals)
    img = build_image((64, 64, 32), (0.5, 0.5, 0.5), fov_to_plate0=30.0)
    return Params(col, det, img, build_physics(), sv=(4, 4, 4), sc=(2, 4, 2), name="pe_large")


def scatter_geometry(grid=(32, 32, 16)) -> Params:
    holes = grid_holes(7, 7, 10.0, 0.5, 5.0, 0.0)
    col = build_collimator([_plate(100.0, 5.0, 100.0, 0.0, holes)])
    crystals = crystal_layer(32, 32, 1.6, (1.6, 6.0, 1.6), 30.0, CZT)
    crystals += crystal_layer(32, 32, 1.6, (1.6, 6.0, 1.6), 36.0, CZT)
    det = build_detector(crystals)
    img = build_image(grid, (1.0, 1.0, 1.0), fov_to_plate0=30.0)
    return Params(col, det, img, build_physics(), sv=(1, 1, 1), sc=(2, 4, 2),
                  name="scatter_%dx%dx%d" % tuple(grid))


def scatter_small() -> Params:
    return scatter_geometry((32, 32, 16))


def scatter_large() -> Params:
    return scatter_geometry((64, 64, 32))


def sweep(seed: int = 2, count: int = 64) -> List[Params]:
    """``count`` geometries of uneven size for the batched persistent kernel."""
    rng = np.random.default_rng(seed)
    out = []
    for g in range(count):
        n = int(rng.integers(16, 49))
        n_plates = int(rng.integers(1, 4))
        plates = []
        fov = 30.0
        for l in range(n_plates):
            nh_side = int(rng.integers(4, 21))        # 16..400 holes per plate
            t = float(rng.choice([2.0, 3.0, 5.0]))
            dist = 8.0 * l
            pitch = 90.0 / nh_side
            r = lambda: float(rng.uniform(0.3, 0.45)) * min(pitch, 2.0)  # noqa: E731
            holes = grid_holes(nh_side, nh_side, pitch, r, t, dist, jitter=0.15 * pitch, rng=rng)
            plates.append(_plate(100.0, t, 100.0, dist, holes))
        nc = int(rng.integers(16, 49))
        n_layers = int(rng.integers(1, 5))
        pitch = float(rng.choice([1.2, 1.6, 2.0]))
        depth = float(rng.choice([3.0, 4.0, 6.0]))
        y0 = 8.0 * (n_plates - 1) + 20.0
        crystals = []
        for l in range(n_layers):
            crystals += crystal_layer(nc, nc, pitch, (pitch, depth, pitch), y0 + l * (depth + 0.5), CZT)
        vox = float(rng.choice([0.5, 1.0]))
        img = build_image((n, n, n), (vox, vox, vox), fov_to_plate0=fov)
        out.append(Params(build_collimator(plates), build_detector(crystals), img, build_physics(),
                          sv=(1, 1, 1), sc=(2, 4, 2), name="sweep_%02d" % g))
    return out


def sweep_small(seed: int = 3, count: int = 64) -> List[Params]:
    """``count`` small geometries (grids 8^3..20^3, 1-2 plates of 16-100 holes,
    8^2..24^2 crystals x 1-2 layers, voxel centres): each one alone fills the
    GPU for only a few waves of CTAs, so launch gaps and tails are a visible
    share of per-geometry launches."""
    rng = np.random.default_rng(seed)
    out = []
    for g in range(count):
        n = int(rng.integers(8, 21))
        n_plates = int(rng.integers(1, 3))
        plates = []
        for l in range(n_plates):
            nh_side = int(rng.integers(4, 11))
            t = float(rng.choice([2.0, 3.0]))
            pitch = 60.0 / nh_side
            r = lambda: float(rng.uniform(0.3, 0.45)) * min(pitch, 2.0)  # noqa: E731
            plates.append(_plate(80.0, t, 80.0, 6.0 * l, grid_holes(nh_side, nh_side, pitch, r, t, 6.0 * l,
                                                                    jitter=0.15 * pitch, rng=rng)))
        nc = int(rng.integers(8, 25))
        n_layers = int(rng.integers(1, 3))
        pitch = float(rng.choice([1.6, 2.0]))
        crystals = []
        for l in range(n_layers):
            crystals += crystal_layer(nc, nc, pitch, (pitch, 4.0, pitch), 6.0 * (n_plates - 1) + 16.0 + 4.5 * l, CZT)
        img = build_image((n, n, n), (1.0, 1.0, 1.0), fov_to_plate0=30.0)
        out.append(Params(build_collimator(plates), build_detector(crystals), img, build_physics(),
                          sv=(1, 1, 1), sc=(2, 4, 2), name="sweep_small_%02d" % g))
    return out


# ---------------------------------------------------------------------------
# Small cases for parity tests: every branch the tracer has, at a size the
# CPU oracle finishes in seconds.
# ---------------------------------------------------------------------------

def tiny(seed: int = 0, layers: int = 2, rotated: bool = False) -> Params:
    """4x4 crystals x ``layers``, one plate with 3x3 holes, 4x4x4 voxels of 2 mm.

    ``rotated`` adds crystal rotations about Y, two image rotations and an FOV
    shift, so that the trigonometric paths of the tracer are exercised.
    """
    rng = np.random.default_rng(seed)
    holes = grid_holes(3, 3, 4.0, lambda: float(rng.uniform(0.5, 0.9)), 4.0, 0.0, jitter=0.5, rng=rng)
    col = build_collimator([_plate(40.0, 4.0, 40.0, 0.0, holes)])
    crystals = []
    for l in range(layers):
        crystals += crystal_layer(4, 4, 2.0, (2.0, 4.0, 2.0), 14.0 + 4.0 * l, CZT)
    if rotated:
        for c in crystals:
            c.rotation = float(rng.uniform(-0.3, 0.3))
    det = build_detector(crystals)
    if rotated:
        img = build_image((4, 4, 4), (2.0, 2.0, 2.0), n_rotations=2, angle_per_rotation=0.1,
                          shift=(0.3, -0.2, 0.5), fov_to_plate0=20.0)
    else:
        img = build_image((4, 4, 4), (2.0, 2.0, 2.0), fov_to_plate0=20.0)
    return Params(col, det, img, build_physics(), sv=(1, 1, 1), sc=(2, 4, 2),
                  name="tiny_rot" if rotated else "tiny")


def two_plates_small(seed: int = 3) -> Params:
    """Two plates with jittered holes of random radius and 3 crystal layers."""
    rng = np.random.default_rng(seed)
    r = lambda: float(rng.uniform(0.3, 0.6))  # noqa: E731
    h0 = grid_holes(5, 5, 4.0, r, 3.0, 0.0, jitter=0.8, rng=rng)
    h1 = grid_holes(5, 5, 4.0, r, 2.0, 6.0, jitter=0.8, rng=rng)
    col = build_collimator([_plate(40.0, 3.0, 40.0, 0.0, h0), _plate(40.0, 2.0, 40.0, 6.0, h1)])
    crystals = []
    for l, y in enumerate((16.0, 19.0, 22.0)):
        crystals += crystal_layer(6, 6, 1.6, (1.6, 3.0, 1.6), y, CZT)
    det = build_detector(crystals)
    img = build_image((6, 6, 4), (1.0, 1.0, 1.0), fov_to_plate0=20.0)
    return Params(col, det, img, build_physics(), sv=(2, 2, 2), sc=(2, 4, 2), name="two_plates_small")


def scatter_mid(seed: int = 5, same_window: int = 1) -> Params:
    """2 layers of 8x8 crystals behind one plate of 5x5 jittered holes; 8x8x6
    voxels of 1.5 mm.  Small enough for the CPU oracle over the full matrix."""
    rng = np.random.default_rng(seed)
    holes = grid_holes(5, 5, 5.0, lambda: float(rng.uniform(0.5, 0.8)), 4.0, 0.0, jitter=0.6, rng=rng)
    col = build_collimator([_plate(40.0, 4.0, 40.0, 0.0, holes)])
    crystals = crystal_layer(8, 8, 2.0, (2.0, 5.0, 2.0), 14.0, CZT)
    crystals += crystal_layer(8, 8, 2.0, (2.0, 5.0, 2.0), 19.5, CZT)
    det = build_detector(crystals)
    img = build_image((8, 8, 6), (1.5, 1.5, 1.5), fov_to_plate0=20.0)
    return Params(col, det, img, build_physics(same_window=same_window), sv=(1, 1, 1), sc=(2, 4, 2),
                  name="scatter_mid")


NAMED = {
    "pe_small": pe_small,
    "pe_large": pe_large,
    "scatter_small": scatter_small,
    "scatter_large": scatter_large,
    "scatter_mid": scatter_mid,
    "tiny": tiny,
    "two_plates_small": two_plates_small,
}
