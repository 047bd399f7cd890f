"""Generate the golden fixtures in this directory from the reference's own code.

Runs the reference kernels compiled for the host by oracle/Makefile
(oracle/_ref/libref_*.so, built from the reference sources where they lie) on
small seeded geometries, and stores inputs and outputs as .npz files:

* ``pe_<case>.npz``     PE sysmat entries: tables, sub-sampling, the sampled
                         (row, voxel, rotation) cells, and the reference's
                         single-precision (f32) and double (f64) results.
* ``prim_<kind>.npz``   ray-primitive calls (random plus axis-aligned and
                         near-tangent rays) with the reference's f32 results.
* ``scatter_<case>.npz`` primary-Compton scatter: tables, the PE sysmat fed in
                         (float32, from the PE oracle), the reference's bitmaps
                         (crystal and collimator words), sampled (row, voxel)
                         cells, and the reference's f32 and f64 crystal- and
                         collimator-scatter values.

Usage: ``python tests/golden/make_golden.py`` (needs oracle/_ref built).
"""
from __future__ import annotations

import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(ROOT, "gpu-spect-pet-sysmat_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from sysmat_b200 import configs  # noqa: E402
import oracle_py  # noqa: E402

PE_CASES = {
    # name: (params factory, sub-sampling override (sv, sc) or None, n samples, rotations)
    "tiny_ref": (lambda: configs.tiny(), ((1, 1, 1), (8, 16, 8)), 48, (0,)),
    "tiny": (lambda: configs.tiny(), None, 96, (0,)),
    "tiny_rot": (lambda: configs.tiny(rotated=True), None, 64, (0, 1)),
    "two_plates": (lambda: configs.two_plates_small(), None, 64, (0,)),
    "pe_small": (lambda: configs.pe_small(), None, 24, (0,)),
}


SCATTER_CASES = {
    # name: (params factory, rotation, sampled cells or None for the full matrix)
    "tiny": (lambda: configs.tiny(), 0, None),
    "tiny_rot": (lambda: _per_crystal_window(configs.tiny(seed=4, rotated=True)), 1, None),
    "mid": (lambda: configs.scatter_mid(), 0, 768),
}


def _per_crystal_window(p):
    """Windows from each crystal's energy resolution (Physics[4] = 0)."""
    p = p.copy()
    p.physics = p.physics.copy()
    p.physics[4] = 0.0
    return p


def scatter_fixture(name, factory, rotation, n_cells):
    p = factory()
    p.sv, p.sc = (1, 1, 1), (2, 4, 2)
    N, V = p.n_crystals, p.n_voxels
    rows = np.repeat(np.arange(N), V)
    vox = np.tile(np.arange(V), N)
    pe = oracle_py.oracle_pe_entries(p, rows, vox, "fp64", rotation=rotation).astype(np.float32).reshape(N, V)
    bm_c = oracle_py.ref_bitmap_crystal(p)
    bm_h = oracle_py.ref_bitmap_collimator(p)
    if n_cells is not None:
        rng = np.random.default_rng(zlib.crc32(("scatter_" + name).encode()))
        pick = rng.choice(N * V, n_cells, replace=False)
        rows, vox = rows[pick], vox[pick]
    out = {}
    for kind in ("crystal", "collimator"):
        bm = bm_c if kind == "crystal" else bm_h
        for variant in ("f32", "f64"):
            out["%s_%s" % (kind, variant)] = oracle_py.ref_scatter_entries(p, kind, rows, vox, bm, pe, variant,
                                                                           rotation=rotation)
    np.savez_compressed(os.path.join(HERE, "scatter_%s.npz" % name),
                        collimator=p.collimator[:100 + 9 * p.n_holes], detector=p.detector[:1 + 12 * N],
                        image=p.image, physics=p.physics, rotation=np.int64(rotation), pe=pe,
                        bitmap_crystal=bm_c, bitmap_collimator=bm_h, rows=rows, voxels=vox,
                        **{"ref_" + k: v for k, v in out.items()})
    print("scatter_%s: %d cells, nonzero crystal %d collimator %d" % (
        name, rows.size, int((out["crystal_f64"] != 0).sum()), int((out["collimator_f64"] != 0).sum())))


def prim_rays(kind: str, n: int, seed: int) -> np.ndarray:
    """Ray/box or ray/cylinder argument rows covering every branch."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        mode = i % 6
        a = rng.uniform(-6, 6, 3).astype(np.float32)
        b = rng.uniform(-6, 6, 3).astype(np.float32)
        if rng.uniform() < 0.5:   # a segment through a point near the origin, so that most rays hit
            c = rng.uniform(-1.0, 1.0, 3)
            u = rng.normal(size=3)
            u /= np.linalg.norm(u)
            a = (c - u * rng.uniform(3, 9)).astype(np.float32)
            b = (c + u * rng.uniform(0.2, 9)).astype(np.float32)
        if mode == 1:      # nearly axis-parallel in x (|dx| < 1e-3)
            b[0] = a[0] + np.float32(rng.uniform(-9e-4, 9e-4))
        elif mode == 2:    # parallel to z only
            b[0] = a[0]; b[1] = a[1]
        elif mode == 3:    # planar in y
            b[1] = a[1] + np.float32(rng.uniform(-5e-4, 5e-4))
        elif mode == 4:    # endpoint inside the box
            b = rng.uniform(-1, 1, 3).astype(np.float32)
        if kind == "cylinder":
            xc, zc = rng.uniform(-0.5, 0.5, 2)
            y1 = rng.uniform(-3, 0)
            y2 = y1 + rng.choice([0.0005, rng.uniform(0.5, 4)])
            R = rng.uniform(0.2, 2.5)
            if mode == 5:  # graze the wall: make the line pass at distance ~R from the axis
                a = np.array([xc + R * 0.9999, -8.0, zc], np.float32)
                b = np.array([xc + R * 1.0001, 8.0, zc + rng.uniform(-1e-3, 1e-3)], np.float32)
            rows.append(np.concatenate([a, b, [xc, y1, y2, zc, R]]).astype(np.float32))
        else:
            lo = rng.uniform(-2.5, 0, 3)
            hi = lo + rng.uniform(0.1, 4, 3)
            if mode == 5:  # touch a face within a few ulps
                a[1] = np.float32(lo[1]); b[1] = np.float32(lo[1] + 1e-6)
            rows.append(np.concatenate([a, b, lo, hi]).astype(np.float32))
    return np.stack(rows)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "scatter":
        for name, (factory, rotation, n_cells) in SCATTER_CASES.items():
            scatter_fixture(name, factory, rotation, n_cells)
        return
    if not oracle_py.ref_available("pe_f32"):
        raise SystemExit("oracle/_ref/libref_pe_f32.so missing: run `make -C oracle ref` first")
    for name, (factory, override, n, rotations) in PE_CASES.items():
        p = factory()
        if override is not None:
            p.sv, p.sc = override
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        rows_all, vox_all, rot_all, f32_all, f64_all = [], [], [], [], []
        for rot in rotations:
            rows = rng.integers(0, p.n_crystals, n)
            vox = rng.integers(0, p.n_voxels, n)
            f32 = oracle_py.ref_pe_entries(p, rows, vox, "f32", rotation=rot)
            f64 = oracle_py.ref_pe_entries(p, rows, vox, "f64", rotation=rot)
            rows_all.append(rows); vox_all.append(vox); rot_all.append(np.full(n, rot)); f32_all.append(f32)
            f64_all.append(f64)
        np.savez_compressed(os.path.join(HERE, "pe_%s.npz" % name),
                            collimator=p.collimator[:100 + 9 * p.n_holes], detector=p.detector[:1 + 12 * p.n_crystals],
                            image=p.image, physics=p.physics, sv=np.asarray(p.sv), sc=np.asarray(p.sc),
                            rows=np.concatenate(rows_all), voxels=np.concatenate(vox_all),
                            rotation=np.concatenate(rot_all), ref_f32=np.concatenate(f32_all),
                            ref_f64=np.concatenate(f64_all))
        print("pe_%s: %d cells, nonzero %d" % (name, len(np.concatenate(f32_all)), int((np.concatenate(f32_all) != 0).sum())))
    if oracle_py.ref_available("scatter_f32"):
        for name, (factory, rotation, n_cells) in SCATTER_CASES.items():
            scatter_fixture(name, factory, rotation, n_cells)
    for kind, seed in (("box", 11), ("inside", 12), ("cylinder", 13)):
        args = prim_rays(kind, 3000, seed)
        out = oracle_py.primitive(kind, args, impl="ref")
        np.savez_compressed(os.path.join(HERE, "prim_%s.npz" % kind), args=args, ref_f32=out)
        print("prim_%s: %d rays, nonzero %d" % (kind, len(out), int((out != 0).sum())))


if __name__ == "__main__":
    main()
