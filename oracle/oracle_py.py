"""TEST INFRASTRUCTURE ONLY -- ctypes access to the CPU oracle.

Imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg; never by the product.  Two families of libraries:

* ``oracle/_build/liboracle.so``: this project's restatement of the reference
  algorithm (oracle_pe.cpp, oracle_scatter.cpp), modes ``fp32`` (the
  reference's single-precision arithmetic, bit-exact), ``fp64`` and ``dual``
  (single-precision decisions, double magnitudes).
* ``oracle/_ref/libref_*.so``: the reference's own kernel code compiled for
  the host (``f32`` and ``f64``) and for sm_100a (``cuda``) by oracle/Makefile.
  Present only where the reference tree was available at build time; the
  shared objects travel with the working tree.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)

_libs = {}

MODES = {"fp32": 0, "fp64": 1, "dual": 2}


def _ptr(a, t):
    return a.ctypes.data_as(t)


def _load(path: str):
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def oracle_lib():
    return _load(os.path.join(BUILD, "liboracle.so"))


def ref_available(kind: str = "pe_f32") -> bool:
    return os.path.exists(os.path.join(REF, "libref_%s.so" % kind))


def ref_lib(kind: str):
    return _load(os.path.join(REF, "libref_%s.so" % kind))


def _tables(params):
    col = np.ascontiguousarray(params.collimator, dtype=np.float32)
    det = np.ascontiguousarray(params.detector, dtype=np.float32)
    img = np.ascontiguousarray(params.image, dtype=np.float32).copy()
    return col, det, img


def fine_cells(params, voxels):
    """Fine-grid voxel indices (n, Sv) covering each coarse voxel, in the
    oracle's sub-point order (x fastest, then y, then z)."""
    nx, ny, nz = params.grid
    kx, ky, kz = params.sv
    v = np.asarray(voxels, dtype=np.int64)
    ix, iy, iz = v % nx, (v // nx) % ny, v // (nx * ny)
    sz, sy, sx = np.meshgrid(np.arange(kz), np.arange(ky), np.arange(kx), indexing="ij")
    sx, sy, sz = sx.ravel(), sy.ravel(), sz.ravel()
    fx = ix[:, None] * kx + sx[None, :]
    fy = iy[:, None] * ky + sy[None, :]
    fz = iz[:, None] * kz + sz[None, :]
    return (fz * (ny * ky) + fy) * (nx * kx) + fx


def fine_image(params):
    img = np.ascontiguousarray(params.image, dtype=np.float32).copy()
    for a in range(3):
        n = int(np.floor(img[a] + np.float32(0.001)))
        img[a] = np.float32(n * params.sv[a])
        img[3 + a] = np.float32(img[3 + a] / np.float32(params.sv[a]))
    img[30] = img[2]
    img[31] = 0.0
    return img


def oracle_pe_entries(params, rows: Sequence[int], voxels: Sequence[int], mode: str = "fp64",
                      rotation: int = 0, nthreads: int = 0) -> np.ndarray:
    """Sysmat entries (row = crystal, voxel = coarse voxel index) from the restatement."""
    lib = oracle_lib()
    col, det, img = _tables(params)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    vox = np.ascontiguousarray(voxels, dtype=np.int64)
    out = np.zeros(rows.size, dtype=np.float64)
    sv = np.asarray(params.sv, dtype=np.int32)
    sc = np.asarray(params.sc, dtype=np.int32)
    lib.oracle_pe_entries(_ptr(col, _f32p), ctypes.c_longlong(col.size), _ptr(det, _f32p),
                          ctypes.c_longlong(det.size), _ptr(img, _f32p), _ptr(sv, _i32p), _ptr(sc, _i32p),
                          ctypes.c_int(rotation), _ptr(rows, _i64p), _ptr(vox, _i64p),
                          ctypes.c_longlong(rows.size), ctypes.c_int(MODES[mode]), _ptr(out, _f64p),
                          ctypes.c_int(nthreads))
    return out


def oracle_pe_hits(params, row: int, voxel: int, rotation: int = 0) -> np.ndarray:
    """Word stream of per-ray hit records for one entry (see oracle_pe.cpp HitLog)."""
    lib = oracle_lib()
    lib.oracle_pe_hits.restype = ctypes.c_longlong
    col, det, img = _tables(params)
    sv = np.asarray(params.sv, dtype=np.int32)
    sc = np.asarray(params.sc, dtype=np.int32)
    cap = 1 << 16
    while True:
        out = np.zeros(cap, dtype=np.int32)
        n = lib.oracle_pe_hits(_ptr(col, _f32p), _ptr(det, _f32p), _ptr(img, _f32p), _ptr(sv, _i32p),
                               _ptr(sc, _i32p), ctypes.c_int(rotation), ctypes.c_longlong(row),
                               ctypes.c_longlong(voxel), _ptr(out, _i32p), ctypes.c_longlong(cap))
        if n >= 0:
            return out[:n]
        cap = -n


def parse_hits(words: np.ndarray):
    """Decode a hit word stream into {ray: (plate_miss_mask, holes tuple, crystals tuple)}."""
    out = {}
    i = 0
    w = words.tolist()
    while i < len(w):
        ray, mask, nh = w[i], w[i + 1], w[i + 2]
        holes = tuple(w[i + 3:i + 3 + nh])
        i += 3 + nh
        nc = w[i]
        crystals = tuple(w[i + 1:i + 1 + nc])
        i += 1 + nc
        out[ray] = (mask, holes, crystals)
    return out


def ref_pe_entries(params, rows: Sequence[int], voxels: Sequence[int], variant: str = "f32",
                   rotation: int = 0, nthreads: int = 0) -> np.ndarray:
    """Entries computed by the reference's own kernel code on the host.

    Voxel sub-sampling runs the reference on the finer grid (one kernel cell
    per sub-point) and averages the sub-point values in double.
    """
    lib = ref_lib("pe_" + variant)
    col, det, _ = _tables(params)
    img = fine_image(params)
    img[20] = np.float32(rotation)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    cells = fine_cells(params, voxels)
    n_sub = cells.shape[1]
    r = np.ascontiguousarray(np.repeat(rows, n_sub), dtype=np.int64)
    c = np.ascontiguousarray(cells.ravel(), dtype=np.int64)
    out = np.zeros(r.size, dtype=np.float64)
    n_fine = int(img[0]) * int(img[1]) * int(img[2])
    lib.ref_pe_entries(_ptr(col, _f32p), ctypes.c_int64(col.size), _ptr(det, _f32p), ctypes.c_int64(det.size),
                       _ptr(img, _f32p), ctypes.c_int(params.sc[0]), ctypes.c_int(params.sc[1]),
                       ctypes.c_int(params.sc[2]), ctypes.c_int(params.n_crystals), ctypes.c_int(n_fine),
                       _ptr(r, _i64p), _ptr(c, _i64p), ctypes.c_int64(r.size), _ptr(out, _f64p),
                       ctypes.c_int(nthreads))
    return out.reshape(-1, n_sub).mean(axis=1)


def _batch(libfn, args: np.ndarray, width: int) -> np.ndarray:
    a = np.ascontiguousarray(args, dtype=np.float32).reshape(-1, width)
    out = np.zeros(a.shape[0], dtype=np.float64)
    libfn(_ptr(a, _f32p), ctypes.c_int64(a.shape[0]), _ptr(out, _f64p))
    return out


def primitive(kind: str, args: np.ndarray, impl: str = "oracle") -> np.ndarray:
    """kind in {box, inside, cylinder}; impl 'oracle' (float), 'dual' (float
    decisions, double values) or 'ref' (the reference's own primitives)."""
    width = 11 if kind == "cylinder" else 12
    name = {"box": "box_ray_batch", "inside": "box_inside_batch", "cylinder": "cylinder_batch"}[kind]
    if impl == "oracle":
        return _batch(getattr(oracle_lib(), "oracle_" + name), args, width)
    if impl == "dual":
        return _batch(getattr(oracle_lib(), "oracle_" + name + "_dual"), args, width)
    return _batch(getattr(ref_lib("pe_f32"), "ref_" + name), args, width)


# ---------------------------------------------------------------------------
# Primary-Compton scatter (oracle_scatter.cpp and the reference's scatter.cu)
# ---------------------------------------------------------------------------

_u32p = ctypes.POINTER(ctypes.c_uint32)


def crystal_bitmap_words(n_crystals: int) -> int:
    """uint32 words of the crystal bitmap: N(N+1)/2 pairs x N bits (scatter.cu:2053-2056)."""
    bits = (n_crystals * (n_crystals + 1) // 2) * n_crystals
    return (bits + 31) // 32


def collimator_bitmap_words(n_crystals: int, n_holes0: int) -> int:
    bits = n_holes0 * n_crystals * n_crystals
    return (bits + 31) // 32


def layer0_holes(params) -> int:
    return int(np.floor(np.float32(params.collimator[10]) + np.float32(0.01)))


def oracle_bitmap_crystal(params) -> np.ndarray:
    det = np.ascontiguousarray(params.detector, dtype=np.float32)
    n = crystal_bitmap_words(params.n_crystals)
    out = np.zeros(n, dtype=np.uint32)
    oracle_lib().oracle_bitmap_crystal(_ptr(det, _f32p), ctypes.c_longlong(det.size), _ptr(out, _u32p),
                                       ctypes.c_longlong(n))
    return out


def oracle_bitmap_collimator(params) -> np.ndarray:
    det = np.ascontiguousarray(params.detector, dtype=np.float32)
    col = np.ascontiguousarray(params.collimator, dtype=np.float32)
    n = collimator_bitmap_words(params.n_crystals, layer0_holes(params))
    out = np.zeros(n, dtype=np.uint32)
    oracle_lib().oracle_bitmap_collimator(_ptr(det, _f32p), ctypes.c_longlong(det.size), _ptr(col, _f32p),
                                          ctypes.c_longlong(col.size), _ptr(out, _u32p), ctypes.c_longlong(n))
    return out


def _scatter_tables(params, rotation):
    col = np.ascontiguousarray(params.collimator, dtype=np.float32)
    det = np.ascontiguousarray(params.detector, dtype=np.float32)
    img = np.zeros(100, np.float32)
    img[:min(100, params.image.size)] = params.image[:100]
    img[20] = np.float32(rotation)
    phy = np.zeros(100, np.float32)
    phy[:min(100, params.physics.size)] = params.physics[:100]
    return col, det, img, phy


def oracle_scatter_entries(params, kind: str, rows, voxels, bitmap: np.ndarray, pe: Optional[np.ndarray] = None,
                           sp=(1, 1, 1), mode: str = "fp64", rotation: int = 0, nthreads: int = 0) -> np.ndarray:
    """Scatter sysmat entries from the restatement.  kind 'crystal' needs the
    [N][V] float32 PE matrix ``pe``; ``sp`` = scatter points per crystal."""
    col, det, img, phy = _scatter_tables(params, rotation)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    vox = np.ascontiguousarray(voxels, dtype=np.int64)
    out = np.zeros(rows.size, dtype=np.float64)
    k = 0 if kind == "crystal" else 1
    if pe is None:
        pe = np.zeros(1, np.float32)
    pe = np.ascontiguousarray(pe, dtype=np.float32)
    bm = np.ascontiguousarray(bitmap, dtype=np.uint32)
    spa = np.asarray(sp, dtype=np.int32)
    oracle_lib().oracle_scatter_entries(ctypes.c_int(k), _ptr(col, _f32p), _ptr(det, _f32p), _ptr(img, _f32p),
                                        _ptr(phy, _f32p), _ptr(pe, _f32p), _ptr(bm, _u32p), _ptr(spa, _i32p),
                                        _ptr(rows, _i64p), _ptr(vox, _i64p), ctypes.c_longlong(rows.size),
                                        ctypes.c_int(0 if mode == "fp32" else 1), _ptr(out, _f64p),
                                        ctypes.c_int(nthreads))
    return out


def oracle_compton_integral(args: np.ndarray, mode: str = "fp64") -> np.ndarray:
    a = np.ascontiguousarray(args, dtype=np.float32).reshape(-1, 3)
    out = np.zeros(a.shape[0], dtype=np.float64)
    oracle_lib().oracle_compton_integral_batch(_ptr(a, _f32p), ctypes.c_longlong(a.shape[0]),
                                               ctypes.c_int(0 if mode == "fp32" else 1), _ptr(out, _f64p))
    return out


def ref_bitmap_crystal(params) -> np.ndarray:
    lib = ref_lib("scatter_f32")
    det = np.ascontiguousarray(params.detector, dtype=np.float32)
    out = np.zeros(crystal_bitmap_words(params.n_crystals), dtype=np.uint32)
    lib.ref_bitmap_crystal(_ptr(det, _f32p), ctypes.c_int64(det.size), _ptr(out, _u32p))
    return out


def ref_bitmap_collimator(params) -> np.ndarray:
    lib = ref_lib("scatter_f32")
    det = np.ascontiguousarray(params.detector, dtype=np.float32)
    col = np.ascontiguousarray(params.collimator, dtype=np.float32)
    out = np.zeros(collimator_bitmap_words(params.n_crystals, layer0_holes(params)), dtype=np.uint32)
    lib.ref_bitmap_collimator(_ptr(det, _f32p), ctypes.c_int64(det.size), _ptr(col, _f32p), ctypes.c_int64(col.size),
                              _ptr(out, _u32p))
    return out


def ref_scatter_entries(params, kind: str, rows, voxels, bitmap: np.ndarray, pe: Optional[np.ndarray] = None,
                        variant: str = "f32", rotation: int = 0, nthreads: int = 0) -> np.ndarray:
    """Entries computed by the reference's own scatter kernel code on the host."""
    lib = ref_lib("scatter_" + variant)
    col, det, img, phy = _scatter_tables(params, rotation)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    vox = np.ascontiguousarray(voxels, dtype=np.int64)
    out = np.zeros(rows.size, dtype=np.float64)
    bm = np.ascontiguousarray(bitmap, dtype=np.uint32)
    if kind == "crystal":
        pe = np.ascontiguousarray(pe, dtype=np.float32)
        lib.ref_crystal_scatter_entries(_ptr(det, _f32p), ctypes.c_int64(det.size), _ptr(img, _f32p),
                                        _ptr(phy, _f32p), _ptr(pe, _f32p), _ptr(bm, _u32p), _ptr(rows, _i64p),
                                        _ptr(vox, _i64p), ctypes.c_int64(rows.size), _ptr(out, _f64p),
                                        ctypes.c_int(nthreads))
    else:
        lib.ref_collimator_scatter_entries(_ptr(col, _f32p), ctypes.c_int64(col.size), _ptr(det, _f32p),
                                           ctypes.c_int64(det.size), _ptr(img, _f32p), _ptr(phy, _f32p),
                                           _ptr(bm, _u32p), _ptr(rows, _i64p), _ptr(vox, _i64p),
                                           ctypes.c_int64(rows.size), _ptr(out, _f64p), ctypes.c_int(nthreads))
    return out


def ref_compton_integral(args: np.ndarray, variant: str = "f32") -> np.ndarray:
    return _batch(ref_lib("scatter_" + variant).ref_compton_integral_batch, args, 3)
