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
* ``pe_shipped_<name>.npz`` the two geometries the reference ships as data files
                         (``PEGen_RayTracing_CircularHole/Params_*.dat``: 5632
                         crystals in 4 layers, one plate with 1865 holes, 64^3
                         voxels of 2 mm; ``Param_*.dat``: one crystal outside a
                         plate whose 4 holes have zero length, 64x64x32 voxels,
                         60 rotations), with the reference's f32 and f64 values
                         on sampled cells in its own mode (voxel centre, 8x16x8
                         crystal sub-cells).  Rows are contiguous blocks spread
                         over the detector layers; within each row the cells mix
                         the largest entries (voxels seen through holes) with
                         random ones.

* ``beams_reference.npz`` the reference's beam post-processing
                         (extract_beam_prop_masks.py, compute_mpxi_3d.py) run
                         here on a synthetic sysmat whose rows cycle through a
                         pool: the pool, its masks, rotation 0's beam
                         properties, MPXI and summary.
* ``mpxi_shipped_rot000.npz`` the MPXI volume the reference ships
                         (``beam_masks/mpxi_3d/mpxi_3d_rot_000.npy``) and the
                         summary text its script wrote for it.

* ``geometry_json_reference.npz`` the reference's json_to_dat.py and
                         check_geometry_sanity.py run here: tables of three
                         JSON geometries, error messages for broken ones, and
                         the printed sanity reports.

Usage: ``python tests/golden/make_golden.py [pe|scatter|shipped|beams|json]``
(needs oracle/_ref built; ``shipped``, ``beams`` and ``json`` read the reference tree named by
SYSMAT_REFERENCE_TREE, default /root/reference).
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


SHIPPED_ROW_BLOCKS = {
    # row blocks [r0, r0 + 8): layers 0, 1, 2 (32 x 16 crystals each) and layer 3 (64 x 64)
    "params": ((0, 8), (712, 720), (1324, 1332), (3600, 3608), (5624, 5632)),
    "param_degenerate": ((0, 1),),
}


def _read_table(path, n_max):
    raw = np.fromfile(path, dtype="<f4")
    return raw[:n_max].astype(np.float32)


def shipped_fixture(tree: str, name: str, prefix: str):
    """Tables of a geometry the reference ships, and the reference's own values
    on sampled cells (reference mode)."""
    from sysmat_b200.params import Params
    d = os.path.join(tree, "PEGen_RayTracing_CircularHole")
    col = _read_table(os.path.join(d, prefix + "_Collimator.dat"), 80000)
    det = _read_table(os.path.join(d, prefix + "_Detector.dat"), 80000)
    img = _read_table(os.path.join(d, prefix + "_Image.dat"), 100)
    phy = _read_table(os.path.join(d, prefix + "_Physics.dat"), 100)
    n_holes = sum(int(np.floor(col[(l + 1) * 10] + np.float32(0.001))) for l in
                  range(int(np.floor(col[0] + np.float32(0.001)))))
    n_crystals = int(np.floor(det[0] + np.float32(0.001)))
    col = col[:100 + 9 * n_holes] if col.size >= 100 + 9 * n_holes else col
    det = det[:1 + 12 * n_crystals] if det.size >= 1 + 12 * n_crystals else det
    padded = lambda a, n: np.concatenate([a, np.zeros(max(0, n - a.size), np.float32)])  # noqa: E731
    p = Params(padded(col, 80000), padded(det, 80000), padded(img, 100), padded(phy, 100), (1, 1, 1),
               (8, 16, 8), "shipped_" + name)
    rng = np.random.default_rng(zlib.crc32(("shipped_" + name).encode()))
    rotations = (0,) if p.n_rotations == 1 else (0, p.n_rotations // 2, p.n_rotations - 1)
    rows_all, vox_all, rot_all = [], [], []
    extra = {}
    if p.n_crystals == 1:
        # One crystal, seen from few voxels: its whole file, every rotation, from the
        # restatement (pinned bit for bit to the reference's code); the nonzero cells
        # are the golden zero pattern and a sample of them gets the reference's values.
        nonzero = []
        for rot in range(p.n_rotations):
            v = oracle_py.oracle_pe_entries(p, np.zeros(p.n_voxels, np.int64), np.arange(p.n_voxels), "fp32",
                                            rotation=rot)
            nonzero.append(rot * p.n_voxels + np.flatnonzero(v))
        nonzero = np.concatenate(nonzero)
        extra["nonzero_cells"] = nonzero
        pick = rng.choice(nonzero, min(96, nonzero.size), replace=False) if nonzero.size else nonzero
        rows_all.append(np.zeros(pick.size, np.int64))
        vox_all.append(pick % p.n_voxels)
        rot_all.append(pick // p.n_voxels)
        rotations = tuple(int(r) for r in np.unique(pick // p.n_voxels)) + rotations
    for rot in sorted(set(rotations)) if p.n_crystals > 1 else (0, p.n_rotations // 2, p.n_rotations - 1):
        for r0, r1 in SHIPPED_ROW_BLOCKS[name]:
            for row in range(r0, r1):
                # a geometry with one crystal sees it from few voxels: look at more of them
                cand = rng.choice(p.n_voxels, 256 if p.n_crystals > 1 else 8192, replace=False)
                v = oracle_py.oracle_pe_entries(p, np.full(cand.size, row), cand, "fp32", rotation=rot)
                top = cand[np.argsort(-v)[:3]]
                nz = cand[v != 0]
                rest = rng.choice(nz, min(3, nz.size), replace=False) if nz.size else cand[:0]
                anyv = rng.choice(cand, 2, replace=False)
                pick = np.unique(np.concatenate([top, rest, anyv]))
                rows_all.append(np.full(pick.size, row))
                vox_all.append(pick)
                rot_all.append(np.full(pick.size, rot))
    rows = np.concatenate(rows_all)
    vox = np.concatenate(vox_all)
    rot = np.concatenate(rot_all)
    f32 = np.zeros(rows.size)
    f64 = np.zeros(rows.size)
    for r in np.unique(rot):
        r = int(r)
        m = rot == r
        f32[m] = oracle_py.ref_pe_entries(p, rows[m], vox[m], "f32", rotation=int(r))
        f64[m] = oracle_py.ref_pe_entries(p, rows[m], vox[m], "f64", rotation=int(r))
    np.savez_compressed(os.path.join(HERE, "pe_shipped_%s.npz" % name), collimator=col, detector=det, image=img,
                        physics=phy, sv=np.asarray(p.sv), sc=np.asarray(p.sc), rows=rows, voxels=vox, rotation=rot,
                        ref_f32=f32, ref_f64=f64,
                        row_blocks=np.asarray(SHIPPED_ROW_BLOCKS[name], dtype=np.int64), **extra)
    print("pe_shipped_%s: %d crystals, %d holes, grid %s, %d cells, nonzero %d" % (
        name, p.n_crystals, p.n_holes, p.grid, rows.size, int((f64 != 0).sum())))


# ---------------------------------------------------------------------------
# Beam masks / MPXI: the reference's own post-processing scripts, run here
# ---------------------------------------------------------------------------

class _Stub:
    """Stands in for a module the reference scripts import but this image lacks
    (h5py, matplotlib): any attribute is another stub, calls return stubs."""

    def __init__(self, name="stub"):
        self._name = name

    def __getattr__(self, item):
        return _Stub(self._name + "." + item)

    def __call__(self, *a, **k):
        return _Stub(self._name + "()")


class _Dataset:
    """h5py dataset stand-in that keeps the rows the test fixture needs."""

    def __init__(self, shape, dtype, keep_rows):
        self.shape = tuple(shape)
        self.keep = keep_rows
        self.data = np.zeros((min(keep_rows, self.shape[0]),) + self.shape[1:], dtype)
        self.count = 0

    def resize(self, shape):
        self.shape = tuple(shape)
        if shape[0] > self.data.shape[0] and self.data.shape[0] < self.keep:
            grow = np.zeros((min(self.keep, shape[0]) - self.data.shape[0],) + self.data.shape[1:], self.data.dtype)
            self.data = np.concatenate([self.data, grow])

    def __setitem__(self, idx, value):
        row = idx[0] if isinstance(idx, tuple) else idx
        if row < self.data.shape[0]:
            self.data[row] = value

    def __getitem__(self, idx):
        return self.data[idx]


class _H5File:
    def __init__(self, path, mode="r", keep_rows=0):
        self.path = path
        self.sets = {}
        self.keep_rows = keep_rows

    def create_dataset(self, name, shape, maxshape=None, dtype="float32"):
        ds = _Dataset(shape, dtype, self.keep_rows)
        self.sets[name] = ds
        return ds

    def close(self):
        pass


def _pool_rows(k=29):
    """k distinct sysmat rows of 4096 voxels: photoelectric rows of the pe_small
    geometry (voxel centres, 2x4x2 sub-cells) from the oracle, an all-zero row
    (threshold 1.0) and a row holding entries exactly at 0.05 * max (strict >)."""
    p = configs.pe_small()
    p.sv = (1, 1, 1)
    rows = []
    for i, crystal in enumerate(np.linspace(0, p.n_crystals - 1, k - 2).astype(int)):
        rows.append(oracle_py.oracle_pe_entries(p, np.full(4096, crystal), np.arange(4096), "fp32").astype(np.float32))
    rows.append(np.zeros(4096, np.float32))
    tie = rows[5].copy()
    mx = tie.max()
    thr = np.float32(0.05) * mx
    tie[::7] = thr
    rows.append(tie)
    return np.stack(rows)


def beams_fixture(tree: str):
    """Runs the reference's extract_3d_beams() (extract_beam_prop_masks.py)
    unmodified on a synthetic 60-rotation x 5632-crystal x 4096-voxel sysmat
    whose rows cycle through a pool, and compute_mpxi_3d.py's
    compute_mpxi_for_rotation / summarize_mpxi on its rotation-0 masks.  Only
    the file layer is replaced (np.memmap by a view that builds each requested
    row from the pool; h5py by in-memory datasets; matplotlib by a stub)."""
    import importlib.util
    import types
    d = os.path.join(tree, "PEGen_RayTracing_CircularHole")
    pool = _pool_rows()
    n_det, n_vox, n_rot = 5632, 4096, 60

    class LazySysmat:
        def __getitem__(self, sl):
            start = sl.start
            g = start // n_vox
            assert sl.stop - start == n_vox and start % n_vox == 0
            return pool[g % len(pool)]

    fake_np = types.SimpleNamespace(**{k: getattr(np, k) for k in dir(np) if not k.startswith("__")})
    fake_np.memmap = lambda *a, **k: LazySysmat()
    files = {}

    def h5file(path, mode="r"):
        f = _H5File(path, mode, keep_rows=n_det)
        files[os.path.basename(path)] = f
        return f

    saved = {m: sys.modules.get(m) for m in ("h5py", "matplotlib", "matplotlib.pyplot")}
    h5 = types.ModuleType("h5py")
    h5.File = h5file
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    plt = _Stub("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules["h5py"], sys.modules["matplotlib"], sys.modules["matplotlib.pyplot"] = h5, mpl, plt
    try:
        spec = importlib.util.spec_from_file_location("ref_extract_beams", os.path.join(d, "extract_beam_prop_masks.py"))
        ext = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(ext)
        ext.np = fake_np
        ext.extract_3d_beams()
        spec = importlib.util.spec_from_file_location("ref_mpxi", os.path.join(d, "compute_mpxi_3d.py"))
        mp = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mp)
    finally:
        for m, v in saved.items():
            if v is None:
                sys.modules.pop(m, None)
            else:
                sys.modules[m] = v
    masks = files["beams_masks_3d.hdf5"].sets["beam_mask"]
    props = files["beams_properties_3d.hdf5"].sets["beam_properties"]
    mpxi = mp.compute_mpxi_for_rotation(masks, 0)
    summary = mp.summarize_mpxi(mpxi)
    n_active0 = int((masks.data[:n_det].sum(axis=1) > 0).sum())
    hist = np.asarray(summary["histogram"], dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "beams_reference.npz"), pool=pool,
                        pool_masks=masks.data[:len(pool)], props_rot0=props.data[:n_active0],
                        n_active_total=np.int64(props.shape[0]), mpxi_rot0=mpxi.astype(np.uint32),
                        summary_hist=hist, summary_scalars=np.asarray(
                            [summary["num_voxels_sampled"], summary["num_voxels_unsampled"],
                             summary["num_voxels_nonmultiplexed"], summary["num_voxels_multiplexed"],
                             summary["max_mpxi"]], np.int64),
                        summary_means=np.asarray([summary["mean_mpxi_all_voxels"], summary["mean_mpxi_sampled_voxels"],
                                                  summary["median_mpxi_sampled_voxels"]], np.float64),
                        dims=np.asarray([n_rot, n_det, n_vox], np.int64))
    shipped = os.path.join(d, "beam_masks", "mpxi_3d")
    vol = np.load(os.path.join(shipped, "mpxi_3d_rot_000.npy"))
    text = open(os.path.join(shipped, "mpxi_3d_rot_000_summary.txt")).read()
    np.savez_compressed(os.path.join(HERE, "mpxi_shipped_rot000.npz"), mpxi=vol, summary_text=np.asarray(text))
    print("beams_reference: pool %d rows, active beams %d (rotation 0: %d), mpxi max %d; shipped mpxi %s %s" % (
        len(pool), int(props.shape[0]), n_active0, int(mpxi.max()), vol.shape, vol.dtype))


# ---------------------------------------------------------------------------
# JSON front-end and sanity report: the reference's json_to_dat.py and
# check_geometry_sanity.py, run here
# ---------------------------------------------------------------------------

def _strip_comments(o):
    if isinstance(o, dict):
        return {k: _strip_comments(v) for k, v in o.items() if not k.startswith("_comment")}
    if isinstance(o, list):
        return [_strip_comments(v) for v in o]
    return o


def geometry_json_fixture(tree: str):
    """Tables json_to_dat.py builds from three JSON geometries (the reference's
    annotated example without its comment keys, and two of this project's
    seeded configurations written in the schema), the error messages it gives
    for broken inputs, and what check_geometry_sanity.py prints for exact-size
    tables of those geometries and of the shipped Params tables."""
    import contextlib
    import copy
    import importlib.util
    import io
    import json
    import tempfile
    from sysmat_b200 import geometry_json
    d = os.path.join(tree, "PEGen_RayTracing_CircularHole")

    def load(name, fname):
        spec = importlib.util.spec_from_file_location(name, os.path.join(d, fname))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        return m

    j2d = load("ref_json_to_dat", "json_to_dat.py")
    san = load("ref_sanity", "check_geometry_sanity.py")
    cases = {"annotated": _strip_comments(json.load(open(os.path.join(d, "geometry.annotated.json")))),
             "two_plates": geometry_json.params_to_json(configs.two_plates_small()),
             "tiny_rot": geometry_json.params_to_json(configs.tiny(seed=4, rotated=True))}
    out = {}
    for name, cfg in cases.items():
        tables = [j2d.build_param_collimator(cfg["collimator"], 10, 100), j2d.build_param_detector(cfg["detector"]),
                  j2d.build_param_image(cfg["image"]), j2d.build_param_physics(cfg["physics"])]
        out["json_" + name] = np.asarray(json.dumps(cfg))
        for key, arr in zip(("collimator", "detector", "image", "physics"), tables):
            out["%s_%s" % (key, name)] = arr
    broken = []
    base = cases["two_plates"]
    edits = [("collimator", lambda c: c["collimator"]["layers"][0].pop("mu_pe")),
             ("detector", lambda c: c["detector"]["bins"][3].pop("cy")),
             ("collimator", lambda c: c["collimator"]["layers"][1].__setitem__("hole_count", 7)),
             ("image", lambda c: c["image"].__setitem__("num_voxel_x", "six")),
             ("detector", lambda c: c["detector"].__setitem__("bins", []))]
    for section, edit in edits:
        cfg = copy.deepcopy(base)
        edit(cfg)
        fn = {"collimator": lambda c: j2d.build_param_collimator(c["collimator"], 10, 100),
              "detector": lambda c: j2d.build_param_detector(c["detector"]),
              "image": lambda c: j2d.build_param_image(c["image"])}[section]
        try:
            fn(cfg)
            msg = ""
        except SystemExit as e:
            msg = str(e)
        broken.append((json.dumps(cfg), msg))
    out["broken_json"] = np.asarray([b[0] for b in broken])
    out["broken_msg"] = np.asarray([b[1] for b in broken])
    shipped = np.load(os.path.join(HERE, "pe_shipped_params.npz"))
    sanity_inputs = {name: (out["collimator_" + name], out["detector_" + name], out["image_" + name])
                     for name in cases}
    sanity_inputs["shipped"] = (shipped["collimator"], shipped["detector"], shipped["image"])
    with tempfile.TemporaryDirectory() as tmp:
        for name, (c, dt, im) in sanity_inputs.items():
            paths = []
            for key, arr in (("col", c), ("det", dt), ("img", im)):
                path = os.path.join(tmp, "%s_%s.dat" % (name, key))
                np.asarray(arr, np.float32).tofile(path)
                paths.append(path)
            argv = sys.argv
            sys.argv = ["check_geometry_sanity.py", "--param_collimator", paths[0], "--param_detector", paths[1],
                        "--param_image", paths[2]]
            buf = io.StringIO()
            try:
                with contextlib.redirect_stdout(buf):
                    san.main()
            finally:
                sys.argv = argv
            out["sanity_" + name] = np.asarray(buf.getvalue())
    np.savez_compressed(os.path.join(HERE, "geometry_json_reference.npz"), **out)
    print("geometry_json_reference: %d geometries, %d broken inputs, %d sanity reports" % (
        len(cases), len(broken), len(sanity_inputs)))


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "json":
        geometry_json_fixture(os.environ.get("SYSMAT_REFERENCE_TREE", "/root/reference"))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "beams":
        beams_fixture(os.environ.get("SYSMAT_REFERENCE_TREE", "/root/reference"))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "shipped":
        tree = os.environ.get("SYSMAT_REFERENCE_TREE", "/root/reference")
        shipped_fixture(tree, "params", "Params")
        shipped_fixture(tree, "param_degenerate", "Param")
        return
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
