"""Photoelectric parity at full size: the headline workload, the sweep's
largest and three-plate members, and the geometries the reference ships.

Tolerances as in test_pe_gpu.py (relative error on nonzero entries): against
FP64 median <= 1e-4 and max <= 1e-3; against the same-decision oracle (dual)
max <= 1e-4; per-ray hit lists identical to the oracle's single-precision
decisions, which are pinned bit for bit to the reference's own code.

Entries are chosen inside whole computed rows: per row the largest entries
(voxels that see the crystal through holes, where the hole chords and the
inter-crystal attenuation decide the value) and random ones.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle_py
import sysmat_b200
from helpers import GOLDEN, rel_err
from sysmat_b200 import configs
from sysmat_b200.params import Params

pytestmark = pytest.mark.gpu

MAX_VS_FP64 = 1e-3
MEDIAN_VS_FP64 = 1e-4
MAX_VS_DUAL = 1e-4


@pytest.fixture(scope="module")
def ctx():
    c = sysmat_b200.Context(0)
    yield c
    c.close()


def pick_entries(block, r0, rng, n_top=4, n_nonzero=4, n_any=2):
    """(rows, voxels) of the largest, random nonzero and random entries of each row of block."""
    rows, vox = [], []
    for i in range(block.shape[0]):
        row = block[i]
        top = np.argsort(-row)[:n_top]
        nz = np.flatnonzero(row)
        extra = rng.choice(nz, min(n_nonzero, nz.size), replace=False) if nz.size else top[:0]
        anyv = rng.choice(row.size, n_any, replace=False)
        v = np.unique(np.concatenate([top, extra, anyv]))
        rows.append(np.full(v.size, r0 + i))
        vox.append(v)
    return np.concatenate(rows), np.concatenate(vox)


def check_vs_oracle(p, got, rows, vox, rotation=0):
    dual = oracle_py.oracle_pe_entries(p, rows, vox, "dual", rotation=rotation)
    fp64 = oracle_py.oracle_pe_entries(p, rows, vox, "fp64", rotation=rotation)
    ed = rel_err(got, dual)
    e64 = rel_err(got, fp64)
    assert ed.size > 0 and ed.max() <= MAX_VS_DUAL, ed.max()
    assert np.median(e64) <= MEDIAN_VS_FP64 and e64.max() <= MAX_VS_FP64, (np.median(e64), e64.max())
    assert np.array_equal(np.asarray(got) == 0, dual == 0)
    return e64


# ---- pe_large (the benchmark workload) ----------------------------------------

PE_LARGE_BLOCKS = [(1600 * layer + 816, 1600 * layer + 824) for layer in range(4)] + [(6392, 6400)]


@pytest.fixture(scope="module")
def pe_large_blocks(ctx):
    p = configs.pe_large()
    g = sysmat_b200.Geometry(ctx, p)
    blocks = {b: g.pe(rows=b) for b in PE_LARGE_BLOCKS}
    g.close()
    return p, blocks


def test_pe_large_entries_in_every_layer_vs_fp64_and_dual(pe_large_blocks):
    p, blocks = pe_large_blocks
    rng = np.random.default_rng(21)
    rows, vox, got = [], [], []
    for (r0, r1), block in blocks.items():
        assert block.shape == (r1 - r0, p.n_voxels) and np.isfinite(block).all()
        r, v = pick_entries(block, r0, rng)
        rows.append(r)
        vox.append(v)
        got.append(block[r - r0, v])
    rows, vox, got = np.concatenate(rows), np.concatenate(vox), np.concatenate(got)
    assert rows.size >= 256
    e64 = check_vs_oracle(p, got, rows, vox)
    assert e64.size >= 200


def test_pe_large_hit_lists_layers_3_and_4(ctx, pe_large_blocks):
    p, blocks = pe_large_blocks
    rows, vox = [], []
    for (r0, r1) in PE_LARGE_BLOCKS[2:]:
        block = blocks[(r0, r1)]
        for i in (0, 5):
            top = np.argsort(-block[i])[:2]        # voxels seen through holes: many hits per ray
            rows += [r0 + i] * 2
            vox += list(top)
    g = sysmat_b200.Geometry(ctx, p)
    rec = g.record_hits(np.asarray(rows), np.asarray(vox))
    g.close()
    assert len(rows) >= 8
    n_crystal_hits = 0
    for i in range(len(rows)):
        mine = sysmat_b200.parse_records(rec[i])
        ref = oracle_py.parse_hits(oracle_py.oracle_pe_hits(p, int(rows[i]), int(vox[i])))
        assert mine == ref, "entry (%d, %d)" % (rows[i], vox[i])
        n_crystal_hits += sum(len(c) for _, _, c in ref.values())
    assert n_crystal_hits > 0   # rays to layers 3 and 4 cross crystals of the layers above


# ---- sweep members: more than 6666 crystals (extended tables), three plates ----

SWEEP_MEMBERS = [5, 22, 41, 45, 2, 35, 58]


@pytest.mark.parametrize("member", SWEEP_MEMBERS)
def test_sweep_member_vs_oracle(ctx, member):
    p = configs.sweep()[member]
    assert p.n_crystals > 6666 or p.n_plates == 3
    g = sysmat_b200.Geometry(ctx, p)
    rng = np.random.default_rng(100 + member)
    starts = sorted({0, (p.n_crystals // 2) // 8 * 8, max(0, p.n_crystals - 8)})
    rows, vox, got = [], [], []
    for r0 in starts:
        block = g.pe(rows=(r0, min(r0 + 8, p.n_crystals)))
        r, v = pick_entries(block, r0, rng, n_top=3, n_nonzero=3, n_any=1)
        rows.append(r)
        vox.append(v)
        got.append(block[r - r0, v])
    g.close()
    check_vs_oracle(p, np.concatenate(got), np.concatenate(rows), np.concatenate(vox))


# ---- the geometries the reference ships -----------------------------------------

def load_shipped(name):
    z = np.load(os.path.join(GOLDEN, "pe_shipped_%s.npz" % name))
    pad = lambda a, n: np.concatenate([a.astype(np.float32), np.zeros(max(0, n - a.size), np.float32)])  # noqa
    p = Params(pad(z["collimator"], 80000), pad(z["detector"], 80000), pad(z["image"], 100), pad(z["physics"], 100),
               tuple(int(v) for v in z["sv"]), tuple(int(v) for v in z["sc"]), "shipped_" + name)
    return p, z


def test_shipped_params_vs_reference_golden(ctx):
    """Params_*.dat as shipped: 5632 crystals in 4 layers, 1865 holes, 64^3
    voxels of 2 mm, reference mode.  Every sampled row is computed in full."""
    p, z = load_shipped("params")
    assert (p.n_crystals, p.n_holes, p.grid) == (5632, 1865, (64, 64, 64))
    g = sysmat_b200.Geometry(ctx, p)
    opts = sysmat_b200.PeOptions.make((1, 1, 1), (8, 16, 8))
    got = np.zeros(z["rows"].size)
    for r0, r1 in z["row_blocks"]:
        block = g.pe(rows=(int(r0), int(r1)), opts=opts)
        m = (z["rows"] >= r0) & (z["rows"] < r1)
        got[m] = block[z["rows"][m] - r0, z["voxels"][m]]
    e64 = rel_err(got, z["ref_f64"])
    assert e64.size == (z["ref_f64"] != 0).sum() and e64.size >= 200
    assert np.median(e64) <= MEDIAN_VS_FP64 and e64.max() <= MAX_VS_FP64, (np.median(e64), e64.max())
    assert np.array_equal(got == 0, z["ref_f32"] == 0)
    # hit lists of the largest sampled entries of layers 2 and 3
    order = np.argsort(-z["ref_f64"] * (z["rows"] >= 1024))
    sel = order[:8]
    rec = g.record_hits(z["rows"][sel], z["voxels"][sel], opts=opts)
    g.close()
    for i, k in enumerate(sel):
        mine = sysmat_b200.parse_records(rec[i])
        ref = oracle_py.parse_hits(oracle_py.oracle_pe_hits(p, int(z["rows"][k]), int(z["voxels"][k])))
        assert mine == ref, "entry (%d, %d)" % (z["rows"][k], z["voxels"][k])


def test_shipped_degenerate_param_through_cli(tmp_path):
    """Param_*.dat as shipped (short tables: one crystal at z = 200 mm, beyond
    the plate's edge, 4 zero-length holes, 64x64x32 voxels, 60 rotations)
    through PEGen_CircularHole: almost every ray misses the plate and is
    blocked (the reference's plate-miss penalty); only corner voxels at some
    rotations see the crystal through the plate.  The file's nonzero cells are
    exactly those of the reference's algorithm, and sampled values match the
    reference's own FP64 values."""
    p, z = load_shipped("param_degenerate")
    for key, fname in (("collimator", "Params_Collimator.dat"), ("detector", "Params_Detector.dat"),
                       ("image", "Params_Image.dat"), ("physics", "Params_Physics.dat")):
        z[key].astype("<f4").tofile(tmp_path / fname)
    binary = os.path.join(os.path.dirname(sysmat_b200.__file__), "..", "bin", "PEGen_CircularHole")
    r = subprocess.run([binary, "-cuda", "0"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    name = "PE_SysMat_shift_%f_%f_%f.sysmat" % tuple(float(v) for v in z["image"][8:11])
    out = np.fromfile(tmp_path / name, np.float32)
    assert out.size == p.n_rotations * p.n_crystals * p.n_voxels == 60 * 64 * 64 * 32
    assert np.array_equal(np.flatnonzero(out), np.sort(z["nonzero_cells"]))
    got = out[z["rotation"] * p.n_voxels + z["voxels"]]
    e64 = rel_err(got, z["ref_f64"])
    assert e64.size == (z["ref_f64"] != 0).sum() > 0
    assert np.median(e64) <= MEDIAN_VS_FP64 and e64.max() <= MAX_VS_FP64, (np.median(e64), e64.max())
