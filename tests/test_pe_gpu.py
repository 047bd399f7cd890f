"""GPU parity of the photoelectric sysmat kernel, through the C ABI.

Oracles: the reference's own code (golden fixtures in tests/golden, produced
by the reference kernels compiled for the host) and the CPU restatement in
oracle/ (fp64; dual = the reference's single-precision decisions with double
magnitudes).  Tolerances (relative error on nonzero entries):

* vs FP64 (reference built with double): median <= 1e-4, max <= 1e-3
  (the accuracy target of the photoelectric tracer);
* vs dual (same decisions, double magnitudes): max <= 1e-4 -- pure arithmetic
  error, no decision flips;
* hit lists (plate misses, holes and crystals with a non-zero chord) of every
  ray: identical to the oracle's single-precision decisions, which are pinned
  bit-exact to the reference's own code.
"""
import numpy as np
import pytest

import oracle_py
import sysmat_b200
from helpers import load_pe_golden, rel_err
from sysmat_b200 import configs

pytestmark = pytest.mark.gpu

MAX_VS_FP64 = 1e-3
MEDIAN_VS_FP64 = 1e-4
MAX_VS_DUAL = 1e-4


@pytest.fixture(scope="module")
def ctx():
    c = sysmat_b200.Context(0)
    yield c
    c.close()


def full_matrix(ctx, p, rotation=0, **kw):
    g = sysmat_b200.Geometry(ctx, p)
    try:
        return g.pe(rotation=rotation, **kw)
    finally:
        g.close()


# ---- primitives -------------------------------------------------------------

@pytest.mark.parametrize("kind", ["box", "inside"])
def test_box_primitives_bit_exact_vs_reference(kind):
    z = np.load("%s/prim_%s.npz" % (oracle_py.HERE + "/../tests/golden", kind))
    got = sysmat_b200.primitive_batch(kind, z["args"]).astype(np.float64)
    assert np.array_equal(got, z["ref_f32"])


def test_hole_primitive_decisions_exact_values_refined():
    z = np.load("%s/prim_cylinder.npz" % (oracle_py.HERE + "/../tests/golden"))
    got = sysmat_b200.primitive_batch("cylinder", z["args"]).astype(np.float64)
    ref = z["ref_f32"]
    assert np.array_equal(got != 0, ref != 0), "hit/miss decisions differ from the reference"
    dual = oracle_py.primitive("cylinder", z["args"], impl="dual")
    err = rel_err(got, dual)
    assert err.max() <= 1e-4


# ---- sysmat values vs the reference's own code (golden) ---------------------

@pytest.mark.parametrize("name", ["tiny_ref", "tiny", "tiny_rot", "two_plates", "pe_small"])
def test_pe_vs_reference_golden(ctx, name):
    p, z = load_pe_golden(name)
    got = np.zeros(z["rows"].size)
    for rot in np.unique(z["rotation"]):
        m = z["rotation"] == rot
        A = full_matrix(ctx, p, rotation=int(rot))
        got[m] = A[z["rows"][m], z["voxels"][m]]
    e64 = rel_err(got, z["ref_f64"])
    assert e64.size == (z["ref_f64"] != 0).sum() and e64.size > 0
    assert np.median(e64) <= MEDIAN_VS_FP64 and e64.max() <= MAX_VS_FP64
    assert np.array_equal(got == 0, z["ref_f32"] == 0)


@pytest.mark.parametrize("factory,rot", [
    (lambda: configs.tiny(layers=3), 0),
    (lambda: configs.tiny(seed=4, rotated=True), 1),
    (lambda: configs.two_plates_small(seed=8), 0),
    (configs.pe_small, 0),
])
def test_pe_vs_oracle_random_entries(ctx, factory, rot):
    p = factory()
    A = full_matrix(ctx, p, rotation=rot)
    rng = np.random.default_rng(11)
    n = 48 if p.n_crystals > 500 else 160
    rows = rng.integers(0, p.n_crystals, n)
    vox = rng.integers(0, p.n_voxels, n)
    got = A[rows, vox]
    dual = oracle_py.oracle_pe_entries(p, rows, vox, "dual", rotation=rot)
    fp64 = oracle_py.oracle_pe_entries(p, rows, vox, "fp64", rotation=rot)
    ed = rel_err(got, dual)
    e64 = rel_err(got, fp64)
    assert ed.size > 0 and ed.max() <= MAX_VS_DUAL
    assert np.median(e64) <= MEDIAN_VS_FP64 and e64.max() <= MAX_VS_FP64


# ---- hit lists ---------------------------------------------------------------

@pytest.mark.parametrize("factory", [lambda: configs.tiny(layers=3), lambda: configs.two_plates_small(seed=8),
                                     lambda: configs.tiny(seed=4, rotated=True)])
def test_hit_lists_identical_to_oracle(ctx, factory):
    p = factory()
    g = sysmat_b200.Geometry(ctx, p)
    rng = np.random.default_rng(3)
    rows = rng.integers(0, p.n_crystals, 12)
    vox = rng.integers(0, p.n_voxels, 12)
    rec = g.record_hits(rows, vox)
    g.close()
    n_hits = 0
    for i in range(len(rows)):
        mine = sysmat_b200.parse_records(rec[i])
        ref = oracle_py.parse_hits(oracle_py.oracle_pe_hits(p, int(rows[i]), int(vox[i])))
        assert mine == ref, "entry (%d, %d)" % (rows[i], vox[i])
        n_hits += sum(len(h) + len(c) for _, h, c in ref.values())
    assert n_hits > 0


def test_hit_lists_pe_small_sample(ctx):
    p = configs.pe_small()
    g = sysmat_b200.Geometry(ctx, p)
    rows = np.array([0, 100, 527, 1023])
    vox = np.array([0, 2047, 1000, 4095])
    rec = g.record_hits(rows, vox)
    g.close()
    for i in range(len(rows)):
        assert sysmat_b200.parse_records(rec[i]) == oracle_py.parse_hits(
            oracle_py.oracle_pe_hits(p, int(rows[i]), int(vox[i])))


# ---- decomposition invariance -------------------------------------------------

def test_tiling_slabs_and_rows_do_not_change_results(ctx):
    p = configs.two_plates_small(seed=8)
    g = sysmat_b200.Geometry(ctx, p)
    full = g.pe()
    for tile in [(1, 1, 1), (6, 6, 4), (3, 2, 1), (8, 8, 2)]:
        assert np.array_equal(g.pe(opts=g.options(tile_voxels=tile)), full), tile
    vxy = g.nx * g.ny
    for z0 in range(g.nz):
        part = g.pe(z=(z0, 1))
        assert np.array_equal(part, full[:, z0 * vxy:(z0 + 1) * vxy])
    part = g.pe(rows=(13, 71))
    assert np.array_equal(part, full[13:71])
    g.close()


def test_voxel_pairs_do_not_change_results(ctx):
    """Entries of at most 16 rays (voxel centre x 2x4x2 sub-cells) go up to 8
    neighbouring voxels to a group of sub-points; which neighbours a voxel is
    grouped with (it depends on the brick) changes no value, and a voxel alone
    in its group gives the same."""
    p = configs.tiny(layers=3)
    g = sysmat_b200.Geometry(ctx, p)
    full = g.pe()
    for tile in [(1, 1, 1), (3, 2, 1), (4, 4, 4), (2, 3, 3), (1, 4, 2)]:
        assert np.array_equal(g.pe(opts=g.options(tile_voxels=tile)), full), tile
    g.close()


def test_legacy_pesysmatgen_slabs_match_api(ctx):
    """PESysMatGen with the reference CLI's slab side channel reproduces the
    sm API in reference mode (voxel centre, 8 x 16 x 8 sub-cells)."""
    p = configs.tiny()
    g = sysmat_b200.Geometry(ctx, p)
    full = g.pe(opts=sysmat_b200.PeOptions.make((1, 1, 1), (8, 16, 8)))
    g.close()
    nx, ny, nz = p.grid
    img = p.image.copy()
    img[30] = nz
    slab = 3
    for z0 in range(0, nz, slab):
        this = min(slab, nz - z0)
        img[2] = this
        img[31] = z0
        img[20] = 0
        dst = np.zeros((p.n_crystals, nx * ny * this), np.float32)
        q = sysmat_b200.PESysMatGen(p.collimator, p.detector, img, dst, 0)
        assert q == nx * ny * this
        assert np.array_equal(dst, full[:, z0 * nx * ny:(z0 + this) * nx * ny])


def test_reference_mode_matches_reference_golden_exactly_where_zero(ctx):
    p, z = load_pe_golden("tiny_ref")
    A = full_matrix(ctx, p)
    got = A[z["rows"], z["voxels"]]
    assert rel_err(got, z["ref_f32"]).max() <= 1e-4


# ---- errors -------------------------------------------------------------------

def test_invalid_arguments_raise(ctx):
    p = configs.tiny()
    g = sysmat_b200.Geometry(ctx, p)
    with pytest.raises(sysmat_b200.SysmatError) as e:
        g.pe(opts=sysmat_b200.PeOptions.make((0, 1, 1), (2, 4, 2)))
    assert e.value.code == -1
    with pytest.raises(sysmat_b200.SysmatError):
        g.pe(rows=(5, 200))
    with pytest.raises(sysmat_b200.SysmatError):
        g.pe(z=(3, 4))
    g.close()
    bad = p.copy()
    bad.detector = bad.detector.copy()
    bad.detector[4] = 0.0     # crystal 0 width
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.Geometry(ctx, bad)
    assert "crystal 0" in str(e.value)
