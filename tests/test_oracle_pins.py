"""The CPU oracle pinned to the reference.

* Against committed golden fixtures produced by the reference's own kernel
  code (tests/golden/make_golden.py): the oracle's single-precision mode must
  reproduce the reference's values bit for bit, its double mode within 1e-12.
* Against the reference build in oracle/_ref when it is present (this
  container): fresh random cells, both precisions, and the ray primitives.
"""
import numpy as np
import pytest

import oracle_py
from helpers import load_pe_golden, rel_err
from sysmat_b200 import configs

PE_GOLDEN = ["tiny_ref", "tiny", "tiny_rot", "two_plates", "pe_small"]


def _oracle_on_golden(p, z, mode):
    out = np.zeros(z["rows"].size)
    for rot in np.unique(z["rotation"]):
        m = z["rotation"] == rot
        out[m] = oracle_py.oracle_pe_entries(p, z["rows"][m], z["voxels"][m], mode, rotation=int(rot))
    return out


@pytest.mark.parametrize("name", PE_GOLDEN)
def test_oracle_fp32_bit_exact_vs_reference_golden(name):
    p, z = load_pe_golden(name)
    got = _oracle_on_golden(p, z, "fp32")
    assert np.array_equal(got, z["ref_f32"]), "oracle fp32 differs from the reference's single-precision values"


@pytest.mark.parametrize("name", PE_GOLDEN)
def test_oracle_fp64_vs_reference_golden(name):
    p, z = load_pe_golden(name)
    got = _oracle_on_golden(p, z, "fp64")
    err = rel_err(got, z["ref_f64"])
    assert err.size > 0 and err.max() <= 1e-12


@pytest.mark.parametrize("name", PE_GOLDEN)
def test_oracle_dual_tracks_fp64(name):
    """Dual mode (single-precision decisions, double magnitudes) agrees with FP64
    except where a decision flips; on these fixtures no decision flips."""
    p, z = load_pe_golden(name)
    got = _oracle_on_golden(p, z, "dual")
    err = rel_err(got, z["ref_f64"])
    assert np.median(err) <= 1e-12


@pytest.mark.parametrize("kind", ["box", "inside", "cylinder"])
def test_primitives_bit_exact_vs_reference_golden(kind):
    z = np.load("%s/prim_%s.npz" % (oracle_py.HERE + "/../tests/golden", kind))
    got = oracle_py.primitive(kind, z["args"], impl="oracle")
    assert np.array_equal(got, z["ref_f32"])
    assert (z["ref_f32"] != 0).sum() > 100   # the fixture exercises hits, not only misses


needs_ref = pytest.mark.skipif(not oracle_py.ref_available("pe_f32"), reason="oracle/_ref not built (no reference tree)")


@needs_ref
@pytest.mark.parametrize("factory,rot", [(lambda: configs.tiny(layers=3), 0), (lambda: configs.tiny(seed=5, rotated=True), 1),
                                         (lambda: configs.two_plates_small(seed=9), 0)])
def test_oracle_vs_reference_build_random_cells(factory, rot):
    p = factory()
    rng = np.random.default_rng(7)
    rows = rng.integers(0, p.n_crystals, 40)
    vox = rng.integers(0, p.n_voxels, 40)
    a = oracle_py.oracle_pe_entries(p, rows, vox, "fp32", rotation=rot)
    b = oracle_py.ref_pe_entries(p, rows, vox, "f32", rotation=rot)
    assert np.array_equal(a, b)
    c = oracle_py.oracle_pe_entries(p, rows, vox, "fp64", rotation=rot)
    d = oracle_py.ref_pe_entries(p, rows, vox, "f64", rotation=rot)
    assert rel_err(c, d).max() <= 1e-12


def test_oracle_reference_mode_matches_finer_grid_average():
    """Voxel sub-sampling k^3 is the reference on the k-times finer grid averaged."""
    p = configs.tiny()
    p.sv = (2, 2, 2)
    rows = np.array([0, 5, 17, 30])
    vox = np.array([0, 21, 42, 63])
    avg = oracle_py.oracle_pe_entries(p, rows, vox, "fp64")
    fine = p.copy()
    fine.sv = (1, 1, 1)
    fine.image = oracle_py.fine_image(p)
    cells = oracle_py.fine_cells(p, vox)
    direct = np.array([oracle_py.oracle_pe_entries(fine, np.full(8, r), c, "fp64").mean() for r, c in zip(rows, cells)])
    assert np.allclose(avg, direct, rtol=1e-14, atol=0)


def test_oracle_hit_log_consistent_with_value():
    """A ray whose record shows a plate miss contributes nothing: entries whose
    every ray misses a plate are exactly zero."""
    p = configs.tiny()
    words = oracle_py.oracle_pe_hits(p, 3, 10)
    recs = oracle_py.parse_hits(words)
    assert len(recs) == p.rays_per_entry
    all_blocked = all(mask != 0 for mask, _, _ in recs.values())
    val = oracle_py.oracle_pe_entries(p, [3], [10], "fp32")[0]
    assert (val == 0.0) == all_blocked
