"""The CPU scatter oracle (oracle/oracle_scatter.cpp) pinned to the reference.

Golden fixtures (tests/golden/scatter_*.npz) hold the reference's own scatter
kernels' results (crystalScatterSysMatCuda, collimatorScatterSysMatCuda,
ScatterGen_RayTracing_CircularHole/scatter.cu, built for the host) and its
bitmaps.  The restatement must reproduce the reference's single-precision
values and bitmaps bit for bit and its double-precision values to 1e-12.
With scatter points (a crystal split into sub-cells) it must reduce to the
reference when the split is 1 x 1 x 1 and converge as the split refines.
"""
import numpy as np
import pytest

import oracle_py
from helpers import load_scatter_golden, rel_err
from sysmat_b200 import configs

SCATTER_GOLDEN = ["tiny", "tiny_rot", "mid"]
KINDS = ["crystal", "collimator"]


@pytest.mark.parametrize("name", SCATTER_GOLDEN)
def test_bitmaps_bit_exact_vs_reference_golden(name):
    p, z = load_scatter_golden(name)
    assert np.array_equal(oracle_py.oracle_bitmap_crystal(p), z["bitmap_crystal"])
    assert np.array_equal(oracle_py.oracle_bitmap_collimator(p), z["bitmap_collimator"])
    assert np.unpackbits(z["bitmap_crystal"].view(np.uint8)).sum() > 0


@pytest.mark.parametrize("name", SCATTER_GOLDEN)
@pytest.mark.parametrize("kind", KINDS)
def test_scatter_fp32_bit_exact_and_fp64_vs_reference_golden(name, kind):
    p, z = load_scatter_golden(name)
    bm = z["bitmap_crystal"] if kind == "crystal" else z["bitmap_collimator"]
    rot = int(z["rotation"])
    f32 = oracle_py.oracle_scatter_entries(p, kind, z["rows"], z["voxels"], bm, z["pe"], mode="fp32", rotation=rot)
    assert np.array_equal(f32, z["ref_%s_f32" % kind])
    f64 = oracle_py.oracle_scatter_entries(p, kind, z["rows"], z["voxels"], bm, z["pe"], mode="fp64", rotation=rot)
    ref = z["ref_%s_f64" % kind]
    assert (ref != 0).sum() > 0
    assert rel_err(f64, ref).max() <= 1e-12


def test_scatter_points_one_equals_reference_and_refinement_converges():
    p, z = load_scatter_golden("mid")
    rows, vox = z["rows"][:48], z["voxels"][:48]
    bm = z["bitmap_crystal"]
    one = oracle_py.oracle_scatter_entries(p, "crystal", rows, vox, bm, z["pe"], sp=(1, 1, 1))
    assert np.array_equal(one, z["ref_crystal_f64"][:48])
    a = oracle_py.oracle_scatter_entries(p, "crystal", rows, vox, bm, z["pe"], sp=(2, 4, 2))
    b = oracle_py.oracle_scatter_entries(p, "crystal", rows, vox, bm, z["pe"], sp=(4, 8, 4))
    nz = b != 0
    assert nz.sum() > 10
    # finer splits move the result less than the first split did
    assert np.median(np.abs(a[nz] - b[nz]) / b[nz]) < np.median(np.abs(one[nz] - b[nz]) / b[nz])


needs_ref = pytest.mark.skipif(not oracle_py.ref_available("scatter_f32"),
                               reason="oracle/_ref not built (no reference tree)")


@needs_ref
def test_compton_integral_bit_exact_vs_reference_build():
    rng = np.random.default_rng(3)
    lo = rng.uniform(0, 3.0, 400).astype(np.float32)
    hi = (lo + rng.uniform(0, 3.14 - lo)).astype(np.float32)
    args = np.stack([np.full(400, 140.5, np.float32), lo, hi], axis=1)
    assert np.array_equal(oracle_py.oracle_compton_integral(args, "fp32"), oracle_py.ref_compton_integral(args, "f32"))
    assert rel_err(oracle_py.oracle_compton_integral(args, "fp64"), oracle_py.ref_compton_integral(args, "f64")).max() <= 1e-12


@needs_ref
@pytest.mark.parametrize("kind", KINDS)
def test_scatter_vs_reference_build_random_cells(kind):
    p = configs.two_plates_small(seed=9)
    p.sv = (1, 1, 1)
    N, V = p.n_crystals, p.n_voxels
    rng = np.random.default_rng(11)
    pe = rng.uniform(0, 1e-4, (N, V)).astype(np.float32) * (rng.uniform(size=(N, V)) < 0.3)
    bm = oracle_py.ref_bitmap_crystal(p) if kind == "crystal" else oracle_py.ref_bitmap_collimator(p)
    rows = rng.integers(0, N, 24)
    vox = rng.integers(0, V, 24)
    a = oracle_py.oracle_scatter_entries(p, kind, rows, vox, bm, pe, mode="fp32")
    b = oracle_py.ref_scatter_entries(p, kind, rows, vox, bm, pe, "f32")
    assert np.array_equal(a, b)
