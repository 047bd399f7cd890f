"""GPU parity of the primary-Compton scatter kernels, through the C ABI.

Oracles: the reference's own scatter kernels built for the host (golden
fixtures in tests/golden/scatter_*.npz: bitmaps, and f64 values of
crystalScatterSysMatCuda / collimatorScatterSysMatCuda), and the CPU
restatement in oracle/ (fp64) for scatter points and for samples of the
full-size workload.

Tolerances, relative error on nonzero entries:
* bitmaps: identical words (the reference's single-precision test);
* values vs FP64: median <= 1e-5, 99th percentile <= 1e-4, maximum <= 1e-3
  (measured on these fixtures and samples: median ~1e-7, maximum ~1e-5).  An
  entry sums up to N x points terms, and a term that sits on one of the
  reference's hard edges (the 2-sigma energy-window cut, the floor in the
  0.01 rad Klein-Nishina rectangle sum, the theta_min = 0 switch) can be decided
  differently in FP32 and FP64; the maximum leaves room for one such term, and
  at most 1% of the entries may exceed 1e-4.
* zero pattern: an entry is zero exactly when the oracle's is, except where
  the oracle's value is below 1e-6 of the row's maximum.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle_py
import sysmat_b200
from helpers import load_scatter_golden, rel_err
from sysmat_b200 import configs

pytestmark = pytest.mark.gpu

MEDIAN = 1e-5
P99 = 1e-4
MAX = 1e-3
FRAC_ABOVE = 0.01


@pytest.fixture(scope="module")
def ctx():
    c = sysmat_b200.Context(0)
    yield c
    c.close()


def check_values(got, ref, what):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    err = rel_err(got, ref)
    assert err.size > 0, what
    stats = "median %.3g p99 %.3g max %.3g above1e-4 %.4f (n=%d)" % (
        np.median(err), np.quantile(err, 0.99), err.max(), (err > 1e-4).mean(), err.size)
    assert np.median(err) <= MEDIAN, what + ": " + stats
    assert np.quantile(err, 0.99) <= P99, what + ": " + stats
    assert err.max() <= MAX, what + ": " + stats
    assert (err > 1e-4).mean() <= FRAC_ABOVE, what + ": " + stats
    scale = np.max(np.abs(ref)) if ref.size else 0.0
    flip = (got == 0) != (ref == 0)
    assert not np.any(flip & (np.abs(ref) > 1e-6 * scale)), what + ": zero pattern differs"


# ---- bitmaps ---------------------------------------------------------------------

@pytest.mark.parametrize("name", ["tiny", "tiny_rot", "mid"])
def test_bitmaps_identical_to_reference(ctx, name):
    p, z = load_scatter_golden(name)
    g = sysmat_b200.Geometry(ctx, p)
    c, h = g.scatter_bitmaps()
    g.close()
    assert np.array_equal(c, z["bitmap_crystal"])
    assert np.array_equal(h, z["bitmap_collimator"])


# ---- values vs the reference's own kernels (golden) ---------------------------------

@pytest.mark.parametrize("name", ["tiny", "tiny_rot", "mid"])
@pytest.mark.parametrize("kind", ["crystal", "collimator"])
def test_scatter_vs_reference_golden(ctx, name, kind):
    p, z = load_scatter_golden(name)
    g = sysmat_b200.Geometry(ctx, p)
    A = g.scatter(pe=z["pe"], rotation=int(z["rotation"]), parts=kind)
    g.close()
    check_values(A[z["rows"], z["voxels"]], z["ref_%s_f64" % kind], "%s/%s" % (name, kind))


def test_both_parts_are_the_sum(ctx):
    p, z = load_scatter_golden("mid")
    g = sysmat_b200.Geometry(ctx, p)
    a = g.scatter(pe=z["pe"], parts="crystal")
    b = g.scatter(pe=z["pe"], parts="collimator")
    both = g.scatter(pe=z["pe"], parts="both")
    g.close()
    np.testing.assert_allclose(both, a.astype(np.float64) + b, rtol=1e-6, atol=0)


def test_reference_bitmaps_from_files_give_same_result(ctx):
    p, z = load_scatter_golden("tiny_rot")
    g = sysmat_b200.Geometry(ctx, p)
    a = g.scatter(pe=z["pe"], rotation=1)
    b = g.scatter(pe=z["pe"], rotation=1, bitmaps=(z["bitmap_crystal"], z["bitmap_collimator"]))
    g.close()
    assert np.array_equal(a, b)


# ---- scatter points and decomposition -------------------------------------------------

def test_scatter_points_vs_oracle(ctx):
    p, z = load_scatter_golden("mid")
    g = sysmat_b200.Geometry(ctx, p)
    A = g.scatter(pe=z["pe"], sp=(2, 4, 2), parts="crystal")
    g.close()
    rng = np.random.default_rng(2)
    rows = rng.integers(0, p.n_crystals, 96)
    vox = rng.integers(0, p.n_voxels, 96)
    ref = oracle_py.oracle_scatter_entries(p, "crystal", rows, vox, z["bitmap_crystal"], z["pe"], sp=(2, 4, 2))
    check_values(A[rows, vox], ref, "mid sp=2x4x2")


def test_row_ranges_and_device_output_match(ctx):
    import torch
    p, z = load_scatter_golden("mid")
    g = sysmat_b200.Geometry(ctx, p)
    full = g.scatter(pe=z["pe"], sp=(1, 2, 1))
    part = g.scatter(pe=z["pe"], sp=(1, 2, 1), rows=(37, 101))
    assert np.array_equal(part, full[37:101])
    V = p.n_voxels
    d_pe = torch.from_numpy(z["pe"]).cuda()
    d_out = torch.zeros((p.n_crystals, V), dtype=torch.float32, device="cuda")
    g.scatter(pe=d_pe.data_ptr(), sp=(1, 2, 1), out=d_out.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy(), full)
    g.close()


# ---- the reference's host entry points ------------------------------------------------

def test_legacy_scatter_writes_and_reads_bitmap_files(ctx, tmp_path):
    p, z = load_scatter_golden("tiny")
    g = sysmat_b200.Geometry(ctx, p)
    api = g.scatter(pe=z["pe"])
    g.close()
    N, V = p.n_crystals, p.n_voxels
    phy = p.physics.copy()
    phy[8] = phy[9] = 1.0
    fc, fh = str(tmp_path / "GeoCrystal"), str(tmp_path / "GeoCollimator")
    dst = np.zeros((N, V), np.float32)
    assert sysmat_b200.scatter_legacy("both", p.collimator, p.detector, p.image, phy, z["pe"], fc, fh, dst) == V
    assert np.array_equal(dst, api)
    assert np.array_equal(np.fromfile(fc, np.uint32), z["bitmap_crystal"])
    assert np.array_equal(np.fromfile(fh, np.uint32), z["bitmap_collimator"])
    phy[8] = phy[9] = 0.0
    dst2 = np.zeros((N, V), np.float32)
    assert sysmat_b200.scatter_legacy("both", p.collimator, p.detector, p.image, phy, z["pe"], fc, fh, dst2) == V
    assert np.array_equal(dst2, api)
    # the combined entry point is the sum of the two single-part ones
    c = np.zeros((N, V), np.float32)
    h = np.zeros((N, V), np.float32)
    sysmat_b200.scatter_legacy("crystal", None, p.detector, p.image, phy, z["pe"], fc, None, c)
    sysmat_b200.scatter_legacy("collimator", p.collimator, p.detector, p.image, phy, None, None, fh, h)
    np.testing.assert_allclose(api, c.astype(np.float64) + h, rtol=1e-6, atol=0)


def test_single_part_shim_libraries(ctx, tmp_path):
    p, z = load_scatter_golden("tiny")
    N, V = p.n_crystals, p.n_voxels
    phy = p.physics.copy()
    phy[8] = phy[9] = 1.0
    libdir = os.path.dirname(sysmat_b200.LIB_PATH)
    f32p = ctypes.POINTER(ctypes.c_float)
    ptr = lambda a: a.ctypes.data_as(f32p)  # noqa: E731
    det = np.ascontiguousarray(p.detector, np.float32)
    col = np.ascontiguousarray(p.collimator, np.float32)
    img = np.ascontiguousarray(p.image, np.float32)
    pe = np.ascontiguousarray(z["pe"], np.float32)
    lc = ctypes.CDLL(os.path.join(libdir, "libsysmat_b200_scatter_crystal.so"))
    c = np.zeros((N, V), np.float32)
    assert lc.scatter(ptr(det), ptr(img), ptr(phy), ptr(pe), str(tmp_path / "gc").encode(), ptr(c), 0) == V
    lh = ctypes.CDLL(os.path.join(libdir, "libsysmat_b200_scatter_collimator.so"))
    h = np.zeros((N, V), np.float32)
    assert lh.scatter(ptr(col), ptr(det), ptr(img), ptr(phy), ptr(pe), str(tmp_path / "gh").encode(), ptr(h), 0) == V
    g = sysmat_b200.Geometry(ctx, p)
    assert np.array_equal(c, g.scatter(pe=z["pe"], parts="crystal"))
    assert np.array_equal(h, g.scatter(pe=z["pe"], parts="collimator"))
    g.close()


def test_missing_bitmap_file_is_an_error_not_an_exit(ctx, tmp_path):
    p, z = load_scatter_golden("tiny")
    phy = p.physics.copy()
    phy[8] = phy[9] = 0.0
    dst = np.zeros((p.n_crystals, p.n_voxels), np.float32)
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.scatter_legacy("both", p.collimator, p.detector, p.image, phy, z["pe"],
                                   str(tmp_path / "absent"), str(tmp_path / "absent2"), dst)
    assert e.value.code == -5


# ---- full-size workload, sampled ---------------------------------------------------

def test_scatter_small_full_size_sampled_vs_oracle(ctx):
    """[2048 x 16384] crystal + collimator scatter with 2 x 4 x 2 scatter points;
    48 sampled entries against the FP64 oracle (the oracle is fed the GPU's
    bitmaps, which are pinned bit-exact above)."""
    import torch
    p = configs.scatter_small()
    g = sysmat_b200.Geometry(ctx, p)
    N, V = p.n_crystals, p.n_voxels
    d_pe = torch.zeros((N, V), dtype=torch.float32, device="cuda")
    g.pe(opts=g.options(sv=(1, 1, 1), sc=(2, 4, 2)), out=d_pe.data_ptr())
    d_out = torch.zeros((N, V), dtype=torch.float32, device="cuda")
    g.scatter(pe=d_pe.data_ptr(), sp=(2, 4, 2), parts="both", out=d_out.data_ptr())
    torch.cuda.synchronize()
    ctx.sync()
    out = d_out.cpu().numpy()
    pe = d_pe.cpu().numpy()
    bc, bh = g.scatter_bitmaps()
    g.close()
    assert np.isfinite(out).all() and (out >= 0).all()
    rng = np.random.default_rng(4)
    # entries where the crystal part can be nonzero: rows of the back layer, voxels some source sees
    seen = np.flatnonzero(pe.any(axis=0))
    rows = rng.integers(N // 2, N, 48)
    vox = rng.choice(seen, 48)
    ref = oracle_py.oracle_scatter_entries(p, "crystal", rows, vox, bc, pe, sp=(2, 4, 2))
    ref = ref + oracle_py.oracle_scatter_entries(p, "collimator", rows, vox, bh, None)
    check_values(out[rows, vox], ref, "scatter_small")


# ---- subsets: the surrogate's re-check and recompute path ---------------------------

def test_subset_rows_and_columns_match_full_matrix(ctx):
    """Row-list and voxel-column modes give exactly the corresponding entries
    of the full matrix (same kernels, same per-entry sums)."""
    import torch
    p, z = load_scatter_golden("mid")
    g = sysmat_b200.Geometry(ctx, p)
    nx, ny, nz = p.grid
    N, V = p.n_crystals, p.n_voxels
    d_pe = torch.from_numpy(z["pe"]).cuda()
    full = g.scatter(pe=z["pe"], sp=(1, 2, 1), parts="both")
    rng = np.random.default_rng(11)
    rows = rng.choice(N, 45, replace=False)
    cols = np.stack([rng.integers(0, nx, 13), rng.integers(0, nz, 13)], 1)
    # rows x all voxels, caller's order kept
    out = torch.full((rows.size, V), float("nan"), device="cuda")
    g.scatter_subset(d_pe.data_ptr(), rows, out.data_ptr(), sp=(1, 2, 1), parts="both")
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), full[rows])
    # rows x voxel columns (repeated columns allowed)
    cols = np.concatenate([cols, cols[:2]])
    out = torch.full((rows.size, cols.shape[0] * ny), float("nan"), device="cuda")
    g.scatter_subset(d_pe.data_ptr(), rows, out.data_ptr(), cols=cols, sp=(1, 2, 1), parts="both")
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(rows.size, cols.shape[0], ny)
    ys = np.arange(ny)
    vox = cols[:, 0][:, None] + nx * (ys[None, :] + ny * cols[:, 1][:, None])     # [c][y]
    assert np.array_equal(got, full[rows][:, vox])
    g.close()


def test_subset_rejects_repeated_rows_and_bad_columns(ctx):
    import torch
    p, z = load_scatter_golden("tiny")
    g = sysmat_b200.Geometry(ctx, p)
    d_pe = torch.from_numpy(z["pe"]).cuda()
    out = torch.zeros((4, p.n_voxels), device="cuda")
    with pytest.raises(sysmat_b200.SysmatError):
        g.scatter_subset(d_pe.data_ptr(), [1, 2, 1], out.data_ptr())
    with pytest.raises(sysmat_b200.SysmatError):
        g.scatter_subset(d_pe.data_ptr(), [1, 2], out.data_ptr(), cols=[(p.grid[0], 0)])
    g.close()
