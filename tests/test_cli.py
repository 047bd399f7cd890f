"""The command-line generators (gpu-spect-pet-sysmat_b200/bin/), run as the
reference's CLIs are run: Params_*.dat in the working directory, the same
flags, the same output files and layout ([rotation][crystal][voxel] float32)."""
import os
import subprocess

import numpy as np
import pytest

import sysmat_b200
from sysmat_b200 import configs

BIN = os.path.abspath(os.path.join(os.path.dirname(sysmat_b200.__file__), "..", "bin"))


def run(tool, args, cwd):
    return subprocess.run([os.path.join(BIN, tool)] + list(args), cwd=cwd, capture_output=True, text=True, timeout=600)


def shift_name(prefix, p):
    return "%s_shift_%f_%f_%f.sysmat" % (prefix, p.image[8], p.image[9], p.image[10])


@pytest.mark.parametrize("tool", ["PEGen_CircularHole", "ScatterGen_CircularHole", "ScatterGen_Crystal",
                                  "ScatterGen_Collimator"])
def test_help_and_unknown_flags(tool, tmp_path):
    configs.tiny().write_dat(str(tmp_path))
    r = run(tool, ["-h"], tmp_path)
    assert r.returncode == 0 and "Usage" in r.stdout
    r = run(tool, ["-bogus"], tmp_path)
    assert r.returncode != 0 and "Unknown parameter" in r.stderr


def test_missing_params_file_is_reported(tmp_path):
    r = run("PEGen_CircularHole", [], tmp_path)
    assert r.returncode != 0 and "Params_Collimator.dat" in r.stderr


@pytest.mark.gpu
def test_pegen_and_scattergen_files(tmp_path):
    p = configs.tiny(seed=4, rotated=True)          # 2 rotations, rotated crystals, shifted FOV
    p.write_dat(str(tmp_path))
    r = run("PEGen_CircularHole", ["-cuda", "0"], tmp_path)
    assert r.returncode == 0, r.stderr
    N, V = p.n_crystals, p.n_voxels
    pe = np.fromfile(tmp_path / shift_name("PE_SysMat", p), np.float32).reshape(2, N, V)
    ctx = sysmat_b200.Context(0)
    g = sysmat_b200.Geometry(ctx, p)
    ref_opts = sysmat_b200.PeOptions.make((1, 1, 1), (8, 16, 8))
    for rot in range(2):
        assert np.array_equal(pe[rot], g.pe(rotation=rot, opts=ref_opts))
    # combined scatter generator: computes and writes the bitmaps, then the sysmats
    r = run("ScatterGen_CircularHole", [], tmp_path)
    assert r.returncode == 0, r.stderr
    sc = np.fromfile(tmp_path / shift_name("Scatter_SysMat", p), np.float32).reshape(2, N, V)
    full = np.fromfile(tmp_path / shift_name("SysMat_withScatter", p), np.float32).reshape(2, N, V)
    for rot in range(2):
        assert np.array_equal(sc[rot], g.scatter(pe=pe[rot], rotation=rot))
    assert np.array_equal(full, pe + sc)
    assert (tmp_path / "GeometryRelationShip_Crystal2Crystal").exists()
    # reading the bitmaps back gives the same matrix
    os.rename(tmp_path / "GeometryRelationShip_Crystal2Crystal", tmp_path / "gc")
    os.rename(tmp_path / "GeometryRelationShip_Collimator2Crystal", tmp_path / "gh")
    os.remove(tmp_path / shift_name("Scatter_SysMat", p))
    r = run("ScatterGen_CircularHole", ["-GeoCrystal", "gc", "-GeoCollimator", "gh"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert np.array_equal(np.fromfile(tmp_path / shift_name("Scatter_SysMat", p), np.float32).reshape(2, N, V), sc)
    # single-part generators
    r1 = run("ScatterGen_Crystal", ["-GeoCrystal", "gc"], tmp_path)
    r2 = run("ScatterGen_Collimator", ["-GeoCollimator", "gh"], tmp_path)
    assert r1.returncode == 0 and r2.returncode == 0, r1.stderr + r2.stderr
    c = np.fromfile(tmp_path / shift_name("Scatter_Crystal_SysMat", p), np.float32).reshape(2, N, V)
    h = np.fromfile(tmp_path / shift_name("Scatter_SysMat", p), np.float32).reshape(2, N, V)
    np.testing.assert_allclose(sc, c.astype(np.float64) + h, rtol=1e-6, atol=0)
    g.close()
    ctx.close()


@pytest.mark.gpu
def test_scattergen_surrogate_flag(tmp_path):
    """`-surrogate TOL`: the same files, the crystal part through the scatter
    surrogate (exact collimator part, exact recompute of rows over TOL)."""
    p = configs.tiny(seed=4, rotated=True)
    p.write_dat(str(tmp_path))
    assert run("PEGen_CircularHole", ["-cuda", "0"], tmp_path).returncode == 0
    N, V = p.n_crystals, p.n_voxels
    assert run("ScatterGen_CircularHole", [], tmp_path).returncode == 0
    exact = np.fromfile(tmp_path / shift_name("Scatter_SysMat", p), np.float32).reshape(2, N, V)
    os.remove(tmp_path / shift_name("Scatter_SysMat", p))
    r = run("ScatterGen_CircularHole", ["-surrogate", "0.01"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "rows recomputed" in r.stdout
    sur = np.fromfile(tmp_path / shift_name("Scatter_SysMat", p), np.float32).reshape(2, N, V)
    pe = np.fromfile(tmp_path / shift_name("PE_SysMat", p), np.float32).reshape(2, N, V)
    full = np.fromfile(tmp_path / shift_name("SysMat_withScatter", p), np.float32).reshape(2, N, V)
    assert np.isfinite(sur).all()
    np.testing.assert_array_equal(full, pe + sur)
    for rot in range(2):
        num = np.sqrt(((sur[rot].astype(np.float64) - exact[rot]) ** 2).sum(1))
        den = np.sqrt((exact[rot].astype(np.float64) ** 2).sum(1))
        err = num[den > 0] / den[den > 0]
        assert np.median(err) <= 0.01 and err.max() <= 0.05, (np.median(err), err.max())
    r = run("ScatterGen_CircularHole", ["-surrogate", "0"], tmp_path)
    assert r.returncode != 0


@pytest.mark.gpu
def test_bitmap_files_carry_a_geometry_hash(tmp_path):
    """Bitmap files come with "<file>.geohash"; a -Geo* file whose hash names
    another geometry is recomputed (the reference would reuse it); a file with
    no .geohash is read as the reference reads it."""
    p = configs.tiny(seed=4, rotated=True)
    p.write_dat(str(tmp_path))
    assert run("PEGen_CircularHole", [], tmp_path).returncode == 0
    r = run("ScatterGen_CircularHole", [], tmp_path)
    assert r.returncode == 0, r.stderr
    ctx = sysmat_b200.Context(0)
    g = sysmat_b200.Geometry(ctx, p)
    hc, hh = g.bitmap_hashes()
    g.close()
    for name, h, kind in (("GeometryRelationShip_Crystal2Crystal", hc, "crystal"),
                          ("GeometryRelationShip_Collimator2Crystal", hh, "collimator")):
        text = (tmp_path / (name + ".geohash")).read_text()
        assert text.startswith("sysmat_b200-bitmap-v1 %s " % kind) and ("fnv1a64=%016x" % h) in text
    for a, b in (("GeometryRelationShip_Crystal2Crystal", "gc"), ("GeometryRelationShip_Collimator2Crystal", "gh")):
        os.rename(tmp_path / a, tmp_path / b)
        os.rename(tmp_path / (a + ".geohash"), tmp_path / (b + ".geohash"))
    r = run("ScatterGen_CircularHole", ["-GeoCrystal", "gc", "-GeoCollimator", "gh"], tmp_path)
    assert r.returncode == 0 and "another geometry" not in r.stderr
    # move one crystal: the PE sysmat and both bitmaps change
    q = p.copy()
    q.detector = q.detector.copy()
    q.detector[1 + 12 * 3] += 0.7
    q.write_dat(str(tmp_path))
    assert run("PEGen_CircularHole", [], tmp_path).returncode == 0
    stale_c, stale_h = (tmp_path / "gc").read_bytes(), (tmp_path / "gh").read_bytes()
    r = run("ScatterGen_CircularHole", ["-GeoCrystal", "gc", "-GeoCollimator", "gh"], tmp_path)
    assert r.returncode == 0, r.stderr
    # once per file: the first rotation refreshes both files, the second reads them
    assert r.stderr.count("computed for another geometry") == 2
    N, V = q.n_crystals, q.n_voxels
    pe = np.fromfile(tmp_path / shift_name("PE_SysMat", q), np.float32).reshape(2, N, V)
    sc = np.fromfile(tmp_path / shift_name("Scatter_SysMat", q), np.float32).reshape(2, N, V)
    g = sysmat_b200.Geometry(ctx, q)
    for rot in range(2):
        assert np.array_equal(sc[rot], g.scatter(pe=pe[rot], rotation=rot))
    fresh_c, fresh_h = g.scatter_bitmaps()
    g.close()
    assert (tmp_path / "gc").read_bytes() == fresh_c.tobytes() != stale_c
    assert (tmp_path / "gh").read_bytes() == fresh_h.tobytes()
    # without .geohash a file is taken as it is (the reference's behaviour)
    (tmp_path / "gc").write_bytes(stale_c)
    os.remove(tmp_path / "gc.geohash")
    r = run("ScatterGen_CircularHole", ["-GeoCrystal", "gc", "-GeoCollimator", "gh"], tmp_path)
    assert r.returncode == 0 and "another geometry" not in r.stderr
    assert (tmp_path / "gc").read_bytes() == stale_c
    ctx.close()


@pytest.mark.gpu
def test_pegen_rotations_as_items_of_one_launch(tmp_path):
    """Several rotations go through one persistent launch (sm_pe_batch with
    per-item rotations); the file equals sm_pe_compute per rotation."""
    p = configs.tiny(seed=2, rotated=True)
    p.image = p.image.copy()
    p.image[6] = 5
    p.image[7] = 0.2
    p.write_dat(str(tmp_path))
    r = run("PEGen_CircularHole", ["-sv", "2", "1", "2", "-sc", "2", "4", "2"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Rotations (0..4) processing in one launch" in r.stdout
    N, V = p.n_crystals, p.n_voxels
    pe = np.fromfile(tmp_path / shift_name("PE_SysMat", p), np.float32).reshape(5, N, V)
    ctx = sysmat_b200.Context(0)
    g = sysmat_b200.Geometry(ctx, p)
    opts = sysmat_b200.PeOptions.make((2, 1, 2), (2, 4, 2))
    for rot in range(5):
        assert np.array_equal(pe[rot], g.pe(rotation=rot, opts=opts)), rot
    assert len({pe[r].tobytes() for r in range(5)}) == 5
    g.close()
    ctx.close()
