"""Beam masks, beam properties and MPXI (sm_beam_metrics, sysmat_b200.beams)
against the reference's own post-processing scripts.

Golden fixtures (tests/golden/make_golden.py beams):
* beams_reference.npz: extract_beam_prop_masks.py and compute_mpxi_3d.py run
  unmodified on a synthetic 60 x 5632 x 4096 sysmat whose rows cycle through a
  29-row pool (photoelectric rows, an all-zero row, a row with entries exactly
  at the threshold): the pool's masks, rotation 0's beam properties, its MPXI
  and the summary of that MPXI.
* mpxi_shipped_rot000.npz: the MPXI volume the reference ships and the summary
  text its script wrote for it.

Masks, counts and MPXI are integer results and must match exactly; row sums
are float32 in the reference (numpy's pairwise sum) and double here, so the
property column holding them matches to 1e-6 relative.
"""
import os

import numpy as np
import pytest

import oracle_beams
from helpers import GOLDEN
from sysmat_b200 import beams


@pytest.fixture(scope="module")
def ref():
    return np.load(os.path.join(GOLDEN, "beams_reference.npz"))


def rotation0_block(ref):
    n_rot, n_det, n_vox = (int(v) for v in ref["dims"])
    pool = ref["pool"]
    return pool[np.arange(n_det) % len(pool)], n_rot


# ---- the oracle against the reference's scripts --------------------------------

def test_oracle_masks_properties_mpxi_match_reference_scripts(ref):
    block, n_rot = rotation0_block(ref)
    mx, sums, mask = oracle_beams.beam_rows(block)
    assert np.array_equal(mask[:len(ref["pool"])], ref["pool_masks"])
    props = oracle_beams.properties(0, n_rot, sums, mask.sum(axis=1))
    assert np.array_equal(props, ref["props_rot0"])
    vol = oracle_beams.mpxi(mask)
    assert np.array_equal(vol.reshape(ref["mpxi_rot0"].shape), ref["mpxi_rot0"])
    s = oracle_beams.summarize(ref["mpxi_rot0"])
    assert [s[k] for k in ("num_voxels_sampled", "num_voxels_unsampled", "num_voxels_nonmultiplexed",
                           "num_voxels_multiplexed", "max_mpxi")] == ref["summary_scalars"].tolist()
    assert np.allclose([s["mean_mpxi_all_voxels"], s["mean_mpxi_sampled_voxels"], s["median_mpxi_sampled_voxels"]],
                       ref["summary_means"], rtol=0, atol=0)
    assert np.array_equal(np.asarray(s["histogram"]), ref["summary_hist"])


# ---- host-side product functions --------------------------------------------------

def test_beam_properties_match_reference_records(ref):
    block, n_rot = rotation0_block(ref)
    _, sums, mask = oracle_beams.beam_rows(block)
    props = beams.beam_properties(0, n_rot, sums.astype(np.float64), mask.sum(axis=1))
    assert np.array_equal(props, ref["props_rot0"])
    later = beams.beam_properties(7, n_rot, sums.astype(np.float64), mask.sum(axis=1), first_row=0)
    assert np.all(later[:, 0] == 7) and np.allclose(later[:, 3], np.float32(7 * 2 * np.pi / 60))


def test_mpxi_summary_text_reproduces_the_shipped_summary_file():
    z = np.load(os.path.join(GOLDEN, "mpxi_shipped_rot000.npz"))
    s = beams.mpxi_summary(z["mpxi"])
    assert beams.mpxi_summary_text(s, 0) == str(z["summary_text"])
    assert s == oracle_beams.summarize(z["mpxi"])


# ---- the GPU kernels -----------------------------------------------------------------

@pytest.mark.gpu
def test_beam_metrics_gpu_match_reference_scripts(ref):
    import torch
    block, n_rot = rotation0_block(ref)
    d = torch.from_numpy(block).cuda()
    for keep_mask in (True, False):
        m = beams.beam_metrics(d, keep_mask=keep_mask)
        torch.cuda.synchronize()
        counts = m["row_count"].cpu().numpy()
        mx, sums, mask = oracle_beams.beam_rows(block)
        assert np.array_equal(m["row_max"].cpu().numpy(), mx)
        assert np.array_equal(counts, mask.sum(axis=1))
        if keep_mask:
            assert np.array_equal(m["mask"].cpu().numpy(), mask)
            assert np.array_equal(m["mask"][:len(ref["pool"])].cpu().numpy(), ref["pool_masks"])
        vol = m["mpxi"].cpu().numpy().view(np.uint32).reshape(ref["mpxi_rot0"].shape)
        assert np.array_equal(vol, ref["mpxi_rot0"])
        props = beams.beam_properties(0, n_rot, m["row_sum"].cpu().numpy(), counts)
        want = ref["props_rot0"]
        assert props.shape == want.shape
        cols = [c for c in range(11) if c != 7]
        assert np.array_equal(props[:, cols], want[:, cols])
        np.testing.assert_allclose(props[:, 7], want[:, 7], rtol=1e-6, atol=0)


@pytest.mark.gpu
def test_beam_metrics_gpu_on_a_computed_sysmat_every_layout():
    """A PE sysmat computed on the device, checked through the vector path, an
    odd row pitch (scalar path) and the MPXI read from the sysmat itself."""
    import torch
    import sysmat_b200
    from sysmat_b200 import configs
    p = configs.two_plates_small()
    ctx = sysmat_b200.Context(0)
    g = sysmat_b200.Geometry(ctx, p)
    A = g.pe()
    g.close()
    ctx.close()
    mx, sums, mask = oracle_beams.beam_rows(A)
    want_mpxi = oracle_beams.mpxi(mask)
    V = A.shape[1]
    for pitch in (V, V + 3):
        buf = torch.zeros((A.shape[0], pitch), dtype=torch.float32, device="cuda:0")
        buf[:, :V] = torch.from_numpy(A).cuda()
        for keep_mask in (True, False):
            m = beams.beam_metrics(buf[:, :V], keep_mask=keep_mask)
            torch.cuda.synchronize()
            assert np.array_equal(m["row_max"].cpu().numpy(), mx)
            assert np.array_equal(m["row_count"].cpu().numpy(), mask.sum(axis=1))
            assert np.array_equal(m["mpxi"].cpu().numpy().view(np.uint32), want_mpxi)
            np.testing.assert_allclose(m["row_sum"].cpu().numpy(), A.astype(np.float64).sum(axis=1), rtol=1e-12)
            if keep_mask:
                assert np.array_equal(m["mask"].cpu().numpy(), mask)


@pytest.mark.gpu
def test_sysmat_file_metrics_pipeline(tmp_path):
    """A two-rotation .sysmat file through the file pipeline, in chunks of a
    few rows, against the oracle on the whole file."""
    import sysmat_b200
    from sysmat_b200 import configs
    p = configs.tiny(seed=4, rotated=True)
    ctx = sysmat_b200.Context(0)
    g = sysmat_b200.Geometry(ctx, p)
    mats = [g.pe(rotation=r) for r in range(2)]
    g.close()
    ctx.close()
    path = tmp_path / "PE.sysmat"
    np.concatenate(mats).astype(np.float32).tofile(path)
    out = tmp_path / "out"
    chunk = 4 * p.n_voxels * 5          # 5 rows per chunk: the last chunk of each rotation is short
    r = beams.sysmat_file_metrics(str(path), 2, p.n_crystals, p.grid, str(out), chunk_bytes=chunk)
    masks = np.load(out / "beam_masks.npy")
    props = np.load(out / "beam_properties.npy")
    want_props = []
    for rot in range(2):
        _, sums, mask = oracle_beams.beam_rows(mats[rot])
        assert np.array_equal(masks[rot * p.n_crystals:(rot + 1) * p.n_crystals], mask)
        vol = np.load(out / ("mpxi_3d_rot_%03d.npy" % rot))
        nx, ny, nz = p.grid
        assert vol.shape == (nz, ny, nx) and np.array_equal(vol.ravel(), oracle_beams.mpxi(mask))
        text = open(out / ("mpxi_3d_rot_%03d_summary.txt" % rot)).read()
        assert text.startswith("3D MPXI Summary | Rotation %d" % rot)
        want_props.append(oracle_beams.properties(rot, 2, sums, mask.sum(axis=1)))
    want_props = np.concatenate(want_props)
    assert r["active_beams"] == len(want_props) == len(props)
    assert np.array_equal(props[:, :7], want_props[:, :7])
    np.testing.assert_allclose(props[:, 7], want_props[:, 7], rtol=1e-6)
