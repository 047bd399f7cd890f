"""Paths that are rare by construction, on the GPU, none of which faults:
candidate sets larger than the shared-memory lists, the device status word,
and the tensor-core GEMM's bounded waits.

Candidates: the tracer stages each tile's candidate crystals and holes in
shared memory (at most 1024 crystals / 384 holes per tile, 512 / 128 per
voxel).  A voxel whose candidates do not fit is traced with its candidates
read straight from the geometry tables: same decisions, same values.  The
geometry below has a plate drilled with 3600 holes at 0.2 mm pitch, so every
voxel sees far more than 128 candidate holes (the reference's own per-plate
list holds 1000, PESysMatGen.cu:485).

Status word: a ray that crosses more crystals than a hit record holds (40) in
record mode sets a bit of the device status word, which the host turns into
SM_ERR_CAPACITY; the context stays usable.
"""
import numpy as np
import pytest

import oracle_py
import sysmat_b200
from helpers import rel_err
from sysmat_b200.params import Params, Plate, build_collimator, build_detector, build_image, build_physics, \
    crystal_layer, grid_holes

pytestmark = pytest.mark.gpu

CZT = (0.35, 0.28, 0.07)


def dense_holes():
    holes = grid_holes(60, 60, 0.2, 0.08, 4.0, 0.0)
    col = build_collimator([Plate(40.0, 4.0, 40.0, 0.0, 3.5, 3.2, 0.3, holes)])
    det = build_detector(crystal_layer(4, 4, 2.0, (2.0, 4.0, 2.0), 14.0, CZT))
    img = build_image((4, 4, 4), (2.0, 2.0, 2.0), fov_to_plate0=20.0)
    return Params(col, det, img, build_physics(), sv=(1, 1, 1), sc=(2, 4, 2), name="dense_holes")


def crystal_stack(n=48):
    """n crystals of 1 x 0.3 x 1 mm stacked along the axis, 0.4 mm apart: a ray
    to the last one crosses the n - 1 in front of it."""
    holes = grid_holes(1, 1, 4.0, 1.5, 2.0, 0.0)
    col = build_collimator([Plate(40.0, 2.0, 40.0, 0.0, 3.5, 3.2, 0.3, holes)])
    crystals = []
    for i in range(n):
        crystals += crystal_layer(1, 1, 1.2, (1.0, 0.3, 1.0), 10.0 + 0.4 * i, CZT)
    det = build_detector(crystals)
    img = build_image((2, 2, 2), (0.2, 0.2, 0.2), fov_to_plate0=20.0)
    return Params(col, det, img, build_physics(), sv=(1, 1, 1), sc=(1, 4, 1), name="crystal_stack")


@pytest.fixture(scope="module")
def ctx():
    c = sysmat_b200.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def dense(ctx):
    p = dense_holes()
    g = sysmat_b200.Geometry(ctx, p)
    A = g.pe()
    g.close()
    return p, A


def test_voxels_beyond_the_list_capacity_match_the_oracle(dense):
    """Every entry of the dense-hole geometry against the same-decision oracle
    (max 1e-4) and FP64 (median 1e-4, max 1e-3), identical zeros."""
    p, A = dense
    N, V = p.n_crystals, p.n_voxels
    rows, vox = np.repeat(np.arange(N), V), np.tile(np.arange(V), N)
    dual = oracle_py.oracle_pe_entries(p, rows, vox, "dual").reshape(N, V)
    fp64 = oracle_py.oracle_pe_entries(p, rows, vox, "fp64").reshape(N, V)
    assert (A != 0).sum() > 0.5 * A.size
    assert np.array_equal(A == 0, dual == 0)
    assert rel_err(A, dual).max() <= 1e-4
    e64 = rel_err(A, fp64)
    assert np.median(e64) <= 1e-4 and e64.max() <= 1e-3


def test_voxels_beyond_the_list_capacity_hit_lists(ctx, dense):
    p, A = dense
    rows = np.array([0, 5, 10, 15])
    vox = np.array([int(np.argmax(A[r])) for r in rows])
    g = sysmat_b200.Geometry(ctx, p)
    rec = g.record_hits(rows, vox)
    g.close()
    n_holes = 0
    for i in range(len(rows)):
        mine = sysmat_b200.parse_records(rec[i])
        ref = oracle_py.parse_hits(oracle_py.oracle_pe_hits(p, int(rows[i]), int(vox[i])))
        assert mine == ref, "entry (%d, %d)" % (rows[i], vox[i])
        n_holes += sum(len(h) for _, h, _ in ref.values())
    assert n_holes > 0


def test_voxels_beyond_the_list_capacity_device_output_and_static_entry(ctx, dense):
    """The same matrix through a device output (asynchronous) and through the
    entry point that allocates nothing."""
    import torch
    torch.cuda.set_device(0)
    p, A = dense
    g = sysmat_b200.Geometry(ctx, p)
    out = torch.zeros((p.n_crystals, p.n_voxels), dtype=torch.float32, device="cuda:0")
    g.pe(out=out.data_ptr())
    ctx.sync()
    g.close()
    assert np.array_equal(out.cpu().numpy(), A)
    dst = torch.zeros((p.n_crystals, p.n_voxels), dtype=torch.float32, device="cuda:0")
    sysmat_b200.pe_compute_static(p, dst.data_ptr(), p.n_voxels)
    assert np.array_equal(dst.cpu().numpy(), A)


def test_hit_record_overflow_is_capacity_error_and_context_stays_usable(ctx):
    p = crystal_stack()
    g = sysmat_b200.Geometry(ctx, p)
    last = p.n_crystals - 1
    with pytest.raises(sysmat_b200.SysmatError) as e:
        g.record_hits(np.array([last]), np.array([0]))
    assert e.value.code == -2 and "hit record" in str(e.value)
    rec = g.record_hits(np.array([0]), np.array([0]))   # the front crystal: nothing in front of it
    assert rec.shape[0] == 1
    A = g.pe()
    g.close()
    assert (A[last] > 0).any() and np.isfinite(A).all()


def test_gemm_wait_running_out_is_reported_skips_epilogue_and_frees_tensor_memory():
    """With a wait limit of 0 polls every bounded wait of the tensor-core GEMM
    gives up at once: the kernel sets the error word, writes nothing, waits for
    its own MMAs and frees its tensor memory; a GEMM launched afterwards with
    the default limit allocates tensor memory again and is correct."""
    import torch
    torch.manual_seed(5)
    m, n, k = 256, 256, 192
    a = torch.randn(m, k, device="cuda").bfloat16()
    b = torch.randn(n, k, device="cuda").bfloat16()
    c = torch.full((m, n), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    prev = sysmat_b200.tc_wait_limit(0)
    try:
        sysmat_b200.gemm_bf16(m, n, k, a.data_ptr(), (k, 1), b.data_ptr(), (k, 1), c.data_ptr(), n, n_tile=256,
                              error=err.data_ptr())
        torch.cuda.synchronize()
    finally:
        assert sysmat_b200.tc_wait_limit(-1) == 0
    assert prev == 1 << 26
    assert int(err.item()) == 1
    assert torch.isnan(c).all()            # epilogue skipped
    err.zero_()
    sysmat_b200.gemm_bf16(m, n, k, a.data_ptr(), (k, 1), b.data_ptr(), (k, 1), c.data_ptr(), n, n_tile=256,
                          error=err.data_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = a.float() @ b.float().T
    assert ((c - ref).abs() / ref.abs().amax(1, keepdim=True)).max().item() <= 1e-4
