"""Error paths on the GPU that fault nothing: capacity overflow reported
through the device status word, and the tensor-core GEMM's bounded waits.

Capacity: the tracer stages each tile's candidate crystals and holes in
shared memory (at most 1024 crystals / 384 holes per tile, 512 / 128 per
voxel).  A kernel that meets more drops nothing silently: it skips the extra
entries' stores (every index stays in bounds), sets a bit of its device status
word, and the host turns that bit into SM_ERR_CAPACITY.  The geometry below
has a plate drilled with 3600 holes at 0.2 mm pitch, so every voxel sees far
more than 128 candidate holes.
"""
import numpy as np
import pytest

import sysmat_b200
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


@pytest.fixture(scope="module")
def ctx():
    c = sysmat_b200.Context(0)
    yield c
    c.close()


def test_candidate_overflow_is_capacity_error_host_output(ctx):
    g = sysmat_b200.Geometry(ctx, dense_holes())
    with pytest.raises(sysmat_b200.SysmatError) as e:
        g.pe()
    g.close()
    assert e.value.code == -2 and "candidate" in str(e.value)


def test_candidate_overflow_is_capacity_error_at_sync(ctx):
    import torch
    torch.cuda.set_device(0)
    p = dense_holes()
    g = sysmat_b200.Geometry(ctx, p)
    out = torch.zeros((p.n_crystals, p.n_voxels), dtype=torch.float32, device="cuda:0")
    g.pe(out=out.data_ptr())                 # device output: asynchronous, returns before the kernel ends
    with pytest.raises(sysmat_b200.SysmatError) as e:
        ctx.sync()
    assert e.value.code == -2
    ctx.sync()                               # the status word was cleared: the context stays usable
    ok = sysmat_b200.Geometry(ctx, sysmat_b200.configs.tiny())
    assert (ok.pe() != 0).any()
    ok.close()
    g.close()


def test_candidate_overflow_is_capacity_error_static_entry():
    import torch
    torch.cuda.set_device(0)
    p = dense_holes()
    dst = torch.zeros((p.n_crystals, p.n_voxels), dtype=torch.float32, device="cuda:0")
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.pe_compute_static(p, dst.data_ptr(), p.n_voxels)
    assert e.value.code == -2 and "candidate" in str(e.value)


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
