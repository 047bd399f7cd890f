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
