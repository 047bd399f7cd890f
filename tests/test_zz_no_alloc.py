"""The photoelectric entry point that allocates no device memory.

``sm_pe_compute_static`` serves callers that cannot call cudaMalloc (a host
application whose own pool or arena owns all device memory, a plugin inside
such a process, code that must avoid the synchronisation cudaMalloc/cudaFree
can cause): its working memory is a fixed array inside the library.  These
tests call it through the C ABI and compare it with ``sm_pe_compute`` (the
allocating entry point, itself checked against the oracle in test_pe_gpu.py)
on several calls in a row, so that a call reading stale contents left in the
shared array by the previous call would be caught.

The file is named to be collected last: if it fails, a run that stops at the
first failure has already run every other test.
"""
import numpy as np
import pytest

import sysmat_b200
from sysmat_b200 import configs

pytestmark = pytest.mark.gpu


def _static_block(p, rotation=0, rows=None, z=None):
    import torch
    r0, r1 = rows if rows is not None else (0, p.n_crystals)
    nx, ny, nz_full = p.grid
    z0, nz = z if z is not None else (0, nz_full)
    ld = nx * ny * nz
    dst = torch.full((r1 - r0, ld), float("nan"), dtype=torch.float32, device="cuda:0")
    sysmat_b200.pe_compute_static(p, dst.data_ptr(), ld, rotation=rotation, rows=(r0, r1), z=(z0, nz))
    return dst.cpu().numpy()


def _allocating_block(ctx, p, rotation=0, rows=None, z=None):
    g = sysmat_b200.Geometry(ctx, p)
    try:
        return g.pe(rotation=rotation, rows=rows, z=z)
    finally:
        g.close()


def _same(got, ref):
    """Both entry points run the same kernel on tables derived by the same
    single-precision expressions, so the results are equal bit for bit."""
    assert got.shape == ref.shape
    assert np.isfinite(got).all(), "entries left unwritten"
    assert (ref != 0).any()
    assert np.array_equal(got, ref)


def test_static_entry_matches_allocating_entry_on_consecutive_calls():
    import torch
    torch.cuda.set_device(0)
    ctx = sysmat_b200.Context(0)
    try:
        big = configs.two_plates_small(seed=8)
        small = configs.tiny(layers=3)
        rotated = configs.tiny(seed=4, rotated=True)
        calls = [
            (big, dict()),
            (small, dict(rows=(5, 40), z=(1, 2))),
            (big, dict(rows=(13, 71))),
            (rotated, dict(rotation=1)),
        ]
        for p, kw in calls:
            _same(_static_block(p, **kw), _allocating_block(ctx, p, **kw))
    finally:
        ctx.close()


def test_static_entry_rejects_geometry_beyond_its_array():
    import torch
    torch.cuda.set_device(0)
    p = configs.tiny()
    n = 60000   # 96 bytes of derived tables per crystal: beyond the 4 MiB array
    det = np.zeros(1 + 12 * n, np.float32)
    det[0] = n
    body = det[1:].reshape(n, 12)
    body[:, 1] = 30.0
    body[:, 3:6] = 1.0
    body[:, 6] = 0.3
    body[:, 7] = 0.25
    p = p.copy()
    p.detector = det
    dst = torch.zeros(16, dtype=torch.float32, device="cuda:0")
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.pe_compute_static(p, dst.data_ptr(), 16, rows=(0, 1), z=(0, 1))
    assert e.value.code == -2 and "at most" in str(e.value)


def test_static_entry_rejects_host_destination_and_autotune():
    import torch
    torch.cuda.set_device(0)
    p = configs.tiny()
    host = np.zeros(64, np.float32)
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.pe_compute_static(p, host.ctypes.data, 64, rows=(0, 1), z=(0, 1))
    assert e.value.code == -1 and "device memory" in str(e.value)
    dst = torch.zeros(64, dtype=torch.float32, device="cuda:0")
    opts = sysmat_b200.PeOptions.make(p.sv, p.sc)
    opts.flags = 1   # SM_PE_AUTOTUNE
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.pe_compute_static(p, dst.data_ptr(), 64, rows=(0, 1), z=(0, 1), opts=opts)
    assert e.value.code == -1 and "autotune" in str(e.value)
