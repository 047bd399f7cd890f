"""The batched photoelectric sysmat (one persistent launch over many
geometries, replayed from a CUDA graph) and the brick autotuner.  Each
geometry's matrix must equal, bit for bit, what sm_pe_compute gives for it
alone: the decomposition into tiles never changes a value."""
import numpy as np
import pytest

import sysmat_b200
from sysmat_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sysmat_b200.Context(0)
    yield c
    c.close()


def test_batch_equals_per_geometry_launches(ctx):
    import torch
    params = [configs.tiny(layers=3), configs.two_plates_small(seed=8), configs.tiny(seed=4, rotated=True),
              configs.sweep()[2]]
    geos = [sysmat_b200.Geometry(ctx, p) for p in params]
    opts = [g.options() for g in geos]
    opts[1] = geos[1].options(tile_voxels=(4, 4, 2))
    rotations = [0, 0, 1, 0]
    outs = [torch.full((g.n_crystals, g.nx * g.ny * g.nz), float("nan"), device="cuda") for g in geos]
    batch = sysmat_b200.PeBatch(ctx, geos, opts, [o.data_ptr() for o in outs], [o.shape[1] for o in outs], rotations)
    info = batch.info()
    assert info["geometries"] == 4 and info["items"] > 0 and info["ctas"] >= 148
    for rep in range(2):                      # first run captures the graph, the second replays it
        for o in outs:
            o.fill_(float("nan"))
        batch.run()
        torch.cuda.synchronize()
        ctx.sync()
        for g, o, op, rot in zip(geos, outs, opts, rotations):
            ref = g.pe(rotation=rot, opts=op)
            assert np.array_equal(o.cpu().numpy(), ref)
    batch.close()
    for g in geos:
        g.close()


def test_autotune_picks_a_brick_and_caches_it(ctx):
    p = configs.two_plates_small(seed=8)
    g = sysmat_b200.Geometry(ctx, p)
    tuned, ms = sysmat_b200.autotune(g)
    brick = tuple(tuned.tile_voxels)
    assert all(b >= 1 for b in brick) and np.prod(brick) <= 128 and ms > 0
    again, ms2 = sysmat_b200.autotune(g)
    assert tuple(again.tile_voxels) == brick and ms2 == -1.0
    # results do not depend on the brick
    assert np.array_equal(g.pe(opts=tuned), g.pe())
    auto = g.options()
    auto.flags = 1
    assert np.array_equal(g.pe(opts=auto), g.pe())
    g.close()


def test_batch_beyond_one_constant_table(ctx):
    """More geometries than one persistent launch takes (64): the graph holds
    one launch per chunk of 64."""
    import torch
    params = [configs.tiny(seed=s, layers=1 + s % 3) for s in range(67)]
    geos = [sysmat_b200.Geometry(ctx, p) for p in params]
    outs = [torch.full((g.n_crystals, g.nx * g.ny * g.nz), float("nan"), device="cuda") for g in geos]
    batch = sysmat_b200.PeBatch(ctx, geos, [g.options() for g in geos], [o.data_ptr() for o in outs],
                                [o.shape[1] for o in outs])
    batch.run()
    torch.cuda.synchronize()
    ctx.sync()
    for g, o in zip(geos, outs):
        assert np.array_equal(o.cpu().numpy(), g.pe())
    batch.close()
    for g in geos:
        g.close()


def _best_ms(fn, reps=5):
    import torch
    best = 1e30
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def _same_up_to_rounding(a, b):
    """Same zeros (the same hit decisions) and values within 1e-5 relative:
    options that change which lane sums which ray change only the rounding."""
    assert np.array_equal(a == 0, b == 0)
    nz = b != 0
    assert (np.abs(a[nz].astype(np.float64) - b[nz]) / np.abs(b[nz])).max() <= 1e-5


@pytest.mark.parametrize("member", [0, 7, 21])
def test_autotuned_options_are_not_slower_and_give_the_same_matrix(ctx, member):
    """The tuner times whole small matrices (bricks x sub-points per group) and
    keeps the fastest; the pick is never slower than the default options by
    more than timing noise.  Bricks change no value; the group changes only
    the rounding of the per-lane sums."""
    import torch
    p = configs.sweep_small()[member]
    g = sysmat_b200.Geometry(ctx, p)
    tuned, ms = sysmat_b200.autotune(g)
    default = g.options()
    out = torch.empty((g.n_crystals, g.nx * g.ny * g.nz), device="cuda")
    t_default = _best_ms(lambda: g.pe(opts=default, out=out.data_ptr()))
    t_tuned = _best_ms(lambda: g.pe(opts=tuned, out=out.data_ptr()))
    assert t_tuned <= 1.05 * t_default + 0.01, (t_tuned, t_default, tuple(tuned.tile_voxels), tuned.group)
    _same_up_to_rounding(g.pe(opts=tuned), g.pe(opts=default))
    same_group = sysmat_b200.PeOptions.make(p.sv, p.sc, tile_voxels=tuple(tuned.tile_voxels), group=tuned.group)
    assert np.array_equal(g.pe(opts=same_group), g.pe(opts=sysmat_b200.PeOptions.make(p.sv, p.sc, group=tuned.group)))
    g.close()


def test_group_option_changes_only_rounding_and_is_validated(ctx):
    p = configs.two_plates_small(seed=8)          # 8 voxel sub-points, 4 depth sub-cells: auto group 8
    g = sysmat_b200.Geometry(ctx, p)
    base = g.pe()
    assert np.array_equal(g.pe(opts=sysmat_b200.PeOptions.make(p.sv, p.sc, group=8)), base)
    for group in (1, 2, 4):
        _same_up_to_rounding(g.pe(opts=sysmat_b200.PeOptions.make(p.sv, p.sc, group=group)), base)
    with pytest.raises(sysmat_b200.SysmatError) as e:
        g.pe(opts=sysmat_b200.PeOptions.make(p.sv, p.sc, group=9))
    assert e.value.code == -1 and "group" in str(e.value)
    g.close()
