"""The batch group planner (pearl_gpu_batch_plan, host only): which blocks of a
batch launch form a group and which instances each group runs.  Only a
group's size bears on an instance's arithmetic; these tests hold the plan to
its invariants and to the balance it is built for."""
from __future__ import annotations

import math

import numpy as np
import pytest

GRID = 296  # 148 SMs x 2 resident blocks


def _tiles(nx, ny):
    return math.ceil(nx / 32) * math.ceil(ny / 16)


def _sweep_tiles(n=256):
    from pearl_gpu import workloads

    return [_tiles(w.nx, w.ny) for w in workloads.sweep(n, seed=0)]


def _modelled(tiles, goi, gsz, o):
    t = np.zeros(len(gsz))
    for i, g in enumerate(goi):
        t[g] += o + math.ceil(tiles[i] / gsz[g])
    return t.max()


def _check(tiles, goi, gsz, grid):
    assert len(gsz) >= 1 and gsz.sum() <= grid
    assert goi.min() >= 0 and goi.max() < len(gsz)
    # every group runs at least one instance unless the groups are of one fixed size
    counts = np.bincount(goi, minlength=len(gsz))
    assert counts.sum() == len(tiles)
    return counts


def test_sized_plan_on_the_sweep(gpu_lib):
    import pearl_gpu

    tiles = _sweep_tiles()
    for o in (1.0, 4.0, 16.0):
        goi, gsz, longest = pearl_gpu.batch_plan(tiles, GRID, pearl_gpu.BATCH_SIZED_GROUPS, o)
        counts = _check(tiles, goi, gsz, GRID)
        assert (counts > 0).all()
        assert all(g & (g - 1) == 0 or g == GRID // len(tiles) for g in gsz)
        assert longest == pytest.approx(_modelled(tiles, goi, gsz, o))
        # at least as balanced as equal groups of 4 under the same model
        _, _, equal4 = pearl_gpu.batch_plan(tiles, GRID, 4, o)
        assert longest <= equal4


def test_equal_groups(gpu_lib):
    import pearl_gpu

    tiles = _sweep_tiles()
    for gb in (1, 4, 8, 16):
        goi, gsz, longest = pearl_gpu.batch_plan(tiles, GRID, gb, 4.0)
        _check(tiles, goi, gsz, GRID)
        assert len(gsz) == GRID // gb and (gsz == gb).all()
        assert longest == pytest.approx(_modelled(tiles, goi, gsz, 4.0))
        # no instance could finish earlier by moving: the longest group is at most
        # the lower bound plus the longest single instance
        per = [4.0 + math.ceil(t / gb) for t in tiles]
        assert longest <= sum(per) / len(gsz) + max(per)


def test_small_instances_get_a_block_per_tile(gpu_lib):
    """With a grid to spare every instance gets at least one block per tile, the
    layout under which a batch instance equals its own context bitwise."""
    import pearl_gpu

    tiles = [_tiles(64, 64), _tiles(40, 48), _tiles(96, 32), _tiles(33, 80)]
    goi, gsz, longest = pearl_gpu.batch_plan(tiles, GRID, pearl_gpu.BATCH_SIZED_GROUPS, 4.0)
    _check(tiles, goi, gsz, GRID)
    for i, t in enumerate(tiles):
        assert gsz[goi[i]] >= t
    assert longest == 5.0


def test_large_instances_share_blocks(gpu_lib):
    import pearl_gpu

    tiles = [_tiles(384, 384)] * 3 + [_tiles(64, 64)]
    goi, gsz, _ = pearl_gpu.batch_plan(tiles, GRID, pearl_gpu.BATCH_SIZED_GROUPS, 4.0)
    _check(tiles, goi, gsz, GRID)
    assert all(gsz[goi[i]] < tiles[i] for i in range(3))
    assert len({goi[i] for i in range(3)}) == 3  # one large instance per group


def test_few_large_instances_use_the_grid(gpu_lib):
    """One instance gets the whole grid, like a context of its own; two large
    ones split it."""
    import pearl_gpu

    big = _tiles(2048, 4096)
    goi, gsz, _ = pearl_gpu.batch_plan([big], GRID, pearl_gpu.BATCH_SIZED_GROUPS, 4.0)
    assert list(gsz) == [GRID] and goi[0] == 0
    goi, gsz, _ = pearl_gpu.batch_plan([big, big], GRID, pearl_gpu.BATCH_SIZED_GROUPS, 4.0)
    assert sorted(gsz) == [GRID // 2, GRID // 2] and goi[0] != goi[1]


@pytest.mark.parametrize("args", [
    dict(grid=0, gb=4), dict(grid=GRID, gb=0), dict(grid=GRID, gb=GRID + 1), dict(grid=GRID, gb=-2),
    dict(grid=GRID, gb=4, o=-1.0), dict(grid=GRID, gb=4, tiles=[3, 0]),
])
def test_invalid_plans(gpu_lib, args):
    import pearl_gpu

    with pytest.raises(pearl_gpu.PearlError) as e:
        pearl_gpu.batch_plan(args.get("tiles", [3, 4]), args["grid"], args["gb"], args.get("o", 4.0))
    assert e.value.status == 1  # PEARL_ERR_INVALID_ARGUMENT
