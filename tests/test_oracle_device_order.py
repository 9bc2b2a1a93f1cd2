"""The oracle's device-order mode (po_set_device_order, oracle/pearl_oracle.c).

libpearl_gpu sums every global quantity in a fixed tree (per-thread running
sums over a block's tiles, warp shuffles, warps in index order, block
partials strided over 32 lanes); the reference sums sequentially in row-major
order.  The oracle's device-order mode restates the tree so that a GPU run can
be compared with the oracle bit for bit.  Here, on the CPU:

  * the C tree equals an independent pure-Python emulation of the device's
    threads (every lane of every warp, shuffles applied to all 32 lanes at
    once, as __shfl_down_sync does) for ragged grids, both block shapes, both
    walk directions and several grid sizes, on values whose sum depends on the
    order;
  * a run in device order takes the same decisions as the reference's order
    and stays within the FP64 bars, while its sums differ in the last bits
    (the order is all that changes);
  * the host threads of the mode change no bit.
"""
from __future__ import annotations

import numpy as np
import pytest


def _emulate_device_sum(v: np.ndarray, warps: int, blocks: int, reverse: bool, warps_x_log2: int = 0) -> float:
    """Python restatement of the kernels' reduction: pair_of's thread-to-cell
    mapping, a running sum per thread over the block's tiles in walk order,
    block_publish's shuffle tree and warp order, grid_gather's strided lanes."""
    ny, nx = v.shape
    tile_w = 32 << warps_x_log2
    tile_h = (2 * warps) >> warps_x_log2
    ntx, nty = -(-nx // tile_w), -(-ny // tile_h)
    ntiles = ntx * nty

    def shfl_down_tree(lanes):
        lanes = list(lanes)
        for o in (16, 8, 4, 2, 1):
            # every lane reads its partner's value from before this step
            lanes = [lanes[i] + (lanes[i + o] if i + o < 32 else lanes[i]) for i in range(32)]
        return lanes[0]

    parts = []
    for b in range(blocks):
        nb = (ntiles - 1 - b) // blocks + 1 if b < ntiles else 0
        tiles = [b + k * blocks for k in range(nb)]
        if reverse:
            tiles = tiles[::-1]
        warp_vals = []
        for w in range(warps):
            wx, wy = w & ((1 << warps_x_log2) - 1), w >> warps_x_log2
            lanes = []
            for lane in range(32):
                s = 0.0
                for t in tiles:
                    x = (t % ntx) * tile_w + (wx << 5) + lane
                    y0 = (t // ntx) * tile_h + 2 * wy
                    if x < nx and y0 < ny:
                        s += float(v[y0, x])
                        if y0 + 1 < ny:
                            s += float(v[y0 + 1, x])
                lanes.append(s)
            warp_vals.append(shfl_down_tree(lanes))
        acc = warp_vals[0]
        for wv in warp_vals[1:]:
            acc += wv
        parts.append(acc)
    lanes = []
    for lane in range(32):
        s = 0.0
        for b in range(lane, blocks, 32):
            s += parts[b]
        lanes.append(s)
    return shfl_down_tree(lanes)


CASES = [
    # nx, ny, warps, blocks, warps_x_log2
    (37, 19, 8, 3, 0),
    (64, 48, 8, 6, 0),
    (100, 72, 16, 5, 0),
    (33, 65, 16, 40, 0),
    (130, 70, 8, 33, 0),
    (96, 40, 8, 7, 1),
    (128, 24, 8, 2, 2),
]


@pytest.mark.parametrize("nx,ny,warps,blocks,wxl2", CASES)
@pytest.mark.parametrize("reverse", [False, True])
def test_device_tree_sum_matches_emulation(port, nx, ny, warps, blocks, wxl2, reverse):
    rng = np.random.default_rng(nx * 1000 + ny)
    # magnitudes over 12 decades, both signs: the sum's rounding depends on the order
    v = rng.standard_normal((ny, nx)) * 10.0 ** rng.integers(-6, 7, size=(ny, nx))
    with port.device_order(warps, blocks, wxl2, threads=1):
        got = port.device_sum(v, reverse)
    want = _emulate_device_sum(v, warps, blocks, reverse, wxl2)
    assert got == want or (np.isnan(got) and np.isnan(want))


def test_device_order_changes_the_rounding(port):
    rng = np.random.default_rng(3)
    v = rng.standard_normal((64, 96)) * 10.0 ** rng.integers(-6, 7, size=(64, 96))
    seq = 0.0
    for x in v.ravel():
        seq += float(x)
    with port.device_order(8, 7):
        fwd, rev = port.device_sum(v, False), port.device_sum(v, True)
    assert fwd != seq or rev != seq
    assert abs(fwd - seq) <= 1e-12 * np.abs(v).sum()


def _run(port, w, n, order=None):
    from oracle import pyoracle

    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    if order is None:
        rc, why, done, infos = port.advance_n(w.params, phi, c, mu, s, n)
    else:
        with port.device_order(*order):
            rc, why, done, infos = port.advance_n(w.params, phi, c, mu, s, n)
    assert rc == 0 and done == n, why
    return phi, c, mu, s, infos


def test_device_order_run_same_decisions_within_bars(port):
    from pearl_gpu import workloads

    w = workloads.scaled(96, 128, seed=7, undercooling=20.0, dt=4e-12, dt_max=8e-12, jitter=0.1, front_jitter=1,
                         front=24.0)
    n = 30
    p0, c0, m0, s0, i0 = _run(port, w, n)
    p1, c1, m1, s1, i1 = _run(port, w, n, order=(8, 24, 0, 1))
    assert [i.retries for i in i0] == [i.retries for i in i1]
    assert [i.cg_iterations for i in i0] == [i.cg_iterations for i in i1]
    assert s0.time == s1.time and s0.rejected == s1.rejected
    assert np.abs(p0 - p1).max() <= 1e-10
    assert np.abs(m0 - m1).max() <= 1e-5
    assert abs(c0.sum() - c1.sum()) <= 1e-12 * abs(c0.sum())
    # the order changes the sums themselves in their last bits (the fields of so
    # short a run may still agree bitwise: the converged CG iterate absorbs it)
    rc, e_seq, m_seq = port.energy_and_mass(w.params, p1, c1)
    with port.device_order(8, 24, 0, 1):
        rc2, e_dev, m_dev = port.energy_and_mass(w.params, p1, c1)
    assert rc == rc2 == 0
    assert (e_seq, m_seq) != (e_dev, m_dev)
    assert abs(e_seq - e_dev) <= 1e-12 * abs(e_seq) and abs(m_seq - m_dev) <= 1e-12 * abs(m_seq)


def test_device_order_host_threads_change_no_bit(port):
    from pearl_gpu import workloads

    w = workloads.scaled(64, 80, seed=9, front=20.0)
    a = _run(port, w, 12, order=(8, 20, 0, 1))
    b = _run(port, w, 12, order=(8, 20, 0, 4))
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
