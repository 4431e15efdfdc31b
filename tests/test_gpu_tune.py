"""The autotuner and the launch shapes it chooses between.

Every tile shape and block size of the solver iteration, and every block size of block matching,
must give the same bytes as the oracle (each element keeps the reference's operation order
whatever the tiling); the tuned table must round-trip through its JSON cache.
"""
import json

import numpy as np
import pytest

import oracle_lib as O
import twixtor_b200 as tw
from twixtor_b200 import synth

pytestmark = pytest.mark.gpu

SHAPES = [(0, 256), (0, 512), (1, 256), (1, 512), (2, 512), (2, 256)]


@pytest.fixture(scope="module")
def dev():
    tw.build()
    d = tw.Device(0)
    yield d
    d.close()


def _pair(w, h, fmt, seed):
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    frames = synth.moving_clip(w, h, 2, depth=depth, seed=seed, square=48, square_velocity=(3.0, 2.0))
    n = w * h * 4
    return O.from_frame(frames[:n], w, h, fmt), O.from_frame(frames[n:], w, h, fmt)


@pytest.mark.parametrize("tile,threads", SHAPES)
@pytest.mark.parametrize("size", [(481, 271), (160, 96), (1920, 1080)])
def test_every_iteration_shape_is_bit_exact(dev, tile, threads, size):
    w, h = size
    if size == (1920, 1080) and (tile, threads) not in [(1, 512), (2, 512)]:
        pytest.skip("1080p: the shapes the tuner picks there")
    a, b = _pair(w, h, 0, seed=w + h)
    s = tw.FlowSettings()
    _, _, levels = tw.flow_geometry(s, w, h)
    for lw, lh in levels:
        dev.tuning_set(lw, lh, tile, threads, 256, 256)
    try:
        fab, fba, _ = dev.solve_pair(a, b, w, h, 0, s)
    finally:
        dev.tuning_clear()
    wab, wba, _ = O.solve_pair(a, b, w, h, 0)
    assert fab.tobytes() == wab.tobytes() and fba.tobytes() == wba.tobytes()


@pytest.mark.parametrize("rows,cols", [(128, 512), (512, 128), (1024, 64), (32, 1024)])
def test_every_block_matching_block_size_is_bit_exact(dev, rows, cols):
    w, h = 481, 271
    a, b = _pair(w, h, 1, seed=7)
    s = tw.FlowSettings()
    _, _, levels = tw.flow_geometry(s, w, h)
    for lw, lh in levels:
        dev.tuning_set(lw, lh, 0, 256, rows, cols)
    try:
        fab, fba, _ = dev.solve_pair(a, b, w, h, 1, s)
    finally:
        dev.tuning_clear()
    wab, wba, _ = O.solve_pair(a, b, w, h, 1)
    assert fab.tobytes() == wab.tobytes() and fba.tobytes() == wba.tobytes()


def test_autotune_table_round_trips_and_keeps_the_bytes(dev, tmp_path):
    path = str(tmp_path / "tune.json")
    s = tw.FlowSettings()
    n = dev.autotune(s, 1920, 1080, path=path)
    _, _, levels = tw.flow_geometry(s, 1920, 1080)
    assert n == len(levels)
    table = json.load(open(path))
    assert set(table["levels"]) == {f"{lw}x{lh}" for lw, lh in levels}
    with tw.Device(0) as other:
        assert other.autotune(s, 1920, 1080, path=path) == 0  # everything came from the cache
        assert json.loads(other.tuning_table()) == table
    # a clip rendered with the tuned shapes is the oracle's
    w, h, nf = 160, 96, 6
    dev.autotune(s, w, h)
    frames = synth.moving_clip(w, h, nf, depth=8, seed=3)
    tp = tw.TimeParams(speed_percent=50.0)
    sels = [tw.select(tp, k, w, h) for k in range(8)]
    got = dev.retime_clip(tw.RetimeSettings(), frames, nf, sels, w, h, 0)
    want = O.retime_clip(frames, nf, w, h, 0, O.retime_params(speed=50.0), 8)
    dev.tuning_clear()
    assert got.tobytes() == want.tobytes()


def test_tuning_entries_are_checked(dev):
    for bad in [(-1, 256, 256, 256), (3, 256, 256, 256), (0, 1024, 256, 256), (0, 100, 256, 256), (0, 256, 2048, 256)]:
        with pytest.raises(tw.BadParam):
            dev.tuning_set(64, 48, *bad)
