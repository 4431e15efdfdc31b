"""Parity of the CUDA masked solve of the layered paths (tw_solve_masked) with the oracle, bit for
bit: soft and hard layer mattes, mattes that move between X and Y, NaN matte values, the three
depths and several geometries; without mattes it is the plain solve."""
import numpy as np
import pytest

import oracle_lib as O
import twixtor_b200 as tw
from twixtor_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    tw.build()
    d = tw.Device(0)
    yield d
    d.close()


def same(a, b):
    return np.asarray(a).view(np.uint8).tobytes() == np.asarray(b).view(np.uint8).tobytes()


def pair(w, h, fmt, seed):
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    frames = synth.moving_clip(w, h, 2, depth=depth, seed=seed)
    n = w * h * 4
    return O.from_frame(frames[:n], w, h, fmt), O.from_frame(frames[n:], w, h, fmt)


def disc(w, h, cx, cy, r, soft=1.0):
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float32)
    d = np.sqrt((xs - cx) ** 2 + (ys - cy) ** 2)
    return np.clip((r - d) / soft + 0.5, 0.0, 1.0).astype(np.float32).reshape(-1)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("size,quality,sens", [((160, 96), 4, 0.7), ((97, 61), 5, 1.0), ((320, 180), 4, 0.5),
                                               ((64, 48), 3, 0.7)])
@pytest.mark.parametrize("above_first", [True, False])
def test_masked_solve_matches_oracle(dev, fmt, size, quality, sens, above_first):
    w, h = size
    x, y = pair(w, h, fmt, seed=w + quality)
    mx = disc(w, h, w * 0.45, h * 0.5, min(w, h) * 0.3, soft=3.0)
    my = disc(w, h, w * 0.5, h * 0.52, min(w, h) * 0.3, soft=3.0)
    s = tw.FlowSettings(quality=quality, sensitivity=np.float32(sens), taps_above_first=above_first)
    got = dev.solve_masked(x, y, w, h, fmt, s, mx, my)
    want, _ = O.solve_masked(x, y, w, h, fmt, mx, my, quality=quality, sensitivity=np.float32(sens),
                             above_first=above_first)
    assert same(got, want)


def test_inverse_mattes_and_nan(dev):
    """The Main_BG style matte (1 - disc), values right at the 0.95 threshold and NaN values."""
    w, h = 128, 80
    x, y = pair(w, h, 0, seed=3)
    mx = 1.0 - disc(w, h, 60, 40, 20)
    my = 1.0 - disc(w, h, 64, 41, 20)
    mx[::7] = np.float32(0.95)
    my[::11] = np.float32(np.nextafter(np.float32(0.95), np.float32(0)))
    mx[5::13] = np.nan
    s = tw.FlowSettings()
    got = dev.solve_masked(x, y, w, h, 0, s, mx, my)
    want, _ = O.solve_masked(x, y, w, h, 0, mx, my)
    assert same(got, want)


def test_without_mattes_is_the_plain_solve(dev):
    w, h = 160, 96
    x, y = pair(w, h, 0, seed=8)
    s = tw.FlowSettings()
    got = dev.solve_masked(x, y, w, h, 0, s)
    want = dev.solve_pair(x, y, w, h, 0, s)[0]
    assert same(got, want)


def test_empty_matte_gives_the_zero_flow(dev):
    """A layer whose matte is empty everywhere: the masked gradient is zero, no pixel moves, and the
    result is the zero flow negated (-0.0), as the reference states (flow/extras.rs:222-230)."""
    w, h = 96, 64
    x, y = pair(w, h, 1, seed=2)
    z = np.zeros(w * h, np.float32)
    got = dev.solve_masked(x, y, w, h, 1, tw.FlowSettings(), z, z)
    want, _ = O.solve_masked(x, y, w, h, 1, z, z)
    assert same(got, want)
    assert (got.view(np.uint32) == 0x80000000).all()


@pytest.mark.parametrize("extras", ["none", "masks", "points", "both"])
def test_solve_pyramids_with_extras_matches_oracle(dev, extras):
    """tw_solve_pyramids (Backend::solve_pyramids_with) on the oracle's pyramids with its mask
    pyramids and user displacement: the flow bit for bit."""
    w, h = 97, 61
    rng = np.random.RandomState(3)
    frames = synth.moving_clip(w, h, 2, depth=8, seed=21)
    n = w * h * 4
    x, y = O.from_frame(frames[:n], w, h, 0), O.from_frame(frames[n:], w, h, 0)
    mx = my = pairs = None
    if extras in ("masks", "both"):
        yy, xx = np.mgrid[0:h, 0:w]
        mx = (((xx - 40) / 30.0) ** 2 + ((yy - 30) / 20.0) ** 2 <= 1).astype(np.float32).ravel()
        my = (((xx - 43) / 30.0) ** 2 + ((yy - 31) / 20.0) ** 2 <= 1).astype(np.float32).ravel()
    if extras in ("points", "both"):
        pairs = rng.uniform([5, 5, 5, 5], [w - 5, h - 5, w - 5, h - 5], (3, 4)).astype(np.float32)
    want, xl, yl, mxl, myl, ud, uw = O.solve_pyramids_with(x, y, w, h, 0, mx, my, pairs)
    got, _ = dev.solve_pyramids(tw.FlowSettings(), w, h, xl, yl, mxl, myl, ud, uw)
    assert got.tobytes() == want.tobytes()
