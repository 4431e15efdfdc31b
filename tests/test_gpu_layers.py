"""Parity of the CUDA layered composition with plates (tw_compose_layers) with the oracle, bit for
bit: one to three FG matte layers moving over a background, Nearest and Blend, warping codes 0 and
1, the three depths, soft mattes and float mattes outside 0..1."""
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


def ellipse(w, h, cx, cy, rx, ry, soft=0.0):
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float32)
    d = np.sqrt(((xs - cx) / rx) ** 2 + ((ys - cy) / ry) ** 2)
    if soft <= 0:
        return (d <= 1.0).astype(np.float32).reshape(-1)
    return np.clip((1.0 - d) * min(rx, ry) / soft + 0.5, 0.0, 1.0).astype(np.float32).reshape(-1)


def scene(w, h, fmt, nfg, seed, soft=0.0):
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    frames = synth.moving_clip(w, h, 2, depth=depth, seed=seed)
    n = w * h * 4
    a, b = O.from_frame(frames[:n], w, h, fmt), O.from_frame(frames[n:], w, h, fmt)
    rng = np.random.RandomState(seed)
    ma, mb = [], []
    for _ in range(nfg):
        cx, cy = rng.uniform(0.3, 0.7) * w, rng.uniform(0.3, 0.7) * h
        rx, ry = rng.uniform(0.12, 0.3) * w, rng.uniform(0.12, 0.3) * h
        vx, vy = rng.uniform(-4, 4), rng.uniform(-3, 3)
        ma.append(ellipse(w, h, cx, cy, rx, ry, soft))
        mb.append(ellipse(w, h, cx + vx, cy + vy, rx, ry, soft))
    return a, b, ma, mb


def run(dev, a, b, w, h, fmt, ma, mb, sens, wa, interp, code, video_360=False):
    s = tw.RetimeSettings(flow=tw.FlowSettings(video_range_luma=video_360),
                          compose=tw.EngineSettings(warp_mode=code, video_360=video_360))
    sel = tw.Selection(wa=np.float32(wa), exact=False, vectors_quality=4, interp=interp)
    got = dev.compose_layers(s, sel, a, b, w, h, fmt, ma, mb, sens)
    want = O.compose_layers(a, b, w, h, fmt, ma, mb, sens, np.float32(wa), interp, warp_mode=code, video_360=video_360)
    assert same(got, want)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("nfg", [1, 3])
@pytest.mark.parametrize("code", [0, 1])
@pytest.mark.parametrize("wa,interp", [(0.4, 1), (0.75, 1), (0.6, 0), (0.3, 0)])
def test_layers_match_oracle(dev, fmt, nfg, code, wa, interp):
    w, h = 96, 64
    a, b, ma, mb = scene(w, h, fmt, nfg, seed=11 + nfg)
    sens = [0.7, 0.5, 0.9][:nfg] + [0.7]
    run(dev, a, b, w, h, fmt, ma, mb, sens, wa, interp, code)


@pytest.mark.parametrize("fmt", [0, 2])
def test_soft_mattes_two_layers(dev, fmt):
    w, h = 160, 96
    a, b, ma, mb = scene(w, h, fmt, 2, seed=5, soft=3.0)
    run(dev, a, b, w, h, fmt, ma, mb, [0.7, 0.7, 0.7], 0.4, 1, 0)


def test_float_mattes_out_of_range(dev):
    """A float matte reaches the cut as it is (plates.rs:50-57): values above 1 and below 0."""
    w, h = 80, 48
    a, b, ma, mb = scene(w, h, 2, 2, seed=9, soft=2.0)
    mb[1][::23] = 1.5
    ma[1][::29] = -0.25
    run(dev, a, b, w, h, 2, ma, mb, [0.7, 0.7, 0.7], 0.4, 1, 1)


def test_integer_mattes_clamped(dev):
    """A matte with a value outside 0..1 is clamped as a whole before its units (matte.rs:106-112)."""
    w, h = 64, 48
    a, b, ma, mb = scene(w, h, 0, 1, seed=3)
    ma[0][::13] = 1.25
    run(dev, a, b, w, h, 0, ma, mb, [0.7, 0.7], 0.4, 1, 0)


def test_no_fg_layer_is_main_bg_alone(dev):
    w, h = 64, 48
    a, b, _, _ = scene(w, h, 0, 0, seed=2)
    run(dev, a, b, w, h, 0, [], [], [0.7], 0.4, 1, 0)


def test_video_360_binary_alpha(dev):
    w, h = 96, 64
    a, b, ma, mb = scene(w, h, 1, 1, seed=4)
    run(dev, a, b, w, h, 1, ma, mb, [0.7, 0.7], 0.4, 1, 1, video_360=True)
