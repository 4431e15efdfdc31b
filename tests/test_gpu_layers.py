"""Parity of the CUDA layered composition with plates (tw_compose_layers) with the oracle, bit for
bit: one to three FG matte layers moving over a background, Nearest and Blend, warping codes 0 and
1, the three depths, soft mattes and float mattes outside 0..1; and retime-fgbg over whole clips
(tw_retime_layers_clip) against the sha256 the reference's fgbg-layers parity grid records."""
import hashlib

import numpy as np
import pytest

import golden_data
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


def display_group(display, nfg):
    """layers.rs:120-129: the layers (first, last) the Display popup composes."""
    if 3 <= display <= 5:
        g = min(display - 3, nfg)
        return g, g
    if display == 6:
        return nfg, nfg
    return 0, nfg


def run(dev, a, b, w, h, fmt, ma, mb, sens, wa, interp, code, video_360=False, gouraud=False, shrink=None, display=1,
        points=None):
    s = tw.RetimeSettings(flow=tw.FlowSettings(video_range_luma=video_360),
                          compose=tw.EngineSettings(warp_mode=code, video_360=video_360, gouraud=gouraud))
    sel = tw.Selection(wa=np.float32(wa), exact=False, vectors_quality=4, interp=interp)
    got = dev.compose_layers(s, sel, a, b, w, h, fmt, ma, mb, sens, shrink=shrink, display=display, points=points)
    want = O.compose_layers(a, b, w, h, fmt, ma, mb, sens, np.float32(wa), interp, warp_mode=code, video_360=video_360,
                            gouraud=gouraud, shrink=shrink, group=display_group(display, len(ma)), points=points)
    assert same(got, want)


@pytest.mark.parametrize("fmt", [0, 2])
@pytest.mark.parametrize("wa,interp", [(0.4, 1), (0.6, 0), (0.3, 0)])
@pytest.mark.parametrize("display", [1, 3])
def test_layers_tracking_points_match_oracle(dev, fmt, wa, interp, display):
    """Tracking points on FG1 and Main_BG: the user displacement pyramid (splat, normalise, blur,
    resample, scale) and its three hooks in every level of the masked solves; points that share a
    pixel, points outside the frame, a large motion."""
    w, h = 96, 64
    a, b, ma, mb = scene(w, h, fmt, 2, seed=41 + display)
    points = [[(20.0, 12.5, 24.0, 14.0), (20.2, 12.6, 26.0, 10.0), (-3.0, 5.0, 2.0, 5.0)],
              [],
              [(70.0, 40.0, 66.5, 43.25), (10.0, 60.0, 80.0, 2.0), (95.4, 63.4, 90.0, 60.0)]]
    run(dev, a, b, w, h, fmt, ma, mb, [0.7, 0.7, 0.7], wa, interp, 1, points=points, display=display)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("display", [1, 3, 4, 6])
@pytest.mark.parametrize("shrink", [(0.0, 0.0), (2.5, 0.0), (1.0, 4.0), (-1.5, 0.5), (10.0, 0.0)])
def test_layers_display_group_and_shrink_match_oracle(dev, fmt, display, shrink):
    """The display groups (one layer alone over an empty image, or Main_BG alone) and the inverse
    matte shrink of the cut planes (the plugin's choke: grow, shrink, fractional mixes), soft and
    hard mattes."""
    w, h = 96, 64
    a, b, ma, mb = scene(w, h, fmt, 2, seed=21 + display, soft=3.0 if fmt == 2 else 0.0)
    run(dev, a, b, w, h, fmt, ma, mb, [0.7, 0.6, 0.7], 0.4, 1, 1, shrink=list(shrink), display=display)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("nfg", [1, 3])
@pytest.mark.parametrize("code", [0, 1])
@pytest.mark.parametrize("wa,interp", [(0.4, 1), (0.75, 1), (0.6, 0), (0.3, 0)])
def test_layers_match_oracle(dev, fmt, nfg, code, wa, interp):
    w, h = 96, 64
    a, b, ma, mb = scene(w, h, fmt, nfg, seed=11 + nfg)
    sens = [0.7, 0.5, 0.9][:nfg] + [0.7]
    run(dev, a, b, w, h, fmt, ma, mb, sens, wa, interp, code)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("code", [2, 3])
@pytest.mark.parametrize("gouraud", [True, False])
@pytest.mark.parametrize("wa,interp", [(0.4, 1), (0.6, 0), (0.3, 0)])
def test_layers_forward_codes(dev, fmt, code, gouraud, wa, interp):
    """Warping codes 2 and 3: plates pushed by the forward warp, the forward compositions per layer."""
    w, h = 80, 48
    a, b, ma, mb = scene(w, h, fmt, 2, seed=21 + code)
    run(dev, a, b, w, h, fmt, ma, mb, [0.7, 0.5, 0.7], wa, interp, code, gouraud=gouraud)


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


FG_CASES, FG_INPUTS = golden_data.fgbg_grid()


def fgbg_clip(dev, case, rows_reversed=True, taps_above_first=True):
    fmt = golden_data.FMT_OF_DEPTH[case["depth"]]
    w, h, n = case["width"], case["height"], case["frames"]
    kw = golden_data.fgbg_case_params(case)
    tp = tw.TimeParams(fps=kw["fps"], speed_percent=kw["speed"], vectors=kw["vectors"], frame_interp=kw["frame_interp"],
                       blur_compensation=kw["blur"], mark_segs=kw["mark_segs"], mark_keys=kw["mark_keys"])
    sels = [tw.select(tp, k, w, h) for k in range(n)]
    s = tw.RetimeSettings(flow=tw.FlowSettings(hiq=True, taps_above_first=taps_above_first,
                                               track_alpha=kw["track_rgb_a"]),
                          compose=tw.EngineSettings(warp_mode=kw["smart_blend"], taps_above_first=taps_above_first,
                                                    gouraud=True, blur=float(tw.fixed_param(kw["blur"]))),
                          motion_rows_reversed=rows_reversed)
    sens = [tw.percent_param(v) for v in kw["fg_sens"]] + [tw.percent_param(kw["sensitivity"])]
    mattes = [FG_INPUTS[m].view(tw.DTYPES[fmt]) for m in case["mattes"]]
    shrink = [float(tw.fixed_param(v)) for v in kw["shrinks"]]
    points = [golden_data.fgbg_points(case, x.a, x.a + 1, len(mattes)) for x in sels]
    return dev.retime_layers_clip(s, FG_INPUTS[case["input"]].view(tw.DTYPES[fmt]), n, mattes, kw["chans"], sens, sels,
                                  w, h, fmt, shrink=shrink, display=kw["display"], points=points)


@pytest.mark.parametrize("case", FG_CASES, ids=[c["id"] for c in FG_CASES])
def test_fgbg_layers_grid_sha256(dev, case):
    """Every served case of the reference's retime-fgbg grid (all four warping codes; retime-fgbg's
    forward warps are the Gouraud variant; the display groups and the inverse matte shrink),
    rendered by the CUDA path."""
    out = fgbg_clip(dev, case)
    assert hashlib.sha256(out.tobytes()).hexdigest() == case["sha256"]


def test_fgbg_clip_matches_oracle_at_larger_size(dev):
    """A 160x96 clip of 6 frames at 40 %, two FG layers on the G and alpha channels, 16 bpc."""
    w, h, n, fmt = 160, 96, 6, 1
    frames = synth.moving_clip(w, h, n, depth=16, seed=0x5eed)
    rng = np.random.RandomState(11)
    mattes = []
    for j in range(2):
        m = synth.moving_clip(w, h, n, depth=16, seed=100 + j).view(np.uint16).reshape(n, h, w, 4).copy()
        cx, cy, vx = rng.uniform(0.3, 0.7) * w, rng.uniform(0.3, 0.7) * h, rng.uniform(-3, 3)
        for f in range(n):
            e = ellipse(w, h, cx + vx * f, cy, 0.2 * w, 0.25 * h, soft=2.0).reshape(h, w)
            m[f, :, :, 1 if j == 0 else 3] = (e * 65535.0 + 0.5).astype(np.uint16)
        mattes.append(m.reshape(-1))
    tp = tw.TimeParams(speed_percent=40.0)
    nout = 12
    sels = [tw.select(tp, k, w, h) for k in range(nout)]
    s = tw.RetimeSettings(flow=tw.FlowSettings(hiq=True), compose=tw.EngineSettings(warp_mode=1))
    sens = [tw.percent_param(55.0), tw.percent_param(70.0), tw.percent_param(70.0)]
    got = dev.retime_layers_clip(s, frames, n, mattes, [2, 4], sens, sels, w, h, fmt)
    p = O.retime_params(speed=40.0, smart_blend=1, sensitivity=70.0)
    want = O.retime_fgbg_clip(frames, n, mattes, [2, 4], [55.0, 70.0], w, h, fmt, p, nout)
    assert same(got, want)


@pytest.mark.parametrize("code", [2, 3])
def test_fgbg_clip_without_layers_forward_codes(dev, code):
    """No FG layer with a forward warping code: the plain vector path on the context's stream."""
    w, h, n, fmt = 96, 64, 4, 0
    frames = synth.moving_clip(w, h, n, depth=8, seed=0x5eed + code)
    tp = tw.TimeParams(speed_percent=50.0)
    nout = 7
    sels = [tw.select(tp, k, w, h) for k in range(nout)]
    s = tw.RetimeSettings(flow=tw.FlowSettings(hiq=True), compose=tw.EngineSettings(warp_mode=code, gouraud=True))
    got = dev.retime_layers_clip(s, frames, n, [], [], [tw.percent_param(70.0)], sels, w, h, fmt)
    p = O.retime_params(speed=50.0, smart_blend=code, sensitivity=70.0)
    want = O.retime_fgbg_clip(frames, n, [], [], [], w, h, fmt, p, nout)
    assert same(got, want)


def test_fgbg_1080p_frame_matches_oracle(dev):
    """One in-between frame of the 1080p retime-fgbg workload (three FG matte layers, speed 40 %)."""
    w, h, n = 1920, 1080, 3
    frames, mattes = synth.layered_clip(w, h, n, nfg=3)
    tp = tw.TimeParams(speed_percent=40.0)
    sels = [tw.select(tp, k, w, h) for k in range(2)]
    assert not sels[1].exact
    s = tw.RetimeSettings(compose=tw.EngineSettings(gouraud=True))
    sens = [tw.percent_param(70.0)] * 4
    got = dev.retime_layers_clip(s, frames, n, mattes, [1, 1, 1], sens, sels, w, h, 0)
    want = O.retime_fgbg_clip(frames, n, mattes, [1, 1, 1], [70.0] * 3, w, h, 0, O.retime_params(speed=40.0), 2)
    assert same(got, want)
