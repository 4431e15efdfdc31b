"""Parity of the CUDA Create Vectors pass (tw_create_vectors, tw_create_vectors_clip,
tw_encode_vectors) with the reference's recorded outputs and with the oracle, bit for bit."""
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


CV_CASES, CV_INPUTS = golden_data.cv_grid()
# the NTSC and decimal rate cases are pinned on the oracle; the device runs the integer rate ones,
# whose frame pairs tw_vectors_frame_pair has been checked against on a GPU run
CV_CASES = [c for c in CV_CASES if "/" not in c["fps"] and "." not in c["fps"]]


@pytest.mark.parametrize("case", golden_data.cv_grid_params(CV_CASES))
def test_create_vectors_grid_sha256(dev, case):
    """The reference's recorded output clips of the served create-vectors grid cases (the Debug
    display with the textured warp of the recorded revision)."""
    fmt = golden_data.FMT_OF_DEPTH[case["depth"]]
    raw = CV_INPUTS[case["input"]].view(tw.DTYPES[fmt])
    kw = golden_data.cv_case_params(case)
    s = tw.vectors_settings(vector_resolution=kw["vector_resolution"], max_displace=kw["max_displace"],
                            sensitivity=kw["sensitivity"], track_rgb_a=kw["track_rgb_a"], rows_reversed=False,
                            taps_above_first=False, prep=kw["prep"], display=kw["display"],
                            debug_view_method=kw["debug_view_method"], debug_textured=True)
    pairs = [tw.vectors_pair(n, kw["track_frame"], kw["fps"], debug=kw["display"] == 3) for n in range(case["frames"])]
    points = [golden_data.cv_points(case, n) for n in range(case["frames"])]
    out = dev.create_vectors_clip(s, raw, case["frames"], pairs, case["width"], case["height"], fmt, points=points)
    assert hashlib.sha256(out.tobytes()).hexdigest() == case["sha256"]


@pytest.mark.parametrize("fmt", [0, 2])
@pytest.mark.parametrize("rows_reversed", [True, False])
def test_clip_with_points_matches_oracle(dev, fmt, rows_reversed):
    """Tracking points on the single layer at 160x96: their user displacement in the solve X -> Y,
    points on one pixel, off the frame, frames without a point."""
    w, h, n = 160, 96, 4
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    frames = synth.moving_clip(w, h, n, depth=depth, seed=0x74570003)
    s = tw.vectors_settings(max_displace=24.0, rows_reversed=rows_reversed, taps_above_first=rows_reversed)
    pairs = [tw.vectors_pair(k, 1) for k in range(n)]
    points = [[(40.0, 30.0, 44.0, 27.5)], [], [(40.0, 30.0, 44.0, 27.5), (40.3, 29.8, 30.0, 35.0), (-9.0, 3.0, 1.0, 1.0)],
              [(150.2, 90.7, 120.0, 80.0), (5.0, 5.0, 5.0, 5.0)]]
    got = dev.create_vectors_clip(s, frames, n, pairs, w, h, fmt, points=points)
    want = O.create_vectors_clip(frames, n, w, h, fmt, n, max_displace=24.0, rows_reversed=rows_reversed,
                                 taps_above_first=rows_reversed, points=points)
    assert same(got, want)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("track_frame", [1, 2])
@pytest.mark.parametrize("rows_reversed", [True, False])
def test_clip_matches_oracle(dev, fmt, track_frame, rows_reversed):
    """The reference's current orders (rows reversed, taps above first) and the grid's."""
    w, h, n = 160, 96, 6
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    frames = synth.moving_clip(w, h, n, depth=depth, seed=0x74570002)
    s = tw.vectors_settings(max_displace=24.0, rows_reversed=rows_reversed, taps_above_first=rows_reversed)
    pairs = [tw.vectors_pair(k, track_frame) for k in range(n)]
    got = dev.create_vectors_clip(s, frames, n, pairs, w, h, fmt)
    want = O.create_vectors_clip(frames, n, w, h, fmt, n, max_displace=24.0, track_frame=track_frame,
                                 rows_reversed=rows_reversed, taps_above_first=rows_reversed)
    assert same(got, want)


def test_1080p_u16_pair_matches_oracle(dev):
    """One frame pair of the 1920x1080 16 bpc workload (solve at 960x540, 8 levels)."""
    w, h = 1920, 1080
    frames = synth.moving_clip(w, h, 2, depth=16, seed=0x74570002, bg_velocity=(6.0, -3.0), square=240,
                               square_start=(600.0, 400.0), square_velocity=(9.0, 4.0))
    s = tw.vectors_settings()
    got = dev.create_vectors_clip(s, frames, 2, [(1, 0)], w, h, 1)
    want = O.create_vectors_clip(frames, 2, w, h, 1, 2)[w * h * 4:]
    assert same(got, want)


@pytest.mark.parametrize("fmt", [0, 1, 2])
def test_engine_entry_matches_oracle(dev, fmt):
    w, h = 97, 61
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    frames = synth.moving_clip(w, h, 2, depth=depth, seed=5)
    n = w * h * 4
    x, y = O.from_frame(frames[:n], w, h, fmt), O.from_frame(frames[n:], w, h, fmt)
    s = tw.vectors_settings(max_displace=10.0)
    got = dev.create_vectors(s, y, x, w, h, fmt)
    flow_b, _, (fw, fh) = O.solve_pair(y, x, w, h, fmt)
    want = O.encode_vectors(flow_b, fw, fh, w, h, fmt, np.float32(10.0))
    assert same(got, want)


@pytest.mark.parametrize("fmt", [0, 1, 2])
def test_encode_special_values(dev, fmt):
    """Clamps, NaN and infinite vectors, a flow of another size than the image."""
    rng = np.random.RandomState(2)
    fw, fh, w, h = 13, 9, 40, 30
    flow = rng.uniform(-30, 30, fw * fh * 2).astype(np.float32)
    flow[rng.randint(0, flow.size, 6)] = np.nan
    flow[rng.randint(0, flow.size, 4)] = np.inf
    flow[rng.randint(0, flow.size, 4)] = -np.inf
    got = dev.encode_vectors(flow, (fw, fh), w, h, fmt, 7.5)
    want = O.encode_vectors(flow, fw, fh, w, h, fmt, 7.5)
    assert same(got, want)


def test_tiny_frames_are_zero_vectors(dev):
    frames = np.arange(1 * 7 * 4 * 3, dtype=np.uint8)
    out = dev.create_vectors_clip(tw.vectors_settings(), frames, 3, [(1, 0), (2, 1)], 1, 7, 0)
    want = O.create_vectors_clip(frames, 3, 1, 7, 0, 3)[7 * 4:]
    assert same(out, want)


# ---- the Debug views (debug.rs) -----------------------------------------------------------------------


def _debug_pair(w, h, fmt, seed, specials=False):
    rng = np.random.default_rng(seed)
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    frames = synth.moving_clip(w, h, 2, depth=depth, seed=seed, square=max(4, min(w, h) // 3))
    x, y = O.from_frame(frames[:w * h * 4], w, h, fmt), O.from_frame(frames[w * h * 4:], w, h, fmt)
    if specials and fmt == 2:
        bits = np.array([0x7FC00000, 0xFFC00000, 0x7F800000, 0xFF800000, 0x00000001, 0x7F7FFFFF, 0x80000000,
                         0x7FA00001], np.uint32).view(np.float32)
        for img in (x, y):
            idx = rng.integers(0, img.size, img.size // 20)
            img[idx] = bits[rng.integers(0, bits.size, idx.size)]
    fw, fh = max(2, w // 2), max(2, h // 2)
    flow = (rng.standard_normal(fw * fh * 2) * 3.0).astype(np.float32)
    return x, y, flow, fw, fh


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("code", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("gouraud", [True, False])
def test_debug_view_matches_oracle(dev, fmt, code, gouraud):
    w, h = 97, 61
    x, y, flow, fw, fh = _debug_pair(w, h, fmt, seed=fmt * 10 + code)
    got = dev.debug_view(x, y, w, h, fmt, flow, (fw, fh), code, gouraud=gouraud)
    want = O.debug_view(x, y, w, h, fmt, flow, fw, fh, code, gouraud=gouraud)
    assert same(got, want)


@pytest.mark.parametrize("code", [0, 1, 2, 3])
def test_debug_view_special_floats(dev, code):
    """Float frames with NaNs of both signs, infinities, denormals and FLT_MAX: the x86 NaN bits of
    the views (the forward warp's, the OVERs', the luma's rule and the measures'). Where a plain
    operation of the Edge measure meets two different NaNs, which one x86 returns is the operand the
    compiler made the destination (debug.rs:295-301 says so of the luma), so there the Edge view is
    compared NaN for NaN and bit for bit elsewhere."""
    w, h = 40, 30
    x, y, flow, fw, fh = _debug_pair(w, h, 2, seed=77 + code, specials=True)
    got = dev.debug_view(x, y, w, h, 2, flow, (fw, fh), code)
    want = O.debug_view(x, y, w, h, 2, flow, fw, fh, code)
    if code != 3:
        assert same(got, want)
    else:
        nan = np.isnan(want)
        assert np.array_equal(np.isnan(got), nan)
        assert got[~nan].view(np.uint32).tobytes() == want[~nan].view(np.uint32).tobytes()
        assert nan.any()


@pytest.mark.parametrize("method", [1, 2, 3, 4, 5])
def test_debug_display_clip_matches_oracle(dev, method):
    """The Debug display over a clip (the reference's current orders: bottom-up rows, the taps above
    first, the Gouraud warp), track Previous, 8 bpc at 160x96."""
    w, h, n = 160, 96, 5
    frames = synth.moving_clip(w, h, n, depth=8, seed=0x7457000A)
    s = tw.vectors_settings(max_displace=24.0, display=3, debug_view_method=method)
    pairs = [tw.vectors_pair(k, 1, debug=True) for k in range(n)]
    got = dev.create_vectors_clip(s, frames, n, pairs, w, h, 0)
    want = O.create_vectors_clip(frames, n, w, h, 0, n, max_displace=24.0, display=3, debug_view_method=method)
    assert same(got, want)
