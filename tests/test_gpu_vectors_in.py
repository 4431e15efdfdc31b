"""Parity of the CUDA Vectors In path (tw_decode_vectors, tw_flow_from_vectors, tw_fill_flow_holes,
tw_invert_flow, tw_retime_frame_vectors, tw_vectors_in_clip) with the reference's fixtures and
with the oracle, bit for bit."""
import hashlib

import numpy as np
import pytest

import golden_data as G
import oracle_lib as O
import twixtor_b200 as tw
from twixtor_b200 import synth

pytestmark = pytest.mark.gpu

CASES = G.vectors_cases()
VI_CASES, VI_INPUTS = G.vi_grid()


@pytest.fixture(scope="module")
def dev():
    tw.build()
    d = tw.Device(0)
    yield d
    d.close()


def same(a, b):
    return np.asarray(a).view(np.uint8).tobytes() == np.asarray(b).view(np.uint8).tobytes()


def vec_wire(w, h, n, depth, seed, md=24.0, holes=0.1, partial=0.02):
    """n wire frames of a vector layer: smooth vectors within +-md encoded like the effect reads
    them (8 bpc ((u / md) + 1) * 127, 16 bpc with 32767, float (u / md + 1) / 2), alpha 0 on a
    fraction `holes` of blobs and partial alpha on `partial` of the pixels."""
    rng = np.random.default_rng(seed)
    out = []
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    for t in range(n):
        u = md * 0.6 * np.sin(xx / (w / 3.0) + t + rng.uniform(0, 6)) * np.cos(yy / (h / 2.0))
        v = md * 0.5 * np.cos(xx / (w / 2.0) - yy / (h / 4.0) + rng.uniform(0, 6))
        a = np.ones((h, w))
        for _ in range(max(1, int(holes * 40))):
            cx, cy, r = rng.uniform(0, w), rng.uniform(0, h), rng.uniform(1, max(2, min(w, h) / 6))
            a[(xx - cx) ** 2 + (yy - cy) ** 2 < r * r] = 0.0
        pm = rng.random((h, w)) < partial
        a[pm] = rng.uniform(0.1, 0.9, pm.sum())
        if depth == 8:
            r8 = np.clip(np.floor((u / md + 1.0) * 127.0 + 0.5), 0, 254)
            g8 = np.clip(np.floor((v / md + 1.0) * 127.0 + 0.5), 0, 254)
            px = np.stack([r8, g8, np.zeros_like(r8), np.round(a * 255)], -1).astype(np.uint8)
            out.append(px.reshape(-1))
        elif depth == 16:
            r16 = np.clip(np.floor((u / md + 1.0) * 32767.0 + 0.5), 0, 65534)
            g16 = np.clip(np.floor((v / md + 1.0) * 32767.0 + 0.5), 0, 65534)
            px = np.stack([r16, g16, np.zeros_like(r16), np.round(a * 65535)], -1).astype(np.uint16)
            out.append(px.reshape(-1))
        else:
            rf, gf = ((u / md + 1.0) / 2.0).astype(np.float32), ((v / md + 1.0) / 2.0).astype(np.float32)
            planes = [gf, np.zeros_like(gf), rf, a.astype(np.float32)]  # wire planes G, B, R, A
            out.append(np.concatenate([p.reshape(-1) for p in planes]))
    return np.concatenate(out)


# ---- the primitives --------------------------------------------------------------------------------------


@pytest.mark.parametrize("c", [c for c in CASES if c["kind"] == "decode"],
                         ids=[f"d{c['depth']}-{c['w']}x{c['h']}" for c in CASES if c["kind"] == "decode"])
def test_decode_model(dev, c):
    """The reference's numpy model of the decode (vectors_cases.hex)."""
    got = dev.decode_vectors(c["image"], c["w"], c["h"], c["depth"], c["scale"])
    assert same(got, c["flow"])


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("size", [(37, 23), (160, 96), (481, 271)])
@pytest.mark.parametrize("above_first", [False, True])
def test_flow_from_vectors(dev, fmt, size, above_first):
    w, h = size
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    wire = vec_wire(w, h, 1, depth, seed=w * 7 + fmt)
    eng = O.from_frame(wire, w, h, fmt)
    md, sc = np.float32(24.0), (np.float32(-1.25), np.float32(0.5))
    got = dev.flow_from_vectors(eng, w, h, fmt, md, sc, taps_above_first=above_first)
    want = O.flow_from_vectors(eng, w, h, fmt, md, sc, above_first=above_first)
    assert same(got, want)


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_fill_flow_holes_with_specials(dev, kind):
    """Flow values with NaNs and infinities beside the holes (the NaN rule repeat of the fill)."""
    w, h = 64, 40
    rng = np.random.default_rng(kind)
    flow = rng.normal(0, 5, w * h * 2).astype(np.float32)
    flow[rng.integers(0, flow.size, 30)] = np.nan
    flow[rng.integers(0, flow.size, 10)] = np.inf
    m = rng.random(w * h) < 0.3
    mask = {1: (m * 255).astype(np.uint8), 2: (m * 65535).astype(np.uint16), 3: m.astype(np.float32)}[kind]
    got = dev.fill_flow_holes(flow, w, h, mask, taps_above_first=False)
    want = O.fill_flow_holes(flow, w, h, mask, kind, above_first=False)
    assert same(got, want)


@pytest.mark.parametrize("pyramid", [True, False])
@pytest.mark.parametrize("size", [(48, 32), (320, 180)])
def test_invert_flow(dev, pyramid, size):
    w, h = size
    wire = vec_wire(w, h, 1, 32, seed=11, holes=0.0, partial=0.0)
    eng = O.from_frame(wire, w, h, 2)
    flow = O.flow_from_vectors(eng, w, h, 2, 12.0)
    got = dev.invert_flow(flow, w, h, pyramid=pyramid, taps_above_first=True)
    want = O.invert_flow(flow, w, h, pyramid=pyramid, above_first=True)
    assert same(got, want)


def test_invert_zero_flow_is_negative_zero(dev):
    w, h = 16, 12
    got = dev.invert_flow(np.zeros(w * h * 2, np.float32), w, h)
    assert np.all(got == 0) and np.all(np.signbit(got))


# ---- the effect ---------------------------------------------------------------------------------------


def grid_frames(c):
    """The selections and Vectors In frames of a grid case as the recorded revision made them: a
    vector layer present where its clip has a frame at the output frame's time."""
    w, h = c["width"], c["height"]
    kw = G.vi_case_params(c)
    tp = tw.TimeParams(fps=kw["fps"], speed_percent=kw["speed"], keys=kw["keys"], frame_interp=kw["frame_interp"],
                       blur_compensation=kw["blur"], remap_mode=kw["remap_mode"], frame_num=kw["frame_num"],
                       fn_keys=kw["fn_keys"], own_input_rate=kw["own_input_rate"],
                       input_frame_rate=kw["input_frame_rate"], mark_segs=kw["mark_segs"], mark_keys=kw["mark_keys"])
    sc = tuple(float(tw.fixed_param(v)) for v in kw["vec_scale"])
    sels, vfs = [], []
    for n in range(c["frames"]):
        sel, vf = tw.select_vectors_in(tp, n, w, h, has_next=c["next"] is not None and n < c["n_next"],
                                       has_prev=c["prev"] is not None and n < c["n_prev"], next_scale=sc, prev_scale=sc)
        sels.append(sel)
        vfs.append(vf)
    return kw, sels, vfs


@pytest.mark.parametrize("c", VI_CASES, ids=[c["id"] for c in VI_CASES])
def test_vectors_in_grid_sha256(dev, c):
    """The reference's recorded output clips of the served vectors-in grid cases (the revision with
    top-down rows, the taps below first, the textured forward warp)."""
    w, h = c["width"], c["height"]
    fmt = G.FMT_OF_DEPTH[c["depth"]]
    dt = tw.DTYPES[fmt]
    kw, sels, vfs = grid_frames(c)
    s = tw.vectors_in_settings(warping=kw["warping"], blur=kw["blur"], rows_reversed=False, taps_above_first=False,
                               gouraud=False)
    clip = lambda key: None if key is None else VI_INPUTS[key].view(dt)
    out = dev.vectors_in_clip(s, clip(c["main"]), c["n_main"], clip(c["next"]), c["n_next"], clip(c["prev"]),
                              c["n_prev"], sels, vfs, float(tw.fixed_param(kw["max_displace"])), w, h, fmt)
    assert hashlib.sha256(out.tobytes()).hexdigest() == c["sha256"]


EFFECT = [(wp, fi, nxt, prv) for wp in (1, 2) for fi in (1, 2, 3) for nxt, prv in ((1, 1), (1, 0), (0, 1))]


@pytest.mark.parametrize("fmt", [0, 2])
@pytest.mark.parametrize("wp,fi,nxt,prv", EFFECT)
def test_vectors_in_clip_matches_oracle(dev, fmt, wp, fi, nxt, prv):
    """The reference's current orders (bottom-up rows, the taps above first, the Gouraud forward
    warp, a set layer present at every time) at 96x64 with holes in the vector layers, both or one
    layer (the other inverted), against the oracle's render of the effect."""
    w, h, n, nout = 96, 64, 5, 8
    depth = {0: 8, 2: 32}[fmt]
    frames = synth.moving_clip(w, h, n, depth=depth, seed=0x7451)
    vn = vec_wire(w, h, 4, depth, seed=5) if nxt else None
    vp = vec_wire(w, h, 4, depth, seed=6) if prv else None
    md, speed, blur, scale = 24.0, 40.0, 0.0 if fi != 2 else 1.5, (1.0, -0.75)
    tp = tw.TimeParams(fps=(30, 1), speed_percent=speed, frame_interp=fi, blur_compensation=blur)
    sels, vfs = zip(*[tw.select_vectors_in(tp, k, w, h, has_next=bool(nxt), has_prev=bool(prv),
                                           next_scale=tuple(map(float, map(tw.fixed_param, scale))),
                                           prev_scale=tuple(map(float, map(tw.fixed_param, scale))))
                      for k in range(nout)])
    s = tw.vectors_in_settings(warping=wp, blur=blur)
    got = dev.vectors_in_clip(s, frames, n, vn, 4, vp, 4, list(sels), list(vfs), float(tw.fixed_param(md)), w, h, fmt)
    p = O.vecin_params(speed=speed, frame_interp=fi, warping=wp, blur=blur, max_displace=md, vec_scale=scale)
    want = O.vectors_in_clip(frames, n, vn, 4, vp, 4, w, h, fmt, p, nout)
    assert same(got, want)


def test_frame_entry_matches_clip(dev):
    """tw_retime_frame_vectors renders what tw_vectors_in_clip renders, frame by frame."""
    w, h, n, nout = 64, 48, 4, 6
    frames = synth.moving_clip(w, h, n, depth=16, seed=3)
    vn, vp = vec_wire(w, h, 4, 16, seed=8), vec_wire(w, h, 4, 16, seed=9)
    tp = tw.TimeParams(fps=(30, 1), speed_percent=50.0, frame_interp=3)
    sv = [tw.select_vectors_in(tp, k, w, h) for k in range(nout)]
    s = tw.vectors_in_settings(warping=1)
    clip = dev.vectors_in_clip(s, frames, n, vn, 4, vp, 4, [x[0] for x in sv], [x[1] for x in sv], 16.0, w, h, 1)
    fs = w * h * 4
    at = lambda c, i: c[i * fs:(i + 1) * fs] if 0 <= i < 4 else None
    for k, (sel, vf) in enumerate(sv):
        one = dev.retime_frame_vectors(s, sel, vf, 16.0, at(frames, vf.a), at(frames, vf.b), at(vn, vf.a), at(vp, vf.b),
                                       w, h, 1)
        assert same(one, clip[k * fs:(k + 1) * fs]), k


def test_no_vector_layer_is_the_error_fill(dev):
    w, h = 8, 6
    frames = synth.moving_clip(w, h, 2, depth=8, seed=1)
    sel, vf = tw.select_vectors_in(tw.TimeParams(fps=(30, 1), speed_percent=50.0), 1, w, h, has_next=False,
                                   has_prev=False)
    out = dev.retime_frame_vectors(tw.vectors_in_settings(), sel, vf, 32.0, frames[:w * h * 4], None, None, None, w, h, 0)
    assert np.all(out.reshape(-1, 4) == np.array([255, 0, 0, 128], np.uint8))


@pytest.mark.parametrize("warping", [1, 2])
def test_vectors_in_at_1080p(dev, warping):
    """1920x1080, 8 bpc, both layers with holes: two in-between frames against the oracle."""
    w, h, n = 1920, 1080, 2
    frames = synth.moving_clip(w, h, n, depth=8, seed=0x1080)
    vn, vp = vec_wire(w, h, 1, 8, seed=21), vec_wire(w, h, 2, 8, seed=22)
    tp = tw.TimeParams(fps=(30, 1), speed_percent=30.0)
    sv = [tw.select_vectors_in(tp, k, w, h) for k in (1, 2)]
    s = tw.vectors_in_settings(warping=warping)
    got = dev.vectors_in_clip(s, frames, n, vn, 1, vp, 2, [x[0] for x in sv], [x[1] for x in sv], 24.0, w, h, 0)
    p = O.vecin_params(speed=30.0, warping=warping, max_displace=24.0)
    fs = w * h * 4
    for i, k in enumerate((1, 2)):
        want = O.vectors_in_clip(frames, n, vn, 1, vp, 2, w, h, 0, p, k + 1)[k * fs:(k + 1) * fs]
        assert same(got[i * fs:(i + 1) * fs], want), k
