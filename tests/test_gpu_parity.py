"""Parity of the CUDA path (through the C ABI) with the oracle, bit for bit.

Every comparison is on bytes: flows as float bits, frames as samples. Inputs are seeded; the
oracle is the pinned CPU restatement of the reference (tests/test_oracle_pins.py). The end to end
cases of the reference's parity grid are checked against its recorded sha256 directly.
"""
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


def rand_engine(rng, w, h, fmt):
    """A random premultiplied engine image through the oracle's own from_frame."""
    if fmt == 0:
        wire = rng.randint(0, 256, w * h * 4).astype(np.uint8)
    elif fmt == 1:
        wire = rng.randint(0, 65536, w * h * 4).astype(np.uint16)
    else:
        wire = rng.random_sample(w * h * 4).astype(np.float32)
    return O.from_frame(wire, w, h, fmt), wire


CASES_ALL, INPUTS_ALL = golden_data.grid()


def grid_settings(kw):
    """The settings of a retime grid case (the grid's revision: rows top down, taps below first)."""
    return tw.RetimeSettings(
        flow=tw.FlowSettings(hiq=True, sensitivity=np.float32(np.float32(kw["sensitivity"]) / np.float32(100.0)),
                             taps_above_first=False, video_range_luma=kw["video_360"],
                             prep_contrast_edge=kw["prep"] == 2, prep_delinearize=kw["prep"] == 3),
        compose=tw.EngineSettings(warp_mode=kw["smart_blend"], video_360=kw["video_360"], taps_above_first=False,
                                  blur=float(tw.fixed_param(kw["blur"]))),
        motion_rows_reversed=False)

# ---- image boundary ------------------------------------------------------------------------------

@pytest.mark.parametrize("fmt", [0, 1, 2])
def test_from_and_to_frame(dev, fmt):
    rng = np.random.RandomState(11 + fmt)
    w, h = 37, 23
    eng, wire = rand_engine(rng, w, h, fmt)
    assert same(dev.from_frame(wire, w, h, fmt), eng)
    # to_frame of arbitrary engine samples (alpha 0 and above-alpha colours included)
    if fmt == 2:
        e = (rng.random_sample(w * h * 4) * 1.5 - 0.1).astype(np.float32)
    else:
        e = rng.randint(0, 256 if fmt == 0 else 65536, w * h * 4).astype(tw.DTYPES[fmt])
        e[::16] = 0
    assert same(dev.to_frame(e, w, h, fmt), O.to_frame(e, w, h, fmt))


# ---- warps and blends ------------------------------------------------------------------------------

WARP = golden_data.warp_cases()


@pytest.mark.parametrize("i", range(len(WARP)))
def test_inverse_warp_reference_fixtures(dev, i):
    """Every case of warp_cases.hex, the 360 ones included."""
    c = WARP[i]
    r = dev.inv_warp(c["src"], c["w"], c["h"], c["fmt"], c["flow"], (c["fw"], c["fh"]), c["amount"], hold=c["hold"],
                     coverage=c["want_cov"], is360=c["is360"])
    out, cov = r if c["want_cov"] else (r, None)
    assert same(out, c["out"])
    if c["want_cov"]:
        assert (cov == c["cov"]).all()


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("w", [0.0, 0.003, 0.25, 0.5, 0.9971, 1.0, -0.4, 1.3])
def test_blend_all_branches(dev, fmt, w):
    rng = np.random.RandomState(5)
    W, H = 19, 13
    a, _ = rand_engine(rng, W, H, fmt)
    b, _ = rand_engine(rng, W, H, fmt)
    want = np.zeros_like(a)
    O.lib().or_blend(O.ptr(want), O.ptr(a), O.ptr(b), W, H, fmt, np.float32(w))
    assert same(dev.blend(a, b, W, H, fmt, w), want)


# ---- pyramid and solver ---------------------------------------------------------------------------

@pytest.mark.parametrize("size", [(160, 96), (33, 31), (7, 9), (2, 2), (3, 3), (64, 48), (241, 17)])
@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("above_first", [True, False])
def test_pyramid_levels(dev, size, fmt, above_first):
    w, h = size
    rng = np.random.RandomState(w * 31 + h + fmt)
    eng, _ = rand_engine(rng, w, h, fmt)
    for q, hiq in ((4, True), (5, True), (3, False)):
        s = tw.FlowSettings(quality=q, hiq=hiq, taps_above_first=above_first)
        got = dev.build_pyramid(eng, w, h, fmt, s)
        want = O.build_pyramid(eng, w, h, fmt, quality=q, hiq=hiq, above_first=above_first)
        assert len(got) == len(want)
        for g, o in zip(got, want):
            assert same(g, o)


@pytest.mark.parametrize("size", [(12, 10), (40, 30), (97, 61), (3, 3), (5, 200), (960, 540)])
@pytest.mark.parametrize("kind", ["noise", "smooth", "constant"])
def test_block_match_sweeps(dev, size, kind):
    """Random fields make long accepted runs and many run starts; the sweep is a loop-carried
    recurrence, so this checks the parallel run decomposition against the sequential oracle."""
    w, h = size
    rng = np.random.RandomState(w + 7 * h)
    a = (rng.random_sample((h, w)) * 50).astype(np.float32)
    b = np.roll(a, 1, axis=1) + (rng.random_sample((h, w)) * 2).astype(np.float32)
    if kind == "noise":
        flow = ((rng.random_sample(w * h * 2) - 0.5) * 6).astype(np.float32)
    elif kind == "smooth":
        yy, xx = np.mgrid[0:h, 0:w]
        flow = np.stack([np.sin(xx / 7.0) * 2 - 1, np.cos(yy / 5.0) * 1.5], -1).astype(np.float32).reshape(-1)
        flow += (rng.random_sample(flow.size) * 0.2).astype(np.float32)
    else:
        flow = np.full(w * h * 2, -1.0, np.float32)
        flow[::7] = 0.5
    want = flow.copy()
    O.lib().or_block_match(O.ptr(a), O.ptr(b), O.ptr(want), w, h)
    got = dev.block_match(a, b, flow, w, h)
    assert same(got, want)


def clip_pair(w, h, fmt, seed, t=3):
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    frames = synth.moving_clip(w, h, t + 2, depth=depth, seed=seed)
    n = w * h * 4
    wa, wb = frames[t * n:(t + 1) * n], frames[(t + 1) * n:(t + 2) * n]
    return O.from_frame(wa, w, h, fmt), O.from_frame(wb, w, h, fmt), wa, wb


@pytest.mark.parametrize("size,fmt", [((160, 96), 0), ((160, 96), 1), ((160, 96), 2), ((97, 61), 0), ((64, 48), 2),
                                      ((6, 5), 0), ((320, 180), 0)])
@pytest.mark.parametrize("sens,quality,hiq", [(0.7, 4, True), (1.0, 5, True), (0.33, 4, True), (0.7, 3, False)])
@pytest.mark.parametrize("above_first", [True, False])
def test_solve_pair_bit_exact(dev, size, fmt, sens, quality, hiq, above_first):
    w, h = size
    a, b, _, _ = clip_pair(w, h, fmt, seed=0x74570001 + w)
    s = tw.FlowSettings(quality=quality, hiq=hiq, sensitivity=np.float32(sens), taps_above_first=above_first)
    f_ab, f_ba, fs = dev.solve_pair(a, b, w, h, fmt, s)
    o_ab, o_ba, ofs = O.solve_pair(a, b, w, h, fmt, quality=quality, hiq=hiq, sensitivity=np.float32(sens),
                                   above_first=above_first)
    assert fs == ofs
    assert same(f_ab, o_ab)
    assert same(f_ba, o_ba)
    if w >= 64 and sens > 0.5:
        assert np.abs(f_ab).max() > 0  # the solve moved


def test_solve_skip_refine(dev):
    w, h = 160, 96
    a, b, _, _ = clip_pair(w, h, 0, seed=3)
    s = tw.FlowSettings(skip_refine=True)
    f_ab, f_ba, _ = dev.solve_pair(a, b, w, h, 0, s)
    o_ab, o_ba, _ = O.solve_pair(a, b, w, h, 0, skip_refine=True)
    assert same(f_ab, o_ab) and same(f_ba, o_ba)


# ---- composition ------------------------------------------------------------------------------------

@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("wa,interp", [(0.5, 1), (0.75, 1), (0.2, 1), (0.999, 1), (1.0, 1), (1.5, 1), (0.6, 0),
                                       (0.3, 0)])
def test_compose_vectors(dev, fmt, wa, interp):
    w, h = 96, 64
    a, b, _, _ = clip_pair(w, h, fmt, seed=9)
    o_ab, o_ba, (fw, fh) = O.solve_pair(a, b, w, h, fmt)
    sel = tw.Selection(wa=np.float32(wa), interp=interp)
    got = dev.compose_vectors(tw.EngineSettings(), sel, a, b, w, h, fmt, o_ab, o_ba, (fw, fh))
    want = O.compose_vectors(a, b, w, h, fmt, o_ab, o_ba, fw, fh, np.float32(wa), interp)
    assert same(got, want)


# ---- Smart Blend and the hole fill --------------------------------------------------------------------

F1 = golden_data.f1_cases()


@pytest.mark.parametrize("i", range(len(F1)))
def test_smart_blend_and_hole_fill_model_fixtures(dev, i):
    """The reference's numpy models of Smart Blend (kind 1), its binary alpha variant (kind 2) and
    the hole fill (kind 3, below first taps), on the device."""
    c = F1[i]
    w, h, fmt = c["w"], c["h"], c["fmt"]
    if c["kind"] in (1, 2):
        out = dev.smart_blend(c["p1"], c["p2"], w, h, fmt, c["weight"], binary=c["kind"] == 2)
    else:
        out = dev.fill_holes(c["p1"], w, h, fmt, c["mask"], taps_above_first=False)
    assert same(out, c["out"])


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("size", [(37, 23), (96, 64), (250, 131)])
@pytest.mark.parametrize("above_first", [False, True])
@pytest.mark.parametrize("kind", [1, 2, 3])
def test_hole_fill_random_masks(dev, fmt, size, above_first, kind):
    """Random images and masks of each kind (sparse holes, a large hole, NaN mask values)."""
    w, h = size
    rng = np.random.RandomState(w * 7 + h + kind * 131 + fmt)
    img, _ = rand_engine(rng, w, h, fmt)
    n = w * h
    if kind == 1:
        mask = (rng.random_sample(n) < 0.3).astype(np.uint8) * rng.randint(1, 256, n).astype(np.uint8)
    elif kind == 2:
        mask = np.where(rng.random_sample(n) < 0.3, rng.randint(1, 65536, n), 0).astype(np.uint16)
    else:
        mask = np.where(rng.random_sample(n) < 0.3, rng.random_sample(n), 0.0).astype(np.float32)
        mask[rng.randint(0, n, 5)] = np.nan
        mask[rng.randint(0, n, 5)] = 3.0e-5  # just below the threshold: not a hole
    m2 = mask.reshape(h, w)
    m2[h // 4:h // 2, w // 3:w // 2] = {1: 255, 2: 65535, 3: 1.0}[kind]
    got = dev.fill_holes(img, w, h, fmt, mask, taps_above_first=above_first)
    want = O.fill_holes(img, w, h, fmt, mask, kind, above_first)
    assert same(got, want)


def test_hole_fill_nan_samples_and_identity(dev):
    """NaN float samples next to holes take the NaN rule's bits; a mask without a hole leaves the
    image unchanged, NaN payloads included."""
    w, h = 64, 40
    rng = np.random.RandomState(5)
    img, _ = rand_engine(rng, w, h, 2)
    img[rng.randint(0, img.size, 40)] = np.float32(np.nan)
    img.view(np.uint32)[rng.randint(0, img.size, 10)] = 0xffc01234
    mask = (rng.random_sample(w * h) < 0.2).astype(np.uint8)
    assert same(dev.fill_holes(img, w, h, 2, mask), O.fill_holes(img, w, h, 2, mask, 1))
    none = np.zeros(w * h, np.uint8)
    assert same(dev.fill_holes(img, w, h, 2, none), img)


def test_hole_fill_side_of_one_pixel(dev):
    img = np.zeros(1 * 9 * 4, np.uint8)
    with pytest.raises(tw.Unsupported):
        dev.fill_holes(img, 1, 9, 0, np.ones(9, np.uint8))
    assert same(dev.fill_holes(img, 1, 9, 0, np.zeros(9, np.uint8)), img)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("wa,interp", [(0.5, 1), (0.75, 1), (0.2, 1), (0.0, 1), (0.6, 0), (0.3, 0), (0.5, 0)])
@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("above_first", [False, True])
def test_compose_smart_blend(dev, fmt, wa, interp, binary, above_first):
    """Warping code 1 through compose_vectors: the warps without hold, Smart Blend and the fill of
    the uncovered pixels. The flows are the solved ones scaled up so that the borders uncover."""
    w, h = 96, 64
    a, b, _, _ = clip_pair(w, h, fmt, seed=21)
    o_ab, o_ba, (fw, fh) = O.solve_pair(a, b, w, h, fmt)
    o_ab = (o_ab * np.float32(6.0) + np.float32(3.5)).astype(np.float32)
    o_ba = (o_ba * np.float32(6.0) - np.float32(2.25)).astype(np.float32)
    sel = tw.Selection(wa=np.float32(wa), interp=interp)
    cs = tw.EngineSettings(warp_mode=1, video_360=binary, taps_above_first=above_first)
    got = dev.compose_vectors(cs, sel, a, b, w, h, fmt, o_ab, o_ba, (fw, fh))
    want = O.compose_vectors2(a, b, w, h, fmt, o_ab, o_ba, fw, fh, np.float32(wa), interp, 1, binary, above_first)
    assert same(got, want)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("code", [2, 3])
@pytest.mark.parametrize("gouraud", [False, True])
@pytest.mark.parametrize("wa,interp", [(0.5, 1), (0.75, 1), (0.2, 1), (0.6, 0), (0.3, 0)])
@pytest.mark.parametrize("binary", [False, True])
def test_compose_forward_codes(dev, fmt, code, gouraud, wa, interp, binary):
    """Warping codes 2 (coverage, Smart Blend, combine, invert, fill) and 3 (the plain blend) through
    compose_vectors: each frame pushed by its own flow with the textured or the Gouraud forward warp.
    The flows are the solved ones scaled up so that the borders uncover."""
    w, h = 96, 64
    a, b, _, _ = clip_pair(w, h, fmt, seed=23)
    o_ab, o_ba, (fw, fh) = O.solve_pair(a, b, w, h, fmt)
    o_ab = (o_ab * np.float32(5.0) + np.float32(2.5)).astype(np.float32)
    o_ba = (o_ba * np.float32(5.0) - np.float32(1.75)).astype(np.float32)
    sel = tw.Selection(wa=np.float32(wa), interp=interp)
    cs = tw.EngineSettings(warp_mode=code, video_360=binary, gouraud=gouraud)
    got = dev.compose_vectors(cs, sel, a, b, w, h, fmt, o_ab, o_ba, (fw, fh))
    want = O.compose_vectors2(a, b, w, h, fmt, o_ab, o_ba, fw, fh, np.float32(wa), interp, code, binary, True, gouraud)
    assert same(got, want)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("code", [0, 1, 2, 3])
@pytest.mark.parametrize("size", [(96, 64), (7, 2), (2, 9), (3, 4), (5, 5), (33, 3)])
@pytest.mark.parametrize("wa", [0.3, 0.5, 0.85])
@pytest.mark.parametrize("above_first", [False, True])
def test_compose_weighted_blend(dev, fmt, code, size, wa, above_first):
    """Weighted Blend (compose/vector.rs:255-272, smartblend.rs:400-456, forward.rs:498-572) for the four
    warping codes: the sharpening step of each warped frame (difference mask and its clean-up,
    the blur with its edge formula, the unsharp lerp, the masked composite), then the blend or the
    Smart Blend with the fill; sizes below 3 take the reference's border copy with its float tests."""
    w, h = size
    rng = np.random.RandomState(w * 131 + h * 7 + fmt)
    a, b, _, _ = clip_pair(w, h, fmt, seed=29 + w + h)
    fw, fh = max(w // 2, 2), max(h // 2, 2)
    f_ab = rng.uniform(-3.0, 3.0, fw * fh * 2).astype(np.float32)
    f_ba = rng.uniform(-3.0, 3.0, fw * fh * 2).astype(np.float32)
    sel = tw.Selection(wa=np.float32(wa), interp=2)
    cs = tw.EngineSettings(warp_mode=code, taps_above_first=above_first, gouraud=code == 3)
    got = dev.compose_vectors(cs, sel, a, b, w, h, fmt, f_ab, f_ba, (fw, fh))
    want = O.compose_vectors2(a, b, w, h, fmt, f_ab, f_ba, fw, fh, np.float32(wa), 2, code, False, above_first,
                              code == 3)
    assert same(got, want)


@pytest.mark.parametrize("size", [(24, 16), (5, 1), (2, 2), (40, 3)])
def test_weighted_blend_without_flows_of_unsound_floats(dev, size):
    """Float frames with NaNs, infinities and huge values take every filter of Weighted Blend on the
    fast path (blend.rs:276-324); sound float frames the plain blend of a + 0 and b + 0. The device
    decides with a flag and gated kernels."""
    w, h = size
    n = 3
    rng = np.random.RandomState(w + h)
    frames = rng.uniform(0.0, 1.0, n * w * h * 4).astype(np.float32)
    special = np.array([np.nan, np.inf, -np.inf, 3e30, -0.0, 1e-40], np.float32)
    idx = rng.choice(frames.size, max(frames.size // 7, 1), replace=False)
    frames[idx] = special[rng.randint(0, len(special), idx.size)]
    sound = rng.uniform(0.0, 1.0, n * w * h * 4).astype(np.float32)
    sound[::5] = -0.0
    for clip in (frames, sound):
        for speed in (50.0, 100.0):
            tp = tw.TimeParams(speed_percent=speed, vectors=1, frame_interp=3)
            got = tw.retime_clip(dev, clip, n, w, h, 2, tp, n)
            want = O.retime_clip(clip, n, w, h, 2, O.retime_params(speed=speed, vectors=1, frame_interp=3), n)
            assert same(got, want)


@pytest.mark.parametrize("case", [c for c in CASES_ALL if c["id"] in golden_data.KNOWN_GAPS],
                         ids=lambda c: c["id"])
def test_known_gap_cases_equal_the_oracle(dev, case):
    """The grid cases the restatement does not reproduce yet: the CUDA path still equals the oracle."""
    fmt = golden_data.FMT_OF_DEPTH[case["depth"]]
    raw = INPUTS_ALL[case["input"]].view(tw.DTYPES[fmt])
    kw = golden_data.case_params(case)
    tp = tw.TimeParams(fps=kw["fps"], speed_percent=kw["speed"], keys=kw["keys"], vectors=kw["vectors"],
                       frame_interp=kw["frame_interp"], blur_compensation=kw["blur"])
    settings = grid_settings(kw)
    out = tw.retime_clip(dev, raw, case["frames"], case["width"], case["height"], fmt, tp, case["frames"], settings)
    want = O.retime_clip(raw, case["frames"], case["width"], case["height"], fmt, O.retime_params(**kw), case["frames"])
    assert same(out, want)


BLUR = golden_data.blur_cases()


@pytest.mark.parametrize("i", range(len(BLUR)))
def test_motion_blur_model_fixtures(dev, i):
    """Blur Compensation's motion blur (warp/blurcomp.rs) against the reference's model fixtures."""
    c = BLUR[i]
    got = dev.motion_blur(c["src"], c["w"], c["h"], c["fmt"], c["flow"], (c["fw"], c["fh"]), c["amount"], c["hiq"],
                          c["shutter"])
    assert same(got, c["out"])


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("code", [0, 1, 2, 3])
@pytest.mark.parametrize("s0,s1,blur", [(3.0, 0.5, 1.0), (1.2, 1.0, 2.0), (0.0, 3.5, 0.25), (1.0, 1.2, 0.004)])
@pytest.mark.parametrize("hiq", [True, False])
def test_compose_blur_compensation(dev, fmt, code, s0, s1, blur, hiq):
    """The Blur Compensation tail of compose_vectors: the motion blur along F_AB of the composite, with
    the clear of a positive amount and the lerp of a negative one; below the slider's threshold none."""
    w, h = 64, 40
    rng = np.random.RandomState(fmt * 7 + code)
    a, b, _, _ = clip_pair(w, h, fmt, seed=31)
    fw, fh = 32, 20
    f_ab = rng.uniform(-4.0, 4.0, fw * fh * 2).astype(np.float32)
    f_ba = rng.uniform(-4.0, 4.0, fw * fh * 2).astype(np.float32)
    sel = tw.Selection(s0=np.float32(s0), s1=np.float32(s1), wa=np.float32(0.6), interp=1)
    cs = tw.EngineSettings(warp_mode=code, blur=blur, quality_high=hiq, gouraud=code == 3)
    got = dev.compose_vectors(cs, sel, a, b, w, h, fmt, f_ab, f_ba, (fw, fh))
    want = O.compose_vectors3(a, b, w, h, fmt, f_ab, f_ba, fw, fh, sel, cs)
    assert same(got, want)


def test_device_powf_traced_vectors(dev):
    """The Delinearize powf on the device equals the plugin runtime's traced values."""
    v = np.array(golden_data.crt_powf_traced(), np.uint32)
    got = dev.check_powf(v[:, 0].view(np.float32), v[:, 1].view(np.float32))
    assert (got.view(np.uint32) == v[:, 2]).all()
    rng = np.random.RandomState(5)
    x = np.concatenate([rng.uniform(0, 4, 200000), rng.uniform(0.93, 1.07, 200000), [0.0, -0.0, np.inf, np.nan, 1e-40,
                                                                                      3e38 / 255]]).astype(np.float32)
    y = np.float32(1.0) / np.float32(2.2)
    assert (dev.check_powf(x, y).view(np.uint32) == O.crt_powf(x, y).view(np.uint32)).all()


@pytest.mark.parametrize("prep", [2, 3])
@pytest.mark.parametrize("fmt", [0, 2])
def test_prep_pyramids(dev, prep, fmt):
    """Image prep on level 0 of the pyramid: Delinearize and Contrast / Edge Enhance at 320x180."""
    w, h = 320, 180
    a, b, _, _ = clip_pair(w, h, fmt, seed=37)
    fs = tw.FlowSettings(prep_contrast_edge=prep == 2, prep_delinearize=prep == 3)
    got = dev.build_pyramid(a, w, h, fmt, fs)
    want = O.build_pyramid(a, w, h, fmt, prep=prep)
    assert len(got) == len(want) and all(same(g, x) for g, x in zip(got, want))


# ---- whole output frames -----------------------------------------------------------------------------

CASES, INPUTS = golden_data.grid()


@pytest.mark.parametrize("case", golden_data.grid_params(CASES))
def test_retime_flow_grid_sha256(dev, case):
    """The reference's recorded output of every served grid case, rendered by the CUDA path."""
    fmt = golden_data.FMT_OF_DEPTH[case["depth"]]
    raw = INPUTS[case["input"]].view(tw.DTYPES[fmt])
    kw = golden_data.case_params(case)
    tp = tw.TimeParams(fps=kw["fps"], speed_percent=kw["speed"], keys=kw["keys"], vectors=kw["vectors"],
                       frame_interp=kw["frame_interp"], blur_compensation=kw["blur"])
    settings = grid_settings(kw)
    out = tw.retime_clip(dev, raw, case["frames"], case["width"], case["height"], fmt, tp, case["frames"], settings)
    assert hashlib.sha256(out.tobytes()).hexdigest() == case["sha256"]


def test_retime_config1_clip_matches_oracle(dev):
    """160x96 8 bpc, 48 frames to 95 output frames at speed 50 %, the reference's current orders."""
    w, h, n = 160, 96, 48
    frames = synth.moving_clip(w, h, n, depth=8)
    tp = tw.TimeParams(speed_percent=50.0)
    out = tw.retime_clip(dev, frames, n, w, h, 0, tp, 95)
    want = O.retime_clip(frames, n, w, h, 0, O.retime_params(speed=50.0), 95)
    assert same(out, want)


@pytest.mark.parametrize("fmt", [0, 1])
def test_1080p_frame_matches_oracle(dev, fmt):
    """One full size in-between frame (1920x1080, solve at 960x540, 8 levels)."""
    w, h = 1920, 1080
    depth = {0: 8, 1: 16}[fmt]
    frames = synth.moving_clip(w, h, 2, depth=depth, seed=0x74570002, bg_velocity=(6.0, -3.0),
                               square=240, square_start=(600.0, 400.0), square_velocity=(9.0, 4.0))
    tp = tw.TimeParams(speed_percent=40.0)
    sel = tw.select(tp, 1, w, h)  # s0 = 0.4
    n = w * h * 4
    out = dev.retime_frame(tw.RetimeSettings(), sel, frames[:n], frames[n:2 * n], w, h, fmt)
    want = O.retime_clip(frames, 2, w, h, fmt, O.retime_params(speed=40.0), 2)[n:2 * n]
    assert same(out, want)


def test_frames_outside_the_clip_are_blank(dev):
    w, h, n = 48, 32, 4
    frames = synth.moving_clip(w, h, n, depth=8, seed=77)
    tp = tw.TimeParams(speed_percent=150.0)
    out = tw.retime_clip(dev, frames, n, w, h, 0, tp, 6)
    want = O.retime_clip(frames, n, w, h, 0, O.retime_params(speed=150.0), 6)
    assert same(out, want)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("w,h", [(24, 16), (97, 61), (320, 180), (12, 8)])
@pytest.mark.parametrize("track_alpha", [False, True])
def test_pyramid_360_mode_matches_oracle(dev, fmt, w, h, track_alpha):
    """The 360 mode of the pyramid's filters (the luma pyramids of retime-fgbg's layered solves with
    Track RGB+A): circular rows, equirectangular columns and resample, odd widths included."""
    depth = {0: 8, 1: 16, 2: 32}[fmt]
    wire = synth.moving_clip(w, h, 1, depth=depth, seed=w + h)
    eng = O.from_frame(wire, w, h, fmt)
    for q, hiq in [(4, True), (3, False)]:
        s = tw.FlowSettings(quality=q, hiq=hiq, wrap=True, track_alpha=track_alpha)
        got = dev.build_pyramid(eng, w, h, fmt, s)
        want = O.build_pyramid(eng, w, h, fmt, quality=q, hiq=hiq, wrap=True, track_alpha=track_alpha)
        for lv, (g, x) in enumerate(zip(got, want)):
            assert g.tobytes() == x.tobytes(), f"level {lv}"


def test_unsupported_settings_fail_loudly(dev):
    w, h = 32, 24
    a, b, _, _ = clip_pair(w, h, 0, seed=1)
    with pytest.raises(tw.Unsupported):
        dev.solve_pair(a, b, w, h, 0, tw.FlowSettings(wrap=True))  # the wrap-around (360) solve
    with pytest.raises(tw.BadParam):
        dev.solve_pair(a, b, w, h, 0, tw.FlowSettings(quality=0))
    # the forward compositions read counts back: not on the lanes of the clip calls
    frames = synth.moving_clip(w, h, 2, depth=8)
    sel = tw.select(tw.TimeParams(speed_percent=50.0), 1, w, h)
    with pytest.raises(tw.Unsupported):
        dev.retime_clip(tw.RetimeSettings(compose=tw.EngineSettings(warp_mode=2)), frames, 2, [sel], w, h, 0)


@pytest.mark.parametrize("speed,n,nout,size", [(50.0, 48, 95, (160, 96)), (150.0, 8, 12, (64, 48)),
                                               (33.3333, 12, 30, (97, 61)), (-50.0, 6, 8, (48, 32))])
def test_retime_clip_host_buffers(dev, speed, n, nout, size):
    """tw_retime_clip: the clip in host memory, a device frame cache with eviction, frames past the
    clip's ends blank, three output frames in flight; every output byte equals the oracle's."""
    w, h = size
    frames = synth.moving_clip(w, h, n, depth=8, seed=int(speed * 10) & 0xffff)
    tp = tw.TimeParams(speed_percent=speed)
    sels = [tw.select(tp, k, w, h) for k in range(nout)]
    out = dev.retime_clip(tw.RetimeSettings(), frames, n, sels, w, h, 0)
    want = O.retime_clip(frames, n, w, h, 0, O.retime_params(speed=speed), nout)
    assert same(out, want)


def test_retime_clip_device_matches_host_clip(dev):
    import torch
    w, h, n = 160, 96, 10
    frames = synth.moving_clip(w, h, n, depth=8, seed=5)
    tp = tw.TimeParams(speed_percent=40.0)
    sels = [tw.select(tp, k, w, h) for k in range(20)]
    host = dev.retime_clip(tw.RetimeSettings(), frames, n, sels, w, h, 0)
    d_in = torch.from_numpy(frames).cuda()
    d_out = torch.zeros(len(sels) * w * h * 4, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    dev.retime_clip_device(tw.RetimeSettings(), d_in.data_ptr(), n, sels, w, h, 0, d_out.data_ptr())
    assert same(d_out.cpu().numpy(), host)


def test_batch_of_uneven_clips_equals_each_clip(dev):
    """tw_retime_batch_device: three clips of different sizes and depths in one call, frames of the
    clips in flight together, each output equal to its own clip call."""
    import torch
    specs = [(96, 64, 0, 50.0), (160, 96, 2, 40.0), (64, 48, 1, 75.0)]
    jobs, keep, want = [], [], []
    for i, (w, h, fmt, speed) in enumerate(specs):
        n = 8
        frames = synth.moving_clip(w, h, n, depth={0: 8, 1: 16, 2: 32}[fmt], seed=40 + i)
        tp = tw.TimeParams(speed_percent=speed)
        sels = [tw.select(tp, k, w, h) for k in range(10)]
        want.append(tw.retime_clip(dev, frames, n, w, h, fmt, tp, 10))
        t = torch.from_numpy(frames).cuda()
        out = torch.zeros(10 * w * h * 4, dtype=t.dtype, device="cuda")
        keep += [t, out]
        jobs.append(dict(settings=tw.RetimeSettings(), frames=t.data_ptr(), nframes=n, sels=sels, width=w, height=h,
                         fmt=fmt, out=out.data_ptr()))
    dev.set_lanes(4)
    dev.retime_batch_device(jobs)
    for (w, h, fmt, _), out, wnt in zip(specs, keep[1::2], want):
        assert same(out.cpu().numpy(), wnt)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("size", [(37, 23), (160, 96), (1920, 1080)])
def test_inverse_warp_360_matches_oracle(dev, fmt, size):
    """The 360 inverse warp with flows of several turns in both axes (the pole reflection on odd
    vertical wraps, the half-width shift below the last row) against the oracle."""
    w, h = size
    rng = np.random.RandomState(w + fmt)
    src, _ = rand_engine(rng, w, h, fmt)
    fw, fh = max(2, w // 2), max(2, h // 2)
    flow = (rng.standard_normal(fw * fh * 2) * np.float32(max(w, h) * 0.8)).astype(np.float32)
    for amount in (1.0, -0.6, 2.5):
        got, cov = dev.inv_warp(src, w, h, fmt, flow, (fw, fh), amount, coverage=True, is360=True)
        want, wcov = O.inv_warp(src, w, h, fmt, flow, fw, fh, amount, coverage=True, is360=True)
        assert same(got, want), amount
        assert (cov == 255).all() and (wcov == 255).all()
