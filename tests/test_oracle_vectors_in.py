"""The oracle of Vectors In pinned to the reference's fixtures (CPU only).

* the reference's numpy model of the vector image coding (plugins/retime-engine/tests/fixtures/
  vectors_cases.hex, its gen_vectors.py): every decode case (vectors.rs:474-528) and every encode
  case (vectors.rs:57-130) bit for bit;
* the reference's parity grid of the `vectors-in` effect (parity/vectors-in, results/base.grid.tsv):
  the sha256 of the whole output clip of every served case (Speed and Frame Number modes, keyed or
  not, the input rate model). That table was recorded by the revision whose render ran on top-down
  rows, with the vertical border taps below first, the
  textured forward warp, and a vector layer probed at the output frame's time (absent past its
  clip's end; the error fill when neither is there), so those cases run with the four orders off.
"""
import hashlib

import numpy as np
import pytest

import golden_data as G
import oracle_lib as O

CASES = G.vectors_cases()
VI_CASES, VI_INPUTS = G.vi_grid()


@pytest.mark.parametrize("c", CASES, ids=[f"{c['kind']}-d{c['depth']}-{c['w']}x{c['h']}" for c in CASES])
def test_vector_coding_model(c):
    if c["kind"] == "decode":
        got = O.decode_vectors(c["image"], c["w"], c["h"], c["depth"], c["scale"])
        assert got.tobytes() == c["flow"].tobytes()
    else:
        got = O.encode_vectors(c["flow"], c["fw"], c["fh"], c["w"], c["h"], c["depth"], c["scale"])
        assert got.tobytes() == c["image"].tobytes()


def vi_render(c, **orders):
    w, h = c["width"], c["height"]
    fmt = G.FMT_OF_DEPTH[c["depth"]]
    p = O.vecin_params(**G.vi_case_params(c), **orders)
    return O.vectors_in_clip(VI_INPUTS[c["main"]], c["n_main"], VI_INPUTS[c["next"]] if c["next"] else None,
                             c["n_next"], VI_INPUTS[c["prev"]] if c["prev"] else None, c["n_prev"], w, h, fmt, p,
                             c["frames"])


GRID_ORDERS = dict(rows_reversed=False, taps_above_first=False, gouraud=False, probe_current_time=True)


def test_vectors_in_grid_is_served():
    assert len(VI_CASES) == 408
    assert sum(any(x.startswith("src_mark_segments=") for x in c["params"]) for c in VI_CASES) == 9
    assert sum("/" in c["fps"] or "." in c["fps"] for c in VI_CASES) == 9
    groups = {c["id"].split(".")[1].split("-")[0] for c in VI_CASES}
    assert {"size", "warp1", "warp2", "vec", "md16", "scalex2", "prev", "next", "short", "spvecR", "spvecA",
            "spsrc", "blur1", "foot", "fnum", "inrate", "ftime", "key"} <= groups, groups


@pytest.mark.parametrize("c", VI_CASES, ids=[c["id"] for c in VI_CASES])
def test_vectors_in_grid(c):
    out = vi_render(c, **GRID_ORDERS)
    assert hashlib.sha256(out.tobytes()).hexdigest() == c["sha256"]


def test_decode_edges():
    """vectors.rs:474-528 by hand: alpha 0 is the zero vector at every depth; 8 bpc 127 is -1/127
    of Max Displace (254 the denominator); float (R * 2 - 1) * md; a NaN alpha decodes."""
    md = np.float32(10.0)
    img8 = np.array([0, 200, 17, 0, 255, 127, 254, 0, 1, 0, 255, 9], np.uint8)
    f = O.decode_vectors(img8, 3, 1, 0, md)
    assert f[0] == 0.0 and f[1] == 0.0
    assert f[2] == np.float32((127 * 2 / 254 - 1) * 10.0) and f[3] == np.float32(10.0)
    assert f[4] == np.float32(-10.0) and f[5] == np.float32((255 * 2 / 254 - 1) * 10.0)
    imgf = np.array([np.nan, 0.75, 0.25, 0.0, -0.0, 0.9, 0.9, 0.0], np.float32)
    f = O.decode_vectors(imgf, 2, 1, 2, md)
    assert f[0] == np.float32(5.0) and f[1] == np.float32(-5.0)
    assert f[2] == 0.0 and f[3] == 0.0


def test_flow_fill_and_scale():
    """compose/vector.rs:335-345: the alpha 0 holes take the pull-push fill of the known vectors
    (a constant field stays constant up to rounding, a known vector exactly), then Vec Scale
    multiplies every vector."""
    w, h = 20, 14
    img = np.zeros((h, w, 4), np.uint8)
    img[..., 0] = 255
    img[..., 1] = 127 + 50
    img[..., 2] = 127 - 20
    img[4:9, 5:12, 0] = 0  # a hole
    f = O.flow_from_vectors(img.reshape(-1), w, h, 0, 16.0, scale=(2.0, -1.0)).reshape(h, w, 2)
    u = np.float32((177 * 2 / 254 - 1) * 16.0)
    v = np.float32((107 * 2 / 254 - 1) * 16.0)
    known = img[..., 0] != 0
    assert np.all(f[known, 0] == np.float32(2.0) * u) and np.all(f[known, 1] == -v)
    assert np.all(np.abs(f[..., 0] - 2.0 * u) <= 1e-5 * abs(u)) and np.all(np.abs(f[..., 1] + v) <= 1e-5 * abs(v))


def test_invert_constant_flow():
    """compose/vector.rs:370-397: the inversion of a constant flow is its negation wherever the push
    lands, and the fill carries it into the band the push leaves empty."""
    w, h = 24, 16
    flow = np.zeros((h, w, 2), np.float32)
    flow[..., 0], flow[..., 1] = 3.0, -2.0
    for pyramid in (True, False):
        inv = O.invert_flow(flow.reshape(-1), w, h, pyramid=pyramid).reshape(h, w, 2)
        assert np.allclose(inv[..., 0], -3.0, atol=1e-5) and np.allclose(inv[..., 1], 2.0, atol=1e-5)


def test_matte_step():
    """plugins/vectors-in/src/vectorin.rs:125-155: the alpha lowered to the matte in the units of the
    depth; at 8 bpc a NaN matte converts to 0 (the saturating cast), in float it keeps the alpha."""
    img = np.array([200, 1, 2, 3, 100, 4, 5, 6, 255, 7, 8, 9], np.uint8)
    m = np.array([0.5, 0.9, np.nan], np.float32)
    got = O.matte_step(img, 3, 1, 0, m)
    assert list(got[::4]) == [128, 100, 0]
    assert list(got[1::4]) == [1, 4, 7]
    imgf = np.array([0.7, 1, 2, 3, 0.2, 4, 5, 6], np.float32)
    got = O.matte_step(imgf, 2, 1, 2, np.array([np.nan, 0.1], np.float32))
    assert got[0] == np.float32(0.7) and got[4] == np.float32(0.1)


@pytest.mark.parametrize("fps", [(30, 1), (24, 1), (25, 1), (12, 1), (60, 1), (30000, 1001), (2997, 100), (24000, 1001)])
@pytest.mark.parametrize("speed", [50.0, 100.0, 33.3333, 150.0, -50.0, 0.5])
def test_selection_of_the_library(fps, speed):
    """tw_select_vectors_in (the product's host time model of the effect) against the oracle's, for
    the first 40 output frames: the selection and the clip frames of the pair."""
    import twixtor_b200 as tw
    p = O.vecin_params(fps=fps, speed=speed, frame_interp=3, blur=2.5)
    tp = tw.TimeParams(fps=fps, speed_percent=speed, frame_interp=3, blur_compensation=2.5)
    for n in range(40):
        want = O.vecin_select(p, n, 16, 12)
        sel, vf = tw.select_vectors_in(tp, n, 16, 12)
        got = dict(s0=np.float32(sel.s0), s1=np.float32(sel.s1), wa=np.float32(sel.wa), a=sel.a, exact=bool(sel.exact),
                   vq=sel.vectors_quality, interp=sel.interp, clip_a=vf.a, clip_b=vf.b)
        assert got == want, (n, got, want)


def test_library_selection_on_the_grid():
    """tw_select_vectors_in against the oracle's selection on every output frame of every served
    grid case (Speed and Frame Number modes, keyed curves, the input rate model, Src: Mark Segments
    constant or keyed, NTSC and decimal rates)."""
    import twixtor_b200 as tw
    for c in VI_CASES:
        w, h = c["width"], c["height"]
        kw = G.vi_case_params(c)
        p = O.vecin_params(**kw, **GRID_ORDERS)
        tp = tw.TimeParams(fps=kw["fps"], speed_percent=kw["speed"], keys=kw["keys"], frame_interp=kw["frame_interp"],
                           blur_compensation=kw["blur"], remap_mode=kw["remap_mode"], frame_num=kw["frame_num"],
                           fn_keys=kw["fn_keys"], own_input_rate=kw["own_input_rate"],
                           input_frame_rate=kw["input_frame_rate"], mark_segs=kw["mark_segs"], mark_keys=kw["mark_keys"])
        for n in range(c["frames"]):
            want = O.vecin_select(p, n, w, h)
            sel, vf = tw.select_vectors_in(tp, n, w, h)
            got = dict(s0=np.float32(sel.s0), s1=np.float32(sel.s1), wa=np.float32(sel.wa), a=sel.a,
                       exact=bool(sel.exact), vq=sel.vectors_quality, interp=sel.interp, clip_a=vf.a, clip_b=vf.b)
            assert got == want, (c["id"], n, got, want)
