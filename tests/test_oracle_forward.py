"""Pins the forward warp of the CPU oracle (forward.rs, forward/{mesh,raster,pyramid}.rs).

* the reference's numpy model fixtures of the textured forward warp (tests/fixtures/f2_cases.hex):
  coverage and the u8 / u16 samples bit for bit, f32 within 2e-6 (the model takes numpy's log for
  the mip level where the engine calls libm's logf, the reference's own tolerance);
* the hand values of the reference's forward warp unit tests (forward/tests.rs).
"""
import numpy as np
import pytest

import golden_data
import oracle_lib as O

F2 = golden_data.f2_cases()


@pytest.mark.parametrize("i", range(len(F2)))
def test_textured_forward_warp_model_fixtures(i):
    c = F2[i]
    out, cov = O.forward_warp(c["src"], c["w"], c["h"], c["fmt"], c["flow"], c["fw"], c["fh"], c["amount"], True, True)
    assert (cov == c["cov"]).all()
    if c["fmt"] == 2:
        assert np.abs(out - c["out"]).max() <= 2e-6
    else:
        assert (out == c["out"]).all()


def const_img(w, h, fmt, px):
    dt = {0: np.uint8, 1: np.uint16, 2: np.float32}[fmt]
    return np.tile(np.asarray(px, dt), w * h)


def const_flow(w, h, v):
    return np.tile(np.asarray(v, np.float32), w * h)


@pytest.mark.parametrize("fmt,px", [(0, [255, 200, 100, 50]), (1, [65535, 51000, 25000, 12800]),
                                    (2, [1.0, 0.8, 0.4, 0.2])])
def test_translation_of_a_constant_image(fmt, px):
    """forward/tests.rs:86-124: flow (2, 0) covers the columns 2.. of every row."""
    w, h = 10, 8
    out, cov = O.forward_warp(const_img(w, h, fmt, px), w, h, fmt, const_flow(w, h, [2.0, 0.0]), w, h, 1.0, True, True)
    cov = cov.reshape(h, w)
    assert (cov[:, 2:] == 255).all() and (cov[:, :2] == 0).all()
    o = out.reshape(h, w, 4)
    assert np.abs(o[:, 2:].astype(np.float64) - np.asarray(px, np.float64)).max() <= 1e-6
    assert (o[:, :2] == 0).all()


def test_vertical_translation_leaves_the_top_rows_as_holes():
    w = h = 8
    out, cov = O.forward_warp(const_img(w, h, 0, [255, 10, 20, 30]), w, h, 0, const_flow(w, h, [0.0, 3.0]), w, h, 1.0,
                              True, True)
    rows = np.arange(h)[:, None].repeat(w, 1)
    assert (cov.reshape(h, w) == np.where(rows >= 3, 255, 0)).all()
    assert (out.reshape(h, w, 4)[:, :, 0] == np.where(rows >= 3, 255, 0)).all()


def test_flow_beyond_the_image():
    w, h = 10, 8
    src = const_img(w, h, 0, [255, 1, 2, 3])
    out, cov = O.forward_warp(src, w, h, 0, const_flow(w, h, [50.0, 0.0]), w, h, 1.0, True, True)
    assert (cov == 0).all() and (out == 0).all()
    out, cov = O.forward_warp(src, w, h, 0, const_flow(w, h, [-3.0, 0.0]), w, h, 1.0, True, True)
    cols = np.arange(w)[None, :].repeat(h, 0)
    assert ((cov.reshape(h, w) != 0) == (cols <= 6)).all()


def test_early_outs_copy_the_source():
    w, h = 9, 7
    rng = np.random.RandomState(3)
    src = rng.randint(0, 256, w * h * 4).astype(np.uint8)
    out, cov = O.forward_warp(src, w, h, 0, const_flow(w, h, [0.0, 0.0]), w, h, 1.0, True, True)
    assert (out == src).all() and (cov == 255).all()
    flow = const_flow(w, h, [1.0, 0.5])
    for a in [0.0, 1e-6, -1e-6, 1e-5]:
        assert (O.forward_warp(src, w, h, 0, flow, w, h, np.float32(a)) == src).all()
    assert (O.forward_warp(src, w, h, 0, flow, w, h, np.float32(1.1e-5)) != src).any()
    assert (O.forward_warp(src, w, h, 0, const_flow(w, h, [1e-4, -1e-4]), w, h, 1.0) == src).all()
    assert (O.forward_warp(src, w, h, 0, const_flow(w, h, [1.0001e-4, 0.0]), w, h, 1.0) != src).any()
    f = const_flow(w, h, [0.0, 0.0])
    f[(6 * w + 8) * 2 + 1] = 0.5
    assert (O.forward_warp(src, w, h, 0, f, w, h, 1.0) != src).any()


def test_pyramid_level_counts():
    L = O.lib()
    for (w, h), n in [((2, 2), 1), ((3, 3), 1), ((4, 4), 2), ((8, 8), 3), ((16, 12), 3), ((5, 100), 2), ((3, 100), 1),
                      ((1920, 1080), 10)]:
        assert L.or_fw_level_count(w, h) == n


def test_mip_level_closed_forms():
    w, h = 16, 12
    L = O.lib()
    xs = np.arange(w, dtype=np.float32)
    flow = np.zeros((h, w, 2), np.float32)
    flow[:, :, 0] = np.float32(-0.5) * xs[None, :]
    m = (4.0 * np.sqrt(1.25) * np.sqrt(0.5) + 2.0 + 1.0) / 8.0
    want = -np.log2(m)
    for c, r in [(5, 5), (3, 7), (10, 2)]:
        assert abs(L.or_fw_mip_level(w, h, O.ptr(flow), w, h, 1.0, c, r) - want) < 2e-6
    t = const_flow(w, h, [2.0, 1.0])
    for c, r in [(0, 0), (5, 5), (15, 11), (0, 11)]:
        assert abs(L.or_fw_mip_level(w, h, O.ptr(t), w, h, 1.0, c, r)) < 3e-7
    e = np.zeros((h, w, 2), np.float32)
    e[:, :, 0] = xs[None, :]
    e[:, :, 1] = np.arange(h, dtype=np.float32)[:, None]
    assert abs(L.or_fw_mip_level(w, h, O.ptr(e), w, h, 1.0, 5, 5) + 1.0) < 1e-6


def test_right_triangle_scan_conversion_by_hand():
    hits = O.fw_triangle([[0, 0, 0, 0, 0], [4, 0, 1, 0, 0], [0, 4, 0, 1, 0]], 7, 7)
    counts = np.bincount(hits[:, 1].astype(int), minlength=8)
    assert list(counts) == [5, 4, 3, 2, 0, 0, 0, 0]
    row1 = hits[hits[:, 1] == 1]
    assert list(row1[:, 0]) == [0, 1, 2, 3]
    assert np.abs(row1[:, 2] - 0.25 * row1[:, 0]).max() < 1e-6 and np.abs(row1[:, 3] - 0.25).max() < 1e-6


def test_degenerate_last_row_pass():
    hits = O.fw_triangle([[4.0, 0.0, 0.5, 0, 0], [3.2, 7.0, 0, 1, 0], [5.9, 7.0, 1, 1, 0]], 9, 7)
    last = hits[hits[:, 1] == 7]
    assert list(last[:, 0]) == [4, 5]
    assert abs(last[0, 2] - 0.8 / 2.7) < 1e-5
    assert (hits[:, 1] < 7).any()
    hits = O.fw_triangle([[4.0, 0.0, 0.5, 0, 0], [3.2, 6.9, 0, 1, 0], [5.9, 6.9, 1, 1, 0]], 9, 7)
    assert (hits[:, 1] <= 6).all()
    assert O.fw_triangle([[4.0, 0.0, 0.5, 0, 0], [9.2, 7.0, 0, 1, 0], [9.6, 7.0, 1, 1, 0]], 7, 7) is None


def test_rejected_and_clipped_triangles():
    assert len(O.fw_triangle([[-3, 0, 0, 0, 0], [-1, 4, 0, 0, 0], [-2, 6, 0, 0, 0]], 7, 7)) == 0
    assert len(O.fw_triangle([[1, 8, 0, 0, 0], [3, 9, 0, 0, 0], [2, 12, 0, 0, 0]], 7, 7)) == 0
    hits = O.fw_triangle([[-20, -20, 0, 0, 0], [40, -10, 1, 0, 0], [5, 50, 0, 1, 0]], 7, 7)
    assert len(hits) == 64 and (hits[:, :2] <= 7).all()


def test_gouraud_variant_interpolates_the_vertex_colours():
    w, h = 16, 12
    src = np.zeros((h, w, 4), np.uint8)
    src[:, :, 0] = 255
    src[6, 7] = 255
    src = src.reshape(-1)
    flow = const_flow(w, h, [1.0, 1.0])
    out, cov = O.forward_warp(src, w, h, 0, flow, w, h, 0.5, False, True)
    red = out.reshape(h, w, 4)[:, :, 1]
    want = np.zeros((h, w), np.uint8)
    want[6, 8] = want[7, 7] = 127
    assert (red == want).all()
    assert cov[0] == 0
    tex = O.forward_warp(src, w, h, 0, flow, w, h, 0.5, True).reshape(h, w, 4)[:, :, 1]
    for x, y in [(7, 6), (8, 6), (7, 7), (8, 7)]:
        assert tex[y, x] == 64
    assert (O.forward_warp(src, w, h, 0, const_flow(w, h, [0.0, 0.0]), w, h, 1.0, False) == src).all()


def test_shape_errors():
    src = np.zeros(6 * 6 * 4, np.uint8)
    with pytest.raises(ValueError):
        O.forward_warp(np.zeros(1 * 6 * 4, np.uint8), 1, 6, 0, const_flow(6, 6, [1, 0]), 6, 6, 1.0)
    with pytest.raises(ValueError):
        O.forward_warp(src, 6, 6, 0, const_flow(1, 6, [1, 0]), 1, 6, 1.0)
