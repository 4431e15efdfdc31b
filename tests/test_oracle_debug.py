"""The Debug views of Create Vectors (debug.rs) in the oracle, pinned to the values of the original
plugin's view generator that the reference's tests record (plugins/retime-engine/src/debug/tests.rs:
Diff, luma, Detail, Edge, overlay and Blend pixels, the traced rows of its special value clip) and
to the reference's numpy model of the Warp view (tests/fixtures/debug_cases.hex). CPU only."""
import numpy as np
import pytest

import golden_data as G
import oracle_lib as O

T = G.debug_tables()
F32 = lambda bits: np.array(bits, np.uint32).view(np.float32)


def px(fmt, vals):
    return np.array(vals, {0: np.uint8, 1: np.uint16}[fmt]) if fmt != 2 else F32(vals)


@pytest.mark.parametrize("fmt,name", [(0, "DIFF8"), (1, "DIFF16"), (2, "DIFF32")])
def test_diff(fmt, name):
    for a, b, want in T[name]:
        out = O.debug_views_of(px(fmt, a), px(fmt, b), 1, 1, fmt, 1)
        white = {0: 255, 1: 65535}.get(fmt, 0x3F800000)
        got = out.view(np.uint32).tolist() if fmt == 2 else out.tolist()
        assert got == [white, want, want, want], (a, b)


@pytest.mark.parametrize("fmt,name", [(0, "LUMA8"), (1, "LUMA16"), (2, "LUMA32")])
def test_luma(fmt, name):
    white = {0: 255, 1: 65535}.get(fmt, 0x3F800000)
    for rgb, want in T[name]:
        l = O.debug_luma(px(fmt, [white] + list(rgb)), 1, 1, fmt)
        assert int(l.view(np.uint32)[0]) == want, rgb


def test_detail_and_edge():
    for patch, want in T["DETAIL"]:
        assert int(O.debug_detail(F32(patch), 3, 3).view(np.uint32)[4]) == want
    for patch, want in T["EDGE"]:
        e = O.debug_edge(F32(patch), 3, 3)[4]
        assert e == np.float32(2.0) * F32([want])[0]


@pytest.mark.parametrize("fmt,name", [(0, "OVERLAY8"), (1, "OVERLAY16"), (2, "OVERLAY32")])
def test_overlay(fmt, name):
    for r, g, want in T[name]:
        out = O.debug_overlay(F32([r]), F32([g]), 1, 1, fmt)
        got = out.view(np.uint32).tolist() if fmt == 2 else out.tolist()
        assert got == list(want)


@pytest.mark.parametrize("fmt,name", [(0, "BLEND8"), (1, "BLEND16"), (2, "BLEND32")])
def test_blend(fmt, name):
    for a, b, want in T[name]:
        out = O.debug_views_of(px(fmt, a), px(fmt, b), 1, 1, fmt, 0)
        got = out.view(np.uint32).tolist() if fmt == 2 else out.tolist()
        assert got == list(want)


def test_traced_special_value_rows():
    """W' = (Y OVER transparent) with W OVER it, and its Blend, on two traced rows of NaNs,
    infinities and denormals; the float luma of those W' rows."""
    for row in range(2):
        y, wimg = F32(T["SPEC_Y"][row]).reshape(-1), F32(T["SPEC_W"][row]).reshape(-1)
        wp = O.debug_compose_over(wimg, y, 6, 1, 2)
        assert wp.view(np.uint32).tolist() == np.array(T["SPEC_WP"][row], np.uint32).reshape(-1).tolist(), row
        bl = O.debug_views_of(wp, y, 6, 1, 2, 0)
        assert bl.view(np.uint32).tolist() == np.array(T["SPEC_BLEND"][row], np.uint32).reshape(-1).tolist(), row
        lum = O.debug_luma(wp, 6, 1, 2)
        assert lum.view(np.uint32).tolist() == T["SPEC_WP_LUMA"][row], row


CASES = G.debug_cases()


@pytest.mark.parametrize("c", [c for c in CASES if c["code"] == 4],
                         ids=[f"f{c['fmt']}-{c['w']}x{c['h']}" for c in CASES if c["code"] == 4])
def test_warp_view_model(c):
    """The Warp view of the reference's numpy model: the textured forward warp at amount 1."""
    got = O.debug_view(c["x"], c["y"], c["w"], c["h"], c["fmt"], c["flow"], c["fw"], c["fh"], 4, gouraud=False)
    assert got.view(np.uint8).tobytes() == c["want"].view(np.uint8).tobytes()


def test_views_are_their_primitives():
    """Every view of a case is views_of over the compose of its Warp view (debug.rs:125-171)."""
    for c in CASES[:10]:
        w, h, fmt = c["w"], c["h"], c["fmt"]
        warp = O.debug_view(c["x"], c["y"], w, h, fmt, c["flow"], c["fw"], c["fh"], 4)
        wp = O.debug_compose_over(warp, c["y"], w, h, fmt)
        for code in range(4):
            want = O.debug_views_of(wp, c["y"], w, h, fmt, code)
            got = O.debug_view(c["x"], c["y"], w, h, fmt, c["flow"], c["fw"], c["fh"], code)
            assert got.view(np.uint8).tobytes() == want.view(np.uint8).tobytes()
