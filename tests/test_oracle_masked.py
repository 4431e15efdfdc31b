"""Pins the masked solve of the layered paths in the CPU oracle (flow/extras.rs, flow.rs:737-845,
:1218-1245) against the reference's numpy models (tests/fixtures/mask_cases.hex): the binary mask
pyramid, the gradient masking, the B step with the warped mask test and the gated block matching
sweeps, bit for bit. The wrap-around (360) cases of the fixture are out of scope."""
import numpy as np
import pytest

import golden_data
import oracle_lib as O

M = [c for c in golden_data.mask_cases() if not c.get("wrap")]


def bits_equal(a, b):
    return (np.asarray(a, np.float32).view(np.uint32) == np.asarray(b, np.float32).view(np.uint32)).all()


@pytest.mark.parametrize("i", range(len(M)), ids=[f"kind{c['kind']}-{k}" for k, c in enumerate(M)])
def test_mask_model_fixtures(i):
    c = M[i]
    w, h = c["w"], c["h"]
    if c["kind"] == 1:
        lv = O.mask_pyramid(c["matte"], w, h, c["quality"], c["hiq"])
        assert [(a, b) for a, b, _ in lv] == [(a, b) for a, b, _ in c["levels"]]
        for (_, _, got), (_, _, want) in zip(lv, c["levels"]):
            assert bits_equal(got, want)
    elif c["kind"] == 2:
        g = np.zeros(w * h * 2, np.float32)
        O.lib().or_calc_grad(O.ptr(c["img"]), w, h, O.ptr(g))
        if c["mask"] is not None:
            O.lib().or_mask_gradient(O.ptr(g), O.ptr(c["mask"]), w, h)
        assert bits_equal(g, c["want"])
    elif c["kind"] == 3:
        b = np.zeros(w * h * 2, np.float32)
        O.lib().or_calc_b_masked(O.ptr(c["i1"]), O.ptr(c["i0"]), O.ptr(c["grad"]), O.ptr(c["flow"]), w, h,
                                 O.ptr(c["mask"]), O.ptr(b))
        assert bits_equal(b, c["want"])
    else:
        f = c["flow"].copy()
        O.lib().or_block_match_gated(O.ptr(c["a"]), O.ptr(c["b"]), O.ptr(f), w, h, O.ptr(c["gate"]))
        assert bits_equal(f, c["want"])


def test_unmasked_solve_is_the_plain_solve():
    """With no mask pyramids the layered driver is the plain one bit for bit (extras.rs:257-259)."""
    w, h = 64, 48
    rng = np.random.RandomState(4)
    ys, xs = np.mgrid[0:h, 0:w]
    base = (128 + 60 * np.sin(xs / 5.0) * np.cos(ys / 7.0)).astype(np.float32)
    a = np.zeros((h, w, 4), np.uint8)
    b = np.zeros((h, w, 4), np.uint8)
    a[..., 0] = b[..., 0] = 255
    a[..., 1:] = np.clip(base, 0, 255)[..., None].astype(np.uint8)
    b[..., 1:] = np.clip(np.roll(base, 2, axis=1), 0, 255)[..., None].astype(np.uint8)
    a, b = a.reshape(-1), b.reshape(-1)
    got, _ = O.solve_masked(a, b, w, h, 0)
    want, _, _ = O.solve_pair(a, b, w, h, 0)
    assert bits_equal(got, want)
