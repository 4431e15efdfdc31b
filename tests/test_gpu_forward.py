"""Parity of the CUDA forward warp (tw_forward_warp) with the oracle, bit for bit.

Covers the textured and the Gouraud variants at the three depths, the reference's f2 model
fixtures, the early outs, folds and collapses of the mesh (long per-pixel hit lists: the shared
memory and the global merge paths of the resolve), NaN and infinite samples, the refusal of the
degenerate last-row pass, and the device's logf against the host C library's.
"""
import numpy as np
import pytest

import golden_data
import oracle_lib as O
import twixtor_b200 as tw

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    tw.build()
    d = tw.Device(0)
    yield d
    d.close()


def same(a, b):
    return np.asarray(a).view(np.uint8).tobytes() == np.asarray(b).view(np.uint8).tobytes()


def rand_img(rng, w, h, fmt):
    if fmt == 0:
        return rng.randint(0, 256, w * h * 4).astype(np.uint8)
    if fmt == 1:
        return rng.randint(0, 65536, w * h * 4).astype(np.uint16)
    return rng.random_sample(w * h * 4).astype(np.float32)


def smooth_flow(rng, fw, fh, amp, bumps=4):
    ys, xs = np.mgrid[0:fh, 0:fw].astype(np.float64)
    f = np.zeros((fh, fw, 2))
    for _ in range(bumps):
        cx, cy = rng.uniform(0, fw), rng.uniform(0, fh)
        s = rng.uniform(0.15, 0.4) * max(fw, fh)
        g = np.exp(-((xs - cx) ** 2 + (ys - cy) ** 2) / (2 * s * s))
        f[:, :, 0] += rng.uniform(-amp, amp) * g
        f[:, :, 1] += rng.uniform(-amp, amp) * g
    return f.astype(np.float32).reshape(-1)


def check(dev, src, w, h, fmt, flow, fw, fh, amount, pyramid):
    got, gcov = dev.forward_warp(src, w, h, fmt, flow, (fw, fh), amount, pyramid, coverage=True)
    want, wcov = O.forward_warp(src, w, h, fmt, flow, fw, fh, amount, pyramid, True)
    assert (gcov == wcov).all()
    assert same(got, want)


def test_logf_matches_the_host_c_library(dev):
    rng = np.random.RandomState(1)
    bits = rng.randint(1, 0x7f800000, 8_000_000, dtype=np.int64).astype(np.uint32)
    extra = np.array([0, 0x80000000, 0x7f800000, 0xff800000, 0x7fc00000, 0x7fc01234, 0xffc00000, 0x7f800001,
                      0xbf800000, 0x80000001, 0x00000001, 0x007fffff, 0x00800000, 0x3f800000, 0x3f800001, 0x3f7fffff,
                      0x40000000, 0x7f7fffff], np.uint32)
    x = np.concatenate([bits, extra, np.arange(0x3f700000, 0x3f900000, dtype=np.uint32)]).view(np.float32)
    got = dev.check_logf(x)
    want = np.zeros_like(x)
    O.lib().or_logf(O.ptr(x), O.ptr(want), x.size)
    assert same(got, want)


F2 = golden_data.f2_cases()


@pytest.mark.parametrize("i", range(len(F2)))
def test_textured_forward_warp_model_fixtures(dev, i):
    c = F2[i]
    got, cov = dev.forward_warp(c["src"], c["w"], c["h"], c["fmt"], c["flow"], (c["fw"], c["fh"]), c["amount"], True, True)
    assert (cov == c["cov"]).all()
    if c["fmt"] == 2:
        assert np.abs(got - c["out"]).max() <= 2e-6
    else:
        assert (got == c["out"]).all()
    want = O.forward_warp(c["src"], c["w"], c["h"], c["fmt"], c["flow"], c["fw"], c["fh"], c["amount"], True)
    assert same(got, want)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("pyramid", [True, False])
@pytest.mark.parametrize("size,fsize,amp,amount", [((64, 48), (64, 48), 6.0, 1.0), ((97, 61), (49, 31), 12.0, 0.7),
                                                   ((160, 96), (80, 48), 25.0, -0.6), ((33, 130), (33, 130), 40.0, 1.3),
                                                   ((256, 200), (128, 100), 4.0, 0.5)])
def test_random_smooth_flows(dev, fmt, pyramid, size, fsize, amp, amount):
    (w, h), (fw, fh) = size, fsize
    rng = np.random.RandomState(w * 131 + h + fmt)
    check(dev, rand_img(rng, w, h, fmt), w, h, fmt, smooth_flow(rng, fw, fh, amp), fw, fh, amount, pyramid)


@pytest.mark.parametrize("fmt", [0, 2])
@pytest.mark.parametrize("pyramid", [True, False])
def test_folding_noise_flows(dev, fmt, pyramid):
    """Uncorrelated vectors: triangles flip, overlap and stack many hits on a pixel."""
    w, h = 80, 60
    rng = np.random.RandomState(7 + fmt)
    flow = rng.uniform(-9, 9, w * h * 2).astype(np.float32)
    check(dev, rand_img(rng, w, h, fmt), w, h, fmt, flow, w, h, 1.0, pyramid)


@pytest.mark.parametrize("pyramid", [True, False])
def test_contraction(dev, pyramid):
    """Every vertex pulled 90 % of the way to one point: small triangles crowd a few pixels."""
    w = h = 128
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float32)
    flow = np.stack([(64.3 - xs) * 0.9, (63.7 - ys) * 0.9], -1).astype(np.float32).reshape(-1)
    check(dev, rand_img(np.random.RandomState(11), w, h, 0), w, h, 0, flow, w, h, 1.0, pyramid)


@pytest.mark.parametrize("size", [40, 72])
def test_every_triangle_covers_half_the_image(dev, size):
    """Vertices thrown 1000 px out in a checkerboard of directions: each triangle covers about half
    the image, so every pixel collects about (w-1)(h-1) hits: above 4096 at 72x72 (the merge in
    global scratch), between 16 and 4096 at 40x40 (the shared memory sort)."""
    w = h = size
    rr, cc = np.mgrid[0:h, 0:w]
    tx = np.where(cc % 2 == 0, -1000.0, 1000.0) + w / 2
    ty = np.where(rr % 2 == 0, -1000.0, 1000.0) + h / 2
    flow = np.stack([tx - cc, ty - rr], -1).astype(np.float32).reshape(-1)
    check(dev, rand_img(np.random.RandomState(5), w, h, 0), w, h, 0, flow, w, h, 1.0, True)


def test_nan_and_infinite_samples(dev):
    w, h = 48, 40
    rng = np.random.RandomState(3)
    src = rand_img(rng, w, h, 2)
    src[rng.randint(0, src.size, 30)] = np.nan
    src.view(np.uint32)[rng.randint(0, src.size, 10)] = 0xffc0abcd
    src[rng.randint(0, src.size, 10)] = np.inf
    src[rng.randint(0, src.size, 10)] = -np.inf
    flow = smooth_flow(rng, w, h, 5.0)
    for pyramid in (True, False):
        check(dev, src, w, h, 2, flow, w, h, 0.8, pyramid)


def test_early_outs_and_errors(dev):
    w, h = 9, 7
    rng = np.random.RandomState(3)
    src = rand_img(rng, w, h, 0)
    out, cov = dev.forward_warp(src, w, h, 0, np.zeros(w * h * 2, np.float32), (w, h), 1.0, True, True)
    assert same(out, src) and (cov == 255).all()
    flow = np.tile(np.float32([1.0, 0.5]), w * h)
    for a in [0.0, 1e-6, -1e-6, 1e-5]:
        assert same(dev.forward_warp(src, w, h, 0, flow, (w, h), np.float32(a)), src)
    check(dev, src, w, h, 0, flow, w, h, np.float32(1.1e-5), True)
    with pytest.raises(tw.Mismatch):
        dev.forward_warp(src[:1 * h * 4], 1, h, 0, flow, (w, h), 1.0)


def test_degenerate_pass_outside_is_refused(dev):
    """Two vertices exactly on the last row (y = 6.9999 + 1e-4 in double = 7.0) at x = 7.2 and 7.6:
    the degenerate pass of their triangle would write x = 8 of an 8 pixel row, which the reference
    refuses (Unsupported)."""
    w = h = 8
    src = np.full(w * h * 4, 200, np.uint8)
    flow = np.zeros((h, w, 2), np.float32)
    flow[7, 1] = (6.2, -0.0001)
    flow[7, 2] = (5.6, -0.0001)
    flow = flow.reshape(-1)
    with pytest.raises(ValueError):
        O.forward_warp(src, w, h, 0, flow, w, h, 1.0, True)
    for pyramid in (True, False):
        with pytest.raises(tw.Unsupported):
            dev.forward_warp(src, w, h, 0, flow, (w, h), 1.0, pyramid)


def test_gouraud_impulse(dev):
    w, h = 16, 12
    src = np.zeros((h, w, 4), np.uint8)
    src[:, :, 0] = 255
    src[6, 7] = 255
    src = src.reshape(-1)
    flow = np.tile(np.float32([1.0, 1.0]), w * h)
    out = dev.forward_warp(src, w, h, 0, flow, (w, h), 0.5, False).reshape(h, w, 4)[:, :, 1]
    want = np.zeros((h, w), np.uint8)
    want[6, 8] = want[7, 7] = 127
    assert (out == want).all()
