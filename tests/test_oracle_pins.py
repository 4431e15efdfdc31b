"""Pins the CPU oracle before any CUDA result is compared with it.

* the Gaussian and binomial kernel tables of the reference (flow/conv.rs tests, bit patterns);
* the hand values of the reference's solver unit tests (flow.rs:1355-1565);
* the reference's bit-exact numpy model fixtures of the inverse warp (tests/fixtures/warp_cases.hex);
* end to end: the sha256 of every served case of the reference's parity grid
  parity/retime-flow/results/base.grid.tsv (whole output clips of the `retime` effect: frame
  selection, pyramids, both solves with block matching, warps, blend, boundary conversions);
* the motion blur of Blur Compensation against the reference's numpy model fixtures
  (tests/fixtures/blur_cases.hex), bit for bit;
* the Delinearize powf against the 72 arguments the reference traced from the plugin's C runtime
  (crt_powf.rs tests) and its fall back cases;
* the same for the layered path with plates: every served case of parity/fgbg-layers/results/base.tsv
  (retime-fgbg with 1 to 3 FG matte layers, recorded at the reference's current revision: rows
  reversed, taps above first).
"""
import ctypes
import hashlib

import numpy as np
import pytest

import golden_data
import oracle_lib as O


def bits(a):
    return [int(x) for x in np.asarray(a, np.float32).view(np.uint32)]


@pytest.mark.parametrize("r,table", [
    (7.0, [0x3e4e2a9a, 0x3e35855c, 0x3df7ca22, 0x3d831b79, 0x3cd71a9b, 0x3c08ca7a, 0x3b06de99, 0x39ce2a9a]),
    (5.0, [0x3e904ee6, 0x3e60e131, 0x3dd4bfc6, 0x3cf46273, 0x3baa6d48, 0x3a104ee6]),
    (2.0, [0x3f33bb04, 0x3e172281, 0x3ab3bb0c]),
])
def test_gaussian_kernel_tables(r, table):
    k = np.zeros(16, np.float32)
    n = O.lib().or_gaussian_kernel(r, O.ptr(k), 16)
    assert bits(k[:n]) == table


@pytest.mark.parametrize("sens,levels,start,damp", [
    (1.0, 8, 7, 1.0), (2.0, 8, 7, 1.0), (0.0, 8, 0, 0.0), (0.1, 3, 0, 0.0), (0.5, 8, 6, 0.0)])
def test_start_level_table(sens, levels, start, damp):
    s, d = ctypes.c_int(), ctypes.c_float()
    O.lib().or_start_level(sens, levels, ctypes.byref(s), ctypes.byref(d))
    assert (s.value, d.value) == (start, damp)


def test_start_level_default_sensitivity():
    s, d = ctypes.c_int(), ctypes.c_float()
    O.lib().or_start_level(0.7, 8, ctypes.byref(s), ctypes.byref(d))
    assert s.value == 6 and abs(d.value - 0.9709) < 1e-4


def cost(b, w, h, p, x2, y2):
    some = ctypes.c_int()
    c = O.lib().or_block_cost(O.ptr(np.asarray(b, np.float32)), w, h, O.ptr(np.asarray(p, np.float32)), x2, y2,
                              ctypes.byref(some))
    return c if some.value else None


def test_block_cost_golden_values():
    zeros = np.zeros(64, np.float32)
    p = np.arange(1, 10, dtype=np.float32)
    assert cost(zeros, 8, 8, p, 3.0, 3.0) == 285.0
    assert cost(zeros, 8, 8, p, 0.5, 3.0) is None
    assert cost(zeros, 8, 8, p, 3.0, 0.0) is None
    assert cost(zeros, 8, 8, p, 6.01, 3.0) is None
    assert cost(zeros, 8, 8, p, 6.0, 6.0) is not None
    p = np.ones(9, np.float32)
    p[8] = 4096.0
    assert cost(zeros, 8, 8, p, 3.0, 3.0) == 16777224.0
    b = np.array([[x + 10.0 * y for x in range(8)] for y in range(8)], np.float32)
    p = np.array([(2.5 + aa) + 10 * (3.25 + bb) for bb in (-1, 0, 1) for aa in (-1, 0, 1)], np.float32)
    assert cost(b, 8, 8, p, 2.5, 3.25) == 0.0
    p[4] += 2.0
    assert cost(b, 8, 8, p, 2.5, 3.25) == 4.0


def test_block_matching_replaces_a_bad_vector_and_spares_the_border():
    w, h = 12, 10
    img = np.array([[((x * 7 + y * 13) % 17) * 3.0 + x * 0.5 for x in range(w)] for y in range(h)], np.float32)
    flow = np.zeros(w * h * 2, np.float32)
    c = (5 * w + 6) * 2
    flow[c], flow[c + 1] = 2.0, 1.0
    for x in range(w):
        flow[x * 2] = 0.25
        flow[((h - 1) * w + x) * 2] = 0.25
    O.lib().or_block_match(O.ptr(img), O.ptr(img), O.ptr(flow), w, h)
    assert (flow[c], flow[c + 1]) == (0.0, 0.0)
    for x in range(w):
        assert flow[x * 2] == 0.25 and flow[((h - 1) * w + x) * 2] == 0.25


def test_new_displacement_and_threshold():
    L = O.lib()
    f = np.array([1.0, 2.0], np.float32)
    L.or_new_disp(O.ptr(f), O.ptr(np.array([100, 0, 100], np.float32)), O.ptr(np.array([50, -20], np.float32)), 1)
    assert list(f) == [1.5, 1.8] or bits(f) == bits([1.5, 1.8])
    f = np.array([1.0, 2.0], np.float32)
    L.or_new_disp(O.ptr(f), O.ptr(np.array([6, 0, 6.5], np.float32)), O.ptr(np.array([50, -20], np.float32)), 1)
    assert list(f) == [1.0, 2.0]
    f = np.zeros(2, np.float32)
    L.or_new_disp(O.ptr(f), O.ptr(np.array([8, 3, 8], np.float32)), O.ptr(np.array([1, 1], np.float32)), 1)
    e = np.float32(np.float32(3.0 * 1.0 - 8.0 * 1.0) / np.float32(-55.0))
    assert f[0] == e and f[1] == e


def test_flow_upsampling_scales_by_the_size_ratio():
    L = O.lib()
    src = np.array([1.0, 2.0] * 4, np.float32)
    d = np.zeros(18, np.float32)
    L.or_upsample_flow(O.ptr(src), 2, 2, 3, 3, O.ptr(d))
    assert (d[0::2] == 2.0).all() and (d[1::2] == 4.0).all()
    src = np.array([0, 0, 2, 0, 4, 0] * 2, np.float32)
    d = np.zeros(20, np.float32)
    L.or_upsample_flow(O.ptr(src), 3, 2, 5, 2, O.ptr(d))
    assert list(d[0:10:2]) == [0.0, 2.0, 4.0, 6.0, 8.0]


def test_gradient_of_ramps():
    w, h = 6, 5
    img = np.array([[3.0 * x + 5.0 * y for x in range(w)] for y in range(h)], np.float32)
    g = np.zeros(w * h * 2, np.float32)
    O.lib().or_calc_grad(O.ptr(img), w, h, O.ptr(g))
    assert (g[0::2] == 3.0).all() and (g[1::2] == 5.0).all()


def test_range_check():
    L = O.lib()
    out = np.array([10.0, 10.0] * 16, np.float32)
    assert L.or_all_out_of_range(O.ptr(out), 4, 4) == 1
    ok = out.copy()
    ok[10] = -1.0
    assert L.or_all_out_of_range(O.ptr(ok), 4, 4) == 1
    ok[0] = ok[1] = 0.0
    assert L.or_all_out_of_range(O.ptr(ok), 4, 4) == 0


def test_quality_to_resolution_table():
    for q, hiq, r, w0, h0 in [(1, True, 3, 240, 135), (2, True, 3, 240, 135), (3, True, 2, 480, 270),
                              (4, True, 1, 960, 540), (5, True, 0, 1920, 1080), (4, False, 2, 480, 270),
                              (3, False, 3, 240, 135), (5, False, 1, 960, 540), (1, False, 3, 240, 135)]:
        red, sizes = O.geometry(q, hiq, 1920, 1080)
        assert (red, sizes[0]) == (r, (w0, h0))
    red, sizes = O.geometry(4, True, 1920, 1080)
    assert sizes == [(960, 540), (480, 270), (240, 135), (120, 67), (60, 33), (30, 16), (15, 8), (7, 4)]


WARP = golden_data.warp_cases()


@pytest.mark.parametrize("i", range(len(WARP)))
def test_inverse_warp_model_fixtures(i):
    """Every case of warp_cases.hex, the 360 ones (wrap, pole reflection, the 360 sampler) included."""
    c = WARP[i]
    r = O.inv_warp(c["src"], c["w"], c["h"], c["fmt"], c["flow"], c["fw"], c["fh"], c["amount"], hold=c["hold"],
                   coverage=c["want_cov"], is360=c["is360"])
    out, cov = r if c["want_cov"] else (r, None)
    assert out.view(np.uint8).tobytes() == c["out"].view(np.uint8).tobytes()
    if c["want_cov"]:
        assert (cov == c["cov"]).all()


CASES, INPUTS = golden_data.grid()


@pytest.mark.parametrize("case", golden_data.grid_params(CASES))
def test_retime_flow_grid_sha256(case):
    fmt = golden_data.FMT_OF_DEPTH[case["depth"]]
    raw = INPUTS[case["input"]].view(O.DTYPE[fmt])
    p = O.retime_params(**golden_data.case_params(case))
    out = O.retime_clip(raw, case["frames"], case["width"], case["height"], fmt, p, case["frames"])
    assert hashlib.sha256(out.tobytes()).hexdigest() == case["sha256"]


F1 = golden_data.f1_cases()


@pytest.mark.parametrize("i", range(len(F1)))
def test_smart_blend_and_hole_fill_model_fixtures(i):
    """The reference's numpy models of Smart Blend (kind 1), its binary alpha variant (kind 2) and the
    hole fill (kind 3, engine tap order: below first) reproduced bit for bit."""
    c = F1[i]
    if c["kind"] in (1, 2):
        out = np.zeros_like(c["p1"])
        O.lib().or_smart_blend(O.ptr(out), O.ptr(c["p1"]), O.ptr(c["p2"]), c["w"], c["h"], c["fmt"], c["weight"],
                               int(c["kind"] == 2))
    else:
        out = c["p1"].copy()
        rc = O.lib().or_fill_holes(O.ptr(out), c["w"], c["h"], c["fmt"], O.ptr(c["mask"]), c["mask_kind"], 0)
        assert rc == 0, O.err()
    assert out.view(np.uint8).tobytes() == c["out"].view(np.uint8).tobytes()


CV_CASES, CV_INPUTS = golden_data.cv_grid()


@pytest.mark.parametrize("case", golden_data.cv_grid_params(CV_CASES))
def test_create_vectors_grid_sha256(case):
    """The reference's recorded output clips of the served create-vectors grid cases (solve + encode,
    frame pairs, blank neighbours outside the clip, tiny frames, the Debug display with the textured
    warp of the recorded revision)."""
    fmt = golden_data.FMT_OF_DEPTH[case["depth"]]
    raw = CV_INPUTS[case["input"]].view(O.DTYPE[fmt])
    kw = golden_data.cv_case_params(case)
    points = [golden_data.cv_points(case, n) for n in range(case["frames"])]
    out = O.create_vectors_clip(raw, case["frames"], case["width"], case["height"], fmt, case["frames"],
                                rows_reversed=False, taps_above_first=False, points=points, debug_textured=True, **kw)
    assert hashlib.sha256(out.tobytes()).hexdigest() == case["sha256"]


FG_CASES, FG_INPUTS = golden_data.fgbg_grid()


@pytest.mark.parametrize("case", FG_CASES, ids=[c["id"] for c in FG_CASES])
def test_fgbg_layers_grid_sha256(case):
    """The reference's recorded output clips of the served retime-fgbg grid cases: matte channels,
    raw and composition planes (with the inverse matte shrink), layer images, masked solves per
    layer, plates, refill, OVER, the single group displays."""
    fmt = golden_data.FMT_OF_DEPTH[case["depth"]]
    w, h, n = case["width"], case["height"], case["frames"]
    kw = golden_data.fgbg_case_params(case)
    chans, sens = kw.pop("chans"), kw.pop("fg_sens")
    shrinks, display = kw.pop("shrinks"), kw.pop("display")
    p = O.retime_params(rows_reversed=True, taps_above_first=True, **kw)
    mattes = [FG_INPUTS[m].view(O.DTYPE[fmt]) for m in case["mattes"]]
    nfg = len(mattes)

    def points(k):
        a = O.select(p, k, w, h)["a"]
        return golden_data.fgbg_points(case, a, a + 1, nfg)
    out = O.retime_fgbg_clip(FG_INPUTS[case["input"]].view(O.DTYPE[fmt]), n, mattes, chans, sens, w, h, fmt, p, n,
                             shrinks=shrinks, display=display, points=points)
    assert hashlib.sha256(out.tobytes()).hexdigest() == case["sha256"]


def test_crt_powf_traced_vectors():
    """The plugin runtime's powf of the Delinearize step, bit for bit on every traced argument."""
    v = np.array(golden_data.crt_powf_traced(), np.uint32)
    got = O.crt_powf(v[:, 0].view(np.float32), v[:, 1].view(np.float32))
    assert (got.view(np.uint32) == v[:, 2]).all()


def test_crt_powf_fall_back_cases():
    """crt_powf.rs:229-232: outside the table path, the double precision pow narrowed to float."""
    f = lambda x, y: float(O.crt_powf([x], [y])[0])  # noqa: E731
    assert f(0.0, 0.5) == 0.0 and f(1.0, 0.45454544) == 1.0 and f(0.25, 1.0) == 0.25 and f(0.5, 0.0) == 1.0
    assert np.isnan(f(-1.0, 0.5)) and np.isnan(f(np.nan, 2.0))
    assert f(np.inf, 2.0) == np.inf and f(2.0, 200.0) == np.inf
    y = np.float32(1.0) / np.float32(2.2)
    x = (np.arange(1, 2000, dtype=np.float32) / np.float32(997.0)).astype(np.float32)
    got = O.crt_powf(x, y).astype(np.float64)
    want = np.power(x.astype(np.float64), np.float64(y))
    assert (np.abs((got - want) / want) < 2.0e-7).all()


BLUR = golden_data.blur_cases()


@pytest.mark.parametrize("i", range(len(BLUR)))
def test_motion_blur_model_fixtures(i):
    """warp/blurcomp.rs motion_blur: bilinear and nearest taps, shutter offsets, every depth."""
    c = BLUR[i]
    out = O.motion_blur(c["src"], c["w"], c["h"], c["fmt"], c["flow"], c["fw"], c["fh"], c["amount"], c["hiq"],
                        c["shutter"])
    assert out.view(np.uint8).tobytes() == c["out"].view(np.uint8).tobytes()


@pytest.mark.parametrize("c", golden_data.flow_models(), ids=lambda c: c["name"])
def test_oracle_solve_matches_the_reference_solver_models(c):
    """The reference's differential fixtures of the solver (its float32 numpy model, no block
    matching; tests/flow_d.rs:224-242): the oracle's solve X -> Y within the reference's own
    tolerances, and the double precision build of the oracle within them too."""
    prep = {0: 1, 1: 2, 2: 3}[c["prep"]]
    kw = dict(quality=c["quality"], hiq=True, sensitivity=c["sens"], skip_refine=True, prep=prep)
    f, _ = O.solve(c["x"], c["y"], c["w"], c["h"], 0, **kw)
    f64, _ = O.solve64(c["x"], c["y"], c["w"], c["h"], 0, **kw)
    assert np.abs(f.astype(np.float64) - c["flow"]).max() < c["tol"]
    assert np.abs(f64 - c["flow"]).max() < c["tol"]
