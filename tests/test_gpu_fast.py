"""The fast mode: the solver's kernels built with FMA contraction, approximate division and flushed
denormals (tw_flow_settings.fast_mode). It is not bit identical to the CPU path; these tests state
how far it is from a double precision restatement of the same solver (oracle/liboracle64.so), in
pixels of flow and in PSNR of the composed frame, next to the strict path's own distance.

Both modes are also checked against the reference's differential fixtures of the solver
(plugins/retime-engine/tests/fixtures/flow_{a..f}.hex: its float32 numpy model without block
matching), with the reference's tolerances for the strict mode (tests/flow_d.rs:231-236).
"""
import numpy as np
import pytest

import golden_data
import oracle_lib as O
import twixtor_b200 as tw
from twixtor_b200 import synth

pytestmark = pytest.mark.gpu

MODELS = golden_data.flow_models()
FAST_MODEL_SCALE = 10.0    # the fast mode's tolerance against the models: ten times the reference's
FAST_MAX_FLOW_PX = 0.5     # the fast mode's flow against FP64: the largest deviation, pixels
FAST_MEAN_FLOW_PX = 2e-3   # and the mean deviation
FAST_MIN_PSNR_DB = 45.0    # the frame composed with the fast flows against the one with the FP64 flows


@pytest.fixture(scope="module")
def dev():
    tw.build()
    d = tw.Device(0)
    yield d
    d.close()


def _settings(c, fast):
    return tw.FlowSettings(quality=c["quality"], hiq=True, sensitivity=c["sens"], skip_refine=True,
                           prep_contrast_edge=c["prep"] == 1, prep_delinearize=c["prep"] == 2, fast_mode=fast)


@pytest.mark.parametrize("c", MODELS, ids=[c["name"] for c in MODELS])
def test_solve_against_the_reference_model(dev, c):
    w, h = c["w"], c["h"]
    strict, _ = dev.solve(c["x"], c["y"], w, h, 0, _settings(c, False))
    fast, _ = dev.solve(c["x"], c["y"], w, h, 0, _settings(c, True))
    ds = np.abs(strict.astype(np.float64) - c["flow"]).max()
    df = np.abs(fast.astype(np.float64) - c["flow"]).max()
    print(f"flow_{c['name']}: strict {ds:.2e}, fast {df:.2e} (reference tolerance {c['tol']:.0e})")
    assert ds < c["tol"], f"strict {ds}"
    assert df < c["tol"] * FAST_MODEL_SCALE, f"fast {df}"


def _psnr(a, b):
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse)


@pytest.mark.parametrize("size", [(160, 96), (1920, 1080)])
def test_fast_mode_against_fp64(dev, size):
    """solve_pair at the retime workload's settings on a synthetic pair (background and square
    moving), strict and fast, against the FP64 solve; then each pair of flows composed (Blend, at
    0.4) into the in-between frame and compared with the frame of the FP64 flows."""
    w, h = size
    kw = dict(seed=0x74570002, bg_velocity=(6.0, -3.0), square=240, square_start=(600.0, 400.0),
              square_velocity=(9.0, 4.0)) if w == 1920 else dict(seed=0x74570001)
    frames = synth.moving_clip(w, h, 2, depth=8, **kw)
    n = w * h * 4
    a, b = O.from_frame(frames[:n], w, h, 0), O.from_frame(frames[n:], w, h, 0)
    s_ab, s_ba, (fw, fh) = dev.solve_pair(a, b, w, h, 0, tw.FlowSettings())
    f_ab, f_ba, _ = dev.solve_pair(a, b, w, h, 0, tw.FlowSettings(fast_mode=True))
    r_ab, r_ba, _ = O.solve_pair64(a, b, w, h, 0)
    o_ab, o_ba, _ = O.solve_pair(a, b, w, h, 0)
    assert s_ab.tobytes() == o_ab.tobytes() and s_ba.tobytes() == o_ba.tobytes()  # strict is the CPU path
    ef = np.abs(np.concatenate([f_ab, f_ba]).astype(np.float64) - np.concatenate([r_ab, r_ba]))
    es = np.abs(np.concatenate([s_ab, s_ba]).astype(np.float64) - np.concatenate([r_ab, r_ba]))
    wa = np.float32(0.6)  # the frame 40 % of the way from A to B
    ref = O.compose_vectors(a, b, w, h, 0, r_ab.astype(np.float32), r_ba.astype(np.float32), fw, fh, wa)
    fast_frame = O.compose_vectors(a, b, w, h, 0, f_ab, f_ba, fw, fh, wa)
    strict_frame = O.compose_vectors(a, b, w, h, 0, s_ab, s_ba, fw, fh, wa)
    pf, ps = _psnr(fast_frame, ref), _psnr(strict_frame, ref)
    print(f"{w}x{h}: flow vs FP64, fast max {ef.max():.3e} px mean {ef.mean():.3e} px; strict max {es.max():.3e} "
          f"mean {es.mean():.3e}; frame PSNR vs FP64 flows: fast {pf:.1f} dB, strict {ps:.1f} dB")
    assert ef.max() < FAST_MAX_FLOW_PX, ef.max()
    assert ef.mean() < FAST_MEAN_FLOW_PX, ef.mean()
    assert pf > FAST_MIN_PSNR_DB, pf


def test_fast_mode_clip_through_the_lanes(dev):
    """The fast mode through the clip call (the flag travels in the retime settings): every frame
    close to the strict render."""
    w, h, nf = 160, 96, 8
    frames = synth.moving_clip(w, h, nf, depth=8)
    tp = tw.TimeParams(speed_percent=50.0)
    sels = [tw.select(tp, k, w, h) for k in range(12)]
    strict = dev.retime_clip(tw.RetimeSettings(), frames, nf, sels, w, h, 0)
    fast = dev.retime_clip(tw.RetimeSettings(flow=tw.FlowSettings(fast_mode=True)), frames, nf, sels, w, h, 0)
    p = _psnr(fast, strict)
    print(f"fast clip against strict clip: {p:.1f} dB")
    assert p > FAST_MIN_PSNR_DB
