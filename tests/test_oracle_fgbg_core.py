"""retime-fgbg without FG matte layers, pinned to the reference's fgbg-core parity grid (CPU only).

The 371 served cases of parity/fgbg-core without 360 Video (the four warping codes with the
effect's Gouraud forward warps, every Motion Vectors quality, the three Frame Interp modes, its Image Prep (2 runs both prep
stages, 3 none: plugins/retime-fgbg/src/glue.rs:153-154), Main_BG sensitivity, Blur Compensation,
Track RGB+A, Speed and Frame Number modes, the input rate model with the effect's plain frame time,
Input: Fields, Src: Mark Segments, NTSC and decimal rates)
against the sha256 of the output clips results/base.tsv records. That table was recorded at the
reference's current code: the motion path on bottom-up rows, the taps above first.
"""
import hashlib

import pytest

import golden_data as G
import oracle_lib as O
import twixtor_b200 as tw

FGC_CASES, FGC_INPUTS = G.fgc_grid()


def test_grid_is_served():
    assert len(FGC_CASES) == 371


@pytest.mark.parametrize("c", FGC_CASES, ids=[c["id"] for c in FGC_CASES])
def test_fgbg_core_grid(c):
    w, h = c["width"], c["height"]
    fmt = G.FMT_OF_DEPTH[c["depth"]]
    p = O.retime_params(rows_reversed=True, taps_above_first=True, **G.fgc_case_params(c))
    out = O.retime_fgbg_clip(FGC_INPUTS[c["input"]], c["frames"], [], [], [], w, h, fmt, p, c["frames"])
    assert hashlib.sha256(out.tobytes()).hexdigest() == c["sha256"]


def test_library_selection_on_the_grid():
    """tw_select with retime-fgbg's plain frame time against the oracle, every output frame."""
    for c in FGC_CASES:
        w, h = c["width"], c["height"]
        kw = G.fgc_case_params(c)
        p = O.retime_params(**kw)
        tp = tw.TimeParams(fps=kw["fps"], speed_percent=kw["speed"], keys=kw["keys"], vectors=kw["vectors"],
                           frame_interp=kw["frame_interp"], blur_compensation=kw["blur"], remap_mode=kw["remap_mode"],
                           frame_num=kw["frame_num"], fn_keys=kw["fn_keys"], own_input_rate=kw["own_input_rate"],
                           input_frame_rate=kw["input_frame_rate"], frame_time_plain=True,
                           input_fields=kw["input_fields"], mark_segs=kw["mark_segs"], mark_keys=kw["mark_keys"])
        for n in range(c["frames"]):
            sel = tw.select(tp, n, w, h)
            want = O.select(p, n, w, h)
            assert (sel.a, sel.b) == O.clip_frames(p, n, w, h), (c["id"], n)
            assert (sel.exact, sel.vectors_quality, sel.interp) == (want["exact"], want["vq"], want["interp"])


FGC360_CASES, FGC360_INPUTS = G.fgc_grid(video_360=True)


def test_360_grid_is_served():
    assert len(FGC360_CASES) == 16


@pytest.mark.parametrize("c", FGC360_CASES, ids=[c["id"] for c in FGC360_CASES])
def test_fgbg_core_360_grid(c):
    """The grid's cases with 360 Video on, which retime-fgbg turns into the engine's wrap-around flag
    (plugins/retime-fgbg/src/glue.rs:146-151): the wrap solve (flow/extras.rs:286-430 with the 360
    gradient, Gaussians, B step, block matching and upsample of flow.rs:625-1246), the 360 inverse
    warps, the 360 passes of the hole fill and the plate refills, the 360 taps of Blur Compensation
    and the 360 Contrast/Edge prep."""
    w, h = c["width"], c["height"]
    fmt = G.FMT_OF_DEPTH[c["depth"]]
    kw = G.fgc_case_params(c)
    assert kw["wrap_360"]
    p = O.retime_params(rows_reversed=True, taps_above_first=True, **kw)
    out = O.retime_fgbg_clip(FGC360_INPUTS[c["input"]], c["frames"], [], [], [], w, h, fmt, p, c["frames"])
    assert hashlib.sha256(out.tobytes()).hexdigest() == c["sha256"]
