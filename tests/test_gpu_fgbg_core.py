"""retime-fgbg without FG matte layers through the CUDA clip call (tw_retime_layers_clip with no
layer) against the sha256 the reference's fgbg-core parity grid records for its 360 served cases."""
import hashlib

import pytest

import golden_data as G
import twixtor_b200 as tw
from test_oracle_fgbg_core import FGC_CASES, FGC_INPUTS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    tw.build()
    d = tw.Device(0)
    yield d
    d.close()


@pytest.mark.parametrize("c", FGC_CASES, ids=[c["id"] for c in FGC_CASES])
def test_fgbg_core_grid_sha256(dev, c):
    fmt = G.FMT_OF_DEPTH[c["depth"]]
    w, h, n = c["width"], c["height"], c["frames"]
    kw = G.fgc_case_params(c)
    tp = tw.TimeParams(fps=kw["fps"], speed_percent=kw["speed"], keys=kw["keys"], vectors=kw["vectors"],
                       frame_interp=kw["frame_interp"], blur_compensation=kw["blur"], remap_mode=kw["remap_mode"],
                       frame_num=kw["frame_num"], fn_keys=kw["fn_keys"], own_input_rate=kw["own_input_rate"],
                       input_frame_rate=kw["input_frame_rate"], frame_time_plain=True,
                       input_fields=kw["input_fields"], mark_segs=kw["mark_segs"], mark_keys=kw["mark_keys"])
    sels = [tw.select(tp, k, w, h) for k in range(n)]
    sens = tw.percent_param(kw["sensitivity"])
    both = kw["prep"] == 4
    s = tw.RetimeSettings(flow=tw.FlowSettings(hiq=True, sensitivity=float(sens), taps_above_first=True,
                                               track_alpha=kw["track_rgb_a"], prep_contrast_edge=both,
                                               prep_delinearize=both),
                          compose=tw.EngineSettings(warp_mode=kw["smart_blend"], taps_above_first=True, gouraud=True,
                                                    blur=float(tw.fixed_param(kw["blur"]))),
                          motion_rows_reversed=True)
    out = dev.retime_layers_clip(s, FGC_INPUTS[c["input"]].view(tw.DTYPES[fmt]), n, [], [], [sens], sels, w, h, fmt)
    assert hashlib.sha256(out.tobytes()).hexdigest() == c["sha256"]
