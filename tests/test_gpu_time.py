"""The time model through the CUDA clip call: the served cases of the reference's retime-time
parity grid (No Vectors: Speed and Frame Number modes, keyed curves, the input rate model, Frame
Interp) rendered by tw_retime_clip with the selections of tw_select, against the sha256 of the
output clips results/base.tsv records (the frame time bias 0.1 of that revision)."""
import hashlib

import pytest

import golden_data as G
import twixtor_b200 as tw
from test_oracle_time import RT_CASES, RT_INPUTS, rt_params, time_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    tw.build()
    d = tw.Device(0)
    yield d
    d.close()


@pytest.mark.parametrize("c", rt_params())
def test_retime_time_grid_sha256(dev, c):
    w, h = c["width"], c["height"]
    fmt = G.FMT_OF_DEPTH[c["depth"]]
    tp = time_params(G.rt_case_params(c), bias=0.1)
    sels = [tw.select(tp, n, w, h) for n in range(c["frames"])]
    s = tw.RetimeSettings(flow=tw.FlowSettings(taps_above_first=False),
                          compose=tw.EngineSettings(taps_above_first=False), motion_rows_reversed=False)
    out = dev.retime_clip(s, RT_INPUTS[c["input"]].view(tw.DTYPES[fmt]), c["frames"], sels, w, h, fmt)
    assert hashlib.sha256(out.tobytes()).hexdigest() == c["sha256"]
