"""The timed paths at their benchmark sizes, byte for byte against the oracle.

bench.py times tw_retime_clip_device and tw_retime_clip at 1920x1080 with four output frames in
flight, tw_retime_batch_device on float clips up to 3840x2160, and tw_retime_layers_clip at 1080p
with its staged second upload slot. The smaller parity cases pin every kernel; these pin the
multi-lane drivers, the frame cache and the staging at the sizes the numbers are quoted at.
"""
import numpy as np
import pytest

import oracle_lib as O
import twixtor_b200 as tw
from twixtor_b200 import synth

pytestmark = pytest.mark.gpu

W, H, SPEED = 1920, 1080, 40.0
CLIP_KW = dict(seed=0x74570002, bg_velocity=(6.0, -3.0), square=240, square_start=(600.0, 400.0),
               square_velocity=(9.0, 4.0))
BATCH_KEYS = [(0.0, 100.0, True), (48.0, 25.0, True), (96.0, 100.0, True)]


@pytest.fixture(scope="module")
def dev():
    tw.build()
    d = tw.Device(0)
    yield d
    d.close()


@pytest.fixture(scope="module")
def clip1080():
    nframes = 8
    return synth.moving_clip(W, H, nframes, depth=8, **CLIP_KW), nframes


def same(a, b):
    return np.asarray(a).view(np.uint8).tobytes() == np.asarray(b).view(np.uint8).tobytes()


def test_clip_device_1080p_four_lanes_matches_oracle(dev, clip1080):
    """12 consecutive output frames (3 exact, 9 in-between) of the 1080p workload through
    tw_retime_clip_device with 4 lanes, the bench's device resident path."""
    import torch
    frames, nframes = clip1080
    tp = tw.TimeParams(speed_percent=SPEED)
    sels = [tw.select(tp, n, W, H) for n in range(12)]
    assert sum(not s.exact for s in sels) >= 8
    dev.set_lanes(4)
    d_in = torch.from_numpy(frames).cuda()
    d_out = torch.zeros(len(sels) * W * H * 4, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    dev.retime_clip_device(tw.RetimeSettings(), d_in.data_ptr(), nframes, sels, W, H, 0, d_out.data_ptr())
    want = O.retime_clip(frames, nframes, W, H, 0, O.retime_params(speed=SPEED), len(sels))
    assert same(d_out.cpu().numpy(), want)


@pytest.mark.parametrize("lanes", [4, 0])
def test_clip_host_1080p_matches_oracle(dev, clip1080, lanes):
    """The e2e path (host buffers, frame cache, copy streams) at 1080p with 4 lanes, and the serial
    mode the benchmark's per-kernel timing uses; output frames 2..13."""
    frames, nframes = clip1080
    tp = tw.TimeParams(speed_percent=SPEED)
    sels = [tw.select(tp, n, W, H) for n in range(2, 14)]
    dev.set_lanes(lanes)
    try:
        got = dev.retime_clip(tw.RetimeSettings(), frames, nframes, sels, W, H, 0)
    finally:
        dev.set_lanes(4)
    want = O.retime_clip(frames, nframes, W, H, 0, O.retime_params(speed=SPEED), 14)[2 * W * H * 4:]
    assert same(got, want)


def test_clip_window_of_a_shard_matches_oracle(dev):
    """A rank of the sharded benchmark: output frames 20..29 of a longer clip rendered from that
    range's source window alone (rebased selections), against the oracle's render from the same
    window."""
    nclip = 40
    tp = tw.TimeParams(speed_percent=SPEED)
    sels = [tw.select(tp, n, W, H) for n in range(20, 30)]
    first, last = tw.source_window(sels, nclip)
    window = synth.moving_clip(W, H, nclip, depth=8, window=(first, last), **CLIP_KW)
    got = dev.retime_clip(tw.RetimeSettings(), window, last - first + 1, tw.rebase(sels, first, nclip), W, H, 0)
    p = O.retime_params(speed=SPEED)
    want = np.concatenate([O.retime_window(window, first, last - first + 1, nclip, W, H, 0, p, n)
                           for n in range(20, 30)])
    assert same(got, want)


def test_batch_config_sizes_match_oracle(dev):
    """The batched retime at its largest and smallest clip sizes (3840x2160 and 1280x720 float RGBA,
    the keyed ramp): the first in-between frame of each and the frame after it, in one call."""
    import torch
    tp = tw.TimeParams(keys=BATCH_KEYS)
    p = O.retime_params(keys=BATCH_KEYS)
    jobs, keep, checks = [], [], []
    for i, (w, h) in [(3, (3840, 2160)), (0, (1280, 720))]:
        all_sels = [tw.select(tp, n, w, h) for n in range(12)]
        k = next(n for n, s in enumerate(all_sels) if not s.exact)
        sels = all_sels[k:k + 2]
        nsrc = max(max(s.a, s.b) for s in sels) + 1
        frames = synth.batch_clip_gpu(w, h, nsrc, seed=0x74570030 + i)
        out = torch.zeros(len(sels) * w * h * 4, dtype=torch.float32, device="cuda")
        keep += [frames, out]
        jobs.append(dict(settings=tw.RetimeSettings(), frames=frames.data_ptr(), nframes=nsrc, sels=sels, width=w,
                         height=h, fmt=2, out=out.data_ptr()))
        checks.append((w, h, k, nsrc, frames, out))
    dev.set_lanes(4)
    dev.retime_batch_device(jobs)
    torch.cuda.synchronize()
    for w, h, k, nsrc, frames, out in checks:
        host = frames.cpu().numpy()
        want = np.concatenate([O.retime_one(host, nsrc, w, h, 2, p, n) for n in (k, k + 1)])
        assert same(out.cpu().numpy(), want), f"{w}x{h}"


def test_fgbg_clip_1080p_five_frames_matches_oracle(dev):
    """tw_retime_layers_clip over 5 output frames of the 1080p three-layer workload (exact and
    in-between frames, the next frame's uploads staged in the second slot while one renders)."""
    nframes = 4
    frames, mattes = synth.layered_clip(W, H, nframes, nfg=3)
    tp = tw.TimeParams(speed_percent=SPEED)
    sels = [tw.select(tp, k, W, H) for k in range(5)]
    s = tw.RetimeSettings(compose=tw.EngineSettings(gouraud=True))
    sens = [tw.percent_param(70.0)] * 4
    got = dev.retime_layers_clip(s, frames, nframes, mattes, [1, 1, 1], sens, sels, W, H, 0)
    want = O.retime_fgbg_clip(frames, nframes, mattes, [1, 1, 1], [70.0] * 3, W, H, 0, O.retime_params(speed=SPEED), 5)
    assert same(got, want)


@pytest.mark.parametrize("lanes,size,nout", [(1, (160, 96), 24), (2, (320, 180), 20), (4, (1920, 1080), 16)])
def test_graph_replay_matches_direct_launches(dev, lanes, size, nout):
    """The clip call with CUDA graphs (captured at a lane's second frame of a shape, replayed with
    updated arguments after) against the same call with graphs off and against the oracle."""
    import torch
    w, h = size
    nframes = int(np.ceil(0.4 * nout)) + 2
    kw = CLIP_KW if w == 1920 else dict(seed=w + h)
    frames = synth.moving_clip(w, h, nframes, depth=8, **kw)
    tp = tw.TimeParams(speed_percent=SPEED)
    sels = [tw.select(tp, n, w, h) for n in range(nout)]
    d_in = torch.from_numpy(frames).cuda()
    outs = []
    dev.set_lanes(lanes)
    try:
        for graphs in (True, False, True):
            dev.set_graphs(graphs)
            d_out = torch.zeros(nout * w * h * 4, dtype=torch.uint8, device="cuda")
            torch.cuda.synchronize()
            dev.retime_clip_device(tw.RetimeSettings(), d_in.data_ptr(), nframes, sels, w, h, 0, d_out.data_ptr())
            outs.append(d_out.cpu().numpy())
    finally:
        dev.set_lanes(4)
        dev.set_graphs(True)
    want = O.retime_clip(frames, nframes, w, h, 0, O.retime_params(speed=SPEED), nout)
    for o in outs:
        assert same(o, want)
