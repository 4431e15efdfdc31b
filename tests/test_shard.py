"""One clip over several ranks (the multi-GPU path of bench.py), checked on CPU with gloo.

An output frame of the retime effect reads only the two clip frames of its selection
(timeline.rs:447-469), so the ranks split the output frames into contiguous ranges (tw_shard), each
rank holds only the clip frames its range reads (tw_source_window), and nothing is exchanged: the
outputs concatenate in rank order. Here two gloo ranks each render their range with the oracle from
their window alone (the oracle refuses a frame outside the window it is given); the ranges are
gathered on rank 0 and must equal the single process render of the whole clip byte for byte.
"""
import datetime
import os
import socket

import numpy as np
import pytest

import oracle_lib as O
import twixtor_b200 as tw
from twixtor_b200 import synth

W, H, N, NOUT, SPEED = 160, 96, 48, 95, 50.0  # the 160x96 retime clip: 48 frames to 95 at speed 50 %


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("nout,nranks", [(95, 2), (95, 8), (7, 3), (3, 5), (0, 2), (1000, 7)])
def test_shard_ranges_partition_the_clip(nout, nranks):
    ranges = [tw.shard(nout, nranks, r) for r in range(nranks)]
    assert ranges[0][0] == 0 and ranges[-1][1] == nout
    for (lo, hi), (lo2, _) in zip(ranges, ranges[1:]):
        assert hi == lo2 and lo <= hi
    sizes = [hi - lo for lo, hi in ranges]
    assert max(sizes) - min(sizes) <= 1


def test_source_windows_cover_each_range_and_overlap_only_at_boundaries():
    tp = tw.TimeParams(speed_percent=SPEED)
    sels = [tw.select(tp, n, W, H) for n in range(NOUT)]
    wins = []
    for r in range(4):
        lo, hi = tw.shard(NOUT, 4, r)
        first, last = tw.source_window(sels[lo:hi], N)
        for s in sels[lo:hi]:
            for f in (s.a, s.b):
                assert not (0 <= f < N) or first <= f <= last
        wins.append((first, last))
    for (_, last), (first2, _) in zip(wins, wins[1:]):
        assert first2 >= last - 1  # neighbours share at most the boundary frames
    # a selection past the clip's end reads nothing from it
    assert tw.source_window([tw.Selection(a=N + 3, b=N + 4)], N) == (0, -1)


def test_clip_window_equals_the_slice_of_the_whole_clip():
    whole = synth.moving_clip(W, H, N, depth=8)
    part = synth.moving_clip(W, H, N, depth=8, window=(10, 17))
    fb = W * H * 4
    assert part.tobytes() == whole[10 * fb:18 * fb].tobytes()


def _rank(rank, ws, port):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=120))
    try:
        O.lib().or_set_threads(2)
        tp = tw.TimeParams(speed_percent=SPEED)
        sels = [tw.select(tp, n, W, H) for n in range(NOUT)]
        lo, hi = tw.shard(NOUT, ws, rank)
        first, last = tw.source_window(sels[lo:hi], N)
        frames = synth.moving_clip(W, H, N, depth=8, window=(first, last))  # this rank's frames only
        p = O.retime_params(speed=SPEED)
        outs = [O.retime_window(frames, first, last - first + 1, N, W, H, 0, p, n) for n in range(lo, hi)]
        mine = np.concatenate(outs) if outs else np.zeros(0, np.uint8)
        got = [None] * ws
        dist.all_gather_object(got, (lo, hi, mine.tobytes()))
        if rank == 0:
            joined = b"".join(b for _, _, b in sorted(got))
            whole = synth.moving_clip(W, H, N, depth=8)
            want = O.retime_clip(whole, N, W, H, 0, p, NOUT)
            assert [(lo_, hi_) for lo_, hi_, _ in sorted(got)] == [tw.shard(NOUT, ws, r) for r in range(ws)]
            assert joined == want.tobytes(), "the ranks' ranges do not concatenate to the whole clip's render"
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_render_one_clip_byte_identical():
    import torch.multiprocessing as mp
    tw.library()
    O.lib()
    mp.spawn(_rank, args=(2, _free_port()), nprocs=2, join=True)
