"""Host-injected failures come back as statuses, and the context stays usable.

The reference's device backend refuses a stage with an error that its executor turns into a CPU
rerun (device/exec/mod.rs:332-369); its tests fake failing backends (device/exec/tests.rs). Here
the failures are made on the host, so nothing faults, traps or hangs the GPU: a device allocation
that fails as cudaMalloc out of memory would (tw_debug_inject), a device status word set by a kernel
as a bounded loop that ran out sets it, and input or output buffers shorter than their images.
After each, the next call on the same context renders the same bytes as the oracle.
"""
import ctypes

import numpy as np
import pytest

import oracle_lib as O
import twixtor_b200 as tw
from twixtor_b200 import synth

pytestmark = pytest.mark.gpu

W, H, N = 160, 96, 8


@pytest.fixture(scope="module")
def clip():
    frames = synth.moving_clip(W, H, N, depth=8, seed=9)
    tp = tw.TimeParams(speed_percent=50.0)
    sels = [tw.select(tp, n, W, H) for n in range(6)]
    want = O.retime_clip(frames, N, W, H, 0, O.retime_params(speed=50.0), 6)
    return frames, sels, want


def test_injected_allocation_failure_is_a_status(clip):
    frames, sels, want = clip
    tw.build()
    for n in (1, 3, 9):  # the first allocation, and ones in the middle of the lanes' set-up
        with tw.Device(0) as dev:
            dev.debug_inject(tw.INJECT_ALLOC, n)
            with pytest.raises(tw.StageError) as e:
                dev.retime_clip(tw.RetimeSettings(), frames, N, sels, W, H, 0)
            assert e.value.code == tw.ERR_CUDA and "injected" in str(e.value)
            got = dev.retime_clip(tw.RetimeSettings(), frames, N, sels, W, H, 0)
            assert got.tobytes() == want.tobytes()


@pytest.mark.parametrize("n", [1, 2, 5])
def test_injected_device_status_is_a_status(clip, n):
    frames, sels, want = clip
    with tw.Device(0) as dev:
        dev.retime_clip(tw.RetimeSettings(), frames, N, sels, W, H, 0)  # buffers already in place
        dev.debug_inject(tw.INJECT_STATUS, n)
        with pytest.raises(tw.StageError) as e:
            dev.retime_clip(tw.RetimeSettings(), frames, N, sels, W, H, 0)
        assert e.value.code == tw.ERR_DEVICE_BOUND
        got = dev.retime_clip(tw.RetimeSettings(), frames, N, sels, W, H, 0)
        assert got.tobytes() == want.tobytes()


def test_injection_disarms_and_rejects_bad_arguments():
    with tw.Device(0) as dev:
        dev.debug_inject(tw.INJECT_ALLOC, 1)
        dev.debug_inject(tw.INJECT_NONE, 0)
        with pytest.raises(tw.BadParam):
            dev.debug_inject(7, 1)
        with pytest.raises(tw.BadParam):
            dev.debug_inject(tw.INJECT_STATUS, 0)
        frames = synth.moving_clip(W, H, 2, depth=8)
        sel = tw.select(tw.TimeParams(speed_percent=50.0), 1, W, H)
        fs = W * H * 4
        dev.retime_frame(tw.RetimeSettings(), sel, frames[:fs], frames[fs:], W, H, 0)


def test_truncated_buffers_are_refused():
    """An image descriptor whose buffer is one byte short, as input and as output."""
    L = tw.library()
    frames = synth.moving_clip(W, H, 2, depth=8)
    a = O.from_frame(frames[:W * H * 4], W, H, 0)
    b = O.from_frame(frames[W * H * 4:], W, H, 0)
    out = np.zeros_like(a)
    with tw.Device(0) as dev:
        ia = tw._Image(W, H, 0, a.ctypes.data, a.nbytes)
        ib_short = tw._Image(W, H, 0, b.ctypes.data, b.nbytes - 1)
        io = tw._Image(W, H, 0, out.ctypes.data, out.nbytes)
        io_short = tw._Image(W, H, 0, out.ctypes.data, out.nbytes - 1)
        rc = L.tw_blend(dev.handle, ctypes.byref(io), ctypes.byref(ia), ctypes.byref(ib_short), ctypes.c_float(0.5))
        assert rc == tw.ERR_BAD_PARAM
        rc = L.tw_blend(dev.handle, ctypes.byref(io_short), ctypes.byref(ia), ctypes.byref(ia), ctypes.c_float(0.5))
        assert rc == tw.ERR_BAD_PARAM
        assert not out.any(), "a refused call wrote its output"
        fw, fh, _ = tw.flow_geometry(tw.FlowSettings(), W, H)
        flow = np.zeros(fw * fh * 2, np.float32)
        fl = tw._Flow(fw, fh, flow.ctypes.data)
        rc = L.tw_solve(dev.handle, ctypes.byref(ia), ctypes.byref(ib_short), ctypes.byref(tw.FlowSettings()._c()),
                        ctypes.byref(fl))
        assert rc == tw.ERR_BAD_PARAM
        # the context still serves a well formed call
        got = dev.blend(a, b, W, H, 0, 0.5)
        want = np.zeros_like(a)
        O.lib().or_blend(O.ptr(want), O.ptr(a), O.ptr(b), W, H, 0, np.float32(0.5))
        assert got.tobytes() == want.tobytes()
