"""The allocation-free block matching entry point, for callers that cannot call cudaMalloc.

A host that owns the device memory pool (a plugin inside a video application) or a real-time
render thread can pass only its own device buffers; tw_block_match_noalloc works on those with a
fixed scratch array inside the library. This checks, through the C ABI, that calls in a row give
exactly what the allocating entry point tw_block_match gives (the tolerance of every parity test
here: bit for bit), on the default stream and on a stream of the caller's own, that a call does
not see the previous call's scratch (a small frame after a large one), that frames above the
scratch limit are refused, and that a call after the host reset the device (a new context, in a
child process) still works on lines long enough to need the raised shared memory limit. The file
is named to run last.
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import twixtor_b200 as tw

pytestmark = pytest.mark.gpu

TOO_LARGE = 7
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _case(seed, w, h):
    rng = np.random.RandomState(seed)
    a = (rng.random_sample((h, w)) * 60).astype(np.float32)
    b = (np.roll(a, 2, axis=1) + rng.random_sample((h, w)).astype(np.float32)).astype(np.float32)
    flow = ((rng.random_sample(w * h * 2) - 0.5) * 5).astype(np.float32)
    return a, b, flow


def _noalloc():
    L = tw.library()
    L.tw_block_match_noalloc.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
    return L


def test_no_alloc_block_match_equals_the_allocating_entry_point():
    import torch

    tw.build()
    L = _noalloc()
    torch.cuda.set_device(0)
    own = torch.cuda.Stream()
    with tw.Device(0) as dev:
        # the small case again after the large one: nothing of the large call's scratch may reach it
        for call, (seed, w, h, stream) in enumerate([(21, 97, 61, None), (22, 960, 540, own), (21, 97, 61, own),
                                                     (23, 1500, 300, None)]):
            a, b, flow = _case(seed, w, h)
            want = dev.block_match(a, b, flow, w, h)
            da = torch.from_numpy(a).cuda()
            db = torch.from_numpy(b).cuda()
            df = torch.from_numpy(flow.copy()).cuda()
            torch.cuda.synchronize()
            handle = stream.cuda_stream if stream is not None else 0
            rc = L.tw_block_match_noalloc(ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(db.data_ptr()),
                                          ctypes.c_void_p(df.data_ptr()), w, h, ctypes.c_void_p(handle))
            assert rc == 0, f"call {call}: status {rc}"
            got = df.cpu().numpy()
            assert got.view(np.uint32).tobytes() == want.view(np.uint32).tobytes(), f"call {call} differs"
            assert not np.array_equal(got, flow), "the sweeps changed nothing: the case does not exercise them"
        # refused before any launch: too many pixels, or a side above 6144 (buffers are never read)
        big = torch.zeros((1 << 19) + 1024, dtype=torch.float32, device="cuda")
        flow_big = torch.zeros(2 * big.numel(), dtype=torch.float32, device="cuda")
        for w, h in [(1024, 513), (6145, 2)]:
            rc = L.tw_block_match_noalloc(ctypes.c_void_p(big.data_ptr()), ctypes.c_void_p(big.data_ptr()),
                                          ctypes.c_void_p(flow_big.data_ptr()), w, h, ctypes.c_void_p(0))
            assert rc == TOO_LARGE, f"{w}x{h}: status {rc}"


_CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import twixtor_b200 as tw
from test_zz_no_alloc import _case, _noalloc

L = _noalloc()
rt = ctypes.CDLL("libcudart.so.12")  # the runtime the library itself loaded
rt.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
rt.cudaFree.argtypes = [ctypes.c_void_p]

def run(a, b, flow, w, h):
    bufs = []
    for x in (a, b, flow):
        p = ctypes.c_void_p()
        assert rt.cudaMalloc(ctypes.byref(p), x.nbytes) == 0
        assert rt.cudaMemcpy(p, x.ctypes.data, x.nbytes, 1) == 0
        bufs.append(p)
    rc = L.tw_block_match_noalloc(bufs[0], bufs[1], bufs[2], w, h, None)
    out = np.empty_like(flow)
    assert rt.cudaMemcpy(out.ctypes.data, bufs[2], out.nbytes, 2) == 0
    for p in bufs:
        rt.cudaFree(p)
    return rc, out

w, h = 2000, 200  # a row of 2000 needs more than the default 48 KiB of shared memory
a, b, flow = _case(31, w, h)
rc1, first = run(a, b, flow, w, h)
assert rt.cudaDeviceReset() == 0  # ends this process's own context; the next call runs in a new one
rc2, second = run(a, b, flow, w, h)
with tw.Device(0) as dev:
    want = dev.block_match(a, b, flow, w, h)
print(json.dumps({"rc": [rc1, rc2], "first": first.tobytes() == want.tobytes(),
                  "second": second.tobytes() == want.tobytes(), "changed": bool(not np.array_equal(want, flow))}))
"""


def test_no_alloc_block_match_after_a_device_reset():
    """In a child process (a reset would pull the device out from under this process's torch): a
    call, cudaDeviceReset, then a call in the new context on a 2000-wide frame."""
    tw.build()
    r = subprocess.run([sys.executable, "-c", _CHILD, ROOT], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["rc"] == [0, 0], res
    assert res["first"] and res["second"] and res["changed"], res
