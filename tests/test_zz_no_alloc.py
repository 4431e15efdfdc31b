"""The allocation-free block matching entry point, for callers that cannot call cudaMalloc.

A host that owns the device memory pool (a plugin inside a video application) or a real-time
render thread can pass only its own device buffers; tw_block_match_noalloc works on those with a
fixed scratch array inside the library. This checks, through the C ABI, that two calls in a row
give exactly what the allocating entry point tw_block_match gives (the tolerance of every parity
test here: bit for bit), that the second call does not see the first call's scratch, and that a
frame above the scratch limit is refused. The file is named to run last.
"""
import ctypes

import numpy as np
import pytest

import twixtor_b200 as tw

pytestmark = pytest.mark.gpu

TOO_LARGE = 7


def _case(seed, w, h):
    rng = np.random.RandomState(seed)
    a = (rng.random_sample((h, w)) * 60).astype(np.float32)
    b = (np.roll(a, 2, axis=1) + rng.random_sample((h, w)).astype(np.float32)).astype(np.float32)
    flow = ((rng.random_sample(w * h * 2) - 0.5) * 5).astype(np.float32)
    return a, b, flow


def test_no_alloc_block_match_equals_the_allocating_entry_point():
    import torch

    tw.build()
    L = tw.library()
    L.tw_block_match_noalloc.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    with tw.Device(0) as dev:
        for call, (seed, w, h) in enumerate([(21, 97, 61), (22, 960, 540)]):
            a, b, flow = _case(seed, w, h)
            want = dev.block_match(a, b, flow, w, h)
            da = torch.from_numpy(a).cuda()
            db = torch.from_numpy(b).cuda()
            df = torch.from_numpy(flow.copy()).cuda()
            torch.cuda.synchronize()
            rc = L.tw_block_match_noalloc(ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(db.data_ptr()),
                                          ctypes.c_void_p(df.data_ptr()), w, h, ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0, f"call {call}: status {rc}"
            got = df.cpu().numpy()
            assert got.view(np.uint32).tobytes() == want.view(np.uint32).tobytes(), f"call {call} differs"
            assert not np.array_equal(got, flow), "the sweeps changed nothing: the case does not exercise them"
        big = torch.zeros((1 << 19) + 1024, dtype=torch.float32, device="cuda")
        flow_big = torch.zeros(2 * big.numel(), dtype=torch.float32, device="cuda")
        rc = L.tw_block_match_noalloc(ctypes.c_void_p(big.data_ptr()), ctypes.c_void_p(big.data_ptr()),
                                      ctypes.c_void_p(flow_big.data_ptr()), 1024, 513, ctypes.c_void_p(stream.cuda_stream))
        assert rc == TOO_LARGE
