"""The FP64 reference of the warp + blend adjoint (oracle/adjoint_fp64.py) against central finite
differences of its own forward: every gradient (frames and both flows), from a given output gradient
and from the L1 loss, at sizes where the flow grid is coarser than, equal to and finer than the
image."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
import adjoint_fp64 as A  # noqa: E402


def case(w, h, fw, fh, seed):
    rng = np.random.RandomState(seed)
    return (rng.rand(w * h * 4), rng.rand(w * h * 4), rng.uniform(-2.5, 2.5, fw * fh * 2),
            rng.uniform(-2.5, 2.5, fw * fh * 2), rng)


@pytest.mark.parametrize("w,h,fw,fh", [(12, 9, 7, 5), (10, 8, 10, 8), (6, 5, 11, 9)])
@pytest.mark.parametrize("wa", [0.25, 0.5, 0.8])
def test_gradients_match_finite_differences(w, h, fw, fh, wa):
    a, b, fab, fba, rng = case(w, h, fw, fh, w * 31 + fw)
    G = rng.randn(w * h * 4)
    _, _, da, db, dfab, dfba = A.warp_blend_grads(a, b, fab, fba, w, h, fw, fh, wa, grad_out=G)

    def f(args):
        return float((A.warp_blend(*args, w, h, fw, fh, wa).reshape(-1) * G).sum())

    eps = 1e-6
    for var, g in ((0, da), (1, db), (2, dfab), (3, dfba)):
        g = g.reshape(-1)
        for i in rng.choice(g.size, 12, replace=False):
            args = [a.copy(), b.copy(), fab.copy(), fba.copy()]
            args[var][i] += eps
            p = f(args)
            args[var][i] -= 2 * eps
            m = f(args)
            assert abs((p - m) / (2 * eps) - g[i]) < 1e-6 * max(1.0, abs(g[i]))


def test_l1_loss_gradient():
    w, h, fw, fh = 12, 9, 7, 5
    a, b, fab, fba, rng = case(w, h, fw, fh, 7)
    t = rng.rand(w * h * 4)
    loss, out, da, db, dfab, dfba = A.warp_blend_grads(a, b, fab, fba, w, h, fw, fh, 0.4, target=t)
    assert abs(loss - np.abs(out.reshape(-1) - t).sum()) < 1e-9
    # a small step along the negative flow gradient lowers the loss
    step = 1e-4
    l2, *_ = A.warp_blend_grads(a, b, fab - step * dfab.reshape(-1), fba - step * dfba.reshape(-1), w, h, fw, fh, 0.4,
                                target=t)
    assert l2 < loss
