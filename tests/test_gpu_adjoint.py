"""The CUDA adjoint of warp + blend (tw_warp_blend_adjoint) against the FP64 reference
(oracle/adjoint_fp64.py) and finite differences, and the photometric flow refinement it drives.

Tolerances (float32 kernels, float32 atomics in an arbitrary order): the forward within 1e-5
absolute of the FP64 values for frames in [0, 1]; every gradient within 1e-3 of the FP64 gradient
relative to its norm; a directional finite difference of the device forward (eps 1e-3) within 2 %
of the device gradient along the same direction. The FP64 reference forms the sample positions in
single precision as the kernel does: a position within rounding of a pixel boundary then lands in
the same bilinear cell on both sides (the image gradient jumps there), and the comparison measures
the arithmetic, not which side of a boundary a rounding picked."""
import os
import sys

import numpy as np
import pytest
import torch

import twixtor_b200 as tw
from twixtor_b200 import adjoint, synth

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
import adjoint_fp64 as A  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    tw.build()
    d = tw.Device(0)
    yield d
    d.close()


def rel(x, ref):
    return float(np.linalg.norm(np.asarray(x, np.float64) - ref) / max(np.linalg.norm(ref), 1e-30))


def batch_case(w, h, fw, fh, n, seed):
    rng = np.random.RandomState(seed)
    a = rng.rand(n, h, w, 4).astype(np.float32)
    b = rng.rand(n, h, w, 4).astype(np.float32)
    fab = rng.uniform(-3, 3, (n, fh, fw, 2)).astype(np.float32)
    fba = rng.uniform(-3, 3, (n, fh, fw, 2)).astype(np.float32)
    t = rng.rand(n, h, w, 4).astype(np.float32)
    g = rng.randn(n, h, w, 4).astype(np.float32)
    cu = lambda x: torch.from_numpy(x).cuda()  # noqa: E731
    return [cu(x) for x in (a, b, fab, fba, t, g)], (a, b, fab, fba, t, g)


@pytest.mark.parametrize("w,h,fw,fh", [(64, 40, 32, 20), (37, 23, 37, 23), (20, 12, 39, 23), (96, 64, 48, 32)])
@pytest.mark.parametrize("wa", [0.3, 0.5, 0.85])
@pytest.mark.parametrize("mode", ["l1", "grad_out"])
def test_matches_fp64(dev, w, h, fw, fh, wa, mode):
    n = 3
    (a, b, fab, fba, t, g), host = batch_case(w, h, fw, fh, n, w * 7 + fw + int(wa * 10))
    if mode == "l1":
        loss, da, db, dfab, dfba = adjoint.l1_loss_and_grads(dev, a, b, fab, fba, t, wa)
    else:
        da, db, dfab, dfba = (torch.zeros_like(x) for x in (a, b, fab, fba))
        dev.set_stream(torch.cuda.current_stream().cuda_stream)
        dev.warp_blend_adjoint(a.data_ptr(), b.data_ptr(), fab.data_ptr(), fba.data_ptr(), w, h, fw, fh, n, wa,
                               grad_out=g.data_ptr(), da=da.data_ptr(), db=db.data_ptr(), df_ab=dfab.data_ptr(),
                               df_ba=dfba.data_ptr())
    out = adjoint.warp_blend(a, b, fab, fba, wa, dev)
    torch.cuda.synchronize()
    for i in range(n):
        args = [x[i].reshape(-1) for x in host[:4]]
        o32 = out[i].cpu().numpy().reshape(-1)
        if mode == "l1":
            # the L1 loss's gradient is sign(out - target): the FP64 backward takes the signs of the
            # device's own output, so that a sample within rounding of its target (whose sign float32
            # and float64 may decide differently) is compared as the same branch
            tt = host[4][i].reshape(-1)
            lref, oref, *_ = A.warp_blend_grads(*args, w, h, fw, fh, wa, target=tt)
            assert abs(loss[i].item() - lref) < 1e-4 * lref
            kw = dict(grad_out=np.sign(o32.astype(np.float64) - tt))
        else:
            kw = dict(grad_out=host[5][i].reshape(-1))
        # positions formed in single precision as on the device (the same bilinear cells), the rest double
        _, oref, daref, dbref, dfabref, dfbaref = A.warp_blend_grads(*args, w, h, fw, fh, wa, pos32=True, **kw)
        assert np.abs(o32.astype(np.float64) - oref.reshape(-1)).max() < 1e-5
        for got, ref in ((da, daref), (db, dbref), (dfab, dfabref), (dfba, dfbaref)):
            assert rel(got[i].cpu().numpy(), ref) < 1e-3


def test_autograd_and_finite_differences(dev):
    """torch.autograd through WarpBlend, and a directional finite difference of the device forward."""
    w, h, fw, fh, n = 48, 32, 24, 16, 2
    (_, _, fab, fba, _, g), _ = batch_case(w, h, fw, fh, n, 3)
    # smooth frames (the refinement workload's noise texture): the sampled image's gradient varies
    # slowly, so a finite difference over 1e-3 of the flows sees the derivative the adjoint takes
    A_, B_, _, _ = synth.adjoint_triples(w, h, n, seed=11)
    a, b = torch.from_numpy(A_).cuda(), torch.from_numpy(B_).cuda()
    wa = 0.4
    xs = [x.clone().requires_grad_(True) for x in (a, b, fab, fba)]
    out = adjoint.warp_blend(*xs, wa, dev)
    (out * g).sum().backward()
    rng = np.random.RandomState(9)
    eps = 1e-3
    for k in range(4):
        d = torch.from_numpy(rng.randn(*xs[k].shape).astype(np.float32)).cuda()
        args_p = [x.detach().clone() for x in xs]
        args_m = [x.detach().clone() for x in xs]
        args_p[k] += eps * d
        args_m[k] -= eps * d
        with torch.no_grad():
            fp = (adjoint.warp_blend(*args_p, wa, dev).double() * g.double()).sum().item()
            fm = (adjoint.warp_blend(*args_m, wa, dev).double() * g.double()).sum().item()
        num = (fp - fm) / (2 * eps)
        ana = (xs[k].grad.double() * d.double()).sum().item()
        assert abs(num - ana) < 2e-2 * max(abs(ana), 1.0), (k, num, ana)


def test_refinement_beats_the_solver(dev):
    """Photometric refinement from the plain solver's flows (50 Adam steps on the L1 loss against the
    middle frame) lowers the loss and raises the PSNR of the interpolated frame."""
    w, h = 320, 180
    A_, B_, M_, _ = synth.adjoint_triples(w, h, 1)
    fs = tw.FlowSettings()
    f_ab, f_ba, (fw, fh) = dev.solve_pair(A_[0].reshape(-1), B_[0].reshape(-1), w, h, 2, fs)
    cu = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    a, b, m = cu(A_), cu(B_), cu(M_)
    fab = cu(f_ab.reshape(1, fh, fw, 2))
    fba = cu(f_ba.reshape(1, fh, fw, 2))
    wa = 0.5

    def psnr(x):
        mse = torch.mean((x - m) ** 2).item()
        return 10 * np.log10(1.0 / mse)

    base = adjoint.warp_blend(a, b, fab, fba, wa, dev)
    rab, rba, hist = adjoint.refine_flows(dev, a, b, fab, fba, m, wa, steps=50, lr=0.05)
    ref = adjoint.warp_blend(a, b, rab, rba, wa, dev)
    assert hist[-1] < hist[0]
    assert psnr(ref) > psnr(base) + 0.5


def test_smooth_flows_match_fp64(dev):
    """Smooth flows (the refinement workload's displacements): neighbouring samples share their
    corners, so the scatter sums them in registers (carried down a column, handed to the next lane)
    before the shared tile; the gradients still match the FP64 reference."""
    w, h, fw, fh, n, wa = 160, 96, 80, 48, 2, 0.5
    A_, B_, M_, D_ = synth.adjoint_triples(w, h, n, seed=5, peak=6.0)
    d_half = np.ascontiguousarray(D_[:, ::2, ::2, :] * np.float32(0.5))
    cu = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    a, b, m, fab, fba = cu(A_), cu(B_), cu(M_), cu(d_half), cu(-d_half)
    loss, da, db, dfab, dfba = adjoint.l1_loss_and_grads(dev, a, b, fab, fba, m, wa)
    out = adjoint.warp_blend(a, b, fab, fba, wa, dev)
    torch.cuda.synchronize()
    for i in range(n):
        args = [np.ascontiguousarray(x[i]).reshape(-1) for x in (A_, B_, d_half, -d_half)]
        tt = M_[i].reshape(-1)
        o32 = out[i].cpu().numpy().reshape(-1)
        kw = dict(grad_out=np.sign(o32.astype(np.float64) - tt))
        _, oref, daref, dbref, dfabref, dfbaref = A.warp_blend_grads(*args, w, h, fw, fh, wa, pos32=True, **kw)
        assert np.abs(o32.astype(np.float64) - oref.reshape(-1)).max() < 1e-5
        for got, ref in ((da, daref), (db, dbref), (dfab, dfabref), (dfba, dfbaref)):
            assert rel(got[i].cpu().numpy(), ref) < 1e-3


@pytest.mark.parametrize("wa", [0.25, 0.5, 0.8])
def test_forward_is_the_library_warp_and_blend(dev, wa):
    """The adjoint's forward is compose_vectors' Blend with warping code 0 on float frames:
    blend(inv_warp(A, F_BA, 1 - wa), inv_warp(B, F_AB, wa), 1 - wa) by tw_inv_warp (hold) and
    tw_blend, wherever no sample leaves the image (there the library slides the point back along
    its segment, the adjoint clamps it). The positions round differently (u * s / r against
    u * (s / r)), so the values agree to float rounding, not bit for bit."""
    w, h, fw, fh = 96, 64, 48, 32
    rng = np.random.RandomState(int(wa * 100))
    a = rng.rand(h, w, 4).astype(np.float32)
    b = rng.rand(h, w, 4).astype(np.float32)
    fab = rng.uniform(-1.5, 1.5, (fh, fw, 2)).astype(np.float32)
    fba = rng.uniform(-1.5, 1.5, (fh, fw, 2)).astype(np.float32)
    cu = lambda x: torch.from_numpy(np.ascontiguousarray(x)[None]).cuda()  # noqa: E731
    out = adjoint.warp_blend(cu(a), cu(b), cu(fab), cu(fba), wa, dev)[0].cpu().numpy()
    ta = dev.inv_warp(a.reshape(-1), w, h, 2, fba.reshape(-1), (fw, fh), 1.0 - wa, hold=True)
    tb = dev.inv_warp(b.reshape(-1), w, h, 2, fab.reshape(-1), (fw, fh), wa, hold=True)
    ref = dev.blend(ta, tb, w, h, 2, 1.0 - wa).reshape(h, w, 4)
    # displacements reach 1.5 / r ~ 3 px: the pixels 4 or more from the border never clip
    inner = (slice(4, h - 4), slice(4, w - 4))
    assert np.abs(out[inner].astype(np.float64) - ref[inner]).max() < 1e-5
