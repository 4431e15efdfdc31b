"""The differentiable warp + blend of the library on torch tensors (CUDA float32), for photometric
flow refinement: a torch.autograd.Function over tw_warp_blend_adjoint, the fused L1 loss with its
gradients, and a refinement loop that moves the solver's flows to lower the photometric loss
against a target frame.

Layouts: frames (batch, height, width, 4) float32, flows (batch, flow_h, flow_w, 2) float32, all on
the device of the ``Device`` handle, contiguous. The kernels run on the torch stream current at the
call (the handle's stream is set to it).
"""
import torch

import twixtor_b200 as tw


def _check(*ts):
    for t in ts:
        if t is not None and (not t.is_cuda or t.dtype != torch.float32 or not t.is_contiguous()):
            raise ValueError("warp + blend needs contiguous float32 CUDA tensors")


def _geometry(a, f):
    batch, h, w, c = a.shape
    if c != 4 or f.dim() != 4 or f.shape[-1] != 2 or f.shape[0] != batch:
        raise ValueError("frames (batch, h, w, 4) and flows (batch, fh, fw, 2) expected")
    return batch, w, h, f.shape[2], f.shape[1]


def _ptr(t):
    return t.data_ptr() if t is not None else 0


class WarpBlend(torch.autograd.Function):
    """out = warp + blend of (a, b) by (f_ab, f_ba) at the weight wa of A; gradients for all four."""

    @staticmethod
    def forward(ctx, a, b, f_ab, f_ba, wa, dev):
        _check(a, b, f_ab, f_ba)
        batch, w, h, fw, fh = _geometry(a, f_ab)
        out = torch.empty_like(a)
        dev.set_stream(torch.cuda.current_stream(a.device).cuda_stream)
        dev.warp_blend_adjoint(_ptr(a), _ptr(b), _ptr(f_ab), _ptr(f_ba), w, h, fw, fh, batch, wa, out=_ptr(out))
        ctx.save_for_backward(a, b, f_ab, f_ba)
        ctx.wa, ctx.dev = wa, dev
        return out

    @staticmethod
    def backward(ctx, grad_out):
        a, b, f_ab, f_ba = ctx.saved_tensors
        batch, w, h, fw, fh = _geometry(a, f_ab)
        g = grad_out.contiguous()
        need = ctx.needs_input_grad
        da = torch.zeros_like(a) if need[0] else None
        db = torch.zeros_like(b) if need[1] else None
        dfab = torch.zeros_like(f_ab) if need[2] else None
        dfba = torch.zeros_like(f_ba) if need[3] else None
        ctx.dev.set_stream(torch.cuda.current_stream(a.device).cuda_stream)
        ctx.dev.warp_blend_adjoint(_ptr(a), _ptr(b), _ptr(f_ab), _ptr(f_ba), w, h, fw, fh, batch, ctx.wa, grad_out=_ptr(g),
                                   da=_ptr(da), db=_ptr(db), df_ab=_ptr(dfab), df_ba=_ptr(dfba))
        return da, db, dfab, dfba, None, None


def warp_blend(a, b, f_ab, f_ba, wa, dev):
    return WarpBlend.apply(a, b, f_ab, f_ba, wa, dev)


def l1_loss_and_grads(dev, a, b, f_ab, f_ba, target, wa, frames_grad=True):
    """The fused path: per batch item sum |out - target| and the gradients of that loss w.r.t. the
    flows (and the frames), in one kernel launch without storing the forward output."""
    _check(a, b, f_ab, f_ba, target)
    batch, w, h, fw, fh = _geometry(a, f_ab)
    loss = torch.zeros(batch, dtype=torch.float32, device=a.device)
    dfab, dfba = torch.zeros_like(f_ab), torch.zeros_like(f_ba)
    da = torch.zeros_like(a) if frames_grad else None
    db = torch.zeros_like(b) if frames_grad else None
    dev.set_stream(torch.cuda.current_stream(a.device).cuda_stream)
    dev.warp_blend_adjoint(_ptr(a), _ptr(b), _ptr(f_ab), _ptr(f_ba), w, h, fw, fh, batch, wa, target=_ptr(target),
                           loss=_ptr(loss), da=_ptr(da), db=_ptr(db), df_ab=_ptr(dfab), df_ba=_ptr(dfba))
    return loss, da, db, dfab, dfba


def refine_flows(dev, a, b, f_ab, f_ba, target, wa, steps=50, lr=0.05):
    """Photometric refinement: ``steps`` Adam steps on the two flows (pixels of the flow grid) that
    lower the L1 loss of warp + blend against ``target``; the frames stay fixed. Returns the refined
    flows and the loss per step (batch sums)."""
    fab = f_ab.clone().requires_grad_(False)
    fba = f_ba.clone().requires_grad_(False)
    m = [torch.zeros_like(fab), torch.zeros_like(fba)]
    v = [torch.zeros_like(fab), torch.zeros_like(fba)]
    b1, b2, eps = 0.9, 0.999, 1e-8
    history = []
    for t in range(1, steps + 1):
        loss, _, _, g_ab, g_ba = l1_loss_and_grads(dev, a, b, fab, fba, target, wa, frames_grad=False)
        history.append(loss.sum().item())
        for k, (p, g) in enumerate(((fab, g_ab), (fba, g_ba))):
            m[k].mul_(b1).add_(g, alpha=1 - b1)
            v[k].mul_(b2).addcmul_(g, g, value=1 - b2)
            mh = m[k] / (1 - b1 ** t)
            vh = v[k] / (1 - b2 ** t)
            p.sub_(lr * mh / (vh.sqrt() + eps))
    return fab, fba, history
