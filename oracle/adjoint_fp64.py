"""Test infrastructure: the FP64 reference of warp + blend and of its adjoint, the checker of the
library's tw_warp_blend_adjoint (which has no counterpart in the reference; the forward model is
compose_vectors' Blend with warping code 0 made differentiable, warp.rs:693-786 / blend.rs:55-114).

Model, per output pixel p and channel c (w = 1 - wa):
    out = ta + (tb - ta) w,  ta = warp(A, F_BA, 1 - wa),  tb = warp(B, F_AB, wa)
    warp(S, F, s)(p) = bilinear(S, clamp(p + F(p r) s / r)),  F(q) bilinear at q = p r,
    r = (flow size - 1) / (image size - 1) per axis; a bilinear footprint whose cell starts at or
    beyond the last column (row) takes the cell before it with fraction 1; a clamped coordinate
    has no positional gradient.
Loss: the L1 sum |out - target| (gradient sign(out - target)) or a given output gradient.
Numpy, float64 throughout, scatters with np.add.at.
"""
import numpy as np


def _footprint(x, n):
    i = np.floor(x).astype(np.int64)
    f = x - i
    hi = i >= n - 1
    i = np.where(hi, n - 2, i)
    f = np.where(hi, 1.0, f)
    lo = i < 0
    i = np.where(lo, 0, i)
    f = np.where(lo, 0.0, f)
    return i, f


def _side(S, F, w, h, fw, fh, amount, pos32=False):
    """S: (h, w, 4), F: (fh, fw, 2) float64; the sample of S and what its gradient needs. With
    pos32 the sample positions (the flow's bilinear value and p + F (s / r)) are formed in single
    precision in the kernel's order, so that a position within rounding of a pixel boundary falls
    in the same bilinear cell as on the device; values and gradients stay double."""
    # the kernel forms r in single precision; keep the same values
    rx32, ry32 = np.float32(fw - 1) / np.float32(w - 1), np.float32(fh - 1) / np.float32(h - 1)
    rx, ry = float(rx32), float(ry32)
    dt = np.float32 if pos32 else np.float64
    Y, X = np.mgrid[0:h, 0:w].astype(dt)
    fix, ffx = _footprint(X * dt(rx32), fw)
    fiy, ffy = _footprint(Y * dt(ry32), fh)
    Fd = F.astype(dt)
    f00, f10 = Fd[fiy, fix], Fd[fiy, fix + 1]
    f01, f11 = Fd[fiy + 1, fix], Fd[fiy + 1, fix + 1]
    fxx, fyy = ffx[..., None].astype(dt), ffy[..., None].astype(dt)
    one = dt(1.0)
    uv = (f00 + (f10 - f00) * fxx) * (one - fyy) + (f01 + (f11 - f01) * fxx) * fyy
    # the step per flow unit, amount / r, formed once as warp.rs forms sx, sy (single precision)
    sx = dt(dt(amount) / dt(rx32)) if pos32 else amount / rx
    sy = dt(dt(amount) / dt(ry32)) if pos32 else amount / ry
    px = (X + uv[..., 0] * sx).astype(np.float64)
    py = (Y + uv[..., 1] * sy).astype(np.float64)
    ffx, ffy = ffx.astype(np.float64), ffy.astype(np.float64)
    cx = ~((px >= 0) & (px <= w - 1))
    cy = ~((py >= 0) & (py <= h - 1))
    px = np.clip(px, 0, w - 1)
    py = np.clip(py, 0, h - 1)
    ix, fx = _footprint(px, w)
    iy, fy = _footprint(py, h)
    c00, c10 = S[iy, ix], S[iy, ix + 1]
    c01, c11 = S[iy + 1, ix], S[iy + 1, ix + 1]
    fxc, fyc = fx[..., None], fy[..., None]
    val = (c00 + (c10 - c00) * fxc) * (1 - fyc) + (c01 + (c11 - c01) * fxc) * fyc
    return dict(val=val, ix=ix, iy=iy, fx=fx, fy=fy, cx=cx, cy=cy, c=(c00, c10, c01, c11), fix=fix, fiy=fiy, ffx=ffx,
                ffy=ffy, rx=rx, ry=ry)


def warp_blend(a, b, f_ab, f_ba, w, h, fw, fh, wa):
    """The forward output (h, w, 4) in float64 for one triple (arrays in the library's layouts)."""
    A, B = _img(a, w, h), _img(b, w, h)
    frac = 1.0 - float(np.float32(wa))
    sa = _side(A, _flow(f_ba, fw, fh), w, h, fw, fh, frac)
    sb = _side(B, _flow(f_ab, fw, fh), w, h, fw, fh, 1.0 - frac)
    return sa["val"] + (sb["val"] - sa["val"]) * frac


def _img(x, w, h):
    return np.asarray(x, np.float64).reshape(h, w, 4)


def _flow(x, fw, fh):
    return np.asarray(x, np.float64).reshape(fh, fw, 2)


def _back(s, g, dS, dF, amount, w, h, fw, fh):
    ix, iy, fx, fy = s["ix"], s["iy"], s["fx"], s["fy"]
    wts = ((1 - fx) * (1 - fy), fx * (1 - fy), (1 - fx) * fy, fx * fy)
    for (ox, oy), wt in zip(((0, 0), (1, 0), (0, 1), (1, 1)), wts):
        np.add.at(dS, (iy + oy, ix + ox), g * wt[..., None])
    c00, c10, c01, c11 = s["c"]
    fxc, fyc = fx[..., None], fy[..., None]
    dx = (c10 - c00) * (1 - fyc) + (c11 - c01) * fyc
    dy = (c01 - c00) * (1 - fxc) + (c11 - c10) * fxc
    gu = np.where(s["cx"], 0.0, (g * dx).sum(-1) * amount / s["rx"])
    gv = np.where(s["cy"], 0.0, (g * dy).sum(-1) * amount / s["ry"])
    fix, fiy, ffx, ffy = s["fix"], s["fiy"], s["ffx"], s["ffy"]
    fw_ = ((1 - ffx) * (1 - ffy), ffx * (1 - ffy), (1 - ffx) * ffy, ffx * ffy)
    for (ox, oy), wt in zip(((0, 0), (1, 0), (0, 1), (1, 1)), fw_):
        np.add.at(dF, (fiy + oy, fix + ox), np.stack([gu * wt, gv * wt], -1))


def warp_blend_grads(a, b, f_ab, f_ba, w, h, fw, fh, wa, target=None, grad_out=None, pos32=False):
    """(loss or None, out, da, db, df_ab, df_ba) in float64 for one triple (pos32: see _side)."""
    A, B = _img(a, w, h), _img(b, w, h)
    frac = float(np.float32(1.0) - np.float32(wa)) if pos32 else 1.0 - float(np.float32(wa))
    amount_b = float(np.float32(wa))
    sa = _side(A, _flow(f_ba, fw, fh), w, h, fw, fh, frac, pos32)
    sb = _side(B, _flow(f_ab, fw, fh), w, h, fw, fh, amount_b, pos32)
    out = sa["val"] + (sb["val"] - sa["val"]) * frac
    loss = None
    if target is not None:
        r = out - _img(target, w, h)
        loss = float(np.abs(r).sum())
        g = np.sign(r)
    else:
        g = _img(grad_out, w, h)
    da, db = np.zeros_like(A), np.zeros_like(B)
    df_ab, df_ba = np.zeros((fh, fw, 2)), np.zeros((fh, fw, 2))
    _back(sa, g * (1.0 - frac), da, df_ba, frac, w, h, fw, fh)
    _back(sb, g * frac, db, df_ab, amount_b, w, h, fw, fh)
    return loss, out, da, db, df_ab, df_ba
