"""Seeded synthetic clips standing in for the reference's `testsrc2` footage (which needs ffmpeg).

The clips have the shapes and motion of the benchmark configurations: a band limited value noise
background (lattice noise on three octaves, smoothly interpolated, rescaled to mean 128 / sd 40 on
an 8 bit scale) translated by a constant velocity, plus a checker textured square moving on its
own. Frames come out as wire frames (8 bpc RGBA interleaved, 16 bpc RGBA, or 32 bpc planar
G, B, R, A), ready for ``tw_retime_frame`` or the oracle.
"""
import numpy as np


def _lattice_noise(rng, w, h, cell):
    gw, gh = w // cell + 4, h // cell + 4
    return rng.standard_normal((gh, gw)).astype(np.float64), cell


def _sample(lat, cell, X, Y):
    # smooth (cubic Hermite) interpolation of the lattice at pixel coordinates; periodic lattice
    gh, gw = lat.shape
    fx, fy = X / cell, Y / cell
    ix, iy = np.floor(fx).astype(np.int64), np.floor(fy).astype(np.int64)
    tx, ty = fx - ix, fy - iy
    sx, sy = tx * tx * (3 - 2 * tx), ty * ty * (3 - 2 * ty)
    ix0, iy0 = ix % gw, iy % gh
    ix1, iy1 = (ix + 1) % gw, (iy + 1) % gh
    a = lat[iy0, ix0] * (1 - sx) + lat[iy0, ix1] * sx
    b = lat[iy1, ix0] * (1 - sx) + lat[iy1, ix1] * sx
    return a * (1 - sy) + b * sy


class NoiseField:
    """Three octaves of value noise; ``at(X, Y)`` gives values with mean 128, sd 40 (8 bit scale)."""

    def __init__(self, seed, w, h):
        rng = np.random.RandomState(seed)
        self.octaves = [(_lattice_noise(rng, w, h, c), a) for c, a in ((24, 1.0), (10, 0.55), (4, 0.3))]
        X, Y = np.meshgrid(np.arange(w, dtype=np.float64), np.arange(h, dtype=np.float64))
        v = self._raw(X, Y)
        self.mu, self.sd = float(v.mean()), float(v.std() or 1.0)

    def _raw(self, X, Y):
        v = 0.0
        for (lat, cell), amp in self.octaves:
            v = v + amp * _sample(lat, cell, X, Y)
        return v

    def at(self, X, Y):
        return 128.0 + 40.0 * (self._raw(X, Y) - self.mu) / self.sd


def _to_wire(rgb, alpha, depth):
    """rgb: (H, W, 3) floats on the 8 bit scale; alpha (H, W) in [0, 1]."""
    h, w = rgb.shape[:2]
    if depth == 8:
        px = np.empty((h, w, 4), np.uint8)
        px[..., :3] = np.clip(np.rint(rgb), 0, 255)
        px[..., 3] = np.clip(np.rint(alpha * 255.0), 0, 255)
        return px.reshape(-1)
    if depth == 16:
        px = np.empty((h, w, 4), np.uint16)
        px[..., :3] = np.clip(np.rint(rgb * 257.0), 0, 65535)
        px[..., 3] = np.clip(np.rint(alpha * 65535.0), 0, 65535)
        return px.reshape(-1)
    f = np.empty((4, h, w), np.float32)  # planes G, B, R, A
    f[0], f[1], f[2] = rgb[..., 1] / 255.0, rgb[..., 2] / 255.0, rgb[..., 0] / 255.0
    f[3] = alpha
    return f.reshape(-1)


def moving_clip(width, height, frames, depth=8, seed=0x74570001, bg_velocity=(1.5, -0.75), square=32,
                square_start=(20.0, 30.0), square_velocity=(2.0, 1.0), alpha=None, window=None):
    """A clip of ``frames`` wire frames back to back (one flat array): the noise background
    translated by ``bg_velocity`` px/frame and a ``square`` x ``square`` checker (8 px cells,
    values 40 / 215) moving by ``square_velocity``. ``alpha`` (optional callable (X, Y, t) -> [0,1])
    makes a straight alpha channel; opaque by default. ``window`` = (first, last): only the frames
    first..last of the clip (the same samples as in the whole clip), for a rank of a sharded render.

    The background is evaluated once over the area every frame's translation covers and each
    frame resamples it bilinearly at its sub-pixel offset."""
    noise = NoiseField(seed, width, height)
    vx, vy = bg_velocity
    span_x = abs(vx) * max(frames - 1, 0)
    span_y = abs(vy) * max(frames - 1, 0)
    ox = -(span_x if vx > 0 else 0.0) - 1.0
    oy = -(span_y if vy > 0 else 0.0) - 1.0
    bw, bh = int(np.ceil(width + span_x)) + 3, int(np.ceil(height + span_y)) + 3
    BX, BY = np.meshgrid(np.arange(bw, dtype=np.float64) + ox, np.arange(bh, dtype=np.float64) + oy)
    base = noise.at(BX, BY)
    X, Y = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64))
    out = []
    t_first, t_last = (0, frames - 1) if window is None else window
    for t in range(t_first, t_last + 1):
        # background value at (X - vx t, Y - vy t): position inside the base grid
        px, py = -vx * t - ox, -vy * t - oy
        ix, iy = int(np.floor(px)), int(np.floor(py))
        fx, fy = px - ix, py - iy
        b00 = base[iy:iy + height, ix:ix + width]
        b10 = base[iy:iy + height, ix + 1:ix + 1 + width]
        b01 = base[iy + 1:iy + 1 + height, ix:ix + width]
        b11 = base[iy + 1:iy + 1 + height, ix + 1:ix + 1 + width]
        g = (b00 * (1 - fx) + b10 * fx) * (1 - fy) + (b01 * (1 - fx) + b11 * fx) * fy
        rgb = np.stack([g, 0.85 * g + 20.0, 1.1 * g - 12.0], -1)
        sx, sy = square_start[0] + square_velocity[0] * t, square_start[1] + square_velocity[1] * t
        inside = (X >= sx) & (X < sx + square) & (Y >= sy) & (Y < sy + square)
        chk = ((np.floor((X - sx) / 8) + np.floor((Y - sy) / 8)) % 2 == 0)
        val = np.where(chk, 40.0, 215.0)
        rgb = np.where(inside[..., None], val[..., None], rgb)
        a = np.ones((height, width)) if alpha is None else alpha(X, Y, t)
        out.append(_to_wire(rgb, a, depth))
    return np.concatenate(out)


def _bilinear(img, X, Y):
    """Bilinear sample of a 2D array at float coordinates, clamped at the edges."""
    h, w = img.shape
    X = np.clip(X, 0.0, w - 1.001)
    Y = np.clip(Y, 0.0, h - 1.001)
    ix, iy = np.floor(X).astype(np.int64), np.floor(Y).astype(np.int64)
    fx, fy = X - ix, Y - iy
    a = img[iy, ix] * (1 - fx) + img[iy, ix + 1] * fx
    b = img[iy + 1, ix] * (1 - fx) + img[iy + 1, ix + 1] * fx
    return a * (1 - fy) + b * fy


def affine_clip(width, height, frames, depth=16, seed=0x74570002):
    """The Create Vectors workload: a seeded value noise texture (uniform octave amplitudes) under a
    random affine motion from each frame to the next (translation U[-16, 16] px, rotation U[-3, 3]
    degrees, scale U[0.97, 1.03] about the centre), opaque, as wire frames back to back."""
    rng = np.random.RandomState(seed)
    pad = 96
    tw_, th_ = width + 2 * pad, height + 2 * pad
    tex = 0.0
    for cell in (32, 12, 5):
        lat, c = _lattice_noise(rng, tw_, th_, cell)
        X, Y = np.meshgrid(np.arange(tw_, dtype=np.float64), np.arange(th_, dtype=np.float64))
        tex = tex + _sample(lat, c, X, Y)
    tex = 128.0 + 40.0 * (tex - tex.mean()) / (tex.std() or 1.0)
    X, Y = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64))
    cx, cy = width / 2.0, height / 2.0
    m = np.eye(3)  # the cumulative map from frame coordinates to texture coordinates
    out = []
    for t in range(frames):
        if t:
            ang = np.deg2rad(rng.uniform(-3.0, 3.0))
            s = rng.uniform(0.97, 1.03)
            tx, ty = rng.uniform(-16.0, 16.0, 2)
            c, sn = np.cos(ang) * s, np.sin(ang) * s
            step = np.array([[c, -sn, cx - c * cx + sn * cy + tx], [sn, c, cy - sn * cx - c * cy + ty], [0, 0, 1]])
            m = m @ step
        U = m[0, 0] * X + m[0, 1] * Y + m[0, 2] + pad
        V = m[1, 0] * X + m[1, 1] * Y + m[1, 2] + pad
        g = _bilinear(tex, U, V)
        rgb = np.stack([g, 0.9 * g + 12.0, 1.05 * g - 6.0], -1)
        out.append(_to_wire(rgb, np.ones((height, width)), depth))
    return np.concatenate(out)


def layered_clip(width, height, frames, nfg=3, depth=8, seed=0x74570004, bg_velocity=(3.0, 0.0)):
    """The retime-fgbg workload: a noise background translating by ``bg_velocity`` px/frame and ``nfg``
    textured ellipses (semi-axes 80 to 300 px) each moving on its own at up to 12 px/frame, FG1 on
    top. Returns (footage, [matte clips]): each matte clip holds its layer's binary ellipse in the
    red channel (the FG matte channel popup's default), white elsewhere in alpha."""
    rng = np.random.RandomState(seed)
    base = moving_clip(width, height, frames, depth=8, seed=seed, bg_velocity=bg_velocity, square=0)
    base = base.reshape(frames, height, width, 4).astype(np.float64)
    X, Y = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64))
    layers = []
    for k in range(nfg):
        ax, ay = rng.uniform(80.0, 300.0, 2) * min(1.0, width / 1920.0)
        cx, cy = rng.uniform(0.25, 0.75) * width, rng.uniform(0.25, 0.75) * height
        speed, ang = rng.uniform(4.0, 12.0), rng.uniform(0, 2 * np.pi)
        vx, vy = speed * np.cos(ang), speed * np.sin(ang)
        tex = NoiseField(seed + 17 * (k + 1), width, height)
        layers.append((ax, ay, cx, cy, vx, vy, tex, 60.0 + 50.0 * k))
    foot, mattes = [], [[] for _ in range(nfg)]
    for t in range(frames):
        rgb = base[t, ..., :3].copy()
        for k in reversed(range(nfg)):  # bottom layer first, FG1 last (on top)
            ax, ay, cx, cy, vx, vy, tex, tint = layers[k]
            px, py = cx + vx * t, cy + vy * t
            inside = ((X - px) / ax) ** 2 + ((Y - py) / ay) ** 2 <= 1.0
            g = tex.at(X - vx * t, Y - vy * t)
            fg = np.stack([g, 0.5 * g + tint, 0.8 * g + 30.0], -1)
            rgb = np.where(inside[..., None], fg, rgb)
            m = np.zeros((height, width, 3))
            m[..., 0] = inside * 255.0
            mattes[k].append(_to_wire(m, np.ones((height, width)), depth))
        foot.append(_to_wire(rgb, np.ones((height, width)), depth))
    return np.concatenate(foot), [np.concatenate(m) for m in mattes]


def adjoint_triples(width, height, batch, seed=0x74570005, peak=10.0):
    """The warp + blend adjoint workload: per batch item a seeded value noise texture T (float RGBA
    in [0, 1], alpha 1) and a smooth ground truth displacement D, the sum of four random Gaussian
    bumps with a peak of ``peak`` px; the middle frame is T, A samples T at p - D(p) / 2 and B at
    p + D(p) / 2. Returns (A, B, M, D) as float32 arrays (batch, height, width, 4) and
    (batch, height, width, 2)."""
    rng = np.random.RandomState(seed)
    Y, X = np.mgrid[0:height, 0:width].astype(np.float64)
    As, Bs, Ms, Ds = [], [], [], []
    for _ in range(batch):
        pad = int(peak) + 4
        tex = NoiseField(int(rng.randint(1 << 30)), width + 2 * pad, height + 2 * pad)
        D = np.zeros((height, width, 2))
        for _ in range(4):
            cx, cy = rng.uniform(0, width), rng.uniform(0, height)
            sg = rng.uniform(0.12, 0.3) * min(width, height)
            amp = rng.uniform(-1.0, 1.0, 2)
            g = np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * sg * sg))
            D += g[..., None] * amp
        D *= peak / max(np.abs(D).max(), 1e-9)

        def frame(dx, dy):
            g = tex.at(X + dx + pad, Y + dy + pad) / 255.0
            rgb = np.stack([g, 0.8 * g + 0.1, 1.0 - 0.7 * g], -1)
            return np.concatenate([rgb, np.ones((height, width, 1))], -1).clip(0, 1)

        Ms.append(frame(0.0, 0.0))
        As.append(frame(-0.5 * D[..., 0], -0.5 * D[..., 1]))
        Bs.append(frame(0.5 * D[..., 0], 0.5 * D[..., 1]))
        Ds.append(D)
    f = lambda v: np.ascontiguousarray(np.stack(v), np.float32)  # noqa: E731
    return f(As), f(Bs), f(Ms), f(Ds)


def batch_clip_gpu(width, height, frames, seed, device="cuda:0"):
    """The batched retime workload, generated on the GPU with torch: float RGBA in [0, 1] as wire
    frames (planes G, B, R, A), a seeded value noise background moving at a random velocity and 3
    to 8 textured ellipses, each moving at up to 24 px/frame (the textures wrap around). Returns a
    flat float32 tensor of ``frames`` wire frames back to back."""
    import torch
    import torch.nn.functional as F
    g = torch.Generator(device="cpu").manual_seed(seed)

    def noise(cell):
        lat = torch.rand((1, 1, height // cell + 4, width // cell + 4), generator=g)
        return F.interpolate(lat.to(device), size=(height, width), mode="bicubic", align_corners=False)[0, 0]

    bg = 0.6 * noise(48) + 0.4 * noise(12)
    bg = ((bg - bg.mean()) / bg.std() * 0.18 + 0.5).clamp(0, 1)
    vb = (torch.rand(2, generator=g) * 2 - 1) * 6.0
    n_ell = int(torch.randint(3, 9, (1,), generator=g))
    ells = []
    for _ in range(n_ell):
        ax, ay = (torch.rand(2, generator=g) * 0.2 + 0.06) * min(width, height)
        cx, cy = torch.rand(1, generator=g) * width, torch.rand(1, generator=g) * height
        ang = torch.rand(1, generator=g) * 6.2832
        sp = torch.rand(1, generator=g) * 24.0
        ells.append((float(ax), float(ay), float(cx), float(cy), float(sp * torch.cos(ang)), float(sp * torch.sin(ang)),
                     noise(8).clamp(0, 1)))
    Y, X = torch.meshgrid(torch.arange(height, device=device, dtype=torch.float32),
                          torch.arange(width, device=device, dtype=torch.float32), indexing="ij")
    out = torch.empty((frames, 4, height, width), device=device, dtype=torch.float32)
    for t in range(frames):
        lum = torch.roll(bg, shifts=(int(round(float(vb[1]) * t)), int(round(float(vb[0]) * t))), dims=(0, 1))
        r, gg, b = lum, 0.85 * lum + 0.08, (1.0 - 0.6 * lum)
        for ax, ay, cx, cy, vx, vy, tex in ells:
            px, py = cx + vx * t, cy + vy * t
            m = ((X - px) / ax) ** 2 + ((Y - py) / ay) ** 2 <= 1.0
            tl = torch.roll(tex, shifts=(int(round(vy * t)), int(round(vx * t))), dims=(0, 1))
            r, gg, b = torch.where(m, tl, r), torch.where(m, 0.5 * tl + 0.3, gg), torch.where(m, 1.0 - tl, b)
        out[t, 0], out[t, 1], out[t, 2], out[t, 3] = gg, b, r, 1.0  # wire planes G, B, R, A
    return out.reshape(-1)


def vector_clip(width, height, frames, velocity, depth=8, max_displace=32.0, sign=1.0, seed=0x74570006, holes=12,
                hole_radius=40.0):
    """A vector layer of ``frames`` wire frames the way the Vectors In effect reads them: every pixel
    the displacement ``sign * velocity`` (plus a slow spatial ripple of a tenth of a pixel) encoded
    against ``max_displace`` (8 bpc R = (u / md + 1) * 127, 16 bpc with 32767, float (u / md + 1) / 2;
    G likewise; B 0), alpha opaque except ``holes`` discs of alpha 0 per frame (the holes the
    effect's flow fill closes)."""
    rng = np.random.RandomState(seed)
    Y, X = np.mgrid[0:height, 0:width].astype(np.float64)
    out = []
    for t in range(frames):
        u = sign * velocity[0] + 0.1 * np.sin(X / 97.0 + t)
        v = sign * velocity[1] + 0.1 * np.cos(Y / 61.0 - t)
        a = np.ones((height, width))
        for _ in range(holes):
            cx, cy = rng.uniform(0, width), rng.uniform(0, height)
            a[(X - cx) ** 2 + (Y - cy) ** 2 < hole_radius ** 2] = 0.0
        if depth == 8:
            r = np.clip(np.floor((u / max_displace + 1.0) * 127.0 + 0.5), 0, 254)
            g = np.clip(np.floor((v / max_displace + 1.0) * 127.0 + 0.5), 0, 254)
            out.append(np.stack([r, g, np.zeros_like(r), a * 255], -1).astype(np.uint8).reshape(-1))
        elif depth == 16:
            r = np.clip(np.floor((u / max_displace + 1.0) * 32767.0 + 0.5), 0, 65534)
            g = np.clip(np.floor((v / max_displace + 1.0) * 32767.0 + 0.5), 0, 65534)
            out.append(np.stack([r, g, np.zeros_like(r), a * 65535], -1).astype(np.uint16).reshape(-1))
        else:
            r = ((u / max_displace + 1.0) / 2.0).astype(np.float32)
            g = ((v / max_displace + 1.0) / 2.0).astype(np.float32)
            out.append(np.concatenate([g.reshape(-1), np.zeros(width * height, np.float32), r.reshape(-1),
                                       a.astype(np.float32).reshape(-1)]))
    return np.concatenate(out)
