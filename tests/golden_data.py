"""Readers of the committed golden fixtures (see tests/golden/make_golden.py)."""
import fractions
import gzip
import json
import os
import struct

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DT = {0: np.uint8, 1: np.uint16, 2: np.float32}
FMT_OF_DEPTH = {8: 0, 16: 1, 32: 2}


def grid():
    """(meta cases, {input name: raw bytes as uint8})."""
    z = np.load(os.path.join(GOLDEN, "retime_flow_grid.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    inputs = {name: z[f"input_{i}"] for i, name in enumerate(meta["inputs"])}
    return meta["cases"], inputs


# Served grid cases whose recorded output the restatement does not reproduce yet: Weighted Blend of
# float frames full of NaNs and infinities (the sharpening of the non finite samples).
KNOWN_GAPS = {
    "retime.spec-all-i3-sb0.spec-all-24x24.d32.ff54dfb4",
    "retime.spec-all-i3-sb1.spec-all-24x24.d32.20e9a0b7",
}


def grid_params(cases):
    """pytest parameters of grid cases, the known gaps marked as strict expected failures."""
    import pytest
    return [pytest.param(c, id=c["id"], marks=pytest.mark.xfail(strict=True, reason="known gap: non finite Weighted Blend"))
            if c["id"] in KNOWN_GAPS else pytest.param(c, id=c["id"]) for c in cases]


# Served create-vectors grid cases of the Debug display whose views (Blend, Diff, Detail, Edge) the
# recorded revision computed with the rules of the reference's numpy model, which predate the rules
# it now follows (read from the original: debug.rs:1-47); its Warp view cases pass.
CV_KNOWN_GAPS = {
    "create-vectors.debug-edge.multi-48x32.d16.3e7cd22e",
    "create-vectors.debug-m2-tf1.disc-16x12.d16.c9272ce2",
    "create-vectors.debug-m2-tf1.disc-16x12.d32.e7374780",
    "create-vectors.debug-m2-tf1.disc-16x12.d8.26c6e7c7",
    "create-vectors.debug-m2-tf2.disc-16x12.d16.655868a1",
    "create-vectors.debug-m2-tf2.disc-16x12.d32.747f4bfc",
    "create-vectors.debug-m2-tf2.disc-16x12.d8.f47a92a8",
    "create-vectors.debug-m3-tf1.disc-16x12.d16.7634a431",
    "create-vectors.debug-m3-tf1.disc-16x12.d32.eb974210",
    "create-vectors.debug-m3-tf1.disc-16x12.d8.69b3d5bc",
    "create-vectors.debug-m3-tf2.disc-16x12.d16.a9b44b89",
    "create-vectors.debug-m3-tf2.disc-16x12.d32.1fcd5d8c",
    "create-vectors.debug-m3-tf2.disc-16x12.d8.39b40b82",
    "create-vectors.debug-m4-tf1.disc-16x12.d16.a596461d",
    "create-vectors.debug-m4-tf1.disc-16x12.d32.ed6a6398",
    "create-vectors.debug-m4-tf1.disc-16x12.d8.8c7fe7e6",
    "create-vectors.debug-m4-tf2.disc-16x12.d16.02548d40",
    "create-vectors.debug-m4-tf2.disc-16x12.d32.12750e18",
    "create-vectors.debug-m4-tf2.disc-16x12.d8.abc37fe3",
    "create-vectors.debug-m5-tf1.disc-16x12.d16.52ff3824",
    "create-vectors.debug-m5-tf1.disc-16x12.d32.53006737",
    "create-vectors.debug-m5-tf1.disc-16x12.d8.48820edb",
    "create-vectors.debug-m5-tf2.disc-16x12.d16.1f4a4a40",
    "create-vectors.debug-m5-tf2.disc-16x12.d32.99f00b21",
    "create-vectors.debug-m5-tf2.disc-16x12.d8.c43cd73e",
    "create-vectors.extreme-dbg.checker-8x6.d16.f40e6f0d",
    "create-vectors.extreme-dbg.checker-8x6.d8.8eb11267",
    "create-vectors.extreme-dbg.white-8x6.d8.238c071a",
    "create-vectors.hdr-debug-diff.hdr-16x12.d32.5decef94",
    "create-vectors.hdr-debug.hdr-16x12.d32.ee0497b1",
    "create-vectors.mix-dbg.specmix-6x4.d32.20503049",
    "create-vectors.mix-dbg.specmix-6x4.d32.4d226157",
    "create-vectors.mix-dbg.specmix-6x4.d32.e7ab55b9",
    "create-vectors.patch-denorm-md1.spp_denorm_min-8x6.d32.2ca98cec",
    "create-vectors.patch-inf-dbg.spp_inf-8x6.d32.72df2219",
    "create-vectors.patch-nan-dbg.spp_nan-8x6.d32.6e58c2ad",
    "create-vectors.tiny-debug.shift-3x3.d16.e0614b79",
}


def cv_grid_params(cases):
    """pytest parameters of create-vectors grid cases, the known gaps marked as strict expected failures."""
    import pytest
    return [pytest.param(c, id=c["id"], marks=pytest.mark.xfail(strict=True, reason="Debug views of the recorded revision"))
            if c["id"] in CV_KNOWN_GAPS else pytest.param(c, id=c["id"]) for c in cases]


def cv_grid():
    """The served cases of the create-vectors parity grid: (meta cases, {input name: raw bytes})."""
    z = np.load(os.path.join(GOLDEN, "create_vectors_grid.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    inputs = {name: z[f"input_{i}"] for i, name in enumerate(meta["inputs"])}
    return meta["cases"], inputs


def crt_powf_traced():
    """(x, y, powf(x, y)) bit patterns traced from the plugin's C runtime."""
    with open(os.path.join(GOLDEN, "crt_powf_traced.json")) as f:
        return json.load(f)


def fgbg_grid():
    """The served cases of the fgbg-layers parity grid: (meta cases, {clip name: raw bytes})."""
    z = np.load(os.path.join(GOLDEN, "fgbg_layers_grid.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    inputs = {name: z[f"input_{i}"] for i, name in enumerate(meta["inputs"])}
    return meta["cases"], inputs


def _fixed_reader(v):
    """A value through 16.16 fixed point and back (crates/fx-core/src/fixed.rs, frontend.rs:131-133)."""
    f = v * 65536.0 + (-0.5 if v < 0 else 0.5)
    fixed = 0 if np.isnan(f) else int(np.clip(np.trunc(f), -2 ** 31, 2 ** 31 - 1))
    return np.float32(np.float64(fixed) * (1.0 / 65536.0))


def _eased(u, ease_start, ease_end):
    """crates/fx-core/src/curves.rs:537-544 (eased_progress)."""
    if ease_start and ease_end:
        return u * u * (3.0 - 2.0 * u)
    if ease_start:
        return u * u * (2.0 - u)
    if ease_end:
        return u * (1.0 + u * (1.0 - u))
    return u


def param_at(text, ticks, kind, default, ticks_per_frame=100):
    """A keyed CLI value ``V@F[h|e];...`` at ``ticks`` (crates/fx-core/src/curves.rs:79-110 and
    348-375): before the first key its value, after the last its value, between two keys the
    first one's value for a hold key or a popup, else the linear (or eased) mix in f64; a point
    moves on the straight line. Keys without handles only. ``kind``: "int" or "point"."""
    def parse(v):
        return int(v) if kind == "int" else [float(x) for x in v.split(",")]
    if text is None:
        return default
    if "@" not in text:
        return parse(text)
    keys = []
    for piece in text.split(";"):
        v, f = piece.rsplit("@", 1)
        hold, ease = f.endswith("h"), f.endswith("e")
        f = f[:-1] if hold or ease else f
        keys.append((int(round(float(f) * ticks_per_frame)), parse(v), hold, ease))
    if ticks <= keys[0][0]:
        return keys[0][1]
    if ticks >= keys[-1][0]:
        return keys[-1][1]
    i = max(j for j, k in enumerate(keys) if k[0] <= ticks)
    a, b = keys[i], keys[i + 1]
    if a[2] or kind == "int":
        return a[1]
    u = _eased((ticks - a[0]) / (b[0] - a[0]), a[3], b[3])
    return [x + (y - x) * u for x, y in zip(a[1], b[1])]


def fgbg_points(case, a, b, nfg, npoints=12):
    """The tracking points of a retime-fgbg grid case for the pair of source frames a, b
    (plugins/retime-fgbg/src/glue.rs:196-211 user_points, 124-133 points_in_use): every point whose
    Use popup is not Don't Use at the layer time T(a) and equal at T(b) (T(f) = trunc(100 f + 0.5),
    integer frame rates) goes to the layer points.rs:64-70 (point_layer) names, its position read
    at both times through the 16.16 reader (points.rs:77-80). One list per layer, Main_BG last, of
    (x, y at A, x, y at B) in output pixels (host rows)."""
    p = dict(x.split("=", 1) for x in case["params"])
    ta, tb = int(100.0 * float(np.float32(a)) + 0.5), int(100.0 * float(np.float32(b)) + 0.5)
    out = [[] for _ in range(nfg + 1)]
    for n in range(1, npoints + 1):
        use = p.get(f"pt{n}_use")
        v1 = param_at(use, ta, "int", 1)
        if v1 == 1 or param_at(use, tb, "int", 1) != v1 or v1 < 2:
            continue
        k = min(v1 - 2, nfg)
        pos = p.get(f"pt{n}_pos")
        pa, pb = param_at(pos, ta, "point", [-5.0, -5.0]), param_at(pos, tb, "point", [-5.0, -5.0])
        out[k].append((float(_fixed_reader(pa[0])), float(_fixed_reader(pa[1])), float(_fixed_reader(pb[0])),
                       float(_fixed_reader(pb[1]))))
    return out


def cv_points(case, n):
    """The tracking points of output frame n of a create-vectors grid case (one layer:
    plugins/create-vectors/src/glue.rs:278-291 layer_points at the layer times of the pair, integer
    frame rates: X = frame n, Y = n - 1 (Track Previous) or n + 1 (Next), T(f) = 100 f)."""
    p = dict(x.split("=", 1) for x in case["params"])
    b = n - 1 if int(p.get("track_frame", 1)) == 1 else n + 1
    return fgbg_points(case, n, b, 0)[0]


def fgbg_case_params(case):
    """The parameters of a fgbg-layers grid case (plugin defaults where the case sets none): the
    retime selection and Main_BG settings (``smart_blend`` carries the warping code, the Warping
    popup minus one, glue.rs:94-100), the Display popup, and per FG layer its channel popup,
    sensitivity and inverse matte shrink."""
    p = dict(x.split("=", 1) for x in case["params"])
    nfg = len(case["mattes"])
    mark_keys, marks = parse_keys(p.get("src_mark_segments", "1"))
    return dict(fps=(int(case["fps"]), 1), speed=float(p.get("speed_percent", 100)), vectors=int(p.get("vectors", 5)),
                mark_segs=1 if mark_keys else int(marks), mark_keys=[(f, v) for f, v, _ in mark_keys] if mark_keys else None,
                frame_interp=int(p.get("frame_interp", 2)), smart_blend=int(p.get("warping", "1")) - 1,
                blur=float(p.get("blur_compensation", 0)),
                sensitivity=float(p.get("main_bg_sensitivity", 70)),
                chans=[int(p.get(f"fg{k + 1}_matte_chan", 1)) for k in range(nfg)],
                fg_sens=[float(p.get(f"fg{k + 1}_sensitivity", 70)) for k in range(nfg)],
                shrinks=[float(p.get(f"fg{k + 1}_inv_matte_shrink", 0)) for k in range(nfg)],
                display=int(p.get("display", 1)), track_rgb_a=p.get("track_rgb_a", "0") == "1")


def cv_case_params(case):
    """The parameter values of a create-vectors grid case (plugin defaults where the case sets none)."""
    p = dict(x.split("=", 1) for x in case["params"])
    fps = fractions.Fraction(case["fps"])
    return dict(fps=(fps.numerator, fps.denominator), vector_resolution=int(p.get("vector_resolution", 1)),
                max_displace=float(p.get("max_displace", 2048)), track_frame=int(p.get("track_frame", 1)),
                sensitivity=float(p.get("main_bg_sensitivity", 70)),
                track_rgb_a=p.get("track_rgb_a", "0") in ("1", "true", "True"), prep=int(p.get("prep", 1)),
                display=int(p.get("display", 2)), debug_view_method=int(p.get("debug_view_method", 1)))


def case_params(case):
    """Keyword arguments of oracle_lib.retime_params for a grid case (grid variant of the orders)."""
    params = dict(p.split("=", 1) for p in case["params"])
    sp = params.pop("speed_percent")
    keys, speed = None, 100.0
    if "@" in sp:
        keys = []
        for k in sp.split(";"):
            v, f = k.split("@")
            keys.append((float(f.rstrip("e")), float(v), f.endswith("e")))
    else:
        speed = float(sp)
    fps = case["fps"]
    fpsp = tuple(int(x) for x in fps.split("/")) if "/" in fps else (int(fps), 1)
    return dict(fps=fpsp, speed=speed, keys=keys, vectors=int(params.get("vectors", 5)),
                frame_interp=int(params.get("frame_interp", 2)), sensitivity=float(params.get("sensitivity", 70)),
                blur=float(params.get("blur_compensation", 0)), smart_blend=int(params.get("smart_blend", 0)),
                video_360=params.get("video_360", "0") == "1", rows_reversed=False, taps_above_first=False,
                prep=int(params.get("prep", 1)))


def f2_cases():
    """The reference's numpy model of the textured forward warp (f2_cases.hex; format in its f2_gen.py)."""
    blob = gzip.open(os.path.join(GOLDEN, "f2_cases.bin.gz")).read()
    assert blob[:4] == b"F2C1"
    n = struct.unpack_from("<I", blob, 4)[0]
    p = 8
    out = []
    for _ in range(n):
        fmt, w, h, fw, fh = struct.unpack_from("<5I", blob, p)
        amount = np.float32(struct.unpack_from("<f", blob, p + 20)[0])
        p += 28
        dt = {0: np.uint8, 1: np.uint16, 2: np.float32}[fmt]
        cnt = w * h * 4 * np.dtype(dt).itemsize
        src = np.frombuffer(blob[p:p + cnt], dt).copy()
        p += cnt
        flow = np.frombuffer(blob[p:p + fw * fh * 8], np.float32).copy()
        p += fw * fh * 8
        want = np.frombuffer(blob[p:p + cnt], dt).copy()
        p += cnt
        cov = np.frombuffer(blob[p:p + w * h], np.uint8).copy()
        p += w * h
        out.append(dict(fmt=fmt, w=w, h=h, fw=fw, fh=fh, amount=amount, src=src, flow=flow, out=want, cov=cov))
    assert p == len(blob)
    return out


def mask_cases():
    """The reference's models of the layered solve's hooks (mask_cases.hex; format in its gen_mask.py):
    dicts with kind 1 (mask pyramid), 2 (gradient masking), 3 (B step), 4 (block matching)."""
    blob = gzip.open(os.path.join(GOLDEN, "mask_cases.bin.gz")).read()
    assert blob[:4] == b"MSK1"
    p = 8
    n = struct.unpack_from("<I", blob, 4)[0]

    def u32():
        nonlocal p
        v = struct.unpack_from("<I", blob, p)[0]
        p += 4
        return v

    def f32s(k):
        nonlocal p
        v = np.frombuffer(blob[p:p + 4 * k], np.float32).copy()
        p += 4 * k
        return v

    out = []
    for _ in range(n):
        kind = u32()
        if kind == 1:
            w, h, q, hiq = u32(), u32(), u32(), u32()
            matte = f32s(w * h)
            levels = []
            for _ in range(u32()):
                lw, lh = u32(), u32()
                levels.append((lw, lh, f32s(lw * lh)))
            out.append(dict(kind=1, w=w, h=h, quality=q, hiq=hiq, matte=matte, levels=levels))
        elif kind == 2:
            w, h, wrap, has = u32(), u32(), u32(), u32()
            img = f32s(w * h)
            mask = f32s(w * h) if has else None
            out.append(dict(kind=2, w=w, h=h, wrap=wrap, img=img, mask=mask, want=f32s(w * h * 2)))
        elif kind == 3:
            w, h, wrap, has = u32(), u32(), u32(), u32()
            i1, i0, grad, flow = f32s(w * h), f32s(w * h), f32s(w * h * 2), f32s(w * h * 2)
            mask = f32s(w * h) if has else None
            out.append(dict(kind=3, w=w, h=h, wrap=wrap, i1=i1, i0=i0, grad=grad, flow=flow, mask=mask,
                            want=f32s(w * h * 2)))
        elif kind == 4:
            w, h, wrap, has = u32(), u32(), u32(), u32()
            a, b, flow = f32s(w * h), f32s(w * h), f32s(w * h * 2)
            gate = f32s(w * h) if has else None
            out.append(dict(kind=4, w=w, h=h, wrap=wrap, a=a, b=b, flow=flow, gate=gate, want=f32s(w * h * 2)))
        else:
            raise ValueError(kind)
    assert p == len(blob)
    return out


def f1_cases():
    """The reference's Smart Blend and hole fill model fixtures (f1_cases.hex; format in its f1_gen.py)."""
    blob = gzip.open(os.path.join(GOLDEN, "f1_cases.bin.gz")).read()
    assert blob[:4] == b"F1C1"
    n = struct.unpack_from("<I", blob, 4)[0]
    p = 8
    out = []
    for _ in range(n):
        kind, depth, w, h = struct.unpack_from("<IIII", blob, p)
        weight = np.float32(struct.unpack_from("<f", blob, p + 16)[0])
        mask_kind = struct.unpack_from("<I", blob, p + 20)[0]
        p += 24
        dt = DT[depth]
        cnt = w * h * 4 * np.dtype(dt).itemsize

        def img():
            nonlocal p
            v = np.frombuffer(blob[p:p + cnt], dt).copy()
            p += cnt
            return v

        p1 = img()
        p2 = mask = None
        if kind == 3:
            msz = {1: 1, 2: 2}.get(mask_kind, 4)
            mask = np.frombuffer(blob[p:p + w * h * msz], {1: np.uint8, 2: np.uint16}.get(mask_kind, np.float32)).copy()
            p += w * h * msz
        else:
            p2 = img()
        exp = img()
        out.append(dict(kind=kind, fmt=depth, w=w, h=h, weight=weight, mask_kind=mask_kind, p1=p1, p2=p2, mask=mask,
                        out=exp))
    assert p == len(blob)
    return out


def blur_cases():
    """The reference's motion blur model fixtures (blur_cases.hex; format in its gen_blur.py): dicts of
    depth, size, flow, amount, shutter, hiq, source and expected output."""
    blob = gzip.open(os.path.join(GOLDEN, "blur_cases.bin.gz")).read()
    assert blob[:4] == b"BLR1"
    n = struct.unpack_from("<I", blob, 4)[0]
    p = 8
    out = []
    for _ in range(n):
        depth, w, h, fw, fh = struct.unpack_from("<IIIII", blob, p)
        amount, shutter = (np.float32(v) for v in struct.unpack_from("<ff", blob, p + 20))
        hiq = struct.unpack_from("<I", blob, p + 28)[0] != 0
        p += 32
        dt = DT[depth]
        cnt = w * h * 4 * np.dtype(dt).itemsize
        src = np.frombuffer(blob[p:p + cnt], dt).copy()
        p += cnt
        flow = np.frombuffer(blob[p:p + fw * fh * 8], np.float32).copy()
        p += fw * fh * 8
        want = np.frombuffer(blob[p:p + cnt], dt).copy()
        p += cnt
        out.append(dict(fmt=depth, w=w, h=h, fw=fw, fh=fh, amount=amount, shutter=shutter, hiq=hiq, src=src, flow=flow,
                        out=want))
    assert p == len(blob)
    return out


def warp_cases():
    """The reference's inverse warp fixtures: list of dicts (src, flow, expected out and coverage)."""
    blob = gzip.open(os.path.join(GOLDEN, "warp_cases.bin.gz")).read()
    assert blob[:4] == b"WRP1"
    p = 4

    def u32():
        nonlocal p
        v = struct.unpack_from("<I", blob, p)[0]
        p += 4
        return v

    def f32():
        nonlocal p
        v = struct.unpack_from("<f", blob, p)[0]
        p += 4
        return np.float32(v)

    def take(n):
        nonlocal p
        v = blob[p:p + n]
        p += n
        return v

    out = []
    for _ in range(u32()):
        depth = u32()
        w, h, fw, fh = u32(), u32(), u32(), u32()
        amount = f32()
        flags = u32()
        dt = DT[depth]
        es = np.dtype(dt).itemsize
        src = np.frombuffer(take(w * h * 4 * es), dt).copy()
        flow = np.frombuffer(take(fw * fh * 8), np.float32).copy()
        exp = np.frombuffer(take(w * h * 4 * es), dt).copy()
        cov = np.frombuffer(take(w * h), np.uint8).copy() if flags & 4 else None
        out.append(dict(fmt=depth, w=w, h=h, fw=fw, fh=fh, amount=amount, hold=bool(flags & 1),
                        is360=bool(flags & 2), want_cov=bool(flags & 4), src=src, flow=flow, out=exp, cov=cov))
    assert p == len(blob)
    return out


FLOW_MODEL_TOL = {"a": 1e-4, "b": 1e-4, "c": 1e-4, "d": 1e-4, "e": 1e-3, "f": 1e-3}  # flow_d.rs:231-236


def flow_models():
    """The reference's differential fixtures of the solver (flow_{a..f}.hex, its float32 numpy model
    without block matching, flow_ref.py): list of dicts with the engine images x and y (8 bit A, R,
    G, B), the settings and the model's flow; the reference accepts FLOW_MODEL_TOL."""
    blob = gzip.open(os.path.join(GOLDEN, "flow_models.bin.gz")).read()
    p, out = 0, []
    for name in "abcdef":
        n = struct.unpack_from("<I", blob, p)[0]
        b = blob[p + 4:p + 4 + n]
        p += 4 + n
        magic, w, h, sens, quality, prep = struct.unpack_from("<IIIfII", b, 0)
        assert magic == 0x32444C46
        o = 24
        x = np.frombuffer(b, np.uint8, w * h * 4, o).copy()
        y = np.frombuffer(b, np.uint8, w * h * 4, o + w * h * 4).copy()
        r = 1 if quality == 4 else 0
        fw, fh = w >> r, h >> r
        flow = np.frombuffer(b, "<f4", fw * fh * 2, o + 2 * w * h * 4).astype(np.float32)
        out.append(dict(name=name, w=w, h=h, sens=np.float32(sens), quality=quality, prep=prep, x=x, y=y,
                        flow=flow, tol=FLOW_MODEL_TOL[name]))
    return out


def vi_grid():
    """The served cases of the vectors-in parity grid: (meta cases, {clip name: raw bytes})."""
    z = np.load(os.path.join(GOLDEN, "vectors_in_grid.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    inputs = {name: z[f"input_{i}"] for i, name in enumerate(meta["inputs"])}
    return meta["cases"], inputs


def vi_case_params(case):
    """Keyword arguments of oracle_lib.vecin_params for a vectors-in grid case (the effect's
    defaults where the case sets none: Speed 100, Max Displace 2048, Blend, Forward, scale 1)."""
    p = dict(x.split("=", 1) for x in case["params"])
    keys, speed = parse_keys(p.get("speed_percent", "100"))
    fn_keys, fnum = parse_keys(p.get("frame_num", "0"))
    fps = fractions.Fraction(case["fps"])
    mark_keys, marks = parse_keys(p.get("src_mark_segments", "1"))
    return dict(fps=(fps.numerator, fps.denominator), speed=speed, keys=keys, remap_mode=int(p.get("time_remap_mode", 1)),
                mark_segs=1 if mark_keys else int(marks), mark_keys=[(f, v) for f, v, _ in mark_keys] if mark_keys else None,
                frame_num=fnum, fn_keys=fn_keys, own_input_rate=p.get("in_fps_is_out_fps", "1") == "0",
                input_frame_rate=float(p.get("input_frame_rate", float(np.float32(29.97)))),
                frame_interp=int(p.get("frame_interp", 2)), warping=int(p.get("warping", 2)),
                blur=float(p.get("blur_compensation", 0)), max_displace=float(p.get("vectors_max_displace", 2048)),
                vec_scale=(float(p.get("vec_scale_x", 1)), float(p.get("vec_scale_y", 1))))


def vectors_cases():
    """The reference's numpy model of the vector encode and decode (vectors_cases.hex, its
    gen_vectors.py): b"VEC1", u32 count, then per case u32 kind (0 encode, 1 decode), depth (0 u8,
    1 u16, 2 f32), W, H,
    FW, FH, f32 scale; a decode case holds the W x H engine image (A, R, G, B samples of the depth)
    and the decoded W x H flow; an encode case the FW x FH flow and the encoded W x H image."""
    blob = gzip.open(os.path.join(GOLDEN, "vectors_cases.bin.gz")).read()
    assert blob[:4] == b"VEC1"
    n = struct.unpack_from("<I", blob, 4)[0]
    p, out = 8, []
    dt = {0: np.dtype("u1"), 1: np.dtype("<u2"), 2: np.dtype("<f4")}
    for _ in range(n):
        kind, depth, w, h, fw, fh = struct.unpack_from("<6I", blob, p)
        scale = struct.unpack_from("<f", blob, p + 24)[0]
        p += 28
        d = dt[depth]
        if kind == 1:
            img = np.frombuffer(blob, d, w * h * 4, p).copy()
            p += w * h * 4 * d.itemsize
            flow = np.frombuffer(blob, "<f4", w * h * 2, p).astype(np.float32)
            p += w * h * 8
            out.append(dict(kind="decode", depth=depth, w=w, h=h, scale=np.float32(scale), image=img, flow=flow))
        else:
            flow = np.frombuffer(blob, "<f4", fw * fh * 2, p).astype(np.float32)
            p += fw * fh * 8
            img = np.frombuffer(blob, d, w * h * 4, p).copy()
            p += w * h * 4 * d.itemsize
            out.append(dict(kind="encode", depth=depth, w=w, h=h, fw=fw, fh=fh, scale=np.float32(scale), flow=flow,
                            image=img))
    assert p == len(blob), (p, len(blob))
    return out


def rt_grid():
    """The served cases of the retime-time parity grid: (meta cases, {clip name: raw bytes})."""
    z = np.load(os.path.join(GOLDEN, "retime_time_grid.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    inputs = {name: z[f"input_{i}"] for i, name in enumerate(meta["inputs"])}
    return meta["cases"], inputs


def parse_keys(text):
    """A keyed CLI value ``V@F[h|e];...`` (crates/fx-core/src/curves.rs:75-115) as (frame, value,
    flags) triples, flags bit 0 ease, bit 1 hold; a plain value gives None and the value."""
    if "@" not in text:
        return None, float(text)
    keys = []
    for piece in text.split(";"):
        v, f = piece.rsplit("@", 1)
        flags = 2 if f.endswith("h") else 1 if f.endswith("e") else 0
        keys.append((float(f.rstrip("he")), float(v), flags))
    return keys, 0.0


def rt_case_params(case):
    """Keyword arguments of oracle_lib.retime_params for a retime-time grid case (the effect's
    defaults elsewhere; Input: Frame Rate defaults to 29.97 narrowed through f32). The composition
    rate is the grid's exact rate (``24``, ``30000/1001``, ``29.97``) in lowest terms, the time base
    the reference's CLI gives it (crates/fx-cli/src/cli.rs:247-257, crates/fx-core/src/time.rs:83-98)."""
    p = dict(x.split("=", 1) for x in case["params"])
    keys, speed = parse_keys(p.get("speed_percent", "100"))
    fn_keys, fnum = parse_keys(p.get("frame_num", "0"))
    fps = fractions.Fraction(case["fps"])
    mark_keys, marks = parse_keys(p.get("src_mark_segments", "1"))
    return dict(fps=(fps.numerator, fps.denominator), input_fields=int(p.get("input_fields", 1)),
                mark_segs=1 if mark_keys else int(marks), mark_keys=[(f, v) for f, v, _ in mark_keys] if mark_keys else None, speed=speed, keys=keys, vectors=int(p.get("vectors", 5)),
                frame_interp=int(p.get("frame_interp", 2)), remap_mode=int(p.get("time_remap_mode", 1)),
                frame_num=fnum, fn_keys=fn_keys, own_input_rate=p.get("in_fps_is_out_fps", "1") == "0",
                input_frame_rate=float(p.get("input_frame_rate", float(np.float32(29.97)))))


def fgc_grid(video_360=False):
    """The served cases of the fgbg-core parity grid: (meta cases, {clip name: raw bytes}); with
    video_360 the cases with 360 Video on."""
    z = np.load(os.path.join(GOLDEN, "fgbg_core_360_grid.npz" if video_360 else "fgbg_core_grid.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    inputs = {name: z[f"input_{i}"] for i, name in enumerate(meta["inputs"])}
    return meta["cases"], inputs


def fgc_case_params(case):
    """Keyword arguments of oracle_lib.retime_params for a fgbg-core grid case (retime-fgbg's
    defaults elsewhere: Warping 1 Inverse, which is warping code Warping - 1, glue.rs:94-100). Its
    Image Prep 2 runs both prep stages and 3 none (plugins/retime-fgbg/src/glue.rs:153-154): the
    oracle's prep code 4 and 1."""
    p = dict(x.split("=", 1) for x in case["params"])
    keys, speed = parse_keys(p.get("speed_percent", "100"))
    fn_keys, fnum = parse_keys(p.get("frame_num", "0"))
    fps = fractions.Fraction(case["fps"])
    mark_keys, marks = parse_keys(p.get("src_mark_segments", "1"))
    return dict(fps=(fps.numerator, fps.denominator), speed=speed, keys=keys, vectors=int(p.get("vectors", 5)),
                input_fields=int(p.get("input_fields", 1)), mark_segs=1 if mark_keys else int(marks),
                mark_keys=[(f, v) for f, v, _ in mark_keys] if mark_keys else None,
                frame_interp=int(p.get("frame_interp", 2)), smart_blend=int(p.get("warping", 1)) - 1,
                sensitivity=float(p.get("main_bg_sensitivity", 70)), blur=float(p.get("blur_compensation", 0)),
                prep={1: 1, 2: 4, 3: 1}[int(p.get("prep", 1))], track_rgb_a=p.get("track_rgb_a", "0") == "1",
                remap_mode=int(p.get("time_remap_mode", 1)), frame_num=fnum, fn_keys=fn_keys,
                own_input_rate=p.get("in_fps_is_out_fps", "1") == "0",
                input_frame_rate=float(p.get("input_frame_rate", float(np.float32(29.97)))), frame_time_plain=True,
                wrap_360=p.get("video_360", "0") == "1")


def debug_tables():
    """The tables of the reference's Debug view tests (values of the original plugin's view
    generator and traced rows of its special value clip; see tests/golden/make_golden.py)."""
    with open(os.path.join(GOLDEN, "debug_tables.json")) as f:
        return json.load(f)


def debug_cases():
    """The reference's numpy model of the Debug views (debug_cases.hex, its gen_debug.py):
    b"DBG1", u32 count, per case u32 fmt, W, H, FW, FH, i32 code, then x, y (W*H*4 samples of the
    format), the flow (FW*FH*2 f32) and the expected view (W*H*4)."""
    blob = gzip.open(os.path.join(GOLDEN, "debug_cases.bin.gz")).read()
    assert blob[:4] == b"DBG1"
    n = struct.unpack_from("<I", blob, 4)[0]
    p, out = 8, []
    dt = {0: np.dtype("u1"), 1: np.dtype("<u2"), 2: np.dtype("<f4")}
    for _ in range(n):
        fmt, w, h, fw, fh = struct.unpack_from("<5I", blob, p)
        code = struct.unpack_from("<i", blob, p + 20)[0]
        p += 24
        d = dt[fmt]
        take = lambda cnt, dtype: (np.frombuffer(blob, dtype, cnt, p).copy(), cnt * np.dtype(dtype).itemsize)
        x, k = take(w * h * 4, d); p += k
        y, k = take(w * h * 4, d); p += k
        flow, k = take(fw * fh * 2, "<f4"); p += k
        want, k = take(w * h * 4, d); p += k
        out.append(dict(fmt=fmt, w=w, h=h, fw=fw, fh=fh, code=code, x=x, y=y, flow=flow.astype(np.float32), want=want))
    assert p == len(blob)
    return out
