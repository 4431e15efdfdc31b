"""ctypes bindings of the CPU oracle (oracle/liboracle.so).

The oracle is the checker of the parity tests: a C++ restatement of the reference CPU engine
(baairon/twixtor, plugins/retime-engine). It is test infrastructure; the product library never
links or calls it.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

FMT = {"u8": 0, "u16": 1, "f32": 2}
DTYPE = {0: np.uint8, 1: np.uint16, 2: np.float32}


class RetimeParams(ctypes.Structure):
    _fields_ = [
        ("fps_num", ctypes.c_int),
        ("fps_den", ctypes.c_int),
        ("quality_high", ctypes.c_int),
        ("speed_percent", ctypes.c_double),
        ("nkeys", ctypes.c_int),
        ("key_frames", ctypes.POINTER(ctypes.c_double)),
        ("key_values", ctypes.POINTER(ctypes.c_double)),
        ("key_ease", ctypes.POINTER(ctypes.c_int)),
        ("vectors", ctypes.c_int),
        ("frame_interp", ctypes.c_int),
        ("smart_blend", ctypes.c_int),
        ("sensitivity", ctypes.c_double),
        ("blur_compensation", ctypes.c_double),
        ("rows_reversed", ctypes.c_int),
        ("taps_above_first", ctypes.c_int),
        ("video_360", ctypes.c_int),
        ("prep", ctypes.c_int),
        ("track_rgb_a", ctypes.c_int),
        ("remap_mode", ctypes.c_int),
        ("frame_num", ctypes.c_double),
        ("nfn_keys", ctypes.c_int),
        ("fn_key_frames", ctypes.POINTER(ctypes.c_double)),
        ("fn_key_values", ctypes.POINTER(ctypes.c_double)),
        ("fn_key_ease", ctypes.POINTER(ctypes.c_int)),
        ("own_input_rate", ctypes.c_int),
        ("input_frame_rate", ctypes.c_double),
        ("frame_time_bias", ctypes.c_double),
        ("frame_time_plain", ctypes.c_int),
        ("wrap_360", ctypes.c_int),
        ("input_fields", ctypes.c_int),
        ("mark_segs", ctypes.c_int),
        ("nmark_keys", ctypes.c_int),
        ("mark_key_frames", ctypes.POINTER(ctypes.c_double)),
        ("mark_key_values", ctypes.POINTER(ctypes.c_double)),
    ]


class VecInParams(ctypes.Structure):
    _fields_ = [
        ("fps_num", ctypes.c_int),
        ("fps_den", ctypes.c_int),
        ("quality_high", ctypes.c_int),
        ("speed_percent", ctypes.c_double),
        ("nkeys", ctypes.c_int),
        ("key_frames", ctypes.POINTER(ctypes.c_double)),
        ("key_values", ctypes.POINTER(ctypes.c_double)),
        ("key_ease", ctypes.POINTER(ctypes.c_int)),
        ("frame_interp", ctypes.c_int),
        ("warping", ctypes.c_int),
        ("blur_compensation", ctypes.c_double),
        ("max_displace", ctypes.c_double),
        ("vec_scale_x", ctypes.c_double),
        ("vec_scale_y", ctypes.c_double),
        ("rows_reversed", ctypes.c_int),
        ("taps_above_first", ctypes.c_int),
        ("gouraud", ctypes.c_int),
        ("probe_current_time", ctypes.c_int),
        ("remap_mode", ctypes.c_int),
        ("frame_num", ctypes.c_double),
        ("nfn_keys", ctypes.c_int),
        ("fn_key_frames", ctypes.POINTER(ctypes.c_double)),
        ("fn_key_values", ctypes.POINTER(ctypes.c_double)),
        ("fn_key_ease", ctypes.POINTER(ctypes.c_int)),
        ("own_input_rate", ctypes.c_int),
        ("input_frame_rate", ctypes.c_double),
        ("mark_segs", ctypes.c_int),
        ("nmark_keys", ctypes.c_int),
        ("mark_key_frames", ctypes.POINTER(ctypes.c_double)),
        ("mark_key_values", ctypes.POINTER(ctypes.c_double)),
    ]


_lib = None


def build():
    """Compiles the oracle with its Makefile (g++ from PATH; no fast math, no FMA contraction)."""
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True, env=env)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        P = ctypes.c_void_p
        i, f = ctypes.c_int, ctypes.c_float
        L.or_last_error.restype = ctypes.c_char_p
        L.or_gaussian_kernel.argtypes = [f, P, i]
        L.or_start_level.argtypes = [f, i, P, P]
        L.or_block_cost.argtypes = [P, i, i, P, f, f, P]
        L.or_block_cost.restype = f
        L.or_convolve.argtypes = [P, i, i, i, P, i, i]
        L.or_calc_grad.argtypes = [P, i, i, P]
        L.or_new_disp.argtypes = [P, P, P, ctypes.c_long]
        L.or_upsample_flow.argtypes = [P, i, i, i, i, P]
        L.or_block_match.argtypes = [P, P, P, i, i]
        L.or_all_out_of_range.argtypes = [P, i, i]
        L.or_geometry.argtypes = [i, i, i, i, P, P, i]
        L.or_build_pyramid.argtypes = [P, i, i, i, i, i, f, i, i, i, i, P]
        L.or_compose_vectors3.argtypes = [P, P, i, i, i, P, P, i, i, f, f, f, i, i, i, i, i, f, i, P]
        L.or_solve_pair.argtypes = [P, P, i, i, i, i, i, f, i, i, P, P]
        L.or_solve.argtypes = [P, P, i, i, i, i, i, f, i, i, i, P]
        L.or_solve_pyramids_with.argtypes = [P, P, i, i, i, i, i, f, i, P, P, P, i, P, P, P, P, P, P, P]
        L.or_inv_warp.argtypes = [P, P, i, i, i, P, i, i, f, i, P]
        L.or_blend.argtypes = [P, P, P, i, i, i, f]
        L.or_compose_vectors.argtypes = [P, P, i, i, i, P, P, i, i, f, i, P]
        L.or_from_frame.argtypes = [P, i, i, i, P]
        L.or_to_frame.argtypes = [P, i, i, i, P]
        L.or_select.argtypes = [ctypes.POINTER(RetimeParams), i, i, i, P, P, P, P, P, P, P]
        L.or_retime_clip.argtypes = [P, i, i, i, i, ctypes.POINTER(RetimeParams), i, P]
        L.or_retime_one.argtypes = [P, i, i, i, i, ctypes.POINTER(RetimeParams), i, P]
        L.or_clip_frames.argtypes = [ctypes.POINTER(RetimeParams), i, i, i, P, P]
        L.or_retime_window.argtypes = [P, i, i, i, i, i, i, ctypes.POINTER(RetimeParams), i, P]
        L.or_crt_powf.argtypes = [P, P, P, i]
        L.or_motion_blur.argtypes = [P, P, i, i, i, P, i, i, f, i, f]
        L.or_retime_fgbg_one.argtypes = [P, i, P, i, P, P, P, i, P, P, i, i, i, ctypes.POINTER(RetimeParams), i, P]
        L.or_set_threads.argtypes = [i]
        L.or_smart_blend.argtypes = [P, P, P, i, i, i, f, i]
        L.or_fill_holes.argtypes = [P, i, i, i, P, i, i]
        L.or_compose_vectors2.argtypes = [P, P, i, i, i, P, P, i, i, f, i, i, i, i, i, P]
        L.or_forward_warp.argtypes = [P, P, i, i, i, P, i, i, f, i, P]
        L.or_fw_mip_level.argtypes = [i, i, P, i, i, f, i, i]
        L.or_fw_mip_level.restype = f
        L.or_fw_level_count.argtypes = [i, i]
        L.or_fw_triangle.argtypes = [P, i, i, P, i]
        L.or_logf.argtypes = [P, P, ctypes.c_long]
        L.or_compose_layers.argtypes = [P, P, i, i, i, i, P, P, P, P, i, i, P, P, i, i, i, i, i, i, f, i, P]
        L.or_mask_pyramid.argtypes = [P, i, i, i, i, i, P, P, i]
        L.or_mask_gradient.argtypes = [P, P, i, i]
        L.or_calc_b_masked.argtypes = [P, P, P, P, i, i, P, P]
        L.or_block_match_gated.argtypes = [P, P, P, i, i, P]
        L.or_solve_masked.argtypes = [P, P, i, i, i, i, i, f, i, P, P, i, P]
        L.or_create_vectors_clip.argtypes = [P, i, i, i, i, ctypes.POINTER(CvParams), i, P, P, P]
        L.or_encode_vectors.argtypes = [P, i, i, i, P, i, i, f]
        L.or_flow_from_vectors.argtypes = [P, i, i, i, f, f, f, i, P]
        L.or_decode_vectors.argtypes = [P, i, i, i, f, P]
        L.or_fill_flow_holes.argtypes = [P, i, i, P, i, i]
        L.or_invert_flow.argtypes = [P, i, i, i, i, P]
        L.or_matte_step.argtypes = [P, i, i, i, P]
        L.or_vectors_in_one.argtypes = [P, i, P, i, P, i, i, i, i, ctypes.POINTER(VecInParams), i, P]
        L.or_debug_luma.argtypes = [P, i, i, i, P]
        L.or_debug_detail.argtypes = [P, i, i, P]
        L.or_debug_edge.argtypes = [P, i, i, P]
        L.or_debug_overlay.argtypes = [P, P, i, i, i, P]
        L.or_debug_views_of.argtypes = [P, P, i, i, i, i, P]
        L.or_debug_compose_over.argtypes = [P, P, i, i, i, P]
        L.or_debug_view.argtypes = [P, P, i, i, i, P, i, i, i, i, P]
        L.or_vecin_select.argtypes = [ctypes.POINTER(VecInParams), i, i, i, P, P]
        _lib = L
    return _lib


_lib64 = None


def lib64():
    """The oracle in double precision (oracle/liboracle64.so, the fast mode's FP64 yardstick)."""
    global _lib64
    if _lib64 is None:
        path = os.path.join(ORACLE_DIR, "liboracle64.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P, i = ctypes.c_void_p, ctypes.c_int
        L.or_solve_pair.argtypes = [P, P, i, i, i, i, i, ctypes.c_double, i, i, P, P]
        L.or_solve.argtypes = [P, P, i, i, i, i, i, ctypes.c_double, i, i, i, P]
        L.or_last_error.restype = ctypes.c_char_p
        L.or_set_threads.argtypes = [i]
        _lib64 = L
    return _lib64


def solve_pair64(a, b, w, h, fmt, quality=4, hiq=True, sensitivity=0.7, skip_refine=False, above_first=True):
    """solve_pair evaluated in double precision: (f_ab, f_ba) as float64 arrays."""
    _, sizes = geometry(quality, hiq, w, h)
    fw, fh = sizes[0]
    f_ab = np.zeros(fw * fh * 2, np.float64)
    f_ba = np.zeros(fw * fh * 2, np.float64)
    rc = lib64().or_solve_pair(ptr(a), ptr(b), w, h, fmt, quality, int(hiq), float(np.float32(sensitivity)),
                               int(skip_refine), int(above_first), ptr(f_ab), ptr(f_ba))
    if rc:
        raise ValueError(lib64().or_last_error().decode())
    return f_ab, f_ba, (fw, fh)


def solve64(x, y, w, h, fmt, quality=4, hiq=True, sensitivity=0.7, skip_refine=False, above_first=True, prep=1):
    """flow::solve X -> Y evaluated in double precision (float64 field)."""
    _, sizes = geometry(quality, hiq, w, h)
    fw, fh = sizes[0]
    out = np.zeros(fw * fh * 2, np.float64)
    rc = lib64().or_solve(ptr(x), ptr(y), w, h, fmt, quality, int(hiq), float(np.float32(sensitivity)),
                          int(skip_refine), int(above_first), prep, ptr(out))
    if rc:
        raise ValueError(lib64().or_last_error().decode())
    return out, (fw, fh)


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def err():
    return lib().or_last_error().decode()


def geometry(quality, hiq, w, h):
    red = ctypes.c_int()
    sizes = np.zeros(64, np.int32)
    n = lib().or_geometry(quality, int(hiq), w, h, ctypes.byref(red), ptr(sizes), 32)
    if n < 0:
        raise ValueError(err())
    return red.value, [(int(sizes[2 * i]), int(sizes[2 * i + 1])) for i in range(n)]


def from_frame(wire, w, h, fmt):
    out = np.zeros(w * h * 4, DTYPE[fmt])
    lib().or_from_frame(ptr(wire), w, h, fmt, ptr(out))
    return out


def to_frame(engine, w, h, fmt):
    out = np.zeros(w * h * 4, DTYPE[fmt])
    lib().or_to_frame(ptr(engine), w, h, fmt, ptr(out))
    return out


def build_pyramid(engine, w, h, fmt, quality=4, hiq=True, sensitivity=0.7, above_first=True, prep=1, wrap=False,
                  track_alpha=False):
    _, sizes = geometry(quality, hiq, w, h)
    total = sum(a * b for a, b in sizes)
    out = np.zeros(total, np.float32)
    n = lib().or_build_pyramid(ptr(engine), w, h, fmt, quality, int(hiq), sensitivity, int(above_first), int(prep),
                               int(wrap), int(track_alpha), ptr(out))
    if n < 0:
        raise ValueError(err())
    levels, off = [], 0
    for lw, lh in sizes:
        levels.append(out[off:off + lw * lh].reshape(lh, lw))
        off += lw * lh
    return levels


def solve_pair(a, b, w, h, fmt, quality=4, hiq=True, sensitivity=0.7, skip_refine=False, above_first=True):
    _, sizes = geometry(quality, hiq, w, h)
    fw, fh = sizes[0]
    f_ab = np.zeros(fw * fh * 2, np.float32)
    f_ba = np.zeros(fw * fh * 2, np.float32)
    rc = lib().or_solve_pair(ptr(a), ptr(b), w, h, fmt, quality, int(hiq), sensitivity, int(skip_refine),
                             int(above_first), ptr(f_ab), ptr(f_ba))
    if rc:
        raise ValueError(err())
    return f_ab, f_ba, (fw, fh)


def solve(x, y, w, h, fmt, quality=4, hiq=True, sensitivity=0.7, skip_refine=False, above_first=True, prep=1):
    """flow::solve X -> Y (prep: 1 none, 2 Contrast/Edge Enhance, 3 Delinearize)."""
    _, sizes = geometry(quality, hiq, w, h)
    fw, fh = sizes[0]
    out = np.zeros(fw * fh * 2, np.float32)
    rc = lib().or_solve(ptr(x), ptr(y), w, h, fmt, quality, int(hiq), np.float32(sensitivity), int(skip_refine),
                        int(above_first), prep, ptr(out))
    if rc:
        raise ValueError(err())
    return out, (fw, fh)


def solve_pyramids_with(x, y, w, h, fmt, matte_x=None, matte_y=None, pairs=None, quality=4, hiq=True, sensitivity=0.7,
                        above_first=True):
    """flow::extras::solve_pyramids_with: returns (flow, x_levels, y_levels, mask_x, mask_y, user_d,
    user_w), the pyramids concatenated finest first; the masks / user displacement None when absent."""
    _, sizes = geometry(quality, hiq, w, h)
    fw, fh = sizes[0]
    pf = sum(a * b for a, b in sizes)
    out = np.zeros(fw * fh * 2, np.float32)
    xl, yl = np.zeros(pf, np.float32), np.zeros(pf, np.float32)
    mxl, myl = np.zeros(pf, np.float32), np.zeros(pf, np.float32)
    ud, uw = np.zeros(2 * pf, np.float32), np.zeros(pf, np.float32)
    pts = np.ascontiguousarray(pairs if pairs is not None else np.zeros((1, 4)), np.float32)
    npts = 0 if pairs is None else len(pairs)
    mx = None if matte_x is None else np.ascontiguousarray(matte_x, np.float32)
    my = None if matte_y is None else np.ascontiguousarray(matte_y, np.float32)
    rc = lib().or_solve_pyramids_with(ptr(x), ptr(y), w, h, fmt, quality, int(hiq), np.float32(sensitivity),
                                      int(above_first), ptr(mx), ptr(my), ptr(pts), npts, ptr(xl), ptr(yl), ptr(mxl),
                                      ptr(myl), ptr(ud), ptr(uw), ptr(out))
    if rc:
        raise ValueError(err())
    return (out, xl, yl, mxl if mx is not None else None, myl if mx is not None else None,
            ud if npts else None, uw if npts else None)


def inv_warp(src, w, h, fmt, flow, fw, fh, amount, hold=True, coverage=False, out=None, is360=False):
    o = np.zeros_like(src) if out is None else out.copy()
    cov = np.zeros(w * h, np.uint8) if coverage else None
    rc = lib().or_inv_warp(ptr(o), ptr(src), w, h, fmt, ptr(flow), fw, fh, amount, int(hold) | (2 if is360 else 0),
                           ptr(cov))
    if rc:
        raise ValueError(err())
    return (o, cov) if coverage else o


def compose_vectors(a, b, w, h, fmt, f_ab, f_ba, fw, fh, wa, interp=1):
    out = np.zeros_like(a)
    rc = lib().or_compose_vectors(ptr(a), ptr(b), w, h, fmt, ptr(f_ab), ptr(f_ba), fw, fh, wa, interp, ptr(out))
    if rc:
        raise ValueError(err())
    return out


def compose_vectors3(a, b, w, h, fmt, f_ab, f_ba, fw, fh, sel, cs):
    """compose_vectors with the selection and compose settings of the library (tw.Selection,
    tw.EngineSettings): the Blur Compensation tail included."""
    out = np.zeros_like(a)
    rc = lib().or_compose_vectors3(ptr(a), ptr(b), w, h, fmt, ptr(f_ab) if f_ab is not None else None,
                                   ptr(f_ba) if f_ba is not None else None, fw, fh, np.float32(sel.s0), np.float32(sel.s1),
                                   np.float32(sel.wa), sel.interp, cs.warp_mode, int(cs.video_360),
                                   int(cs.taps_above_first), int(cs.gouraud), np.float32(cs.blur), int(cs.quality_high),
                                   ptr(out))
    if rc:
        raise ValueError(err())
    return out


def compose_vectors2(a, b, w, h, fmt, f_ab, f_ba, fw, fh, wa, interp, warp_mode, video_360=False,
                     taps_above_first=True, gouraud=False):
    """compose_vectors with a warping code (1: Smart Blend with the hole fill, 2 / 3 the forward warps
    with / without coverage and fill; ``gouraud`` their Gouraud variant) and the binary alpha flag."""
    out = np.zeros_like(a)
    rc = lib().or_compose_vectors2(ptr(a), ptr(b), w, h, fmt, ptr(f_ab) if f_ab is not None else None,
                                   ptr(f_ba) if f_ba is not None else None, fw, fh, wa, interp, warp_mode,
                                   int(video_360), int(taps_above_first), int(gouraud), ptr(out))
    if rc:
        raise ValueError(err())
    return out


def fill_holes(img, w, h, fmt, mask, mask_kind, above_first=True):
    out = np.array(img, copy=True)
    rc = lib().or_fill_holes(ptr(out), w, h, fmt, ptr(mask), mask_kind, int(above_first))
    if rc:
        raise ValueError(err())
    return out


class CvParams(ctypes.Structure):
    _fields_ = [("fps_num", ctypes.c_int), ("fps_den", ctypes.c_int), ("quality_high", ctypes.c_int),
                ("vector_resolution", ctypes.c_int), ("max_displace", ctypes.c_double), ("track_frame", ctypes.c_int),
                ("sensitivity", ctypes.c_double), ("track_rgb_a", ctypes.c_int), ("rows_reversed", ctypes.c_int),
                ("taps_above_first", ctypes.c_int), ("prep", ctypes.c_int), ("display", ctypes.c_int),
                ("debug_view_method", ctypes.c_int), ("debug_textured", ctypes.c_int)]


def create_vectors_clip(frames, nframes, w, h, fmt, nout, fps=(24, 1), vector_resolution=1, max_displace=2048.0,
                        track_frame=1, sensitivity=70.0, track_rgb_a=False, rows_reversed=True, taps_above_first=True,
                        prep=1, points=None, display=2, debug_view_method=1, debug_textured=False):
    """Output frames 0..nout-1 of the Create Vectors effect (plugin 02, one layer) over a raw clip;
    ``points[n]`` the tracking points of output frame n (x, y at X, x, y at Y; host rows); display 3
    is the Debug display of ``debug_view_method`` (its forward warp the Gouraud variant, or textured
    with ``debug_textured``: the revision the parity grid records)."""
    p = CvParams(fps[0], fps[1], 1, vector_resolution, max_displace, track_frame, sensitivity, int(track_rgb_a),
                 int(rows_reversed), int(taps_above_first), int(prep), int(display), int(debug_view_method),
                 int(debug_textured))
    out = np.zeros(nout * w * h * 4, DTYPE[fmt])
    pts = npts = None
    if points is not None:
        npts = np.array([len(x) for x in points], np.int32)
        pts = np.array([q for x in points for q in x] or [[0, 0, 0, 0]], np.float32).reshape(-1)
    rc = lib().or_create_vectors_clip(ptr(np.ascontiguousarray(frames)), nframes, w, h, fmt, ctypes.byref(p), nout,
                                      ptr(pts), ptr(npts), ptr(out))
    if rc:
        raise ValueError(err())
    return out


def encode_vectors(flow, fw, fh, w, h, fmt, scale):
    out = np.zeros(w * h * 4, DTYPE[fmt])
    rc = lib().or_encode_vectors(ptr(out), w, h, fmt, ptr(np.ascontiguousarray(flow, np.float32)), fw, fh,
                                 np.float32(scale))
    if rc:
        raise ValueError(err())
    return out


def mask_pyramid(matte, w, h, quality=4, hiq=True, above_first=True):
    """flow/extras.rs MaskPyramid::build: the binary mask levels (finest first) as (w, h, values)."""
    out = np.zeros(2 * w * h + 64, np.float32)
    sizes = np.zeros(64, np.int32)
    n = lib().or_mask_pyramid(ptr(np.ascontiguousarray(matte, np.float32)), w, h, quality, int(hiq), int(above_first),
                              ptr(out), ptr(sizes), 32)
    if n < 0:
        raise ValueError(err())
    levels, off = [], 0
    for i in range(n):
        lw, lh = int(sizes[2 * i]), int(sizes[2 * i + 1])
        levels.append((lw, lh, out[off:off + lw * lh].copy()))
        off += lw * lh
    return levels


def solve_masked(x, y, w, h, fmt, matte_x=None, matte_y=None, quality=4, hiq=True, sensitivity=0.7, above_first=True,
                 gate=False):
    """flow::extras::solve_pyramids_with with the mask pyramids of two mattes: the flow of X -> Y."""
    _, sizes = geometry(quality, hiq, w, h)
    fw, fh = sizes[0]
    out = np.zeros(fw * fh * 2, np.float32)
    mx = None if matte_x is None else np.ascontiguousarray(matte_x, np.float32)
    my = None if matte_y is None else np.ascontiguousarray(matte_y, np.float32)
    rc = lib().or_solve_masked(ptr(x), ptr(y), w, h, fmt, quality, int(hiq), np.float32(sensitivity), int(above_first),
                               ptr(mx), ptr(my), int(gate), ptr(out))
    if rc:
        raise ValueError(err())
    return out, (fw, fh)


def compose_layers(a, b, w, h, fmt, mattes_a, mattes_b, sensitivity, wa, interp=1, quality=4, hiq=True,
                   above_first=True, warp_mode=0, video_360=False, gouraud=False, shrink=None, group=None, points=None):
    """layers/plates.rs solve_and_compose_plates of one in-between frame (engine images in and out);
    ``shrink`` the inverse matte shrink per FG layer, ``group`` the displayed (first, last)."""
    nfg = len(mattes_a)
    ma = np.ascontiguousarray(np.concatenate(mattes_a) if nfg else np.zeros(1), np.float32)
    mb = np.ascontiguousarray(np.concatenate(mattes_b) if nfg else np.zeros(1), np.float32)
    sens = np.ascontiguousarray(sensitivity, np.float32)
    sh = np.ascontiguousarray(list(shrink) if shrink is not None else [0.0] * max(nfg, 1), np.float32)
    first, last = group if group is not None else (0, -1)
    lists = points if points is not None else [[] for _ in range(nfg + 1)]
    npts = np.array([len(x) for x in lists], np.int32)
    pts = np.array([q for x in lists for q in x] or [[0, 0, 0, 0]], np.float32).reshape(-1)
    out = np.zeros_like(a)
    rc = lib().or_compose_layers(ptr(a), ptr(b), w, h, fmt, nfg, ptr(ma), ptr(mb), ptr(sens), ptr(sh), first, last,
                                 ptr(pts), ptr(npts), quality, int(hiq), int(above_first), warp_mode, int(video_360), int(gouraud),
                                 np.float32(wa), interp, ptr(out))
    if rc:
        raise ValueError(err())
    return out


def forward_warp(src, w, h, fmt, flow, fw, fh, amount, pyramid=True, coverage=False):
    """forward.rs forward_warp_with: (out, cov) with coverage, else out."""
    out = np.zeros_like(src)
    cov = np.zeros(w * h, np.uint8) if coverage else None
    rc = lib().or_forward_warp(ptr(out), ptr(src), w, h, fmt, ptr(np.ascontiguousarray(flow, np.float32)), fw, fh,
                               np.float32(amount), int(pyramid), ptr(cov))
    if rc:
        raise ValueError(err())
    return (out, cov) if coverage else out


def fw_triangle(verts, w1, h1, cap=4096):
    """forward/raster.rs triangle: the hits (x, y, u, v, d) in order, or None for an outside write."""
    v = np.asarray(verts, np.float32).reshape(-1)
    hits = np.zeros(cap * 5, np.float32)
    n = lib().or_fw_triangle(ptr(v), w1, h1, ptr(hits), cap)
    return None if n < 0 else hits[:n * 5].reshape(n, 5)


def _keys(p, keys, prefix):
    """Keyed curve fields of a params struct: (frame, value, ease) triples."""
    fr = (ctypes.c_double * len(keys))(*[k[0] for k in keys])
    va = (ctypes.c_double * len(keys))(*[k[1] for k in keys])
    ea = (ctypes.c_int * len(keys))(*[int(k[2]) for k in keys])
    setattr(p, "n" + prefix + "keys" if prefix else "nkeys", len(keys))
    pre = prefix + "key_" if prefix else "key_"
    setattr(p, pre + "frames", ctypes.cast(fr, ctypes.POINTER(ctypes.c_double)))
    setattr(p, pre + "values", ctypes.cast(va, ctypes.POINTER(ctypes.c_double)))
    setattr(p, pre + "ease", ctypes.cast(ea, ctypes.POINTER(ctypes.c_int)))
    p.__dict__.setdefault("_keep", []).append((fr, va, ea))


def retime_params(fps=(24, 1), quality_high=True, speed=100.0, keys=None, vectors=5, frame_interp=2, smart_blend=0,
                  sensitivity=70.0, blur=0.0, rows_reversed=True, taps_above_first=True, video_360=False, prep=1,
                  track_rgb_a=False, remap_mode=1, frame_num=0.0, fn_keys=None, own_input_rate=False,
                  input_frame_rate=30.0, frame_time_bias=0.05, frame_time_plain=False, wrap_360=False, input_fields=1,
                  mark_segs=1, mark_keys=None):
    """The `retime` parameters of one render. rows_reversed / taps_above_first at their defaults
    are the reference's current code; both False is the revision the parity grid records.
    remap_mode 2 is Frame Number (frame_num or the keyed fn_keys); own_input_rate turns "In FPS is
    Out FPS" off (the input rate input_frame_rate, the output rate fps); frame_time_bias 0.1 is the
    revision the parity grids record (the reference's current value is 0.05); frame_time_plain is
    retime-fgbg's frame time (trunc(dur * k + 0.5) at every rate); wrap_360 is retime-fgbg's "360 Video"
    (the engine's wrap-around flag); input_fields the Input: Fields popup (1 None); mark_segs the Src:
    Mark Segments popup, or mark_keys its (frame, value) keys."""
    p = RetimeParams()
    p.remap_mode, p.frame_num = remap_mode, frame_num
    p.own_input_rate, p.input_frame_rate = int(own_input_rate), input_frame_rate
    p.frame_time_bias = frame_time_bias
    p.frame_time_plain = int(frame_time_plain)
    p.wrap_360 = int(wrap_360)
    p.input_fields, p.mark_segs = int(input_fields), int(mark_segs)
    if mark_keys:
        fr = (ctypes.c_double * len(mark_keys))(*[k[0] for k in mark_keys])
        va = (ctypes.c_double * len(mark_keys))(*[k[1] for k in mark_keys])
        p.nmark_keys = len(mark_keys)
        p.mark_key_frames = ctypes.cast(fr, ctypes.POINTER(ctypes.c_double))
        p.mark_key_values = ctypes.cast(va, ctypes.POINTER(ctypes.c_double))
        p.__dict__.setdefault("_keep", []).append((fr, va))
    if fn_keys:
        _keys(p, fn_keys, "fn_")
    p.rows_reversed, p.taps_above_first = int(rows_reversed), int(taps_above_first)
    p.video_360 = int(video_360)
    p.prep = int(prep)
    p.track_rgb_a = int(track_rgb_a)
    p.fps_num, p.fps_den = fps
    p.quality_high = int(quality_high)
    p.speed_percent = speed
    p.vectors, p.frame_interp, p.smart_blend = vectors, frame_interp, smart_blend
    p.sensitivity, p.blur_compensation = sensitivity, blur
    p.nkeys = 0
    if keys:
        fr = (ctypes.c_double * len(keys))(*[k[0] for k in keys])
        va = (ctypes.c_double * len(keys))(*[k[1] for k in keys])
        ea = (ctypes.c_int * len(keys))(*[int(k[2]) for k in keys])
        p.nkeys = len(keys)
        p.key_frames = ctypes.cast(fr, ctypes.POINTER(ctypes.c_double))
        p.key_values = ctypes.cast(va, ctypes.POINTER(ctypes.c_double))
        p.key_ease = ctypes.cast(ea, ctypes.POINTER(ctypes.c_int))
        p._keep = (fr, va, ea)
    return p


def select(params, n, w, h):
    s0, s1, wa = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    a, ex, vq, it = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib().or_select(ctypes.byref(params), n, w, h, ctypes.byref(s0), ctypes.byref(s1), ctypes.byref(a),
                    ctypes.byref(wa), ctypes.byref(ex), ctypes.byref(vq), ctypes.byref(it))
    return dict(s0=s0.value, s1=s1.value, a=a.value, wa=wa.value, exact=bool(ex.value), vq=vq.value,
                interp=it.value)


def clip_frames(params, n, w, h):
    """The clip frames output frame n's pair shows (its positions through frame_time)."""
    a, b = ctypes.c_int(), ctypes.c_int()
    lib().or_clip_frames(ctypes.byref(params), n, w, h, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def retime_one(frames, nframes, w, h, fmt, params, n):
    """Output frame n alone (the oracle's renderer is stateless per output frame)."""
    out = np.zeros(w * h * 4, DTYPE[fmt])
    rc = lib().or_retime_one(ptr(frames), nframes, w, h, fmt, ctypes.byref(params), n, ptr(out))
    if rc:
        raise ValueError(err())
    return out


def retime_window(frames, first, count, nframes, w, h, fmt, params, n):
    """Output frame n of a clip of nframes frames from the clip frames [first, first + count) alone;
    raises when the frame needs one outside that window."""
    out = np.zeros(w * h * 4, DTYPE[fmt])
    rc = lib().or_retime_window(ptr(frames), first, count, nframes, w, h, fmt, ctypes.byref(params), n, ptr(out))
    if rc:
        raise RuntimeError(f"or_retime_window: {rc} {err()}")
    return out


def retime_fgbg_clip(frames, nframes, mattes, chans, sens, w, h, fmt, params, nout, shrinks=None, display=1,
                     points=None):
    """retime-fgbg with FG matte layers (FG1 first): ``mattes`` the matte clips (nframes wire frames
    each), ``chans`` their channel popups, ``sens`` their sensitivities 0..100, ``shrinks`` their
    inverse matte shrinks; Main_BG's sensitivity is params.sensitivity; ``display`` the Display
    popup; ``points(n)`` the tracking points of output frame n, one list per layer (Main_BG last)
    of (x, y at A, x, y at B) in host rows. Output frames 0..nout-1 back to back."""
    nfg = len(mattes)
    mattes = [np.ascontiguousarray(m) for m in mattes]
    arr = (ctypes.c_void_p * max(nfg, 1))(*[m.ctypes.data for m in mattes])
    ch = (ctypes.c_int * 3)(*(list(chans) + [1] * (3 - nfg)))
    se = (ctypes.c_double * 3)(*(list(sens) + [70.0] * (3 - nfg)))
    shr = list(shrinks) if shrinks is not None else [0.0] * nfg
    sh = (ctypes.c_double * 3)(*(shr + [0.0] * (3 - nfg)))
    fb = w * h * 4
    out = np.zeros(nout * fb, DTYPE[fmt])
    for n in range(nout):
        lists = points(n) if points else [[] for _ in range(nfg + 1)]
        npts = np.array([len(x) for x in lists], np.int32)
        pts = np.array([q for x in lists for q in x] or [[0, 0, 0, 0]], np.float32).reshape(-1)
        rc = lib().or_retime_fgbg_one(ptr(frames), nframes, arr, nfg, ch, se, sh, display, ptr(pts), ptr(npts), w, h,
                                      fmt, ctypes.byref(params), n, ptr(out[n * fb:]))
        if rc:
            raise ValueError(err())
    return out


def retime_clip(frames, nframes, w, h, fmt, params, nout):
    out = np.zeros(nout * w * h * 4, DTYPE[fmt])
    rc = lib().or_retime_clip(ptr(frames), nframes, w, h, fmt, ctypes.byref(params), nout, ptr(out))
    if rc:
        raise ValueError(err())
    return out


def crt_powf(x, y):
    """The Delinearize powf of the plugin's runtime (crt_powf.rs) over float32 arrays."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(np.broadcast_to(np.asarray(y, np.float32), x.shape), np.float32)
    out = np.zeros_like(x)
    lib().or_crt_powf(ptr(x), ptr(y), ptr(out), x.size)
    return out


def motion_blur(src, w, h, fmt, flow, fw, fh, amount, hiq, shutter):
    """warp::blurcomp::motion_blur (is360 off) of an engine image."""
    out = np.zeros_like(src)
    rc = lib().or_motion_blur(ptr(out), ptr(src), w, h, fmt, ptr(np.ascontiguousarray(flow, np.float32)), fw, fh,
                              np.float32(amount), int(hiq), np.float32(shutter))
    if rc:
        raise ValueError(err())
    return out


# ---- Vectors In ----------------------------------------------------------------------------------


def decode_vectors(vec, w, h, fmt, max_displace):
    """vectors::decode_vectors of an engine image: the (w, h, 2) float32 flow."""
    out = np.zeros(w * h * 2, np.float32)
    lib().or_decode_vectors(ptr(np.ascontiguousarray(vec)), w, h, fmt, np.float32(max_displace), ptr(out))
    return out


def flow_from_vectors(vec, w, h, fmt, max_displace, scale=(1.0, 1.0), above_first=False):
    """compose::flow_from_vector_image_with: decode, flow hole fill, Vec Scale."""
    out = np.zeros(w * h * 2, np.float32)
    rc = lib().or_flow_from_vectors(ptr(np.ascontiguousarray(vec)), w, h, fmt, np.float32(max_displace),
                                    np.float32(scale[0]), np.float32(scale[1]), int(above_first), ptr(out))
    if rc:
        raise ValueError(err())
    return out


def fill_flow_holes(flow, w, h, mask, mask_kind, above_first=False):
    out = np.array(flow, np.float32, copy=True)
    rc = lib().or_fill_flow_holes(ptr(out), w, h, ptr(np.ascontiguousarray(mask)), mask_kind, int(above_first))
    if rc:
        raise ValueError(err())
    return out


def invert_flow(flow, w, h, pyramid=True, above_first=False):
    """compose::invert_flow_on: the inversion of a (w, h) flow (textured or Gouraud forward warp)."""
    out = np.zeros(w * h * 2, np.float32)
    rc = lib().or_invert_flow(ptr(np.ascontiguousarray(flow, np.float32)), w, h, int(pyramid), int(above_first),
                              ptr(out))
    if rc:
        raise ValueError(err())
    return out


def matte_step(vec, w, h, fmt, matte):
    out = np.array(vec, copy=True)
    lib().or_matte_step(ptr(out), w, h, fmt, ptr(np.ascontiguousarray(matte, np.float32)))
    return out


def vecin_params(fps=(30, 1), quality_high=True, speed=100.0, keys=None, frame_interp=2, warping=2, blur=0.0,
                 max_displace=2048.0, vec_scale=(1.0, 1.0), rows_reversed=True, taps_above_first=True, gouraud=True,
                 probe_current_time=False, remap_mode=1, frame_num=0.0, fn_keys=None, own_input_rate=False,
                 input_frame_rate=30.0, mark_segs=1, mark_keys=None):
    """The `vectors-in` parameters of one render (the effect's defaults; the three orders at the
    plugin's: bottom-up rows, the tap above first, the Gouraud forward warp; a set vector layer
    present at every time). All four False is the revision the parity grid records."""
    p = VecInParams()
    p.fps_num, p.fps_den = fps
    p.quality_high = int(quality_high)
    p.speed_percent = speed
    p.frame_interp, p.warping = frame_interp, warping
    p.blur_compensation, p.max_displace = blur, max_displace
    p.vec_scale_x, p.vec_scale_y = vec_scale
    p.rows_reversed, p.taps_above_first, p.gouraud = int(rows_reversed), int(taps_above_first), int(gouraud)
    p.probe_current_time = int(probe_current_time)
    p.remap_mode, p.frame_num = remap_mode, frame_num
    p.own_input_rate, p.input_frame_rate = int(own_input_rate), input_frame_rate
    if fn_keys:
        _keys(p, fn_keys, "fn_")
    p.nkeys = 0
    if keys:
        fr = (ctypes.c_double * len(keys))(*[k[0] for k in keys])
        va = (ctypes.c_double * len(keys))(*[k[1] for k in keys])
        ea = (ctypes.c_int * len(keys))(*[int(k[2]) for k in keys])
        p.nkeys = len(keys)
        p.key_frames = ctypes.cast(fr, ctypes.POINTER(ctypes.c_double))
        p.key_values = ctypes.cast(va, ctypes.POINTER(ctypes.c_double))
        p.key_ease = ctypes.cast(ea, ctypes.POINTER(ctypes.c_int))
        p._keep = (fr, va, ea)
    p.mark_segs, p.nmark_keys = int(mark_segs), 0
    if mark_keys:
        mf = (ctypes.c_double * len(mark_keys))(*[k[0] for k in mark_keys])
        mv = (ctypes.c_double * len(mark_keys))(*[k[1] for k in mark_keys])
        p.nmark_keys = len(mark_keys)
        p.mark_key_frames = ctypes.cast(mf, ctypes.POINTER(ctypes.c_double))
        p.mark_key_values = ctypes.cast(mv, ctypes.POINTER(ctypes.c_double))
        p.__dict__.setdefault("_keep_marks", []).append((mf, mv))
    return p


def vectors_in_clip(frames, nframes, vec_next, n_next, vec_prev, n_prev, w, h, fmt, params, nout):
    """Output frames 0..nout-1 of the single layer `vectors-in` render, back to back. vec_next /
    vec_prev: wire clips of the vector layers (None: the layer is not set)."""
    fb = w * h * 4
    out = np.zeros(nout * fb, DTYPE[fmt])
    vn = None if vec_next is None else np.ascontiguousarray(vec_next)
    vp = None if vec_prev is None else np.ascontiguousarray(vec_prev)
    for n in range(nout):
        rc = lib().or_vectors_in_one(ptr(frames), nframes, None if vn is None else ptr(vn), n_next,
                                     None if vp is None else ptr(vp), n_prev, w, h, fmt, ctypes.byref(params), n,
                                     ptr(out[n * fb:]))
        if rc:
            raise ValueError(f"or_vectors_in_one: {rc} {err()}")
    return out


def vecin_select(params, n, w, h):
    """The Vectors In effect's selection of output frame n and the clip frames of its pair."""
    f3, i6 = np.zeros(3, np.float32), np.zeros(6, np.int32)
    lib().or_vecin_select(ctypes.byref(params), n, w, h, ptr(f3), ptr(i6))
    return dict(s0=f3[0], s1=f3[1], wa=f3[2], a=int(i6[0]), exact=bool(i6[1]), vq=int(i6[2]), interp=int(i6[3]),
                clip_a=int(i6[4]), clip_b=int(i6[5]))


# ---- the Debug views of Create Vectors -------------------------------------------------------------


def debug_luma(img, w, h, fmt):
    out = np.zeros(w * h, np.float32)
    lib().or_debug_luma(ptr(np.ascontiguousarray(img)), w, h, fmt, ptr(out))
    return out


def debug_detail(plane, w, h):
    out = np.zeros(w * h, np.float32)
    lib().or_debug_detail(ptr(np.ascontiguousarray(plane, np.float32)), w, h, ptr(out))
    return out


def debug_edge(plane, w, h):
    out = np.zeros(w * h, np.float32)
    lib().or_debug_edge(ptr(np.ascontiguousarray(plane, np.float32)), w, h, ptr(out))
    return out


def debug_overlay(r, g, w, h, fmt):
    out = np.zeros(w * h * 4, DTYPE[fmt])
    lib().or_debug_overlay(ptr(np.ascontiguousarray(r, np.float32)), ptr(np.ascontiguousarray(g, np.float32)), w, h,
                           fmt, ptr(out))
    return out


def debug_views_of(wp, y, w, h, fmt, code):
    out = np.zeros(w * h * 4, DTYPE[fmt])
    lib().or_debug_views_of(ptr(np.ascontiguousarray(wp)), ptr(np.ascontiguousarray(y)), w, h, fmt, code, ptr(out))
    return out


def debug_compose_over(wimg, y, w, h, fmt):
    out = np.zeros(w * h * 4, DTYPE[fmt])
    lib().or_debug_compose_over(ptr(np.ascontiguousarray(wimg)), ptr(np.ascontiguousarray(y)), w, h, fmt, ptr(out))
    return out


def debug_view(x, y, w, h, fmt, flow, fw, fh, code, gouraud=True):
    """debug::debug_view_on: view code 0 Blend, 1 Diff, 2 Detail, 3 Edge, 4 Warp."""
    out = np.zeros(w * h * 4, DTYPE[fmt])
    rc = lib().or_debug_view(ptr(np.ascontiguousarray(x)), ptr(np.ascontiguousarray(y)), w, h, fmt,
                             ptr(np.ascontiguousarray(flow, np.float32)), fw, fh, code, int(gouraud), ptr(out))
    if rc:
        raise ValueError(err())
    return out
