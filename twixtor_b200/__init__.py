"""twixtor_b200: the retime hot path of baairon/twixtor on B200 (sm_100a CUDA behind a C ABI).

This module is the Python face of the library ``libtwixtor_b200.so`` (declared in
``include/twixtor_b200.h``). It mirrors the reference's stage seam
(``plugins/retime-engine/src/stages.rs:33-71``, trait ``Stages``; its device side is
``device/exec/backend.rs:27-46``, trait ``Backend``): ``solve``, ``solve_pair`` and
``compose_vectors`` take the same arguments (engine images, ``FlowSettings``, a ``Selection``) and
return what the CPU functions return. Every computation runs in the library's CUDA kernels; when
the library is missing, importing a ``Device`` raises instead of falling back to anything else.

Images are numpy arrays of ``width * height * 4`` samples (uint8, uint16 or float32) in the engine
layout (A, R, G, B premultiplied, top row first); flows are float32 arrays of
``width * height * 2`` values, (dx, dy) interleaved.
"""
import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtwixtor_b200.so")

U8, U16, F32 = 0, 1, 2
DTYPES = {U8: np.uint8, U16: np.uint16, F32: np.float32}
FMT_OF_DTYPE = {np.dtype(np.uint8): U8, np.dtype(np.uint16): U16, np.dtype(np.float32): F32}

OK, ERR_CUDA, ERR_NAN_OUTPUT, ERR_UNSUPPORTED, ERR_MISMATCH, ERR_BAD_PARAM, ERR_DEVICE_BOUND = range(7)


class StageError(RuntimeError):
    """A stage the device did not serve (the reference's ``device::image::StageError``)."""

    def __init__(self, code, message):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


class Unsupported(StageError):
    pass


class NanOutput(StageError):
    pass


class Mismatch(StageError):
    pass


class BadParam(StageError):
    pass


INJECT_NONE, INJECT_ALLOC, INJECT_STATUS = 0, 1, 2

_ERRORS = {ERR_UNSUPPORTED: Unsupported, ERR_NAN_OUTPUT: NanOutput, ERR_MISMATCH: Mismatch, ERR_BAD_PARAM: BadParam,
           ERR_DEVICE_BOUND: Unsupported}


# ---- C ABI structs (include/twixtor_b200.h) --------------------------------------------------------

class _Image(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("fmt", ctypes.c_int32),
                ("data", ctypes.c_void_p), ("bytes", ctypes.c_size_t)]


class _Flow(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("data", ctypes.c_void_p)]


class _FlowSettings(ctypes.Structure):
    _fields_ = [("quality", ctypes.c_int32), ("hiq", ctypes.c_int32), ("sensitivity", ctypes.c_float),
                ("prep_contrast_edge", ctypes.c_int32), ("prep_delinearize", ctypes.c_int32),
                ("track_alpha", ctypes.c_int32), ("video_range_luma", ctypes.c_int32),
                ("skip_refine", ctypes.c_int32), ("wrap", ctypes.c_int32), ("taps_above_first", ctypes.c_int32),
                ("fast_mode", ctypes.c_int32)]


class _Selection(ctypes.Structure):
    _fields_ = [("s0", ctypes.c_float), ("s1", ctypes.c_float), ("a", ctypes.c_int32), ("b", ctypes.c_int32),
                ("wa", ctypes.c_float), ("exact", ctypes.c_int32), ("vectors_quality", ctypes.c_int32),
                ("interp", ctypes.c_int32)]


class _EngineSettings(ctypes.Structure):
    _fields_ = [("warp_mode", ctypes.c_int32), ("video_360", ctypes.c_int32), ("wrap_360", ctypes.c_int32),
                ("quality_high", ctypes.c_int32), ("blur", ctypes.c_float), ("taps_above_first", ctypes.c_int32),
                ("gouraud", ctypes.c_int32)]


class _RetimeSettings(ctypes.Structure):
    _fields_ = [("flow", _FlowSettings), ("compose", _EngineSettings), ("motion_rows_reversed", ctypes.c_int32)]


class _ClipJob(ctypes.Structure):
    _fields_ = [("settings", ctypes.POINTER(_RetimeSettings)), ("frames", ctypes.c_void_p), ("nframes", ctypes.c_int32),
                ("sels", ctypes.POINTER(_Selection)), ("nout", ctypes.c_int32), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("fmt", ctypes.c_int32), ("out", ctypes.c_void_p)]


class _LayerJob(ctypes.Structure):
    _fields_ = [("nfg", ctypes.c_int32), ("matte_chan", ctypes.c_int32 * 3), ("sensitivity", ctypes.c_float * 4),
                ("shrink", ctypes.c_float * 3), ("display", ctypes.c_int32), ("points", ctypes.c_void_p),
                ("npoints", ctypes.c_void_p)]


def _layer_job(nfg, sensitivity, matte_chan=None, shrink=None, display=1, points=None, per_frame=False):
    """The tw_layer_job of ``nfg`` FG layers: ``sensitivity`` nfg + 1 values (Main_BG last),
    ``matte_chan`` and ``shrink`` one value per FG layer; ``points`` a list of per-layer lists
    (Main_BG last) of tracking points (x, y at A, x, y at B), or with ``per_frame`` one such list
    per output frame (the clip call)."""
    j = _LayerJob()
    if points is not None:
        frames = points if per_frame else [points]
        counts = np.array([len(layer) for f in frames for layer in f], np.int32)
        flat = np.array([q for f in frames for layer in f for q in layer] or [[0, 0, 0, 0]], np.float32).reshape(-1)
        j.points, j.npoints = flat.ctypes.data, counts.ctypes.data
        j._keep = (flat, counts)
    j.nfg = nfg
    for k, v in enumerate(matte_chan or []):
        j.matte_chan[k] = int(v)
    for k, v in enumerate(sensitivity):
        j.sensitivity[k] = float(v)
    for k, v in enumerate(shrink or []):
        j.shrink[k] = float(v)
    j.display = int(display)
    return j


class _VectorsSettings(ctypes.Structure):
    _fields_ = [("flow", _FlowSettings), ("max_displace", ctypes.c_float), ("rows_reversed", ctypes.c_int32),
                ("display", ctypes.c_int32), ("debug_view", ctypes.c_int32), ("debug_textured", ctypes.c_int32)]


class _TimeParams(ctypes.Structure):
    _fields_ = [("fps_num", ctypes.c_int32), ("fps_den", ctypes.c_int32), ("speed_percent", ctypes.c_double),
                ("nkeys", ctypes.c_int32), ("key_frames", ctypes.POINTER(ctypes.c_double)),
                ("key_values", ctypes.POINTER(ctypes.c_double)), ("key_ease", ctypes.POINTER(ctypes.c_int32)),
                ("vectors", ctypes.c_int32), ("frame_interp", ctypes.c_int32),
                ("blur_compensation", ctypes.c_double), ("remap_mode", ctypes.c_int32), ("frame_num", ctypes.c_double),
                ("nfn_keys", ctypes.c_int32), ("fn_key_frames", ctypes.POINTER(ctypes.c_double)),
                ("fn_key_values", ctypes.POINTER(ctypes.c_double)), ("fn_key_flags", ctypes.POINTER(ctypes.c_int32)),
                ("own_input_rate", ctypes.c_int32), ("input_frame_rate", ctypes.c_double),
                ("frame_time_bias", ctypes.c_double), ("frame_time_plain", ctypes.c_int32),
                ("input_fields", ctypes.c_int32), ("mark_segs", ctypes.c_int32), ("nmark_keys", ctypes.c_int32),
                ("mark_key_frames", ctypes.POINTER(ctypes.c_double)),
                ("mark_key_values", ctypes.POINTER(ctypes.c_double))]


class _VecInFrame(ctypes.Structure):
    _fields_ = [("a", ctypes.c_int32), ("b", ctypes.c_int32), ("has_next", ctypes.c_int32), ("has_prev", ctypes.c_int32),
                ("next_scale", ctypes.c_float * 2), ("prev_scale", ctypes.c_float * 2)]


# ---- the Python mirrors of the reference types -----------------------------------------------------

@dataclass
class FlowSettings:
    """``flow::FlowSettings`` (flow.rs:83-123). ``taps_above_first`` is the vertical tap order of the
    solver's filters: True is the reference's order; False the order of the revision its parity grid
    records."""
    quality: int = 4
    hiq: bool = True
    sensitivity: float = 0.7
    prep_contrast_edge: bool = False
    prep_delinearize: bool = False
    track_alpha: bool = False
    video_range_luma: bool = False
    skip_refine: bool = False
    wrap: bool = False
    taps_above_first: bool = True
    fast_mode: bool = False

    def _c(self):
        return _FlowSettings(self.quality, int(self.hiq), np.float32(self.sensitivity), int(self.prep_contrast_edge),
                             int(self.prep_delinearize), int(self.track_alpha), int(self.video_range_luma),
                             int(self.skip_refine), int(self.wrap), int(self.taps_above_first), int(self.fast_mode))


@dataclass
class Selection:
    """``timeline::Selection`` (timeline.rs:391-414)."""
    s0: float = 0.0
    s1: float = 0.0
    a: int = 0
    b: int = 1
    wa: float = 1.0
    exact: bool = True
    vectors_quality: int = 4
    interp: int = 1

    def _c(self):
        return _Selection(self.s0, self.s1, self.a, self.b, self.wa, int(self.exact), self.vectors_quality,
                          self.interp)

    @staticmethod
    def _from_c(c):
        return Selection(c.s0, c.s1, c.a, c.b, c.wa, bool(c.exact), c.vectors_quality, c.interp)


@dataclass
class EngineSettings:
    """The fields of ``host::EngineSettings`` (host.rs:20-100) that ``compose_vectors`` reads;
    ``gouraud``: the forward warps of codes 2 and 3 as the Gouraud variant (retime-fgbg's stage set)."""
    warp_mode: int = 0
    video_360: bool = False
    wrap_360: bool = False
    quality_high: bool = True
    blur: float = 0.0
    taps_above_first: bool = True
    gouraud: bool = False

    def _c(self):
        return _EngineSettings(self.warp_mode, int(self.video_360), int(self.wrap_360), int(self.quality_high),
                               self.blur, int(self.taps_above_first), int(self.gouraud))


@dataclass
class RetimeSettings:
    """One output frame's settings of the ``retime`` effect beyond its selection."""
    flow: FlowSettings = field(default_factory=FlowSettings)
    compose: EngineSettings = field(default_factory=EngineSettings)
    motion_rows_reversed: bool = True

    def _c(self):
        return _RetimeSettings(self.flow._c(), self.compose._c(), int(self.motion_rows_reversed))


@dataclass
class VectorsSettings:
    """The Create Vectors pass of one layer (create_vectors.rs:97-135): the solver settings (quality 4
    Normal (half res) / 5 Full res, ``track_alpha`` for Track RGB+A), Max Displace in output pixels,
    and whether the engine sees the frames upside down (plugin 02's glue); ``display`` 3 is the Debug
    display of the engine view code ``debug_view`` (0 Blend, 1 Diff, 2 Detail, 3 Edge, 4 Warp),
    its forward warp the Gouraud variant (textured with ``debug_textured``)."""
    flow: FlowSettings = field(default_factory=FlowSettings)
    max_displace: float = 2048.0
    rows_reversed: bool = True
    display: int = 2
    debug_view: int = 4
    debug_textured: bool = False

    def _c(self):
        return _VectorsSettings(self.flow._c(), np.float32(self.max_displace), int(self.rows_reversed), self.display,
                                self.debug_view, int(self.debug_textured))


def fixed_param(v) -> np.float32:
    """A slider value as the plugin reads it: through 16.16 fixed point (crates/fx-core/src/fixed.rs:
    8-10, rounded half away from zero, saturated) and back (frontend.rs:131-133)."""
    f = v * 65536.0 + (-0.5 if v < 0 else 0.5)
    fixed = 0 if np.isnan(f) else int(np.clip(np.trunc(f), -2 ** 31, 2 ** 31 - 1))
    return np.float32(np.float64(fixed) * (1.0 / 65536.0))


def percent_param(v) -> np.float32:
    """A percent slider (a sensitivity) as the fraction the solver takes."""
    return np.float32(fixed_param(v) / np.float32(100.0))


DEBUG_VIEW_CODE = {1: 4, 2: 0, 3: 1, 4: 2, 5: 3}  # Debug View Method -> engine view code (glue.rs:120-130)


def vectors_settings(vector_resolution=1, max_displace=2048.0, sensitivity=70.0, track_rgb_a=False, hiq=True,
                     rows_reversed=True, taps_above_first=True, prep=1, display=2, debug_view_method=1,
                     debug_textured=False) -> VectorsSettings:
    """The settings of plugin 02 (create-vectors) from its parameter values (glue.rs:133-146): the
    popup Vector Resolution, the 16.16 readers of Max Displace and Sensitivity (percent), the Image
    Prep popup (2 Contrast/Edge Enhance, 3 Delinearize), the Display popup (3 Debug) and the Debug
    View Method popup."""
    reader = fixed_param
    sens = percent_param(sensitivity)
    fs = FlowSettings(quality=5 if vector_resolution == 2 else 4, hiq=hiq, sensitivity=sens, track_alpha=track_rgb_a,
                      taps_above_first=taps_above_first, prep_contrast_edge=prep == 2, prep_delinearize=prep == 3)
    return VectorsSettings(flow=fs, max_displace=float(np.float32(1.0) * reader(max_displace)), rows_reversed=rows_reversed,
                           display=display, debug_view=DEBUG_VIEW_CODE.get(debug_view_method, 3),
                           debug_textured=debug_textured)


@dataclass
class TimeParams:
    """The parameters the time map reads (plugins/retime/src/lib.rs:59-99). Popups carry their
    1-based values; ``keys`` / ``fn_keys`` are lists of (frame, value, flags) of a keyed Speed % /
    Frame Num (flags: True or 1 ease, 2 hold); ``remap_mode`` 2 is Frame Number; ``own_input_rate``
    turns "In FPS is Out FPS" off (the input rate ``input_frame_rate``); ``frame_time_bias`` 0.1 is
    the revision the reference's parity grids record (0 reads as its current 0.05);
    ``frame_time_plain`` is retime-fgbg's frame time (no bias branch); ``input_fields`` the Input:
    Fields popup (2 and 3 double the source rate); ``mark_segs`` the Src: Mark Segments popup, or
    ``mark_keys`` its (frame, value) keys (held from one key to the next)."""
    fps: Tuple[int, int] = (24, 1)
    speed_percent: float = 100.0
    keys: Optional[Sequence[Tuple[float, float, int]]] = None
    vectors: int = 5
    frame_interp: int = 2
    blur_compensation: float = 0.0
    remap_mode: int = 1
    frame_num: float = 0.0
    fn_keys: Optional[Sequence[Tuple[float, float, int]]] = None
    own_input_rate: bool = False
    input_frame_rate: float = float(np.float32(29.97))
    frame_time_bias: float = 0.0
    frame_time_plain: bool = False
    input_fields: int = 1
    mark_segs: int = 1
    mark_keys: Optional[Sequence[Tuple[float, float]]] = None

    def _c(self):
        p = _TimeParams()
        p.fps_num, p.fps_den = self.fps
        p.speed_percent = self.speed_percent
        p.vectors, p.frame_interp = self.vectors, self.frame_interp
        p.blur_compensation = self.blur_compensation
        p.remap_mode, p.frame_num = self.remap_mode, self.frame_num
        p.own_input_rate, p.input_frame_rate = int(self.own_input_rate), self.input_frame_rate
        p.frame_time_bias = self.frame_time_bias
        p.frame_time_plain = int(self.frame_time_plain)
        keep = []
        for keys, n_attr, f_attr, v_attr, e_attr in ((self.keys, "nkeys", "key_frames", "key_values", "key_ease"),
                                                     (self.fn_keys, "nfn_keys", "fn_key_frames", "fn_key_values",
                                                      "fn_key_flags")):
            setattr(p, n_attr, 0)
            if keys:
                n = len(keys)
                fr = (ctypes.c_double * n)(*[k[0] for k in keys])
                va = (ctypes.c_double * n)(*[k[1] for k in keys])
                ea = (ctypes.c_int32 * n)(*[int(k[2]) for k in keys])
                setattr(p, n_attr, n)
                setattr(p, f_attr, ctypes.cast(fr, ctypes.POINTER(ctypes.c_double)))
                setattr(p, v_attr, ctypes.cast(va, ctypes.POINTER(ctypes.c_double)))
                setattr(p, e_attr, ctypes.cast(ea, ctypes.POINTER(ctypes.c_int32)))
                keep.append((fr, va, ea))
        p.input_fields, p.mark_segs, p.nmark_keys = self.input_fields, self.mark_segs, 0
        if self.mark_keys:
            n = len(self.mark_keys)
            fr = (ctypes.c_double * n)(*[k[0] for k in self.mark_keys])
            va = (ctypes.c_double * n)(*[k[1] for k in self.mark_keys])
            p.nmark_keys = n
            p.mark_key_frames = ctypes.cast(fr, ctypes.POINTER(ctypes.c_double))
            p.mark_key_values = ctypes.cast(va, ctypes.POINTER(ctypes.c_double))
            keep.append((fr, va))
        p._keep = keep
        return p


# ---- library loading ----------------------------------------------------------------------------

_lib = None


def build(force=False):
    """Compiles the library in tree (nvcc, sm_100a)."""
    from . import buildlib
    return buildlib.build(force=force)


def library():
    """The loaded library; raises when it is not built (there is no other implementation)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built: run `python -c 'import twixtor_b200; twixtor_b200.build()'`")
    L = ctypes.CDLL(LIB_PATH)
    P, i32 = ctypes.c_void_p, ctypes.c_int32
    pimg, pflow = ctypes.POINTER(_Image), ctypes.POINTER(_Flow)
    L.tw_open.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.tw_close.argtypes = [P]
    L.tw_close.restype = None
    L.tw_last_error.argtypes = [P, ctypes.c_char_p, ctypes.c_size_t]
    L.tw_last_error.restype = ctypes.c_size_t
    L.tw_stats.argtypes = [P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.tw_set_stream.argtypes = [P, P]
    L.tw_debug_inject.argtypes = [P, i32, i32]
    L.tw_set_graphs.argtypes = [P, i32]
    L.tw_autotune.argtypes = [P, ctypes.POINTER(_FlowSettings), i32, i32, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32)]
    L.tw_tuning_table.argtypes = [P, ctypes.c_char_p, ctypes.c_size_t]
    L.tw_tuning_table.restype = ctypes.c_size_t
    L.tw_tuning_set.argtypes = [P, i32, i32, i32, i32, i32, i32]
    L.tw_tuning_clear.argtypes = [P]
    L.tw_profile_begin.argtypes = [P, ctypes.c_char_p]
    L.tw_profile_end.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64),
                                 ctypes.POINTER(ctypes.c_double)]
    L.tw_profile_report.argtypes = [P, ctypes.c_char_p, ctypes.c_size_t]
    L.tw_profile_report.restype = ctypes.c_size_t
    L.tw_flow_geometry.argtypes = [ctypes.POINTER(_FlowSettings), i32, i32, P, P, P, P, i32]
    L.tw_solve.argtypes = [P, pimg, pimg, ctypes.POINTER(_FlowSettings), pflow]
    L.tw_solve_pair.argtypes = [P, pimg, pimg, ctypes.POINTER(_FlowSettings), pflow, pflow]
    L.tw_solve_pyramids.argtypes = [P, ctypes.POINTER(_FlowSettings), i32, i32, P, P, P, P, P, P, pflow]
    L.tw_compose_vectors.argtypes = [P, ctypes.POINTER(_EngineSettings), ctypes.POINTER(_Selection), pimg, pimg,
                                     pflow, pflow, pimg]
    L.tw_build_pyramid.argtypes = [P, pimg, ctypes.POINTER(_FlowSettings), P]
    L.tw_inv_warp.argtypes = [P, pimg, pimg, pflow, ctypes.c_float, i32, P]
    L.tw_block_match.argtypes = [P, P, P, P, i32, i32]
    L.tw_blend.argtypes = [P, pimg, pimg, pimg, ctypes.c_float]
    L.tw_smart_blend.argtypes = [P, pimg, pimg, pimg, ctypes.c_float, i32]
    L.tw_set_lanes.argtypes = [P, i32]
    L.tw_compose_layers.argtypes = [P, ctypes.POINTER(_RetimeSettings), ctypes.POINTER(_Selection), pimg, pimg,
                                    ctypes.POINTER(_LayerJob), P, P, pimg]
    L.tw_solve_masked.argtypes = [P, pimg, pimg, ctypes.POINTER(_FlowSettings), P, P, pflow]
    L.tw_forward_warp.argtypes = [P, pimg, pimg, pflow, ctypes.c_float, i32, P]
    L.tw_encode_vectors.argtypes = [P, pimg, pflow, ctypes.c_float]
    L.tw_create_vectors.argtypes = [P, ctypes.POINTER(_VectorsSettings), pimg, pimg, pimg]
    L.tw_vectors_pair.argtypes = [i32, i32, i32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.tw_vectors_frame_pair.argtypes = [i32, i32, i32, i32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.tw_debug_view.argtypes = [P, pimg, pimg, pflow, i32, i32, pimg]
    L.tw_create_vectors_clip.argtypes = [P, ctypes.POINTER(_VectorsSettings), P, i32, P, i32, P, P, i32, i32, i32, P]
    L.tw_check_logf.argtypes = [P, P, P, ctypes.c_int64]
    L.tw_check_powf.argtypes = [P, P, P, P, ctypes.c_int64]
    L.tw_motion_blur.argtypes = [P, pimg, pimg, pflow, ctypes.c_float, i32, ctypes.c_float]
    L.tw_retime_batch_device.argtypes = [P, ctypes.POINTER(_ClipJob), i32]
    L.tw_warp_blend_adjoint.argtypes = [P, P, P, P, P, i32, i32, i32, i32, i32, ctypes.c_float, P, P, P, P, P, P, P, P]
    L.tw_fill_holes.argtypes = [P, pimg, P, i32, i32]
    L.tw_from_frame.argtypes = [P, P, i32, i32, i32, P]
    L.tw_to_frame.argtypes = [P, P, i32, i32, i32, P]
    L.tw_select.argtypes = [ctypes.POINTER(_TimeParams), i32, i32, i32, ctypes.POINTER(_Selection)]
    L.tw_shard.argtypes = [i32, i32, i32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.tw_source_window.argtypes = [ctypes.POINTER(_Selection), i32, i32, ctypes.POINTER(ctypes.c_int32),
                                   ctypes.POINTER(ctypes.c_int32)]
    L.tw_retime_frame.argtypes = [P, ctypes.POINTER(_RetimeSettings), ctypes.POINTER(_Selection), P, P, i32, i32,
                                  i32, P]
    L.tw_retime_clip.argtypes = [P, ctypes.POINTER(_RetimeSettings), P, i32, ctypes.POINTER(_Selection), i32, i32,
                                 i32, i32, P]
    L.tw_retime_clip_device.argtypes = [P, ctypes.POINTER(_RetimeSettings), P, i32, ctypes.POINTER(_Selection), i32,
                                        i32, i32, i32, P]
    L.tw_retime_layers_clip.argtypes = [P, ctypes.POINTER(_RetimeSettings), P, i32, ctypes.POINTER(_LayerJob), P, P,
                                        ctypes.POINTER(_Selection), i32, i32, i32, i32, P]
    pvf = ctypes.POINTER(_VecInFrame)
    L.tw_select_vectors_in.argtypes = [ctypes.POINTER(_TimeParams), i32, i32, i32, ctypes.POINTER(_Selection), pvf]
    L.tw_decode_vectors.argtypes = [P, pimg, ctypes.c_float, pflow]
    L.tw_flow_from_vectors.argtypes = [P, pimg, ctypes.c_float, ctypes.c_float, ctypes.c_float, i32, pflow]
    L.tw_fill_flow_holes.argtypes = [P, pflow, P, i32, i32]
    L.tw_invert_flow.argtypes = [P, pflow, i32, i32, pflow]
    L.tw_retime_frame_vectors.argtypes = [P, ctypes.POINTER(_RetimeSettings), ctypes.POINTER(_Selection), pvf,
                                          ctypes.c_float, P, P, P, P, i32, i32, i32, P]
    L.tw_vectors_in_clip.argtypes = [P, ctypes.POINTER(_RetimeSettings), P, i32, P, i32, P, i32,
                                     ctypes.POINTER(_Selection), pvf, i32, ctypes.c_float, i32, i32, i32, P]
    L.tw_vectors_in_clip_device.argtypes = L.tw_vectors_in_clip.argtypes
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _img(a, w, h, fmt):
    a = np.ascontiguousarray(a)
    assert a.dtype == DTYPES[fmt] and a.size == w * h * 4, "engine image of the wrong size or depth"
    return _Image(w, h, fmt, a.ctypes.data, a.nbytes), a


def vectors_pair(n: int, track_frame: int = 1, fps: Tuple[int, int] = (24, 1), debug: bool = False) -> Tuple[int, int]:
    """The clip frames (X, Y) of output frame ``n`` of Create Vectors (create_vectors.rs:59-97); with
    ``debug`` the Debug display's pair."""
    ts = 100 if fps[1] == 1 else fps[1]
    a, b = ctypes.c_int32(), ctypes.c_int32()
    rc = library().tw_vectors_frame_pair(n, ts, track_frame, int(debug), ctypes.byref(a), ctypes.byref(b))
    if rc:
        raise BadParam(rc, "bad argument")
    return a.value, b.value


def select(params: TimeParams, n: int, width: int, height: int) -> Selection:
    """``timeline::select`` of output frame ``n`` (the Speed map, host scalars in the library)."""
    out = _Selection()
    rc = library().tw_select(ctypes.byref(params._c()), n, width, height, ctypes.byref(out))
    if rc:
        raise BadParam(rc, "tw_select")
    return Selection._from_c(out)


@dataclass
class VecInFrame:
    """One output frame of the Vectors In render beyond its selection (tw_vecin_frame): the clip
    frames of the pair, which vector layers are present and their Vec Scale at the fetch times."""
    a: int = 0
    b: int = 1
    has_next: bool = True
    has_prev: bool = True
    next_scale: Tuple[float, float] = (1.0, 1.0)
    prev_scale: Tuple[float, float] = (1.0, 1.0)

    def _c(self):
        return _VecInFrame(self.a, self.b, int(self.has_next), int(self.has_prev),
                           (ctypes.c_float * 2)(*self.next_scale), (ctypes.c_float * 2)(*self.prev_scale))


def select_vectors_in(params: TimeParams, n: int, width: int, height: int, has_next=True, has_prev=True,
                      next_scale=(1.0, 1.0), prev_scale=(1.0, 1.0)) -> Tuple[Selection, VecInFrame]:
    """The selection and the clip frames of output frame ``n`` of the Vectors In effect (its time
    map: the input rate 30, the output rate ``params.fps``; tw_select_vectors_in)."""
    out, fr = _Selection(), _VecInFrame()
    rc = library().tw_select_vectors_in(ctypes.byref(params._c()), n, width, height, ctypes.byref(out),
                                        ctypes.byref(fr))
    if rc:
        raise BadParam(rc, "tw_select_vectors_in")
    return Selection._from_c(out), VecInFrame(fr.a, fr.b, has_next, has_prev, tuple(next_scale), tuple(prev_scale))


def vectors_in_settings(warping: int = 2, quality_high=True, blur=0.0, rows_reversed=True, taps_above_first=True,
                        gouraud=True) -> "RetimeSettings":
    """The settings of the Vectors In render (plugins/vectors-in/src/glue.rs:204-243): the Warping
    popup (1 Inverse, 2 Forward) as the warp code, the blur compensation, and its three orders
    (bottom-up rows, the tap above first in the fills, the Gouraud forward warp); all three False
    is the revision the reference's parity grid records."""
    return RetimeSettings(FlowSettings(), EngineSettings(warp_mode=2 if warping == 2 else 0, quality_high=quality_high,
                                                         blur=float(fixed_param(blur)),
                                                         taps_above_first=taps_above_first, gouraud=gouraud),
                          motion_rows_reversed=rows_reversed)


def shard(nout: int, nranks: int, rank: int) -> Tuple[int, int]:
    """The output frames [lo, hi) rank ``rank`` of ``nranks`` renders (tw_shard)."""
    lo, hi = ctypes.c_int32(), ctypes.c_int32()
    rc = library().tw_shard(nout, nranks, rank, ctypes.byref(lo), ctypes.byref(hi))
    if rc:
        raise BadParam(rc, "tw_shard")
    return lo.value, hi.value


def source_window(sels, nframes: int) -> Tuple[int, int]:
    """The clip frames [first, last] the selections read (tw_source_window); first > last: none."""
    arr = (_Selection * max(len(sels), 1))(*[s._c() for s in sels])
    first, last = ctypes.c_int32(), ctypes.c_int32()
    rc = library().tw_source_window(arr, len(sels), nframes, ctypes.byref(first), ctypes.byref(last))
    if rc:
        raise BadParam(rc, "tw_source_window")
    return first.value, last.value


def rebase(sels, first: int, nframes: int):
    """The selections with their frames counted from the window's first frame (a frame outside the
    clip stays outside: -1), for a rank that holds only frames [first, ...] of the clip."""
    out = []
    for s in sels:
        c = Selection._from_c(s._c())
        c.a = c.a - first if 0 <= c.a < nframes else -1
        c.b = c.b - first if 0 <= c.b < nframes else -1
        out.append(c)
    return out


def flow_geometry(settings: FlowSettings, width: int, height: int):
    """(flow width, flow height, [(w, h) per level]) of a solve (FlowSettings::geometry)."""
    fw, fh, nl = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    sizes = np.zeros(64, np.int32)
    rc = library().tw_flow_geometry(ctypes.byref(settings._c()), width, height, ctypes.byref(fw), ctypes.byref(fh),
                                    ctypes.byref(nl), _ptr(sizes), 32)
    if rc:
        raise (_ERRORS.get(rc, StageError))(rc, "flow geometry")
    return fw.value, fh.value, [(int(sizes[2 * i]), int(sizes[2 * i + 1])) for i in range(nl.value)]


class Device:
    """One CUDA device with the library's context (the reference's ``exec::open``,
    device/exec/open.rs:72-116). Implements the ``Stages`` methods."""

    def __init__(self, device: int = 0):
        L = library()
        h = ctypes.c_void_p()
        rc = L.tw_open(device, ctypes.byref(h))
        if rc:
            raise StageError(rc, f"tw_open({device}) failed")
        self._h = h
        self._L = L

    def close(self):
        if self._h:
            self._L.tw_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc):
        if rc:
            n = self._L.tw_last_error(self._h, None, 0)
            buf = ctypes.create_string_buffer(n + 1)
            self._L.tw_last_error(self._h, buf, n + 1)
            raise (_ERRORS.get(rc, StageError))(rc, buf.value.decode())

    def autotune(self, settings: FlowSettings, width: int, height: int, path: Optional[str] = None) -> int:
        """Times the launch shapes of every level size of a width x height solve and keeps the
        fastest (tw_autotune); ``path``: the JSON cache read first and written after. Returns the
        number of level sizes measured."""
        n = ctypes.c_int32()
        self._check(self._L.tw_autotune(self._h, ctypes.byref(settings._c()), width, height,
                                        None if path is None else path.encode(), ctypes.byref(n)))
        return n.value

    def tuning_table(self) -> str:
        n = self._L.tw_tuning_table(self._h, None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        self._L.tw_tuning_table(self._h, buf, n + 1)
        return buf.value.decode()

    def tuning_set(self, width, height, iter_tile, iter_threads, bm_rows_threads, bm_cols_threads):
        self._check(self._L.tw_tuning_set(self._h, width, height, iter_tile, iter_threads, bm_rows_threads,
                                          bm_cols_threads))

    def tuning_clear(self):
        self._check(self._L.tw_tuning_clear(self._h))

    def set_graphs(self, on: bool):
        """CUDA graphs of the clip calls' per-frame pipeline (tw_set_graphs; on by default)."""
        self._check(self._L.tw_set_graphs(self._h, int(bool(on))))

    def debug_inject(self, kind: int, n: int = 1):
        """Arms a host-injected failure (tw_debug_inject): INJECT_ALLOC fails the n-th device
        allocation, INJECT_STATUS sets the device status word of the n-th output frame."""
        self._check(self._L.tw_debug_inject(self._h, int(kind), int(n)))

    def set_stream(self, stream_handle: int):
        """Enqueue on a caller's CUDA stream (e.g. ``torch.cuda.current_stream().cuda_stream``)."""
        self._check(self._L.tw_set_stream(self._h, ctypes.c_void_p(stream_handle)))

    def profile_begin(self, kernel: str):
        self._check(self._L.tw_profile_begin(self._h, kernel.encode()))

    def profile_report(self) -> str:
        """Per-kernel table of the launches since ``profile_begin("*")``."""
        n = self._L.tw_profile_report(self._h, None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        self._L.tw_profile_report(self._h, buf, n + 1)
        return buf.value.decode()

    def profile_end(self):
        """(device ms, launches, algorithmic bytes) of the profiled kernel since profile_begin."""
        ms, n, b = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_double()
        self._check(self._L.tw_profile_end(self._h, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(b)))
        return ms.value, n.value, b.value

    def stats(self):
        k, b = ctypes.c_uint64(), ctypes.c_uint64()
        self._L.tw_stats(self._h, ctypes.byref(k), ctypes.byref(b))
        return {"kernel_launches": k.value, "device_bytes": b.value}

    # ---- Stages ---------------------------------------------------------------------------------

    def solve(self, x, y, width, height, fmt, settings: FlowSettings):
        """``flow::solve``: X(p) ~ Y(p + out(p)) at the working resolution."""
        fw, fh, _ = flow_geometry(settings, width, height)
        out = np.zeros(fw * fh * 2, np.float32)
        xi, xa = _img(x, width, height, fmt)
        yi, ya = _img(y, width, height, fmt)
        fo = _Flow(fw, fh, out.ctypes.data)
        self._check(self._L.tw_solve(self._h, ctypes.byref(xi), ctypes.byref(yi), ctypes.byref(settings._c()),
                                     ctypes.byref(fo)))
        return out, (fw, fh)

    def solve_pyramids(self, settings: FlowSettings, width, height, x_levels, y_levels, mask_x=None, mask_y=None,
                       user_d=None, user_w=None):
        """``flow::extras::solve_pyramids_with`` on given band pyramids (levels concatenated finest
        first) with the optional mask pyramids and user displacement: the flow and its size."""
        fw, fh, _ = flow_geometry(settings, width, height)
        out = np.zeros(fw * fh * 2, np.float32)
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32)
                for a in (x_levels, y_levels, mask_x, mask_y, user_d, user_w)]
        fo = _Flow(fw, fh, out.ctypes.data)
        self._check(self._L.tw_solve_pyramids(self._h, ctypes.byref(settings._c()), width, height,
                                              *[_ptr(a) for a in arrs], ctypes.byref(fo)))
        return out, (fw, fh)

    def solve_pair(self, a, b, width, height, fmt, settings: FlowSettings):
        """``flow::solve_pair``: (f_ab, f_ba, (flow width, flow height))."""
        fw, fh, _ = flow_geometry(settings, width, height)
        f_ab = np.zeros(fw * fh * 2, np.float32)
        f_ba = np.zeros(fw * fh * 2, np.float32)
        ai, aa = _img(a, width, height, fmt)
        bi, ba = _img(b, width, height, fmt)
        fa, fb = _Flow(fw, fh, f_ab.ctypes.data), _Flow(fw, fh, f_ba.ctypes.data)
        self._check(self._L.tw_solve_pair(self._h, ctypes.byref(ai), ctypes.byref(bi), ctypes.byref(settings._c()),
                                          ctypes.byref(fa), ctypes.byref(fb)))
        return f_ab, f_ba, (fw, fh)

    def compose_vectors(self, settings: EngineSettings, sel: Selection, a, b, width, height, fmt, f_ab, f_ba,
                        flow_size):
        """``compose::compose_vectors`` (warping code 0): the engine image of the output frame."""
        fw, fh = flow_size
        out = np.zeros(width * height * 4, DTYPES[fmt])
        ai, aa = _img(a, width, height, fmt)
        bi, ba = _img(b, width, height, fmt)
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        fab = _Flow(fw, fh, f_ab.ctypes.data) if f_ab is not None else None
        fba = _Flow(fw, fh, f_ba.ctypes.data) if f_ba is not None else None
        self._check(self._L.tw_compose_vectors(self._h, ctypes.byref(settings._c()), ctypes.byref(sel._c()),
                                               ctypes.byref(ai), ctypes.byref(bi),
                                               ctypes.byref(fab) if fab else None, ctypes.byref(fba) if fba else None,
                                               ctypes.byref(oi)))
        return out

    # ---- single stages ----------------------------------------------------------------------------

    def build_pyramid(self, img, width, height, fmt, settings: FlowSettings):
        _, _, sizes = flow_geometry(settings, width, height)
        out = np.zeros(sum(w * h for w, h in sizes), np.float32)
        ii, ia = _img(img, width, height, fmt)
        self._check(self._L.tw_build_pyramid(self._h, ctypes.byref(ii), ctypes.byref(settings._c()), _ptr(out)))
        levels, off = [], 0
        for w, h in sizes:
            levels.append(out[off:off + w * h].reshape(h, w))
            off += w * h
        return levels

    def block_match(self, a, b, flow, width, height):
        """``flow::block_match`` on one level: returns the refined flow (interleaved)."""
        a = np.ascontiguousarray(a, np.float32).reshape(-1)
        b = np.ascontiguousarray(b, np.float32).reshape(-1)
        f = np.array(flow, np.float32).reshape(-1)
        self._check(self._L.tw_block_match(self._h, _ptr(a), _ptr(b), _ptr(f), width, height))
        return f

    def inv_warp(self, src, width, height, fmt, flow, flow_size, amount, hold=True, coverage=False, is360=False):
        """``warp::inv_warp`` (mode 1): hold edges, or the fade with coverage, or the 360 wrap."""
        fw, fh = flow_size
        out = np.zeros(width * height * 4, DTYPES[fmt])
        si, sa = _img(src, width, height, fmt)
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        flow = np.ascontiguousarray(flow, np.float32)
        fl = _Flow(fw, fh, flow.ctypes.data)
        cov = np.zeros(width * height, np.uint8) if coverage else None
        self._check(self._L.tw_inv_warp(self._h, ctypes.byref(oi), ctypes.byref(si), ctypes.byref(fl),
                                        np.float32(amount), int(hold) | (2 if is360 else 0), _ptr(cov)))
        return (out, cov) if coverage else out

    def blend(self, a, b, width, height, fmt, w):
        out = np.zeros(width * height * 4, DTYPES[fmt])
        ai, aa = _img(a, width, height, fmt)
        bi, ba = _img(b, width, height, fmt)
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        self._check(self._L.tw_blend(self._h, ctypes.byref(oi), ctypes.byref(ai), ctypes.byref(bi), np.float32(w)))
        return out

    def forward_warp(self, src, width, height, fmt, flow, flow_size, amount, pyramid=True, coverage=False):
        """``forward::forward_warp_with``: the engine image (and the coverage bytes with coverage=True).
        pyramid=False is the Gouraud variant."""
        fw, fh = flow_size
        out = np.zeros(width * height * 4, DTYPES[fmt])
        si, sa = _img(src, width, height, fmt)
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        flow = np.ascontiguousarray(flow, np.float32)
        fl = _Flow(fw, fh, flow.ctypes.data)
        cov = np.zeros(width * height, np.uint8) if coverage else None
        self._check(self._L.tw_forward_warp(self._h, ctypes.byref(oi), ctypes.byref(si), ctypes.byref(fl), np.float32(amount),
                                            int(pyramid), _ptr(cov)))
        return (out, cov) if coverage else out

    def encode_vectors(self, flow, flow_size, width, height, fmt, scale):
        """``vectors::encode_vectors``: the encoded vector image (engine samples) of a flow."""
        fw, fh = flow_size
        out = np.zeros(width * height * 4, DTYPES[fmt])
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        flow = np.ascontiguousarray(flow, np.float32)
        fl = _Flow(fw, fh, flow.ctypes.data)
        self._check(self._L.tw_encode_vectors(self._h, ctypes.byref(oi), ctypes.byref(fl), np.float32(scale)))
        return out

    def create_vectors(self, settings: VectorsSettings, x, y, width, height, fmt):
        """``create_vectors::create_vectors_on`` for one layer: engine images in, the encoded engine image out."""
        out = np.zeros(width * height * 4, DTYPES[fmt])
        xi, xa = _img(x, width, height, fmt)
        yi, ya = _img(y, width, height, fmt)
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        self._check(self._L.tw_create_vectors(self._h, ctypes.byref(settings._c()), ctypes.byref(xi), ctypes.byref(yi),
                                              ctypes.byref(oi)))
        return out

    def create_vectors_clip(self, settings: VectorsSettings, frames, nframes, pairs, width, height, fmt, out=None,
                            points=None):
        """Create Vectors over a clip in host memory: output frame k encodes the flow from clip frame
        pairs[k][0] to pairs[k][1]; ``points[k]`` the tracking points in use of frame k (x, y at X,
        x, y at Y; host rows). Returns the output wire frames back to back."""
        frames = np.ascontiguousarray(frames)
        fs = width * height * 4
        pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1)
        nout = pairs.size // 2
        if out is None:
            out = np.zeros(nout * fs, DTYPES[fmt])
        pts = npts = None
        if points is not None:
            npts = np.array([len(x) for x in points], np.int32)
            pts = np.array([q for x in points for q in x] or [[0, 0, 0, 0]], np.float32).reshape(-1)
        self._check(self._L.tw_create_vectors_clip(self._h, ctypes.byref(settings._c()), _ptr(frames), nframes, _ptr(pairs),
                                                   nout, _ptr(pts), _ptr(npts), width, height, fmt, _ptr(out)))
        return out

    def solve_masked(self, x, y, width, height, fmt, settings: FlowSettings, matte_x=None, matte_y=None):
        """``flow::extras::solve_pyramids_with`` with the (ungated) mask pyramids of a layer's mattes
        (``width * height`` values 0..1 at X and at Y): the flow X -> Y at the working size."""
        _, _, sizes = flow_geometry(settings, width, height)
        fw, fh = sizes[0]
        out = np.zeros(fw * fh * 2, np.float32)
        xi, xa = _img(x, width, height, fmt)
        yi, ya = _img(y, width, height, fmt)
        fl = _Flow(fw, fh, out.ctypes.data)
        mx = None if matte_x is None else np.ascontiguousarray(matte_x, np.float32)
        my = None if matte_y is None else np.ascontiguousarray(matte_y, np.float32)
        self._check(self._L.tw_solve_masked(self._h, ctypes.byref(xi), ctypes.byref(yi), ctypes.byref(settings._c()),
                                            _ptr(mx), _ptr(my), ctypes.byref(fl)))
        return out

    def compose_layers(self, settings: RetimeSettings, sel: Selection, a, b, width, height, fmt, mattes_a, mattes_b,
                       sensitivity, shrink=None, display=1, points=None):
        """The layered composition with plates of one in-between frame (layers/plates.rs): ``mattes_a`` /
        ``mattes_b`` the FG raw mattes at A and B (FG1 first, ``width * height`` floats each),
        ``sensitivity`` one value per layer, Main_BG last, ``shrink`` the inverse matte shrink per FG
        layer, ``display`` the Display popup (the group composed), ``points`` the tracking points per
        layer (x, y at A, x, y at B in the images' rows). Returns the engine image."""
        nfg = len(mattes_a)
        job = _layer_job(nfg, sensitivity, shrink=shrink, display=display, points=points)
        out = np.zeros(width * height * 4, DTYPES[fmt])
        ai, aa = _img(a, width, height, fmt)
        bi, ba = _img(b, width, height, fmt)
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        ma = np.ascontiguousarray(np.concatenate(mattes_a) if nfg else np.zeros(1), np.float32)
        mb = np.ascontiguousarray(np.concatenate(mattes_b) if nfg else np.zeros(1), np.float32)
        self._check(self._L.tw_compose_layers(self._h, ctypes.byref(settings._c()), ctypes.byref(sel._c()), ctypes.byref(ai),
                                              ctypes.byref(bi), ctypes.byref(job), _ptr(ma), _ptr(mb), ctypes.byref(oi)))
        return out

    def set_lanes(self, lanes):
        """Output frames in flight in the clip calls (1..8)."""
        self._check(self._L.tw_set_lanes(self._h, int(lanes)))

    def check_logf(self, x):
        """The device's logf of the forward warp's mip level (equal to the host C library's)."""
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros_like(x)
        self._check(self._L.tw_check_logf(self._h, _ptr(x), _ptr(out), x.size))
        return out

    def motion_blur(self, src, width, height, fmt, flow, flow_size, amount, hiq, shutter):
        """``warp::blurcomp::motion_blur`` of an engine image (the Blur Compensation primitive)."""
        fw, fh = flow_size
        out = np.zeros(width * height * 4, DTYPES[fmt])
        si, sa = _img(src, width, height, fmt)
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        fl = np.ascontiguousarray(flow, np.float32)
        self._check(self._L.tw_motion_blur(self._h, ctypes.byref(oi), ctypes.byref(si), ctypes.byref(_Flow(fw, fh, fl.ctypes.data)),
                                           np.float32(amount), int(hiq), np.float32(shutter)))
        return out

    def warp_blend_adjoint(self, a, b, f_ab, f_ba, width, height, flow_w, flow_h, batch, wa, target=0, grad_out=0,
                           out=0, loss=0, da=0, db=0, df_ab=0, df_ba=0):
        """tw_warp_blend_adjoint on DEVICE pointers (ints, e.g. tensor.data_ptr(); 0 for none): the
        forward of warp + blend and, from the L1 loss against ``target`` or from ``grad_out``, the
        gradients added into ``da``, ``db``, ``df_ab``, ``df_ba``. Enqueued on the device's stream."""
        vp = ctypes.c_void_p
        self._check(self._L.tw_warp_blend_adjoint(self._h, vp(a), vp(b), vp(f_ab), vp(f_ba), width, height, flow_w, flow_h,
                                                  batch, np.float32(wa), vp(target or None), vp(grad_out or None),
                                                  vp(out or None), vp(loss or None), vp(da or None), vp(db or None),
                                                  vp(df_ab or None), vp(df_ba or None)))

    def check_powf(self, x, y):
        """The device's powf of the Delinearize prep (the plugin runtime's, crt_powf.rs)."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(np.broadcast_to(np.asarray(y, np.float32), x.shape), np.float32)
        out = np.zeros_like(x)
        self._check(self._L.tw_check_powf(self._h, _ptr(x), _ptr(y), _ptr(out), x.size))
        return out

    def smart_blend(self, p1, p2, width, height, fmt, w, binary=False):
        """``smartblend::smart_blend`` (or ``smart_blend_binary``) of two engine images."""
        out = np.zeros(width * height * 4, DTYPES[fmt])
        ai, aa = _img(p1, width, height, fmt)
        bi, ba = _img(p2, width, height, fmt)
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        self._check(self._L.tw_smart_blend(self._h, ctypes.byref(oi), ctypes.byref(ai), ctypes.byref(bi), np.float32(w),
                                           int(binary)))
        return out

    def fill_holes(self, img, width, height, fmt, mask, taps_above_first=True):
        """``holefill::fill_holes_masked_with`` (is360 off): the filled copy of an engine image. The
        mask's dtype picks its kind: uint8, uint16 or float32 (one value per pixel)."""
        kind = {np.dtype(np.uint8): 1, np.dtype(np.uint16): 2, np.dtype(np.float32): 3}[np.asarray(mask).dtype]
        mask = np.ascontiguousarray(mask)
        if mask.size != width * height:
            raise Mismatch(ERR_MISMATCH, f"hole fill: mask has {mask.size} entries for an image of {width}x{height}")
        out = np.array(img, DTYPES[fmt], copy=True).reshape(-1)
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        self._check(self._L.tw_fill_holes(self._h, ctypes.byref(oi), _ptr(mask), kind, int(taps_above_first)))
        return out

    def decode_vectors(self, vec, width, height, fmt, max_displace):
        """``vectors::decode_vectors`` of an engine image: the interleaved (w x h x 2) flow."""
        vi, vec = _img(vec, width, height, fmt)
        out = np.zeros(width * height * 2, np.float32)
        fo = _Flow(width, height, out.ctypes.data)
        self._check(self._L.tw_decode_vectors(self._h, ctypes.byref(vi), np.float32(max_displace), ctypes.byref(fo)))
        return out

    def flow_from_vectors(self, vec, width, height, fmt, max_displace, scale=(1.0, 1.0), taps_above_first=True):
        """``compose::flow_from_vector_image_with``: decode, flow hole fill, Vec Scale."""
        vi, vec = _img(vec, width, height, fmt)
        out = np.zeros(width * height * 2, np.float32)
        fo = _Flow(width, height, out.ctypes.data)
        self._check(self._L.tw_flow_from_vectors(self._h, ctypes.byref(vi), np.float32(max_displace),
                                                 np.float32(scale[0]), np.float32(scale[1]), int(taps_above_first),
                                                 ctypes.byref(fo)))
        return out

    def fill_flow_holes(self, flow, width, height, mask, taps_above_first=True):
        """``holefill::fill_flow_holes_with`` (is360 off): the filled copy of an interleaved flow; the
        mask's dtype picks its kind as in fill_holes."""
        kind = {np.dtype(np.uint8): 1, np.dtype(np.uint16): 2, np.dtype(np.float32): 3}[np.asarray(mask).dtype]
        mask = np.ascontiguousarray(mask)
        out = np.array(flow, np.float32, copy=True).reshape(-1)
        fo = _Flow(width, height, out.ctypes.data)
        self._check(self._L.tw_fill_flow_holes(self._h, ctypes.byref(fo), _ptr(mask), kind, int(taps_above_first)))
        return out

    def invert_flow(self, flow, width, height, pyramid=True, taps_above_first=True):
        """``compose::invert_flow_on``: the inversion of a (w x h) interleaved flow."""
        flow = np.ascontiguousarray(flow, np.float32)
        out = np.zeros(width * height * 2, np.float32)
        fi, fo = _Flow(width, height, flow.ctypes.data), _Flow(width, height, out.ctypes.data)
        self._check(self._L.tw_invert_flow(self._h, ctypes.byref(fi), int(pyramid), int(taps_above_first),
                                           ctypes.byref(fo)))
        return out

    def retime_frame_vectors(self, settings: "RetimeSettings", sel: "Selection", vf: VecInFrame, max_displace,
                             wire_a, wire_b, wire_next, wire_prev, width, height, fmt, out=None):
        """One output wire frame of the single layer Vectors In render (tw_retime_frame_vectors)."""
        if out is None:
            out = np.zeros(width * height * 4, DTYPES[fmt])
        keep = [None if w is None else np.ascontiguousarray(w) for w in (wire_a, wire_b, wire_next, wire_prev)]
        self._check(self._L.tw_retime_frame_vectors(self._h, ctypes.byref(settings._c()), ctypes.byref(sel._c()),
                                                    ctypes.byref(vf._c()), np.float32(max_displace),
                                                    *[_ptr(k) for k in keep], width, height, fmt, _ptr(out)))
        return out

    def vectors_in_clip(self, settings: "RetimeSettings", frames, nframes, next_clip, n_next, prev_clip, n_prev, sels,
                        vfs, max_displace, width, height, fmt, out=None):
        """Output frames ``sels`` / ``vfs`` of the single layer Vectors In render over clips in host
        memory (tw_vectors_in_clip); a vector clip None is a layer that is not set."""
        fs = width * height * 4
        if out is None:
            out = np.zeros(len(sels) * fs, DTYPES[fmt])
        frames = np.ascontiguousarray(frames)
        nc = None if next_clip is None else np.ascontiguousarray(next_clip)
        pc = None if prev_clip is None else np.ascontiguousarray(prev_clip)
        sa = (_Selection * max(len(sels), 1))(*[s._c() for s in sels])
        va = (_VecInFrame * max(len(vfs), 1))(*[v._c() for v in vfs])
        self._check(self._L.tw_vectors_in_clip(self._h, ctypes.byref(settings._c()), _ptr(frames), nframes, _ptr(nc),
                                               n_next if nc is not None else 0, _ptr(pc),
                                               n_prev if pc is not None else 0, sa, va, len(sels),
                                               np.float32(max_displace), width, height, fmt, _ptr(out)))
        return out

    def vectors_in_clip_device(self, settings: "RetimeSettings", frames_ptr, nframes, next_ptr, n_next, prev_ptr,
                               n_prev, sels, vfs, max_displace, width, height, fmt, out_ptr):
        """tw_vectors_in_clip_device on device pointers (ints; 0 or None for a layer that is not set)."""
        sa = (_Selection * max(len(sels), 1))(*[s._c() for s in sels])
        va = (_VecInFrame * max(len(vfs), 1))(*[v._c() for v in vfs])
        self._check(self._L.tw_vectors_in_clip_device(self._h, ctypes.byref(settings._c()), frames_ptr, nframes,
                                                      next_ptr or None, n_next, prev_ptr or None, n_prev, sa, va,
                                                      len(sels), np.float32(max_displace), width, height, fmt,
                                                      out_ptr))

    def debug_view(self, x, y, width, height, fmt, flow, flow_size, code, gouraud=True):
        """``debug::debug_view_on``: view code 0 Blend, 1 Diff, 2 Detail, 3 Edge, 4 Warp of engine
        images x and y by the interleaved flow of ``flow_size``."""
        xi, x = _img(x, width, height, fmt)
        yi, y = _img(y, width, height, fmt)
        flow = np.ascontiguousarray(flow, np.float32)
        fi = _Flow(flow_size[0], flow_size[1], flow.ctypes.data)
        out = np.zeros(width * height * 4, DTYPES[fmt])
        oi = _Image(width, height, fmt, out.ctypes.data, out.nbytes)
        self._check(self._L.tw_debug_view(self._h, ctypes.byref(xi), ctypes.byref(yi), ctypes.byref(fi), code,
                                          int(gouraud), ctypes.byref(oi)))
        return out

    def from_frame(self, wire, width, height, fmt):
        wire = np.ascontiguousarray(wire)
        out = np.zeros(width * height * 4, DTYPES[fmt])
        self._check(self._L.tw_from_frame(self._h, _ptr(wire), width, height, fmt, _ptr(out)))
        return out

    def to_frame(self, engine, width, height, fmt):
        engine = np.ascontiguousarray(engine)
        out = np.zeros(width * height * 4, DTYPES[fmt])
        self._check(self._L.tw_to_frame(self._h, _ptr(engine), width, height, fmt, _ptr(out)))
        return out

    # ---- whole frames -------------------------------------------------------------------------------

    def retime_frame(self, settings: RetimeSettings, sel: Selection, wire_a, wire_b, width, height, fmt, out=None):
        """One output wire frame of the ``retime`` core; ``wire_a`` / ``wire_b`` None are blank frames."""
        if out is None:
            out = np.zeros(width * height * 4, DTYPES[fmt])
        self._check(self._L.tw_retime_frame(self._h, ctypes.byref(settings._c()), ctypes.byref(sel._c()),
                                            _ptr(wire_a), _ptr(wire_b), width, height, fmt, _ptr(out)))
        return out

    def retime_clip(self, settings: RetimeSettings, frames, nframes: int, sels, width, height, fmt, out=None):
        """Output frames ``sels`` of a clip in host memory (wire frames back to back in ``frames``;
        page-locked memory makes the copies asynchronous). Returns the output frames back to back."""
        frames = np.ascontiguousarray(frames)
        fs = width * height * 4
        if out is None:
            out = np.zeros(len(sels) * fs, DTYPES[fmt])
        arr = (_Selection * len(sels))(*[s._c() for s in sels])
        self._check(self._L.tw_retime_clip(self._h, ctypes.byref(settings._c()), _ptr(frames), nframes, arr, len(sels),
                                           width, height, fmt, _ptr(out)))
        return out

    def retime_layers_clip(self, settings: RetimeSettings, frames, nframes: int, mattes, matte_chan, sensitivity, sels,
                           width, height, fmt, matte_nframes=None, out=None, shrink=None, display=1, points=None):
        """retime-fgbg with FG matte layers over a clip in host memory: ``mattes`` the FG1.. matte
        clips (wire frames back to back, the footage's size and format), ``matte_chan`` their channel
        popups (1 R, 2 G, 3 B, else alpha), ``sensitivity`` one value 0..1 per layer, Main_BG last,
        ``shrink`` the inverse matte shrink per FG layer (pixels), ``display`` the Display popup,
        ``points`` per output frame the tracking points of every layer (x, y at A, x, y at B, host
        rows). Returns the output frames ``sels`` back to back."""
        frames = np.ascontiguousarray(frames)
        fs = width * height * 4
        if out is None:
            out = np.zeros(len(sels) * fs, DTYPES[fmt])
        nfg = len(mattes)
        mattes = [np.ascontiguousarray(m) for m in mattes]
        clips = (ctypes.c_void_p * max(nfg, 1))(*[m.ctypes.data for m in mattes])
        job = _layer_job(nfg, sensitivity, matte_chan=matte_chan, shrink=shrink, display=display, points=points,
                         per_frame=True)
        counts = None if matte_nframes is None else np.ascontiguousarray(matte_nframes, np.int32)
        arr = (_Selection * max(len(sels), 1))(*[x._c() for x in sels])
        self._check(self._L.tw_retime_layers_clip(self._h, ctypes.byref(settings._c()), _ptr(frames), nframes,
                                                  ctypes.byref(job), clips, _ptr(counts),
                                                  arr, len(sels), width, height, fmt, _ptr(out)))
        return out

    def retime_batch_device(self, jobs):
        """Several clips in one call (tw_retime_batch_device): ``jobs`` is a list of dicts with
        settings (RetimeSettings), frames (device pointer), nframes, sels, width, height, fmt and out
        (device pointer, len(sels) output frames)."""
        keep = []
        arr = (_ClipJob * max(len(jobs), 1))()
        for i, j in enumerate(jobs):
            st = j["settings"]._c()
            sl = (_Selection * max(len(j["sels"]), 1))(*[x._c() for x in j["sels"]])
            keep += [st, sl]
            arr[i] = _ClipJob(ctypes.pointer(st), ctypes.c_void_p(j["frames"]), j["nframes"], sl, len(j["sels"]),
                              j["width"], j["height"], j["fmt"], ctypes.c_void_p(j["out"]))
        self._check(self._L.tw_retime_batch_device(self._h, arr, len(jobs)))

    def retime_clip_device(self, settings: RetimeSettings, frames_ptr: int, nframes: int, sels, width, height, fmt,
                           out_ptr: int):
        """A clip resident in device memory (raw device pointers, e.g. ``tensor.data_ptr()``)."""
        arr = (_Selection * len(sels))(*[s._c() for s in sels])
        self._check(self._L.tw_retime_clip_device(self._h, ctypes.byref(settings._c()), ctypes.c_void_p(frames_ptr),
                                                  nframes, arr, len(sels), width, height, fmt,
                                                  ctypes.c_void_p(out_ptr)))


def retime_clip(dev: Device, frames, nframes, width, height, fmt, params: TimeParams, nout,
                settings: Optional[RetimeSettings] = None):
    """Renders ``nout`` output frames of the ``retime`` effect over a raw clip (wire frames back to
    back in one array), frame by frame through the library: the host part of the reference's
    ``vfx apply retime`` loop (crates/fx-cli/src/temporal.rs:183-250) around ``tw_retime_frame``."""
    settings = settings or RetimeSettings()
    frame_samples = width * height * 4
    frames = np.ascontiguousarray(frames).reshape(-1)
    out = np.zeros(nout * frame_samples, DTYPES[fmt])
    for n in range(nout):
        sel = select(params, n, width, height)
        sel_flow = FlowSettings(**{**settings.flow.__dict__})
        fa = frames[sel.a * frame_samples:(sel.a + 1) * frame_samples] if 0 <= sel.a < nframes else None
        fb = frames[sel.b * frame_samples:(sel.b + 1) * frame_samples] if 0 <= sel.b < nframes else None
        s = RetimeSettings(sel_flow, settings.compose, settings.motion_rows_reversed)
        dev.retime_frame(s, sel, fa, fb, width, height, fmt, out=out[n * frame_samples:(n + 1) * frame_samples])
    return out
