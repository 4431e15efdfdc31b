"""The C-ABI library: it builds, loads, and exports every function include/twixtor_b200.h declares
(no device call: these run without a GPU). The host-side time model is checked against the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle_lib as O
import twixtor_b200 as tw

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "twixtor_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tw_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_seam():
    names = declared()
    for must in ("tw_open", "tw_close", "tw_solve", "tw_solve_pair", "tw_compose_vectors", "tw_retime_frame",
                 "tw_select", "tw_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    tw.build()
    lib = ctypes.CDLL(tw.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_built_for_sm_100a_in_tree():
    assert os.path.dirname(tw.LIB_PATH) == os.path.join(ROOT, "twixtor_b200")
    from twixtor_b200 import buildlib as b
    assert "arch=compute_100a,code=sm_100a" in " ".join(b.FLAGS)
    assert "-fmad=false" in b.FLAGS


@pytest.mark.parametrize("speed,fps,keys,n", [
    (50.0, (24, 1), None, 7), (33.3333, (30000, 1001), None, 5), (62.5, (24, 1), None, 11), (-50.0, (24, 1), None, 6),
    (0.0, (24, 1), None, 3), (150.0, (60, 1), None, 9), (0.0, (24, 1), [(0, 100, 0), (5, 40, 0)], 8),
    (0.0, (24, 1), [(0, 60, 1), (5, 30, 1)], 8), (40.0, (24, 1), None, 95)])
def test_time_model_matches_the_oracle(speed, fps, keys, n):
    p = O.retime_params(fps=fps, speed=speed, keys=keys)
    tp = tw.TimeParams(fps=fps, speed_percent=speed, keys=keys)
    for k in range(n):
        o = O.select(p, k, 64, 48)
        s = tw.select(tp, k, 64, 48)
        assert np.float32(o["s0"]).tobytes() == np.float32(s.s0).tobytes()
        assert np.float32(o["s1"]).tobytes() == np.float32(s.s1).tobytes()
        assert np.float32(o["wa"]).tobytes() == np.float32(s.wa).tobytes()
        assert (o["a"], o["exact"], o["vq"], o["interp"]) == (s.a, s.exact, s.vectors_quality, s.interp)


def test_flow_geometry_matches_the_oracle():
    for q in (1, 2, 3, 4, 5):
        for hiq in (True, False):
            for (w, h) in ((1920, 1080), (160, 96), (2, 2), (7, 9), (3840, 2160)):
                red, sizes = O.geometry(q, hiq, w, h)
                fw, fh, s2 = tw.flow_geometry(tw.FlowSettings(quality=q, hiq=hiq), w, h)
                assert sizes == s2 and (fw, fh) == sizes[0]
