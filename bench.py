#!/usr/bin/env python3
"""Benchmark of the retime hot path on B200: strict-mode 1080p `retime` output frames per second.

Workload: the `retime` effect at its defaults (Motion Vectors Best, Frame Interp Blend, Sensitivity
70, no Smart Blend) on a synthetic 1920x1080 8 bpc RGBA clip, Speed 40 % (the speed of the
reference's own 1080p timings). A step renders 10 consecutive output frames (two exact source
frames and eight in-between frames, each with a full solve_pair and composition), byte identical to
the reference CPU path.

* ``value``: output frames/s with the source clip resident in HBM (tw_retime_clip_device), timed
  with CUDA events on the library's stream, L2 flushed between steps, max over ranks.
* ``e2e``: the same frames through the C ABI's host-buffer clip call (tw_retime_clip): every
  source frame the step references is uploaded from pinned host memory and every output frame is
  read back into pinned host memory inside the timed region.
* ``roofline``: after the timed region the last step runs once more in the library's serial mode
  (every kernel alone on the stream, CUDA events around each launch): the dominant kernel's
  algorithmic bytes per launch over its average launch time, against the measured HBM bandwidth,
  with the next kernels of that table.
* ``parity``: the last timed step's output frames (device resident, serial and e2e) compared byte
  for byte with the oracle's render of the same frames; any difference fails the run (exit 3).
* ``cpu_baseline``: the time of that oracle render (the reference CPU path restated in C++, OpenMP
  over all host cores): a bounded sample of the same workload.

``--workload create-vectors``, ``--workload fgbg`` and ``--workload vectors-in`` measure the other
single-GPU configurations the same way through their host-buffer C ABI calls (tw_create_vectors_clip
on a 1920x1080 16 bpc clip under random affine motion; tw_retime_layers_clip on a 1920x1080 8 bpc
clip with three FG matte layers at speed 40 %; tw_vectors_in_clip on the retime clip with both
vector layers, holes in them, the effect's defaults), with the oracle beside them on a small sample.

``--impl reference`` times the reference's CPU path the same way (the oracle port: the reference
is Rust and no Rust toolchain exists on these machines). Under torchrun the output frames of ONE
clip are split into contiguous ranges, one per rank (tw_shard), each rank holding only the clip
frames its range reads (tw_source_window): weak scaling, no collective on the data path (NCCL only
for the barrier and the max over ranks of the timings).
"""
import argparse
import hashlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H = 1920, 1080
SPEED = 40.0
FRAMES_PER_STEP = 10
METRIC = "1080p retime output frames/s (strict byte-exact GPU vs CPU)"
METRIC_FAST = "1080p retime output frames/s (fast mode: FMA contraction, approximate division; PSNR vs CPU)"
WORKLOAD = "retime 1920x1080 8bpc RGBA, speed 40%, defaults (vectors Best, Blend, sensitivity 70)"
CLIP_KW = dict(seed=0x74570002, bg_velocity=(6.0, -3.0), square=240, square_start=(600.0, 400.0),
               square_velocity=(9.0, 4.0))


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return int(os.environ.get("RANK", "0")), ws, int(os.environ.get("LOCAL_RANK", "0"))


def emit(obj):
    print(json.dumps(obj), flush=True)


def source_frames_needed(nout):
    return int(math.ceil(SPEED / 100.0 * nout)) + 2


def make_clip(nframes, window=None):
    """The 1080p clip of nframes frames, or only its frames window = (first, last)."""
    from twixtor_b200 import synth
    return synth.moving_clip(W, H, nframes, depth=8, window=window, **CLIP_KW)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_of(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return t.get(kernel)
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx = float(p[2])
                except ValueError:
                    continue
                for n, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference(args):
    """The reference CPU path (restated in C++, all host threads) on the same workload and step as
    the CUDA arm: 10 consecutive output frames of the 1080p clip (2 exact, 8 in-between)."""
    rank, ws, _ = dist_env()
    if rank != 0:
        return 0
    nout = FRAMES_PER_STEP
    total = (args.warmup + args.steps) * nout
    nframes = source_frames_needed(total)
    frames = make_clip(nframes)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    threads = os.cpu_count() or 1
    O.lib().or_set_threads(threads)
    p = O.retime_params(speed=SPEED)

    def step(k):
        for j in range(nout):
            O.retime_one(frames, nframes, W, H, 0, p, k * nout + j)

    for k in range(args.warmup):
        step(k)
    t = time.perf_counter()
    for k in range(args.warmup, args.warmup + args.steps):
        step(k)
    dt = time.perf_counter() - t
    value = args.steps * nout / dt
    emit({"impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": ws,
          "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
          "config": {"workload": WORKLOAD, "output_frames_per_step": nout},
          "cpu_baseline": {"value": value, "unit": "frames/s", "cores": threads, "kind": "port",
                           "sample": f"{args.steps} steps of {nout} output frames (2 exact, 8 in-between) "
                                     f"of the 1080p clip on {threads} OpenMP threads"},
          "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    return 0


def ncu_case(tune_cache=None):
    """One step of the workload (10 output frames of the 1080p clip, 2 exact and 8 in-between), for
    an ncu capture: a few hundred kernel launches, 0.1 GB on the device. The autotuner's table comes
    from `tune_cache` when given (a run without ncu writes it; under ncu it is only read, so the
    launch list holds the step alone)."""
    import twixtor_b200 as tw
    nframes = source_frames_needed(FRAMES_PER_STEP)
    frames_np = make_clip(nframes)
    dev = tw.Device(0)
    dev.autotune(tw.FlowSettings(quality=4), W, H, path=tune_cache)
    tp = tw.TimeParams(speed_percent=SPEED)
    sels = [tw.select(tp, n, W, H) for n in range(FRAMES_PER_STEP)]
    out = np.zeros(FRAMES_PER_STEP * W * H * 4, np.uint8)
    dev.retime_clip(tw.RetimeSettings(), frames_np, nframes, sels, W, H, 0, out=out)
    print(json.dumps({"ncu_case": "ok", "frames": FRAMES_PER_STEP, "launches": dev.stats()["kernel_launches"]}))
    dev.close()
    return 0


def _timed(stream, fn, k, flush):
    import torch
    flush.fill_(k & 0xff)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn(k)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_workload(args):
    """The create-vectors (1080p 16 bpc, frame pairs n -> n - 1), retime-fgbg (1080p 8 bpc, three FG
    layers, speed 40 %) and vectors-in (1080p 8 bpc, both vector layers, speed 40 %) configurations
    through their host-buffer clip calls, one GPU."""
    import torch
    import twixtor_b200 as tw
    from twixtor_b200 import synth
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    dev = tw.Device(0)
    dev.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda:0")
    steps, warmup = args.steps, args.warmup
    if args.workload == "create-vectors":
        per, nsrc, fmt = 8, 24, 1
        frames = synth.affine_clip(W, H, nsrc, depth=16)
        pinned = torch.from_numpy(frames).pin_memory().numpy()
        vs = tw.vectors_settings()
        pairs = [(1 + (n % (nsrc - 1)), n % (nsrc - 1)) for n in range((warmup + steps) * per)]
        out = torch.empty(per * W * H * 4, dtype=torch.int16).pin_memory().numpy().view(np.uint16)

        def step(k):
            dev.create_vectors_clip(vs, pinned, nsrc, pairs[k * per:(k + 1) * per], W, H, fmt, out=out)
        metric = "1080p create-vectors output frames/s (strict byte-exact GPU vs CPU)"
        workload = "create-vectors 1920x1080 16bpc RGBA, pairs n -> n-1 under random affine motion, defaults (half res)"
        h2d = per * 2 * W * H * 8
    elif args.workload == "vectors-in":
        per, fmt, md = 5, 0, 32.0
        nsrc = int(math.ceil(SPEED / 100.0 * (warmup + steps) * per)) + 2
        frames = synth.moving_clip(W, H, nsrc, depth=8, **CLIP_KW)
        vnext = synth.vector_clip(W, H, nsrc, CLIP_KW["bg_velocity"], max_displace=md)
        vprev = synth.vector_clip(W, H, nsrc, CLIP_KW["bg_velocity"], max_displace=md, sign=-1.0, seed=0x74570007)
        fs = W * H * 4
        tp = tw.TimeParams(fps=(30, 1), speed_percent=SPEED)
        settings = tw.vectors_in_settings()  # the effect's defaults: Warping Forward, Blend
        step_args = []
        for k in range(warmup + steps):  # per step the clip frames its output frames read
            sv = [tw.select_vectors_in(tp, n, W, H) for n in range(k * per, (k + 1) * per)]
            lo = min(min(v.a, v.b) for _, v in sv)
            hi = max(max(v.a, v.b) for _, v in sv)
            lo, hi = max(lo, 0), min(hi, nsrc - 1)
            vfs = [tw.VecInFrame(v.a - lo, v.b - lo) for _, v in sv]
            cut = lambda c: torch.from_numpy(np.ascontiguousarray(c[lo * fs:(hi + 1) * fs])).pin_memory().numpy()
            step_args.append(([s for s, _ in sv], vfs, cut(frames), cut(vnext), cut(vprev), hi - lo + 1))
        out = torch.empty(per * W * H * 4, dtype=torch.uint8).pin_memory().numpy()

        def step(k):
            sels, vfs, f, vn, vp, n = step_args[k]
            dev.vectors_in_clip(settings, f, n, vn, n, vp, n, sels, vfs, md, W, H, fmt, out=out)
        metric = "1080p vectors-in output frames/s (strict byte-exact GPU vs CPU)"
        workload = ("vectors-in 1920x1080 8bpc RGBA, speed 40%, both vector layers (12 alpha-0 holes a frame), "
                    "defaults (Warping Forward, Blend)")
        h2d = sum(3 * a[5] * fs for a in step_args[warmup:]) // steps
    else:
        per, fmt, nfg = 5, 0, 3
        nsrc = int(math.ceil(SPEED / 100.0 * (warmup + steps) * per)) + 2
        frames, mattes = synth.layered_clip(W, H, nsrc, nfg=nfg)
        pin = [torch.from_numpy(x).pin_memory().numpy() for x in [frames] + mattes]
        tp = tw.TimeParams(speed_percent=SPEED)
        sels = [tw.select(tp, n, W, H) for n in range((warmup + steps) * per)]
        settings = tw.RetimeSettings(compose=tw.EngineSettings(gouraud=True))
        sens = [tw.percent_param(70.0)] * (nfg + 1)
        out = torch.empty(per * W * H * 4, dtype=torch.uint8).pin_memory().numpy()

        def step(k):
            dev.retime_layers_clip(settings, pin[0], nsrc, pin[1:], [1] * nfg, sens, sels[k * per:(k + 1) * per], W, H,
                                   fmt, out=out)
        metric = "1080p retime-fgbg output frames/s, 3 FG layers (strict byte-exact GPU vs CPU)"
        workload = "retime-fgbg 1920x1080 8bpc RGBA, 3 FG matte layers (binary ellipses, red channel), speed 40%"
        h2d = per * 2 * (nfg + 1) * W * H * 4
    dev.autotune(tw.FlowSettings(quality=4), W, H)
    if args.ncu_case:  # the profiling driver: one step (5 output frames), no timing
        step(0)
        torch.cuda.synchronize()
        print(json.dumps({"ncu_case": "ok", "workload": args.workload, "frames": per,
                          "launches": dev.stats()["kernel_launches"]}))
        dev.close()
        return 0
    for k in range(warmup):
        step(k)
    torch.cuda.synchronize()
    l0 = dev.stats()["kernel_launches"]
    with Clocks(0) as clk:
        times = [_timed(stream, step, k, flush) for k in range(warmup, warmup + steps)]
    launches = dev.stats()["kernel_launches"] - l0
    total_ms = sum(times)
    value = steps * per / (total_ms / 1e3)
    kernels, serial_ms = roofline_pass(dev, stream, flush, lambda: step(warmup + steps - 1))
    peak, which = peaks()
    line = {"metric": metric, "value": value, "unit": "frames/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": total_ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload, "output_frames_per_step": per,
                       "timing": "host buffers through the C ABI clip call (uploads and downloads inside)",
                       "l2": "flushed between steps (256 MiB write)"},
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": per * W * H * 4 * (2 if fmt == 1 else 1)},
            "gpu_launches": launches,
            "roofline": roofline_entry(kernels, serial_ms, launches / steps, total_ms / steps, peak, which),
            "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        import oracle_lib as O
        threads = os.cpu_count() or 1
        O.lib().or_set_threads(threads)
        t = time.perf_counter()
        if args.workload == "create-vectors":
            O.create_vectors_clip(frames, 3, W, H, fmt, 2)
            n = 2
        elif args.workload == "vectors-in":
            O.vectors_in_clip(frames, nsrc, vnext, nsrc, vprev, nsrc, W, H, fmt, O.vecin_params(speed=SPEED, max_displace=md),
                              2)
            n = 2
        else:
            O.retime_fgbg_clip(frames, nsrc, mattes, [1] * nfg, [70.0] * nfg, W, H, fmt, O.retime_params(speed=SPEED), 2)
            n = 2
        dt = time.perf_counter() - t
        line["cpu_baseline"] = {"value": n / dt, "unit": "frames/s", "cores": threads, "kind": "port",
                                "sample": f"{n} output frame(s) of the same clip, {dt:.2f} s on {threads} OpenMP threads"}
    emit(line)
    dev.close()
    return 0


def run_adjoint(args):
    """The adjoint of warp + blend: per step the L1 loss against the middle frame and its gradients
    w.r.t. both frames and both flows for a batch of 64 triples of 1280x720 float RGBA (flows at
    640x360), the gradient buffers zeroed first; triples/s with everything resident in HBM."""
    import torch
    import twixtor_b200 as tw
    from twixtor_b200 import adjoint, synth
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    dev = tw.Device(0)
    dev.set_stream(stream.cuda_stream)
    w, h, fw, fh, batch, base = 1280, 720, 640, 360, 64, 8
    if args.ncu_case:  # the profiling driver: one launch on 8 triples (0.7 GB on the device)
        batch = 8
    A_, B_, M_, D_ = synth.adjoint_triples(w, h, base)
    d_half = np.ascontiguousarray(D_[:, ::2, ::2, :] * np.float32(0.5))  # flow grid units (r ~ 0.5)
    # 64 distinct triples: each generated triple (texture, displacement) and 7 copies rolled by an
    # even pixel offset (the flows by half of it), the same shift for the three frames and the flows
    shifts = [(0, 0)] + [(2 * ((97 * k) % (h // 2)), 2 * ((211 * k) % (w // 2))) for k in range(1, batch // base)]
    def spread(x, flow):  # noqa: E306
        t = torch.from_numpy(x).cuda()
        out = [torch.roll(t, (dy // 2, dx // 2) if flow else (dy, dx), dims=(1, 2)) for dy, dx in shifts]
        return torch.cat(out, 0).contiguous()
    a, b, m = spread(A_, False), spread(B_, False), spread(M_, False)
    fab, fba = spread(d_half, True), spread(-d_half, True)
    wts = (torch.arange(a[0].numel(), device=a.device, dtype=torch.float64) % 1013) + 1.0
    distinct = len({float((a[i].reshape(-1).double() * wts).sum()) for i in range(batch)})  # position weighted sums
    loss = torch.zeros(batch, device="cuda:0")
    da, db = torch.zeros_like(a), torch.zeros_like(b)
    dfab, dfba = torch.zeros_like(fab), torch.zeros_like(fba)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda:0")

    def step(k):
        for t in (loss, da, db, dfab, dfba):
            t.zero_()
        dev.warp_blend_adjoint(a.data_ptr(), b.data_ptr(), fab.data_ptr(), fba.data_ptr(), w, h, fw, fh, batch, 0.5,
                               target=m.data_ptr(), loss=loss.data_ptr(), da=da.data_ptr(), db=db.data_ptr(),
                               df_ab=dfab.data_ptr(), df_ba=dfba.data_ptr())

    if args.ncu_case:
        step(0)
        torch.cuda.synchronize()
        print(json.dumps({"ncu_case": "ok", "workload": "adjoint", "batch": batch}))
        dev.close()
        return 0
    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    dev.profile_begin("k_warp_blend_adjoint")
    with Clocks(0) as clk:
        times = [_timed(stream, step, k, flush) for k in range(args.warmup, args.warmup + args.steps)]
    kms, klaunch, kbytes = dev.profile_end()
    total_ms = sum(times)
    value = args.steps * batch / (total_ms / 1e3)
    # the torch harness (l1_loss_and_grads allocates its zeroed gradients per call)
    for k in range(args.warmup):
        adjoint.l1_loss_and_grads(dev, a, b, fab, fba, m, 0.5)
    torch.cuda.synchronize()
    etimes = [_timed(stream, lambda k: adjoint.l1_loss_and_grads(dev, a, b, fab, fba, m, 0.5), k, flush)
              for k in range(args.steps)]
    peak, which = peaks()
    achieved = (kbytes / (kms / 1e3)) / 1e9 if kms > 0 else None
    tr = traffic_of("k_warp_blend_adjoint")
    if isinstance(tr, dict):
        tr = tr["dram_bytes"] / tr["algorithmic_bytes"] * (kbytes / max(klaunch, 1))
    emit({"metric": "adjoint of warp + blend, triples/s (L1 loss, gradients for both frames and both flows)",
          "value": value, "unit": "triples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
          "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
          "dtype": "f32", "data": "synthetic",
          "config": {"workload": "64 triples of 1280x720 float RGBA, flows 640x360, wa 0.5, L1 against the middle frame",
                     "batch": batch, "distinct_triples": distinct,
                     "l2": "flushed between steps (256 MiB write); inputs 2.8 GB > L2"},
          "e2e": {"value": args.steps * batch / (sum(etimes) / 1e3), "unit": "triples/s", "h2d_bytes_per_step": 0,
                  "d2h_bytes_per_step": 0, "note": "through the torch harness (device tensors)"},
          "gpu_launches": dev.stats()["kernel_launches"],
          "roofline": {"bound": "hbm", "kernel": "k_warp_blend_adjoint", "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": (achieved / peak) if achieved else None, "traffic": tr, "peak_source": which,
                       "algorithmic_bytes_per_launch": kbytes / max(klaunch, 1),
                       "avg_launch_us": 1e3 * kms / max(klaunch, 1)},
          "clocks": clk.summary()})
    dev.close()
    return 0


BATCH_SIZES = [(1280, 720), (1440, 1080), (1920, 1080), (3840, 2160)]
BATCH_KEYS = [(0.0, 100.0, True), (48.0, 25.0, True), (96.0, 100.0, True)]


def run_batch(args):
    """Four clips of uneven size (1280x720, 1440x1080, 1920x1080, 3840x2160; float RGBA), the keyed
    speed ramp 100@0e;25@48e;100@96e, in one batched call per step (tw_retime_batch_device): every
    step renders the next 8 output frames of every clip, frames of different clips in flight
    together. Clips generated and resident on the device."""
    import torch
    import twixtor_b200 as tw
    from twixtor_b200 import synth
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    dev = tw.Device(0)
    dev.set_stream(stream.cuda_stream)
    per = 8
    total = (args.warmup + args.steps) * per
    tp = tw.TimeParams(keys=BATCH_KEYS)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda:0")
    jobs, keep = [], []
    for i, (w, h) in enumerate(BATCH_SIZES):
        sels = [tw.select(tp, n, w, h) for n in range(total)]
        nsrc = max(max(s.a, s.b) for s in sels) + 1
        frames = synth.batch_clip_gpu(w, h, nsrc, seed=0x74570030 + i)
        out = torch.empty(per * w * h * 4, dtype=torch.float32, device="cuda:0")
        keep += [frames, out]
        jobs.append(dict(settings=tw.RetimeSettings(), frames=frames.data_ptr(), nframes=nsrc, sels=sels, width=w,
                         height=h, fmt=2, out=out.data_ptr()))

    for w, h in BATCH_SIZES:
        dev.autotune(tw.FlowSettings(quality=4), w, h)

    def step(k):
        dev.retime_batch_device([dict(j, sels=j["sels"][k * per:(k + 1) * per]) for j in jobs])

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    l0 = dev.stats()["kernel_launches"]
    with Clocks(0) as clk:
        times = [_timed(stream, step, k, flush) for k in range(args.warmup, args.warmup + args.steps)]
    launches = dev.stats()["kernel_launches"] - l0
    total_ms = sum(times)
    nframes = args.steps * per * len(jobs)
    kernels, serial_ms = roofline_pass(dev, stream, flush, lambda: step(args.warmup + args.steps - 1))
    peak, which = peaks()
    mpx = args.steps * per * sum(w * h for w, h in BATCH_SIZES) / 1e6
    line = {"metric": "batched retime output frames/s, 4 clips of uneven size (strict byte-exact GPU vs CPU)",
            "value": nframes / (total_ms / 1e3), "unit": "frames/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "retime of 1280x720, 1440x1080, 1920x1080 and 3840x2160 float RGBA clips, keyed speed "
                                   "100@0e;25@48e;100@96e, 8 output frames of each clip per step in one batched call",
                       "megapixels_per_s": mpx / (total_ms / 1e3), "output_frames_per_step": per * len(jobs),
                       "l2": "flushed between steps (256 MiB write); clips resident in HBM"},
            "gpu_launches": launches,
            "roofline": roofline_entry(kernels, serial_ms, launches / args.steps, total_ms / args.steps, peak, which),
            "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib as O
        threads = os.cpu_count() or 1
        O.lib().or_set_threads(threads)
        p = O.retime_params(keys=BATCH_KEYS)
        t = time.perf_counter()
        px = 0
        for (w, h), j, fr in zip(BATCH_SIZES, jobs, keep[0::2]):
            k = next(n for n, s in enumerate(j["sels"]) if not s.exact)
            need = j["sels"][k].a + 2  # only the frames up to the pair go to the host
            O.retime_one(fr[:need * w * h * 4].cpu().numpy(), need, w, h, 2, p, k)
            px += w * h
        dt = time.perf_counter() - t
        line["cpu_baseline"] = {"value": 4 / dt, "unit": "frames/s", "cores": threads, "kind": "port",
                                "sample": f"one in-between frame of each clip ({px / 1e6:.1f} Mpx), {dt:.2f} s on "
                                          f"{threads} OpenMP threads", "megapixels_per_s": px / 1e6 / dt}
    emit(line)
    dev.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ncu-case", action="store_true",
                    help="profiling driver, no timing: renders the first 10 output frames of the 1080p workload once "
                         "(device resident clip) and exits; the command the committed ncu summaries name")
    ap.add_argument("--fast", action="store_true",
                    help="retime: the fast mode (tw_flow_settings.fast_mode); parity becomes PSNR against the strict render")
    ap.add_argument("--tune-cache", default=None,
                    help="--ncu-case: the autotuner's JSON table, read when present, written otherwise")
    ap.add_argument("--workload", default="retime", choices=["retime", "create-vectors", "fgbg", "vectors-in", "adjoint",
                                                           "batch"],
                    help="retime (the headline, default), create-vectors (1080p 16 bpc), fgbg (1080p, 3 FG layers) or "
                         "adjoint (warp + blend gradients, 64 triples of 1280x720) or batch (4 clips of uneven size)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload != "retime":
        return run_workload(args)
    if args.ncu_case and args.workload == "retime":
        return ncu_case(args.tune_cache)

    import torch
    import twixtor_b200 as tw

    rank, ws, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    # One clip; under torchrun its output frames are split into contiguous ranges, one per rank
    # (tw_shard), and each rank holds only the clip frames its range reads (tw_source_window).
    per_rank = (args.warmup + args.steps) * FRAMES_PER_STEP
    total_out = ws * per_rank
    nclip = source_frames_needed(total_out)
    tp = tw.TimeParams(speed_percent=SPEED)
    all_sels = [tw.select(tp, n, W, H) for n in range(total_out)]
    lo, hi = tw.shard(total_out, ws, rank)
    first, last = tw.source_window(all_sels[lo:hi], nclip)
    nframes = last - first + 1
    frames_np = make_clip(nclip, window=(first, last))
    sels = tw.rebase(all_sels[lo:hi], first, nclip)  # frame indices into this rank's window
    fs = W * H * 4
    stream = torch.cuda.current_stream()
    dev = tw.Device(local)
    dev.set_stream(stream.cuda_stream)
    settings = tw.RetimeSettings(flow=tw.FlowSettings(fast_mode=args.fast))

    # the autotuner's launch shapes for every level of the 1080p solve (measured once, before the
    # warm-up; the table only changes the time, never the bytes)
    tuned = dev.autotune(tw.FlowSettings(quality=sels[0].vectors_quality or 4), W, H)
    clip = torch.from_numpy(frames_np).to(f"cuda:{local}")
    out = torch.empty(FRAMES_PER_STEP * fs, dtype=torch.uint8, device=f"cuda:{local}")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")

    def step_device(k):
        s = sels[k * FRAMES_PER_STEP:(k + 1) * FRAMES_PER_STEP]
        dev.retime_clip_device(settings, clip.data_ptr(), nframes, s, W, H, 0, out.data_ptr())

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # ---- value: device resident -------------------------------------------------------------
    for k in range(args.warmup):
        step_device(k)
    barrier()
    l0 = dev.stats()["kernel_launches"]
    times = []
    with Clocks(local) as clk:
        for k in range(args.warmup, args.warmup + args.steps):
            flush.fill_(k & 0xff)  # L2 flush between steps, outside the timed events
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step_device(k)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    launches = dev.stats()["kernel_launches"] - l0
    last_k = args.warmup + args.steps - 1
    dev_out = out.cpu().numpy()  # the last timed step's output frames
    barrier()
    total_ms = max_over_ranks(sum(times))
    clocks = clk.summary()
    value = ws * args.steps * FRAMES_PER_STEP / (total_ms / 1e3)

    # ---- roofline: the same step once more in serial mode (every kernel alone on the stream) -------
    kernels, serial_ms = roofline_pass(dev, stream, flush, lambda: step_device(last_k))
    serial_out = out.cpu().numpy()

    # ---- e2e: host buffers through the C ABI ------------------------------------------------
    pinned = torch.from_numpy(frames_np).pin_memory()
    pin_np = pinned.numpy()
    out_host = torch.empty(FRAMES_PER_STEP * fs, dtype=torch.uint8).pin_memory().numpy()

    def step_host(k):
        # the step's source frames (the ones its selections reference) are uploaded from pinned host
        # memory inside the call, and every output frame is copied back into pinned host memory
        s = sels[k * FRAMES_PER_STEP:(k + 1) * FRAMES_PER_STEP]
        dev.retime_clip(settings, pin_np, nframes, s, W, H, 0, out=out_host)

    for k in range(args.warmup):
        step_host(k)
    barrier()
    etimes = []
    for k in range(args.warmup, args.warmup + args.steps):
        flush.fill_(k & 0xff)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step_host(k)
        e1.record(stream)
        e1.synchronize()
        etimes.append(e0.elapsed_time(e1))
    barrier()
    e2e_ms = max_over_ranks(sum(etimes))
    e2e_value = ws * args.steps * FRAMES_PER_STEP / (e2e_ms / 1e3)
    step_sels = sels[:FRAMES_PER_STEP]
    h2d = fs * len({f for s in step_sels for f in (s.a, s.b) if 0 <= f < nframes})
    d2h = FRAMES_PER_STEP * fs

    # ---- parity: the last timed step, device resident, serial and e2e, against the oracle --------
    threads = max(1, (os.cpu_count() or 1) // ws)
    glob = [lo + last_k * FRAMES_PER_STEP + j for j in range(FRAMES_PER_STEP)]
    want, cpu_dt = oracle_frames(frames_np, first, nframes, nclip, glob, threads)
    if not args.fast:
        equal = {"device": dev_out.tobytes() == want.tobytes(), "serial": serial_out.tobytes() == want.tobytes(),
                 "e2e": out_host.tobytes() == want.tobytes()}
    else:  # the fast mode is not byte identical: its PSNR against the strict render, at least 45 dB
        equal = {k: psnr(v, want) for k, v in (("device", dev_out), ("serial", serial_out), ("e2e", out_host))}
    ok = all(equal.values()) if not args.fast else min(equal.values()) > 45.0
    if ws > 1:
        t = torch.tensor([0 if ok else 1], dtype=torch.int32, device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ok_all = int(t.item()) == 0
    else:
        ok_all = ok
    parity = {"frames": FRAMES_PER_STEP * ws, "equal": ok_all, "paths": equal,
              "sha256_rank0": hashlib.sha256(dev_out.tobytes()).hexdigest(),
              "checked": "the last timed step's output frames of every rank, byte for byte against the oracle"
                         if not args.fast else
                         "fast mode: PSNR (dB) of the last timed step's output frames against the oracle's strict "
                         "render, every path above 45 dB"}

    if rank == 0:
        peak, which = peaks()
        line = {
            "metric": METRIC if not args.fast else METRIC_FAST, "value": value, "unit": "frames/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD + (", fast mode" if args.fast else ""),
                       "output_frames_per_step": FRAMES_PER_STEP * ws,
                       "in_between_frames_per_step": sum(1 for s in step_sels if not s.exact),
                       "source_frames_resident": nframes, "frame_bytes": fs,
                       "l2": "flushed between steps (256 MiB write), inputs resident 0.5 GB > L2",
                       "parallelism": (f"one clip of {total_out} output frames split into {ws} contiguous ranges "
                                       f"of {per_rank} (one per GPU, each holding only its source window); "
                                       "no collective on the data path") if ws > 1 else "1 GPU",
                       "autotuned_levels": tuned, "tuning": json.loads(dev.tuning_table())["levels"]},
            "e2e": {"value": e2e_value, "unit": "frames/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roofline_entry(kernels, serial_ms, launches / args.steps, total_ms / args.steps, peak,
                                       which),
            "parity": parity,
            "clocks": clocks,
        }
        if not args.no_cpu_baseline and ws == 1:
            line["cpu_baseline"] = {"value": FRAMES_PER_STEP / cpu_dt, "unit": "frames/s", "cores": threads,
                                    "kind": "port",
                                    "sample": f"the parity render: the {FRAMES_PER_STEP} output frames of the last timed "
                                              f"step ({sum(1 for s in step_sels if not s.exact)} in-between) of the "
                                              f"same 1080p clip, {cpu_dt:.2f} s on {threads} OpenMP threads"}
        emit(line)
    if ws > 1:
        torch.distributed.destroy_process_group()
    dev.close()
    return 0 if ok_all else 3


def psnr(a, b):
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = float(np.mean(d * d))
    return 1e9 if mse == 0 else round(10.0 * math.log10(255.0 ** 2 / mse), 2)


def oracle_frames(window, first, count, nclip, outputs, threads):
    """The oracle's render of the given output frames from the clip window a rank holds (test
    infrastructure, after the timed regions): the parity reference and the CPU baseline's sample."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    O.lib().or_set_threads(threads)
    p = O.retime_params(speed=SPEED)
    t = time.perf_counter()
    res = [O.retime_window(window, first, count, nclip, W, H, 0, p, n) for n in outputs]
    return np.concatenate(res), time.perf_counter() - t


def roofline_pass(dev, stream, flush, run):
    """One more step in the library's serial mode (tw_set_lanes(0): every kernel in issue order on the
    stream, nothing overlapping), with every launch bracketed by CUDA events on that stream: per
    kernel its launches, device time and algorithmic bytes. Outside the timed region."""
    import torch
    dev.set_lanes(0)
    flush.fill_(7)
    torch.cuda.synchronize()
    dev.profile_begin("*")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run()
    e1.record(stream)
    e1.synchronize()
    table = dev.profile_report()
    dev.profile_end()
    dev.set_lanes(4)
    kernels = []
    for row in table.splitlines()[1:]:
        p = row.split()
        if len(p) >= 6:
            kernels.append({"kernel": p[0], "launches": int(p[1]), "ms": float(p[2]), "us_per_launch": float(p[3]),
                            "share": float(p[4].rstrip("%")) / 100.0, "alg_gbs": float(p[5])})
    # the tile shapes of one kernel (k_level_iter_32x32, _64x32, ...) count as that kernel
    fam = {}
    for k in kernels:
        name = k["kernel"].rsplit("_", 1)[0] if k["kernel"].startswith("k_level_iter_") else k["kernel"]
        f = fam.setdefault(name, {"kernel": name, "launches": 0, "ms": 0.0, "bytes": 0.0, "share": 0.0,
                                  "shapes": []})
        f["launches"] += k["launches"]
        f["ms"] += k["ms"]
        f["bytes"] += k["alg_gbs"] * 1e9 * k["ms"] * 1e-3
        f["share"] += k["share"]
        if name != k["kernel"]:
            f["shapes"].append({x: k[x] for x in ("kernel", "launches", "us_per_launch", "alg_gbs")})
    kernels = []
    for f in sorted(fam.values(), key=lambda f: -f["ms"]):
        row = {"kernel": f["kernel"], "launches": f["launches"], "ms": f["ms"],
               "us_per_launch": 1e3 * f["ms"] / max(f["launches"], 1), "share": f["share"],
               "alg_gbs": f["bytes"] / (f["ms"] * 1e-3) / 1e9 if f["ms"] > 0 else 0.0}
        if f["shapes"]:
            row["shapes"] = f["shapes"]
        kernels.append(row)
    return kernels, e0.elapsed_time(e1)


def roofline_entry(kernels, serial_ms, launches_per_step, ms_per_step, peak, which):
    """The dominant kernel by serial device time: its algorithmic bytes per launch over its average
    launch duration (measured alone), as a fraction of the measured HBM copy bandwidth; with the
    next kernels of the table beside it."""
    top = kernels[0]
    achieved = top["alg_gbs"]
    bytes_per_launch = achieved * 1e9 * top["us_per_launch"] * 1e-6
    tr = traffic_of(top["kernel"])
    if isinstance(tr, dict):
        # DRAM bytes of the captured launch scaled to the average launch by the algorithmic bytes
        # each moves (traffic grows in proportion to the units processed)
        tr = tr["dram_bytes"] / tr["algorithmic_bytes"] * bytes_per_launch
    return {"bound": "hbm", "kernel": top["kernel"], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if peak else None, "traffic": tr, "peak_source": which,
            "launches_per_step": top["launches"], "avg_launch_us": top["us_per_launch"],
            "algorithmic_bytes_per_launch": bytes_per_launch,
            "timing": "one step in serial mode (each kernel alone on the stream, CUDA events per launch), "
                      "after the timed region",
            "serial_step_ms": serial_ms, "kernel_ms_per_step": top["ms"],
            "kernel_ms_fits_step": top["ms"] <= serial_ms,
            "timed_ms_per_step": ms_per_step, "timed_launches_per_step": launches_per_step,
            "kernels": [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()} |
                        {"frac": round(r["alg_gbs"] / peak, 4) if peak else None} for r in kernels[:8]]}


if __name__ == "__main__":
    sys.exit(main())
