#!/usr/bin/env python3
"""1080p turbo encode benchmark of the B200 encode backend.

Workload (the reference's 1080p turbo configuration): a seeded synthetic
1920x1080 8-bit 4:2:0 clip of 120 frames (pan (+2.5, +1.0) px/frame, 12
moving rectangles of 64-256 px, noise sigma 2), coded with --turbo -q 125
--keyint 60 --tiles 2 (deblocking and CDEF on, loop restoration off). One
step = the whole clip in coding order (2 key frames, 58 hidden ALTREF frames,
58 leaf frames, 2 regular frames).

value: frames/s with the source frames resident in HBM (CUDA events on the
       session stream, max over ranks): every device stage of the backend.
e2e:   the encoder's public API end to end: libmav1.so (the reference's
       src/mav1.h) fed the clip's frames from host memory, producing the IVF
       temporal units. Per step the clip's two closed GOPs go to two live
       encoders, each driven by its own host thread (mav1_send_frame /
       mav1_receive_packet / mav1_get_recon, as tools/mav1enc.c does), until
       every temporal unit of the clip has come back. Inside the timed region:
       the copy of every source into page-locked memory and to the device,
       every device stage, the export of the writer inputs and
       reconstructions to the host, entropy coding and OBU assembly on the
       host thread pool, and the reconstruction copies of mav1_get_recon.
       Wall clock (the host is part of the path), max over ranks. The first
       timed step's temporal units are hashed and checked against the
       oracle's hashes of the same clip (tests/golden/oracle_hashes.json).
--impl reference: the reference encoder's own CPU path (oracle/_ref, built
       from the reference sources: its scalar backend with OpenMP-parallel
       stages, its entropy coder and OBU writer) on the host cores, all
       threads, through the same mav1.h calls; each step codes a bounded
       sample of the clip (its first frames) and is timed by wall clock.

Multi-GPU: the path does not shard (one stream is a serial reference
chain); --gpus N runs N independent replicas, one per GPU.
"""
import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mav1-encoder_b200"))
# Every encoder runs several CUDA streams (two frame engines, their transfer,
# upload and status streams); with the default 8 hardware work queues they
# alias and serialise. Read when the CUDA context is created, so set here,
# before anything touches the device (measured: the 16-stream batch 766 ->
# 786 fps, the clip through the API 970 -> 980 fps).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import synthetic  # noqa: E402

METRIC = "1080p turbo encode fps on 1 B200 (bit-exact to --cpu)"
GOLDEN = os.path.join(ROOT, "tests", "golden", "oracle_hashes.json")
GOLDEN_CASE = "c1_1080p_turbo_120"
REF_SAMPLE = 30  # frames of the clip per reference-arm step
FLAGS = dict(q=125, turbo=1, keyint=60, tiles=2)
SPEC = synthetic.CONFIGS["c1_1080p"]
CONFIG = {"workload": "1920x1080 synthetic 120-frame clip, --turbo -q 125 --keyint 60 --tiles 2 (LF+CDEF on, LR off)",
          "frames_per_step": SPEC.frames, "width": SPEC.width, "height": SPEC.height,
          "l2": "inputs larger than L2 (373 MB of source frames per step) and a 256 MiB L2 flush between steps"}


def load_clip(spec):
    cache = f"/tmp/mav1cu_clip_{spec.name}_{spec.seed}_{spec.frames}.npy"
    if os.path.exists(cache):
        return np.load(cache)
    frames = np.stack([np.frombuffer(synthetic.packed(f), np.uint8) for f in synthetic.generate(spec)])
    np.save(cache, frames)
    return frames


class Clocks:
    """nvidia-smi samples of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index, self.samples, self.proc = index, [], None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        sm, mx, reasons = [], 0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[0]))
                mx = max(mx, float(s[1]))
                for n, v in zip(names, s[3:7]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def split_gops(jobs):
    """Coding-order jobs grouped by key frame: each group is independent of
    the others (a key frame refreshes every reference slot)."""
    gops = []
    for j in jobs:
        if j["is_key"] or not gops:
            gops.append([])
        gops[-1].append(j)
    return gops


def batch_bench(args):
    """The batching workload (16 streams: 4 each of 640x360, 1280x720,
    1920x1080, 2560x1440; 60 frames each, --turbo, q from {80, 125, 170}):
    every stream through its own live encoder, all at once, against the same
    streams coded one after another. Each stream's IVF is checked against the
    oracle's hashes (tests/golden/batch_hashes.json). Wall clock, sources from
    host memory, entropy coding included."""
    import batch
    import mav1cu

    specs = synthetic.batch_streams()
    frames = batch.load_streams([s for s, _ in specs])
    # keyint = clip length: the clip codes as with keyint 0 (one key frame),
    # and a live encoder codes it again as a new closed GOP at every pass
    cfgs = [mav1cu.cli_config(s.width, s.height, q=q, turbo=1, keyint=s.frames) for s, q in specs]
    B = batch.Batch(list(zip(cfgs, frames)))
    try:
        want = {}
        path = os.path.join(ROOT, "tests", "golden", "batch_hashes.json")
        if os.path.exists(path):
            want = json.load(open(path))
        _, out = B.code(concurrent=True)
        bitexact = None
        if want:
            bitexact = all(batch.stream_hashes(o, s.width, s.height) == want[s.name]["ivf"]
                           for (s, _), o in zip(specs, out))
        n = max(1, args.batch_passes)
        seq = [B.code(concurrent=False)[0] for _ in range(n)]
        conc = [B.code(concurrent=True)[0] for _ in range(n)]
    finally:
        B.close()
    nframes = sum(s.frames for s, _ in specs)
    npx = sum(s.frames * s.width * s.height for s, _ in specs)
    fps_seq, fps_conc = nframes / (sum(seq) / n), nframes / (sum(conc) / n)
    return {"workload": "16 streams (4 x 640x360, 4 x 1280x720, 4 x 1920x1080, 4 x 2560x1440), 60 frames each, "
                        "--turbo, q in {80, 125, 170}; host frames in, IVF out",
            "frames": nframes, "fps_concurrent": round(fps_conc, 1), "fps_sequential": round(fps_seq, 1),
            "speedup": round(fps_conc / fps_seq, 3), "passes": n,
            "mpx_per_s_concurrent": round(npx / (sum(conc) / n) / 1e6, 1),
            "bitexact_to_oracle": bitexact}


def serving_bench(args, capacity_pxs):
    """The serving workload: an open-loop Poisson arrival of sessions
    (resolution mix 640x360 0.3, 1280x720 0.4, 1920x1080 0.25, 3840x2160
    0.05; 30-300 frames; q 60-200; --turbo), frames arriving in real time at
    30 per second, admitted against a 150 GB device-memory budget. The arrival
    rate offers 80% of the batched capacity (capacity_pxs: pixels per second
    of the batching workload, all streams at once). Reports per-frame latency
    percentiles and the aggregate rate; a sample of the sessions is coded
    again alone and must give the same bitstream as in the mix."""
    import batch
    import mav1api
    import serve

    specs = serve.content_specs()
    flat = [c for v in specs.values() for c in v]
    clips = dict(zip([c.name for c in flat], batch.load_streams(flat)))
    mean_len = 165.0
    px_per_frame = serve.mean_pixels_per_second() / serve.FPS
    rate = 0.8 * capacity_pxs / (px_per_frame * mean_len)
    sessions = serve.poisson_sessions(args.serving_sessions, rate, seed=11)
    for s in sessions:
        cands = specs[(s.width, s.height)]
        s.clip = clips[cands[s.sid % len(cands)].name]
    os.environ.setdefault("MAV1_CUDA_IMAGES", "2")
    srv = serve.Server(budget_bytes=150e9)
    try:
        wall = srv.run(sessions)
    finally:
        srv.close()
    res = serve.summary(sessions, wall)
    # alone == in the mix: re-code a sample of the sessions, each alone
    sample = [s for s in sessions if s.latencies][:: max(1, len(sessions) // 8)][:8]
    same = []
    for s in sample:
        pk, _ = mav1api.encode([s.frame(i) for i in range(s.frames)], s.config(), recon=False)
        same.append(hashlib.sha256(mav1api.ivf_bytes(pk, s.width, s.height)).hexdigest() == s.ivf_sha256)
    res.update({"arrival_rate_per_s": round(rate, 3), "offered_load": 0.8, "capacity_mpx_s": round(capacity_pxs / 1e6, 1),
                "hbm_budget_gb": 150, "peak_active_sessions": srv.peak_active,
                "peak_device_gb": round(srv.peak_bytes / 1e9, 2), "encoders_created": srv.encoders_created,
                "alone_equals_mix": f"{sum(same)}/{len(same)}"})
    return res


def full4k_bench(args):
    """The full filter and search chain (3840x2160, 32 frames with a scene cut
    at frame 16, -q 90, tx search, tx depth, switchable / dual filter, CDEF,
    loop restoration searched on the device, --altref 16 --golden --tiles 3,
    ME range 64) through the encoder API from host frames, wall clock per
    pass; the bitstream is checked against the oracle's hashes
    (tests/golden/dropin_hashes.json) when they are present."""
    import batch
    import mav1api
    import mav1cu

    spec = synthetic.CONFIGS["c2_2160p"]
    frames = batch.load_streams([spec])[0]
    cfg = mav1cu.cli_config(spec.width, spec.height, q=90, altref=16, golden=1, tiles=3, me_range=64)
    want = json.load(open(os.path.join(ROOT, "tests", "golden", "dropin_hashes.json"))).get("c2_2160p_full_32f")
    walls, bitexact = [], None
    for i in range(1 + max(1, args.full4k_passes)):
        t0 = time.perf_counter()
        packets, _ = mav1api.encode(list(frames), cfg, recon=False)
        dt = time.perf_counter() - t0
        if i == 0:
            if want:
                bitexact = hashlib.sha256(mav1api.ivf_bytes(packets, spec.width, spec.height)).hexdigest() == want["ivf"]
            continue
        walls.append(dt)
    return {"workload": "3840x2160 synthetic clip, 32 frames (scene cut at 16), -q 90 --altref 16 --golden --tiles 3 "
                        "--me-range 64, every tool on (tx search, tx depth, dual filter, CDEF, loop restoration)",
            "fps": round(spec.frames * len(walls) / sum(walls), 3), "passes": len(walls),
            "s_per_pass": round(sum(walls) / len(walls), 2), "bitexact_to_oracle": bitexact}


def max_over_ranks(values, device):
    """Element-wise maximum of this rank's timings over the process group:
    each replica times its own GPU, and the slowest one defines the step. The
    only collectives of a multi-GPU run are this and the barriers around the
    timed region (the replicas share no data)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def run_ours(args, rank, world):
    import torch
    import mav1cu

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    frames_host = load_clip(SPEC)
    cfg = mav1cu.cli_config(SPEC.width, SPEC.height, **FLAGS)
    jobs = mav1cu.plan(cfg, SPEC.frames)
    gops = split_gops(jobs)
    streams = [mav1cu.Stream(cfg) for _ in gops]
    # round-robin over the GOPs, so every stream always has work queued
    order = [(g, gop[i]) for i in range(max(len(x) for x in gops)) for g, gop in enumerate(gops) if i < len(gop)]
    seq_order = [(0, j) for j in jobs]
    S = torch.cuda.Stream()
    frames_dev = torch.from_numpy(frames_host).to(f"cuda:{dev}")
    fbytes = frames_host.shape[1]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    def step_device(order=order):
        for g, j in order:
            streams[g].encode(j, frames_dev[j["disp"]].data_ptr(), True)

    def step_sequential():
        step_device(seq_order)

    def launches():
        return sum(st.launches() for st in streams)

    def timed(fn, k, w):
        for _ in range(w):
            with torch.cuda.stream(S):
                for st in streams:
                    st.wait(S.cuda_stream)
                fn()
                for st in streams:
                    st.join(S.cuda_stream)
        S.synchronize()
        l0 = launches()
        ms = []
        for _ in range(k):
            with torch.cuda.stream(S):
                flush.fill_(1)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(S)
                for st in streams:
                    st.wait(S.cuda_stream)
                fn()
                for st in streams:
                    st.join(S.cuda_stream)
                b.record(S)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        for st in streams:
            st.synchronize()
        return ms, (launches() - l0) // k

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(dev) as clk:
        ms, nlaunch = timed(step_device, args.steps, args.warmup)
    ms_seq, _ = timed(step_sequential, max(1, args.steps // 2), 1)
    per_step = sum(ms) / len(ms)
    per_seq = sum(ms_seq) / len(ms_seq)
    kern = kernel_times(frames_dev) if (rank == 0 and not args.no_roofline) else None
    for st in streams:
        st.close()
    del frames_dev, flush
    torch.cuda.synchronize()
    e2e = e2e_api(args, frames_host, world)
    if world > 1:
        per_step, per_seq, e2e["ms"], e2e["ms_one"] = max_over_ranks(
            [per_step, per_seq, e2e["ms"], e2e["ms_one"]], f"cuda:{dev}")
    return dict(ms=per_step, ms_seq=per_seq, launches=nlaunch, clocks=clk.summary(), kern=kern, gops=len(gops),
                e2e=e2e)


def e2e_api(args, frames_host, world):
    """The clip through the encoder's public API (libmav1.so), timed by wall
    clock per step: two live encoders, one per closed GOP, each on its own
    host thread; then one encoder coding the whole clip. The encoders are
    created before the timed region (a key frame starts each GOP, so every
    step codes the same bitstream again)."""
    import hashlib
    import torch
    import mav1api
    import mav1cu

    cfg = mav1cu.cli_config(SPEC.width, SPEC.height, **FLAGS)
    keyint = FLAGS["keyint"]
    gops = [frames_host[i:i + keyint] for i in range(0, len(frames_host), keyint)]
    want = json.load(open(GOLDEN))[GOLDEN_CASE]

    def run_parallel(encs, parts, out):
        def one(i):
            out[i] = mav1api.code_frames(encs[i], parts[i], len(parts[i]))
        th = [threading.Thread(target=one, args=(i,)) for i in range(len(parts))]
        t0 = time.perf_counter()
        for t in th:
            t.start()
        for t in th:
            t.join()
        return time.perf_counter() - t0

    def measure(parts, steps, warmup, check):
        encs = [mav1api.Encoder(cfg) for _ in parts]
        try:
            times, bitexact = [], None
            for i in range(warmup + steps):
                if world > 1:
                    import torch.distributed as dist
                    dist.barrier()
                out = [None] * len(parts)
                dt = run_parallel(encs, parts, out)
                if any(o is None for o in out):
                    raise RuntimeError("an encoder thread failed")
                if i >= warmup:
                    times.append(dt)
                    if check and bitexact is None:
                        packets = [p for pk, _ in out for p in pk]
                        recons = [r for _, rc in out for r in rc]
                        bitexact = (len(packets) == want["packets"] and
                                    hashlib.sha256(mav1api.ivf_bytes(packets, SPEC.width, SPEC.height)).hexdigest()
                                    == want["ivf"] and
                                    hashlib.sha256(b"".join(p.tobytes() for r in recons for p in r)).hexdigest()
                                    == want["recon"])
            c = [e.counters() for e in encs]
            tot = dict(frames=sum(x.frames for x in c), h2d=sum(x.h2d_bytes for x in c),
                       d2h=sum(x.d2h_bytes for x in c), entropy_s=sum(x.entropy_s for x in c))
        finally:
            for e in encs:
                e.close()
        return times, bitexact, tot

    steps = max(3, args.steps)
    times, bitexact, tot = measure(gops, steps, args.warmup, True)
    runs = args.warmup + steps
    times_one, bitexact_one, _ = measure([frames_host], max(1, steps // 4), 1, True)
    if not (bitexact and bitexact_one):
        raise SystemExit("e2e: the timed encode's bitstream or reconstructions differ from the oracle's hashes")
    return dict(ms=1e3 * sum(times) / len(times), ms_one=1e3 * sum(times_one) / len(times_one),
                h2d=tot["h2d"] // runs, d2h=tot["d2h"] // runs, entropy_ms=1e3 * tot["entropy_s"] / runs,
                bitexact=bool(bitexact and bitexact_one), encoders=len(gops),
                threads=int(os.environ.get("MAV1_CUDA_THREADS", os.cpu_count())))


def stage_calls(sess, presets, intra):
    """The backend's stages of one frame on an engine session, in order."""
    calls = [] if intra else [("motion_search", sess.motion_search)]
    return calls + [("analyze", sess.analyze), ("edge_types", sess.edge_types), ("recon", sess.recon),
                    ("filter_info", sess.filter_info), ("filter", lambda: sess.filter(presets)),
                    ("cdef_select", lambda: sess.cdef_select(4))]


def frame_stages(frames_dev, fn, kinds=("key", "arf")):
    """Codes the clip's first key and ALTREF frames through a fresh stream,
    and after each one calls fn(kind, engine session, stage list) while the
    engine still holds that frame's inputs (a stage re-run reproduces its
    outputs from them; the frame's reference slots were written already)."""
    import mav1cu

    cfg = mav1cu.cli_config(SPEC.width, SPEC.height, **FLAGS)
    jobs = mav1cu.plan(cfg, SPEC.frames)
    picks = {"key": jobs[0], "arf": next(j for j in jobs if j["kind"] == 1)}
    st = mav1cu.Stream(cfg)
    out = {}
    try:
        for kind in ("key", "arf"):
            j = picks[kind]
            st.encode(j, frames_dev[j["disp"]].data_ptr(), True)
            st.synchronize()
            if kind not in kinds:
                continue
            es = st.engines[st.engine_of(j)]
            fp, presets = mav1cu.frame_params(cfg, j)
            es.set_params(fp)
            out[kind] = fn(kind, es, stage_calls(es, presets, kind == "key"))
            es.synchronize()
    finally:
        st.close()
    return out


def kernel_times(frames_dev):
    """Device time of every stage of the clip's first key and ALTREF frames
    (CUDA events on the engine's own stream, median of 5 after 2 warm-up
    runs). The key frame's recon stage is the dominant kernel k_recon_blocks
    (the intra block workers) plus four short set-up launches."""
    import torch

    def timeit(kind, es, calls):
        ext = torch.cuda.ExternalStream(es.lib.mav1cu_get_stream(es.h))
        res = {}
        for _ in range(2):
            for name, fn in calls:
                fn()
        es.synchronize()
        for name, fn in calls:
            tt = []
            for _ in range(5):
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                ev[0].record(ext)
                fn()
                ev[1].record(ext)
                ev[1].synchronize()
                tt.append(ev[0].elapsed_time(ev[1]))
            res[name] = statistics.median(tt)
        return res

    return frame_stages(frames_dev, timeit)


def work_counts():
    """The counting build's work units of every stage of the same two frames
    (one run of each stage between a reset and a read), and the device's
    measured integer-operation peak. Runs in its own process (the counting
    library's kernels and counters)."""
    import ctypes
    import torch
    import mav1cu

    mav1cu._lib = lib_ = mav1cu.load_count_library()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    frames_dev = torch.from_numpy(load_clip(SPEC)[:8]).cuda()

    def count(kind, es, calls):
        res = {}
        for name, fn in calls:
            es.synchronize()
            lib_.mav1cu_work_reset()
            fn()
            es.synchronize()
            res[name] = {k: v for k, v in mav1cu.work_read(lib_).items() if v}
        return res

    out = frame_stages(frames_dev, count)
    peak = ctypes.c_double()
    if lib_.mav1cu_work_int_peak(ctypes.byref(peak)) != 0:
        raise RuntimeError("mav1cu_work_int_peak failed")
    out["int_peak_ops_s"] = peak.value
    return out


# Integer operations per counted unit (include/mav1cu_count.h): a SAD byte
# pair is an absolute difference and an add; a 4x4 SATD unit 16 differences,
# the two Hadamard passes (64 adds), 16 absolute values and 16 adds; an
# inter-predicted sample 8 + 8 multiply-accumulates; an intra-predicted
# sample about 4 (DC none, SMOOTH 4 multiply-adds); a CfL SSE term a
# multiply, round, clip, difference and square-add; a multiply-accumulate 2;
# a quantised coefficient about 8 (scale, round, 64-bit reciprocal multiply,
# shifts, sign); inverse-transform and loop-restoration counts are operations
# and taps of 2; a CDEF tap about 6 (difference, constrain, weight, add).
WORK_OPS = {"me_sad": 2, "me_dec_sad": 2, "me_satd": 112, "qpel_taps": 2, "ana_satd": 112, "ana_inter_px": 32,
            "ana_intra_px": 4, "ana_cfl": 6, "rec_inter_px": 32, "rec_intra_px": 4, "fwd_mac": 2, "quant": 8,
            "inv_ops": 1, "lf_taps": 2, "cdef_taps": 6, "lr_taps": 2}


def run_work_counts():
    """work_counts() in a child process (the counting library must not share
    a process with the product library); None if it fails."""
    try:
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--work-counts"], capture_output=True, text=True,
                           timeout=600)
        return json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else None
    except Exception:
        return None


def int_roofline(times, counts):
    """Counted integer operations of every stage of the key and ALTREF
    frames over the stage's device time, against the measured peak."""
    peak = counts.get("int_peak_ops_s")
    out = []
    for kind in ("key", "arf"):
        for stage, ms in times.get(kind, {}).items():
            units = counts.get(kind, {}).get(stage, {})
            ops = sum(WORK_OPS[k] * v for k, v in units.items())
            ent = {"frame": kind, "stage": stage, "ms": round(ms, 4), "int_ops": ops, "units": units}
            if ops and ms > 0:
                ent["int_ops_per_s"] = round(ops / (ms * 1e-3) / 1e12, 4)
                ent["frac_of_int_peak"] = round(ops / (ms * 1e-3) / peak, 5) if peak else None
            out.append(ent)
    return {"unit": "Tops/s", "peak_int_ops_per_s": round(peak / 1e12, 2) if peak else None,
            "peak_source": "measured (mav1cu_work_int_peak: multiply-add, xor, add chains on every SM)",
            "stages": out}


# Bytes the key-frame reconstruction must move at 1080p, each once: source
# read (3,133,440), reconstruction written (3,133,440), block records read and
# written (510 superblocks x 64 x 108 bytes, twice), coefficients written
# (510 x 6144 x 4), forward matrices read (61,440 x 4).
KEY_RECON_BYTES = 2 * 3133440 + 2 * 510 * 64 * 108 + 510 * 6144 * 4 + 61440 * 4
# dram__bytes_read.sum + dram__bytes_write.sum of that launch of k_recon_blocks
# in one ncu capture (the key frame of `bench.py --profile-frames 3
# --profile-export`: 18.467 MB read + 1.447 MB written,
# profiles/k_recon_blocks_1080p_turbo_3frames.md).
KEY_RECON_DRAM_BYTES = 19914752


# Integer-pipe figures of each stage's main kernel from the committed ncu
# captures (profiles/*_1080p_turbo_3frames.md: the clip's first key, ALTREF
# and leaf frames): the ALU pipe's share of its peak and the issue slots
# active, ranges over the captured launches.
STAGE_NCU = {
    "motion_search": ("k_me_level", "31-48", "27-55", "profiles/k_me_level_1080p_turbo_3frames.md"),
    "analyze": ("k_analyze_level", "23-31", "33-42", "profiles/k_analyze_level_1080p_turbo_3frames.md"),
    "recon": ("k_recon_inter", "22", "31-33", "profiles/k_recon_inter_1080p_turbo_3frames.md"),
    "filter": ("k_deblock, k_cdef", "49-59", "63-67", "profiles/k_deblock_1080p_turbo_3frames.md"),
}


def roofline(kern, peaks, counts=None):
    """Roofline of the dominant kernel (k_recon_blocks) through its stage on
    the key frame: algorithmic bytes over the measured stage time, against the
    measured HBM copy bandwidth. The kernel is a dependency chain (latency
    bound), so the fraction is small by nature; `stages_altref_frame` gives
    every stage's live time on an ALTREF frame with its main kernel's
    integer-pipe utilisation from the committed ncu captures, and `int_ops`
    the counted integer operations of every stage of the key and ALTREF
    frames against the measured integer peak (counts: work_counts())."""
    if not kern:
        return None
    key_recon_ms = kern["key"]["recon"]
    t = key_recon_ms * 1e-3
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = KEY_RECON_BYTES / t / 1e9
    stages = []
    for name, ms in kern["arf"].items():
        ent = {"stage": name, "ms": round(ms, 4)}
        if name in STAGE_NCU:
            k, alu, issue, src = STAGE_NCU[name]
            ent.update({"kernel": k, "alu_pipe_pct_of_peak": alu, "issue_active_pct": issue, "ncu": src})
        stages.append(ent)
    return {"bound": "hbm", "kernel": "k_recon_blocks (key-frame recon stage)", "achieved": round(achieved, 2),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 6), "traffic": KEY_RECON_DRAM_BYTES,
            "algorithmic_bytes": KEY_RECON_BYTES, "ms_per_launch": round(key_recon_ms, 3),
            "stages_altref_frame": stages,
            "int_ops": int_roofline(kern, counts) if counts else None,
            "peak_source": "MEASURED_PEAKS.json" if "hbm_gbs" in peaks else "fallback"}


def cpu_reference(sample_frames):
    """The reference encoder's own CPU path (oracle/_ref: its scalar backend
    with OpenMP-parallel stages over all host threads, its entropy coder and
    OBU writer) through the mav1.h queue API, like its CLI, on the clip's
    first `sample_frames` frames. Returns (fps by wall clock, wall seconds,
    fps if the process's CPU time were spread over every host core: a bound
    for the reference's frame-engine mode, which this build of its driver
    does not run)."""
    import resource
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    w, h = SPEC.width, SPEC.height
    cw, ch = (w + 1) // 2, (h + 1) // 2
    frames = []
    for f in load_clip(SPEC)[:sample_frames]:
        y, u, v = np.split(f, [w * h, w * h + cw * ch])
        frames.append([y.reshape(h, w), u.reshape(ch, cw), v.reshape(ch, cw)])
    cfg = oracle.cli_config(w, h, **FLAGS)
    r0 = resource.getrusage(resource.RUSAGE_SELF)
    t0 = time.perf_counter()
    packets, _ = oracle.encode(frames, cfg)
    wall = time.perf_counter() - t0
    r1 = resource.getrusage(resource.RUSAGE_SELF)
    cpu = (r1.ru_utime - r0.ru_utime) + (r1.ru_stime - r0.ru_stime)
    assert len(packets) == sample_frames
    return sample_frames / wall, wall, sample_frames * os.cpu_count() / cpu


def profile_run(n, export=False, lr=False):
    """Codes the first n planned frames once (a short run for ncu): the
    benchmark clip, or with lr a 640x360 clip with every tool on (loop
    restoration searched on the device); with export, every frame's writer
    inputs and reconstruction are exported into page-locked memory."""
    import torch
    import mav1cu

    if lr:
        spec = synthetic.ClipSpec(640, 360, n, seed=35, rects=5, rect_size=(32, 96))
        frames_host = np.stack([np.frombuffer(synthetic.packed(f), np.uint8) for f in synthetic.generate(spec)])
        cfg = mav1cu.cli_config(spec.width, spec.height, q=110, altref=4, tiles=2)
    else:
        spec = SPEC
        frames_host = load_clip(SPEC)
        cfg = mav1cu.cli_config(SPEC.width, SPEC.height, **FLAGS)
    jobs = mav1cu.plan(cfg, spec.frames)[:n]
    st = mav1cu.Stream(cfg)
    frames_dev = torch.from_numpy(frames_host[: max(j["disp"] for j in jobs) + 1]).cuda()
    image = torch.empty(st.session.export_capacity(), dtype=torch.uint8).pin_memory() if export else None
    for j in jobs:
        sess = st.encode(j, frames_dev[j["disp"]].data_ptr(), True)
        if export:
            sess.export(image.data_ptr(), image.numel(), rec=True)
            st.synchronize()
    st.synchronize()
    print(json.dumps({"profile_frames": n, "kinds": [int(j["kind"]) for j in jobs], "launches": int(st.launches())}))
    st.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=REF_SAMPLE, help="frames of the CPU baseline sample")
    ap.add_argument("--no-roofline", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 16-stream batching measurement")
    ap.add_argument("--batch-passes", type=int, default=2)
    ap.add_argument("--workload", default="clip", choices=["clip", "serving", "full4k"],
                    help="serving: the session-serving measurement alone (about two minutes); full4k: the 4K "
                         "full-tool configuration")
    ap.add_argument("--full4k-passes", type=int, default=1)
    ap.add_argument("--serving-sessions", type=int, default=400)
    ap.add_argument("--work-counts", action="store_true",
                    help="print the counting build's per-stage work units of the clip's first key and ALTREF frames "
                         "and the measured integer peak (JSON), then exit")
    ap.add_argument("--profile-frames", type=int, default=0,
                    help="code the clip's first N planned frames once and exit (a short run for ncu)")
    ap.add_argument("--profile-export", action="store_true", help="with --profile-frames: export every frame")
    ap.add_argument("--profile-lr", action="store_true",
                    help="with --profile-frames: a 640x360 clip with every tool on (loop restoration)")
    args = ap.parse_args()
    if args.work_counts:
        print(json.dumps(work_counts()))
        return
    if args.profile_frames:
        profile_run(args.profile_frames, export=args.profile_export, lr=args.profile_lr)
        return
    if args.workload == "full4k":
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        print(json.dumps(full4k_bench(args)))
        return
    if args.workload == "serving":
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        b = batch_bench(args)
        with Clocks(int(os.environ.get("LOCAL_RANK", 0))) as clk:
            res = serving_bench(args, b["mpx_per_s_concurrent"] * 1e6)
        res["clocks"] = clk.summary()
        res["batch"] = b
        print(json.dumps({"workload": "serving", **res}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    cores = os.cpu_count()

    if args.impl == "reference":
        if rank != 0:
            return
        walls, fps_ideal = [], []
        for i in range(args.warmup + args.steps):
            fps, wall, ideal = cpu_reference(REF_SAMPLE)
            if i >= args.warmup:
                walls.append(wall)
                fps_ideal.append(ideal)
        v = REF_SAMPLE * len(walls) / sum(walls)
        sample = (f"per step: the clip's first {REF_SAMPLE} frames (1 key, 14 hidden ALTREF, 14 leaf and 1 regular "
                  f"frame), coded and entropy-coded through the reference's mav1.h calls, wall clock; its driver runs "
                  f"frames one after another (serial frame mode), its stages in parallel on all host threads")
        line = {"metric": METRIC, "value": round(v, 3), "unit": "fps", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(1e3 * sum(walls) / len(walls), 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32",
                "data": "synthetic", "config": CONFIG, "impl": "reference",
                "cpu_baseline": {"value": round(v, 3), "unit": "fps", "cores": cores, "kind": "reference",
                                 "sample": sample,
                                 "fps_if_all_cores_busy": round(sum(fps_ideal) / len(fps_ideal), 3)},
                "e2e": {"value": round(v, 3), "unit": "fps", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    r = run_ours(args, rank, world)
    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        frames = SPEC.frames * world
        value = frames / (r["ms"] * 1e-3)
        x = r["e2e"]
        e2e = frames / (x["ms"] * 1e-3)
        line = {"metric": METRIC, "value": round(value, 2), "unit": "fps", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(r["ms"], 3), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u8/int32", "data": "synthetic", "config": CONFIG,
                "parallelism": "replicas" if world > 1 else "single",
                "e2e": {"value": round(e2e, 2), "unit": "fps", "h2d_bytes_per_step": x["h2d"],
                        "d2h_bytes_per_step": x["d2h"], "ms_per_step": round(x["ms"], 2),
                        "path": "libmav1.so (mav1.h): host frames in, IVF temporal units and reconstructions out",
                        "bitexact_to_oracle": x["bitexact"], "encoders": x["encoders"],
                        "host_entropy_threads": x["threads"], "entropy_thread_ms_per_step": round(x["entropy_ms"], 1),
                        "fps_one_encoder": round(frames / (x["ms_one"] * 1e-3), 2)},
                "schedule": {"gop_parallel_streams": r["gops"], "frame_engines_per_stream": 2,
                             "fps_one_stream": round(frames / (r["ms_seq"] * 1e-3), 2)},
                "gpu_launches": int(r["launches"]), "clocks": r["clocks"],
                "roofline": roofline(r["kern"], peaks, run_work_counts() if r["kern"] else None)}
        if not args.no_batch:
            try:
                line["batch"] = batch_bench(args)
            except Exception as ex:  # reported in the line; the clip's numbers stand on their own
                line["batch"] = {"error": f"{type(ex).__name__}: {ex}"}
        if not args.no_cpu_baseline:
            fps, wall, ideal = cpu_reference(args.cpu_sample)
            line["cpu_baseline"] = {"value": round(fps, 3), "unit": "fps", "cores": cores, "kind": "reference",
                                    "sample": f"the clip's first {args.cpu_sample} frames through the reference's "
                                              f"mav1.h calls, entropy coding included ({wall:.1f} s wall clock); "
                                              f"serial frame mode, stages parallel on all host threads",
                                    "fps_if_all_cores_busy": round(ideal, 3)}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
