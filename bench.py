#!/usr/bin/env python3
"""1080p turbo encode benchmark of the B200 encode backend.

Workload (the reference's 1080p turbo configuration): a seeded synthetic
1920x1080 8-bit 4:2:0 clip of 120 frames (pan (+2.5, +1.0) px/frame, 12
moving rectangles of 64-256 px, noise sigma 2), coded with --turbo -q 125
--keyint 60 --tiles 2 (deblocking and CDEF on, loop restoration off). One
step = the whole clip in coding order (2 key frames, 58 hidden ALTREF frames,
58 leaf frames, 2 regular frames) through every device stage of the encode
backend: source load, motion search, mode/partition analysis, edge types,
reconstruction, filter info, deblocking, CDEF and CDEF selection, reference
slot refresh. Entropy coding and OBU assembly (host steps of the encoder,
not part of this path) are not timed.

value: frames/s with the source frames resident in HBM (CUDA events on the
       session stream, max over ranks).
e2e:   the same through the C ABI from pinned host memory: every frame's
       source is copied host->device (an upload stream per engine, ahead of
       the engine), and its entropy-coder inputs (superblock table, CDEF
       choices, the blocks in use, the levels of coded planes) plus, for
       shown frames, the visible I420 reconstruction are packed on the device
       and stored into mapped pinned host memory (mav1cu_export, on each
       engine's transfer stream), all inside the timed region.
       d2h_bytes_per_step counts the bytes the export images hold (their
       headers' byte counts, read in an untimed pass over the same step).
--impl reference: the reference encoder's own scalar CPU path (oracle/_ref,
       built from the reference sources) on the host cores, all threads.

Multi-GPU: the path does not shard (one stream is a serial reference
chain); --gpus N runs N independent replicas, one per GPU.
"""
import argparse
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

import synthetic  # noqa: E402

METRIC = "1080p turbo encode fps on 1 B200 (bit-exact to --cpu)"
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
    pinned = torch.from_numpy(frames_host).pin_memory()
    geom = mav1cu.geometry(SPEC.width, SPEC.height)
    # one export image per engine of each GOP stream: a frame's image stays
    # intact until that engine's next frame
    cap = streams[0].session.export_capacity()
    images = {(g, k): torch.empty(cap, dtype=torch.uint8).pin_memory()
              for g in range(len(gops)) for k in range(len(streams[0].engines))}

    def step_device(order=order):
        for g, j in order:
            streams[g].encode(j, frames_dev[j["disp"]].data_ptr(), True)

    def step_sequential():
        step_device(seq_order)

    def e2e_frame(g, j):
        sess = streams[g].encode(j, pinned[j["disp"]].data_ptr(), False)
        img = images[(g, mav1cu.Stream.engine_of(j))]
        sess.export(img.data_ptr(), cap, rec=not j["hidden"])
        return img

    def step_e2e():
        for g, j in order:
            e2e_frame(g, j)

    def d2h_bytes():
        """Bytes one e2e step moves device->host, frame by frame (untimed)."""
        total = 0
        for g, j in order:
            img = e2e_frame(g, j)
            streams[g].synchronize()
            h = img[:mav1cu.EXPORT_HEADER_DTYPE.itemsize].numpy().view(mav1cu.EXPORT_HEADER_DTYPE)[0]
            assert h["status"] == 0
            total += int(h["bytes"])
        return total

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
    ms_e2e, _ = timed(step_e2e, max(1, args.steps // 2), 1)
    d2h_per_step = d2h_bytes()
    per_step = sum(ms) / len(ms)
    per_e2e = sum(ms_e2e) / len(ms_e2e)
    per_seq = sum(ms_seq) / len(ms_seq)
    if world > 1:
        per_step, per_e2e, per_seq = max_over_ranks([per_step, per_e2e, per_seq], f"cuda:{dev}")
    kern = kernel_times(streams[0].session, S, frames_dev) if (rank == 0 and not args.no_roofline) else None
    for st in streams:
        st.close()
    return dict(ms=per_step, ms_e2e=per_e2e, ms_seq=per_seq, launches=nlaunch, clocks=clk.summary(),
                h2d=SPEC.frames * fbytes, d2h=d2h_per_step, kern=kern, gops=len(gops))


def kernel_times(sess, stream, frames_dev):
    """Device times for the roofline, with CUDA events on the stream the
    kernels are launched on.

    dominant: the reconstruction stage of the clip's first key frame, which is
    the dominant kernel k_recon_blocks (the intra block workers, 28% of the
    clip's device time in the ncu launch list) plus four short set-up
    launches.
    A fresh stream codes the key frame, then the stage is re-run on the engine
    session that holds the frame's analysis output (recon reproduces its
    outputs from the same inputs). stage_ms: every stage of one ALTREF frame,
    for reference."""
    import torch
    import mav1cu

    cfg = mav1cu.cli_config(SPEC.width, SPEC.height, **FLAGS)
    jobs = mav1cu.plan(cfg, SPEC.frames)
    key = jobs[0]
    st = mav1cu.Stream(cfg)
    st.encode(key, frames_dev[key["disp"]].data_ptr(), True)
    st.synchronize()
    es = st.engines[st.engine_of(key)]
    ext = torch.cuda.ExternalStream(st.lib.mav1cu_get_stream(es.h))
    ts = []
    for i in range(8):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(ext)
        es.recon()
        ev[1].record(ext)
        ev[1].synchronize()
        if i >= 3:
            ts.append(ev[0].elapsed_time(ev[1]))
    es.synchronize()
    key_recon_ms = statistics.median(ts)
    st.close()

    # every stage of one ALTREF frame (inputs: whatever the session holds)
    sess.set_stream(stream.cuda_stream)
    arf = next(j for j in jobs if j["kind"] == 1)
    fp, presets = mav1cu.frame_params(cfg, arf)
    sess.set_params(fp)
    stages = [("motion_search", sess.motion_search), ("analyze", sess.analyze), ("edge_types", sess.edge_types),
              ("recon", sess.recon), ("filter_info", sess.filter_info), ("filter", lambda: sess.filter(presets)),
              ("cdef_select", lambda: sess.cdef_select(4))]
    res = {}
    with torch.cuda.stream(stream):
        for _ in range(3):
            for name, fn in stages:
                fn()
        stream.synchronize()
        for name, fn in stages:
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            tt = []
            for _ in range(5):
                ev[0].record(stream)
                fn()
                ev[1].record(stream)
                ev[1].synchronize()
                tt.append(ev[0].elapsed_time(ev[1]))
            res[name] = statistics.median(tt)
    return {"key_recon_ms": key_recon_ms, "arf_stage_ms": res}


# Bytes the key-frame reconstruction must move at 1080p, each once: source
# read (3,133,440), reconstruction written (3,133,440), block records read and
# written (510 superblocks x 64 x 108 bytes, twice), coefficients written
# (510 x 6144 x 4), forward matrices read (61,440 x 4).
KEY_RECON_BYTES = 2 * 3133440 + 2 * 510 * 64 * 108 + 510 * 6144 * 4 + 61440 * 4
# dram__bytes_read.sum + dram__bytes_write.sum of that launch of k_recon_blocks
# in one ncu capture (the key frame of `bench.py --profile-frames 3`).
KEY_RECON_DRAM_BYTES = 19850000


def roofline(kern, peaks):
    """Roofline of the dominant kernel (k_recon_blocks) through its stage on
    the key frame: algorithmic bytes over the measured stage time, against the
    measured HBM copy bandwidth. The kernel is a dependency chain (latency
    bound), so the fraction is small by nature."""
    if not kern:
        return None
    t = kern["key_recon_ms"] * 1e-3
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = KEY_RECON_BYTES / t / 1e9
    return {"bound": "hbm", "kernel": "k_recon_blocks (key-frame recon stage)", "achieved": round(achieved, 2),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 6), "traffic": KEY_RECON_DRAM_BYTES,
            "algorithmic_bytes": KEY_RECON_BYTES, "ms_per_launch": round(kern["key_recon_ms"], 3),
            "arf_stage_ms": {k: round(v, 4) for k, v in kern["arf_stage_ms"].items()},
            "peak_source": "MEASURED_PEAKS.json" if "hbm_gbs" in peaks else "fallback"}


def cpu_reference(args, sample_frames, per_kind=True):
    """The reference's scalar CPU path (oracle/_ref) on the host cores: the
    backend stages of the first `sample_frames` frames of the clip, timed per
    frame between run_frame_core's first and last stage hook; fps of the
    120-frame clip from the per-kind mean times weighted by the clip's kind
    counts."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    frames = [np.split(f, [SPEC.width * SPEC.height, SPEC.width * SPEC.height + ((SPEC.width + 1) // 2) * ((SPEC.height + 1) // 2)])
              for f in load_clip(SPEC)[:sample_frames]]
    frames = [[f[0].reshape(SPEC.height, SPEC.width), f[1].reshape((SPEC.height + 1) // 2, -1),
               f[2].reshape((SPEC.height + 1) // 2, -1)] for f in frames]
    cfg = oracle.cli_config(SPEC.width, SPEC.height, **FLAGS)
    times = []

    class Tr:
        pass

    tr = Tr()
    state = {}

    def hook(user, stage, e):
        if stage == oracle.STAGE["PARAMS"]:
            state["t0"] = time.perf_counter()
            state["kind"] = oracle.frame_state(e)
        elif stage == oracle.STAGE["DONE"]:
            k = state["kind"]
            kind = "key" if k["is_key"] else {0: "regular", 1: "arf", 2: "leaf", 3: "arf"}[k["frame_kind"]]
            times.append((kind, time.perf_counter() - state["t0"]))

    tr.cb = oracle.HOOK(hook)
    oracle.encode(frames, cfg, trace=tr)
    by = {}
    for k, t in times:
        by.setdefault(k, []).append(t)
    mean = {k: sum(v) / len(v) for k, v in by.items()}
    counts = {"key": 2, "arf": 58, "leaf": 58, "regular": 2}
    total = sum(counts[k] * mean.get(k, mean.get("arf")) for k in counts)
    return SPEC.frames / total, sum(t for _, t in times), mean


def profile_run(n):
    import torch
    import mav1cu

    frames_host = load_clip(SPEC)
    cfg = mav1cu.cli_config(SPEC.width, SPEC.height, **FLAGS)
    jobs = mav1cu.plan(cfg, SPEC.frames)[:n]
    st = mav1cu.Stream(cfg)
    frames_dev = torch.from_numpy(frames_host[: max(j["disp"] for j in jobs) + 1]).cuda()
    for j in jobs:
        st.encode(j, frames_dev[j["disp"]].data_ptr(), True)
    st.synchronize()
    print(json.dumps({"profile_frames": n, "kinds": [int(j["kind"]) for j in jobs], "launches": int(st.launches())}))
    st.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=16, help="frames of the CPU baseline sample")
    ap.add_argument("--no-roofline", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-frames", type=int, default=0,
                    help="code the clip's first N planned frames once and exit (a short run for ncu)")
    args = ap.parse_args()
    if args.profile_frames:
        profile_run(args.profile_frames)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    cores = os.cpu_count()

    if args.impl == "reference":
        if rank != 0:
            return
        per_step = []
        for i in range(args.warmup + args.steps):
            fps, secs, mean = cpu_reference(args, 8)
            if i >= args.warmup:
                per_step.append(fps)
        v = sum(per_step) / len(per_step)
        line = {"metric": METRIC, "value": round(v, 3), "unit": "fps", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(1000 * SPEC.frames / v, 1), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32", "data": "synthetic",
                "config": CONFIG, "impl": "reference",
                "cpu_baseline": {"value": round(v, 3), "unit": "fps", "cores": cores, "kind": "reference",
                                 "sample": "per step: the backend stages of the clip's first 8 frames (key, ALTREF and "
                                           "leaf frames), per-kind mean time weighted to the 120-frame clip"},
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
        e2e = frames / (r["ms_e2e"] * 1e-3)
        line = {"metric": METRIC, "value": round(value, 2), "unit": "fps", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(r["ms"], 3), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u8/int32", "data": "synthetic", "config": CONFIG,
                "parallelism": "replicas" if world > 1 else "single",
                "e2e": {"value": round(e2e, 2), "unit": "fps", "h2d_bytes_per_step": r["h2d"],
                        "d2h_bytes_per_step": r["d2h"]},
                "schedule": {"gop_parallel_streams": r["gops"], "frame_engines_per_stream": 2,
                             "fps_one_stream": round(frames / (r["ms_seq"] * 1e-3), 2)},
                "gpu_launches": int(r["launches"]), "clocks": r["clocks"],
                "roofline": roofline(r["kern"], peaks)}
        if not args.no_cpu_baseline:
            fps, secs, mean = cpu_reference(args, args.cpu_sample)
            line["cpu_baseline"] = {"value": round(fps, 3), "unit": "fps", "cores": cores, "kind": "reference",
                                    "sample": f"backend stages of the clip's first {args.cpu_sample} frames "
                                              f"({secs:.1f} s of CPU work), per-kind mean time weighted to the 120-frame clip",
                                    "per_kind_ms": {k: round(v * 1e3, 1) for k, v in mean.items()}}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
