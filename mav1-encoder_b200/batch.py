"""Batched encoding of many streams of uneven size on one GPU.

A batch codes N streams (each its own configuration and resolution) at the
same time through the encoder API (libmav1.so): every stream has a live
encoder with its device state resident in HBM (its frame engines and their
CUDA streams), all of them share the device and the process-wide host
entropy pool, and a host thread per stream feeds its frames and collects its
temporal units. The device interleaves the streams' stage kernels; the host
pool codes whichever frames are ready. The same streams coded one after
another, each alone on the GPU, are the baseline the batch is measured
against; every stream's bitstream is the same either way.

Clip generation for the batching workload is CPU-heavy (about 5 minutes on
one core for the 16-stream mix), so load_streams() generates clips in a pool
of processes started with `spawn` (safe next to a CUDA context) and caches
them on local disk.
"""
import hashlib
import multiprocessing as mp
import os
import threading
import time

import numpy as np

import synthetic


def _gen(spec):
    return synthetic.packed_clip(spec)


def load_streams(specs, cache_dir="/tmp", workers=None):
    """The packed I420 frames of every clip ([frames, bytes] uint8 arrays),
    from the cache when present, otherwise generated in parallel."""
    paths = [os.path.join(cache_dir, f"mav1_clip_{s.name}_{s.seed}_{s.frames}.npy") for s in specs]
    out = [np.load(p) if os.path.exists(p) else None for p in paths]
    todo = [i for i, o in enumerate(out) if o is None]
    if todo:
        ctx = mp.get_context("spawn")
        n = workers or min(len(todo), os.cpu_count() or 1)
        with ctx.Pool(n) as pool:
            for i, arr in zip(todo, pool.map(_gen, [specs[i] for i in todo])):
                out[i] = arr
                try:
                    np.save(paths[i] + ".tmp.npy", arr)
                    os.replace(paths[i] + ".tmp.npy", paths[i])
                except OSError:
                    pass
    return out


def _code_stream(enc, frames, out, i, recon):
    import mav1api
    try:
        out[i] = mav1api.code_frames(enc, frames, len(frames), recon=recon)
    except Exception as e:  # reported by the caller
        out[i] = e


class Batch:
    """N streams [(mav1cu config record, frames)] with a live encoder each.

    Each stream is a closed GOP run (its clip starts with a key frame and has
    no key frame inside, or its key frames fall on its keyint boundaries):
    every call of code() codes every stream's clip once more, to the same
    bitstream, without re-creating the encoders."""

    def __init__(self, streams):
        import mav1api
        self.streams = streams
        self.encoders = [mav1api.Encoder(cfg) for cfg, _ in streams]

    def code(self, concurrent=True, recon=False):
        """Codes every stream's frames; returns (wall seconds, [(packets,
        reconstructions)] per stream). concurrent: all streams at once (a
        host thread each); else one after another."""
        out = [None] * len(self.streams)
        t0 = time.perf_counter()
        if concurrent:
            th = [threading.Thread(target=_code_stream, args=(e, fr, out, i, recon))
                  for i, (e, (_, fr)) in enumerate(zip(self.encoders, self.streams))]
            for t in th:
                t.start()
            for t in th:
                t.join()
        else:
            for i, (e, (_, fr)) in enumerate(zip(self.encoders, self.streams)):
                _code_stream(e, fr, out, i, recon)
        wall = time.perf_counter() - t0
        for o in out:
            if isinstance(o, Exception):
                raise o
        return wall, out

    def close(self):
        for e in self.encoders:
            e.close()
        self.encoders = []


def stream_hashes(result, width, height):
    """IVF SHA-256 of one stream's temporal units."""
    import mav1api
    packets, _ = result
    return hashlib.sha256(mav1api.ivf_bytes(packets, width, height)).hexdigest()
