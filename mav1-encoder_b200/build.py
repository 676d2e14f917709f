"""Builds libmav1cu.so (the sm_100a kernels and their C ABI) and libmav1.so
(the mav1 encoder API over it) in-tree.

nvcc compiles the translation units csrc/session.cu (the session and stream
API over every stage) and csrc/edge_noalloc.cu (the entry point that
allocates nothing) for compute_100a / sm_100a with line info; host code is
compiled without
floating-point contraction (the forward-matrix derivation must round like
the reference's). The library lands next to this file so it travels with
the working tree.

libmav1.so is the encoder's public API (src/mav1.h of the reference,
unchanged) on this backend: the host driver host/encoder_cuda.c, the glue
host/writer.c and the reference's own entropy coder and OBU writer
(src/obu.c, tile_writer.c, mvpred.c, entenc.c, cdfs.c, bitwriter.c and the
LR-unit rate coding of lr_search.c), compiled in place from the reference
checkout named by MAV1_REFERENCE. Where that checkout is absent, an existing
libmav1.so is kept as it is.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmav1cu.so")
API_LIB = os.path.join(HERE, "libmav1.so")
HOST = os.path.join(HERE, "host")
REFERENCE = os.environ.get("MAV1_REFERENCE", "/root/reference")
# the reference's host sources of entropy coding and OBU assembly, linked unchanged
REF_WRITER_SRCS = ["obu.c", "cdfs.c", "entenc.c", "bitwriter.c", "mvpred.c", "lr_search.c"]
CC = os.environ.get("CC", "gcc")
CFLAGS = ["-O2", "-g", "-std=gnu11", "-fPIC", "-ffp-contract=off", "-pthread", "-Wall", "-Wno-unused-function",
          "-Wno-unused-parameter", "-Wno-unused-variable", "-Wno-unused-but-set-variable"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-shared",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-O2",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.inc")) +
                  [os.path.join(ROOT, "include", "mav1cu.h")])


def stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=(), out=LIB):
    deps = sources()
    if not force and not stale(out, deps):
        return out
    cmd = [NVCC, *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           os.path.join(CSRC, "session.cu"), os.path.join(CSRC, "edge_noalloc.cu"), "-o", out + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    os.replace(out + ".tmp", out)
    return out


COUNT_LIB = os.path.join(HERE, "libmav1cu_count.so")


def build_count(force=False, verbose=False):
    """libmav1cu_count.so: the same kernels with their work counters compiled
    in (-DMAV1CU_COUNT, include/mav1cu_count.h), for the per-stage integer
    operation counts of the benchmark; never on the coding path."""
    deps = sources() + [os.path.join(ROOT, "include", "mav1cu_count.h")]
    if not force and not stale(COUNT_LIB, deps):
        return COUNT_LIB
    return build(force=True, verbose=verbose, extra=("-DMAV1CU_COUNT",), out=COUNT_LIB)


def build_api(force=False, verbose=False):
    """libmav1.so: the mav1.h API over libmav1cu.so (needs the reference's
    sources for its entropy coder; kept as built where they are absent)."""
    src = os.path.join(REFERENCE, "src")
    if not os.path.isdir(src):
        if os.path.exists(API_LIB):
            return API_LIB
        raise RuntimeError(f"libmav1.so needs the reference sources (MAV1_REFERENCE={REFERENCE})")
    ours = [os.path.join(HOST, "encoder_cuda.c"), os.path.join(HOST, "writer.c")]
    ref = [os.path.join(src, f) for f in REF_WRITER_SRCS]
    deps = ours + ref + glob.glob(os.path.join(HOST, "*.h")) + glob.glob(os.path.join(src, "*.h")) + \
        glob.glob(os.path.join(src, "kernels", "*.h")) + [LIB, os.path.join(ROOT, "include", "mav1cu.h")]
    if not force and not stale(API_LIB, deps):
        return API_LIB
    cmd = [CC, *CFLAGS, "-shared", "-I", os.path.join(ROOT, "include"), "-I", HOST, "-I", src,
           "-I", os.path.join(HOST, "compat"), *ours, *ref, "-L", HERE, "-lmav1cu", "-Wl,-rpath,$ORIGIN",
           "-lm", "-o", API_LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("gcc failed:\n" + r.stdout + r.stderr)
    os.replace(API_LIB + ".tmp", API_LIB)
    build_cli(verbose)
    return API_LIB


def build_cli(verbose=False):
    """The reference's command-line encoder (tools/mav1enc.c, unchanged)
    linked against libmav1.so: y4m in, IVF out, on this backend."""
    tool = os.path.join(REFERENCE, "tools", "mav1enc.c")
    out = os.path.join(HERE, "mav1enc")
    cmd = [CC, "-O2", "-std=gnu11", tool, "-L", HERE, "-lmav1", "-lmav1cu", "-Wl,-rpath,$ORIGIN", "-lm",
           "-o", out + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("gcc failed:\n" + r.stdout + r.stderr)
    os.replace(out + ".tmp", out)
    return out


def build_all(force=False, verbose=False):
    build(force=force, verbose=verbose)
    build_count(force=force, verbose=verbose)
    return build_api(force=force, verbose=verbose)


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv, verbose=True))
