"""Host side of the product without a GPU: the C-ABI library loads and
exports every declared entry point, its record layouts and tables equal the
reference's, the host helpers reproduce the reference's outputs, and bad
arguments are rejected before any device work."""
import ctypes
import os
import re

import numpy as np
import pytest

import mav1cu
import oracle
import parity

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mav1cu.h")


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    return sorted(set(re.findall(r"\b(mav1cu_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = mav1cu.lib()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(not oracle.available(), reason="oracle not built")
def test_record_layouts_match_reference():
    sizes = oracle.struct_sizes()
    assert sizes[:4] == [mav1cu.PARAMS_DTYPE.itemsize, mav1cu.BLOCK_DTYPE.itemsize, mav1cu.SB_DTYPE.itemsize,
                         mav1cu.LRUNIT_DTYPE.itemsize]
    assert sizes[4] == mav1cu.PARAMS_DTYPE.fields["turbo"][1]
    assert sizes[5] == mav1cu.PARAMS_DTYPE.fields["lr_unit_off"][1]
    assert sizes[6] == mav1cu.BLOCK_DTYPE.fields["mv1_col"][1]
    assert sizes[7] == mav1cu.SB_DTYPE.fields["part"][1]


@pytest.mark.skipif(not oracle.available(), reason="oracle not built")
def test_forward_matrices_equal_reference():
    import synthetic
    tr = oracle.Trace(stages={oracle.STAGE["PARAMS"]})
    spec = synthetic.ClipSpec(64, 64, 1, seed=1)
    oracle.encode(list(synthetic.generate(spec)), oracle.cli_config(64, 64, q=100), trace=tr)
    ref = tr.mats[: 15 * 4096 * 4].view(np.int32)
    assert np.array_equal(mav1cu.fwd_matrices(), ref)


def test_spec_table_digest():
    import hashlib
    T = parity.spec_tables()
    text = open(os.path.join(ROOT, "mav1-encoder_b200", "csrc", "spec_tables_gen.h")).read()
    digest = re.search(r'MAV1T_DIGEST "(\w+)"', text).group(1)
    order = re.findall(r"#define MAV1T_(\w+)_DIMS", text)
    h = hashlib.sha256()
    for name in order:
        h.update(name.encode())
        h.update(",".join(str(int(v)) for v in T[name].ravel()).encode())
    assert h.hexdigest() == digest


REFERENCE = os.environ.get("MAV1_REFERENCE", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE, "src")), reason="reference checkout absent")
def test_spec_tables_regenerate_identically(tmp_path):
    import subprocess
    import sys
    gen = os.path.join(ROOT, "mav1-encoder_b200", "csrc", "gen_spec_tables.py")
    out = tmp_path / "t.h"
    subprocess.run([sys.executable, gen, os.path.join(REFERENCE, "src"), str(out)], check=True, capture_output=True)
    assert out.read_bytes() == open(os.path.join(ROOT, "mav1-encoder_b200", "csrc", "spec_tables_gen.h"), "rb").read()


def test_bad_arguments_rejected_without_device_work():
    lib = mav1cu.lib()
    h = ctypes.c_void_p()
    err = ctypes.create_string_buffer(256)
    assert lib.mav1cu_session_create(8, 8, 4, ctypes.byref(h), err, 256) == -1
    assert b"unsupported" in err.value
    assert lib.mav1cu_session_create(64, 64, 5, ctypes.byref(h), err, 256) == -1
    jobs = np.zeros(2, mav1cu.JOB_DTYPE)
    assert lib.mav1cu_plan(mav1cu.cli_config(64, 64, turbo=1).ctypes.data, 10, jobs.ctypes.data, 2) == -1


def test_plan_turbo_gop_structure():
    cfg = mav1cu.cli_config(1920, 1080, q=125, turbo=1, keyint=60, tiles=2)
    jobs = mav1cu.plan(cfg, 120)
    kinds = {}
    for j in jobs:
        k = "key" if j["is_key"] else ("arf", "leaf", "mid")[j["kind"] - 1] if j["kind"] else "regular"
        kinds[k] = kinds.get(k, 0) + 1
    assert kinds == {"key": 2, "arf": 58, "leaf": 58, "regular": 2}
    assert sorted(int(j["disp"]) for j in jobs) == list(range(120))


def test_split_large_inverse_dct_is_exact(tmp_path):
    """The two-thread form of the 32- and 64-point inverse DCT equals the
    spec-order butterfly list on the host (tests/native/idct_split_check.cpp)."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "idct_split_check"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "mav1-encoder_b200", "csrc"), "-x", "c++",
                    os.path.join(ROOT, "tests", "native", "idct_split_check.cpp"), "-o", str(exe)],
                   check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr

def test_butterfly_sums_fit_32_bits(tmp_path):
    """Every inverse transform's butterfly sums stay inside 32 bits on
    extreme 16-bit inputs (tests/native/butterfly_range_check.cpp), so the
    32-bit tx::B equals the specification's rotation."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "butterfly_range_check"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "mav1-encoder_b200", "csrc"), "-x", "c++",
                    os.path.join(ROOT, "tests", "native", "butterfly_range_check.cpp"), "-o", str(exe)],
                   check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_forward_matrices_identical_from_concurrent_threads():
    """Sessions are created from several host threads at once (one encoder per
    thread); the forward-matrix table each one gets must be the same."""
    import threading
    want = mav1cu.fwd_matrices()
    out = [None] * 8

    def one(i):
        out[i] = [mav1cu.fwd_matrices() for _ in range(4)]

    th = [threading.Thread(target=one, args=(i,)) for i in range(8)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert all(np.array_equal(m, want) for ms in out for m in ms)


def test_api_ivf_container_equals_the_reference_cli_container():
    """mav1api.ivf_bytes (the container the bench and the API tests hash)
    equals the oracle's, which the oracle tests pin to the reference CLI's
    own output file byte for byte."""
    import mav1api
    rng = np.random.default_rng(9)
    packets = [rng.integers(0, 256, int(n), dtype=np.uint8).tobytes() for n in rng.integers(1, 5000, 17)]
    for (w, h) in ((1920, 1080), (203, 131), (64, 48)):
        a = mav1api.ivf_bytes(packets, w, h)
        assert a == oracle.ivf_bytes(packets, w, h)
        assert a[:4] == b"DKIF" and int.from_bytes(a[24:28], "little") == len(packets)
    assert mav1api.ivf_bytes([], 64, 48) == oracle.ivf_bytes([], 64, 48)
