"""The oracle (the reference's scalar CPU path built from its own sources)
pinned: the reference's unit tests pass, its output matches the committed
hashes, its Python path equals the reference CLI, it is deterministic across
thread counts, and lossless coding reconstructs the source exactly. CPU."""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
import synthetic

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "oracle", "_ref")
GOLDEN = json.load(open(os.path.join(HERE, "golden", "oracle_hashes.json")))

pytestmark = pytest.mark.skipif(not oracle.available(), reason="oracle not built")


def test_reference_unit_tests():
    out = subprocess.run([os.path.join(REF, "test_txfm")], capture_output=True, text=True, check=True).stdout
    assert "transform consistency OK" in out
    out = subprocess.run([os.path.join(REF, "test_entropy")], capture_output=True, text=True, check=True).stdout
    assert "entropy round-trip OK" in out


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_oracle_matches_golden(name):
    import importlib.util
    spec_ = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec_)
    spec_.loader.exec_module(mg)
    assert mg.run(name) == GOLDEN[name]


def test_python_path_equals_cli_and_threads(tmp_path):
    spec = synthetic.ClipSpec(160, 96, 6, seed=51, rects=2)
    y4m = tmp_path / "in.y4m"
    synthetic.write_y4m(str(y4m), spec)
    flags = ["--cpu", "--turbo", "-q", "125", "--keyint", "30", "--tiles", "0"]
    outs = []
    for threads in ("1", "8"):
        ivf = tmp_path / f"out{threads}.ivf"
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        subprocess.run([os.path.join(REF, "mav1enc"), "-i", str(y4m), "-o", str(ivf)] + flags, env=env, check=True,
                       capture_output=True)
        outs.append(ivf.read_bytes())
    assert outs[0] == outs[1]
    packets, _ = oracle.encode(list(synthetic.generate(spec)),
                               oracle.cli_config(160, 96, q=125, turbo=1, keyint=30, tiles=0))
    assert oracle.ivf_bytes(packets, 160, 96) == outs[0]


def test_lossless_reconstructs_source():
    spec = synthetic.ClipSpec(64, 48, 2, seed=52, rects=1, rect_size=(8, 16))
    frames = list(synthetic.generate(spec))
    _, recons = oracle.encode(frames, oracle.cli_config(64, 48, q=0, fast=1))
    for f, r in zip(frames, recons):
        for a, b in zip(f, r):
            assert np.array_equal(a, b)
