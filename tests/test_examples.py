"""The programs under examples/ build from the public header, the library and
the CUDA runtime alone, as strict C99 (on any host), and do what they print
on a GPU: decode_batch's five chunks report the documented statuses, and
decode_frame writes exactly the frame's content."""
import os
import subprocess

import numpy as np
import pytest

import cudec_b200 as cd
from cudec_b200 import workload as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_example(name, out_dir):
    exe = os.path.join(str(out_dir), name)
    libdir = os.path.dirname(cd.LIB_PATH)
    cudart = os.path.join(CUDA, "lib64")
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"), "-isystem", os.path.join(CUDA, "include"),
                    os.path.join(ROOT, "examples", name + ".c"), "-o", exe,
                    "-L" + libdir, "-lcudec_b200", "-Wl,-rpath," + libdir,
                    "-L" + cudart, "-lcudart", "-Wl,-rpath," + cudart], check=True)
    return exe


@pytest.mark.parametrize("name", ["decode_batch", "decode_frame"])
def test_examples_build_as_c99(tmp_path, name):
    assert os.path.exists(build_example(name, tmp_path))


def test_decode_frame_usage_and_missing_file(tmp_path):
    exe = build_example("decode_frame", tmp_path)
    assert subprocess.run([exe], capture_output=True).returncode == 1
    r = subprocess.run([exe, str(tmp_path / "absent.lz4"), str(tmp_path / "o")],
                       capture_output=True)
    assert r.returncode == 1


@pytest.mark.gpu
def test_decode_batch_runs(tmp_path):
    r = subprocess.run([build_example("decode_batch", tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    assert lines[-1] == "all chunks as expected"
    want = ["OK", "CORRUPT_INPUT", "OUTPUT_TOO_SMALL", "OK", "OUTPUT_TOO_SMALL"]
    got = [ln.split("->")[1].split()[0] for ln in lines if "->" in ln]
    assert got == want


@pytest.mark.gpu
def test_decode_frame_runs(tmp_path):
    exe = build_example("decode_frame", tmp_path)
    rng = np.random.default_rng(3)
    raw = bytes(rng.integers(0, 8, 300000, dtype=np.uint8))
    # the second frame states no size and compresses ~200:1, so the program
    # doubles its buffer several times before the output fits
    rep = b"0123456789abcdef" * 131072
    cases = {"sized": (raw, W.lz4f_compress(raw, content_size=True)),
             "unsized": (rep, W.lz4f_compress(rep, content_size=False, content_checksum=True))}
    for label, (raw, frame) in cases.items():
        src, dst = tmp_path / (label + ".lz4"), tmp_path / (label + ".out")
        src.write_bytes(frame)
        r = subprocess.run([exe, str(src), str(dst)], capture_output=True, text=True)
        assert r.returncode == 0, (label, r.stdout + r.stderr)
        assert dst.read_bytes() == raw, label
    bad = bytearray(cases["unsized"][1])
    bad[-1] ^= 1  # content checksum
    src = tmp_path / "bad.lz4"
    src.write_bytes(bytes(bad))
    r = subprocess.run([exe, str(src), str(tmp_path / "bad.out")], capture_output=True, text=True)
    assert r.returncode == 2 and "CORRUPT_INPUT" in r.stderr
