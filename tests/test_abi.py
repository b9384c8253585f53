"""ABI conformance without a GPU (the reference's tests/conformance_c.c:34-120
checks, plus the exported-symbol set).

Validation rejects make no CUDA call, so they run on a host with no device.
"""
import ctypes
import os
import re
import subprocess

import pytest

import cudec_b200 as cd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cudec.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cudec_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol():
    names = declared_functions()
    assert "cudec_lz4_decompress_batch" in names
    out = subprocess.run(["nm", "-D", "--defined-only", cd.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (cudec_[a-z0-9_]+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # and the Python mirror binds each of them
    assert set(names) <= set(cd.SIGNATURES), set(names) - set(cd.SIGNATURES)
    lib = cd.lib()
    for n in names:
        assert getattr(lib, n) is not None


def test_version_matches_header():
    text = open(HEADER).read()
    maj = int(re.search(r"CUDEC_VERSION_MAJOR (\d+)", text).group(1))
    mnr = int(re.search(r"CUDEC_VERSION_MINOR (\d+)", text).group(1))
    pat = int(re.search(r"CUDEC_VERSION_PATCH (\d+)", text).group(1))
    assert cd.version() == maj * 10000 + mnr * 100 + pat


def test_result_record_layout():
    assert ctypes.sizeof(cd.ChunkResult) == 16
    assert cd.ChunkResult.bytes_written.offset == 8


def _fake(n=8):
    # Non-NULL host addresses: validation must reject before touching them.
    buf = (ctypes.c_uint8 * (64 * n + 64))()
    base = ctypes.addressof(buf)
    aligned = (base + 15) & ~15
    return buf, aligned


def test_batch_validation_rejects_synchronously():
    buf, a = _fake()
    for entry in cd.BATCH_ENTRIES.values():
        ok_args = [a, a, a, a, 4, a]
        for i in range(4):
            args = list(ok_args)
            args[i] = None
            assert entry(*args, None) == cd.ERR_INVALID_ARGUMENT
        assert entry(a, a, a, a, 4, None, None) == cd.ERR_INVALID_ARGUMENT
        assert entry(a, a, a, a, 4, a + 8, None) == cd.ERR_INVALID_ARGUMENT
        assert entry(a, a, a, a, 0, a, None) == cd.ERR_INVALID_ARGUMENT
        assert entry(a, a, a, a, 2**64 - 1, a, None) == cd.ERR_INVALID_ARGUMENT
        assert entry(a, a, a, a, (2**31 - 1) * 32 + 1, a, None) == cd.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("std", ["c99", "c11"])
def test_c_conformance_program(tmp_path, std):
    """tests/conformance_c.c, built as strict C99 and C11 against the header and
    linked against the library: every entry point resolves with C linkage and
    its documented synchronous rejects hold for a C caller (the reference pins
    the same in tests/conformance_c.c)."""
    exe = tmp_path / ("conformance_" + std)
    libdir = os.path.dirname(cd.LIB_PATH)
    subprocess.run(["gcc", "-std=" + std, "-pedantic", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "conformance_c.c"),
                    "-o", str(exe), "-L" + libdir, "-lcudec_b200", "-Wl,-rpath," + libdir],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "PASS: every public entry point called from C"


def test_zstd_workspace_rejects_synchronously():
    buf, a = _fake()
    ws = cd.zstd_workspace_bytes(4)
    assert ws == 4 * 128 * 1024
    assert cd.zstd_workspace_bytes(1) == ws  # rounded up to a CTA's warps
    assert cd.zstd_workspace_bytes(1 << 20) == cd.zstd_workspace_bytes(4096)
    z = cd.zstd_decompress_batch
    assert z(a, a, a, a, 4, a, None, ws, None) == cd.ERR_INVALID_ARGUMENT
    assert z(a, a, a, a, 4, a, a, ws - 1, None) == cd.ERR_INVALID_ARGUMENT
    assert z(None, a, a, a, 4, a, a, ws, None) == cd.ERR_INVALID_ARGUMENT
    assert z(a, a, a, a, 0, a, a, ws, None) == cd.ERR_INVALID_ARGUMENT
    assert z(a, a, a, a, 4, a + 8, a, ws, None) == cd.ERR_INVALID_ARGUMENT


def test_mixed_plan_rejects_without_cuda():
    buf, a = _fake()
    assert cd.lib().cudec_mixed_plan_create(None) == cd.ERR_INVALID_ARGUMENT
    assert cd.lib().cudec_mixed_plan_destroy(None) == cd.ERR_INVALID_ARGUMENT
    m = cd.lib().cudec_mixed_decompress
    assert m(None, a, a, a, a, a, 4, a, None) == cd.ERR_INVALID_ARGUMENT
    assert cd.lib().cudec_mixed_plan_tune(None, a, a, a, a, a, 4, a, None) == cd.ERR_INVALID_ARGUMENT
    assert cd.lib().cudec_mixed_plan_get_tuning(None, a) == cd.ERR_INVALID_ARGUMENT
    assert cd.lib().cudec_mixed_plan_get_shape(None, a) == cd.ERR_INVALID_ARGUMENT
    assert cd.lib().cudec_mixed_plan_set_shape(None, a) == cd.ERR_INVALID_ARGUMENT


def test_server_rejects_without_cuda():
    buf, a = _fake()
    h = ctypes.c_void_p()
    c = cd.lib().cudec_server_create
    assert c(0, 4, cd.SERVER_MIXED, 4096, ctypes.byref(h)) == cd.ERR_INVALID_ARGUMENT
    assert c(1 << 20, 0, cd.SERVER_MIXED, 4096, ctypes.byref(h)) == cd.ERR_INVALID_ARGUMENT
    assert c(1 << 20, 2, cd.SERVER_PLAIN, 4096, ctypes.byref(h)) == cd.ERR_INVALID_ARGUMENT
    assert c(1 << 20, 4, 7, 4096, ctypes.byref(h)) == cd.ERR_INVALID_ARGUMENT
    assert c(1 << 20, 4, cd.SERVER_MIXED, 0, ctypes.byref(h)) == cd.ERR_INVALID_ARGUMENT
    assert c(1 << 20, 4, cd.SERVER_MIXED, 4096, None) == cd.ERR_INVALID_ARGUMENT
    t = ctypes.c_uint64()
    assert cd.lib().cudec_server_submit(None, a, 8, a, a, a, a, 1, ctypes.byref(t)) == \
        cd.ERR_INVALID_ARGUMENT
    assert cd.lib().cudec_server_wait(None, 1, None, None, None) == cd.ERR_INVALID_ARGUMENT
    done = ctypes.c_int(7)
    assert cd.lib().cudec_server_wait_for(None, 1, 5.0, ctypes.byref(done), None, None,
                                          None) == cd.ERR_INVALID_ARGUMENT
    assert cd.lib().cudec_server_release(None, 1) == cd.ERR_INVALID_ARGUMENT
    assert cd.lib().cudec_server_destroy(None) == cd.ERR_INVALID_ARGUMENT
