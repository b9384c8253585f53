"""The install surface (the reference's packaging, CMakeLists.txt:395-471 and
cmake/cudec-config.cmake.in): `python -m cudec_b200.build install --prefix P`
gives a prefix that a CMake consumer finds with find_package(cudec) and links
through the imported target cudec::cudec, and that pkg-config describes. The
consumer here is the C conformance program (tests/conformance_c.c, C99),
built against the installed header and library only and run (its checks need
no GPU). Version requests follow the 0.x rule (met by the same major.minor
at an installed patch level at or above the one requested), and the prefix
still works after it is moved."""
import os
import shutil
import subprocess

import pytest

from cudec_b200 import build as B

HERE = os.path.dirname(os.path.abspath(__file__))
CMAKE = shutil.which("cmake")
PKGCONFIG = shutil.which("pkg-config")

CONSUMER = """\
cmake_minimum_required(VERSION 3.24)
project(cudec_consumer C)
find_package(cudec {want} REQUIRED)
add_executable(conformance "{src}")
set_property(TARGET conformance PROPERTY C_STANDARD 99)
set_property(TARGET conformance PROPERTY C_STANDARD_REQUIRED ON)
target_link_libraries(conformance PRIVATE cudec::cudec)
"""


def configure(tmp, prefix, want, tag):
    src = os.path.join(tmp, "consumer_" + tag)
    os.makedirs(src, exist_ok=True)
    with open(os.path.join(src, "CMakeLists.txt"), "w") as f:
        f.write(CONSUMER.format(want=want, src=os.path.join(HERE, "conformance_c.c")))
    bld = os.path.join(tmp, "build_" + tag)
    r = subprocess.run([CMAKE, "-S", src, "-B", bld, "-DCMAKE_PREFIX_PATH=" + prefix],
                       capture_output=True, text=True)
    return r, bld


@pytest.fixture(scope="module")
def prefix(tmp_path_factory):
    p = str(tmp_path_factory.mktemp("prefix"))
    B.install(p)
    return p


def test_installed_files(prefix):
    ver = "%d.%d.%d" % B.version()
    for rel in ("lib/libcudec_b200.so", "include/cudec.h", "lib/cmake/cudec/cudec-config.cmake",
                "lib/cmake/cudec/cudec-config-version.cmake", "lib/pkgconfig/cudec.pc"):
        assert os.path.isfile(os.path.join(prefix, rel)), rel
    assert "Version: " + ver in open(os.path.join(prefix, "lib/pkgconfig/cudec.pc")).read()
    if shutil.which("readelf"):
        soname = subprocess.run(["readelf", "-d", os.path.join(prefix, "lib/libcudec_b200.so")],
                                capture_output=True, text=True).stdout
        assert "[libcudec_b200.so]" in soname


@pytest.mark.skipif(CMAKE is None, reason="cmake not installed")
def test_find_package_builds_and_runs_the_conformance_program(prefix, tmp_path):
    major, minor, patch = B.version()
    r, bld = configure(str(tmp_path), prefix, "%d.%d" % (major, minor), "ok")
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([CMAKE, "--build", bld], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([os.path.join(bld, "conformance")], capture_output=True, text=True)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.skipif(CMAKE is None, reason="cmake not installed")
def test_version_requests(prefix, tmp_path):
    major, minor, patch = B.version()
    ok = ["%d.%d" % (major, minor), "%d.%d.%d" % (major, minor, patch),
          "%d.%d...%d.%d" % (major, minor, major + 1, 0)]
    bad = ["%d.%d" % (major, minor + 1), "%d.%d.%d" % (major, minor, patch + 1),
           "%d.0" % (major + 1)]
    if minor > 0:
        bad.append("%d.%d" % (major, minor - 1))
    for k, want in enumerate(ok):
        assert configure(str(tmp_path), prefix, want, "v%d" % k)[0].returncode == 0, want
    for k, want in enumerate(bad):
        assert configure(str(tmp_path), prefix, want, "b%d" % k)[0].returncode != 0, want


@pytest.mark.skipif(CMAKE is None, reason="cmake not installed")
def test_moved_prefix(prefix, tmp_path):
    moved = str(tmp_path / "moved")
    shutil.copytree(prefix, moved)
    r, bld = configure(str(tmp_path), moved, "", "moved")
    assert r.returncode == 0, r.stdout + r.stderr
    cache = open(os.path.join(bld, "CMakeCache.txt")).read()
    assert os.path.join(moved, "lib", "cmake", "cudec") in cache


@pytest.mark.skipif(PKGCONFIG is None, reason="pkg-config not installed")
def test_pkg_config(prefix, tmp_path):
    env = dict(os.environ, PKG_CONFIG_PATH=os.path.join(prefix, "lib", "pkgconfig"))
    flags = subprocess.run([PKGCONFIG, "--cflags", "--libs", "cudec"], env=env,
                           capture_output=True, text=True, check=True).stdout.split()
    exe = str(tmp_path / "conformance_pc")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", os.path.join(HERE, "conformance_c.c"),
                    "-o", exe] + flags, check=True)
    r = subprocess.run([exe], capture_output=True, text=True,
                       env=dict(os.environ, LD_LIBRARY_PATH=os.path.join(prefix, "lib")))
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr
