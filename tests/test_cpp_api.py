"""The C++ API (include/turbosort.hpp) on the crate's README examples and
larger slices: compiled with g++ against libturbosort_b200.so and run."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "turbosort_b200")


def _build(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "api_example")
    cmd = [cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp",
           "api_example.cpp"), "-L", LIBDIR, "-lturbosort_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_api_compiles(tmp_path):
    import turbosort_b200  # noqa: F401  (the library must exist)

    assert os.path.exists(turbosort_b200.LIB_PATH)
    _build(tmp_path)


@pytest.mark.gpu
def test_cpp_api_examples(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"


def test_copy_pool_copies_every_byte(tmp_path):
    """The transfer pipeline's host copy threads (ts_staging.h), on the CPU."""
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "copy_pool_test")
    subprocess.run([cxx, "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "turbosort_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "copy_pool_test.cpp"), "-o", exe],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"


def test_copy_pool_has_no_data_race(tmp_path):
    """The same program under ThreadSanitizer: the pool's hand-off between the
    caller and its workers (one mutex, two condition variables) is race-free."""
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no g++")
    exe = str(tmp_path / "copy_pool_tsan")
    r = subprocess.run([cxx, "-std=c++17", "-O1", "-g", "-fsanitize=thread", "-pthread", "-I",
                        os.path.join(ROOT, "turbosort_b200", "csrc"),
                        os.path.join(ROOT, "tests", "cpp", "copy_pool_test.cpp"), "-o", exe],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("no ThreadSanitizer runtime: " + r.stderr[-200:])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert "ThreadSanitizer" not in r.stderr, r.stderr[-2000:]
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr[-2000:]
