"""The device kernel bodies that also compile for the host (compression, source/loss solves,
production/loss rates, dt selection) run over every index of their launch ranges under
AddressSanitizer: an index that leaves its array fails here, on the CPU, before the same code
reaches a GPU.  The host tests themselves run in a child process with the sanitizer runtime
preloaded and the harnesses built with -fsanitize=address."""
import os
import shutil
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
MODULES = ["test_compression_host.py", "test_sources_host.py", "test_rates_host.py", "test_clock_host.py"]


def _asan_runtime():
    cxx = shutil.which("g++")
    if not cxx:
        return None
    p = subprocess.run([cxx, "-print-file-name=libasan.so"], capture_output=True, text=True).stdout.strip()
    return os.path.realpath(p) if p and os.path.isabs(p) and os.path.exists(p) else None


def test_kernel_bodies_stay_in_bounds():
    rt = _asan_runtime()
    if rt is None:
        pytest.skip("no AddressSanitizer runtime")
    env = dict(os.environ, LD_PRELOAD=rt, ASAN_OPTIONS="detect_leaks=0",
               GEMINI_HARNESS_CFLAGS="-fsanitize=address -fno-omit-frame-pointer")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", "-x"] +
                       [os.path.join(HERE, m) for m in MODULES], env=env, capture_output=True, text=True,
                       timeout=900)
    out = r.stdout + r.stderr
    assert r.returncode == 0 and "AddressSanitizer" not in out, out[-4000:]
