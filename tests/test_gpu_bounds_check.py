"""The bounds-checked build (-DCUDIL_BOUNDS_CHECK, libcudilithium_b200_bc.so) on the GPU.

compute-sanitizer is not available where these tests run, so this build is the memory-safety
check: device-side range checks on pool rows, attempt slots, item indices and key-cache rows that
record the first failure in an error word instead of trapping.  Small batches of all three
parameter sets run through every signing and verification path in that build, with outputs
bit-exact against the oracle, and the error word must stay 0 (needs a B200)."""
import ctypes
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
BC_LIB = ROOT / "cudilithium_b200" / "libcudilithium_b200_bc.so"


def test_bounds_checked_build_clean(cuda_ok):
    if not BC_LIB.exists():
        subprocess.run([sys.executable, str(ROOT / "cudilithium_b200" / "build.py"), "--bounds-check"], check=True)
    env = dict(os.environ, CUDIL_LIB=str(BC_LIB))
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "bounds_check_run.py")], env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert r.stdout.strip().splitlines()[-1] == "bounds error word: 0", r.stdout[-2000:]


def test_normal_build_reports_no_checks(cuda_ok):
    from cudilithium_b200._lib import CUDIL_ERR_INVALID, lib
    err = ctypes.c_uint32(7)
    assert lib.cudil_bounds_check_status(ctypes.byref(err), 0) == CUDIL_ERR_INVALID
    assert err.value == 0
