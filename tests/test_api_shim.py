"""The reference-compatible C++ header include/api.cuh: a caller written against the reference's
API (tests/shim/kat_shim.cpp) compiles for every parameter set and links with the library (CPU);
on a GPU it reproduces the reference's known-answer digests through that header."""
import hashlib
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "shim" / "kat_shim.cpp"
LIBDIR = ROOT / "cudilithium_b200"
CUDA = Path("/usr/local/cuda")


def build_shim(mode: int, out: Path, extra=()) -> Path:
    exe = out / f"kat_shim{mode}"
    cmd = ["g++", "-O1", "-std=c++17", f"-DDILITHIUM_MODE={mode}", *extra, f"-I{ROOT / 'include'}",
           f"-I{CUDA / 'include'}", str(SRC), "-o", str(exe), f"-L{LIBDIR}", "-lcudilithium_b200",
           f"-Wl,-rpath,{LIBDIR}", f"-L{CUDA / 'lib64'}", "-lcudart", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
@pytest.mark.parametrize("mode", [2, 3, 5])
def test_api_shim_compiles_and_links(tmp_path, mode):
    if not (LIBDIR / "libcudilithium_b200.so").exists():
        pytest.skip("library not built")
    exe = build_shim(mode, tmp_path)
    assert exe.exists()


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_api_shim_randomized_compiles_and_links(tmp_path):
    if not (LIBDIR / "libcudilithium_b200.so").exists():
        pytest.skip("library not built")
    assert build_shim(5, tmp_path, extra=["-DDILITHIUM_RANDOMIZED_SIGNING"]).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [2, 3, 5])
def test_api_shim_known_answer_digest(tmp_path, cuda_ok, oracle, golden_digests, mode):
    n, mlen = golden_digests["nvectors"], golden_digests["mlen"]
    exe = build_shim(mode, tmp_path)
    m = oracle.messages_from_ctr(n, mlen)
    (tmp_path / "m.bin").write_bytes(m.tobytes())
    r = subprocess.run([str(exe), str(tmp_path), str(n), str(mlen)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    p = oracle.params(mode)
    pk = np.fromfile(tmp_path / "pk.bin", np.uint8).reshape(n, p.pk_bytes)
    sk = np.fromfile(tmp_path / "sk.bin", np.uint8).reshape(n, p.sk_bytes)
    sig = np.fromfile(tmp_path / "sig.bin", np.uint8).reshape(n, p.sig_bytes)
    ret = np.fromfile(tmp_path / "ret.bin", np.int32)
    assert np.all(ret == 0)
    data = oracle.tvecs_from_outputs(m, pk, sk, sig, ret)
    assert hashlib.sha256(data).hexdigest() == golden_digests["sha256"][str(mode)]
