"""Driver for test_gpu_bounds_check.py, run in a fresh process whose CUDIL_LIB selects the
bounds-checked library: small batches of every parameter set through the plain path, the fused
engine (phased and asynchronous signers) and the parse step, each checked against the oracle,
then the library's bounds error word, which must be 0 (printed as the last line)."""
import ctypes
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402
import torch  # noqa: E402

import cudilithium_b200 as cd  # noqa: E402
from cudilithium_b200._lib import LIB_PATH, lib  # noqa: E402
from cudilithium_b200.engine import Engine  # noqa: E402
from oracle import pyoracle as ora  # noqa: E402


def main():
    assert LIB_PATH.name == "libcudilithium_b200_bc.so", LIB_PATH
    rng = np.random.default_rng(4242)
    for mode in (2, 3, 5):
        n = 40
        d = cd.Dilithium(mode)
        pk, sk = d.keypair(n, rand_index=900 + mode)
        opk, osk = ora.keypair_batch(mode, n, rand_index=900 + mode)
        assert np.array_equal(pk, opk) and np.array_equal(sk, osk), mode
        m = rng.integers(0, 256, (n, 60), dtype=np.uint8)
        want = ora.sign_batch(mode, m, sk)
        assert np.array_equal(d.sign(m, sk, exec_threshold=32), want), mode
        bad = want.copy()
        bad[::3, 50] ^= 1
        assert np.array_equal(d.verify(bad, m, pk), ora.verify_batch(mode, bad, m, pk)), mode
        assert np.array_equal(d.sig_check(bad), ora.sig_check(mode, bad)), mode
        for variant in (0, 2):
            eng = Engine(mode, max_keys=n, max_items=n)
            eng.set_sign_kernel(variant)
            eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
            eng.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
            keys = rng.permutation(n).astype(np.uint32)
            sig = eng.sign_np(m, keys)
            assert np.array_equal(sig, ora.sign_batch(mode, m, sk[keys])), (mode, variant)
            assert np.all(eng.verify_np(sig, m, keys) == 0), (mode, variant)
            eng.close()
    err = ctypes.c_uint32(0xFFFFFFFF)
    assert lib.cudil_bounds_check_status(ctypes.byref(err), 1) == 0
    print(f"bounds error word: {err.value}")


if __name__ == "__main__":
    main()
