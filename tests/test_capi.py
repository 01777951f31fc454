"""The C-ABI library without a GPU: loads, exports every declared symbol, sizes agree."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = "\n".join(p.read_text() for p in (ROOT / "include").glob("*.h"))
    return sorted(set(re.findall(r"\b(cudil_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from cudilithium_b200._lib import LIB_PATH, SIGNATURES
    lib = ctypes.CDLL(str(LIB_PATH))
    syms = declared_symbols()
    assert syms, "no declarations found"
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/ but not exported"
        assert s in SIGNATURES, f"{s} has no ctypes signature"


def ref_rows(mode, mlen):
    """The reference's per-row pool formulas (tests/test_vectors.cu:62-166)."""
    import oracle.pyoracle as o
    p = o.params(mode)
    A = lambda x: (x + 255) // 256 * 256
    N = 256
    k, l = p.k, p.l
    w1 = k * p.polyw1_packed
    kp = A(p.pk_bytes) + A(p.sk_bytes) + k * N * 4
    sg = (A(p.sig_bytes) + A(p.sk_bytes) + A(32) + A(32 + mlen) + A(32 + 64 + w1) + A(64)
          + (k * l + 3 * l + 4 * k + 1) * N * 4)
    tp = A(p.sig_bytes) + A(64 + w1) + (2 * l + 3 * k) * N * 4
    vf = (A(p.sig_bytes) + A(p.pk_bytes) + A(32 + mlen) + A(64 + w1) + A(32)
          + (k * l + l + 3 * k + 1) * N * 4 + 4)
    return kp, sg, tp, vf


@pytest.mark.parametrize("mode", [2, 3, 5])
@pytest.mark.parametrize("mlen", [0, 32, 1000, 65536])
def test_row_sizes_equal_reference_formulas(mode, mlen):
    from cudilithium_b200._lib import lib
    kp, sg, tp, vf = ref_rows(mode, mlen)
    assert lib.cudil_keypair_row_bytes(mode) == kp
    assert lib.cudil_sign_row_bytes(mode, mlen) == sg
    assert lib.cudil_sign_temp_row_bytes(mode) == tp
    assert lib.cudil_verify_row_bytes(mode, mlen) == vf


@pytest.mark.parametrize("mode", [2, 3, 5])
def test_params_match_oracle(mode):
    import oracle.pyoracle as o
    from cudilithium_b200._lib import params
    a, b = params(mode), o.params(mode)
    for f in ("k", "l", "eta", "tau", "beta", "gamma1", "gamma2", "omega", "pk_bytes", "sk_bytes", "sig_bytes"):
        assert getattr(a, f) == getattr(b, f), f


def test_invalid_mode_and_args_rejected_without_gpu():
    from cudilithium_b200._lib import CUDIL_ERR_INVALID, lib, cudil_params
    assert lib.cudil_get_params(4, ctypes.byref(cudil_params())) == CUDIL_ERR_INVALID
    assert lib.cudil_keypair_row_bytes(7) == 0
    # null pools are rejected before any CUDA call
    assert lib.cudil_keypair(2, None, None, None, 0, 1, None, 0) == CUDIL_ERR_INVALID
    assert lib.cudil_ntt_mul(None, None, None, 4, None) == CUDIL_ERR_INVALID
