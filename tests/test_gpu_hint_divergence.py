"""Where verification deliberately differs from the reference: non-canonical hint encodings.

The reference combines its hint-check ballots with XOR (src/verify.cu:66, :85), so it accepts a
valid signature re-encoded with two violations 32 positions apart (see hint_cases.py).  This
library applies the checks as the scheme states them: the plain verify, the fused verifier, the
allocation-free verify and the standalone parse step must all reject those re-encodings, while
the oracle's restatement of the reference's own form accepts them (needs a B200)."""
import numpy as np
import pytest

from hint_cases import all_cases

pytestmark = pytest.mark.gpu


def _noalloc_verify(mode, sig, m, pk):
    import torch

    from cudilithium_b200._lib import lib
    from cudilithium_b200.api import pinned
    n, mlen = m.shape
    hs, hm, hp = pinned(sig.size), pinned(m.size), pinned(pk.size)
    hs.numpy()[: sig.size] = sig.reshape(-1)
    hm.numpy()[: m.size] = m.reshape(-1)
    hp.numpy()[: pk.size] = pk.reshape(-1)
    ret = torch.full((n,), 7, dtype=torch.int32, pin_memory=True)
    assert lib.cudil_verify_noalloc(mode, ret.data_ptr(), hs.data_ptr(), sig.shape[1], sig.shape[1], hm.data_ptr(),
                                    mlen, mlen, hp.data_ptr(), n, None) == 0
    torch.cuda.synchronize()
    return ret.numpy().copy()


@pytest.mark.parametrize("label", ["padding-d2", "padding-d3", "padding-d5", "order-d2"])
def test_noncanonical_hints_rejected_everywhere(cuda_ok, oracle, label):
    import torch

    import cudilithium_b200 as cd
    from cudilithium_b200.engine import Engine
    case = {c[0]: c for c in all_cases(oracle)}[label]
    _, mode, pk, m, sig, bad = case
    # the reference's own evaluation accepts the re-encoding; the scheme's does not
    assert oracle.verify_xor_ballots(mode, bad, m.tobytes(), pk) == 0
    assert oracle.verify_batch(mode, bad[None], m[None], pk[None])[0] == -1

    sigs = np.stack([sig, bad])
    ms = np.stack([m, m])
    pks = np.stack([pk, pk])
    want = np.array([0, -1], np.int32)
    d = cd.Dilithium(mode)
    assert np.array_equal(d.verify(sigs, ms, pks), want)                 # plain stage-by-stage path
    assert np.array_equal(_noalloc_verify(mode, sigs, ms, pks), want)     # allocation-free entry point
    eng = Engine(mode, max_keys=1, max_items=2)
    eng.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    assert np.array_equal(eng.verify_np(sigs, [m.tobytes()] * 2, np.zeros(2, np.uint32)), want)  # fused
    st = d.sig_check(sigs)                                                # standalone parse step
    assert st[0] == 0 and (st[1] & 1) == 1
    assert np.array_equal(st, oracle.sig_check(mode, sigs))
