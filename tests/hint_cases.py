"""Valid signatures re-encoded so that the reference's hint checks and the scheme's disagree.

The reference verifies the hint encoding with one warp per signature and combines the lanes'
failure ballots with XOR across passes (src/verify.cu:66 for the strictly-increasing positions,
:85 for the zero padding), so two violations in the same lane -- 32 positions apart -- cancel.
The scheme (and this library, and the oracle's ora_verify) rejects every violation.  Two
constructions keep the decoded hint vectors, hence the signature's validity, unchanged:

* padding: a signature with fewer than omega - 32 hints gets nonzero bytes at the first unused
  slot and 32 slots later;
* order: a polynomial with 33 hints gets its first position duplicated (one violation at relative
  index 1) and its last two positions swapped (a violation at relative index 33); the end counts
  from that polynomial on grow by one.  Only Dilithium2 (omega = 80) has room for this.

Items come from the reference's seed scheme (seed SHAKE128(le64(2i+1)), message SHAKE128(le64(2i)),
32 bytes) and were picked with the oracle; the builders assert the property they rely on.
"""
import numpy as np

# item of the seed scheme with fewer than omega - 32 hints in its signature, per parameter set
PADDING_ITEMS = {2: 9, 3: 159, 5: 112}
# Dilithium2 item whose first polynomial carries 33 hints (79 in total)
ORDER_ITEM = 1547


def seed_scheme_item(oracle, mode, i):
    seeds = oracle.seeds_from_ctr(1, rand_index=2 * i)
    pk, sk = oracle.keypair_seeds(mode, seeds)
    m = np.frombuffer(oracle.shake128((2 * i).to_bytes(8, "little"), 32), np.uint8).copy()
    sig = oracle.sign_batch(mode, m.reshape(1, -1), sk)[0]
    return pk[0], m, sig


def _hint_section(oracle, mode):
    p = oracle.params(mode)
    return p, 32 + p.l * p.polyz_packed


def padding_case(oracle, mode):
    """(pk, m, sig, noncanonical sig) with two nonzero padding bytes 32 slots apart."""
    pk, m, sig = seed_scheme_item(oracle, mode, PADDING_ITEMS[mode])
    p, h0 = _hint_section(oracle, mode)
    total = int(sig[h0 + p.omega + p.k - 1])
    assert total + 32 < p.omega, "item no longer has room for the padding construction"
    bad = sig.copy()
    bad[h0 + total] = 17
    bad[h0 + total + 32] = 200
    return pk, m, sig, bad


def order_case(oracle):
    """Dilithium2 (pk, m, sig, noncanonical sig) with two order violations 32 positions apart."""
    mode = 2
    pk, m, sig = seed_scheme_item(oracle, mode, ORDER_ITEM)
    p, h0 = _hint_section(oracle, mode)
    ends = [int(e) for e in sig[h0 + p.omega: h0 + p.omega + p.k]]
    pos = [int(x) for x in sig[h0: h0 + ends[-1]]]
    assert ends[0] == 33 and ends[-1] < p.omega, "item no longer fits the order construction"
    first = pos[: ends[0]]
    first = [first[0], first[0]] + first[1:]        # duplicate: violation at relative index 1
    first[32], first[33] = first[33], first[32]     # swap: violation at relative index 33
    newpos = first + pos[ends[0]:]
    bad = sig.copy()
    bad[h0: h0 + p.omega] = 0
    bad[h0: h0 + len(newpos)] = newpos
    bad[h0 + p.omega: h0 + p.omega + p.k] = [e + 1 for e in ends]
    return pk, m, sig, bad


def all_cases(oracle):
    """[(label, mode, pk, m, sig, bad)] for every construction."""
    out = [(f"padding-d{mode}", mode, *padding_case(oracle, mode)) for mode in (2, 3, 5)]
    out.append(("order-d2", 2, *order_case(oracle)))
    return out
