"""World pool slot allocation (src/main.cu:364-390): nsb_pool_claim replays
claim_slot one claim after another. Compared with a Python restatement of the
reference's rules and, where oracle/_ref is present, with the reference's own
claim_slot run on one device thread (oracle/ref_world_harness.cu)."""
import ctypes as ct

import numpy as np
import pytest

from oracle.pyoracle import ref_world_lib

pytestmark = pytest.mark.gpu


def claim_python(used, capacity, hints):
    used = used.copy()
    words = (capacity + 31) // 32
    out = []
    for h in hints:
        slot = -1
        start = h % words
        for off in range(words):
            w = (start + off) % words
            occ = int(used[w])
            if occ != 0xFFFFFFFF:
                free = ~occ & 0xFFFFFFFF
                bit = (free & -free).bit_length() - 1
                s = w * 32 + bit
                if s < capacity:
                    used[w] = np.uint32(occ | (1 << bit))
                    slot = s
                break
        out.append(slot)
    return np.array(out, np.int32), used


@pytest.mark.parametrize("capacity", [10000, 4096])
def test_pool_claims_match_reference(nsb, capacity):
    import torch
    rng = np.random.default_rng(capacity)
    words = (capacity + 31) // 32
    bits = rng.random(words * 32) < 0.8
    used = np.packbits(bits.reshape(-1, 32)[:, ::-1], axis=1).view(">u4").ravel().astype(np.uint32)
    hints = rng.integers(0, 5 * words, 3000).astype(np.int32)
    want, want_used = claim_python(used, capacity, hints)
    assert (want >= 0).sum() > 500 and (want < 0).sum() > 0       # claims succeed, then the pool fills
    lib = nsb.native.library()
    d = torch.from_numpy(used.view(np.int32).copy()).cuda()
    got = np.zeros(len(hints), np.int32)
    assert lib.nsb_pool_claim(ct.c_void_p(d.data_ptr()), capacity, hints.ctypes.data_as(ct.POINTER(ct.c_int32)),
                              len(hints), got.ctypes.data_as(ct.POINTER(ct.c_int32))) == 0
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(d.cpu().numpy().view(np.uint32), want_used)
    ref = ref_world_lib()
    if ref is not None:
        r = torch.from_numpy(used.view(np.int32).copy()).cuda()
        h = torch.from_numpy(hints).cuda()
        s = torch.zeros(len(hints), dtype=torch.int32, device="cuda")
        assert ref.ref_world_claim_sequential(r.data_ptr(), capacity, h.data_ptr(), len(hints), s.data_ptr()) == 0
        np.testing.assert_array_equal(s.cpu().numpy(), want)
        np.testing.assert_array_equal(r.cpu().numpy().view(np.uint32), want_used)
    # release returns the bits
    claimed = got[got >= 0]
    assert lib.nsb_pool_release(ct.c_void_p(d.data_ptr()), claimed.ctypes.data_as(ct.POINTER(ct.c_int32)),
                                len(claimed)) == 0
    np.testing.assert_array_equal(d.cpu().numpy().view(np.uint32), used)
