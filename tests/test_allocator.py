"""A caller-supplied device allocator (clb_controls_set_allocator): every
buffer of a product goes through it and comes back, and buffers it refuses
make the library take its other way (bitmap rows without step records are
expanded a row per CTA; without room for B's word runs the bitmap rows insert
B's entries), with the same C."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from util import assert_dcsr_equal, from_device, to_device

pytestmark = pytest.mark.gpu

ALLOC = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)
FREE = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_void_p)
STEP_RECORD_BYTES = (2 + 2 * 256) * 4  # one deferred row's step record


class TorchAllocator:
    """Device buffers from torch's caching allocator on the library's stream;
    sizes in `refuse` are refused (NULL)."""

    def __init__(self, device: int):
        self.device = device
        self.live = {}
        self.refuse = set()
        self.refused = []
        self.requests = 0
        self.alloc_cb = ALLOC(self._alloc)
        self.free_cb = FREE(self._free)

    def _alloc(self, ctx, nbytes, stream):
        import torch
        self.requests += 1
        if nbytes in self.refuse:
            self.refused.append(nbytes)
            return None
        s = torch.cuda.ExternalStream(stream, device=self.device) if stream else None
        p = torch.cuda.caching_allocator_alloc(nbytes, self.device, s)
        self.live[p] = nbytes
        return p

    def _free(self, ctx, ptr, stream):
        import torch
        if ptr in self.live:
            del self.live[ptr]
            torch.cuda.caching_allocator_delete(ptr)


def quarter_dense_pair(ncols=1 << 18, seed=5):
    rng = np.random.default_rng(seed)
    nb = 4000
    rb = np.repeat(np.arange(nb, dtype=np.uint32), 60)
    cbb = rng.integers(0, ncols, rb.size).astype(np.uint32)
    b = O.coo_to_dcsr(O.Coo(nb, ncols, *O.unique_pairs(*O.sort_pairs(rb, cbb))))
    lens = np.array([20, 50, 90, 160, 200, 3] * 4)
    ra = np.repeat(np.arange(lens.size, dtype=np.uint32), lens)
    ca = rng.integers(0, nb, ra.size).astype(np.uint32)
    a = O.coo_to_dcsr(O.Coo(lens.size, nb, *O.unique_pairs(*O.sort_pairs(ra, ca))))
    return a, b


@pytest.mark.parametrize("refuse_records", [False, True])
def test_caller_allocator_serves_and_gets_back_every_buffer(refuse_records):
    import clbool_b200 as cb
    from clbool_b200 import sizing
    a, b = quarter_dense_pair()
    want = O.spgemm(a, b)
    nbmp = int((O.workload(a, b) > 4096).sum())  # rows in the bitmap bins
    assert nbmp >= 8
    ctl = cb.create_controls(0, 0)
    al = TorchAllocator(ctl.device)
    try:
        assert cb.lib.clb_controls_set_allocator(ctl.handle, al.alloc_cb, al.free_cb, None) == 0
        if refuse_records:
            al.refuse.add(nbmp * STEP_RECORD_BYTES)
        A, B = to_device(ctl, a), to_device(ctl, b)
        s = sizing.RowSizer.load(ctl)
        got = sizing.matrix_multiplication_learned(ctl, None, A, B, s)
        ctl.sync()
        assert_dcsr_equal(from_device(ctl, got), want, f"learned, records refused={refuse_records}")
        assert al.requests > 10
        if refuse_records:
            assert al.refused == [nbmp * STEP_RECORD_BYTES]  # the expansion fell back to a CTA per row
        del got, A, B, s
        import gc
        gc.collect()
        ctl.sync()
        assert al.live == {}, f"{len(al.live)} buffers not given back"
    finally:
        ctl.close()


def test_refused_word_runs_fall_back_to_entries():
    """Without B's word-run buffers the bitmap rows insert B's entries."""
    import clbool_b200 as cb
    rng = np.random.default_rng(11)
    n = 1 << 17
    nb = 5000  # B of at least 2^16 entries, each read more than 4 times: the word runs are tried
    rb = np.repeat(np.arange(nb, dtype=np.uint32), 100)
    cbb = rng.integers(0, n, rb.size).astype(np.uint32)
    b = O.coo_to_dcsr(O.Coo(nb, n, *O.unique_pairs(*O.sort_pairs(rb, cbb))))
    lens = np.array([2500, 3000, 40, 4000] * 3)
    ra = np.repeat(np.arange(lens.size, dtype=np.uint32), lens)
    ca = rng.integers(0, nb, ra.size).astype(np.uint32)
    a = O.coo_to_dcsr(O.Coo(lens.size, nb, *O.unique_pairs(*O.sort_pairs(ra, ca))))
    want = O.spgemm(a, b)
    nnz_b = len(b.cols)
    ctl = cb.create_controls(0, 0)
    al = TorchAllocator(ctl.device)
    try:
        assert cb.lib.clb_controls_set_allocator(ctl.handle, al.alloc_cb, al.free_cb, None) == 0
        al.refuse.add(nnz_b * 8)  # the (word, bits) pairs
        A, B = to_device(ctl, a), to_device(ctl, b)
        got = cb.dcsr.matrix_multiplication_hash(ctl, None, A, B)
        assert_dcsr_equal(from_device(ctl, got), want, "two-pass, word runs refused")
        assert al.refused and al.refused[0] == nnz_b * 8
        del got, A, B
    finally:
        ctl.close()


def test_refused_kept_bitmaps_fall_back_to_two_passes():
    """The two-pass form keeping its bitmaps (tuning form 2) without room for
    them inserts the bitmap rows' products again in its numeric pass."""
    import clbool_b200 as cb
    from clbool_b200 import gen
    r, c = gen.rmat(14, seed=4)
    n = 1 << 14
    a = O.coo_to_dcsr(O.Coo(n, n, r, c))
    want = O.spgemm(a, a)
    nbmp = int((O.workload(a, a) > 4096).sum())
    words = n // 32  # bitmap words of a 2^14-column row
    assert nbmp >= 8
    ctl = cb.create_controls(0, 0)
    al = TorchAllocator(ctl.device)
    try:
        assert cb.lib.clb_controls_set_allocator(ctl.handle, al.alloc_cb, al.free_cb, None) == 0
        al.refuse.add(nbmp * words * 4)
        A = to_device(ctl, a)
        got = cb.dcsr.matrix_multiplication_tuned(ctl, None, A, A, cb.dcsr.tuning("two_pass_kept"))
        assert_dcsr_equal(from_device(ctl, got), want, "kept form, bitmaps refused")
        assert al.refused == [nbmp * words * 4]
        del got, A
    finally:
        ctl.close()
