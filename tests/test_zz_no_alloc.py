"""The spike compaction that allocates nothing, against the one that allocates.

Callers that cannot allocate device memory where they need a compaction -- a
serving or data-assimilation loop whose device-memory budget is fixed at start-up,
or a runtime that owns all device memory through its own pool -- call
``dtb_compact_spikes_noalloc``, whose scratch is a fixed array inside the library.
This file checks, through the C-ABI, that two calls in a row give exactly the same
index lists and counts as ``dtb_compact_spikes`` on the same inputs (integer
results, so the tolerance is zero), and that inputs beyond the array's limit are
rejected.  It is named to run last.
"""
import ctypes as C

import numpy as np
import pytest

from dtb_b200 import engine as E

pytestmark = pytest.mark.gpu

MAX_NEURONS = 1 << 26


def _bitmap(n, seed, density):
    rng = np.random.default_rng(seed)
    flags = rng.random(n) < density
    words = np.packbits(flags, bitorder="little")
    pad = (-words.size) % 4
    return flags, np.concatenate([words, np.zeros(pad, np.uint8)]).view(np.uint32)


def _run(fn, bits_dev, n, torch, stream):
    idx = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    st = fn(C.c_void_p(bits_dev.data_ptr()), n, C.c_void_p(idx.data_ptr()), C.c_void_p(cnt.data_ptr()),
            C.c_void_p(stream))
    assert st == E.OK, E.LIB.dtb_last_error().decode()
    torch.cuda.synchronize()
    c = int(cnt.item())
    return c, idx[:c].cpu().numpy()


def test_noalloc_matches_allocating_compaction(gpu):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(5_000_000, 0.02, 1), (4097, 0.5, 2), (MAX_NEURONS, 0.001, 3), (33, 0.9, 4)]
    for n, density, seed in cases:
        # two different inputs, each through both entry points; the no-alloc calls come back to back
        inputs = [_bitmap(n, seed, density), _bitmap(n, seed + 100, density * 0.5)]
        devs = [torch.from_numpy(w.view(np.int32)).cuda() for _, w in inputs]
        ref = [_run(E.LIB.dtb_compact_spikes, d, n, torch, stream) for d in devs]
        got = [_run(E.LIB.dtb_compact_spikes_noalloc, d, n, torch, stream) for d in devs]
        for (flags, _), (rc, ri), (gc, gi) in zip(inputs, ref, got):
            assert gc == rc == int(flags.sum())
            assert np.array_equal(gi, ri)
            assert np.array_equal(gi.astype(np.int64), np.nonzero(flags)[0])


def test_noalloc_rejects_inputs_beyond_its_limit(gpu):
    import torch
    n = MAX_NEURONS + 1
    # buffers sized for n, so that even a broken limit check could not write out of bounds
    bits = torch.zeros((n + 31) // 32, dtype=torch.int32, device="cuda")
    idx = torch.zeros(n, dtype=torch.int32, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    st = E.LIB.dtb_compact_spikes_noalloc(C.c_void_p(bits.data_ptr()), n, C.c_void_p(idx.data_ptr()),
                                          C.c_void_p(cnt.data_ptr()), None)
    assert st == E.INVALID_PARAMETER
    assert "limit" in E.LIB.dtb_last_error().decode()
    torch.cuda.synchronize()
    assert int(cnt.item()) == -1          # rejected before anything ran
