"""The allocation-free link list (tlbm_link_list_noalloc) against the regular one.

Some host programs cannot allocate device memory while they run: they hand a
fixed budget of the GPU to a solver framework or a caching allocator at start-up,
and a cudaMalloc in the time loop could fail or stall the device.  For them the
library offers one entry point whose scratch lives in a static device array.
This test calls it through the C ABI twice in a row (the second call reuses the
array the first one left behind) and checks both results against
tlbm_link_count + tlbm_link_list with caller-provided scratch, which must agree
exactly (integer indices).  It also checks the size limit and the truncation to
the caller's output capacity.  This file is collected last on purpose.
"""

from __future__ import annotations

import pytest
import torch

pytestmark = pytest.mark.gpu


def _regular(lib, stream, mask):
    """tlbm_link_count + tlbm_link_list with a caller-provided block-count buffer."""
    from tensorlbm_b200 import _lib

    count = mask.numel()
    nb = lib.tlbm_link_blocks(count)
    blocks = torch.empty(max(nb, 1), dtype=torch.int64, device=mask.device)
    total = torch.zeros(1, dtype=torch.int64, device=mask.device)
    _lib.check(lib.tlbm_link_count(mask.data_ptr(), count, blocks.data_ptr(), total.data_ptr(), stream), "count")
    out = torch.empty(int(total.item()), dtype=torch.int64, device=mask.device)
    if out.numel():
        _lib.check(lib.tlbm_link_list(mask.data_ptr(), count, blocks.data_ptr(), out.data_ptr(), stream), "list")
    return out


def _noalloc(lib, stream, mask, capacity):
    from tensorlbm_b200 import _lib

    out = torch.full((max(capacity, 1),), -1, dtype=torch.int64, device=mask.device)
    total = torch.full((1,), -1, dtype=torch.int64, device=mask.device)
    st = lib.tlbm_link_list_noalloc(mask.data_ptr(), mask.numel(), out.data_ptr(), capacity, total.data_ptr(),
                                    stream)
    _lib.check(st, "tlbm_link_list_noalloc")
    torch.cuda.synchronize(mask.device)
    return out[:capacity], int(total.item())


def test_noalloc_link_list_matches_regular_two_calls(cuda):
    from tensorlbm_b200 import _lib

    lib = _lib.load()
    stream = _lib.stream_of(cuda)
    g = torch.Generator(device=cuda).manual_seed(7)
    # first call: a dense mask; second call: a sparser, shorter mask, so stale
    # block counts from the first call would show up if they leaked
    m1 = (torch.rand((19, 40, 50, 60), device=cuda, generator=g) < 0.05).view(torch.uint8).reshape(-1)
    m2 = (torch.rand((27, 10, 33, 17), device=cuda, generator=g) < 0.01).view(torch.uint8).reshape(-1)
    for m in (m1, m2):
        ref = _regular(lib, stream, m)
        got, total = _noalloc(lib, stream, m, m.numel())
        assert total == ref.numel()
        assert torch.equal(got[:total], ref)
        assert bool((got[total:] == -1).all())  # nothing written past the count


def test_noalloc_capacity_and_limit(cuda):
    from tensorlbm_b200 import _lib

    lib = _lib.load()
    stream = _lib.stream_of(cuda)
    m = (torch.arange(5000, device=cuda) % 7 == 0).view(torch.uint8)
    ref = _regular(lib, stream, m)
    got, total = _noalloc(lib, stream, m, 100)
    assert total == ref.numel() and total > 100
    assert torch.equal(got, ref[:100])
    # count-only query: no output buffer at all (null pointer, capacity 0)
    n0 = torch.full((1,), -1, dtype=torch.int64, device=cuda)
    _lib.check(lib.tlbm_link_list_noalloc(m.data_ptr(), m.numel(), None, 0, n0.data_ptr(), stream), "count only")
    torch.cuda.synchronize(cuda)
    assert int(n0.item()) == ref.numel()
    cap = lib.tlbm_link_list_static_capacity()
    assert cap == 128 * 1024 * 1024
    out = torch.empty(1, dtype=torch.int64, device=cuda)
    n = torch.empty(1, dtype=torch.int64, device=cuda)
    # the size check comes before any access, so a one-byte buffer is enough here
    st = lib.tlbm_link_list_noalloc(m.data_ptr(), cap + 1, out.data_ptr(), 1, n.data_ptr(), stream)
    assert st == _lib.ERR_TOO_LARGE
    with pytest.raises(ValueError, match="static scratch"):
        _lib.check(st, "tlbm_link_list_noalloc")
