"""The allocation-free search entry point, hm_search_noalloc.

Some callers cannot allocate device memory when they search: a host runtime
that owns all device memory and hands the library only its buffers, a serving
loop held to a fixed budget, or a caller that cannot afford the device-wide
synchronisation cudaFree implies.  hm_search_noalloc serves them from a fixed
array the library keeps in device memory.  This test calls it through the C ABI and
checks it against the allocating entry point, hm_search, on two calls in a
row (the second with other queries and another size, so whatever the first
call left in the shared array must not matter).  Results are integers:
equality is exact.  The file sorts last so that a run stopping at the first
failure has already run every other test; it also passes on its own in a
fresh process."""
import numpy as np
import pytest

from harmonia_b200 import BPlusTree, datagen as dg, native

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_noalloc_matches_hm_search_on_two_calls():
    lib = native.lib()
    keys = dg.gen_keys(1 << 20, seed=123)
    vals = dg.values_for(keys)
    with BPlusTree.bulk_load(torch.from_numpy(keys).cuda(), torch.from_numpy(vals).cuda()) as t:
        for call, m in enumerate((native.HM_NOALLOC_MAX_QUERIES, 300001)):
            q = torch.from_numpy(dg.gen_point_queries(keys, m, 0.7, seed=200 + call)).cuda()
            expected = t.search(q)  # hm_search, the allocating entry point
            out = torch.full_like(q, -99)
            rc = lib.hm_search_noalloc(t.handle, q.data_ptr(), m, out.data_ptr(), None)
            assert rc == 0, native.ERRORS.get(rc, rc)
            torch.cuda.synchronize()
            assert torch.equal(out, expected), f"call {call}"
            assert int((out >= 0).sum()) > m // 2


def test_noalloc_rejects_oversize_and_host_buffers():
    lib = native.lib()
    keys = dg.gen_keys(4096, seed=5)
    with BPlusTree.bulk_load(keys, dg.values_for(keys)) as t:
        big = native.HM_NOALLOC_MAX_QUERIES + 1
        q = torch.zeros(big, dtype=torch.int64, device="cuda")
        out = torch.empty_like(q)
        assert lib.hm_search_noalloc(t.handle, q.data_ptr(), big, out.data_ptr(), None) == -11
        hq = np.zeros(16, np.int64)
        ho = np.zeros(16, np.int64)
        assert lib.hm_search_noalloc(t.handle, hq.ctypes.data, 16, ho.ctypes.data, None) == -1
        assert lib.hm_search_noalloc(t.handle, q.data_ptr(), 0, out.data_ptr(), None) == 0
