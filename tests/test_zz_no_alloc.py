"""The allocation-free exact flat search (ann_flat_query_noalloc), called through the C ABI.

It serves callers that cannot let a library allocate device memory -- an application that owns
every device allocation through its own pool, or a serving thread that must not call cudaMalloc /
cudaFree because those can synchronise the device. Its output must equal the allocating entry
point's (ann_flat_query, exact mode) on the same inputs, on two calls in a row (the fixed scratch
keeps the previous call's contents), and it must reject batches whose scratch exceeds the fixed
array. This file is collected last so a failure here leaves every other test already run.
"""
import numpy as np
import pytest

from annvedi_b200 import synth

pytestmark = pytest.mark.gpu


def _noalloc(ix, q, k, ids, dists):
    import torch
    from annvedi_b200 import _lib
    lib = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    return lib.ann_flat_query_noalloc(ix._h, q.data_ptr(), q.shape[0], q.stride(0), k, ids.data_ptr(),
                                      dists.data_ptr(), st)


@pytest.mark.parametrize("n,dim,nq,k", [(60000, 384, 64, 100), (20011, 100, 9, 37)])
def test_no_alloc_matches_allocating_entry_point(cuda, n, dim, nq, k):
    import torch
    from annvedi_b200 import _lib
    from annvedi_b200.linear import LinearIndex
    w = synth.flat_normal(n, dim, 2 * nq, seed=n + k)
    ix = LinearIndex(device=0, mode="exact")
    ix.fit(torch.from_numpy(w.base).cuda())
    queries = torch.from_numpy(w.queries).cuda()
    for call in range(2):  # two calls in a row, different queries
        q = queries[call * nq:(call + 1) * nq]
        want_ids, want_d = ix.search(q, k, mode="exact")
        ids = torch.full((nq, k), -7, dtype=torch.int64, device=cuda)
        dists = torch.full((nq, k), float("nan"), dtype=torch.float32, device=cuda)
        before = ix.total_distances_count()
        _lib.check(_noalloc(ix, q, k, ids, dists))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(ids.cpu().numpy(), want_ids.cpu().numpy())
        np.testing.assert_allclose(dists.cpu().numpy(), want_d.cpu().numpy(), rtol=1e-5, atol=1e-6)
        assert ix.total_distances_count() == before + n * nq


def test_no_alloc_rejects_oversized_batch(cuda):
    import torch
    from annvedi_b200 import _lib
    from annvedi_b200.linear import LinearIndex
    w = synth.flat_normal(4096, 384, 1, seed=1)
    ix = LinearIndex(device=0, mode="exact")
    ix.fit(w.base)
    nq, k = 20000, 512  # 20000 * 512 * 8 bytes of per-split lists alone exceed the fixed scratch
    q = torch.zeros(nq, 384, device=cuda)
    ids = torch.empty(nq, k, dtype=torch.int64, device=cuda)
    dists = torch.empty(nq, k, dtype=torch.float32, device=cuda)
    rc = _noalloc(ix, q, k, ids, dists)
    assert rc == _lib.ANN_ERR_INVALID
    assert "scratch" in _lib.last_error()
