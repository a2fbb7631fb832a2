"""CUDA graphs of fixed-shape searches (annvedi_b200.graphs): a replay returns what the eager call returns,
for new query contents each time (the plain exact scan at 1 and 4 queries, IVF-SQ8 at 1 and 8)."""
import numpy as np
import pytest

from annvedi_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("batch", [1, 4])
def test_graphed_flat_scan_equals_eager(cuda, batch):
    import torch
    from annvedi_b200 import graphs
    from annvedi_b200.linear import LinearIndex
    w = synth.flat_normal(100_000, 384, 64, seed=batch)
    ix = LinearIndex(device=0, mode="exact")
    ix.fit(torch.from_numpy(w.base).cuda())
    g = graphs.flat_exact(ix, batch, 100)
    q = torch.from_numpy(w.queries).cuda()
    for s in range(0, 3 * batch, batch):
        gi, gd = g(q[s:s + batch])
        torch.cuda.synchronize()
        ei, ed = ix.search(q[s:s + batch], 100, mode="exact")
        np.testing.assert_array_equal(gi.cpu().numpy(), ei.cpu().numpy())
        np.testing.assert_array_equal(gd.cpu().numpy(), ed.cpu().numpy())


@pytest.mark.parametrize("batch", [1, 8])
def test_graphed_ivf_equals_eager(cuda, batch):
    import torch
    from annvedi_b200 import graphs
    from annvedi_b200.ivf import IVFIndex
    w = synth.zipf_mixture(60_000, 128, 64, c=64, lo=20, hi=6000, seed=batch)
    ix = IVFIndex(device=0, mode="exact")
    ix.fit(torch.from_numpy(w.base).cuda(), 1, 0, 64, centroids=w.centres)
    g = graphs.ivf_exact(ix, batch, 100, 8, 300)
    q = torch.from_numpy(w.queries).cuda()
    before = ix.total_distances_count()
    for s in range(0, 3 * batch, batch):
        gi, gd = g(q[s:s + batch])
        torch.cuda.synchronize()
        ei, ed = ix.search(q[s:s + batch], 100, 0, 8, 300, max_candidates=0, mode="exact")
        np.testing.assert_array_equal(gi.cpu().numpy(), ei.cpu().numpy())
        np.testing.assert_array_equal(gd.cpu().numpy(), ed.cpu().numpy())
    assert ix.total_distances_count() > before  # the device-side counter advances on replays
