"""The per-query selection of the best R keys (ann_select_smallest, the radix select of the tensor-core
forms) against numpy's (key, position) order, exactly, over the stream lengths that take each of its
paths: shorter than R, below 8R (histogram bins), the sampled bar (>= 8R) with up to 1,024 and with up to
2,048 keys under the bar, heavy ties, all keys equal, and infinite keys."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _select(keys, lens, r):
    import torch
    from annvedi_b200 import _lib
    lib = _lib.load()
    k = torch.from_numpy(keys).cuda()
    ln = torch.from_numpy(lens.astype(np.int64)).cuda()
    nq, ld = keys.shape
    ok = torch.empty(nq, r, dtype=torch.float32, device="cuda")
    op = torch.empty(nq, r, dtype=torch.int32, device="cuda")
    _lib.check(lib.ann_select_smallest(_lib.ptr(k), ld, _lib.ptr(ln), nq, r, _lib.ptr(ok), _lib.ptr(op),
                                       _lib.stream_ptr(k)))
    torch.cuda.synchronize()
    return ok.cpu().numpy(), op.cpu().numpy()


def _check(keys, lens, r):
    gk, gp = _select(keys, lens, r)
    for q in range(keys.shape[0]):
        n = int(lens[q])
        want = np.lexsort((np.arange(n), keys[q, :n]))[:r]
        m = len(want)
        o = np.lexsort((gp[q], gk[q]))  # the set by (key, position)
        np.testing.assert_array_equal(gp[q][o][:m], want, err_msg=f"row {q} len {n}")
        np.testing.assert_array_equal(gk[q][o][:m], keys[q, want])
        assert (gp[q][o][m:] == np.iinfo(np.int32).max).all() and np.isinf(gk[q][o][m:]).all()


@pytest.mark.parametrize("r", [1, 100, 300, 512])
def test_random_streams(cuda, r):
    rng = np.random.default_rng(r)
    nq, ld = 48, 40000
    keys = rng.standard_normal((nq, ld)).astype(np.float32) ** 2
    # lengths across the paths: < r, < 8r, >= 8r, the full row
    lens = np.concatenate([rng.integers(1, max(2, r), 8), rng.integers(r, 8 * r, 12),
                           rng.integers(8 * r, ld, 20), np.full(8, ld)])
    _check(keys, lens, r)


def test_skewed_and_tied_streams(cuda):
    rng = np.random.default_rng(7)
    nq, ld, r = 40, 30000, 300
    keys = rng.standard_normal((nq, ld)).astype(np.float32) ** 2
    keys[0:8] = np.round(keys[0:8] * 4) / 4          # few distinct values: long runs of ties
    keys[8:12] = 1.0                                   # all equal
    keys[12:16] = np.sort(keys[12:16], axis=1)         # ascending: the sample over-represents small keys
    keys[16:20] = np.sort(keys[16:20], axis=1)[:, ::-1]
    keys[20:24, ::50] = np.inf                         # infinite keys spread in
    keys[24:28] = rng.exponential(1e-3, (4, ld)).astype(np.float32) + 5.0   # narrow range, high offset
    # 1,500 tied keys below all others: the bar lets all of them through (between 1,024 and 2,048)
    keys[28:32] += 1.0
    for q in range(28, 32):
        keys[q, rng.choice(ld, 1500, replace=False)] = 0.5
    lens = np.full(nq, ld)
    _check(keys, lens, r)
