"""GPU tests of the captured search (CUDA graph) and of the autotuner.

A graph replays exactly the launches of one device search of a fixed batch, so its results
equal the direct call's bit for bit; it reads the queries through the captured pointer (new
queries in the same buffer give their own results); a launch after the engine reallocated a
buffer is refused. The autotuner only chooses among forms with identical results."""
import os
import tempfile

import numpy as np
import pytest

from pdx_b200 import compiled
from pdx_b200.builder import GaussianMixture, build_index

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tree_index():
    gm = GaussianMixture(256, 30, 0.4, seed=31, unit_norm=True)
    X = gm.sample(8000, 0)
    f = build_index(X, "pdx_tree_u8", num_clusters=64, num_meso_clusters=8, normalize=True, seed=9)
    td = tempfile.TemporaryDirectory()
    p = os.path.join(td.name, "ix.pdx")
    f.save(p)
    yield p, gm
    td.cleanup()


def _buffers(Q, k):
    import torch
    nq = len(Q)
    q = torch.from_numpy(np.ascontiguousarray(Q, np.float32)).cuda()
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    ds = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
    return q, ids, ds, cnt


def _host(ids, ds, cnt):
    return ids.cpu().numpy().view(np.uint32).copy(), ds.cpu().numpy().copy(), cnt.cpu().numpy().copy()


def test_graph_replay_equals_direct_search(tree_index):
    import torch
    p, gm = tree_index
    ix = compiled.load_index(p)
    ix.set_nprobe(12)
    k = 10
    Q1, Q2 = gm.sample(600, 1), gm.sample(600, 2)
    q, ids, ds, cnt = _buffers(Q1, k)
    stream = torch.cuda.current_stream().cuda_stream
    ix.search_device(q.data_ptr(), len(Q1), k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(), stream=stream)
    torch.cuda.synchronize()
    direct1 = _host(ids, ds, cnt)
    q.copy_(torch.from_numpy(Q2))
    ix.search_device(q.data_ptr(), len(Q2), k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(), stream=stream)
    torch.cuda.synchronize()
    direct2 = _host(ids, ds, cnt)
    q.copy_(torch.from_numpy(Q1))
    torch.cuda.synchronize()
    g = ix.capture(q.data_ptr(), len(Q1), k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr())
    for Q, ref in ((Q1, direct1), (Q2, direct2), (Q1, direct1)):
        q.copy_(torch.from_numpy(Q))
        ids.zero_()
        torch.cuda.synchronize()
        g.launch(stream)
        torch.cuda.synchronize()
        for a, b in zip(_host(ids, ds, cnt), ref):
            np.testing.assert_array_equal(a, b)
    # a larger batch grows the engine's buffers: the old graph must refuse to launch
    Q3 = gm.sample(3000, 3)
    q3, ids3, ds3, cnt3 = _buffers(Q3, k)
    ix.search_device(q3.data_ptr(), len(Q3), k, ids3.data_ptr(), ds3.data_ptr(), cnt3.data_ptr(), stream=stream)
    torch.cuda.synchronize()
    with pytest.raises(ValueError):
        g.launch(stream)
    del g


def test_autotune_keeps_results(tree_index):
    import torch
    p, gm = tree_index
    ix = compiled.load_index(p)
    ix.set_nprobe(12)
    k = 10
    Q = gm.sample(2000, 4)
    q, ids, ds, cnt = _buffers(Q, k)
    stream = torch.cuda.current_stream().cuda_stream
    ix.search_device(q.data_ptr(), len(Q), k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(), stream=stream)
    torch.cuda.synchronize()
    before = _host(ids, ds, cnt)
    choice = ix.autotune(q.data_ptr(), len(Q), k)
    assert choice["threads_per_query"] in (64, 128, 256)
    assert choice["top_level_mode"] in (2, 3)
    assert choice["start_mode"] in (0, 1)
    ix.search_device(q.data_ptr(), len(Q), k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(), stream=stream)
    torch.cuda.synchronize()
    for a, b in zip(_host(ids, ds, cnt), before):
        np.testing.assert_array_equal(a, b)
