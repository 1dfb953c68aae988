"""GPU parity of the cluster-major scan (pdxg_scan.cu) for U8 indexes.

After a batched Start, the first warmup step of every (query, visited cluster) pair is computed
per cluster and a warp per query replays PDXearch on it (scan mode 0, the default); scan mode 1
runs the per-query kernel for every query. Both must return bit-identical results, and both must
equal the oracle port on the same prepared queries (ids as sets inside tied distances). The cases
cover the replay's own fallbacks -- a warmup that does not stop after its first step (pruning
off), Start clusters smaller than k (those queries go to the per-query kernel), filtered queries
mixed into a batch, per-request k -- and dimensions whose first checkpoint is short (d_v < 16).
"""
import os
import tempfile

import numpy as np
import pytest

from pdx_b200 import compiled
from pdx_b200.builder import GaussianMixture, build_index
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def port_cls(built_oracle):
    from oracle.oracle import Port
    return Port


def _index(itype, d, n, nlist, nmeso, nq, seed, sigma=0.3, comps=24):
    gm = GaussianMixture(d, comps, sigma, seed=seed + 7 * d, unit_norm=True)
    X = gm.sample(n, 0)
    Q = gm.sample(nq, 1)
    f = build_index(X, itype, num_clusters=nlist, num_meso_clusters=nmeso, normalize=True, seed=seed)
    td = tempfile.mkdtemp()
    p = os.path.join(td, "ix.pdx")
    f.save(p)
    return p, Q


def _both_modes(ix, R, k):
    """Results with the cluster-major scan and with the per-query kernel, and the launch counts."""
    out = []
    for mode in (0, 1):
        ix.set_scan_mode(mode)
        ids, ds, cnt = ix.search_batch(R, k, transformed=True)
        out.append((ids, ds, cnt, ix.last_launch_count()))
    ix.set_scan_mode(0)
    return out


def test_stats_are_the_same_in_both_scan_forms():
    """The algorithmic byte counts (PDXG_COLLECT_STATS) do not depend on the scan form."""
    import torch
    path, Q = _index("pdx_tree_u8", 256, 6000, 16, 4, 96, seed=13)
    ix = compiled.load_index(path)
    ix.set_nprobe(6)
    R = torch.from_numpy(ix.prepare_queries(Q)).cuda()
    nq, k = len(Q), 20
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    ds = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
    stats = []
    for mode in (0, 1):
        ix.set_scan_mode(mode)
        ix.search_device(R.data_ptr(), nq, k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(),
                         stream=torch.cuda.current_stream().cuda_stream, transformed=True, stats=True)
        torch.cuda.synchronize()
        stats.append(ix.last_stats())
    ix.set_scan_mode(0)
    assert stats[0]["bytes_by_phase"] == stats[1]["bytes_by_phase"]
    assert stats[0]["clusters_visited"] == stats[1]["clusters_visited"]
    assert stats[0]["merged"] == stats[1]["merged"]


def _same(a, b, ctx):
    np.testing.assert_array_equal(a[2], b[2], err_msg=f"{ctx}: counts")
    for i in range(len(a[2])):
        c = a[2][i]
        np.testing.assert_array_equal(a[0][i, :c], b[0][i, :c], err_msg=f"{ctx}: ids q{i}")
        np.testing.assert_array_equal(a[1][i, :c], b[1][i, :c], err_msg=f"{ctx}: dists q{i}")


def _vs_port(port, got, R, k, ctx):
    ids, ds, cnt = got[:3]
    for i in range(len(R)):
        pi, pd = port.search(R[i], k, transformed=True)
        assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd, ctx=f"{ctx} q{i}")


@pytest.mark.parametrize("itype", ["pdx_u8", "pdx_tree_u8"])
@pytest.mark.parametrize("d,k,nprobe", [(256, 20, 6), (100, 10, 0), (44, 7, 3), (12, 5, 4), (1024, 100, 5)])
def test_cluster_major_equals_per_query_and_port(port_cls, itype, d, k, nprobe):
    n = 3000 if d >= 1024 else 6000
    path, Q = _index(itype, d, n, 16, 4, 96, seed=11)
    ix = compiled.load_index(path)
    port = port_cls(path)
    ix.set_nprobe(nprobe)
    port.set_nprobe(nprobe)
    R = ix.prepare_queries(Q)
    cm, pq = _both_modes(ix, R, k)
    assert cm[3] == pq[3] + 3, f"cluster-major scan did not run: {cm[3]} vs {pq[3]} launches"
    _same(cm, pq, f"{itype} d={d} k={k}")
    _vs_port(port, cm, R, k, f"{itype} d={d} k={k} nprobe={nprobe}")
    # pruning off: no warmup stops after its first step, so every visit takes the replay's
    # full warmup
    ix.set_pruning_aggressiveness(1e30)
    port.set_pruning_aggressiveness(1e30)
    cm, pq = _both_modes(ix, R, k)
    _same(cm, pq, f"{itype} d={d} unpruned")
    _vs_port(port, cm, R[:24], k, f"{itype} d={d} unpruned")
    port.close()


def test_small_start_clusters_go_to_the_per_query_kernel(port_cls):
    # about 12 vectors per cluster and k = 20: every Start leaves the heap short of k
    path, Q = _index("pdx_tree_u8", 64, 2400, 200, 14, 64, seed=5)
    ix = compiled.load_index(path)
    port = port_cls(path)
    for k, nprobe in ((20, 16), (8, 16), (3, 0)):
        ix.set_nprobe(nprobe)
        port.set_nprobe(nprobe)
        R = ix.prepare_queries(Q)
        cm, pq = _both_modes(ix, R, k)
        _same(cm, pq, f"small clusters k={k}")
        _vs_port(port, cm, R, k, f"small clusters k={k}")
    port.close()


def test_filtered_queries_mixed_into_a_batch(port_cls):
    path, Q = _index("pdx_tree_u8", 128, 6000, 16, 4, 64, seed=9)
    ix = compiled.load_index(path)
    port = port_cls(path)
    ix.set_nprobe(6)
    port.set_nprobe(6)
    R = ix.prepare_queries(Q)
    rng = np.random.default_rng(1)
    lists = [None if i % 3 else rng.choice(6000, 900, replace=False).astype(np.uint64) for i in range(len(R))]
    res = []
    for mode in (0, 1):
        ix.set_scan_mode(mode)
        res.append(ix.filtered_search_batch(R, 10, lists, transformed=True))
    ix.set_scan_mode(0)
    _same(res[0], res[1], "mixed filters")
    ids, ds, cnt = res[0]
    for i in range(len(R)):
        if lists[i] is None:
            pi, pd = port.search(R[i], 10, transformed=True)
        else:
            pi, pd = port.filtered_search(R[i], 10, lists[i], transformed=True)
        assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd, ctx=f"mixed filters q{i}")
    port.close()


def test_per_request_k_and_nprobe():
    import torch
    path, Q = _index("pdx_tree_u8", 256, 6000, 16, 4, 128, seed=21)
    ix = compiled.load_index(path)
    rng = np.random.default_rng(4)
    req = compiled.request_table(len(Q))
    req["k"] = rng.choice([1, 10, 20, 100], len(Q))
    req["nprobe"] = rng.choice([2, 6, 16], len(Q))
    q = torch.from_numpy(Q).cuda()
    outs = []
    for mode in (0, 1):
        ix.set_scan_mode(mode)
        ctx = compiled.Context(ix)
        ids = torch.full((len(Q), 100), -1, dtype=torch.int32, device="cuda")
        ds = torch.full((len(Q), 100), -1.0, dtype=torch.float32, device="cuda")
        cnt = torch.zeros(len(Q), dtype=torch.int32, device="cuda")
        ctx.search_requests(q.data_ptr(), len(Q), req, None, 100, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr())
        torch.cuda.synchronize()
        outs.append((ids.cpu().numpy(), ds.cpu().numpy(), cnt.cpu().numpy()))
        ctx.close()
    ix.set_scan_mode(0)
    _same(outs[0], outs[1], "per-request k / nprobe")
