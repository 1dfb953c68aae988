"""Serving-form parity: batches of requests with their own k, nprobe and row-id filter
(pdxg_search_requests) give, for every request, exactly the result of the same request searched
alone -- through the per-call API and through the oracle port -- and the continuous-batching
server returns each request's result unchanged by the mix it ran in."""
import os
import tempfile

import numpy as np
import pytest

from pdx_b200 import compiled
from pdx_b200.builder import GaussianMixture, build_index
from pdx_b200.serving import Server, Workload, make_filters, poisson_mix
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu

N_ROWS = 4000


@pytest.fixture(scope="module")
def port_cls(built_oracle):
    from oracle.oracle import Port
    return Port


def _index(itype, d, seed):
    gm = GaussianMixture(d, 16, 0.5, seed=seed + d, unit_norm=False)
    X = gm.sample(N_ROWS, 0)
    Q = gm.sample(48, 1)
    f = build_index(X, itype, num_clusters=24, num_meso_clusters=5 if "tree" in itype else 0, seed=seed)
    return f, Q


def _mix(nq, seed, ks=(1, 10, 20, 100), nprobes=(0, 1, 3, 8, 24, 40)):
    """Request parameters: k, nprobe and half of the queries with filters of log-uniform
    selectivity, plus the filter edge cases (empty, one row, every row, unknown ids)."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(nq):
        k = int(rng.choice(ks))
        npb = int(rng.choice(nprobes))
        rows = None
        if i % 2 == 1:
            edge = i // 2 % 8
            if edge == 0:
                rows = np.zeros(0, np.uint32)
            elif edge == 1:
                rows = np.array([int(rng.integers(N_ROWS))], np.uint32)
            elif edge == 2:
                rows = np.arange(N_ROWS, dtype=np.uint32)
            elif edge == 3:
                rows = np.array([N_ROWS + 5, 3, 2 ** 31, 77], np.uint32)
            else:
                sel = float(np.exp(rng.uniform(np.log(0.001), np.log(0.5))))
                rows = np.sort(rng.choice(N_ROWS, max(1, int(sel * N_ROWS)), replace=False)).astype(np.uint32)
        reqs.append((k, npb, rows))
    return reqs


def _table(reqs):
    """reqs: (k, nprobe, filter) with filter None, a row-id array, or a registered filter id."""
    table = compiled.request_table(len(reqs))
    parts, pos = [], 0
    for j, (k, npb, rows) in enumerate(reqs):
        table[j]["k"] = k
        table[j]["nprobe"] = npb
        if isinstance(rows, int):
            table[j]["filter_id"] = rows
        elif rows is not None:
            table[j]["filter_begin"] = pos
            table[j]["filter_end"] = pos + len(rows)
            parts.append(rows)
            pos += len(rows)
    rows = np.concatenate(parts).astype(np.uint32) if parts else None
    return table, rows


def _run_requests(ctx, R, reqs, k_max):
    import torch
    dev = torch.device("cuda", 0)
    nq = len(reqs)
    table, rows = _table(reqs)
    q = torch.from_numpy(np.ascontiguousarray(R, dtype=np.float32)).to(dev)
    ids = torch.empty((nq, k_max), dtype=torch.int32, device=dev)
    ds = torch.empty((nq, k_max), dtype=torch.float32, device=dev)
    cnt = torch.empty(nq, dtype=torch.int32, device=dev)
    ctx.search_requests(q.data_ptr(), nq, table, rows, k_max, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(),
                        transformed=True)
    torch.cuda.synchronize()
    return ids.cpu().numpy().view(np.uint32), ds.cpu().numpy(), cnt.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("itype,d", [("pdx_u8", 96), ("pdx_f32", 130), ("pdx_tree_u8", 130),
                                     ("pdx_tree_f32", 96)])
def test_requests_match_single_searches(port_cls, itype, d):
    f, Q = _index(itype, d, seed=4)
    reqs = _mix(len(Q), seed=d)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        port = port_cls(p)
        ix = compiled.load_index(p)
        R = ix.prepare_queries(Q)
        ctx = compiled.Context(ix)
        ids, ds, cnt = _run_requests(ctx, R, reqs, 100)
        for i, (k, npb, rows) in enumerate(reqs):
            port.set_nprobe(npb)
            if rows is None:
                pi, pd = port.search(R[i], k, transformed=True)
            else:
                pi, pd = port.filtered_search(R[i], k, rows.astype(np.uint64), transformed=True)
                assert set(ids[i, :cnt[i]].tolist()) <= set(rows.tolist())
            assert cnt[i] <= k
            assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd,
                        ctx=f"{itype} d={d} q{i} k={k} nprobe={npb} filtered={rows is not None}")
            # the unused tail of each output row is marked empty
            assert np.all(ids[i, cnt[i]:] == 0xFFFFFFFF)
        # the same requests through the per-call API
        for i in range(0, len(reqs), 5):
            k, npb, rows = reqs[i]
            ix.set_nprobe(npb)
            if rows is None:
                a, b, c = ix.search_batch(R[i:i + 1], k, transformed=True)
            else:
                a, b, c = ix.filtered_search_batch(R[i:i + 1], k, [rows.astype(np.uint64)], transformed=True)
            np.testing.assert_array_equal(a[0, :c[0]], ids[i, :cnt[i]])
            np.testing.assert_array_equal(b[0, :c[0]], ds[i, :cnt[i]])
        ctx.close()
        port.close()


def test_requests_alone_equals_in_batch_and_duplicates():
    f, Q = _index("pdx_tree_u8", 200, seed=7)
    reqs = _mix(len(Q), seed=11)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        R = ix.prepare_queries(Q)
        ctx = compiled.Context(ix)
        ids, ds, cnt = _run_requests(ctx, R, reqs, 100)
        for i in range(len(reqs)):
            a, b, c = _run_requests(ctx, R[i:i + 1], [reqs[i]], reqs[i][0])
            np.testing.assert_array_equal(a[0, :c[0]], ids[i, :cnt[i]])
            np.testing.assert_array_equal(b[0, :c[0]], ds[i, :cnt[i]])
        # a filter that repeats row ids selects the same rows as its distinct ids
        dup = [(k, npb, None if rows is None else np.concatenate([rows, rows[::-1]]))
               for (k, npb, rows) in reqs]
        a, b, c = _run_requests(ctx, R, dup, 100)
        np.testing.assert_array_equal(c, cnt)
        for i in range(len(reqs)):
            np.testing.assert_array_equal(a[i, :c[i]], ids[i, :cnt[i]])
        # invalid requests fail with a clear error
        with pytest.raises(ValueError):
            _run_requests(ctx, R[:1], [(0, 4, None)], 10)
        with pytest.raises(ValueError):
            _run_requests(ctx, R[:1], [(20, 4, None)], 10)
        ctx.close()


def test_registered_filters_match_row_lists():
    f, Q = _index("pdx_tree_u8", 130, seed=6)
    reqs = _mix(len(Q), seed=3)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        R = ix.prepare_queries(Q)
        ctx = compiled.Context(ix)
        ids, ds, cnt = _run_requests(ctx, R, reqs, 100)
        reg = [(k, npb, None if rows is None else ix.register_filter(rows)) for (k, npb, rows) in reqs]
        a, b, c = _run_requests(ctx, R, reg, 100)
        np.testing.assert_array_equal(c, cnt)
        for i in range(len(reqs)):
            np.testing.assert_array_equal(a[i, :c[i]], ids[i, :cnt[i]])
            np.testing.assert_array_equal(b[i, :c[i]], ds[i, :cnt[i]])
        # release + re-register reuses slots; unknown ids are rejected
        fid = reg[1][2]
        ix.release_filter(fid)
        with pytest.raises(ValueError):
            _run_requests(ctx, R[:1], [(10, 4, fid)], 10)
        with pytest.raises(ValueError):
            ix.release_filter(fid)
        assert ix.register_filter(reqs[1][2]) == fid
        ctx.close()


@pytest.mark.parametrize("max_batch,n_contexts,rate", [(7, 3, 20000.0), (64, 2, 5000.0), (4096, 3, 0.0)])
def test_server_mix_equals_alone(max_batch, n_contexts, rate):
    f, Q = _index("pdx_u8", 128, seed=5)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        filters = make_filters(ix, 6, seed=2)
        Qs = np.concatenate([Q] * 4)
        w = poisson_mix(Qs, rate, filters, seed=9, ks=(10, 20, 100), nprobes=(8, 16, 24))
        # a few requests carry their own row-id lists instead of a registered filter
        rng = np.random.default_rng(4)
        w.rows = [None] * len(w)
        for i in range(0, len(w), 9):
            w.filter_id[i] = -1
            w.rows[i] = np.sort(rng.choice(N_ROWS, 300, replace=False)).astype(np.uint32)
        srv = Server(ix, max_batch=max_batch, n_contexts=n_contexts, k_max=100)
        served = srv.run(w, realtime=rate > 0)
        if max_batch < len(w):
            assert len(np.unique(served.batch)) > 1
        assert np.all(served.latency >= 0)
        ctx = compiled.Context(ix)
        import torch
        for i in range(len(w)):
            k = int(w.k[i])
            q = torch.from_numpy(Qs[i:i + 1].astype(np.float32)).cuda()
            a = torch.empty((1, k), dtype=torch.int32, device="cuda")
            b = torch.empty((1, k), dtype=torch.float32, device="cuda")
            c = torch.empty(1, dtype=torch.int32, device="cuda")
            filt = w.rows[i] if w.rows[i] is not None else (int(w.filter_id[i]) if w.filter_id[i] >= 0 else None)
            table, rows = _table([(k, int(w.nprobe[i]), filt)])
            ctx.search_requests(q.data_ptr(), 1, table, rows, k, a.data_ptr(), b.data_ptr(), c.data_ptr())
            torch.cuda.synchronize()
            n = int(c.item())
            si, sd = served.result(i)
            np.testing.assert_array_equal(si, a.cpu().numpy().view(np.uint32)[0, :n])
            np.testing.assert_array_equal(sd, b.cpu().numpy()[0, :n])
        ctx.close()
        srv.close()
