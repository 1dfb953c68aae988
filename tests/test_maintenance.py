"""Append / Delete on tree indexes (PDXTreeIndex::Append / Delete, index.hpp:580-638).

CPU tests pin the oracle (the reference's own Cluster code behind oracle/_ref, with the few
index.hpp lines restated) against the properties of the reference's tests/test_maintenance.cpp:
an appended row is found, appended rows pass a filter on them, a deleted row is gone; plus the
tombstone reuse, compaction and capacity-growth paths.

GPU tests hold the engine to the oracle after the same sequence of appends and deletes: search
results bit-identical (distances equal, ids equal up to ties), the same live row ids in the same
slot order in every cluster, the same maintenance counters, and after Save (which compacts) the
same file contents. Appended rows are passed pre-rotated to both (the engine's own rotation), so
the stored values are identical; raw rows go through each side's rotation in the property tests."""
import os
import tempfile

import numpy as np
import pytest

from pdx_b200.builder import GaussianMixture, build_index
from pdx_b200.layout import Level, read_index
from tests.helpers import assert_same


def _tree_file(path, itype, d=128, n=3000, nlist=24, nmeso=4, seed=3, full_clusters=()):
    """A tree index file; clusters listed in full_clusters get max_capacity == n (so the first
    delete there makes the health check compact)."""
    gm = GaussianMixture(d, 16, 0.35, seed=seed, unit_norm=True)
    X = gm.sample(n, 0)
    f = build_index(X, itype, num_clusters=nlist, num_meso_clusters=nmeso, normalize=True, seed=seed)
    if full_clusters:
        caps = f.l1.caps()
        for c in full_clusters:
            caps[c] = f.l1.embeddings[c].shape[0]
        f.l1 = Level(f.l1.embeddings, f.l1.row_ids, f.l1.centroids, caps)
    f.save(path)
    return f, gm, X


@pytest.fixture(scope="module")
def ref_cls(built_oracle):
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("oracle/_ref not built")
    return Reference


# ----------------------------------------------------------------------------- oracle (CPU)

@pytest.mark.parametrize("itype", ["pdx_tree_f32", "pdx_tree_u8"])
def test_oracle_reference_maintenance_properties(ref_cls, itype):
    """tests/test_maintenance.cpp: InsertSingleAndSearch, InsertMultipleAndFilteredSearch,
    InsertDeleteAndSearch (raw rows through the reference's rotation, normalize on)."""
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f, gm, X = _tree_file(p, itype)
        n = X.shape[0]
        extra = gm.sample(12, 7)
        ref = ref_cls(p)
        ref.set_append_normalization(True)
        ref.set_nprobe(0)
        ref.append(n, extra[0])
        ids, _ = ref.search(extra[0], 10)
        assert n in ids.tolist()
        for i in range(1, 11):
            ref.append(n + i, extra[i])
        fids, _ = ref.filtered_search(extra[1], 10, np.arange(n + 1, n + 11, dtype=np.uint64))
        assert set(fids.tolist()) == set(range(n + 1, n + 11))
        ref.append(n + 11, extra[11])
        ref.delete(n + 11)
        ids, _ = ref.search(extra[11], 10)
        assert n + 11 not in ids.tolist()
        with pytest.raises(ValueError, match="not sequential"):
            ref.append(n + 20, extra[0])
        with pytest.raises(ValueError, match="already deleted"):
            ref.delete(n + 11)
        with pytest.raises(ValueError, match="not in the index"):
            ref.delete(n + 50)
        ref.close()


def test_oracle_tombstone_reuse_compaction_growth(ref_cls):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f, gm, X = _tree_file(p, "pdx_tree_u8", full_clusters=(0,))
        ref = ref_cls(p)
        n = X.shape[0]
        # deleting from the full cluster 0 compacts it at once (used == max_capacity)
        victim = int(f.l1.row_ids[0][0])
        before = len(f.l1.row_ids[0])
        ref.delete(victim)
        st = ref.maintenance_stats()
        assert st["compactions"] == 1
        ids0 = ref.cluster_row_ids(0)
        assert len(ids0) == before - 1 and victim not in ids0.tolist()
        # a tombstoned slot is reused by the next append landing in its cluster
        R = ref.rotate(X[7:8] / np.linalg.norm(X[7]))
        ref.append(n, R[0], transformed=True)
        c = next(c for c in range(ref.nclusters) if n in ref.cluster_row_ids(c).tolist())
        v = int(ref.cluster_row_ids(c)[3])
        ref.delete(v)
        ref.append(n + 1, R[0], transformed=True)  # the same row: the same cluster
        ids = ref.cluster_row_ids(c).tolist()
        assert ids.index(n + 1) == 3 and v not in ids
        # appending near-duplicates of that row fills its cluster to max_capacity: growth
        rng = np.random.default_rng(0)
        for i in range(2, 300):
            ref.append(n + i, R[0] + rng.normal(0, 1e-3, R.shape[1]).astype(np.float32), transformed=True)
        assert ref.maintenance_stats()["capacity_growths"] >= 1
        assert len(ref.cluster_row_ids(c)) > 256
        ref.close()


# ----------------------------------------------------------------------------- engine (GPU)

def _compare(ix, ref, R, k, filters=None, ctx=""):
    ids, ds, cnt = ix.search_batch(R, k, transformed=True)
    for i in range(len(R)):
        pi, pd = ref.search(R[i], k, transformed=True)
        assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd, ctx=f"{ctx} q{i}")
    if filters is not None:
        fids, fds, fcnt = ix.filtered_search_batch(R, k, filters, transformed=True)
        for i in range(len(R)):
            pi, pd = ref.filtered_search(R[i], k, filters[i], transformed=True)
            assert_same(fids[i, :fcnt[i]], fds[i, :fcnt[i]], pi, pd, ctx=f"{ctx} filtered q{i}")


def _same_clusters(ix, ref):
    for c in range(ref.nclusters):
        a = ix.get_cluster_row_ids(c)
        b = ref.cluster_row_ids(c)
        assert ix.get_cluster_size(c) == len(b)
        np.testing.assert_array_equal(a, b, err_msg=f"cluster {c}")


@pytest.mark.gpu
@pytest.mark.parametrize("itype", ["pdx_tree_f32", "pdx_tree_u8"])
def test_engine_matches_oracle_through_appends_and_deletes(ref_cls, itype):
    from pdx_b200 import compiled
    rng = np.random.default_rng(11)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f, gm, X = _tree_file(p, itype, full_clusters=(2, 5))
        n = X.shape[0]
        ix = compiled.load_index(p)
        ref = ref_cls(p)
        Q = gm.sample(20, 3)
        R = ix.prepare_queries(Q)
        live = set(range(n))
        next_id = n
        new_rows = ix.prepare_queries(gm.sample(400, 5))
        anchor = new_rows[0]
        k = 10
        # clusters 2 and 5 are full (used == max_capacity): a delete there compacts at once, and
        # only then do they take appends (AppendEmbedding would overflow, in both)
        for c in (2, 5):
            victim = int(f.l1.row_ids[c][1])
            ix.delete(victim)
            ref.delete(victim)
            live.discard(victim)
        assert ix.maintenance_stats()["compactions"] == 2
        for rnd in range(6):
            # round 0 fills one cluster past its capacity (growth); later rounds mix appends of
            # new rows with deletes (tombstones, reuse, compaction of the full clusters 2 and 5)
            for _ in range(160 if rnd == 0 else 50):
                u = rng.random()
                if rnd == 0 or u < 0.55:
                    row = anchor + rng.normal(0, 2e-3, anchor.shape).astype(np.float32) if rnd == 0 else \
                        new_rows[(next_id - n) % len(new_rows)]
                    ix.append(next_id, row, transformed=True)
                    ref.append(next_id, row, transformed=True)
                    live.add(next_id)
                    next_id += 1
                else:
                    victim = int(rng.choice(sorted(live)))
                    ix.delete(victim)
                    ref.delete(victim)
                    live.discard(victim)
            assert ix.get_num_embeddings() == len(live)
            _same_clusters(ix, ref)
            st_e, st_r = ix.maintenance_stats(), ref.maintenance_stats()
            for key in ("appends", "deletes", "compactions", "capacity_growths", "merges_not_performed"):
                assert st_e[key] == st_r[key], (key, st_e, st_r)
            filters = [np.array(sorted(rng.choice(sorted(live), 300, replace=False)), np.uint64)
                       for _ in range(len(R))]
            for nprobe in (0, 6):
                ix.set_nprobe(nprobe)
                ref.set_nprobe(nprobe)
                _compare(ix, ref, R, k, filters if nprobe == 0 else None, ctx=f"{itype} round {rnd} nprobe {nprobe}")
        st = ix.maintenance_stats()
        assert st["compactions"] >= 2 and st["capacity_growths"] >= 1 and st["tombstones"] > 0
        # Save compacts every cluster, in the engine and in the reference alike
        out = os.path.join(td, "after.pdx")
        ix.save(out)
        ref.compact_all()
        _same_clusters(ix, ref)
        g = read_index(open(out, "rb").read())
        for c in range(ref.nclusters):
            np.testing.assert_array_equal(g.l1.row_ids[c], ref.cluster_row_ids(c))
        ix.set_nprobe(0)
        ref.set_nprobe(0)
        _compare(ix, ref, R, k, ctx=f"{itype} after save")
        # the saved file, loaded fresh, searches like the live index
        ref2 = ref_cls(out)
        ref2.set_nprobe(0)
        _compare(ix, ref2, R, k, ctx=f"{itype} reloaded")
        ref2.close()
        ref.close()


@pytest.mark.gpu
@pytest.mark.parametrize("itype", ["pdx_tree_f32", "pdx_tree_u8"])
def test_engine_reference_maintenance_properties(itype):
    """tests/test_maintenance.cpp on the engine: an index built with normalize, raw rows."""
    from pdx_b200 import compiled
    gm = GaussianMixture(384, 16, 0.35, seed=5, unit_norm=False)
    X = gm.sample(4001, 0)
    n = 4000
    ix = compiled.PDXIndex(itype, 384, normalize=True, num_clusters=40, num_meso_clusters=6)
    ix.build_index(X[:n])
    ix.set_nprobe(0)
    ix.append(n, X[n])
    ids, _ = ix.search(X[n], 10)
    assert n in ids.tolist()
    extra = gm.sample(11, 9)
    for i in range(10):
        ix.append(n + 1 + i, extra[i])
    fids, _ = ix.filtered_search(extra[0], 10, np.arange(n + 1, n + 11, dtype=np.uint64))
    assert set(fids.tolist()) == set(range(n + 1, n + 11))
    ix.append(n + 11, extra[10])
    ix.delete(n + 11)
    ids, _ = ix.search(extra[10], 10)
    assert n + 11 not in ids.tolist()
    assert ix.get_num_embeddings() == n + 11
    with pytest.raises(ValueError, match="not sequential"):
        ix.append(n + 30, extra[0])
    with pytest.raises(ValueError, match="already deleted"):
        ix.delete(n + 11)
    with pytest.raises(ValueError, match="not in the index"):
        ix.delete(n + 100)


@pytest.mark.gpu
def test_flat_index_append_is_not_implemented():
    from pdx_b200 import compiled
    with tempfile.TemporaryDirectory() as td:
        gm = GaussianMixture(64, 8, 0.3, seed=1, unit_norm=True)
        X = gm.sample(800, 0)
        p = os.path.join(td, "flat.pdx")
        build_index(X, "pdx_u8", num_clusters=8, seed=1).save(p)
        ix = compiled.load_index(p)
        with pytest.raises(RuntimeError, match="Append is not implemented in PDXIndex"):
            ix.append(800, X[0])


@pytest.mark.gpu
@pytest.mark.parametrize("itype", ["pdx_tree_f32", "pdx_tree_u8"])
def test_batch_append_equals_row_appends(ref_cls, itype):
    """append_batch over chunks of several sizes (one crossing a capacity growth) leaves the same
    clusters, counters and search results as one append per row, and as the oracle."""
    from pdx_b200 import compiled
    rng = np.random.default_rng(4)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f, gm, X = _tree_file(p, itype, seed=8)
        n = X.shape[0]
        rows_ix = compiled.load_index(p)
        batch_ix = compiled.load_index(p)
        ref = ref_cls(p)
        new = rows_ix.prepare_queries(gm.sample(300, 6))
        near = new[0] + rng.normal(0, 2e-3, (200, new.shape[1])).astype(np.float32)
        rows = np.concatenate([near, new]).astype(np.float32)
        victims = rng.choice(n, 60, replace=False)
        for v in victims[:30]:
            for ix in (rows_ix, batch_ix):
                ix.delete(int(v))
            ref.delete(int(v))
        for i, r in enumerate(rows):
            rows_ix.append(n + i, r, transformed=True)
            ref.append(n + i, r, transformed=True)
        a = 0
        for size in (1, 7, 250, len(rows)):
            b = min(len(rows), a + size)
            batch_ix.append_batch(n + a, rows[a:b], transformed=True)
            a = b
            if a == len(rows):
                break
        for v in victims[30:]:
            for ix in (rows_ix, batch_ix):
                ix.delete(int(v))
            ref.delete(int(v))
        assert rows_ix.maintenance_stats() == batch_ix.maintenance_stats()
        assert batch_ix.maintenance_stats()["capacity_growths"] >= 1
        _same_clusters(batch_ix, ref)
        _same_clusters(rows_ix, ref)
        Q = batch_ix.prepare_queries(gm.sample(16, 9))
        for ix in (rows_ix, batch_ix):
            ix.set_nprobe(0)
        ref.set_nprobe(0)
        _compare(batch_ix, ref, Q, 10, ctx=f"{itype} batch")
        _compare(rows_ix, ref, Q, 10, ctx=f"{itype} rows")
        with pytest.raises(ValueError, match="not sequential"):
            batch_ix.append_batch(n, rows[:2], transformed=True)
        ref.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tree_f32_d130", "tree_u8_d256"])
def test_engine_matches_oracle_on_reference_files(ref_cls, name):
    """The same parity on index files the reference itself wrote (golden fixtures)."""
    from pdx_b200 import compiled
    from tests.helpers import load_golden
    path, queries, rotated, exp = load_golden(name)
    ix = compiled.load_index(path)
    ref = ref_cls(path)
    n = ix.get_num_embeddings()
    rng = np.random.default_rng(2)
    live = list(range(n))
    base = ix.prepare_queries(queries)
    next_id = n
    for step in range(120):
        if rng.random() < 0.6:
            row = (base[step % len(base)] + rng.normal(0, 0.02, base.shape[1])).astype(np.float32)
            ix.append(next_id, row, transformed=True)
            ref.append(next_id, row, transformed=True)
            live.append(next_id)
            next_id += 1
        else:
            v = live.pop(int(rng.integers(len(live))))
            ix.delete(v)
            ref.delete(v)
    _same_clusters(ix, ref)
    for nprobe in (0, exp["nprobe"]):
        ix.set_nprobe(nprobe)
        ref.set_nprobe(nprobe)
        _compare(ix, ref, rotated, exp["k"], ctx=f"{name} nprobe {nprobe}")
    ref.close()


@pytest.mark.gpu
def test_request_batches_after_maintenance(ref_cls):
    """Serving batches (a context's pdxg_search_requests) after Append / Delete: per-request k and
    nprobe, row-list filters and a filter registered before the changes (rebuilt from its row ids,
    which name deleted rows and rows appended later) equal the oracle's searches."""
    from pdx_b200 import compiled
    from tests.test_gpu_serving import _run_requests
    rng = np.random.default_rng(21)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f, gm, X = _tree_file(p, "pdx_tree_u8", seed=5)
        n = X.shape[0]
        ix = compiled.load_index(p)
        ref = ref_cls(p)
        ctx = compiled.Context(ix)
        victims = rng.choice(n, 200, replace=False)
        fl_rows = np.concatenate([victims[:40], rng.choice(n, 300, replace=False), np.arange(n, n + 60)])
        fid = ix.register_filter(fl_rows.astype(np.uint64))
        R = ix.prepare_queries(gm.sample(32, 4))
        new = ix.prepare_queries(gm.sample(150, 5))
        for i, r in enumerate(new):
            ix.append(n + i, r, transformed=True)
            ref.append(n + i, r, transformed=True)
        for v in victims:
            ix.delete(int(v))
            ref.delete(int(v))
        live = np.array(sorted(set(range(n + len(new))) - set(victims.tolist())), np.uint32)
        reqs = []
        for i in range(len(R)):
            k = int(rng.choice((1, 10, 20)))
            npb = int(rng.choice((0, 3, 8)))
            kind = i % 3
            rows = None if kind == 0 else (fid if kind == 1 else
                                           np.sort(rng.choice(live, 250, replace=False)).astype(np.uint32))
            reqs.append((k, npb, rows))
        ids, ds, cnt = _run_requests(ctx, R, reqs, 20)
        for i, (k, npb, rows) in enumerate(reqs):
            ref.set_nprobe(npb)
            if rows is None:
                pi, pd = ref.search(R[i], k, transformed=True)
            else:
                sel = fl_rows if isinstance(rows, int) else rows
                pi, pd = ref.filtered_search(R[i], k, sel.astype(np.uint64), transformed=True)
            assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd, ctx=f"request {i} k={k} nprobe={npb}")
            assert not set(ids[i, :cnt[i]].tolist()) & set(victims.tolist())
        ctx.close()
        ref.close()


@pytest.mark.gpu
@pytest.mark.parametrize("itype", ["pdx_tree_f32", "pdx_tree_u8"])
def test_tombstones_in_start_and_masked_heaps(ref_cls, itype):
    """Clusters of about 8 rows with most rows deleted and k = 10: Start pushes tombstoned slots
    at the mask distance (searcher.hpp:169-179, 256-280) and later clusters prune against a heap
    top that is the mask; the results, deleted ids and mask distances included, are the oracle's.
    A cluster with every row deleted is skipped (num_embeddings == 0)."""
    from pdx_b200 import compiled
    rng = np.random.default_rng(13)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f, gm, X = _tree_file(p, itype, d=96, n=400, nlist=50, nmeso=5, seed=12)
        ix = compiled.load_index(p)
        ref = ref_cls(p)
        deleted = set()
        for c, rid in enumerate(f.l1.row_ids):
            drop = rid[: max(0, len(rid) - (1 if c % 3 else 0) - 1)] if c % 2 == 0 else rid[:1]
            for v in drop:
                ix.delete(int(v))
                ref.delete(int(v))
                deleted.add(int(v))
        R = ix.prepare_queries(gm.sample(24, 3))
        for nprobe in (1, 2, 3, 0):
            ix.set_nprobe(nprobe)
            ref.set_nprobe(nprobe)
            _compare(ix, ref, R, 10, ctx=f"{itype} nprobe {nprobe}")
            if nprobe == 1:  # the case is reached: masked slots come back, as in the reference
                ids, _, cnt = ix.search_batch(R, 10, transformed=True)
                assert sum(int(i) in deleted for q in range(len(R)) for i in ids[q, :cnt[q]]) > 0
        ref.close()
