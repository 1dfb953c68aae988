"""Parity at the benchmark's scale: the production forms against the reference's own search.

The other GPU tests pin bit-exactness on small indexes. The forms that only run at scale --
128-query tiles of the tiled top level, the batched Start with its per-cluster query groups,
persistent scan CTAs over a 10,000-query batch, the CUDA graph the benchmark launches and the
two-chunk host pipeline of pdxg_search -- are checked here on the benchmark's own workloads
(bench.py builds and caches them):

* IVF2 SQ8, 1,000,000 x 1024, 1,000 L1 / 32 meso clusters, nprobe 32, k 20, one 10,000-query
  batch: 500 queries spread over the batch against oracle/_ref (the reference's PDXearch and
  tree search, AVX2 build) with pruning on, 100 with pruning off (SetPruningAggresiveness(1e30));
* IVF F32, 100,000 x 128, nlist 316, nprobe 16, k 10: the whole 1,000-query batch.

Both sides search the same prepared queries (the engine's rotation; rotation parity is tested
at FP32 tolerance elsewhere), so the bar is bit-identical distances and ids equal as sets inside
groups of tied distances (tests/helpers.py). Reference: searcher.hpp:596-724, index.hpp:545-566.
"""
import ctypes as C
import os

import numpy as np
import pytest

from tests.helpers import assert_same

pytestmark = pytest.mark.gpu


def _reference_available():
    from oracle.oracle import Reference
    return Reference.available("avx2")


def _workload(name):
    import bench
    cfg = dict(bench.CONFIGS[name])
    path, gm, gt = bench.dataset(name, "cuda:0")
    Q = gm.sample(cfg["nq"], 1)  # the benchmark's rank-0 batch
    return cfg, path, Q, gt


def _graph_search(ix, Q, k, forms=None):
    """The benchmark's step: one CUDA graph launch for the whole batch, in the given forms (threads
    per query, top-level mode, Start mode) or the autotuner's."""
    import torch
    nq = len(Q)
    q = torch.from_numpy(np.ascontiguousarray(Q)).cuda()
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    ds = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
    if forms is None:
        tuned = ix.autotune(q.data_ptr(), nq, k)
    else:
        ix.set_threads_per_query(forms[0])
        ix.set_top_level_mode(forms[1])
        ix.set_start_mode(forms[2])
        tuned = {"threads_per_query": forms[0], "top_level_mode": forms[1], "start_mode": forms[2]}
    g = ix.capture(q.data_ptr(), nq, k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr())
    ids.fill_(-1)
    cnt.fill_(-1)
    torch.cuda.synchronize()
    g.launch(0)
    torch.cuda.synchronize()
    out = (ids.cpu().numpy().view(np.uint32), ds.cpu().numpy(), cnt.cpu().numpy().view(np.uint32))
    del g
    return out, tuned


def _host_search(ix, Q, k):
    """pdxg_search with pinned host buffers (the two-chunk pipeline for large batches)."""
    import torch
    from pdx_b200 import compiled
    nq = len(Q)
    q = torch.from_numpy(np.ascontiguousarray(Q)).pin_memory()
    ids = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    ds = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    cnt = torch.empty(nq, dtype=torch.int32).pin_memory()
    lib = compiled.library()
    rc = lib.pdxg_search(ix.handle.ptr, C.c_void_p(q.data_ptr()), nq, k, 0, C.c_void_p(ids.data_ptr()),
                         C.c_void_p(ds.data_ptr()), C.c_void_p(cnt.data_ptr()))
    assert rc == 0, lib.pdxg_last_error().decode()
    return ids.numpy().view(np.uint32).copy(), ds.numpy().copy(), cnt.numpy().view(np.uint32).copy()


def _compare(got, ref_ids, ref_ds, ref_cnt, rows, ctx):
    ids, ds, cnt = got
    for j, i in enumerate(rows):
        assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], ref_ids[j, :ref_cnt[j]], ref_ds[j, :ref_cnt[j]],
                    ctx=f"{ctx} q{i}")


def test_ivf2_sq8_1m_d1024_production_forms_vs_reference(built_oracle):
    if not _reference_available():
        pytest.skip("oracle/_ref not built (the reference sources were not present at build time)")
    from oracle.oracle import Reference
    from pdx_b200 import compiled
    cfg, path, Q, gt = _workload("ivf2_sq8_1m_d1024")
    k, nq = cfg["k"], cfg["nq"]
    ix = compiled.load_index(path)
    ix.set_nprobe(cfg["nprobe"])
    prepared = ix.prepare_queries(Q)
    # the forms the autotuner picks for this batch on B200: 128 threads per query, tiled top
    # level, batched Start
    got, _ = _graph_search(ix, Q, k, forms=(128, 3, 0))
    # the host pipeline rotates in two chunks; per-row results are those of the whole batch
    host = _host_search(ix, Q, k)
    np.testing.assert_array_equal(host[2], got[2])
    for i in range(nq):
        c = got[2][i]
        np.testing.assert_array_equal(host[0][i, :c], got[0][i, :c], err_msg=f"host ids q{i}")
        np.testing.assert_array_equal(host[1][i, :c], got[1][i, :c], err_msg=f"host dists q{i}")
    # transformed queries through the same graph form give the same results
    ref = Reference(path, "avx2")
    ref.set_nprobe(cfg["nprobe"])
    rows = np.linspace(0, nq - 1, 500).astype(np.int64)
    rids, rds, rcnt = ref.search_batch(prepared[rows], k, transformed=True, n_threads=os.cpu_count() or 1)
    _compare(got, rids, rds, rcnt, rows, "ivf2 sq8 pruned")
    # pruning off: every vector of the 32 visited clusters is scored exactly
    ix.set_pruning_aggressiveness(1e30)
    ref.set_pruning_aggressiveness(1e30)
    rows_u = rows[::5]
    got_u, _ = _graph_search(ix, Q[rows_u], k, forms=(128, 3, 0))
    rids, rds, rcnt = ref.search_batch(prepared[rows_u], k, transformed=True, n_threads=os.cpu_count() or 1)
    _compare(got_u, rids, rds, rcnt, range(len(rows_u)), "ivf2 sq8 unpruned")
    ref.close()


def test_ivf_f32_100k_d128_batch_vs_reference(built_oracle):
    if not _reference_available():
        pytest.skip("oracle/_ref not built (the reference sources were not present at build time)")
    from oracle.oracle import Reference
    from pdx_b200 import compiled
    cfg, path, Q, gt = _workload("ivf_f32_100k_d128")
    k, nq = cfg["k"], cfg["nq"]
    ix = compiled.load_index(path)
    ix.set_nprobe(cfg["nprobe"])
    prepared = ix.prepare_queries(Q)
    got, _ = _graph_search(ix, Q, k)
    ref = Reference(path, "avx2")
    ref.set_nprobe(cfg["nprobe"])
    rids, rds, rcnt = ref.search_batch(prepared, k, transformed=True, n_threads=os.cpu_count() or 1)
    _compare(got, rids, rds, rcnt, range(nq), "ivf f32")
    ref.close()
