"""GPU parity tests: the CUDA search path (through the C ABI) against the reference's own results
(golden fixtures) and against the oracle port on freshly generated indexes.

Parity bar: on the same prepared (rotated) queries, distances are bit-identical and ids equal
(as sets inside groups of tied distances) for every index type -- U8 and F32, pruning on and
off, plain, fixed-order and filtered search. Raw queries additionally go through the GPU
rotation, compared with the reference's BLAS rotation at FP32 tolerance (rtol 1e-5)."""
import os
import tempfile

import numpy as np
import pytest

from pdx_b200 import compiled
from pdx_b200.builder import GaussianMixture, build_index
from pdx_b200.layout import IndexFile, Level, max_capacity, quantization_params, quantize
from tests.helpers import assert_same, golden_cases, load_golden, recall

pytestmark = pytest.mark.gpu
CASES = [c["name"] for c in golden_cases()]


@pytest.fixture(scope="module")
def port_cls(built_oracle):
    from oracle.oracle import Port
    return Port


@pytest.mark.parametrize("name", CASES)
def test_golden_plain(name):
    path, q, r, exp = load_golden(name)
    ix = compiled.load_index(path)
    ix.set_nprobe(exp["nprobe"])
    ids, ds, cnt = ix.search_batch(r, exp["k"], transformed=True)
    for i in range(len(r)):
        assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], exp["plain_ids"][i], exp["plain_dists"][i],
                    ctx=f"{name} q{i}")


@pytest.mark.parametrize("name", CASES)
def test_golden_order_filtered_unpruned(name):
    path, q, r, exp = load_golden(name)
    ix = compiled.load_index(path)
    k = exp["k"]
    ix.set_nprobe(exp["nprobe"])
    ids, ds, cnt = ix.search_with_order(r, k, np.array(exp["order"], np.uint32), transformed=True)
    for i in range(len(r)):
        assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], exp["order_ids"][i], exp["order_dists"][i],
                    ctx=f"{name} order q{i}")
    fids, fds, fcnt = ix.filtered_search_batch(r, k, [np.array(f, np.uint64) for f in exp["filters"]],
                                               transformed=True)
    for i in range(len(r)):
        assert_same(fids[i, :fcnt[i]], fds[i, :fcnt[i]], exp["filt_ids"][i], exp["filt_dists"][i],
                    ctx=f"{name} filtered q{i}")
    ix.set_pruning_aggressiveness(1e30)
    eids, eds, ecnt = ix.search_batch(r, k, transformed=True)
    for i in range(len(r)):
        assert_same(eids[i, :ecnt[i]], eds[i, :ecnt[i]], exp["exh_ids"][i], exp["exh_dists"][i],
                    ctx=f"{name} unpruned q{i}")


@pytest.mark.parametrize("name", CASES)
def test_golden_raw_queries(name):
    path, q, r, exp = load_golden(name)
    ix = compiled.load_index(path)
    prepared = ix.prepare_queries(q)
    np.testing.assert_allclose(prepared, r, rtol=1e-5, atol=1e-6)
    ix.set_nprobe(exp["nprobe"])
    ids, ds, cnt = ix.search_batch(q, exp["k"])
    for i in range(len(q)):
        assert recall(ids[i, :cnt[i]], exp["raw_ids"][i], exp["k"]) >= 0.9
        common = set(ids[i, :cnt[i]].tolist()) & set(exp["raw_ids"][i])
        for rid in common:
            a = ds[i, list(ids[i, :cnt[i]]).index(rid)]
            b = exp["raw_dists"][i][exp["raw_ids"][i].index(rid)]
            assert abs(a - b) <= 1e-4 * max(abs(b), 1e-3) + 1e-5


def _fresh(itype, d, n, nlist, nmeso=0, norm=False, seed=0, sigma=0.5, comps=16):
    gm = GaussianMixture(d, comps, sigma, seed=seed + d, unit_norm=norm)
    X = gm.sample(n, 0)
    Q = gm.sample(24, 1)
    f = build_index(X, itype, num_clusters=nlist, num_meso_clusters=nmeso, normalize=norm, seed=seed)
    return f, X, Q


def _compare_with_port(port_cls, f, Q, k, nprobes, threads=(256,)):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        port = port_cls(p)
        ix = compiled.load_index(p)
        R = ix.prepare_queries(Q)
        for nprobe in nprobes:
            ix.set_nprobe(nprobe)
            port.set_nprobe(nprobe)
            for t in threads:
                ix.set_threads_per_query(t)
                ids, ds, cnt = ix.search_batch(R, k, transformed=True)
                for i in range(len(R)):
                    pi, pd = port.search(R[i], k, transformed=True)
                    assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd,
                                ctx=f"type={f.index_type} d={f.d} k={k} nprobe={nprobe} T={t} q{i}")
        port.close()


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8", "pdx_tree_f32", "pdx_tree_u8"])
@pytest.mark.parametrize("d", [3, 5, 63, 65, 127, 129, 200, 384])
def test_fresh_vs_port_dims(port_cls, itype, d):
    f, X, Q = _fresh(itype, d, 1500, 12, 3, norm=(d % 2 == 0), seed=1)
    _compare_with_port(port_cls, f, Q, 10, (0, 4))


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8", "pdx_tree_f32", "pdx_tree_u8"])
def test_fresh_vs_port_k_and_threads(port_cls, itype):
    f, X, Q = _fresh(itype, 160, 3000, 20, 4, norm=True, seed=4)
    for k in (1, 7, 100):
        _compare_with_port(port_cls, f, Q, k, (0, 1, 6, 25), threads=(64, 128, 256, 512))


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8", "pdx_tree_u8"])
def test_large_d(port_cls, itype):
    f, X, Q = _fresh(itype, 1024, 3000, 16, 4, norm=True, seed=7, sigma=0.25)
    _compare_with_port(port_cls, f, Q, 20, (5,))


def _manual_index(itype, d, sizes, seed=0):
    """Index with exactly the given cluster sizes (0 allowed) from random data."""
    rng = np.random.default_rng(seed)
    n = sum(sizes)
    X = rng.standard_normal((max(n, 1), d)).astype(np.float32)[:n]
    rot = np.linalg.qr(rng.standard_normal((d, d)))[0].astype(np.float32)
    R = (X.astype(np.float64) @ rot.astype(np.float64)).astype(np.float32)
    is_u8 = itype in ("pdx_u8", "pdx_tree_u8")
    base, scale = quantization_params(R) if n else (0.0, 1.0)
    stored = quantize(R, base, scale) if is_u8 else R
    embs, ids, cents = [], [], []
    perm = rng.permutation(n).astype(np.uint32)
    s = 0
    for m in sizes:
        sel = perm[s:s + m]
        s += m
        embs.append(np.ascontiguousarray(stored[sel]) if m else np.zeros((0, d), stored.dtype))
        ids.append(sel)
        cents.append(R[sel].mean(0) if m else rng.standard_normal(d).astype(np.float32))
    cents = np.array(cents, np.float32)
    l1 = Level(embs, ids, cents)
    itype_id = {"pdx_f32": 0, "pdx_u8": 1, "pdx_tree_f32": 2, "pdx_tree_u8": 3}[itype]
    l0 = None
    if itype_id >= 2:
        half = len(sizes) // 2
        groups = [np.arange(half, dtype=np.uint32), np.arange(half, len(sizes), dtype=np.uint32)]
        l0 = Level([cents[g] for g in groups], groups, np.array([cents[g].mean(0) for g in groups], np.float32))
    return IndexFile(itype_id, rot, d, l1, l0, False, float(base), float(scale)), X


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8", "pdx_tree_f32", "pdx_tree_u8"])
def test_edge_cluster_sizes(port_cls, itype):
    f, X = _manual_index(itype, 72, [0, 1, 31, 33, 0, 5, 64, 257, 2, 0])
    Q = np.random.default_rng(5).standard_normal((16, 72)).astype(np.float32)
    _compare_with_port(port_cls, f, Q, 10, (0, 3, 11))
    _compare_with_port(port_cls, f, Q, 500, (0,))  # k larger than the index


@pytest.mark.parametrize("itype", ["pdx_u8", "pdx_tree_f32", "pdx_f32"])
def test_dct_rotation_files(port_cls, itype):
    """FFTW-built files (1 x d sign vector + orthonormal DCT-II): the engine rotates as the
    reference's DCT does (FP32 rounding level against scipy's DCT), searches exactly like the
    oracle on the same prepared queries, and saves the file back byte for byte."""
    from tests.helpers import dct_index, dct_rotate
    nmeso = 6 if "tree" in itype else 0
    f, Q, signs = dct_index(itype, 512, 6000, 40, nmeso, seed=7)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "dct.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        R = ix.prepare_queries(Q)
        np.testing.assert_allclose(R, dct_rotate(Q, signs), rtol=0, atol=2e-6)
        port = port_cls(p)
        ix.set_nprobe(6)
        port.set_nprobe(6)
        ids, ds, cnt = ix.search_batch(R, 10, transformed=True)
        for i in range(len(R)):
            pi, pd = port.search(R[i], 10, transformed=True)
            assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd, ctx=f"dct {itype} q{i}")
        ids2, _, cnt2 = ix.search_batch(Q, 10)
        hits = sum(len(set(ids2[i, :cnt2[i]].tolist()) & set(port.search(Q[i], 10)[0].tolist()))
                   for i in range(len(Q)))
        assert hits >= 0.95 * 10 * len(Q)
        port.close()
        out = os.path.join(td, "saved.pdx")
        ix.save(out)
        assert open(out, "rb").read() == open(p, "rb").read()


def test_save_roundtrip_bytes():
    for name in CASES:
        path, *_ = load_golden(name)
        ix = compiled.load_index(path)
        with tempfile.TemporaryDirectory() as td:
            out = os.path.join(td, "saved.pdx")
            ix.save(out)
            assert open(out, "rb").read() == open(path, "rb").read(), name


def test_getters_match_file():
    from pdx_b200.layout import read_index
    for name in CASES:
        path, *_ = load_golden(name)
        f = read_index(open(path, "rb").read())
        ix = compiled.load_index(path)
        assert ix.get_num_dimensions() == f.d
        assert ix.get_num_clusters() == f.l1.nclusters
        for c in range(f.l1.nclusters):
            assert ix.get_cluster_size(c) == f.l1.embeddings[c].shape[0]
            np.testing.assert_array_equal(ix.get_cluster_row_ids(c), f.l1.row_ids[c])
        assert ix.get_in_memory_size_in_bytes() > 0


def test_batch_equals_single_queries():
    path, q, r, exp = load_golden("tree_u8_d256")
    ix = compiled.load_index(path)
    ix.set_nprobe(exp["nprobe"])
    ids, ds, cnt = ix.search_batch(q, exp["k"])
    for i in range(len(q)):
        si, sd = ix.search(q[i], exp["k"])
        np.testing.assert_array_equal(si, ids[i, :cnt[i]])
        np.testing.assert_array_equal(sd, ds[i, :cnt[i]])


def test_filtered_mixed_batch(port_cls):
    f, X, Q = _fresh("pdx_u8", 96, 4000, 24, seed=9)
    rng = np.random.default_rng(3)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        port = port_cls(p)
        ix = compiled.load_index(p)
        R = ix.prepare_queries(Q)
        lists = []
        for i in range(len(Q)):
            if i % 3 == 0:
                lists.append(None)
            else:
                sel = float(np.exp(rng.uniform(np.log(0.001), np.log(0.5))))
                lists.append(np.sort(rng.choice(4000, max(1, int(4000 * sel)), replace=False)).astype(np.uint64))
        for nprobe in (0, 5):
            ix.set_nprobe(nprobe)
            port.set_nprobe(nprobe)
            ids, ds, cnt = ix.filtered_search_batch(R, 10, lists, transformed=True)
            for i in range(len(Q)):
                if lists[i] is None:
                    pi, pd = port.search(R[i], 10, transformed=True)
                else:
                    pi, pd = port.filtered_search(R[i], 10, lists[i], transformed=True)
                    assert set(ids[i, :cnt[i]].tolist()) <= set(lists[i].tolist())
                assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd, ctx=f"filtered nprobe={nprobe} q{i}")
        port.close()


def test_filtered_edge_cases():
    path, q, r, exp = load_golden("f32_d64")
    ix = compiled.load_index(path)
    ix.set_nprobe(0)
    ids, ds = ix.filtered_search(q[0], 10, np.array([], np.uint64))
    assert len(ids) == 0
    ids, ds = ix.filtered_search(q[0], 10, np.array([17], np.uint64))
    assert ids.tolist() == [17]
    all_rows = np.arange(1200, dtype=np.uint64)
    a = ix.filtered_search(q[1], 10, all_rows)
    b = ix.search(q[1], 10)
    np.testing.assert_array_equal(a[1], b[1])


def _tiled_ok(d):
    """The tiled top level needs d and the vertical dims to be multiples of 4."""
    from pdx_b200.layout import dimension_split
    h, v = dimension_split(d)
    return d % 4 == 0 and v % 4 == 0


@pytest.mark.parametrize("itype", ["pdx_tree_f32", "pdx_tree_u8"])
@pytest.mark.parametrize("d", [65, 130, 384, 512, 1024])
def test_tree_top_level_modes(port_cls, itype, d):
    """Every form of the top level -- inside the search CTA (1), per-query CTAs (2) and tiled
    probe + exact partials + replay (3) -- gives the oracle's results."""
    gm = GaussianMixture(d, 20, 0.5, seed=d + 3, unit_norm=True)
    X = gm.sample(4000, 0)
    Q = gm.sample(80, 1)
    f = build_index(X, itype, num_clusters=40, num_meso_clusters=7, normalize=True, seed=3)
    modes = (1, 2, 3) if _tiled_ok(d) else (1, 2)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        port = port_cls(p)
        ix = compiled.load_index(p)
        R = ix.prepare_queries(Q)
        if not _tiled_ok(d):
            ix.set_top_level_mode(3)
            with pytest.raises(RuntimeError):
                ix.search_batch(R, 10, transformed=True)
        for nprobe in (0, 3, 12, 39):
            ix.set_nprobe(nprobe)
            port.set_nprobe(nprobe)
            res = {}
            for mode in modes:
                ix.set_top_level_mode(mode)
                res[mode] = ix.search_batch(R, 10, transformed=True)
            for i in range(len(R)):
                pi, pd = port.search(R[i], 10, transformed=True)
                for mode in modes:
                    ids, ds, cnt = res[mode]
                    assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd,
                                ctx=f"{itype} d={d} nprobe={nprobe} mode={mode} q{i}")
        port.close()


def test_tree_top_level_tiled_stats_match():
    """The tiled top level replays the per-query search's decisions: the same index bytes and
    clusters are accounted for as by the per-query kernel."""
    import torch
    gm = GaussianMixture(256, 30, 0.4, seed=11, unit_norm=True)
    X = gm.sample(6000, 0)
    Q = gm.sample(300, 1)
    f = build_index(X, "pdx_tree_u8", num_clusters=60, num_meso_clusters=8, normalize=True, seed=5)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        ix.set_nprobe(10)
        R = torch.from_numpy(ix.prepare_queries(Q)).cuda()
        nq, k = len(Q), 10
        ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
        ds = torch.empty((nq, k), dtype=torch.float32, device="cuda")
        cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
        out = {}
        for mode in (2, 3):
            ix.set_top_level_mode(mode)
            ix.search_device(R.data_ptr(), nq, k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(),
                             stream=torch.cuda.current_stream().cuda_stream, transformed=True, stats=True)
            torch.cuda.synchronize()
            out[mode] = (ix.last_stats(), ids.cpu().numpy().copy(), ds.cpu().numpy().copy())
        assert out[2][0]["bytes_by_phase"] == out[3][0]["bytes_by_phase"]
        assert out[2][0]["clusters_visited"] == out[3][0]["clusters_visited"]
        np.testing.assert_array_equal(out[2][1], out[3][1])
        np.testing.assert_array_equal(out[2][2], out[3][2])


@pytest.mark.parametrize("top_mode", [2, 3])
def test_batched_start_matches_scan_start(port_cls, top_mode):
    """The batched first-cluster Start (exact U8 distances computed once per cluster and query
    group) gives the same results, and the same algorithmic byte count, as the scan's own
    Start, and the oracle's results; k above the first cluster's size continues with the
    scan's Start on the next clusters."""
    import torch
    gm = GaussianMixture(256, 30, 0.4, seed=13, unit_norm=True)
    X = gm.sample(8000, 0)
    Q = gm.sample(200, 1)
    f = build_index(X, "pdx_tree_u8", num_clusters=64, num_meso_clusters=8, normalize=True, seed=6)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        port = port_cls(p)
        ix = compiled.load_index(p)
        ix.set_top_level_mode(top_mode)
        ix.set_scan_mode(1)  # the per-query scan in both Start forms (tests/test_gpu_scan.py covers the other)
        R = ix.prepare_queries(Q)
        Rd = torch.from_numpy(R).cuda()
        nq = len(Q)
        for nprobe, k in ((6, 10), (20, 500)):
            ix.set_nprobe(nprobe)
            port.set_nprobe(nprobe)
            ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
            ds = torch.empty((nq, k), dtype=torch.float32, device="cuda")
            cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
            out = {}
            for mode in (1, 0):
                ix.set_start_mode(mode)
                ix.search_device(Rd.data_ptr(), nq, k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(),
                                 stream=torch.cuda.current_stream().cuda_stream, transformed=True, stats=True)
                torch.cuda.synchronize()
                out[mode] = (ix.last_stats(), ix.last_launch_count(), ids.cpu().numpy().copy(),
                             ds.cpu().numpy().copy(), cnt.cpu().numpy().copy())
            assert out[0][1] == out[1][1] + 3  # count, plan and distance kernels ran
            assert out[0][0]["bytes_by_phase"] == out[1][0]["bytes_by_phase"]
            for j in (2, 3, 4):
                np.testing.assert_array_equal(out[0][j], out[1][j])
            gi, gd, gc = out[0][2].view(np.uint32), out[0][3], out[0][4]
            for i in range(0, nq, 7):
                pi, pd = port.search(R[i], k, transformed=True)
                assert_same(gi[i, :gc[i]], gd[i, :gc[i]], pi, pd, ctx=f"top_mode={top_mode} k={k} q{i}")
        port.close()


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8"])
def test_flat_probe_ahead_matches_port(port_cls, itype):
    """Batches of >= 32 queries on flat indexes probe ahead of the scan (probe_exact_kernel);
    the visit order and the results are the oracle's."""
    gm = GaussianMixture(192, 25, 0.4, seed=23, unit_norm=True)
    X = gm.sample(5000, 0)
    Q = gm.sample(64, 1)
    f = build_index(X, itype, num_clusters=70, normalize=True, seed=12)
    _compare_with_port(port_cls, f, Q, 10, (0, 3, 17), threads=(64, 128))


@pytest.mark.parametrize("itype", ["pdx_tree_u8", "pdx_tree_f32", "pdx_u8"])
def test_host_pipelined_equals_device_search(itype):
    """Host-buffer batches of >= 4096 queries upload in chunks overlapped with the per-chunk
    rotation and top level; results equal the device-buffer search of the whole batch."""
    import torch
    gm = GaussianMixture(256, 30, 0.4, seed=17, unit_norm=True)
    X = gm.sample(6000, 0)
    Q = gm.sample(5000, 1)
    nmeso = 8 if "tree" in itype else 0
    f = build_index(X, itype, num_clusters=60, num_meso_clusters=nmeso, normalize=True, seed=8)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        ix.set_nprobe(9)
        k = 10
        hi, hd, hc = ix.search_batch(Q, k)
        q = torch.from_numpy(Q).cuda()
        ids = torch.empty((len(Q), k), dtype=torch.int32, device="cuda")
        ds = torch.empty((len(Q), k), dtype=torch.float32, device="cuda")
        cnt = torch.empty(len(Q), dtype=torch.int32, device="cuda")
        ix.search_device(q.data_ptr(), len(Q), k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(),
                         stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(hc, cnt.cpu().numpy().view(np.uint32))
        np.testing.assert_array_equal(hi, ids.cpu().numpy().view(np.uint32))
        np.testing.assert_array_equal(hd, ds.cpu().numpy())


def test_tree_top_level_batched_edge_sizes(port_cls):
    for itype in ("pdx_tree_f32", "pdx_tree_u8"):
        f, X = _manual_index(itype, 200, [0, 1, 31, 33, 0, 5, 64, 257, 2, 0, 90, 7])
        Q = np.random.default_rng(5).standard_normal((40, 200)).astype(np.float32)
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "ix.pdx")
            f.save(p)
            port = port_cls(p)
            ix = compiled.load_index(p)
            R = ix.prepare_queries(Q)
            for mode in (2, 3):
                ix.set_top_level_mode(mode)
                for nprobe, k in ((0, 10), (2, 10), (5, 500)):
                    ix.set_nprobe(nprobe)
                    port.set_nprobe(nprobe)
                    ids, ds, cnt = ix.search_batch(R, k, transformed=True)
                    for i in range(len(R)):
                        pi, pd = port.search(R[i], k, transformed=True)
                        assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd,
                                    ctx=f"{itype} mode={mode} nprobe={nprobe} k={k} q{i}")
            port.close()


@pytest.mark.parametrize("d", [100, 512, 1024])
def test_few_row_rotation_against_fp64(d):
    """Batches of up to 8 rows rotate with the FP32 GEMV (one CTA per 32 columns, fixed order);
    larger ones with the tensor-core or SIMT GEMM. Every size agrees with the FP64 rotation of the
    normalized rows at FP32 rounding level (rtol 1e-5)."""
    gm = GaussianMixture(d, 8, 0.4, seed=d, unit_norm=False)
    X = gm.sample(1200, 0)
    f = build_index(X, "pdx_tree_u8", num_clusters=12, num_meso_clusters=3, normalize=True, seed=2)
    Q = gm.sample(20, 1)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        rot = np.asarray(f.rotation, np.float64)
        Qn = Q.astype(np.float64) / np.linalg.norm(Q.astype(np.float64), axis=1, keepdims=True)
        R64 = Qn @ rot
        for m in (1, 3, 8, 9, 20):
            got = ix.prepare_queries(Q[:m])
            np.testing.assert_allclose(got, R64[:m], rtol=1e-5, atol=1e-6, err_msg=f"{m} rows")
        # a single raw query searches like its prepared form within the rotation's rounding
        ix.set_nprobe(0)
        a, _, ca = ix.search_batch(Q[:1], 10)
        b, _, cb = ix.search_batch(ix.prepare_queries(Q[:1]), 10, transformed=True)
        assert ca[0] == cb[0] and set(a[0, :ca[0]].tolist()) == set(b[0, :cb[0]].tolist())
