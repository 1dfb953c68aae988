"""GPU tests of the native index build (pdxg_build, PDXIndex.build_index).

The clustering is the engine's own (BF16 tensor-core k-means), so cluster contents are not the
reference's. What the tests hold it to:
* the file is the reference's format and layout: every row id once, headers, capacities, the
  stored values equal to normalize(x) . M (FP32 rotation, rtol 1e-5 against FP64) or to its SQ8
  quantization with the global min / max parameters (at most 1 step where the rotation's
  rounding moves a value across a rounding boundary);
* rows sit in the cluster of their nearest stored centroid (BF16 assignment: at least 99 %
  agree with the FP32 nearest centroid), trees' L0 level holds every L1 centroid once;
* the same inputs and seed give the same file bytes;
* the search over a built index equals the oracle port's on the same file, bit for bit, and
  reaches the recall the Python builder's index reaches."""
import os
import tempfile

import numpy as np
import pytest

from pdx_b200 import compiled
from pdx_b200.builder import GaussianMixture, build_index, random_rotation
from pdx_b200.layout import max_capacity, quantization_params, read_index
from tests.helpers import assert_same, recall

pytestmark = pytest.mark.gpu
TYPES = ["pdx_f32", "pdx_u8", "pdx_tree_f32", "pdx_tree_u8"]


def _data(d, n, seed, norm=True):
    gm = GaussianMixture(d, 24, 0.35, seed=seed, unit_norm=norm)
    return gm.sample(n, 0), gm.sample(32, 1)


def _native(X, itype, nlist, nmeso, norm, seed, iters=10):
    ix = compiled.PDXIndex(itype, X.shape[1], seed=seed, num_clusters=nlist, num_meso_clusters=nmeso,
                           normalize=norm, kmeans_iters=iters)
    ix.build_index(X)
    return ix


def _saved(ix):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        ix.save(p)
        with open(p, "rb") as fh:
            return fh.read()


@pytest.fixture(scope="module")
def port_cls(built_oracle):
    from oracle.oracle import Port
    return Port


@pytest.mark.parametrize("itype", TYPES)
@pytest.mark.parametrize("d,norm", [(128, True), (200, False)])
def test_built_file_layout(itype, d, norm):
    X, _ = _data(d, 5000, 11 + d, norm)
    nlist, nmeso = 40, (6 if "tree" in itype else 0)
    ix = _native(X, itype, nlist, nmeso, norm, seed=3)
    f = read_index(_saved(ix))
    assert f.index_type == compiled.INDEX_TYPES[itype] and f.d == d and f.is_normalized == norm
    rot = random_rotation(d, 3)
    np.testing.assert_array_equal(f.rotation, rot)
    Xn = X.astype(np.float64)
    if norm:
        Xn = Xn / np.linalg.norm(Xn, axis=1, keepdims=True)
    R = Xn @ rot.astype(np.float64)
    ids = np.concatenate(f.l1.row_ids)
    assert np.array_equal(np.sort(ids), np.arange(len(X)))
    assert f.l1.nclusters == nlist
    for e, cap in zip(f.l1.embeddings, f.l1.caps()):
        assert cap == max_capacity(e.shape[0])
    for e, rid in zip(f.l1.embeddings, f.l1.row_ids):
        assert np.all(np.diff(rid.astype(np.int64)) > 0)  # row-id order inside a cluster
        if e.dtype == np.float32:
            np.testing.assert_allclose(e, R[rid], rtol=1e-5, atol=1e-5 * np.abs(R).max())
    if "u8" in itype:
        base, scale = quantization_params(R.astype(np.float32))
        assert abs(f.base - base) <= 1e-5 * max(1.0, abs(base))
        assert abs(f.scale - scale) <= 1e-4 * scale
        for e, rid in zip(f.l1.embeddings, f.l1.row_ids):
            ref = np.clip(np.round((R[rid] - f.base) * f.scale), 0, 255)
            diff = np.abs(e.astype(np.int64) - ref.astype(np.int64))
            assert diff.max() <= 1
    if "tree" in itype:
        assert f.l0.nclusters == nmeso
        l0ids = np.concatenate(f.l0.row_ids)
        assert np.array_equal(np.sort(l0ids), np.arange(nlist))
        cents = np.concatenate(f.l0.embeddings)
        if norm:  # spherical k-means: unit centroids
            np.testing.assert_allclose(np.linalg.norm(cents, axis=1), 1.0, rtol=1e-5)
    else:
        # rows in the cluster of their nearest stored centroid (BF16 assignment)
        C = f.l1.centroids.astype(np.float64)
        lab = np.empty(len(X), np.int64)
        for c, rid in enumerate(f.l1.row_ids):
            lab[rid] = c
        d2 = (C ** 2).sum(1)[None, :] - 2.0 * R @ C.T
        agree = np.mean(np.argmin(d2, axis=1) == lab)
        assert agree >= 0.99, f"assignment agreement {agree:.4f}"


@pytest.mark.parametrize("itype", ["pdx_u8", "pdx_tree_u8"])
def test_build_is_reproducible(itype):
    X, _ = _data(256, 4000, 5)
    a = _saved(_native(X, itype, 32, 5 if "tree" in itype else 0, True, seed=8))
    b = _saved(_native(X, itype, 32, 5 if "tree" in itype else 0, True, seed=8))
    assert a == b
    c = _saved(_native(X, itype, 32, 5 if "tree" in itype else 0, True, seed=9))
    assert a != c


@pytest.mark.parametrize("itype", TYPES)
def test_search_on_built_index_vs_port(port_cls, itype):
    X, Q = _data(384, 6000, 23)
    ix = _native(X, itype, 48, 7 if "tree" in itype else 0, True, seed=4)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        ix.save(p)
        port = port_cls(p)
        R = ix.prepare_queries(Q)
        for nprobe in (0, 6):
            ix.set_nprobe(nprobe)
            port.set_nprobe(nprobe)
            ids, ds, cnt = ix.search_batch(R, 10, transformed=True)
            for i in range(len(R)):
                pi, pd = port.search(R[i], 10, transformed=True)
                assert_same(ids[i, :cnt[i]], ds[i, :cnt[i]], pi, pd, ctx=f"{itype} nprobe={nprobe} q{i}")
        port.close()


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_tree_u8"])
def test_recall_matches_python_builder(itype):
    X, Q = _data(256, 20000, 31)
    nmeso = 10 if "tree" in itype else 0
    Xn = X / np.linalg.norm(X, axis=1, keepdims=True)
    Qn = Q / np.linalg.norm(Q, axis=1, keepdims=True)
    Xd, Qd = Xn.astype(np.float64), Qn.astype(np.float64)
    d2 = (Qd ** 2).sum(1)[:, None] - 2.0 * Qd @ Xd.T + (Xd ** 2).sum(1)[None, :]
    truth = np.argsort(d2, axis=1, kind="stable")[:, :10]
    ix = _native(X, itype, 100, nmeso, True, seed=2)
    ix.set_nprobe(10)
    ids, _, cnt = ix.search_batch(Q, 10)
    rn = np.mean([recall(ids[i, :cnt[i]], truth[i].tolist(), 10) for i in range(len(Q))])
    f = build_index(X, itype, num_clusters=100, num_meso_clusters=nmeso, normalize=True, seed=2)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ref = compiled.load_index(p)
        ref.set_nprobe(10)
        rids, _, rcnt = ref.search_batch(Q, 10)
    rp = np.mean([recall(rids[i, :rcnt[i]], truth[i].tolist(), 10) for i in range(len(Q))])
    assert rn >= rp - 0.05, f"native build recall {rn:.3f} vs Python builder {rp:.3f}"
    assert rn >= 0.8


def test_unsupported_dims_use_the_torch_builder():
    X, Q = _data(100, 2000, 3)  # d % 8 != 0: the native build answers UNSUPPORTED
    assert compiled.build_handle(X, "pdx_u8", random_rotation(100, 1), 16) is None
    ix = _native(X, "pdx_u8", 16, 0, True, seed=1)
    assert ix.get_num_clusters() == 16 and ix.get_num_embeddings() == len(X)
    ids, _, cnt = ix.search_batch(Q, 5)
    assert (cnt == 5).all()


def test_build_rejects_bad_arguments():
    X, _ = _data(64, 300, 2)
    with pytest.raises(ValueError):
        compiled.build_handle(X, "pdx_f32", random_rotation(64, 1), num_clusters=400)
    with pytest.raises(ValueError):
        compiled.build_handle(X, "pdx_tree_f32", random_rotation(64, 1), num_clusters=20, num_meso_clusters=20)
    with pytest.raises(ValueError):
        compiled.build_handle(X, "pdx_f32", random_rotation(32, 1))


# --- the reference's tests/test_index_properties.cpp on indexes this engine builds ---

def _props_data(n, d=128, seed=42):
    gm = GaussianMixture(d, 20, 0.4, seed=seed, unit_norm=False)
    return gm.sample(n, 0), gm.sample(50, 1)


@pytest.mark.parametrize("itype", TYPES)
def test_properties_cluster_ids_sizes_dims_memory(itype):
    """ClusterRowIdsCoverAllPoints, ClusterSizeMatchesRowIdCount, GetNumDimensionsMatchesInput,
    InMemorySizeIsPositive (test_index_properties.cpp:18-66)."""
    X, _ = _props_data(3000)
    ix = compiled.PDXIndex(itype, 128, normalize=True)
    ix.build_index(X)
    ids = np.concatenate([ix.get_cluster_row_ids(c) for c in range(ix.get_num_clusters())])
    assert np.array_equal(np.sort(ids), np.arange(len(X)))
    for c in range(ix.get_num_clusters()):
        assert ix.get_cluster_size(c) == len(ix.get_cluster_row_ids(c))
    assert ix.get_num_dimensions() == 128
    assert ix.get_in_memory_size_in_bytes() > 0


@pytest.mark.parametrize("itype", TYPES)
def test_properties_knn_larger_than_data(itype):
    """KnnLargerThanDataReturnsAvailable (test_index_properties.cpp:69-82): 5 points, k = 100."""
    X, Q = _props_data(5)
    ix = compiled.PDXIndex(itype, 128, normalize=True)
    ix.build_index(X)
    ix.set_nprobe(ix.get_num_clusters())
    ids, _ = ix.search(Q[0], 100)
    assert 0 < len(ids) <= 5


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8"])
def test_properties_num_clusters_and_full_nprobe(itype):
    """NumClustersMatchesConfig (test_index_properties.cpp:84-140): the requested cluster count,
    and nprobe = n, n + 1 and 0 give identical results."""
    X, Q = _props_data(3000)
    for requested in (10, 50, 100):
        ix = compiled.PDXIndex(itype, 128, num_clusters=requested, normalize=True)
        ix.build_index(X)
        assert ix.get_num_clusters() == requested
        outs = []
        for nprobe in (requested, requested + 1, 0):
            ix.set_nprobe(nprobe)
            outs.append(ix.search_batch(Q, 10))
        for o in outs[1:]:
            for a, b in zip(outs[0], o):
                np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8"])
def test_edge_single_and_two_points(itype):
    """SinglePointIndex, TwoPointIndex (test_index_properties.cpp:151-205)."""
    X, _ = _props_data(2, seed=3)
    one = compiled.PDXIndex(itype, 128, num_clusters=1, normalize=True)
    one.build_index(X[:1])
    assert one.get_num_clusters() == 1 and one.get_cluster_size(0) == 1
    one.set_nprobe(0)
    ids, _ = one.search(X[0], 10)
    assert ids.tolist() == [0]
    two = compiled.PDXIndex(itype, 128, num_clusters=1, normalize=True)
    two.build_index(X)
    two.set_nprobe(0)
    ids, ds = two.search(X[0], 2)
    assert len(ids) == 2 and ds[0] <= ds[1] + 1e-6


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8"])
def test_edge_num_clusters_exceeds_points(itype):
    """NumClustersExceedsNumPointsThrows (test_index_properties.cpp:207-230)."""
    X, _ = _props_data(10)
    ix = compiled.PDXIndex(itype, 128, num_clusters=100, normalize=True)
    with pytest.raises(ValueError):
        ix.build_index(X)
