"""GPU tests of the reduced-precision centroid probe (probe modes 1 and 2): BF16 tensor-core
rotation and centroid scores (FP8-E4M3 scores in mode 2), the nprobe list widened by 10 %, and
an FP32 rescore of the candidates with the reference's probe arithmetic.

Bars: with every centroid probed the widened list is the whole level, so the visit order and
the results equal the reference probe's bit for bit on the same prepared queries; with a partial
probe, the probe set against the FP64 nearest centroids and the search results against the
exact form stay within the tolerances written in each test."""
import os
import tempfile

import numpy as np
import pytest

from pdx_b200 import compiled
from pdx_b200.builder import GaussianMixture, build_index

pytestmark = pytest.mark.gpu


def _index(itype, d, n, nlist, nmeso, seed, sigma=0.3):
    gm = GaussianMixture(d, 40, sigma, seed=seed, unit_norm=True)
    X = gm.sample(n, 0)
    Q = gm.sample(256, 1)
    f = build_index(X, itype, num_clusters=nlist, num_meso_clusters=nmeso, normalize=True, seed=seed)
    return f, X, Q


def _device_search(ix, Q, k, transformed):
    import torch
    nq = len(Q)
    q = torch.from_numpy(np.ascontiguousarray(Q, np.float32)).cuda()
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    ds = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
    ix.search_device(q.data_ptr(), nq, k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(),
                     stream=torch.cuda.current_stream().cuda_stream, transformed=transformed)
    torch.cuda.synchronize()
    return ids.cpu().numpy().view(np.uint32), ds.cpu().numpy(), cnt.cpu().numpy()


def _fp64_nearest(R, C, m):
    d2 = (R.astype(np.float64) ** 2).sum(1)[:, None] - 2.0 * R.astype(np.float64) @ C.astype(np.float64).T \
        + (C.astype(np.float64) ** 2).sum(1)[None, :]
    return np.argsort(d2, axis=1, kind="stable")[:, :m]


def _l1_centroids(f):
    return np.asarray(f.l1.centroids, np.float32)


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8"])
def test_full_probe_equals_reference_probe(itype):
    """nprobe = 0: every centroid is a candidate and rescored in FP32, so the order and the
    results are the reference probe's, bit for bit."""
    f, X, Q = _index(itype, 256, 6000, 48, 0, seed=21)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        R = ix.prepare_queries(Q)
        ix.set_nprobe(0)
        ref = _device_search(ix, R, 10, True)
        for mode in (1, 2):
            ix.set_probe_mode(mode)
            got = _device_search(ix, R, 10, True)
            for a, b in zip(ref, got):
                np.testing.assert_array_equal(a, b)
            orders, counts = ix.last_visit_orders(len(R), 48)
            assert (counts == 48).all()
        ix.set_probe_mode(0)


@pytest.mark.parametrize("mode,max_mismatch", [(1, 0.02), (2, 0.06)])
@pytest.mark.parametrize("itype", ["pdx_u8", "pdx_tree_u8", "pdx_f32"])
def test_partial_probe_against_fp64(itype, mode, max_mismatch):
    """Probe-set error against the FP64 nearest centroids of the FP64-rotated queries, and the
    overlap of the results with the exact form's."""
    nmeso = 8 if "tree" in itype else 0
    f, X, Q = _index(itype, 512, 12000, 96, nmeso, seed=5 + mode)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        nprobe = 10
        ix.set_nprobe(nprobe)
        exact = ix.search_batch(Q, 10)
        ix.set_probe_mode(mode)
        got = _device_search(ix, Q, 10, False)
        orders, counts = ix.last_visit_orders(len(Q), nprobe)
        assert (counts == nprobe).all()
        rot = np.asarray(f.rotation, np.float64)
        Qn = Q.astype(np.float64) / np.linalg.norm(Q.astype(np.float64), axis=1, keepdims=True)
        R64 = Qn @ rot
        truth = _fp64_nearest(R64, _l1_centroids(f), nprobe)
        miss = 1.0 - np.mean([len(set(orders[i].tolist()) & set(truth[i].tolist())) / nprobe
                              for i in range(len(Q))])
        assert miss <= max_mismatch, f"probe-set mismatch {miss:.4f}"
        ids_e, _, cnt_e = exact
        ids_g, _, cnt_g = got
        overlap = np.mean([len(set(ids_e[i, :cnt_e[i]].tolist()) & set(ids_g[i, :cnt_g[i]].tolist()))
                           / max(1, cnt_e[i]) for i in range(len(Q))])
        assert overlap >= 0.9, f"result overlap with the exact form {overlap:.4f}"
        ix.set_probe_mode(0)


def test_probe_mode_rejects_unsupported_dims():
    f, X, Q = _index("pdx_f32", 72, 2000, 16, 0, seed=3)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        with pytest.raises(RuntimeError):
            ix.set_probe_mode(1)
        with pytest.raises(ValueError):
            ix.set_probe_mode(3)
