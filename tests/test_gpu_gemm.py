"""Tensor-core (tcgen05) query rotation: the TF32x3 GEMM against an FP64 rotation of the same
queries and against the FP32 SIMT GEMM, and the searches built on it.

Tolerance: the reference rotates with an FP32 BLAS sgemm (adsampling.hpp:192-246), so rotated
queries are compared at FP32 rounding level: |y - y64| <= 2e-6 * max|y64| per element, for the
TF32x3 tensor-core GEMM (accumulated in FP32 registers) and for the FP32 SIMT GEMM alike."""
import os
import tempfile

import numpy as np
import pytest

from pdx_b200 import compiled
from pdx_b200.builder import GaussianMixture, build_index
from tests.helpers import recall

pytestmark = pytest.mark.gpu


def _index(itype, d, n=3000, norm=True, seed=3):
    gm = GaussianMixture(d, 12, 0.4, seed=seed + d, unit_norm=False)
    X = gm.sample(n, 0)
    Q = gm.sample(300, 1)
    f = build_index(X, itype, num_clusters=16, num_meso_clusters=4 if "tree" in itype else 0,
                    normalize=norm, seed=seed)
    return f, Q


def _fp64_rotation(f, Q, normalize):
    q = Q.astype(np.float64)
    if normalize:
        n = np.linalg.norm(q, axis=1, keepdims=True)
        n[n == 0] = 1.0
        q = q / n
    return q @ f.rotation.astype(np.float64)


@pytest.mark.parametrize("d,norm", [(1024, True), (1024, False), (768, True), (516, False)])
def test_tensor_core_rotation_vs_fp64(d, norm):
    f, Q = _index("pdx_f32", d, norm=norm)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        assert ix.rotation_uses_tensor_cores()
        ref = _fp64_rotation(f, Q, norm)
        tc = ix.prepare_queries(Q)
        scale = np.abs(ref).max()
        err = np.abs(tc - ref).max()
        ix.set_rotation_mode(1)
        assert not ix.rotation_uses_tensor_cores()
        simt = ix.prepare_queries(Q)
        err_simt = np.abs(simt - ref).max()
        print(f"d={d}: tensor-core error {err:.3g}, SIMT error {err_simt:.3g}, scale {scale:.3g}")
        assert err <= 2e-6 * scale, f"tensor-core rotation error {err:.3g} (scale {scale:.3g})"
        assert err_simt <= 2e-6 * scale
        # batch edge sizes: one query, a partial 128-row tile, several tiles
        ix.set_rotation_mode(0)
        for nq in (1, 127, 129, 300):
            part = ix.prepare_queries(Q[:nq])
            assert np.abs(part - ref[:nq]).max() <= 2e-6 * scale


@pytest.mark.parametrize("d", [130, 256, 514])
def test_rotation_uses_simt_below_512_or_unpitched(d):
    """d < 512 (SIMT is the more accurate there) or a row pitch that is not a multiple of 16
    bytes (d = 514) keep the FP32 SIMT GEMM."""
    f, Q = _index("pdx_f32", d)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        assert not ix.rotation_uses_tensor_cores()
        ref = _fp64_rotation(f, Q, True)
        assert np.abs(ix.prepare_queries(Q) - ref).max() <= 2e-6 * np.abs(ref).max()


@pytest.mark.parametrize("itype", ["pdx_u8", "pdx_tree_u8", "pdx_f32"])
def test_search_with_tensor_core_rotation(itype):
    """Raw-query search with the tensor-core rotation against the same search after the FP32
    SIMT rotation: the rotated queries differ at FP32 rounding level only, so the results agree
    up to quantization ties (recall >= 0.95 per query, equal distances on common ids)."""
    f, Q = _index(itype, 768)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
        assert ix.rotation_uses_tensor_cores()
        ix.set_nprobe(6)
        a_ids, a_d, a_c = ix.search_batch(Q, 10)
        ix.set_rotation_mode(1)
        b_ids, b_d, b_c = ix.search_batch(Q, 10)
        same = 0
        for i in range(len(Q)):
            assert recall(a_ids[i, :a_c[i]], b_ids[i, :b_c[i]], 10) >= 0.9
            same += int(np.array_equal(a_ids[i, :a_c[i]], b_ids[i, :b_c[i]]))
        print(f"{itype}: {same} of {len(Q)} result lists identical")
        assert same >= 0.95 * len(Q)
