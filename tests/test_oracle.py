"""CPU tests of the oracle: the C restatement (oracle/pdx_port.c) is pinned bit-for-bit against
the reference's own outputs stored in tests/golden/, and -- where the reference build exists --
against the reference on freshly generated indexes."""
import os
import tempfile

import numpy as np
import pytest

from pdx_b200.builder import GaussianMixture, build_index
from pdx_b200.layout import adsampling_ratio, dimension_split, read_index
from tests.helpers import assert_same, golden_cases, load_golden, recall

CASES = [c["name"] for c in golden_cases()]


def test_dimension_split_known_answers():
    # the static_asserts of common.hpp:161-189
    known = {4: (0, 4), 33: (0, 33), 64: (0, 64), 65: (0, 65), 100: (0, 100), 127: (0, 127),
             128: (64, 64), 256: (192, 64), 1024: (768, 256), 1028: (768, 260)}
    for d, (h, v) in known.items():
        assert dimension_split(d) == (h, v), d


def test_port_dimension_split_and_ratios(built_oracle):
    import ctypes as C
    from oracle.oracle import PORT_LIB
    lib = C.CDLL(PORT_LIB)
    lib.pdxport_dim_split.argtypes = [C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    for d in range(1, 2100, 7):
        h, v = C.c_uint32(), C.c_uint32()
        lib.pdxport_dim_split(d, C.byref(h), C.byref(v))
        assert (h.value, v.value) == dimension_split(d)


def test_ratio_table_properties():
    d = 768
    r = [adsampling_ratio(i, d) for i in range(d + 1)]
    assert r[0] == 1.0 and r[d] == 1.0
    assert all(x > 0 for x in r)
    # epsilon0 = 1.5: i/d * (1 + 1.5/sqrt(i))^2
    assert abs(float(r[64]) - 64 / 768 * (1 + 1.5 / 8) ** 2) < 1e-6


@pytest.mark.parametrize("name", CASES)
def test_file_roundtrip(name):
    path, *_ = load_golden(name)
    raw = open(path, "rb").read()
    assert read_index(raw).to_bytes() == raw


@pytest.mark.parametrize("name", CASES)
def test_port_matches_reference_golden(built_oracle, name):
    from oracle.oracle import Port
    path, q, r, exp = load_golden(name)
    port = Port(path)
    k = exp["k"]
    port.set_nprobe(exp["nprobe"])
    order = np.array(exp["order"], np.uint32)
    for i in range(len(r)):
        a = port.search(r[i], k, transformed=True)
        assert_same(*a, exp["plain_ids"][i], exp["plain_dists"][i], ctx=f"{name} plain q{i}")
        b = port.search_with_order(r[i], k, order, transformed=True)
        assert_same(*b, exp["order_ids"][i], exp["order_dists"][i], ctx=f"{name} order q{i}")
        c = port.filtered_search(r[i], k, np.array(exp["filters"][i], np.uint64), transformed=True)
        assert_same(*c, exp["filt_ids"][i], exp["filt_dists"][i], ctx=f"{name} filtered q{i}")
        # raw queries go through the port's own rotation (not the reference's BLAS): same
        # neighbours, distances at FP32 rounding level
        e = port.search(q[i], k)
        assert recall(e[0], exp["raw_ids"][i], k) >= 0.8
    port.set_pruning_aggressiveness(1e30)
    for i in range(len(r)):
        g = port.search(r[i], k, transformed=True)
        assert_same(*g, exp["exh_ids"][i], exp["exh_dists"][i], ctx=f"{name} unpruned q{i}")


def _ref_available():
    from oracle.oracle import Reference
    return Reference.available()


@pytest.mark.parametrize("itype", ["pdx_f32", "pdx_u8", "pdx_tree_f32", "pdx_tree_u8"])
@pytest.mark.parametrize("d", [5, 63, 129, 384])
def test_port_matches_reference_fresh(built_oracle, itype, d):
    if not _ref_available():
        pytest.skip("reference oracle not built (reference sources absent)")
    from oracle.oracle import Port, Reference
    gm = GaussianMixture(d, 12, 0.5, seed=d, unit_norm=(d % 2 == 1))
    X = gm.sample(1500, 0)
    Q = gm.sample(20, 1)
    f = build_index(X, itype, num_clusters=9, num_meso_clusters=3, normalize=(d % 2 == 1), seed=2)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ref, port = Reference(p), Port(p)
        for nprobe in (0, 3):
            ref.set_nprobe(nprobe)
            port.set_nprobe(nprobe)
            R = ref.rotate(Q / np.linalg.norm(Q, axis=1, keepdims=True) if d % 2 == 1 else Q)
            for i in range(len(Q)):
                assert_same(*port.search(R[i], 10, transformed=True),
                            *ref.search(R[i], 10, transformed=True), ctx=f"{itype} d={d} q{i}")
        ref.close()
        port.close()


def test_port_recall_against_bruteforce(built_oracle):
    from oracle.oracle import Port, brute_force_knn
    gm = GaussianMixture(96, 16, 0.6, seed=3)
    X = gm.sample(4000, 0)
    Q = gm.sample(50, 1)
    f = build_index(X, "pdx_f32", num_clusters=20, seed=1)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        port = Port(p)
        gt, _ = brute_force_knn(X, Q, 10)
        port.set_nprobe(0)
        ids, ds, cnt = port.search_batch(Q, 10, n_threads=2)
        r = np.mean([recall(ids[i], gt[i], 10) for i in range(len(Q))])
        assert r >= 0.97  # exhaustive with ADSampling pruning


def test_port_dct_rotation(built_oracle, tmp_path):
    """FFTW-built files (1 x d sign vector): the port's rotation is the orthonormal DCT-II of
    the sign-flipped query (adsampling.hpp:192-246)."""
    from oracle.oracle import Port
    from tests.helpers import dct_index, dct_rotate
    f, Q, signs = dct_index("pdx_f32", 64, 3000, 12, seed=4)
    p = str(tmp_path / "dct.pdx")
    f.save(p)
    port = Port(p)
    ref = dct_rotate(Q[:8], signs)
    for i in range(8):
        np.testing.assert_allclose(port.prepare_query(Q[i]), ref[i], rtol=0, atol=2e-6)
    port.close()
