"""The allocation-free entry point, pdxg_search_device_noalloc.

It exists for callers that must not have the library allocate GPU memory (a host framework
that owns the device's memory pool, a serving loop that cannot take the synchronisation
cudaMalloc may cause). It must return exactly what pdxg_search_device returns for the same
batch -- the parity bar of the other GPU tests is bit-identical distances and ids -- and it
must keep doing so on a second call, since the fixed scratch array keeps the previous call's
contents. The cases cover both rotations pdxg_search_device picks for raw queries (the FP32 SIMT
kernels below d = 512, the TF32x3 tensor-core GEMM for more than 8 queries at d = 1024), an index
after Append / Delete, and the refusals (a batch beyond the scratch, the reduced-precision
probe). This file is collected last so that a failure here never hides another test.
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from pdx_b200 import compiled
from tests.helpers import load_golden

pytestmark = pytest.mark.gpu

PDXG_ERR_UNSUPPORTED = 5
PDXG_ERR_CAPACITY = 6


def _lib():
    lib = compiled.library()
    vp = C.c_void_p
    lib.pdxg_search_device_noalloc.restype = C.c_int
    lib.pdxg_search_device_noalloc.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp,
                                               vp, vp]
    lib.pdxg_noalloc_scratch_bytes.restype = C.c_uint64
    lib.pdxg_noalloc_scratch_bytes.argtypes = []
    return lib


def _run(lib, fn_name, ix, q, k, flags, stream):
    import torch
    nq = q.shape[0]
    ids = torch.full((nq, k), -1, dtype=torch.int32, device="cuda")
    ds = torch.full((nq, k), -1.0, dtype=torch.float32, device="cuda")
    cnt = torch.full((nq,), -1, dtype=torch.int32, device="cuda")
    fn = getattr(lib, fn_name)
    rc = fn(ix.handle.ptr, C.c_void_p(q.data_ptr()), nq, k, flags, C.c_void_p(ids.data_ptr()),
            C.c_void_p(ds.data_ptr()), C.c_void_p(cnt.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == 0, lib.pdxg_last_error().decode()
    stream.synchronize()
    return ids.cpu().numpy(), ds.cpu().numpy(), cnt.cpu().numpy()


def _check_twice(lib, ix, host_q, k, flags, noalloc_first=False):
    """Two noalloc calls in a row against one pdxg_search_device call: bit-identical. With
    noalloc_first the first noalloc call runs before pdxg_search_device."""
    import torch
    stream = torch.cuda.Stream()
    q = torch.from_numpy(np.ascontiguousarray(host_q, dtype=np.float32)).cuda()
    first = _run(lib, "pdxg_search_device_noalloc", ix, q, k, flags, stream) if noalloc_first else None
    want = _run(lib, "pdxg_search_device", ix, q, k, flags, stream)
    assert (want[2] > 0).all()
    for call in range(2):
        got = first if (call == 0 and first is not None) else \
            _run(lib, "pdxg_search_device_noalloc", ix, q, k, flags, stream)
        np.testing.assert_array_equal(got[2], want[2], err_msg=f"counts, call {call}")
        for i in range(q.shape[0]):
            c = want[2][i]
            np.testing.assert_array_equal(got[0][i, :c], want[0][i, :c], err_msg=f"ids q{i} call {call}")
            np.testing.assert_array_equal(got[1][i, :c], want[1][i, :c], err_msg=f"dists q{i} call {call}")


@pytest.mark.parametrize("name", ["tree_u8_d256", "f32_d64"])
def test_noalloc_matches_search_device_twice(name):
    lib = _lib()
    path, queries, rotated, exp = load_golden(name)
    ix = compiled.load_index(path)
    ix.set_nprobe(exp["nprobe"])
    for flags, host_q in ((0, queries), (compiled.PDXG_QUERY_TRANSFORMED, rotated)):
        _check_twice(lib, ix, host_q, exp["k"], flags)


@pytest.fixture(scope="module")
def d1024_index():
    """A 3,000 x 1024 SQ8 tree index: raw batches of more than 8 queries at d >= 512 are rotated
    on the tensor cores by pdxg_search_device."""
    from pdx_b200.builder import GaussianMixture, build_index
    gm = GaussianMixture(1024, 16, 0.25, seed=1031, unit_norm=True)
    X = gm.sample(3000, 0)
    Q = gm.sample(48, 1)
    f = build_index(X, "pdx_tree_u8", num_clusters=16, num_meso_clusters=4, normalize=True, seed=7)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ix.pdx")
        f.save(p)
        ix = compiled.load_index(p)
    return ix, Q


def test_noalloc_tensor_core_rotation_d1024(d1024_index):
    lib = _lib()
    ix, Q = d1024_index
    assert ix.rotation_uses_tensor_cores()
    ix.set_nprobe(6)
    _check_twice(lib, ix, Q, 20, 0)          # 48 raw queries: TF32x3 rotation in both
    _check_twice(lib, ix, Q[:5], 20, 0)      # 5 raw queries: the FP32 GEMV in both
    ix.set_rotation_mode(1)
    _check_twice(lib, ix, Q, 20, 0)          # the FP32 SIMT GEMM in both
    ix.set_rotation_mode(0)


def test_noalloc_after_append_delete():
    lib = _lib()
    path, queries, rotated, exp = load_golden("tree_u8_d256")
    ix = compiled.load_index(path)
    ix.set_nprobe(exp["nprobe"])
    n = ix.get_num_embeddings()
    rng = np.random.default_rng(3)
    new_rows = rotated[rng.integers(0, len(rotated), 40)] + rng.normal(0, 0.01, (40, rotated.shape[1])).astype(np.float32)
    ix.append_batch(n, new_rows.astype(np.float32), transformed=True)
    for r in rng.choice(n, 60, replace=False):
        ix.delete(int(r))
    # the first search after the changes (a noalloc call) uploads them on its own stream
    _check_twice(lib, ix, rotated, exp["k"], compiled.PDXG_QUERY_TRANSFORMED, noalloc_first=True)
    _check_twice(lib, ix, queries, exp["k"], 0)
    assert ix.maintenance_stats()["deletes"] == 60


def test_noalloc_rejects_reduced_precision_probe(d1024_index):
    import torch
    lib = _lib()
    ix, Q = d1024_index
    ix.set_probe_mode(1)
    try:
        q = torch.from_numpy(Q).cuda()
        out = torch.zeros((len(Q), 20), dtype=torch.int32, device="cuda")
        rc = lib.pdxg_search_device_noalloc(ix.handle.ptr, C.c_void_p(q.data_ptr()), len(Q), 20, 0,
                                            C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()),
                                            C.c_void_p(out.data_ptr()), None)
        assert rc == PDXG_ERR_UNSUPPORTED
        assert "reduced-precision probe" in lib.pdxg_last_error().decode()
    finally:
        ix.set_probe_mode(0)


@pytest.mark.parametrize("d_case", ["simt", "tensor_cores"])
def test_noalloc_rejects_batches_beyond_its_scratch(d_case, d1024_index):
    import torch
    lib = _lib()
    if d_case == "simt":
        path, queries, rotated, exp = load_golden("tree_u8_d256")
        ix = compiled.load_index(path)
        d = queries.shape[1]
        too_many = int(lib.pdxg_noalloc_scratch_bytes() // (4 * d)) + 1
    else:
        ix, Q = d1024_index
        d = Q.shape[1]
        too_many = int(lib.pdxg_noalloc_scratch_bytes() // (12 * d)) + 1
    q = torch.zeros((too_many, d), dtype=torch.float32, device="cuda")
    out = torch.zeros((too_many, 4), dtype=torch.int32, device="cuda")
    rc = lib.pdxg_search_device_noalloc(ix.handle.ptr, C.c_void_p(q.data_ptr()), too_many, 1, 0,
                                        C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()),
                                        C.c_void_p(out.data_ptr()), None)
    assert rc == PDXG_ERR_CAPACITY
    assert "too large" in lib.pdxg_last_error().decode()
