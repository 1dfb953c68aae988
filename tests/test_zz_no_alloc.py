"""The allocation-free entry point, pdxg_search_device_noalloc.

It exists for callers that must not have the library allocate GPU memory (a host framework
that owns the device's memory pool, a serving loop that cannot take the synchronisation
cudaMalloc may cause). It must return exactly what pdxg_search_device returns for the same
batch -- the parity bar of the other GPU tests is bit-identical distances and ids -- and it
must keep doing so on a second call, since the fixed scratch array keeps the previous call's
contents. This file is collected last so that a failure here never hides another test.
"""
import ctypes as C

import numpy as np
import pytest

from pdx_b200 import compiled
from tests.helpers import load_golden

pytestmark = pytest.mark.gpu

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


@pytest.mark.parametrize("name", ["tree_u8_d256", "f32_d64"])
def test_noalloc_matches_search_device_twice(name):
    import torch
    lib = _lib()
    path, queries, rotated, exp = load_golden(name)
    ix = compiled.load_index(path)
    ix.set_nprobe(exp["nprobe"])
    k = exp["k"]
    stream = torch.cuda.Stream()
    for flags, host_q in ((0, queries), (compiled.PDXG_QUERY_TRANSFORMED, rotated)):
        q = torch.from_numpy(np.ascontiguousarray(host_q, dtype=np.float32)).cuda()
        want = _run(lib, "pdxg_search_device", ix, q, k, flags, stream)
        for call in range(2):
            got = _run(lib, "pdxg_search_device_noalloc", ix, q, k, flags, stream)
            np.testing.assert_array_equal(got[2], want[2], err_msg=f"counts, call {call}")
            for i in range(q.shape[0]):
                c = want[2][i]
                np.testing.assert_array_equal(got[0][i, :c], want[0][i, :c], err_msg=f"ids q{i} call {call}")
                np.testing.assert_array_equal(got[1][i, :c], want[1][i, :c], err_msg=f"dists q{i} call {call}")


def test_noalloc_rejects_batches_beyond_its_scratch():
    import torch
    lib = _lib()
    path, queries, rotated, exp = load_golden("tree_u8_d256")
    ix = compiled.load_index(path)
    d = queries.shape[1]
    too_many = int(lib.pdxg_noalloc_scratch_bytes() // (4 * d)) + 1
    q = torch.zeros((too_many, d), dtype=torch.float32, device="cuda")
    out = torch.zeros((too_many, 4), dtype=torch.int32, device="cuda")
    rc = lib.pdxg_search_device_noalloc(ix.handle.ptr, C.c_void_p(q.data_ptr()), too_many, 1, 0,
                                        C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()),
                                        C.c_void_p(out.data_ptr()), None)
    assert rc == PDXG_ERR_CAPACITY
    assert "too large" in lib.pdxg_last_error().decode()
