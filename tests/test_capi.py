"""CPU tests of the drop-in boundary: the C-ABI library loads and exports every entry point the
header declares, host-side validation rejects bad input before any GPU work, and without a GPU
the search path fails loudly instead of falling back to the CPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from pdx_b200 import compiled
from tests.helpers import load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pdx_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pdxg_[a-z_0-9]+)\s*\(", txt)))


def test_header_symbols_exported():
    lib = compiled.library()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def _load_status(data: bytes):
    lib = compiled.library()
    out = C.c_void_p()
    rc = lib.pdxg_load_buffer(data, len(data), 0, C.byref(out))
    return rc, lib.pdxg_last_error().decode()


def test_rejects_unknown_type():
    rc, msg = _load_status(bytes([7]) + b"\0" * 64)
    assert rc == 3 and "Unknown PDX index type" in msg


def test_rejects_truncated_files():
    path, *_ = load_golden("u8_d100")
    raw = open(path, "rb").read()
    for cut in (0, 5, 9, 400, len(raw) // 2, len(raw) - 1):
        rc, msg = _load_status(raw[:cut])
        assert rc == 3, (cut, rc, msg)


def test_rejects_inconsistent_split():
    path, *_ = load_golden("f32_d64")
    raw = bytearray(open(path, "rb").read())
    d = 64
    off = 9 + 4 * d * d
    raw[off + 4:off + 8] = (60).to_bytes(4, "little")  # d_v no longer matches the split
    rc, msg = _load_status(bytes(raw))
    assert rc == 3 and "split" in msg


def test_missing_file_is_io_error():
    with pytest.raises(RuntimeError, match="Failed to open"):
        compiled.load_index("/nonexistent/file.pdx")


def test_config_validation():
    # PDXIndexConfig::Validate (index.hpp:39-62)
    with pytest.raises(ValueError):
        compiled.PDXIndex("pdx_f32", 0)
    with pytest.raises(ValueError):
        compiled.PDXIndex("pdx_f32", 16385)
    with pytest.raises(ValueError):
        compiled.PDXIndex("pdx_f32", 8, sampling_fraction=1.5)
    with pytest.raises(ValueError):
        compiled.PDXIndex("pdx_tree_f32", 8, num_clusters=10, num_meso_clusters=10)
    with pytest.raises(ValueError):
        compiled.PDXIndex("pdx_f32", 8, kmeans_iters=100)
    with pytest.raises(RuntimeError, match="Unknown index type"):
        compiled.PDXIndex("pdx_f16", 8)
    with pytest.raises(RuntimeError):
        compiled.PDXIndex("pdx_f32", 8, distance_metric=7)


def test_flat_index_rejects_maintenance():
    ix = compiled.PDXIndex("pdx_f32", 8)
    with pytest.raises(RuntimeError, match="Append is not implemented in PDXIndex"):
        ix.append(0, np.zeros(8, np.float32))
    with pytest.raises(RuntimeError, match="Delete is not implemented in PDXIndex"):
        ix.delete(0)


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    path, *_ = load_golden("f32_d64")
    with pytest.raises(RuntimeError, match="cuda|CUDA"):
        compiled.load_index(path)


def test_build_and_maintenance_argument_checks():
    """pdxg_build / pdxg_append / pdxg_delete reject bad arguments on the host, before any GPU
    work (BuildIndex's config checks, index.hpp:27-62; the C ABI's NULL checks)."""
    lib = compiled.library()
    rng = np.random.default_rng(0)
    X = rng.standard_normal((300, 64)).astype(np.float32)
    rot = np.eye(64, dtype=np.float32)
    out = C.c_void_p()
    # more clusters than rows
    rc = lib.pdxg_build(X, 300, 64, 0, 400, 0, 0, rot, 42, 10, 0, C.byref(out))
    assert rc == compiled.PDXG_ERR_INVALID_ARGUMENT and "exceeds" in lib.pdxg_last_error().decode()
    # meso clusters not fewer than clusters (trees)
    rc = lib.pdxg_build(X, 300, 64, 2, 20, 20, 0, rot, 42, 10, 0, C.byref(out))
    assert rc == compiled.PDXG_ERR_INVALID_ARGUMENT
    # unknown index type, empty data, d out of range
    assert lib.pdxg_build(X, 300, 64, 4, 10, 0, 0, rot, 42, 10, 0, C.byref(out)) == compiled.PDXG_ERR_INVALID_ARGUMENT
    assert lib.pdxg_build(X, 0, 64, 0, 10, 0, 0, rot, 42, 10, 0, C.byref(out)) == compiled.PDXG_ERR_INVALID_ARGUMENT
    assert lib.pdxg_build(X, 300, 0, 0, 10, 0, 0, rot, 42, 10, 0, C.byref(out)) == compiled.PDXG_ERR_INVALID_ARGUMENT
    # NULL index handles
    e = np.zeros(64, np.float32)
    assert lib.pdxg_append(None, 0, e, 0) == compiled.PDXG_ERR_INVALID_ARGUMENT
    assert lib.pdxg_append_batch(None, 0, 1, e, 0) == compiled.PDXG_ERR_INVALID_ARGUMENT
    assert lib.pdxg_delete(None, 0) == compiled.PDXG_ERR_INVALID_ARGUMENT
    assert lib.pdxg_maintenance_stats(None, np.zeros(6, np.uint64)) == compiled.PDXG_ERR_INVALID_ARGUMENT
    # the Python layer: flat types refuse maintenance with the reference's message
    ix = compiled.PDXIndex("pdx_u8", 64)
    with pytest.raises(RuntimeError, match="Append is not implemented in PDXIndex"):
        ix.append_batch(0, np.zeros((2, 64), np.float32))
    tree = compiled.PDXIndex("pdx_tree_u8", 64)
    with pytest.raises(RuntimeError, match="empty"):
        tree.append(0, np.zeros(64, np.float32))
    with pytest.raises(RuntimeError, match="1D"):
        tree.append(0, np.zeros((1, 64), np.float32))
