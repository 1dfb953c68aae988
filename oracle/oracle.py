"""ctypes access to the CPU oracles. TEST INFRASTRUCTURE ONLY.

Only tests/, `__graft_entry__.smoke()` and bench.py's CPU-baseline / reference arm import this
module, and only as the checker or the timed CPU baseline. The product package (`pdx_b200`)
never imports it.

* `Port`      -- oracle/libpdx_port.so, the C restatement of the search path (pdx_port.c).
* `Reference` -- oracle/_ref/libpdx_ref*.so, the reference's own search headers compiled by
                 oracle/Makefile (present only where the reference sources were available
                 at build time; the built files travel with the repository snapshot).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "libpdx_port.so")
REF_LIB = os.path.join(HERE, "_ref", "libpdx_ref.so")
REF_LIB_AVX512 = os.path.join(HERE, "_ref", "libpdx_ref_avx512.so")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def cpu_has_avx512_vnni() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = set()
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        return False
    need = {"avx512f", "avx512bw", "avx512vl", "avx512dq", "avx512_vnni", "bmi2", "fma", "avx2"}
    return need <= flags


class _Base:
    prefix = ""

    def _fn(self, name, res, *args):
        f = getattr(self.lib, self.prefix + name)
        f.restype = res
        f.argtypes = list(args)
        return f


class Port(_Base):
    """Own C restatement of PDXearch (see oracle/pdx_port.c)."""
    prefix = "pdxport_"
    _lib = None

    def __init__(self, path: str):
        if Port._lib is None:
            if not os.path.exists(PORT_LIB):
                raise FileNotFoundError(f"{PORT_LIB} missing: run `make -C oracle port`")
            Port._lib = C.CDLL(PORT_LIB)
        self.lib = Port._lib
        vp = C.c_void_p
        self._load = self._fn("load", vp, C.c_char_p)
        self._free = self._fn("free", None, vp)
        self._dims = self._fn("num_dimensions", C.c_uint32, vp)
        self._ncl = self._fn("num_clusters", C.c_uint32, vp)
        self._type = self._fn("type", C.c_int, vp)
        self._setnp = self._fn("set_nprobe", None, vp, C.c_uint32)
        self._setagg = self._fn("set_pruning_aggressiveness", None, vp, C.c_float)
        self._search = self._fn("search", C.c_int, vp, _f32p, C.c_uint32, C.c_int, _u32p, _f32p)
        self._search_order = self._fn("search_with_order", C.c_int, vp, _f32p, C.c_uint32, _u32p,
                                      C.c_uint32, C.c_int, _u32p, _f32p)
        self._fsearch = self._fn("filtered_search", C.c_int, vp, _f32p, C.c_uint32, _u64p,
                                 C.c_uint64, C.c_int, _u32p, _f32p)
        self._batch = self._fn("search_batch", C.c_int, vp, _f32p, C.c_uint32, C.c_uint32, C.c_int,
                               C.c_int, _u32p, _f32p, _u32p)
        self._prep = self._fn("prepare_query", None, vp, _f32p, _f32p)
        self._quant = self._fn("quantize", None, vp, _f32p, _u8p)
        self._tree_order = self._fn("tree_order", C.c_int, vp, _f32p, C.c_int, _u32p)
        self._access_order = self._fn("access_order", None, vp, _f32p, C.c_int, _u32p)
        self.h = self._load(path.encode())
        if not self.h:
            raise RuntimeError(f"port failed to load {path}")
        self.d = self._dims(self.h)
        self.nclusters = self._ncl(self.h)
        self.index_type = self._type(self.h)

    def close(self):
        if self.h:
            self._free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_nprobe(self, n: int):
        self._setnp(self.h, n)

    def set_pruning_aggressiveness(self, eps0: float):
        self._setagg(self.h, eps0)

    def search(self, q, k: int, transformed: bool = False):
        q = np.ascontiguousarray(q, dtype=np.float32)
        ids = np.zeros(k, np.uint32)
        ds = np.zeros(k, np.float32)
        m = self._search(self.h, q, k, int(transformed), ids, ds)
        return ids[:m], ds[:m]

    def search_with_order(self, q, k: int, order, transformed: bool = False):
        q = np.ascontiguousarray(q, dtype=np.float32)
        order = np.ascontiguousarray(order, dtype=np.uint32)
        ids = np.zeros(k, np.uint32)
        ds = np.zeros(k, np.float32)
        m = self._search_order(self.h, q, k, order, len(order), int(transformed), ids, ds)
        return ids[:m], ds[:m]

    def filtered_search(self, q, k: int, row_ids, transformed: bool = False):
        q = np.ascontiguousarray(q, dtype=np.float32)
        r = np.ascontiguousarray(row_ids, dtype=np.uint64)
        ids = np.zeros(k, np.uint32)
        ds = np.zeros(k, np.float32)
        m = self._fsearch(self.h, q, k, r, len(r), int(transformed), ids, ds)
        return ids[:m], ds[:m]

    def search_batch(self, Q, k: int, transformed: bool = False, n_threads: int = 0):
        Q = np.ascontiguousarray(Q, dtype=np.float32)
        nq = Q.shape[0]
        ids = np.zeros((nq, k), np.uint32)
        ds = np.zeros((nq, k), np.float32)
        cnt = np.zeros(nq, np.uint32)
        self._batch(self.h, Q, nq, k, int(transformed), n_threads or (os.cpu_count() or 1), ids, ds, cnt)
        return ids, ds, cnt

    def prepare_query(self, q):
        q = np.ascontiguousarray(q, dtype=np.float32)
        out = np.zeros(self.d, np.float32)
        self._prep(self.h, q, out)
        return out

    def quantize(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros(self.d, np.uint8)
        self._quant(self.h, x, out)
        return out

    def tree_order(self, q, transformed: bool = False):
        q = np.ascontiguousarray(q, dtype=np.float32)
        out = np.zeros(self.nclusters + 1, np.uint32)
        m = self._tree_order(self.h, q, int(transformed), out)
        return out[:m]

    def access_order(self, q, transformed: bool = False):
        q = np.ascontiguousarray(q, dtype=np.float32)
        out = np.zeros(self.nclusters, np.uint32)
        self._access_order(self.h, q, int(transformed), out)
        return out


class Reference(_Base):
    """The reference's own search code (oracle/_ref), loaded from a file index."""
    prefix = "pdxref_"
    _libs = {}

    @staticmethod
    def available(flavour: str = "avx2") -> bool:
        return os.path.exists(REF_LIB if flavour == "avx2" else REF_LIB_AVX512)

    def __init__(self, path: str, flavour: str = "avx2"):
        lib_path = REF_LIB if flavour == "avx2" else REF_LIB_AVX512
        if lib_path not in Reference._libs:
            # the reference's sgemm_ comes from a pthreads OpenBLAS while its searchers run on an
            # OpenMP pool: one BLAS thread per caller avoids the nested pools (OpenBLAS reads
            # this when the library loads)
            os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
            if not os.path.exists(lib_path):
                raise FileNotFoundError(f"{lib_path} missing: run `make -C oracle ref`")
            Reference._libs[lib_path] = C.CDLL(lib_path)
        self.lib = Reference._libs[lib_path]
        vp = C.c_void_p
        self._load = self._fn("load", vp, C.c_char_p)
        self._err = self._fn("last_error", C.c_char_p)
        self._free = self._fn("free", None, vp)
        self._dims = self._fn("num_dimensions", C.c_uint32, vp)
        self._ncl = self._fn("num_clusters", C.c_uint32, vp)
        self._type = self._fn("type", C.c_int, vp)
        self._csize = self._fn("cluster_size", C.c_uint32, vp, C.c_uint32)
        self._cids = self._fn("cluster_row_ids", None, vp, C.c_uint32, _u32p)
        self._setnp = self._fn("set_nprobe", None, vp, C.c_uint32)
        self._setagg = self._fn("set_pruning_aggressiveness", None, vp, C.c_float)
        self._rotate = self._fn("rotate", None, vp, _f32p, _f32p, C.c_uint32)
        self._search = self._fn("search", C.c_int, vp, _f32p, C.c_uint32, C.c_int, _u32p, _f32p)
        self._search_order = self._fn("search_with_order", C.c_int, vp, _f32p, C.c_uint32, _u32p,
                                      C.c_uint32, C.c_int, _u32p, _f32p)
        self._fsearch = self._fn("filtered_search", C.c_int, vp, _f32p, C.c_uint32, _u64p,
                                 C.c_uint64, C.c_int, _u32p, _f32p)
        self._batch = self._fn("search_batch", C.c_int, vp, _f32p, C.c_uint32, C.c_uint32, C.c_int,
                               C.c_int, _u32p, _f32p, _u32p)
        self._append = self._fn("append", C.c_int, vp, C.c_uint64, _f32p, C.c_int)
        self._delete = self._fn("delete", C.c_int, vp, C.c_uint64)
        self._set_append_norm = self._fn("set_append_normalization", None, vp, C.c_int)
        self._compact_all = self._fn("compact_all", None, vp)
        self._mstats = self._fn("maintenance_stats", None, vp, _u64p)
        self.h = self._load(path.encode())
        if not self.h:
            raise RuntimeError(self._err().decode())
        self.d = self._dims(self.h)
        self.nclusters = self._ncl(self.h)
        self.index_type = self._type(self.h)

    def close(self):
        if self.h:
            self._free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_nprobe(self, n: int):
        self._setnp(self.h, n)

    def set_pruning_aggressiveness(self, eps0: float):
        self._setagg(self.h, eps0)

    def cluster_row_ids(self, c: int):
        out = np.zeros(self._csize(self.h, c), np.uint32)
        self._cids(self.h, c, out)
        return out

    # -- maintenance: PDXTreeIndex::Append / Delete on the reference's clusters ------------------
    def _raise(self, rc: int):
        msg = self._err().decode()
        raise (ValueError if rc == 1 else RuntimeError)(msg)

    def append(self, row_id: int, embedding, transformed: bool = False):
        e = np.ascontiguousarray(embedding, dtype=np.float32)
        rc = self._append(self.h, row_id, e, int(transformed))
        if rc:
            self._raise(rc)

    def delete(self, row_id: int):
        rc = self._delete(self.h, row_id)
        if rc:
            self._raise(rc)

    def set_append_normalization(self, on: bool):
        self._set_append_norm(self.h, int(on))

    def compact_all(self):
        """The compaction PDXTreeIndex::Save applies before writing (index.hpp:484-494)."""
        self._compact_all(self.h)

    def maintenance_stats(self) -> dict:
        out = np.zeros(5, np.uint64)
        self._mstats(self.h, out)
        keys = ("appends", "deletes", "compactions", "capacity_growths", "merges_not_performed")
        return {k: int(v) for k, v in zip(keys, out)}

    def rotate(self, X):
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float32)
        out = np.zeros_like(X)
        self._rotate(self.h, X, out, X.shape[0])
        return out

    def search(self, q, k: int, transformed: bool = False):
        q = np.ascontiguousarray(q, dtype=np.float32)
        ids = np.zeros(k, np.uint32)
        ds = np.zeros(k, np.float32)
        m = self._search(self.h, q, k, int(transformed), ids, ds)
        if m < 0:
            raise RuntimeError(self._err().decode())
        return ids[:m], ds[:m]

    def search_with_order(self, q, k: int, order, transformed: bool = False):
        q = np.ascontiguousarray(q, dtype=np.float32)
        order = np.ascontiguousarray(order, dtype=np.uint32)
        ids = np.zeros(k, np.uint32)
        ds = np.zeros(k, np.float32)
        m = self._search_order(self.h, q, k, order, len(order), int(transformed), ids, ds)
        return ids[:m], ds[:m]

    def filtered_search(self, q, k: int, row_ids, transformed: bool = False):
        q = np.ascontiguousarray(q, dtype=np.float32)
        r = np.ascontiguousarray(row_ids, dtype=np.uint64)
        ids = np.zeros(k, np.uint32)
        ds = np.zeros(k, np.float32)
        m = self._fsearch(self.h, q, k, r, len(r), int(transformed), ids, ds)
        return ids[:m], ds[:m]

    def search_batch(self, Q, k: int, transformed: bool = False, n_threads: int = 0):
        Q = np.ascontiguousarray(Q, dtype=np.float32)
        nq = Q.shape[0]
        ids = np.zeros((nq, k), np.uint32)
        ds = np.zeros((nq, k), np.float32)
        cnt = np.zeros(nq, np.uint32)
        rc = self._batch(self.h, Q, nq, k, int(transformed), n_threads, ids, ds, cnt)
        if rc != 0:
            raise RuntimeError("reference batch search failed")
        return ids, ds, cnt


def brute_force_knn(data: np.ndarray, queries: np.ndarray, k: int, chunk: int = 4096):
    """FP64 brute-force L2 ground truth (ids [nq, k], squared distances [nq, k])."""
    X = np.asarray(data, dtype=np.float64)
    Q = np.asarray(queries, dtype=np.float64)
    xn = np.einsum("ij,ij->i", X, X)
    ids = np.zeros((Q.shape[0], k), np.int64)
    ds = np.zeros((Q.shape[0], k), np.float64)
    for s in range(0, Q.shape[0], chunk):
        q = Q[s:s + chunk]
        d2 = xn[None, :] - 2.0 * q @ X.T + np.einsum("ij,ij->i", q, q)[:, None]
        part = np.argpartition(d2, min(k, d2.shape[1] - 1), axis=1)[:, :k]
        pd = np.take_along_axis(d2, part, 1)
        o = np.argsort(pd, axis=1, kind="stable")
        ids[s:s + chunk] = np.take_along_axis(part, o, 1)
        ds[s:s + chunk] = np.take_along_axis(pd, o, 1)
    return ids, ds


def recall_at_k(found_ids: np.ndarray, gt_ids: np.ndarray, k: int) -> float:
    """Mean |found[:k] ∩ gt[:k]| / k (test_utils.hpp:212-243)."""
    tot = 0.0
    for f, g in zip(found_ids, gt_ids):
        tot += len(set(np.asarray(f[:k]).tolist()) & set(np.asarray(g[:k]).tolist())) / float(min(k, len(g)))
    return tot / max(1, len(gt_ids))
