"""ctypes binding of libpdx_b200.so with the reference's pybind surface.

Mirrors module `pdxearch.compiled` (python/lib.cpp:6-60, include/pdx/lib/lib.hpp:15-175):
class `PDXIndex` with the same constructor arguments and methods (`build_index` builds on the
GPU, `append` / `delete` maintain tree indexes), and `load_index(path)`. Additions: batched and
device-pointer searches, `append_batch`, `maintenance_stats`, CUDA-graph capture, the autotuner
and serving contexts (`Context`).
Errors map like pybind's: invalid arguments -> ValueError, everything else -> RuntimeError.

There is no CPU fallback: if the CUDA engine cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from typing import Optional, Tuple

import numpy as np

from . import build as _build
from .layout import INDEX_TYPES

_LIB_PATH = _build.LIB
_lib = None

PDXG_OK = 0
PDXG_ERR_INVALID_ARGUMENT = 1
PDXG_QUERY_TRANSFORMED = 1
PDXG_COLLECT_STATS = 2
PDXG_TIME_KERNELS = 4

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


def library() -> C.CDLL:
    """Loads (building first if missing or stale) the engine library."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or _build._stale():
            _build.build()
        lib = C.CDLL(_LIB_PATH)
        vp = C.c_void_p

        def fn(name, res, *args):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = list(args)

        fn("pdxg_last_error", C.c_char_p)
        fn("pdxg_load", C.c_int, C.c_char_p, C.c_int, C.POINTER(vp))
        fn("pdxg_load_buffer", C.c_int, C.c_char_p, C.c_uint64, C.c_int, C.POINTER(vp))
        fn("pdxg_free", None, vp)
        fn("pdxg_build", C.c_int, _f32p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
           C.c_int, _f32p, C.c_uint64, C.c_uint32, C.c_int, C.POINTER(vp))
        fn("pdxg_set_nprobe", C.c_int, vp, C.c_uint32)
        fn("pdxg_set_pruning_aggressiveness", C.c_int, vp, C.c_float)
        fn("pdxg_set_threads_per_query", C.c_int, vp, C.c_uint32)
        fn("pdxg_set_scan_mode", C.c_int, vp, C.c_uint32)
        fn("pdxg_set_top_level_mode", C.c_int, vp, C.c_uint32)
        fn("pdxg_last_launch_count", C.c_uint32, vp)
        fn("pdxg_set_start_mode", C.c_int, vp, C.c_uint32)
        fn("pdxg_set_probe_mode", C.c_int, vp, C.c_uint32)
        fn("pdxg_graph_create", C.c_int, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, vp, C.POINTER(vp))
        fn("pdxg_graph_launch", C.c_int, vp, vp)
        fn("pdxg_graph_free", None, vp)
        fn("pdxg_autotune", C.c_int, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp)
        fn("pdxg_kernel_times_ex", C.c_int, vp, vp, C.c_uint32)
        fn("pdxg_last_visit_orders", C.c_int, vp, C.c_uint32, C.c_uint32, vp, vp)
        fn("pdxg_search", C.c_int, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, vp)
        fn("pdxg_search_device", C.c_int, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, vp, vp)
        fn("pdxg_search_with_order", C.c_int, vp, _f32p, C.c_uint32, C.c_uint32, _u32p, C.c_uint32,
           C.c_uint32, _u32p, _f32p, _u32p)
        fn("pdxg_filtered_search", C.c_int, vp, _f32p, C.c_uint32, _u64p, C.c_uint64, C.c_uint32,
           _u32p, _f32p, _u32p)
        fn("pdxg_filtered_search_batch", C.c_int, vp, _f32p, C.c_uint32, C.c_uint32, _u64p, _u64p,
           C.c_uint32, _u32p, _f32p, _u32p)
        fn("pdxg_save", C.c_int, vp, C.c_char_p)
        fn("pdxg_index_type", C.c_int, vp)
        fn("pdxg_num_dimensions", C.c_uint32, vp)
        fn("pdxg_num_clusters", C.c_uint32, vp)
        fn("pdxg_nprobe", C.c_uint32, vp)
        fn("pdxg_cluster_size", C.c_uint32, vp, C.c_uint32)
        fn("pdxg_cluster_row_ids", C.c_int, vp, C.c_uint32, _u32p, C.c_uint32)
        fn("pdxg_in_memory_size_in_bytes", C.c_uint64, vp)
        fn("pdxg_num_embeddings", C.c_uint64, vp)
        fn("pdxg_prepare_queries", C.c_int, vp, _f32p, C.c_uint32, _f32p)
        fn("pdxg_get_stats", C.c_int, vp, _u64p)
        fn("pdxg_get_scan_stats", C.c_int, vp, C.c_void_p)
        fn("pdxg_kernel_times", C.c_int, vp, _f32p)
        fn("pdxg_set_rotation_mode", C.c_int, vp, C.c_uint32)
        fn("pdxg_rotation_uses_tensor_cores", C.c_int, vp)
        fn("pdxg_context_create", C.c_int, vp, C.POINTER(vp))
        fn("pdxg_context_free", None, vp)
        fn("pdxg_context_stream", vp, vp)
        fn("pdxg_search_requests", C.c_int, vp, vp, C.c_uint32, vp, vp, C.c_uint32, C.c_uint32, vp, vp, vp)
        fn("pdxg_filter_register", C.c_int, vp, vp, C.c_uint64, C.POINTER(C.c_int32))
        fn("pdxg_filter_release", C.c_int, vp, C.c_int32)
        fn("pdxg_append", C.c_int, vp, C.c_uint64, _f32p, C.c_uint32)
        fn("pdxg_append_batch", C.c_int, vp, C.c_uint64, C.c_uint32, _f32p, C.c_uint32)
        fn("pdxg_delete", C.c_int, vp, C.c_uint64)
        fn("pdxg_set_append_normalization", C.c_int, vp, C.c_int)
        fn("pdxg_maintenance_stats", C.c_int, vp, _u64p)
        _lib = lib
    return _lib


def _check(rc: int) -> None:
    if rc != PDXG_OK:
        msg = library().pdxg_last_error().decode(errors="replace")
        if rc == PDXG_ERR_INVALID_ARGUMENT:
            raise ValueError(msg)
        raise RuntimeError(msg)


class SearchGraph:
    """A captured device search; launch() replays it on a stream."""

    def __init__(self, ptr, owner):
        self.ptr = ptr
        self._owner = owner  # the index outlives the graph

    def launch(self, stream: int = 0) -> None:
        _check(library().pdxg_graph_launch(self.ptr, C.c_void_p(stream)))

    def __del__(self):
        if getattr(self, "ptr", None) and self.ptr.value:
            library().pdxg_graph_free(self.ptr)
            self.ptr = C.c_void_p()


class Handle:
    """Owns one pdxg_index*."""

    def __init__(self, ptr: int):
        self.ptr = C.c_void_p(ptr)

    def __del__(self):
        if getattr(self, "ptr", None) and self.ptr.value and _lib is not None:
            _lib.pdxg_free(self.ptr)
            self.ptr = C.c_void_p(0)


def _load_handle(path: Optional[str] = None, data: Optional[bytes] = None, device: int = 0) -> Handle:
    lib = library()
    out = C.c_void_p()
    if path is not None:
        _check(lib.pdxg_load(os.fsencode(path), device, C.byref(out)))
    else:
        _check(lib.pdxg_load_buffer(data, len(data), device, C.byref(out)))
    return Handle(out.value)


PDXG_ERR_UNSUPPORTED = 5


def build_handle(data: np.ndarray, index_type: str, rotation: np.ndarray, num_clusters: int = 0,
                 num_meso_clusters: int = 0, normalize: bool = False, seed: int = 42,
                 kmeans_iters: int = 10, device: int = 0) -> Optional[Handle]:
    """Builds an index on the GPU (pdxg_build). None when the engine cannot build this shape
    (d not a multiple of 8); raises on every other error."""
    lib = library()
    data = np.ascontiguousarray(data, dtype=np.float32)
    rot = np.ascontiguousarray(rotation, dtype=np.float32)
    n, d = data.shape
    if rot.shape != (d, d):
        raise ValueError(f"rotation must be {d} x {d}")
    out = C.c_void_p()
    rc = lib.pdxg_build(data, n, d, INDEX_TYPES[index_type], num_clusters, num_meso_clusters,
                        1 if normalize else 0, rot, seed, kmeans_iters, device, C.byref(out))
    if rc == PDXG_ERR_UNSUPPORTED:
        return None
    _check(rc)
    return Handle(out.value)


_METRICS = {0: "l2sq", 1: "cosine", 2: "ip"}


class PDXIndex:
    """GPU-resident PDX index with the reference's `compiled.PDXIndex` interface."""

    def __init__(self, index_type: str, num_dimensions: int, distance_metric: int = 0, seed: int = 42,
                 num_clusters: int = 0, num_meso_clusters: int = 0, normalize: bool = False,
                 sampling_fraction: float = 0.0, kmeans_iters: int = 10,
                 hierarchical_indexing: bool = True, n_threads: int = 0, device: int = 0):
        if index_type not in INDEX_TYPES:
            raise RuntimeError(f"Unknown index type: {index_type}. Valid types: pdx_f32, pdx_u8, "
                               "pdx_tree_f32, pdx_tree_u8")
        if distance_metric not in _METRICS:
            raise RuntimeError(f"Unknown distance metric: {distance_metric}")
        # PDXIndexConfig::Validate (index.hpp:39-62)
        if num_dimensions == 0 or num_dimensions > 16384:
            raise ValueError(f"num_dimensions must be between 1 and 16384, got {num_dimensions}")
        if sampling_fraction < 0.0 or sampling_fraction > 1.0:
            raise ValueError(f"sampling_fraction must be between 0.0 and 1.0, got {sampling_fraction}")
        if num_meso_clusters > 0 and num_clusters > 0 and num_meso_clusters >= num_clusters:
            raise ValueError(f"num_meso_clusters ({num_meso_clusters}) must be smaller than "
                             f"num_clusters ({num_clusters})")
        if kmeans_iters == 0 or kmeans_iters >= 100:
            raise ValueError(f"kmeans_iters must be between 1 and 99, got {kmeans_iters}")
        self._type = index_type
        self._d = num_dimensions
        self._metric = distance_metric
        self._seed = seed
        self._num_clusters = num_clusters
        self._num_meso = num_meso_clusters
        self._normalize = normalize or distance_metric in (1, 2)
        self._kmeans_iters = kmeans_iters
        self._device = device
        self._nprobe = 0
        self._h: Optional[Handle] = None

    # -- construction --------------------------------------------------------------------
    @classmethod
    def _from_handle(cls, h: Handle) -> "PDXIndex":
        self = cls.__new__(cls)
        lib = library()
        t = lib.pdxg_index_type(h.ptr)
        self._type = {v: k for k, v in INDEX_TYPES.items()}[t]
        self._d = lib.pdxg_num_dimensions(h.ptr)
        self._metric = 0
        self._seed = 42
        self._num_clusters = lib.pdxg_num_clusters(h.ptr)
        self._num_meso = 0
        self._normalize = False
        self._kmeans_iters = 10
        self._device = 0
        self._nprobe = 0
        self._h = h
        return self

    def build_index(self, data: np.ndarray) -> None:
        from .builder import build_index as _build_index
        data = np.ascontiguousarray(data, dtype=np.float32)
        if data.ndim != 2:
            raise RuntimeError("data must be a 2D numpy array (n_embeddings x dimensions)")
        if data.shape[1] != self._d:
            raise ValueError(f"data has {data.shape[1]} dimensions, index expects {self._d}")
        from .builder import random_rotation
        rotation = random_rotation(self._d, self._seed)
        h = build_handle(data, self._type, rotation, self._num_clusters, self._num_meso, self._normalize,
                         self._seed, self._kmeans_iters, self._device)
        if h is None:  # d not a multiple of 8: k-means on torch's GPU GEMMs, same file layout
            f = _build_index(data, self._type, num_clusters=self._num_clusters,
                             num_meso_clusters=self._num_meso, normalize=self._normalize,
                             seed=self._seed, kmeans_iters=self._kmeans_iters, rotation=rotation,
                             device=f"cuda:{self._device}")
            h = _load_handle(data=f.to_bytes(), device=self._device)
            _check(library().pdxg_set_append_normalization(h.ptr, 1 if self._normalize else 0))
        self._h = h
        _check(library().pdxg_set_nprobe(self._h.ptr, self._nprobe))

    def _handle(self) -> Handle:
        if self._h is None:
            raise RuntimeError("index is empty: call build_index() or load_index() first")
        return self._h

    # -- search ----------------------------------------------------------------------------
    def set_nprobe(self, nprobe: int) -> None:
        self._nprobe = int(nprobe)
        if self._h is not None:
            _check(library().pdxg_set_nprobe(self._h.ptr, self._nprobe))

    def search(self, query: np.ndarray, knn: int) -> Tuple[np.ndarray, np.ndarray]:
        q = np.ascontiguousarray(query, dtype=np.float32)
        if q.ndim != 1:
            raise RuntimeError("query must be a 1D numpy array")
        ids, ds, cnt = self.search_batch(q[None, :], knn)
        return ids[0, :cnt[0]].copy(), ds[0, :cnt[0]].copy()

    def search_batch(self, queries: np.ndarray, knn: int, transformed: bool = False):
        """Batched search (extension): returns ids [nq, k], distances [nq, k], counts [nq]."""
        h = self._handle()
        Q = np.ascontiguousarray(queries, dtype=np.float32)
        if Q.ndim != 2 or Q.shape[1] != self.get_num_dimensions():
            raise ValueError("queries must be a 2D array (n_queries x num_dimensions)")
        nq = Q.shape[0]
        ids = np.empty((nq, knn), np.uint32)
        ds = np.empty((nq, knn), np.float32)
        cnt = np.empty(nq, np.uint32)
        _check(library().pdxg_search(h.ptr, Q.ctypes.data, nq, knn,
                                     PDXG_QUERY_TRANSFORMED if transformed else 0,
                                     ids.ctypes.data, ds.ctypes.data, cnt.ctypes.data))
        return ids, ds, cnt

    def search_with_order(self, queries: np.ndarray, knn: int, order, transformed: bool = False):
        """PDXearch::SetClusterAccessOrder + Search (searcher.hpp:48-54), batched."""
        h = self._handle()
        Q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        o = np.ascontiguousarray(order, dtype=np.uint32)
        nq = Q.shape[0]
        ids = np.empty((nq, knn), np.uint32)
        ds = np.empty((nq, knn), np.float32)
        cnt = np.empty(nq, np.uint32)
        _check(library().pdxg_search_with_order(h.ptr, Q, nq, knn, o, len(o),
                                                PDXG_QUERY_TRANSFORMED if transformed else 0,
                                                ids, ds, cnt))
        return ids, ds, cnt

    def filtered_search(self, query: np.ndarray, knn: int, row_ids: np.ndarray):
        h = self._handle()
        q = np.ascontiguousarray(query, dtype=np.float32)
        if q.ndim != 1:
            raise RuntimeError("query must be a 1D numpy array")
        r = np.ascontiguousarray(row_ids, dtype=np.uint64)
        if r.ndim != 1:
            raise RuntimeError("row_ids must be a 1D numpy array")
        ids = np.empty(knn, np.uint32)
        ds = np.empty(knn, np.float32)
        cnt = np.zeros(1, np.uint32)
        _check(library().pdxg_filtered_search(h.ptr, q, knn, r, len(r), 0, ids, ds, cnt))
        return ids[:cnt[0]].copy(), ds[:cnt[0]].copy()

    def filtered_search_batch(self, queries: np.ndarray, knn: int, row_id_lists, transformed=False):
        """Batched filtered search (extension): row_id_lists[i] is None (unfiltered) or ids."""
        h = self._handle()
        Q = np.ascontiguousarray(queries, dtype=np.float32)
        nq = Q.shape[0]
        offsets = np.zeros(nq + 1, np.uint64)
        parts = []
        pos = 0
        for i, lst in enumerate(row_id_lists):
            if lst is None:
                offsets[i] = np.uint64(np.iinfo(np.uint64).max)
            else:
                a = np.asarray(lst, dtype=np.uint64)
                offsets[i] = pos
                parts.append(a)
                pos += len(a)
        offsets[nq] = pos
        # unfiltered queries need the next filtered start as their successor's bound
        rows = np.concatenate(parts) if parts else np.zeros(1, np.uint64)
        ids = np.empty((nq, knn), np.uint32)
        ds = np.empty((nq, knn), np.float32)
        cnt = np.empty(nq, np.uint32)
        _check(library().pdxg_filtered_search_batch(h.ptr, Q, nq, knn, rows, offsets,
                                                    PDXG_QUERY_TRANSFORMED if transformed else 0,
                                                    ids, ds, cnt))
        return ids, ds, cnt

    def prepare_queries(self, queries: np.ndarray) -> np.ndarray:
        """Normalized (if the index is) and rotated queries as the engine searches them."""
        h = self._handle()
        Q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        out = np.empty_like(Q)
        _check(library().pdxg_prepare_queries(h.ptr, Q, Q.shape[0], out))
        return out

    def search_device(self, queries_ptr: int, nq: int, knn: int, ids_ptr: int, dists_ptr: int,
                      counts_ptr: int, stream: int = 0, transformed: bool = False,
                      stats: bool = False, time_kernels: bool = False) -> None:
        """Enqueues a search on GPU-resident buffers (raw device pointers) on `stream`."""
        flags = (PDXG_QUERY_TRANSFORMED if transformed else 0) | (PDXG_COLLECT_STATS if stats else 0)
        flags |= PDXG_TIME_KERNELS if time_kernels else 0
        _check(library().pdxg_search_device(self._handle().ptr, C.c_void_p(queries_ptr), nq, knn,
                                            flags, C.c_void_p(ids_ptr), C.c_void_p(dists_ptr),
                                            C.c_void_p(counts_ptr), C.c_void_p(stream)))

    def last_stats(self) -> dict:
        out = np.zeros(12, np.uint64)
        _check(library().pdxg_get_stats(self._handle().ptr, out))
        names = ["top_level", "start", "warmup", "survivor_horizontal", "survivor_vertical", "probe"]
        return {"bytes": int(out[0]), "clusters_visited": int(out[1]), "merged": int(out[2]),
                "bytes_by_phase": {n: int(v) for n, v in zip(names, out[3:9])},
                "cycles_by_phase": {n: int(v) for n, v in zip(["top_level", "start", "rest"], out[9:12])}}

    def last_scan_stats(self) -> dict:
        """Cluster-major scan counters of the last search_device(..., stats=True)."""
        out = np.zeros(4, np.uint64)
        _check(library().pdxg_get_scan_stats(self._handle().ptr, out.ctypes.data))
        return {"candidates": int(out[0]), "first_step_survivors": int(out[1]),
                "visits_first_step_exit": int(out[2]), "visits_full_warmup": int(out[3])}

    def last_launch_count(self) -> int:
        """Engine kernels launched by the last search_device call."""
        return int(library().pdxg_last_launch_count(self._handle().ptr))

    def kernel_times(self) -> dict:
        """Durations (ms) of the last search_device(..., time_kernels=True): query preparation,
        tree top level or reduced-precision probe, batched Start, scan kernel ("scan" is the
        batched Start plus the scan kernel)."""
        out = np.zeros(11, np.float32)
        _check(library().pdxg_kernel_times_ex(self._handle().ptr, out.ctypes.data, 11))
        return {"prepare": float(out[0]), "top_level": float(out[1]), "start": float(out[2]),
                "search_kernel": float(out[3]), "scan": float(out[2] + out[3]),
                "scan_plan": float(out[4]), "scan_bitmap": float(out[5]), "scan_replay": float(out[6]),
                "scan_per_query": float(out[7]), "top_probe": float(out[8]), "top_partials": float(out[9]),
                "top_replay": float(out[10])}

    def set_pruning_aggressiveness(self, epsilon0: float) -> None:
        _check(library().pdxg_set_pruning_aggressiveness(self._handle().ptr, float(epsilon0)))

    def set_top_level_mode(self, mode: int) -> None:
        """Tree indexes: 0 automatic, 1 top level inside each query's CTA, 2 per-query CTAs,
        3 tiled (probe, exact partials with reuse across queries, replay)."""
        _check(library().pdxg_set_top_level_mode(self._handle().ptr, int(mode)))

    def set_start_mode(self, mode: int) -> None:
        """U8 tree indexes: 0 batched first-cluster Start when it fits, 1 inside the scan."""
        _check(library().pdxg_set_start_mode(self._handle().ptr, int(mode)))

    def autotune(self, queries_ptr: int, nq: int, knn: int, transformed: bool = False) -> dict:
        """Times the engine's forms on this batch of device queries and keeps the fastest."""
        out = np.zeros(3, np.uint32)
        _check(library().pdxg_autotune(self._handle().ptr, C.c_void_p(queries_ptr), nq, knn,
                                       PDXG_QUERY_TRANSFORMED if transformed else 0, out.ctypes.data))
        return {"threads_per_query": int(out[0]), "top_level_mode": int(out[1]), "start_mode": int(out[2])}

    def capture(self, queries_ptr: int, nq: int, knn: int, ids_ptr: int, dists_ptr: int, counts_ptr: int,
                transformed: bool = False) -> "SearchGraph":
        """CUDA graph of one device search of this batch (see pdxg_graph_create)."""
        g = C.c_void_p()
        _check(library().pdxg_graph_create(self._handle().ptr, C.c_void_p(queries_ptr), nq, knn,
                                           PDXG_QUERY_TRANSFORMED if transformed else 0, C.c_void_p(ids_ptr),
                                           C.c_void_p(dists_ptr), C.c_void_p(counts_ptr), C.byref(g)))
        return SearchGraph(g, self)

    def set_probe_mode(self, mode: int) -> None:
        """0 reference probe; 1 BF16 tensor-core rotation + centroid scores, widened list, FP32
        rescore; 2 the same with FP8-E4M3 centroid scores."""
        _check(library().pdxg_set_probe_mode(self._handle().ptr, int(mode)))

    def last_visit_orders(self, nq: int, nprobe: int):
        """Visit orders computed ahead of the scan by the last search_device call."""
        orders = np.zeros((nq, nprobe), np.uint32)
        counts = np.zeros(nq, np.uint32)
        _check(library().pdxg_last_visit_orders(self._handle().ptr, nq, nprobe, orders.ctypes.data,
                                                counts.ctypes.data))
        return orders, counts

    def set_rotation_mode(self, mode: int) -> None:
        """0: tcgen05 TF32x3 rotation when available, 1: FP32 SIMT GEMM."""
        _check(library().pdxg_set_rotation_mode(self._handle().ptr, int(mode)))

    def rotation_uses_tensor_cores(self) -> bool:
        return bool(library().pdxg_rotation_uses_tensor_cores(self._handle().ptr))

    def set_threads_per_query(self, threads: int) -> None:
        _check(library().pdxg_set_threads_per_query(self._handle().ptr, int(threads)))

    def set_scan_mode(self, mode: int) -> None:
        """U8 scan after a batched Start: 0 cluster-major (default), 1 the per-query kernel only."""
        _check(library().pdxg_set_scan_mode(self._handle().ptr, int(mode)))

    def register_filter(self, row_ids: np.ndarray) -> int:
        """Keeps the filter of `row_ids` resident on the GPU (extension); returns its id for
        requests of Context.search_requests."""
        r = np.ascontiguousarray(row_ids, dtype=np.uint64)
        out = C.c_int32()
        _check(library().pdxg_filter_register(self._handle().ptr, C.c_void_p(r.ctypes.data), len(r),
                                              C.byref(out)))
        return int(out.value)

    def release_filter(self, filter_id: int) -> None:
        _check(library().pdxg_filter_release(self._handle().ptr, int(filter_id)))

    # -- persistence & getters -----------------------------------------------------------
    def save(self, path: str) -> None:
        _check(library().pdxg_save(self._handle().ptr, os.fsencode(path)))

    def get_num_dimensions(self) -> int:
        return library().pdxg_num_dimensions(self._handle().ptr) if self._h else self._d

    def get_num_clusters(self) -> int:
        return library().pdxg_num_clusters(self._handle().ptr)

    def get_cluster_size(self, cluster_id: int) -> int:
        if cluster_id >= self.get_num_clusters():
            raise ValueError("cluster_id out of range")
        return library().pdxg_cluster_size(self._handle().ptr, cluster_id)

    def get_cluster_row_ids(self, cluster_id: int) -> np.ndarray:
        n = self.get_cluster_size(cluster_id)
        out = np.empty(max(n, 1), np.uint32)
        _check(library().pdxg_cluster_row_ids(self._handle().ptr, cluster_id, out, len(out)))
        return out[:n].copy()

    def get_in_memory_size_in_bytes(self) -> int:
        return int(library().pdxg_in_memory_size_in_bytes(self._handle().ptr))

    def get_num_embeddings(self) -> int:
        return int(library().pdxg_num_embeddings(self._handle().ptr))

    @property
    def handle(self) -> Handle:
        return self._handle()

    # -- maintenance (tree indexes in the reference) -----------------------------------
    def append(self, row_id: int, embedding: np.ndarray, transformed: bool = False) -> None:
        """PDXTreeIndex::Append (index.hpp:580-616); transformed: the embedding is already
        normalized and rotated (extension)."""
        if self._type in ("pdx_f32", "pdx_u8"):
            raise RuntimeError("Append is not implemented in PDXIndex. Use PDXTreeIndex instead.")
        e = np.ascontiguousarray(embedding, dtype=np.float32)
        if e.ndim != 1:
            raise RuntimeError("embedding must be a 1D numpy array")
        if e.shape[0] != self._d:
            raise ValueError(f"embedding has {e.shape[0]} dimensions, index expects {self._d}")
        if row_id < 0:
            raise ValueError(f"Append: row_id {row_id} is not sequential")
        _check(library().pdxg_append(self._handle().ptr, int(row_id), e,
                                     PDXG_QUERY_TRANSFORMED if transformed else 0))

    def append_batch(self, first_row_id: int, embeddings: np.ndarray, transformed: bool = False) -> None:
        """Rows first_row_id, first_row_id + 1, ... appended in order (extension): the results of
        one append() per row, with one rotation and top-level search for the batch."""
        if self._type in ("pdx_f32", "pdx_u8"):
            raise RuntimeError("Append is not implemented in PDXIndex. Use PDXTreeIndex instead.")
        e = np.ascontiguousarray(embeddings, dtype=np.float32)
        if e.ndim != 2 or e.shape[1] != self._d:
            raise ValueError(f"embeddings must be n x {self._d}")
        if first_row_id < 0:
            raise ValueError(f"Append: row_id {first_row_id} is not sequential")
        _check(library().pdxg_append_batch(self._handle().ptr, int(first_row_id), e.shape[0], e,
                                           PDXG_QUERY_TRANSFORMED if transformed else 0))

    def delete(self, row_id: int) -> None:
        """PDXTreeIndex::Delete (index.hpp:619-638)."""
        if self._type in ("pdx_f32", "pdx_u8"):
            raise RuntimeError("Delete is not implemented in PDXIndex. Use PDXTreeIndex instead.")
        if row_id < 0:
            raise ValueError(f"Delete: row_id {row_id} is not in the index")
        _check(library().pdxg_delete(self._handle().ptr, int(row_id)))

    def maintenance_stats(self) -> dict:
        out = np.zeros(6, np.uint64)
        _check(library().pdxg_maintenance_stats(self._handle().ptr, out))
        keys = ("appends", "deletes", "compactions", "capacity_growths", "merges_not_performed", "tombstones")
        return {k: int(v) for k, v in zip(keys, out)}


# pdxg_request (include/pdx_b200.h)
# pdxg_request: a filter is a registered filter (filter_id >= 0) or else the row-id range
# rows[filter_begin, filter_end) (filter_id = -1 and filter_begin = NO_FILTER: unfiltered)
REQUEST_DTYPE = np.dtype([("k", np.uint32), ("nprobe", np.uint32), ("filter_begin", np.uint64),
                          ("filter_end", np.uint64), ("filter_id", np.int32), ("reserved", np.uint32)])
NO_FILTER = np.uint64(np.iinfo(np.uint64).max)


def request_table(n: int) -> np.ndarray:
    """n unfiltered requests (k and nprobe still to be filled in)."""
    t = np.zeros(n, dtype=REQUEST_DTYPE)
    t["filter_begin"] = NO_FILTER
    t["filter_end"] = NO_FILTER
    t["filter_id"] = -1
    return t


class Context:
    """A workspace + CUDA stream of one index (pdxg_context): batches issued on different
    contexts run concurrently."""

    def __init__(self, index: "PDXIndex"):
        self.index = index
        out = C.c_void_p()
        _check(library().pdxg_context_create(index.handle.ptr, C.byref(out)))
        self.ptr = out

    @property
    def stream(self) -> int:
        return int(library().pdxg_context_stream(self.ptr) or 0)

    def search_requests(self, queries_ptr: int, nq: int, requests: np.ndarray, rows: Optional[np.ndarray],
                        k_max: int, ids_ptr: int, dists_ptr: int, counts_ptr: int,
                        transformed: bool = False) -> None:
        """Enqueues a batch (device queries/outputs, host requests/rows) on this context."""
        req = np.ascontiguousarray(requests, dtype=REQUEST_DTYPE)
        rws = None if rows is None else np.ascontiguousarray(rows, dtype=np.uint32)
        _check(library().pdxg_search_requests(
            self.ptr, C.c_void_p(queries_ptr), nq, C.c_void_p(req.ctypes.data),
            C.c_void_p(rws.ctypes.data if rws is not None and len(rws) else 0), k_max,
            PDXG_QUERY_TRANSFORMED if transformed else 0, C.c_void_p(ids_ptr), C.c_void_p(dists_ptr),
            C.c_void_p(counts_ptr)))

    def close(self):
        if getattr(self, "ptr", None) and self.ptr.value and _lib is not None:
            _lib.pdxg_context_free(self.ptr)
            self.ptr = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_index(path: str, device: int = 0) -> PDXIndex:
    """Load a PDX index from a single file (auto-detects type)."""
    return PDXIndex._from_handle(_load_handle(path=path, device=device))
