"""IndexPDXIVF* wrappers with the reference's Python API (python/pdxearch/index_factory.py:10-250).

Each class owns one GPU-resident `compiled.PDXIndex`; `search` / `filtered_search` take the
same arguments and return the same (ids uint32[<=k], distances float32[<=k]) tuples. The
batched `search_batch` is an addition for throughput-oriented callers.
"""
from __future__ import annotations

import numpy as np

from .compiled import PDXIndex as _PDXIndex, load_index as _load_index

METRIC_MAP = {"l2sq": 0, "cosine": 1, "ip": 2}
DEFAULT_NPROBE = 32


class _IndexBase:
    _index_type = ""
    _tree = False

    def __init__(self, *, num_dimensions: int, distance_metric: str = "l2sq", normalize: bool = True,
                 seed: int = 42, num_clusters: int = 0, num_meso_clusters: int = 0,
                 sampling_fraction: float = 0.0, kmeans_iters: int = 10,
                 hierarchical_indexing: bool = True, n_threads: int = 0, device: int = 0) -> None:
        if not self._tree and num_meso_clusters:
            raise TypeError("num_meso_clusters applies to tree indexes only")
        self._index = _PDXIndex(self._index_type, num_dimensions, METRIC_MAP[distance_metric], seed,
                                num_clusters, num_meso_clusters if self._tree else 0, normalize,
                                sampling_fraction, kmeans_iters, hierarchical_indexing, n_threads,
                                device)

    def build(self, data: np.ndarray) -> None:
        self._index.build_index(np.ascontiguousarray(data, dtype=np.float32))

    def search(self, query: np.ndarray, knn: int, nprobe: int = DEFAULT_NPROBE):
        self._index.set_nprobe(nprobe)
        return self._index.search(np.ascontiguousarray(query, dtype=np.float32), knn)

    def search_batch(self, queries: np.ndarray, knn: int, nprobe: int = DEFAULT_NPROBE):
        """Batched search: ids [nq, k], distances [nq, k], counts [nq]."""
        self._index.set_nprobe(nprobe)
        return self._index.search_batch(np.ascontiguousarray(queries, dtype=np.float32), knn)

    def filtered_search(self, query: np.ndarray, knn: int, row_ids: np.ndarray,
                        nprobe: int = DEFAULT_NPROBE):
        self._index.set_nprobe(nprobe)
        return self._index.filtered_search(np.ascontiguousarray(query, dtype=np.float32), knn,
                                           np.ascontiguousarray(row_ids, dtype=np.uint64))

    def append(self, row_id: int, embedding: np.ndarray) -> None:
        self._index.append(row_id, np.ascontiguousarray(embedding, dtype=np.float32))

    def delete(self, row_id: int) -> None:
        self._index.delete(row_id)

    def save(self, path: str) -> None:
        self._index.save(path)

    @property
    def num_dimensions(self) -> int:
        return self._index.get_num_dimensions()

    @property
    def num_clusters(self) -> int:
        return self._index.get_num_clusters()

    @property
    def in_memory_size_bytes(self) -> int:
        return self._index.get_in_memory_size_in_bytes()


class IndexPDXIVF(_IndexBase):
    """Single-level IVF index (F32)."""
    _index_type = "pdx_f32"


class IndexPDXIVFSQ8(_IndexBase):
    """Single-level IVF index (U8 scalar quantization)."""
    _index_type = "pdx_u8"


class IndexPDXIVFTree(_IndexBase):
    """Two-level IVF index (F32)."""
    _index_type = "pdx_tree_f32"
    _tree = True


class IndexPDXIVFTreeSQ8(_IndexBase):
    """Two-level IVF index (U8 scalar quantization)."""
    _index_type = "pdx_tree_u8"
    _tree = True


def load_index(path: str, device: int = 0):
    """Load a PDX index from a single file (auto-detects type)."""
    return _load_index(path, device)
