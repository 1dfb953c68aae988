"""PDX layout constants and the serialized index format (reader/writer side in numpy).

The byte layout is the reference's `Save` format, kept identical so files move freely between
the reference library and this engine:

* header: ``u8 type`` (0 F32, 1 U8, 2 TREE_F32, 3 TREE_U8), ``u32 rows, u32 cols``, then the
  row-major ``f32[rows*cols]`` rotation matrix (index.hpp:213-239, 483-514).
* flat payload (ivf_wrapper.hpp:133-165): ``u32 d, d_v, d_h, nlist``; ``nlist x {u32 n,
  u32 max_capacity}``; every cluster's compact PDX block; every cluster's ``u32[n]`` row ids;
  ``u8 is_normalized``; ``f32[nlist*d]`` centroids; U8 only ``f32 base, f32 scale``.
* tree payload (ivf_wrapper.hpp:314-380): ``u32 d, d_v, d_h, n_l1, n_l0``; the L0 level
  (always F32, its vectors are the L1 centroids, its row ids the L1 cluster ids) as headers,
  blocks and ids; the L1 level likewise; ``u8 is_normalized``; ``f32[n_l0*d]`` meso
  centroids; U8 only ``f32 base, f32 scale``. No L1 centroid array is stored.
* compact PDX block of one cluster (cluster.hpp:185-221): F32 -- ``d_v`` dimension rows of
  ``n`` floats, then ``d_h/64`` row-major ``n x 64`` blocks; U8 -- ``d_v//4`` groups of
  ``n x 4`` bytes (4 dims interleaved per vector), an ``n x (d_v % 4)`` tail, then the
  ``n x 64`` byte blocks.
"""
from __future__ import annotations

import io
import math
import struct
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

H_DIM_SIZE = 64  # common.hpp:45
U8_INTERLEAVE_SIZE = 4  # common.hpp:46
PDX_MAX_DIMS = 16384  # common.hpp:44
DIMENSIONS_FETCHING_SIZES = (16, 16, 32, 32, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128,
                             256, 256, 512, 1024, 2048, 16384)  # common.hpp:47-49
ADSAMPLING_EPSILON0 = 1.5  # common.hpp:67
SELECTIVITY_THRESHOLD = np.float32(0.80)  # searcher.hpp:57

INDEX_TYPES = {"pdx_f32": 0, "pdx_u8": 1, "pdx_tree_f32": 2, "pdx_tree_u8": 3}
TYPE_NAMES = {v: k for k, v in INDEX_TYPES.items()}


def dimension_split(d: int):
    """(horizontal, vertical) dims of GetPDXDimensionSplit (common.hpp:133-159)."""
    prop = np.float32(0.75) if d > 128 else np.float32(0.25)
    h = int(np.float32(d) * prop)
    v = d - h
    if h % H_DIM_SIZE > 0:
        h = ((h + H_DIM_SIZE // 2) // H_DIM_SIZE) * H_DIM_SIZE
        v = d - h
    if not v:
        h = H_DIM_SIZE
        v = d - h
    if d <= H_DIM_SIZE:
        h, v = 0, d
    return h, v


def adsampling_ratio(visited: int, d: int, eps0: float = ADSAMPLING_EPSILON0) -> np.float32:
    """ADSamplingPruner::GetRatio (adsampling.hpp:147-157), same float/double steps."""
    if visited == 0 or visited == d:
        return np.float32(1.0)
    a = 1.0 + float(np.float32(eps0)) / math.sqrt(visited)
    r = float(np.float32(visited) / np.float32(d))
    return np.float32(r * a * a)


def max_capacity(n: int) -> int:
    """Cluster::max_capacity = max(uint32(n * 1.3f), 256) (cluster.hpp:22-33)."""
    return max(int(np.float32(n) * np.float32(1.3)), 256)


def round_half_away(x: np.ndarray) -> np.ndarray:
    """std::round on float32 values, exactly (half away from zero)."""
    x64 = np.asarray(x, dtype=np.float32).astype(np.float64)
    return np.trunc(x64 + np.copysign(0.5, x64))


def quantize(x: np.ndarray, base: float, scale: float) -> np.ndarray:
    """ScalarQuantizer::QuantizeEmbedding (scalar.hpp:76-94) in float32."""
    v = (np.asarray(x, dtype=np.float32) - np.float32(base)) * np.float32(scale)
    r = round_half_away(v)
    return np.clip(r, 0, 255).astype(np.uint8)


def quantization_params(x: np.ndarray):
    """Global min/max parameters (scalar.hpp:60-74): base = min, scale = 255 / range."""
    lo = np.float32(np.min(x))
    hi = np.float32(np.max(x))
    rng = np.float32(hi - lo)
    scale = np.float32(np.float32(255.0) / rng) if rng > 0 else np.float32(1.0)
    return lo, scale


def pdx_block_bytes(emb: np.ndarray, d_v: int, d_h: int) -> bytes:
    """Compact PDX block of one cluster from its row-major embeddings (cluster.hpp:185-221)."""
    n = emb.shape[0]
    out = io.BytesIO()
    if emb.dtype == np.float32:
        out.write(np.ascontiguousarray(emb[:, :d_v].T).tobytes())
    else:
        g = 0
        while g + U8_INTERLEAVE_SIZE <= d_v:
            out.write(np.ascontiguousarray(emb[:, g:g + U8_INTERLEAVE_SIZE]).tobytes())
            g += U8_INTERLEAVE_SIZE
        if g < d_v:
            out.write(np.ascontiguousarray(emb[:, g:d_v]).tobytes())
    for j in range(0, d_h, H_DIM_SIZE):
        out.write(np.ascontiguousarray(emb[:, d_v + j:d_v + j + H_DIM_SIZE]).tobytes())
    assert n == 0 or out.tell() == emb.nbytes
    return out.getvalue()


@dataclass
class Level:
    """One IVF level: per-cluster row-major embeddings (f32 or u8) and row ids."""
    embeddings: List[np.ndarray]
    row_ids: List[np.ndarray]
    centroids: Optional[np.ndarray] = None  # f32 [nclusters, d]
    max_caps: Optional[List[int]] = None

    @property
    def nclusters(self) -> int:
        return len(self.embeddings)

    def caps(self) -> List[int]:
        if self.max_caps is not None:
            return list(self.max_caps)
        return [max_capacity(e.shape[0]) for e in self.embeddings]


@dataclass
class IndexFile:
    index_type: int
    rotation: np.ndarray  # f32 [d, d]
    d: int
    l1: Level
    l0: Optional[Level] = None
    is_normalized: bool = False
    base: float = 0.0
    scale: float = 1.0
    extra: dict = field(default_factory=dict)

    def to_bytes(self) -> bytes:
        d = self.d
        d_h, d_v = dimension_split(d)
        out = io.BytesIO()
        rot = np.ascontiguousarray(self.rotation, dtype=np.float32)
        out.write(struct.pack("<BII", self.index_type, rot.shape[0], rot.shape[1]))
        out.write(rot.tobytes())
        tree = self.index_type >= 2
        if not tree:
            out.write(struct.pack("<IIII", d, d_v, d_h, self.l1.nclusters))
            _write_level(out, self.l1, d_v, d_h)
            out.write(struct.pack("<B", 1 if self.is_normalized else 0))
            out.write(np.ascontiguousarray(self.l1.centroids, dtype=np.float32).tobytes())
        else:
            out.write(struct.pack("<IIIII", d, d_v, d_h, self.l1.nclusters, self.l0.nclusters))
            _write_level(out, self.l0, d_v, d_h)
            _write_level(out, self.l1, d_v, d_h)
            out.write(struct.pack("<B", 1 if self.is_normalized else 0))
            out.write(np.ascontiguousarray(self.l0.centroids, dtype=np.float32).tobytes())
        if self.index_type in (1, 3):
            out.write(struct.pack("<ff", float(self.base), float(self.scale)))
        return out.getvalue()

    def save(self, path: str) -> None:
        with open(path, "wb") as f:
            f.write(self.to_bytes())


def _write_level(out, lv: Level, d_v: int, d_h: int) -> None:
    caps = lv.caps()
    for e, c in zip(lv.embeddings, caps):
        out.write(struct.pack("<II", e.shape[0], c))
    for e in lv.embeddings:
        out.write(pdx_block_bytes(e, d_v, d_h))
    for ids in lv.row_ids:
        out.write(np.ascontiguousarray(ids, dtype=np.uint32).tobytes())


def read_index(buf: bytes) -> IndexFile:
    """Parses a serialized index back into row-major per-cluster embeddings."""
    mv = memoryview(buf)
    itype, rows, cols = struct.unpack_from("<BII", mv, 0)
    p = 9
    rot = np.frombuffer(mv, dtype=np.float32, count=rows * cols, offset=p).reshape(rows, cols)
    p += 4 * rows * cols
    is_u8 = itype in (1, 3)
    if itype < 2:
        d, d_v, d_h, ncl = struct.unpack_from("<IIII", mv, p)
        p += 16
        l1, p = _read_level(mv, p, d, d_v, d_h, ncl, is_u8)
        norm = mv[p]
        p += 1
        l1.centroids = np.frombuffer(mv, dtype=np.float32, count=ncl * d, offset=p).reshape(ncl, d).copy()
        p += 4 * ncl * d
        l0 = None
    else:
        d, d_v, d_h, n1, n0 = struct.unpack_from("<IIIII", mv, p)
        p += 20
        l0, p = _read_level(mv, p, d, d_v, d_h, n0, False)
        l1, p = _read_level(mv, p, d, d_v, d_h, n1, is_u8)
        norm = mv[p]
        p += 1
        l0.centroids = np.frombuffer(mv, dtype=np.float32, count=n0 * d, offset=p).reshape(n0, d).copy()
        p += 4 * n0 * d
    base, scale = 0.0, 1.0
    if is_u8:
        base, scale = struct.unpack_from("<ff", mv, p)
        p += 8
    if p != len(buf):
        raise ValueError(f"trailing bytes in index file: parsed {p} of {len(buf)}")
    return IndexFile(itype, rot.copy(), d, l1, l0, bool(norm), base, scale)


def _read_level(mv, p, d, d_v, d_h, ncl, is_u8):
    hdr = np.frombuffer(mv, dtype=np.uint32, count=2 * ncl, offset=p).reshape(ncl, 2)
    p += 8 * ncl
    embs = []
    for i in range(ncl):
        n = int(hdr[i, 0])
        if is_u8:
            raw = np.frombuffer(mv, dtype=np.uint8, count=n * d, offset=p)
            e = np.empty((n, d), dtype=np.uint8)
            q = 0
            g = 0
            while g + 4 <= d_v:
                e[:, g:g + 4] = raw[q:q + 4 * n].reshape(n, 4)
                q += 4 * n
                g += 4
            if g < d_v:
                r = d_v - g
                e[:, g:d_v] = raw[q:q + r * n].reshape(n, r)
                q += r * n
            for j in range(0, d_h, H_DIM_SIZE):
                e[:, d_v + j:d_v + j + H_DIM_SIZE] = raw[q:q + 64 * n].reshape(n, 64)
                q += 64 * n
            p += n * d
        else:
            raw = np.frombuffer(mv, dtype=np.float32, count=n * d, offset=p)
            e = np.empty((n, d), dtype=np.float32)
            e[:, :d_v] = raw[:d_v * n].reshape(d_v, n).T
            q = d_v * n
            for j in range(0, d_h, H_DIM_SIZE):
                e[:, d_v + j:d_v + j + H_DIM_SIZE] = raw[q:q + 64 * n].reshape(n, 64)
                q += 64 * n
            p += 4 * n * d
        embs.append(e)
    ids = []
    for i in range(ncl):
        n = int(hdr[i, 0])
        ids.append(np.frombuffer(mv, dtype=np.uint32, count=n, offset=p).copy())
        p += 4 * n
    return Level(embs, ids, None, [int(c) for c in hdr[:, 1]]), p
