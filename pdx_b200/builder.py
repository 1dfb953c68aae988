"""Index construction for the PDX layout: seeded synthetic data, rotation, k-means, SQ8, files.

The reference builds with SuperKMeans (an absent submodule); this builder follows the same
pipeline as `PDXIndex::BuildIndex` / `PDXTreeIndex::BuildIndex` (index.hpp:329-403, 640-758):
normalize (optional) -> rotate with a random orthogonal matrix -> global SQ8 parameters (U8
only) -> k-means into nlist clusters -> PDX blocks; the tree adds a second k-means over the L1
centroids into sqrt(nlist) meso-clusters whose PDX "vectors" are the L1 centroids.

Clustering uses plain Lloyd iterations (k-means++-free, seeded sample init). The search engine
only needs *a* valid index in the reference's format; clustering quality parity with SuperKMeans
is out of scope. The heavy assignment step runs on the GPU through torch when a device is
given, else in numpy.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .layout import (INDEX_TYPES, IndexFile, Level, dimension_split, quantization_params,
                     quantize)


# ----------------------------------------------------------------------------- synthetic data

class GaussianMixture:
    """Isotropic Gaussian mixture: centres ~ N(0, 1), per-point noise sigma."""

    def __init__(self, d: int, n_components: int, sigma: float, seed: int,
                 unit_norm: bool = False):
        self.d = d
        self.sigma = np.float32(sigma)
        self.unit_norm = unit_norm
        rng = np.random.default_rng(seed)
        self.centres = rng.standard_normal((n_components, d), dtype=np.float32)
        self.seed = seed

    def sample(self, n: int, stream: int) -> np.ndarray:
        """n points of sample stream `stream`; sample(m, s) is a prefix of sample(n, s), m <= n."""
        out = np.empty((n, self.d), dtype=np.float32)
        chunk = 1 << 16
        for c, s in enumerate(range(0, n, chunk)):
            e = min(n, s + chunk)
            labels = np.random.default_rng([self.seed, stream, c, 0]).integers(
                0, self.centres.shape[0], e - s)
            x = np.random.default_rng([self.seed, stream, c, 1]).standard_normal(
                (e - s, self.d), dtype=np.float32)
            x *= self.sigma
            x += self.centres[labels]
            if self.unit_norm:
                x /= np.linalg.norm(x, axis=1, keepdims=True).astype(np.float32)
            out[s:e] = x
        return out


def random_rotation(d: int, seed: int) -> np.ndarray:
    """Random orthogonal d x d matrix (QR of a Gaussian matrix in float64, stored f32)."""
    rng = np.random.default_rng([seed, 7919])
    g = rng.standard_normal((d, d))
    q, r = np.linalg.qr(g)
    q *= np.sign(np.diag(r))[None, :]
    return q.astype(np.float32)


def normalize_rows(x: np.ndarray) -> np.ndarray:
    """NormalizeQuery over rows (scalar.hpp:23-40); all-zero rows are left unchanged."""
    x = np.asarray(x, dtype=np.float32)
    s = np.sqrt(np.einsum("ij,ij->i", x, x, dtype=np.float32)).astype(np.float32)
    s[s == 0] = 1.0
    return (x / s[:, None]).astype(np.float32)


def compute_num_clusters(n: int) -> int:
    """ComputeNumberOfClusters (common.hpp:191-199)."""
    if n < 500000:
        return int(math.ceil(2 * math.sqrt(n)))
    if n < 2500000:
        return int(math.ceil(4 * math.sqrt(n)))
    return int(math.ceil(8 * math.sqrt(n)))


# ----------------------------------------------------------------------------- k-means

def _assign_numpy(x: np.ndarray, c: np.ndarray) -> np.ndarray:
    cn = np.einsum("ij,ij->i", c, c)
    out = np.empty(x.shape[0], dtype=np.int64)
    step = 1 << 14
    for s in range(0, x.shape[0], step):
        xs = x[s:s + step]
        dots = xs @ c.T
        out[s:s + step] = np.argmin(cn[None, :] - 2.0 * dots, axis=1)
    return out


def kmeans(x: np.ndarray, k: int, iters: int = 10, seed: int = 42, device: Optional[str] = None,
           angular: bool = False):
    """Lloyd k-means. Returns (centroids f32 [k, d], assignment int64 [n]).

    angular: spherical k-means (unit-norm centroids, nearest = largest inner product), what the
    reference's SuperKMeans does for normalized data (clustering.hpp:55-56). Without it, plain
    L2 Lloyd on unit vectors lets the smallest-norm centroid absorb most points. Empty clusters
    are re-seeded from random points.
    """
    n, d = x.shape
    rng = np.random.default_rng([seed, 104729])
    init = rng.choice(n, size=k, replace=False) if k <= n else rng.integers(0, n, k)
    if device is not None:
        import torch
        xt = torch.from_numpy(np.ascontiguousarray(x)).to(device)
        ct = xt[torch.from_numpy(init).to(device)].clone()
        gen = torch.Generator(device="cpu").manual_seed(int(seed) * 7 + 3)

        def norm_rows(c):
            return c / c.norm(dim=1, keepdim=True).clamp(min=1e-30)

        if angular:
            ct = norm_rows(ct)
        step = max(1, (1 << 28) // max(1, k))
        for it in range(iters + 1):
            cn = (ct * ct).sum(1)
            assign = torch.empty(n, dtype=torch.int64, device=device)
            for s0 in range(0, n, step):
                xs = xt[s0:s0 + step]
                assign[s0:s0 + step] = torch.argmin(cn[None, :] - 2.0 * (xs @ ct.T), dim=1)
            if it == iters:
                break
            sums = torch.zeros_like(ct).index_add_(0, assign, xt)
            cnt = torch.bincount(assign, minlength=k).to(ct.dtype)
            empty = cnt == 0
            new_c = sums / cnt.clamp(min=1)[:, None]
            if bool(empty.any()):
                ridx = torch.randint(0, n, (int(empty.sum()),), generator=gen).to(device)
                new_c[empty] = xt[ridx]
            ct = norm_rows(new_c) if angular else new_c
        return ct.float().cpu().numpy(), assign.cpu().numpy()
    c = x[init].astype(np.float32).copy()

    def norm_np(c):
        nrm = np.linalg.norm(c, axis=1, keepdims=True)
        nrm[nrm == 0] = 1.0
        return (c / nrm).astype(np.float32)

    if angular:
        c = norm_np(c)
    for it in range(iters + 1):
        assign = _assign_numpy(x, c)
        if it == iters:
            break
        cnt = np.bincount(assign, minlength=k)
        sums = np.zeros_like(c, dtype=np.float64)
        np.add.at(sums, assign, x)
        nz = cnt > 0
        c[nz] = (sums[nz] / cnt[nz, None]).astype(np.float32)
        if (~nz).any():
            c[~nz] = x[rng.integers(0, n, int((~nz).sum()))]
        if angular:
            c = norm_np(c)
    return c, assign


# ----------------------------------------------------------------------------- index build

def _split_by_assignment(values: np.ndarray, row_ids: np.ndarray, assign: np.ndarray, k: int):
    order = np.argsort(assign, kind="stable")
    bounds = np.searchsorted(assign[order], np.arange(k + 1))
    embs, ids = [], []
    for c in range(k):
        sel = order[bounds[c]:bounds[c + 1]]
        embs.append(np.ascontiguousarray(values[sel]))
        ids.append(row_ids[sel].astype(np.uint32))
    return embs, ids


def build_index(data: np.ndarray, index_type: str = "pdx_f32", num_clusters: int = 0,
                num_meso_clusters: int = 0, normalize: bool = False, seed: int = 42,
                kmeans_iters: int = 10, rotation: Optional[np.ndarray] = None,
                device: Optional[str] = None) -> IndexFile:
    """Builds an index in the reference's file layout from row-major float32 data."""
    if index_type not in INDEX_TYPES:
        raise ValueError(f"Unknown index type: {index_type}")
    itype = INDEX_TYPES[index_type]
    data = np.ascontiguousarray(data, dtype=np.float32)
    n, d = data.shape
    if num_clusters == 0:
        num_clusters = compute_num_clusters(n)
    if num_clusters > n:
        raise ValueError(f"num_clusters ({num_clusters}) exceeds num_embeddings ({n})")
    if rotation is None:
        rotation = random_rotation(d, seed)
    x = normalize_rows(data) if normalize else data
    rot = _rotate(x, rotation, device)
    del x
    base, scale = 0.0, 1.0
    is_u8 = itype in (1, 3)
    if is_u8:
        base, scale = quantization_params(rot)
    cents, assign = kmeans(rot, num_clusters, kmeans_iters, seed, device, angular=normalize)
    stored = _quantize(rot, base, scale, device) if is_u8 else rot
    row_ids = np.arange(n, dtype=np.uint32)
    embs, ids = _split_by_assignment(stored, row_ids, assign, num_clusters)
    l1 = Level(embs, ids, cents)
    l0 = None
    if itype >= 2:
        n0 = num_meso_clusters or int(math.sqrt(num_clusters))
        if n0 >= num_clusters:
            raise ValueError("num_meso_clusters must be smaller than num_clusters")
        c0, a0 = kmeans(cents, n0, 10, seed, None, angular=normalize)
        e0, i0 = _split_by_assignment(cents, np.arange(num_clusters, dtype=np.uint32), a0, n0)
        l0 = Level(e0, i0, c0)
    return IndexFile(itype, rotation, d, l1, l0, bool(normalize), float(base), float(scale))


def _quantize(x: np.ndarray, base: float, scale: float, device: Optional[str]) -> np.ndarray:
    """quantize() of layout.py, chunked on the GPU when a device is given (same float32 steps,
    round half away from zero)."""
    if device is None:
        return quantize(x, base, scale)
    import torch
    out = np.empty(x.shape, dtype=np.uint8)
    b = torch.tensor(np.float32(base), device=device)
    s = torch.tensor(np.float32(scale), device=device)
    step = 1 << 17
    for i in range(0, x.shape[0], step):
        v = (torch.from_numpy(x[i:i + step]).to(device) - b) * s
        v64 = v.double()
        r = torch.trunc(v64 + torch.copysign(torch.full_like(v64, 0.5), v64))
        out[i:i + step] = r.clamp(0, 255).to(torch.uint8).cpu().numpy()
    return out


def _rotate(x: np.ndarray, rotation: np.ndarray, device: Optional[str]) -> np.ndarray:
    """Row form of y = M^T x (adsampling.hpp:225-245): Y = X @ M."""
    if device is not None:
        import torch
        out = np.empty_like(x)
        mt = torch.from_numpy(rotation).to(device).double()
        step = 1 << 17
        for s in range(0, x.shape[0], step):
            xs = torch.from_numpy(x[s:s + step]).to(device).double()
            out[s:s + step] = (xs @ mt).float().cpu().numpy()
        return out
    return (x.astype(np.float64) @ rotation.astype(np.float64)).astype(np.float32)
