"""Result comparison helpers shared by the parity tests."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_cases():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def load_golden(name):
    with open(os.path.join(GOLDEN, f"{name}.expected.json")) as f:
        exp = json.load(f)
    q = np.load(os.path.join(GOLDEN, f"{name}.queries.npy"))
    r = np.load(os.path.join(GOLDEN, f"{name}.rotated.npy"))
    return os.path.join(GOLDEN, f"{name}.pdx"), q, r, exp


def same_results(ids_a, d_a, ids_b, d_b, rtol: float = 0.0):
    """True when two top-k lists agree: distances equal (or within rtol), and ids equal as sets
    inside every group of tied distances; the tie group at the k-th distance may differ in which
    ids it keeps (the reference's heap order among equal distances is unspecified)."""
    ids_a, ids_b = np.asarray(ids_a), np.asarray(ids_b)
    d_a = np.asarray(d_a, dtype=np.float32)
    d_b = np.asarray(d_b, dtype=np.float32)
    if len(ids_a) != len(ids_b):
        return False, f"length {len(ids_a)} != {len(ids_b)}"
    if len(ids_a) == 0:
        return True, ""
    if rtol == 0.0:
        if not np.array_equal(d_a, d_b):
            bad = np.nonzero(d_a != d_b)[0]
            return False, f"distances differ at {bad[:5]}: {d_a[bad[:5]]} vs {d_b[bad[:5]]}"
    else:
        if not np.allclose(d_a, d_b, rtol=rtol, atol=0.0):
            return False, f"distances differ beyond rtol={rtol}"
        return True, ""
    last = d_a[-1]
    for v in np.unique(d_a):
        if v == last:
            continue
        sa = set(ids_a[d_a == v].tolist())
        sb = set(ids_b[d_b == v].tolist())
        if sa != sb:
            return False, f"ids differ for distance {v}: {sorted(sa)} vs {sorted(sb)}"
    return True, ""


def assert_same(ids_a, d_a, ids_b, d_b, rtol=0.0, ctx=""):
    ok, why = same_results(ids_a, d_a, ids_b, d_b, rtol)
    assert ok, f"{ctx}: {why}\n a={list(zip(np.asarray(ids_a).tolist(), np.asarray(d_a).tolist()))}\n b={list(zip(np.asarray(ids_b).tolist(), np.asarray(d_b).tolist()))}"


def recall(found, truth, k):
    return len(set(np.asarray(found)[:k].tolist()) & set(np.asarray(truth)[:k].tolist())) / max(1, min(k, len(truth)))


def dct_index(itype, d, n, nlist, nmeso=0, seed=0):
    """An index whose file stores the FFTW-style rotation: a 1 x d sign vector (flip where
    negative) followed by the orthonormal DCT-II. The data are rotated with the same transform
    in float64 (scipy.fft.dct, norm="ortho")."""
    import scipy.fft
    from pdx_b200.builder import GaussianMixture, build_index
    rng = np.random.default_rng(seed)
    signs = np.where(rng.random(d) < 0.5, -1.0, 1.0).astype(np.float32)
    # dense form of x -> dct(x * s): rows j of the matrix are the images of the unit vectors
    dense = scipy.fft.dct(np.diag(signs.astype(np.float64)), type=2, norm="ortho", axis=1).astype(np.float32)
    gm = GaussianMixture(d, 20, 0.4, seed=seed + 1, unit_norm=True)
    X = gm.sample(n, 0)
    Q = gm.sample(64, 1)
    f = build_index(X, itype, num_clusters=nlist, num_meso_clusters=nmeso, normalize=True, seed=seed,
                    rotation=dense)
    f.rotation = signs.reshape(1, d)
    return f, Q, signs


def dct_rotate(Q, signs, normalize=True):
    import scipy.fft
    Q = Q.astype(np.float64)
    if normalize:
        Q = Q / np.linalg.norm(Q, axis=1, keepdims=True)
    return scipy.fft.dct(Q * signs.astype(np.float64)[None, :], type=2, norm="ortho", axis=1)
