"""Generates the golden fixtures in this directory.

For a handful of small seeded indexes (all four index types, odd and even dimensions) it
writes the index file in the reference's format, a set of queries, the queries as the
reference rotates them (ADSamplingPruner::PreprocessQuery through its sgemm_ call), and the
reference's own search results -- plain, with a fixed cluster order, filtered, and with
pruning disabled -- computed by the reference's search code compiled from its headers
(oracle/_ref/libpdx_ref.so, AVX2 flavour: exact U8 arithmetic).

Run from the repository root, where the reference sources were available to build oracle/_ref:
    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import zlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference  # noqa: E402
from pdx_b200.builder import GaussianMixture, build_index  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name, index type, d, n, nlist, n_meso, normalize, k, nprobe
CASES = [
    ("f32_d64", "pdx_f32", 64, 1200, 12, 0, False, 10, 4),
    ("u8_d100", "pdx_u8", 100, 1200, 10, 0, True, 10, 3),
    ("tree_f32_d130", "pdx_tree_f32", 130, 1000, 16, 4, True, 10, 6),
    ("tree_u8_d256", "pdx_tree_u8", 256, 1000, 16, 4, True, 20, 5),
    ("u8_d33", "pdx_u8", 33, 1500, 8, 0, False, 10, 0),
]
N_QUERIES = 12


def main():
    manifest = []
    for name, itype, d, n, nlist, nmeso, norm, k, nprobe in CASES:
        gm = GaussianMixture(d, 24, 0.4, seed=zlib.crc32(name.encode()) % 1000 + 11, unit_norm=norm)
        X = gm.sample(n, 0)
        Q = gm.sample(N_QUERIES, 1)
        f = build_index(X, itype, num_clusters=nlist, num_meso_clusters=nmeso, normalize=norm,
                        seed=5)
        path = os.path.join(OUT, f"{name}.pdx")
        f.save(path)
        ref = Reference(path)
        ref.set_nprobe(nprobe)
        Qn = Q / np.linalg.norm(Q, axis=1, keepdims=True) if norm else Q
        R = ref.rotate(Qn)
        res = {"plain_ids": [], "plain_dists": [], "raw_ids": [], "raw_dists": [],
               "order_ids": [], "order_dists": [], "filt_ids": [], "filt_dists": [],
               "exh_ids": [], "exh_dists": [], "filters": []}
        rng = np.random.default_rng(99)
        order = rng.permutation(ref.nclusters)[: max(3, ref.nclusters // 2)].astype(np.uint32)
        for i in range(N_QUERIES):
            a = ref.search(R[i], k, transformed=True)
            res["plain_ids"].append(a[0].tolist())
            res["plain_dists"].append(a[1].tolist())
            b = ref.search(Q[i], k)
            res["raw_ids"].append(b[0].tolist())
            res["raw_dists"].append(b[1].tolist())
            c = ref.search_with_order(R[i], k, order, transformed=True)
            res["order_ids"].append(c[0].tolist())
            res["order_dists"].append(c[1].tolist())
            rows = np.sort(rng.choice(n, size=max(1, int(n * rng.uniform(0.01, 0.6))), replace=False))
            res["filters"].append(rows.tolist())
            e = ref.filtered_search(R[i], k, rows, transformed=True)
            res["filt_ids"].append(e[0].tolist())
            res["filt_dists"].append(e[1].tolist())
        ref.set_pruning_aggressiveness(1e30)
        for i in range(N_QUERIES):
            g = ref.search(R[i], k, transformed=True)
            res["exh_ids"].append(g[0].tolist())
            res["exh_dists"].append(g[1].tolist())
        ref.close()
        np.save(os.path.join(OUT, f"{name}.queries.npy"), Q)
        np.save(os.path.join(OUT, f"{name}.rotated.npy"), R)
        with open(os.path.join(OUT, f"{name}.expected.json"), "w") as fh:
            json.dump({"k": k, "nprobe": nprobe, "order": order.tolist(), **res}, fh)
        manifest.append({"name": name, "type": itype, "d": d, "n": n, "k": k, "nprobe": nprobe})
        print(name, os.path.getsize(path), "bytes")
    with open(os.path.join(OUT, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1)


if __name__ == "__main__":
    main()
