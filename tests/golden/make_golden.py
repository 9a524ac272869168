"""Regenerates the golden fixtures of this directory from the reference itself.

Runs the reference's own CPU tree code, compiled from its sources by
`make -C oracle ref` (oracle/_ref/libref_tree.so): its AppData point
generator and its per-element functions wired with the canonical dataflow
(oracle/ref_driver.cpp).  Usage, from the repository root, where the
reference sources are present:

    make -C oracle && python tests/golden/make_golden.py

Writes:
  config1_kat.json  - the reference's default cloud (n = 640*480,
                      mt19937(114514)): counts and an FNV-1a-64 digest of every
                      output array.
  small_cases.npz   - small clouds (duplicates, clusters, odd sizes) with every
                      canonical output array in full.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import Oracle, RefTree  # noqa: E402

FIELDS = ("sorted_keys", "unique_keys", "prefix_n", "has_leaf_left", "has_leaf_right",
          "left_child", "parents", "edge_count", "edge_offset", "children", "corner",
          "cell_size", "child_node_mask", "child_leaf_mask")


def digests(res, orc):
    t = res.trimmed()
    out = {k: f"{orc.fnv1a64(np.ascontiguousarray(t[k])):#018x}" for k in FIELDS}
    out["morton_keys"] = f"{orc.fnv1a64(res.morton_keys):#018x}"
    return out


def small_inputs():
    rng = np.random.default_rng(20240601)
    cases = {}
    # coarse grid -> heavy duplicates
    for n in (5, 31, 32, 33, 100, 1000, 1025, 4097):
        p = np.zeros((n, 4), np.float32)
        p[:, :3] = rng.integers(0, 64, size=(n, 3)).astype(np.float32) * 16.0
        p[:, 3] = 1.0
        cases[f"grid_{n}"] = p
    # clusters with fractional coordinates
    for n in (257, 3000):
        c = rng.uniform(0, 1024, size=(4, 3))
        k = rng.integers(0, 4, size=n)
        p = np.zeros((n, 4), np.float32)
        p[:, :3] = np.clip(c[k] + rng.normal(0, 3.0, size=(n, 3)), 0,
                           np.nextafter(np.float32(1024), np.float32(0)))
        p[:, 3] = 1.0
        cases[f"cluster_{n}"] = p
    # edges of the box: exactly min and the largest float below min+range
    p = np.zeros((64, 4), np.float32)
    top = np.nextafter(np.float32(1024), np.float32(0))
    p[:, :3] = rng.choice(np.array([0.0, top, 512.0, 1.0, 1023.0], np.float32), size=(64, 3))
    p[:, 3] = 1.0
    cases["box_edges_64"] = p
    return cases


def main():
    ref, orc = RefTree(), Oracle()
    pts = ref.default_points(640 * 480)
    res = ref.canonical(pts)
    assert res.status == 0, res.status
    kat = {
        "n_input": 640 * 480,
        "generator": "AppData: std::mt19937(114514), uniform_real_distribution<float>(0,1024), "
                     "draws z, y, x per point (g++ argument order), w = 1",
        "points_fnv1a64": f"{orc.fnv1a64(pts):#018x}",
        "n_unique": res.n_unique,
        "n_brt_nodes": res.n_brt_nodes,
        "n_octree_nodes": res.n_octree_nodes,
        "prefix_n0": int(res.prefix_n[0]),
        "edge_count0": int(res.edge_count[0]),
        "edge_offset_last": int(res.edge_offset[res.n_brt_nodes - 1]),
        "child_slots_written": int(sum(bin(int(x) & 0xffffffff).count("1")
                                       for x in res.child_node_mask[:res.n_octree_nodes + 1])),
        "fnv1a64": digests(res, orc),
    }
    with open(os.path.join(HERE, "config1_kat.json"), "w") as f:
        json.dump(kat, f, indent=1, sort_keys=True)

    arrays = {}
    for name, p in small_inputs().items():
        r = ref.canonical(p)
        arrays[f"{name}/points"] = p
        arrays[f"{name}/status"] = np.array([r.status], np.int32)
        arrays[f"{name}/counts"] = np.array([r.n_unique, r.n_brt_nodes, r.n_octree_nodes], np.uint32)
        arrays[f"{name}/morton_keys"] = r.morton_keys
        t = r.trimmed()
        for k in FIELDS:
            if k in t:
                arrays[f"{name}/{k}"] = np.ascontiguousarray(t[k])
    np.savez_compressed(os.path.join(HERE, "small_cases.npz"), **arrays)
    print("wrote", len(arrays), "arrays;", kat["n_unique"], kat["n_octree_nodes"])


if __name__ == "__main__":
    main()
