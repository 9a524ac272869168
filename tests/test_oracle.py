"""The oracle (oracle/tree_oracle.c) pinned against the reference.

Two pins: the committed golden fixtures (made by tests/golden/make_golden.py
from the reference's own CPU code) and, where oracle/_ref is built, the
reference's functions run live on fresh inputs.  CPU only.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR
from oracle import (ORC_ERR_CAPACITY, ORC_ERR_DEGENERATE, ORC_OK, RefTree, compare,
                    octree_capacity, ref_available)

FIELDS = ("sorted_keys", "unique_keys", "prefix_n", "has_leaf_left", "has_leaf_right",
          "left_child", "parents", "edge_count", "edge_offset", "children", "corner",
          "cell_size", "child_node_mask", "child_leaf_mask")


def _kat():
    with open(os.path.join(GOLDEN_DIR, "config1_kat.json")) as f:
        return json.load(f)


def _small_cases():
    z = np.load(os.path.join(GOLDEN_DIR, "small_cases.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    return z, names


def config1_points(rw=None):
    """The reference's default cloud, from the product's generator."""
    if rw is None:
        from conftest import load_package
        rw = load_package()
    return rw.generate_points(640 * 480, rw.GEN_APPDATA, 114514)


def test_capacity_matches_appdata():
    # floor(n * 0.6f) in float, app_data.hpp:13,28
    assert octree_capacity(640 * 480) == 184320
    assert octree_capacity(16777216) == int(np.float32(16777216) * np.float32(0.6))
    assert octree_capacity(5) == 3


def test_config1_generator_matches_reference_fixture(rw, oracle):
    pts = config1_points(rw)
    assert f"{oracle.fnv1a64(pts):#018x}" == _kat()["points_fnv1a64"]


def test_config1_kat(rw, oracle):
    kat = _kat()
    res = oracle.run(config1_points(rw))
    assert res.status == ORC_OK
    assert res.n_unique == kat["n_unique"] == 307151
    assert res.n_brt_nodes == kat["n_brt_nodes"]
    assert res.n_octree_nodes == kat["n_octree_nodes"] == 150716
    assert int(res.prefix_n[0]) == kat["prefix_n0"] == 1
    assert int(res.edge_count[0]) == kat["edge_count0"] == 0
    assert int(res.edge_offset[res.n_brt_nodes - 1]) == kat["edge_offset_last"] == 150715
    t = res.trimmed()
    for k in FIELDS:
        assert f"{oracle.fnv1a64(np.ascontiguousarray(t[k])):#018x}" == kat["fnv1a64"][k], k
    assert f"{oracle.fnv1a64(res.morton_keys):#018x}" == kat["fnv1a64"]["morton_keys"]


def test_small_golden_cases(oracle):
    z, names = _small_cases()
    assert len(names) >= 10
    for name in names:
        res = oracle.run(z[f"{name}/points"])
        assert res.status == int(z[f"{name}/status"][0]), name
        assert [res.n_unique, res.n_brt_nodes, res.n_octree_nodes] == list(z[f"{name}/counts"]) \
            or res.status != ORC_OK, name
        assert res.morton_keys.tobytes() == z[f"{name}/morton_keys"].tobytes(), name
        t = res.trimmed()
        for k in FIELDS:
            key = f"{name}/{k}"
            if key in z.files:
                assert np.ascontiguousarray(t[k]).tobytes() == z[key].tobytes(), (name, k)


def test_oracle_sort_is_stable_ascending(oracle):
    rng = np.random.default_rng(1)
    for bits, dt in ((32, np.uint32), (64, np.uint64)):
        top = (1 << 30) if bits == 32 else (1 << 63)
        keys = rng.integers(0, top, size=10007, dtype=np.uint64).astype(dt)
        assert np.array_equal(oracle.sort(keys), np.sort(keys))


def test_oracle_morton_bit_layout(oracle):
    # one set bit per axis lands at 3b, 3b+1, 3b+2 (func_morton.hpp:15-39)
    pts = np.zeros((3, 4), np.float32)
    pts[0, 0] = 1.0  # x bit 0
    pts[1, 1] = 2.0  # y bit 1
    pts[2, 2] = 512.0  # z bit 9
    k = oracle.morton(pts)
    assert list(k) == [1 << 0, 1 << 4, 1 << 29]
    k64 = oracle.morton(pts, key_bits=64)
    # 21 bits per axis: 1.0 * 2^21 / 1024 = 2048 = bit 11 of x
    assert list(k64) == [1 << 33, 1 << 37, 1 << 62]


def test_degenerate_inputs(oracle):
    pts = np.zeros((10, 4), np.float32)
    res = oracle.run(pts)  # one distinct key
    assert res.status == ORC_ERR_DEGENERATE and res.n_unique == 1
    pts[:5, 0] = 100.0  # two distinct keys
    assert oracle.run(pts).status == ORC_ERR_DEGENERATE
    pts[:2, 1] = 700.0  # three distinct keys: the smallest tree
    res = oracle.run(pts)
    assert res.status == ORC_OK and res.n_unique == 3


def test_capacity_overflow_reported(oracle):
    rng = np.random.default_rng(3)
    pts = np.zeros((2000, 4), np.float32)
    pts[:, :3] = rng.uniform(0, 1024, size=(2000, 3))
    assert oracle.run(pts, capacity=2).status == ORC_ERR_CAPACITY


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (no reference sources)")
def test_oracle_matches_reference_live():
    """Fresh seeded clouds: the restatement equals the reference's functions."""
    from oracle import Oracle
    ref, orc = RefTree(), Oracle()
    rng = np.random.default_rng(7)
    for n, spread in ((3, 1024), (17, 1024), (300, 8), (5000, 1024), (20000, 40), (100000, 1024)):
        pts = np.zeros((n, 4), np.float32)
        pts[:, :3] = np.clip(rng.normal(512, spread, size=(n, 3)), 0,
                             np.nextafter(np.float32(1024), np.float32(0)))
        pts[:, 3] = 1.0
        a, b = orc.run(pts), ref.canonical(pts)
        assert a.status == b.status, n
        assert (a.n_unique, a.n_octree_nodes) == (b.n_unique, b.n_octree_nodes), n
        assert compare(a, b) == [], n


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (no reference sources)")
def test_reference_verbatim_stage1_equals_oracle(rw):
    """The verbatim reference path's Morton keys equal the oracle's."""
    from oracle import Oracle
    ref = RefTree()
    pts = config1_points(rw)
    keys, n_unique, _ = ref.verbatim(pts, 4)
    assert np.array_equal(keys, Oracle().morton(pts))
    assert n_unique == 307151


@pytest.mark.parametrize("kind,kw", [(1, {}), (2, dict(n_components=32, sigma_lo=4.0,
                                                        sigma_hi=40.0)),
                                     (2, dict(n_components=9, sigma_lo=2.0, sigma_hi=20.0))])
def test_oracle_generators_equal_the_library(rw, oracle, kind, kw):
    """The C restatement of the counter-based generators gives the library's
    clouds byte for byte (the reference arm of the benchmark relies on it)."""
    for n, seed in ((1, 3), (1000, 20260101), (70001, 7)):
        want = rw.generate_points(n, kind, seed, **kw)
        got = oracle.generate_points(n, kind, seed, **kw)
        assert got.tobytes() == want.tobytes(), (kind, n, seed)


def _oracle_linked(oracle, pts, **kw):
    from oracle import OPT_LINK_LEAVES
    return oracle.run(pts, options=OPT_LINK_LEAVES, **kw)


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_leaf_links_equal_the_reference_function(rw, oracle):
    """The restated leaf linker equals the reference's own process_link_leaf
    (func_octree.hpp:114-163) run after the canonical stage 7, on every output,
    on clouds where the reference's unbounded walk ends."""
    ref = RefTree()
    compared = 0
    for i, (n, kind) in enumerate(((307200, "appdata"), (50000, "uniform"), (65537, "gauss"),
                                   (4096, "gauss"), (200000, "uniform"))):
        if kind == "appdata":
            pts = ref.default_points(n)
        elif kind == "uniform":
            pts = rw.generate_points(n, rw.GEN_UNIFORM, 900 + i)
        else:
            pts = rw.generate_points(n, rw.GEN_GAUSSIAN_MIXTURE, 900 + i, n_components=6,
                                     sigma_lo=2.0, sigma_hi=20.0)
        want = ref.canonical(pts, link_leaves=True)
        if want.status == 4:
            continue
        assert want.status == ORC_OK
        got = _oracle_linked(oracle, pts)
        assert compare(got, want) == [], (n, kind)
        # the links did change the octree relative to the default contract
        plain = oracle.run(pts)
        assert plain.trimmed()["children"].tobytes() != got.trimmed()["children"].tobytes()
        compared += 1
    assert compared >= 3


def _octree_is_nested(res, key_bits):
    """Geometric check of an octree: every child link (node mask bit set)
    names a row whose cell is half its parent's and lies in the parent's
    octant `which`; returns the number of violations.  Row 0 is left out as a
    parent: the reference's layout gives it the root's links but the corner
    and cell size of the first chain node (edge offset 0), which overwrite the
    root's initialisation (07_octree.cu:188-198 then func_octree.hpp:62-87)."""
    t = res.trimmed()
    ch, mask, corner, cell = t["children"], t["child_node_mask"], t["corner"], t["cell_size"]
    bad = 0
    for p in range(1, t["n_octree_nodes"]):
        for w in range(8):
            if not (mask[p] >> w) & 1:
                continue
            c = ch[p, w]
            half = cell[p] / 2
            if cell[c] != half:
                bad += 1
                continue
            for a in range(3):
                lo = corner[p, a] + (half if (w >> a) & 1 else 0)
                if corner[c, a] != lo:
                    bad += 1
                    break
    return bad


def test_geometric_delta_gives_a_nested_octree(rw, oracle):
    """With the clz - 2 delta every octree link is geometrically exact (a
    child cell is the parent's octant at half its size); the reference's
    clz - 1 shifts levels and breaks that on ordinary clouds.  64-bit keys
    are unchanged by the option (their clz - 1 is already exact)."""
    from oracle import OPT_GEOMETRIC_DELTA
    pts = rw.generate_points(20000, rw.GEN_UNIFORM, 77)
    geo = oracle.run(pts, options=OPT_GEOMETRIC_DELTA)
    assert geo.status == ORC_OK
    assert _octree_is_nested(geo, 32) == 0
    assert _octree_is_nested(oracle.run(pts), 32) > 0
    a = oracle.run(pts, key_bits=64)
    b = oracle.run(pts, key_bits=64, options=OPT_GEOMETRIC_DELTA)
    assert compare(a, b) == []
    assert _octree_is_nested(a, 64) == 0
