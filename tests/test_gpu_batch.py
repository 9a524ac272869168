"""Batched form: every cloud of a batch equals the oracle's run on that cloud
alone, bit for bit, with and without the CUDA graph."""
import numpy as np
import pytest

from oracle import ORC_ERR_CAPACITY, ORC_ERR_DEGENERATE, ORC_OK

pytestmark = pytest.mark.gpu

FIELDS = ("sorted_keys", "unique_keys", "prefix_n", "has_leaf_left", "has_leaf_right",
          "left_child", "parents", "edge_count", "edge_offset", "children", "corner",
          "cell_size", "child_node_mask", "child_leaf_mask")


def make_clouds(rw, n_clouds, lo, hi, seed):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_clouds)).astype(np.int64)
    clouds = []
    for c, n in enumerate(sizes):
        kind = rw.GEN_UNIFORM if rng.random() < 0.5 else rw.GEN_GAUSSIAN_MIXTURE
        clouds.append(rw.generate_points(int(n), kind, seed * 1000 + c,
                                         n_components=int(rng.integers(8, 65))))
    return clouds


def check_batch(rw, oracle, batch, clouds, key_bits):
    counted = {"ok": 0, "degenerate": 0, "capacity": 0}
    for c, pts in enumerate(clouds):
        want = oracle.run(pts, key_bits=key_bits, capacity=batch.capacity(c))
        if want.status == ORC_ERR_DEGENERATE:
            assert batch.status[c] == rw.RW_ERR_DEGENERATE, c
            assert batch.n_unique[c] == want.n_unique, c
            counted["degenerate"] += 1
            continue
        if want.status == ORC_ERR_CAPACITY:
            # a plain run with this capacity reports the same overflow
            assert batch.status[c] == rw.RW_ERR_CAPACITY, c
            assert batch.n_octree_nodes[c] == want.n_octree_nodes, c
            counted["capacity"] += 1
            continue
        counted["ok"] += 1
        assert want.status == ORC_OK
        assert batch.status[c] == 0, (c, batch.status[c])
        got = batch.results(c)
        w = want.trimmed()
        assert got["n_unique"] == w["n_unique"], c
        assert got["n_octree_nodes"] == w["n_octree_nodes"], c
        bad = [k for k in FIELDS
               if np.ascontiguousarray(got[k]).tobytes() != np.ascontiguousarray(w[k]).tobytes()]
        assert not bad, (c, pts.shape[0], bad)
    return counted


@pytest.mark.parametrize("key_bits", [32, 64])
def test_batch_every_cloud_exact(rw, oracle, key_bits):
    clouds = make_clouds(rw, 48, 1000, 70000, 3)
    # degenerate and tiny clouds in the middle of the batch
    clouds[5] = np.zeros((7, 4), np.float32)
    clouds[9] = rw.generate_points(1, rw.GEN_UNIFORM, 1)
    clouds[17] = rw.generate_points(3, rw.GEN_UNIFORM, 2)
    batch = rw.Batch(clouds, key_bits)
    batch.run(graph=False)
    counted = check_batch(rw, oracle, batch, clouds, key_bits)
    assert counted["degenerate"] >= 2 and counted["ok"] >= 10
    # with room for every octree no cloud overflows
    roomy = rw.Batch(clouds, key_bits, octree_ratio=1.5)
    roomy.run(graph=True)
    assert check_batch(rw, oracle, roomy, clouds, key_bits)["capacity"] == 0
    # the graph, twice, on new points of the same sizes
    clouds2 = [rw.generate_points(c.shape[0], rw.GEN_UNIFORM, 77 + i) for i, c in enumerate(clouds)]
    batch.set_points(clouds2)
    batch.run(graph=True)
    batch.run(graph=True)
    check_batch(rw, oracle, batch, clouds2, key_bits)


def test_batch_sort_variant_change(rw, oracle):
    clouds = make_clouds(rw, 20, 2000, 40000, 9)
    batch = rw.Batch(clouds, 32)
    batch.run(graph=True)
    for v in rw.sort_variants():
        if v["key_bits"] == 32 and v["radix_bits"] == 8 and v["index"] in (1, 3):
            batch.set_sort_variant(v["index"])
            batch.run(graph=True)
            check_batch(rw, oracle, batch, clouds, 32)


def test_batch_eleven_bit_digits(rw, oracle):
    clouds = make_clouds(rw, 16, 1000, 30000, 12)
    batch = rw.Batch(clouds, 32, radix_bits=11)
    batch.run(graph=True)
    check_batch(rw, oracle, batch, clouds, 32)


def test_batch_size_classes(rw, oracle):
    """Three size classes, each with its own onesweep variant, in one batch."""
    clouds = make_clouds(rw, 40, 500, 120000, 21)
    v32 = [v["index"] for v in rw.sort_variants() if v["key_bits"] == 32 and v["radix_bits"] == 8]
    batch = rw.Batch(clouds, 32, octree_ratio=1.5, tuning=None)
    batch.set_classes([(4000, v32[2]), (30000, v32[1]), (1 << 30, v32[0])])
    batch.run(graph=True)
    assert check_batch(rw, oracle, batch, clouds, 32)["ok"] == len(clouds)


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_with_learned_sort_every_cloud_exact(rw, oracle, mode):
    """Stage 2 of every cloud by the learned-CDF sort inside the batch (the
    combined form): clouds above and below the 65,536-key sample, starting at
    offsets that are not 16-byte aligned, one of them with a dense spot that
    overflows its bucket region (the gated onesweep fallback), through the
    CUDA graph and without it - every cloud equals the oracle's run on it."""
    from redwood_comp_b200 import learned
    clouds = [learned.mixture_cloud(rw, 200_003, 41_001),
              rw.generate_points(1_001, rw.GEN_UNIFORM, 41_002),
              rw.generate_points(150_001, rw.GEN_UNIFORM, 41_003),
              learned.mixture_cloud(rw, 65_537, 41_004),
              rw.generate_points(120_000, rw.GEN_UNIFORM, 41_005)]
    clouds[4][:30_000] = np.float32(700.5)  # a quarter of the cloud on one spot
    largest = max(c.shape[0] for c in clouds)
    L = rw.Learned(largest)
    if L.params is None:
        L.set_params(learned.init_params(1))
    fallback = rw.ImStorage(largest, 32)
    batch = rw.Batch(clouds, 32, octree_ratio=1.0)
    batch.set_learned(L, mode, fallback)
    for graph in (False, True, True):
        batch.run(graph=graph)
        counted = check_batch(rw, oracle, batch, clouds, 32)
        assert counted["ok"] == len(clouds), counted
    batch.set_learned(None)
    batch.run(graph=True)
    assert check_batch(rw, oracle, batch, clouds, 32)["ok"] == len(clouds)
    batch.close()
