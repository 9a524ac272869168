"""GPU parity: every output of the sm_100a pipeline equals the oracle's,
bit for bit, through the C ABI (per-stage calls and the fused pipeline)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR
from oracle import ORC_OK, compare  # noqa: F401

pytestmark = pytest.mark.gpu

FIELDS = ("sorted_keys", "unique_keys", "prefix_n", "has_leaf_left", "has_leaf_right",
          "left_child", "parents", "edge_count", "edge_offset", "children", "corner",
          "cell_size", "child_node_mask", "child_leaf_mask")


def run_gpu(rw, pts, key_bits=32, radix_bits=0, fused=True, app=None, im=None):
    n = pts.shape[0]
    if app is None:
        app = rw.AppData(n, key_bits, points=pts)
    else:
        app.set_points(pts)
    im = im or rw.ImStorage(n, key_bits, radix_bits)
    if fused:
        rw.run_pipeline(app, im)
    else:
        for k in range(1, 8):
            getattr(rw, f"run_stage{k}")(app, im)
    return app.results()


def assert_same(got, want_res, label=""):
    want = want_res.trimmed()
    assert got["n_unique"] == want["n_unique"], label
    assert got["n_octree_nodes"] == want["n_octree_nodes"], label
    bad = [k for k in FIELDS
           if np.ascontiguousarray(got[k]).tobytes() != np.ascontiguousarray(want[k]).tobytes()]
    assert not bad, f"{label}: mismatching outputs {bad}"


def cloud(rw, n, kind, seed):
    if kind == "appdata":
        return rw.generate_points(n, rw.GEN_APPDATA, seed)
    if kind == "uniform":
        return rw.generate_points(n, rw.GEN_UNIFORM, seed)
    return rw.generate_points(n, rw.GEN_GAUSSIAN_MIXTURE, seed, n_components=8,
                              sigma_lo=2.0, sigma_hi=20.0)


def test_config1_stagewise_and_fused(rw, oracle):
    pts = rw.generate_points(640 * 480, rw.GEN_APPDATA, 114514)
    want = oracle.run(pts)
    with open(os.path.join(GOLDEN_DIR, "config1_kat.json")) as f:
        kat = json.load(f)
    for fused in (False, True):
        got = run_gpu(rw, pts, fused=fused)
        assert_same(got, want, f"config1 fused={fused}")
        assert got["n_unique"] == kat["n_unique"]
        assert got["n_octree_nodes"] == kat["n_octree_nodes"]
        for k in FIELDS:
            assert f"{oracle.fnv1a64(np.ascontiguousarray(got[k])):#018x}" == kat["fnv1a64"][k], k


def test_golden_small_cases(rw, oracle):
    z = np.load(os.path.join(GOLDEN_DIR, "small_cases.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    for name in names:
        pts = z[f"{name}/points"]
        if int(z[f"{name}/status"][0]) != ORC_OK:
            continue
        for fused in (False, True):
            got = run_gpu(rw, pts, fused=fused)
            for k in FIELDS:
                assert np.ascontiguousarray(got[k]).tobytes() == z[f"{name}/{k}"].tobytes(), \
                    (name, fused, k)


SIZES = (3, 31, 32, 33, 255, 256, 257, 1023, 1024, 1025, 4095, 4096, 4097,
         6143, 6144, 6145, 8191, 8192, 8193, 65537)


@pytest.mark.parametrize("key_bits,radix_bits", [(32, 8), (32, 10), (32, 11), (64, 8),
                                               (64, 10), (64, 11)])
def test_ragged_sizes(rw, oracle, key_bits, radix_bits):
    for i, n in enumerate(SIZES):
        for kind in ("uniform", "gauss"):
            pts = cloud(rw, n, kind, 1000 + i)
            want = oracle.run(pts, key_bits=key_bits)
            for fused in (False, True):
                if want.status != ORC_OK:
                    continue
                got = run_gpu(rw, pts, key_bits, radix_bits, fused)
                assert_same(got, want, f"n={n} {kind} k{key_bits} r{radix_bits} f{fused}")


@pytest.mark.parametrize("key_bits", [32, 64])
def test_one_million_both_forms(rw, oracle, key_bits):
    for kind in ("uniform", "gauss"):
        pts = cloud(rw, (1 << 20) + 1, kind, 77)
        want = oracle.run(pts, key_bits=key_bits)
        assert want.status == ORC_OK
        for fused in (False, True):
            assert_same(run_gpu(rw, pts, key_bits, 0, fused), want, f"{kind} fused={fused}")


def test_buffers_reused_across_inputs(rw, oracle):
    """A second cloud through the same AppData/ImStorage leaves no trace of the first."""
    n = 50000
    a, b = cloud(rw, n, "uniform", 1), cloud(rw, n, "gauss", 2)
    app = rw.AppData(n, 32, points=a)
    im = rw.ImStorage(n, 32)
    rw.run_pipeline(app, im)
    app.set_points(b)
    rw.run_pipeline(app, im)
    assert_same(app.results(), oracle.run(b), "reuse fused")
    app.set_points(a)
    for k in range(1, 8):
        getattr(rw, f"run_stage{k}")(app, im)
    assert_same(app.results(), oracle.run(a), "reuse stagewise")


def test_two_clouds_in_flight_on_two_streams(rw, oracle):
    """Two AppData/ImStorage pairs on two streams, their pipelines enqueued in
    turn with no host wait in between (how a stream of clouds keeps two in
    flight, as bench.py's device-resident region does): each pair ends with the
    oracle's outputs for its own cloud, so scratch sets share no device state."""
    import torch
    n = 300000
    pts = [cloud(rw, n, "uniform", 31), cloud(rw, n, "gauss", 32)]
    pairs = [(rw.AppData(n, 32, points=p), rw.ImStorage(n, 32), torch.cuda.Stream())
             for p in pts]
    torch.cuda.synchronize()
    for app, im, s in pairs:
        rw.run_pipeline(app, im, s)
    torch.cuda.synchronize()
    for i in range(6):
        app, im, s = pairs[i % 2]
        rw.pipeline_enqueue(app, im, s)
    for app, im, s in pairs:
        rw.pipeline_finish(app, im, s)
    for k, ((app, _, _), p) in enumerate(zip(pairs, pts)):
        assert_same(app.results(), oracle.run(p), f"pair {k} of two in flight")


def test_pipeline_replayed_from_a_cuda_graph(rw, oracle):
    """rw_tree_pipeline_enqueue captured once into a CUDA graph (the kernels use
    programmatic dependent launch) and replayed on new clouds in the same
    buffers: every replay exact, counts read by pipeline_finish."""
    import torch
    n = 100000
    app = rw.AppData(n, 32, points=cloud(rw, n, "uniform", 21))
    im = rw.ImStorage(n, 32)
    rw.run_pipeline(app, im)  # first run outside the capture
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        rw.pipeline_enqueue(app, im)
    for kind, seed in (("gauss", 22), ("uniform", 23), ("appdata", 24)):
        pts = cloud(rw, n, kind, seed)
        app.set_points(pts)
        g.replay()
        rw.pipeline_finish(app, im)
        assert_same(app.results(), oracle.run(pts), f"graph replay {kind}")
    del g


def test_sort_stage_matches_numpy(rw):
    """Stage 2 alone on adversarial key sets."""
    import torch
    rng = np.random.default_rng(5)
    for n, top in ((100000, 1 << 30), (100000, 2), (77777, 1), (8192 * 3 + 5, 1 << 8)):
        keys = rng.integers(0, top, size=n, dtype=np.uint64).astype(np.uint32)
        app = rw.AppData(n, 32, points=np.zeros((n, 4), np.float32))
        app.u_morton_keys.copy_(torch.from_numpy(keys.view(np.int32)))
        im = rw.ImStorage(n, 32)
        rw.run_stage2(app, im)
        got = app.u_morton_keys_alt.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, np.sort(keys)), (n, top)


def test_degenerate_and_counts(rw):
    n = 1000
    pts = np.zeros((n, 4), np.float32)
    app = rw.AppData(n, 32, points=pts)
    im = rw.ImStorage(n, 32)
    with pytest.raises(RuntimeError):
        app.get_n_unique()  # unset, as app_data.hpp:110-116
    for k in (1, 2, 3):
        getattr(rw, f"run_stage{k}")(app, im)
    assert app.get_n_unique() == 1
    with pytest.raises(rw.RwTreeError) as e:
        rw.run_stage4(app, im)
    assert e.value.code == rw.RW_ERR_DEGENERATE
    with pytest.raises(rw.RwTreeError) as e:
        rw.run_pipeline(app, im)
    assert e.value.code == rw.RW_ERR_DEGENERATE
    # the device is still usable afterwards
    good = cloud(rw, n, "uniform", 3)
    app.set_points(good)
    rw.run_pipeline(app, im)
    assert app.get_n_unique() > 900


@pytest.mark.gpu
def test_capacity_error_keeps_stages_1_to_6(rw, oracle):
    """An octree too large for its rows stops stage 7 with RW_ERR_CAPACITY
    (the reference would write past the buffer); the fused pipeline still
    leaves every output of stages 1-6 exact, the edge offsets included, as a
    stage-by-stage run does."""
    n = 20000
    pts = cloud(rw, n, "uniform", 11)
    want = oracle.run(pts)
    assert want.status == ORC_OK
    u, b = want.n_unique, want.n_brt_nodes
    for run in ("fused", "stagewise"):
        app = rw.AppData(n, 32, points=pts, octree_ratio=0.01)
        im = rw.ImStorage(n, 32)
        with pytest.raises(rw.RwTreeError) as e:
            if run == "fused":
                rw.run_pipeline(app, im)
            else:
                for k in range(1, 8):
                    getattr(rw, f"run_stage{k}")(app, im)
        assert e.value.code == rw.RW_ERR_CAPACITY, run
        got = {
            "sorted_keys": app.u_morton_keys_alt.cpu().numpy(),
            "unique_keys": app.u_morton_keys[:u].cpu().numpy(),
            "prefix_n": app.brt_prefix_n[:b].cpu().numpy(),
            "parents": app.brt_parents[:b].cpu().numpy(),
            "left_child": app.brt_left_child[:b].cpu().numpy(),
            "edge_count": app.u_edge_count[:b].cpu().numpy(),
            "edge_offset": app.u_edge_offset[:b].cpu().numpy(),
        }
        ref = {"sorted_keys": want.sorted_keys, "unique_keys": want.unique_keys[:u],
               "prefix_n": want.prefix_n[:b], "parents": want.parents[:b],
               "left_child": want.left_child[:b], "edge_count": want.edge_count[:b],
               "edge_offset": want.edge_offset[:b]}
        for k, v in ref.items():
            assert np.ascontiguousarray(got[k]).view(np.uint8).tobytes() == \
                np.ascontiguousarray(v).view(np.uint8).tobytes(), (run, k)


def test_stage_order_enforced(rw):
    n = 1000
    app = rw.AppData(n, 32, points=cloud(rw, n, "uniform", 4))
    im = rw.ImStorage(n, 32)
    with pytest.raises(rw.RwTreeError) as e:
        rw.run_stage4(app, im)
    assert e.value.code == rw.RW_ERR_NOT_READY


def test_every_sort_variant_is_exact(rw, oracle):
    """Each onesweep variant of the autotuner's menu sorts exactly and keeps
    the whole pipeline bit-exact."""
    import torch
    rng = np.random.default_rng(11)
    for v in rw.sort_variants():
        kb, rb = v["key_bits"], v["radix_bits"]
        kt = np.uint32 if kb == 32 else np.uint64
        top = (1 << 30) if kb == 32 else (1 << 63)
        for n in (1, 4097, 100003):
            keys = rng.integers(0, top, size=n, dtype=np.uint64).astype(kt)
            keys[: n // 3] = keys[0]  # a long run of one key
            app = rw.AppData(n, kb, points=np.zeros((n, 4), np.float32))
            app.u_morton_keys.copy_(torch.from_numpy(keys.view(np.int32 if kb == 32 else np.int64)))
            im = rw.ImStorage(n, kb, rb)
            im.set_sort_variant(v["index"])
            try:
                rw.run_stage2(app, im)
            except rw.RwTreeError as e:
                raise AssertionError(f"variant {v}: {e}")
            got = app.u_morton_keys_alt.cpu().numpy().view(kt)
            assert np.array_equal(got, np.sort(keys)), (v, n)
        pts = cloud(rw, 30001, "gauss", 5)
        app = rw.AppData(30001, kb, points=pts)
        im = rw.ImStorage(30001, kb, rb)
        im.set_sort_variant(v["index"])
        rw.run_pipeline(app, im)
        assert_same(app.results(), oracle.run(pts, key_bits=kb), f"variant {v}")


@pytest.mark.parametrize("key_bits", [32, 64])
@pytest.mark.parametrize("box", [(-3.5, 2048.0), (7.25, 1000.0), (0.0, 0.375)])
def test_other_bounds(rw, oracle, key_bits, box):
    """Quantisation against the oracle for bounds other than [0, 1024): a
    power-of-two range (multiplication by the exact reciprocal) and ranges
    that are not (IEEE division), with a nonzero minimum."""
    mn, rg = box
    n = 300_001
    rng = np.random.default_rng(int(rg * 8) + key_bits)
    pts = np.zeros((n, 4), np.float32)
    pts[:, :3] = (mn + rng.random((n, 3)) * rg * 0.999).astype(np.float32)
    pts[:, 3] = 1.0
    app = rw.AppData(n, key_bits, points=pts, min_coord=mn, range_=rg)
    im = rw.ImStorage(n, key_bits)
    rw.run_pipeline(app, im)
    want = oracle.run(pts, key_bits=key_bits, min_coord=mn, range_=rg)
    assert_same(app.results(), want, f"box {box} key_bits {key_bits}")
