"""GPU parity at the benchmark's own scale: 16,777,216 points, uniform and a
32-component Gaussian mixture (sigma 4-40), 32- and 64-bit keys; the fused
pipeline, the host-facing calls the end-to-end number runs through
(rw_tree_run_host and the rw_tree_host_submit / rw_tree_host_collect
rotation) and the pipeline with the learned-CDF sort in stage 2 - every output
array and both counts against the oracle, bit for bit."""
import numpy as np
import pytest

from oracle import ORC_OK

pytestmark = pytest.mark.gpu

N_SCALE = 1 << 24
FIELDS = ("sorted_keys", "unique_keys", "prefix_n", "has_leaf_left", "has_leaf_right",
          "left_child", "parents", "edge_count", "edge_offset", "children", "corner",
          "cell_size", "child_node_mask", "child_leaf_mask")


def scale_cloud(rw, dist, n=N_SCALE, seed=20260101):
    """The benchmark's clouds (bench.py make_points)."""
    if dist == "uniform":
        return rw.generate_points(n, rw.GEN_UNIFORM, seed)
    return rw.generate_points(n, rw.GEN_GAUSSIAN_MIXTURE, seed, n_components=32,
                              sigma_lo=4.0, sigma_hi=40.0)


def assert_same(got, want_res, label):
    want = want_res.trimmed()
    assert got["n_unique"] == want["n_unique"], label
    assert got["n_octree_nodes"] == want["n_octree_nodes"], label
    bad = [k for k in FIELDS
           if np.ascontiguousarray(got[k]).tobytes() != np.ascontiguousarray(want[k]).tobytes()]
    assert not bad, f"{label}: mismatching outputs {bad}"


@pytest.mark.parametrize("dist,key_bits", [("uniform", 32), ("gauss", 32), ("uniform", 64),
                                           ("gauss", 64)])
def test_fused_pipeline_at_16M(rw, oracle, dist, key_bits):
    pts = scale_cloud(rw, dist)
    want = oracle.run(pts, key_bits=key_bits)
    assert want.status == ORC_OK
    app = rw.AppData(N_SCALE, key_bits, points=pts)
    im = rw.ImStorage(N_SCALE, key_bits)
    rw.run_pipeline(app, im)
    assert_same(app.results(), want, f"{dist} k{key_bits}")
    # a second run on the same buffers (the benchmark's steps) is exact too
    rw.run_pipeline(app, im)
    assert_same(app.results(), want, f"{dist} k{key_bits} second run")


def _host_out(rw, n, key_bits):
    """Pinned host buffers for every output rw_tree_host_out names."""
    import torch
    cap = rw.octree_capacity(n)
    kt = torch.int32 if key_bits == 32 else torch.int64
    shapes = {
        "sorted_keys": ((n,), kt), "unique_keys": ((n,), kt),
        "prefix_n": ((n,), torch.uint8), "has_leaf_left": ((n,), torch.uint8),
        "has_leaf_right": ((n,), torch.uint8), "left_child": ((n,), torch.int32),
        "parents": ((n,), torch.int32), "edge_count": ((n,), torch.int32),
        "edge_offset": ((n,), torch.int32), "children": ((cap, 8), torch.int32),
        "corner": ((cap, 4), torch.float32), "cell_size": ((cap,), torch.float32),
        "child_node_mask": ((cap,), torch.int32), "child_leaf_mask": ((cap,), torch.int32)}
    return {k: torch.zeros(*sh, dtype=dt).pin_memory().numpy() for k, (sh, dt) in shapes.items()}


def _host_results(app, out):
    """The host buffers cut to their meaningful lengths, as AppData.results()."""
    u, m = app.get_n_unique(), app.get_n_octree_nodes()
    b = u - 1
    kdt = np.uint32 if app.key_bits == 32 else np.uint64
    r = {"n_unique": u, "n_octree_nodes": m,
         "sorted_keys": out["sorted_keys"].view(kdt),
         "unique_keys": out["unique_keys"].view(kdt)[:u]}
    for k in ("prefix_n", "has_leaf_left", "has_leaf_right", "left_child", "parents",
              "edge_count", "edge_offset"):
        r[k] = out[k][:b]
    for k in ("children", "corner", "cell_size", "child_node_mask", "child_leaf_mask"):
        r[k] = out[k][:m]
    return r


@pytest.mark.parametrize("dist,key_bits,n", [("uniform", 32, N_SCALE),
                                             ("gauss", 64, (1 << 20) + 3)])
def test_run_host_equals_oracle(rw, oracle, dist, key_bits, n):
    """rw_tree_run_host: pinned host points in, all 14 outputs back in host
    memory, every one equal to the oracle's."""
    import torch
    pts = scale_cloud(rw, dist, n, seed=31337)
    want = oracle.run(pts, key_bits=key_bits)
    assert want.status == ORC_OK
    h_pts = torch.from_numpy(pts).pin_memory().numpy()
    app = rw.AppData(n, key_bits, points=np.zeros_like(pts))
    im = rw.ImStorage(n, key_bits)
    out = _host_out(rw, n, key_bits)
    rw.run_host(app, im, h_pts, out)
    assert_same(_host_results(app, out), want, f"run_host {dist} k{key_bits}")


def test_host_stream_rotation_equals_oracle(rw, oracle):
    """The rotation the end-to-end number times (three AppData/scratch pairs
    on three streams, submit(k) then collect(k-2)) over four clouds: every
    cloud's 14 outputs equal the oracle's."""
    import torch
    n = 1 << 21
    clouds = [scale_cloud(rw, "uniform", n, 11), scale_cloud(rw, "gauss", n, 12),
              scale_cloud(rw, "gauss", n, 13), scale_cloud(rw, "uniform", n, 14)]
    wants = [oracle.run(c) for c in clouds]
    pinned = [torch.from_numpy(c).pin_memory().numpy() for c in clouds]
    n_slots, lag = 3, 2
    slots = [(rw.AppData(n, 32, points=np.zeros_like(clouds[0])), rw.ImStorage(n, 32),
              torch.cuda.Stream(), _host_out(rw, n, 32)) for _ in range(n_slots)]
    got = {}
    for k in range(len(clouds) + lag):
        if k < len(clouds):
            cur = slots[k % n_slots]
            rw.host_submit(cur[0], cur[1], pinned[k], cur[2])
        if k >= lag:
            j = k - lag
            prev = slots[j % n_slots]
            rw.host_collect(prev[0], prev[1], prev[3], prev[2])
            prev[2].synchronize()
            got[j] = {kk: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v)
                      for kk, v in _host_results(prev[0], prev[3]).items()}
    for j, want in enumerate(wants):
        assert_same(got[j], want, f"rotation cloud {j}")


def test_learned_pipeline_equals_oracle_at_16M(rw, oracle):
    """The pipeline with the learned-CDF sort in stage 2, both boundary
    methods, on 16,777,216 Gaussian-mixture points: every output equals the
    oracle's (not only the plain GPU pipeline's)."""
    from redwood_comp_b200 import learned
    n = N_SCALE
    pts = learned.mixture_cloud(rw, n, 950_003)  # not a training seed
    want = oracle.run(pts)
    assert want.status == ORC_OK
    L = rw.Learned(n)
    if L.params is None:
        L.set_params(learned.init_params(1))
    app = rw.AppData(n, 32, points=pts)
    im = rw.ImStorage(n, 32)
    for mode in (rw.LEARNED_MLP, rw.LEARNED_SAMPLE_QUANTILES):
        im.set_learned(L, mode)
        rw.run_pipeline(app, im)
        assert_same(app.results(), want, f"learned mode {mode}")
        assert im.learned_stats()["fell_back"] == 0
    im.set_learned(None)
    L.close()
