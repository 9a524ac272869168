"""Streaming from host memory: rw_tree_host_submit / rw_tree_host_collect on
two AppData/scratch pairs and two streams give every cloud exactly the outputs
rw_tree_run_host gives it (the reference's callers read results from host
memory, apps/tree/main.cpp:48-88)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("children", "corner", "cell_size", "child_node_mask", "child_leaf_mask")


def _outs(rw, n):
    import torch
    cap = rw.octree_capacity(n)
    shapes = {"children": ((cap, 8), torch.int32), "corner": ((cap, 4), torch.float32),
              "cell_size": ((cap,), torch.float32), "child_node_mask": ((cap,), torch.int32),
              "child_leaf_mask": ((cap,), torch.int32)}
    return {k: torch.zeros(*sh, dtype=dt).pin_memory().numpy() for k, (sh, dt) in shapes.items()}


def test_two_slot_stream_equals_run_host(rw):
    import torch
    n = 1 << 20
    clouds = [rw.generate_points(n, rw.GEN_UNIFORM, 101),
              rw.generate_points(n, rw.GEN_GAUSSIAN_MIXTURE, 102, n_components=16)]
    pinned = [torch.from_numpy(c).pin_memory().numpy() for c in clouds]
    # reference results, one cloud at a time
    want = []
    app = rw.AppData(n, 32)
    im = rw.ImStorage(n, 32)
    for p in pinned:
        out = _outs(rw, n)
        rw.run_host(app, im, p, out)
        want.append((app.get_n_octree_nodes(), out))
    # streamed: steps alternate the two clouds over two slots
    slots = []
    for _ in range(2):
        slots.append((rw.AppData(n, 32), rw.ImStorage(n, 32), torch.cuda.Stream(), _outs(rw, n)))
    order = [0, 1, 0, 1, 1]
    got = []
    rw.host_submit(slots[0][0], slots[0][1], pinned[order[0]], slots[0][2])
    for k in range(1, len(order)):
        cur, prev = slots[k % 2], slots[(k - 1) % 2]
        rw.host_submit(cur[0], cur[1], pinned[order[k]], cur[2])
        rw.host_collect(prev[0], prev[1], prev[3], prev[2])
        prev[2].synchronize()
        got.append((prev[0].get_n_octree_nodes(), {f: prev[3][f].copy() for f in FIELDS}))
    last = slots[(len(order) - 1) % 2]
    rw.host_collect(last[0], last[1], last[3], last[2])
    last[2].synchronize()
    got.append((last[0].get_n_octree_nodes(), {f: last[3][f].copy() for f in FIELDS}))
    for k, (m, out) in enumerate(got):
        wm, wout = want[order[k]]
        assert m == wm, k
        for f in FIELDS:
            assert np.array_equal(out[f][:m], wout[f][:m]), (k, f)
