"""The onesweep sort's bounded look-back wait, made to run out without any
fault: rw_tree_sort_lookback_probe leaves the first tile of a pass out, so
every other tile waits on a descriptor that nothing publishes.  The reference's
look-back has no bound (cu_dispatcher.cu:376); here the wait must end with
RW_ERR_TIMEOUT, keep every write inside the output buffer, and leave the
scratch fit for the next normal run, which must be exact."""
import numpy as np
import pytest

from oracle import ORC_OK

pytestmark = pytest.mark.gpu

FIELDS = ("sorted_keys", "unique_keys", "prefix_n", "has_leaf_left", "has_leaf_right",
          "left_child", "parents", "edge_count", "edge_offset", "children", "corner",
          "cell_size", "child_node_mask", "child_leaf_mask")
GUARD = 4096  # keys of guard on each side of the output (16-byte multiple)
PATTERN = 0x5A5A5A5A


@pytest.mark.parametrize("key_bits", [32, 64])
def test_lookback_wait_runs_out_and_the_next_run_is_exact(rw, oracle, key_bits):
    import torch
    n = 300_007
    pts = rw.generate_points(n, rw.GEN_GAUSSIAN_MIXTURE, 4242, n_components=12)
    want = oracle.run(pts, key_bits=key_bits).trimmed()
    app = rw.AppData(n, key_bits, points=pts)
    im = rw.ImStorage(n, key_bits)
    rw.run_stage1(app, im)
    kt = torch.int32 if key_bits == 32 else torch.int64
    fill = PATTERN if key_bits == 32 else (PATTERN << 32) | PATTERN
    guarded = torch.full((n + 2 * GUARD,), fill, dtype=kt, device="cuda")
    app.c.u_morton_keys_alt = guarded.data_ptr() + guarded.element_size() * GUARD
    rc = rw.sort_lookback_probe(app, im, 64)
    assert rc == rw.RW_ERR_TIMEOUT, rw.STATUS_NAMES.get(rc, rc)
    g = guarded.cpu().numpy()
    assert (g[:GUARD] == fill).all() and (g[GUARD + n:] == fill).all(), \
        "a write landed outside the output"
    # the same scratch, the real buffers again: a normal run is exact
    app.c.u_morton_keys_alt = app.u_morton_keys_alt.data_ptr()
    rw.run_pipeline(app, im)
    got = app.results()
    assert got["n_unique"] == want["n_unique"]
    assert got["n_octree_nodes"] == want["n_octree_nodes"]
    bad = [k for k in FIELDS
           if np.ascontiguousarray(got[k]).tobytes() != np.ascontiguousarray(want[k]).tobytes()]
    assert not bad, bad


def test_probe_rejects_a_zero_limit_and_a_single_tile(rw):
    n = 5000  # fewer keys than one tile of the default variant
    app = rw.AppData(n, 32, points=rw.generate_points(n, rw.GEN_UNIFORM, 1))
    im = rw.ImStorage(n, 32)
    assert rw.sort_lookback_probe(app, im, 64) == rw.RW_ERR_ARG
    big = rw.AppData(100_000, 32, points=rw.generate_points(100_000, rw.GEN_UNIFORM, 2))
    im2 = rw.ImStorage(100_000, 32)
    assert rw.sort_lookback_probe(big, im2, 0) == rw.RW_ERR_ARG
