"""Options outside the bit-exact contract (rw_tree_im_storage_set_options):
the clz - 2 delta of 32-bit keys and the reference's leaf linker.  Each is
compared with the oracle run under the same option, output by output, through
the stage calls and the fused pipeline; with the options cleared the outputs
are the reference's again."""
import numpy as np
import pytest

from oracle import OPT_GEOMETRIC_DELTA, OPT_LINK_LEAVES, ORC_OK

pytestmark = pytest.mark.gpu

FIELDS = ("sorted_keys", "unique_keys", "prefix_n", "has_leaf_left", "has_leaf_right",
          "left_child", "parents", "edge_count", "edge_offset", "children", "corner",
          "cell_size", "child_node_mask", "child_leaf_mask")


def assert_same(got, want_res, label):
    want = want_res.trimmed()
    assert got["n_unique"] == want["n_unique"], label
    assert got["n_octree_nodes"] == want["n_octree_nodes"], label
    bad = [k for k in FIELDS
           if np.ascontiguousarray(got[k]).tobytes() != np.ascontiguousarray(want[k]).tobytes()]
    assert not bad, f"{label}: mismatching outputs {bad}"


def clouds(rw):
    yield "appdata", rw.generate_points(640 * 480, rw.GEN_APPDATA, 114514)
    yield "gauss", rw.generate_points(65537, rw.GEN_GAUSSIAN_MIXTURE, 5, n_components=6,
                                      sigma_lo=2.0, sigma_hi=20.0)
    yield "uniform", rw.generate_points((1 << 20) + 7, rw.GEN_UNIFORM, 6)


@pytest.mark.parametrize("key_bits", [32, 64])
@pytest.mark.parametrize("options", [OPT_GEOMETRIC_DELTA, OPT_LINK_LEAVES,
                                     OPT_GEOMETRIC_DELTA | OPT_LINK_LEAVES])
def test_options_equal_the_oracle(rw, oracle, key_bits, options):
    for name, pts in clouds(rw):
        n = pts.shape[0]
        want = oracle.run(pts, key_bits=key_bits, options=options)
        assert want.status == ORC_OK, name
        app = rw.AppData(n, key_bits, points=pts)
        im = rw.ImStorage(n, key_bits)
        im.set_options(options)
        rw.run_pipeline(app, im)
        assert_same(app.results(), want, f"{name} fused k{key_bits} opt{options}")
        for k in range(1, 8):
            getattr(rw, f"run_stage{k}")(app, im)
        assert_same(app.results(), want, f"{name} stagewise k{key_bits} opt{options}")
        # cleared again: the reference's own outputs
        im.set_options(0)
        rw.run_pipeline(app, im)
        assert_same(app.results(), oracle.run(pts, key_bits=key_bits), f"{name} cleared")


def test_leaf_links_change_the_children(rw, oracle):
    pts = rw.generate_points(100_000, rw.GEN_UNIFORM, 8)
    app = rw.AppData(100_000, 32, points=pts)
    im = rw.ImStorage(100_000, 32)
    rw.run_pipeline(app, im)
    plain = app.results()["children"].copy()
    im.set_options(OPT_LINK_LEAVES)
    rw.run_pipeline(app, im)
    linked = app.results()["children"]
    assert not np.array_equal(plain, linked)
    with pytest.raises(rw.RwTreeError):
        im.set_options(4)
