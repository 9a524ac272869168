"""The C++ front end (include/redwood_tree/): the reference's CUDA demo and its
timing loop, rebuilt on cuda::run_stage1..7 / futures / run_pipeline, produce
the reference's canonical outputs on its own default cloud."""
import json
import os
import subprocess

import pytest

from conftest import GOLDEN_DIR, PKG_DIR

BIN = os.path.join(PKG_DIR, "bin")


def _run(args, timeout=300):
    out = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    assert out.returncode == 0, out.stderr[-2000:]
    kv = {}
    for line in out.stdout.splitlines():
        if " = " in line:
            k, v = line.split(" = ", 1)
            kv[k.strip()] = v.strip()
    return kv


def test_cpp_drivers_are_built():
    for name in ("tree_demo", "pipe_baseline"):
        assert os.access(os.path.join(BIN, name), os.X_OK), f"{name} not built (make -C redwood-comp_b200)"


@pytest.mark.gpu
def test_tree_demo_matches_reference_fixture():
    with open(os.path.join(GOLDEN_DIR, "config1_kat.json")) as f:
        kat = json.load(f)
    kv = _run([os.path.join(BIN, "tree_demo")])
    assert kv["stagewise.sorted"] == "1"
    assert kv["done"] == "1"
    assert kv["engine.buffer_sum"] == str(sum(range(1024)))
    for form in ("stagewise", "futures", "fused"):
        assert int(kv[f"{form}.num_unique"]) == kat["n_unique"], form
        assert int(kv[f"{form}.num_brt"]) == kat["n_brt_nodes"], form
        assert int(kv[f"{form}.num_octree_nodes"]) == kat["n_octree_nodes"], form
        for field in ("prefix_n", "parents", "edge_offset", "children", "corner", "cell_size",
                      "child_node_mask"):
            assert int(kv[f"{form}.fnv_{field}"], 16) == int(kat["fnv1a64"][field], 16), (form, field)
    assert kv["edge_count[0]"] == "0"
    assert kv["edge_offset[0]"] == "0"


@pytest.mark.gpu
def test_pipe_baseline_loop_runs():
    kv = _run([os.path.join(BIN, "pipe_baseline"), str(640 * 480), "20"])
    assert float(kv["stagewise.ms_per_iteration"]) > 0
    assert float(kv["fused.ms_per_iteration"]) > 0
    assert int(kv["num_unique"]) == 307151
    assert int(kv["num_octree_nodes"]) == 150716


REF_DEMO = os.path.join(os.path.dirname(GOLDEN_DIR), "..", "oracle", "_ref", "ref_appdata_demo")


@pytest.mark.gpu
@pytest.mark.skipif(not os.access(REF_DEMO, os.X_OK),
                    reason="oracle/_ref/ref_appdata_demo is built only where the reference's "
                           "sources are (make -C oracle ref)")
def test_reference_appdata_drives_our_stages():
    """The reference's own AppData type (apps/tree/app_data.hpp: static
    constexpr bounds, glm::vec4 corners, its own seeded generator) bound to
    cuda::run_stage1..7 of include/redwood_tree/cu_dispatcher.hpp with the
    reference's call shapes, in the stage, future and fused forms: every
    output equals the fixture made from the reference's CPU functions."""
    with open(os.path.join(GOLDEN_DIR, "config1_kat.json")) as f:
        kat = json.load(f)
    kv = _run([REF_DEMO])
    assert kv["done"] == "1"
    for form in ("stagewise", "futures", "fused"):
        assert int(kv[f"{form}.fnv_points"], 16) == int(kat["points_fnv1a64"], 16), form
        assert int(kv[f"{form}.num_unique"]) == kat["n_unique"], form
        assert int(kv[f"{form}.num_brt"]) == kat["n_brt_nodes"], form
        assert int(kv[f"{form}.num_octree_nodes"]) == kat["n_octree_nodes"], form
        for field in ("sorted_keys", "unique_keys", "prefix_n", "has_leaf_left",
                      "has_leaf_right", "left_child", "parents", "edge_count", "edge_offset",
                      "children", "corner", "cell_size", "child_node_mask", "child_leaf_mask"):
            assert int(kv[f"{form}.fnv_{field}"], 16) == int(kat["fnv1a64"][field], 16), \
                (form, field)
