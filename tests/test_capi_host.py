"""Host-side checks of the C ABI that need no GPU: the library loads, exports
every function include/rw_tree.h declares, validates arguments before touching
the device, and generates the documented seeded inputs."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "rw_tree.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rw_tree_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported(rw):
    lib = rw.lib()
    names = declared_functions()
    assert len(names) >= 19
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(rw.EXPORTS)


def test_version_and_capacity(rw):
    assert b"sm_100a" in rw.lib().rw_tree_version()
    assert rw.octree_capacity(307200) == 184320


def test_argument_validation_without_device(rw):
    lib = rw.lib()
    h = ctypes.c_void_p()
    assert lib.rw_tree_im_storage_create_ex(0, 32, 0, ctypes.byref(h)) == rw.RW_ERR_ARG
    assert lib.rw_tree_im_storage_create_ex(100, 48, 0, ctypes.byref(h)) == rw.RW_ERR_ARG
    assert lib.rw_tree_im_storage_create_ex(100, 32, 9, ctypes.byref(h)) == rw.RW_ERR_ARG
    assert lib.rw_tree_im_storage_create_ex(1 << 30, 32, 0, ctypes.byref(h)) == rw.RW_ERR_ARG
    # null app / storage
    assert lib.rw_tree_run_stage1(None, None, None) == rw.RW_ERR_ARG
    assert lib.rw_tree_pipeline_enqueue(None, None, None) == rw.RW_ERR_ARG


def test_app_data_init(rw):
    c = rw._AppDataC()
    rw.lib().rw_tree_app_data_init(ctypes.byref(c), 1000, 64)
    assert (c.n_input, c.key_bits, c.oct_capacity) == (1000, 64, 600)
    assert (c.min_coord, c.range) == (0.0, 1024.0)
    assert c.n_unique == c.n_brt_nodes == c.n_octree_nodes == rw.COUNT_UNSET
    assert c.u_input_points is None


def test_generators(rw):
    a = rw.generate_points(1000, rw.GEN_UNIFORM, 5)
    b = rw.generate_points(1000, rw.GEN_UNIFORM, 5)
    c = rw.generate_points(1000, rw.GEN_UNIFORM, 6)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a[:, :3].min() >= 0 and a[:, :3].max() < 1024 and (a[:, 3] == 1).all()
    g = rw.generate_points(200000, rw.GEN_GAUSSIAN_MIXTURE, 9, n_components=32)
    assert g[:, :3].min() >= 0 and g[:, :3].max() < 1024
    # a mixture with sigma 4..40 puts the points in far fewer 8-unit cells
    u = rw.generate_points(200000, rw.GEN_UNIFORM, 9)
    cells = lambda p: len(np.unique(np.floor(p[:, :3] / 8), axis=0))
    assert cells(g) < 0.5 * cells(u)
    # multithreaded generation is chunk-independent
    big = rw.generate_points(300000, rw.GEN_GAUSSIAN_MIXTURE, 9, n_components=32)
    assert np.array_equal(big[:200000], g)


def test_new_entry_points_validate_before_the_device(rw):
    """The entry points added for options, the bounded-wait probe and the
    batch's learned stage 2 reject bad arguments before any device access."""
    lib = rw.lib()
    assert lib.rw_tree_im_storage_set_options(None, 0) == rw.RW_ERR_ARG
    assert lib.rw_tree_sort_lookback_probe(None, None, 64, None) == rw.RW_ERR_ARG
    assert lib.rw_tree_batch_set_learned(None, None, 0, None) == rw.RW_ERR_ARG
    assert lib.rw_tree_learned_sort(None, None, None, 0, 0, None, None, None) == rw.RW_ERR_ARG
    # the option bits and the learned modes the header defines
    text = open(os.path.join(ROOT, "include", "rw_tree.h")).read()
    assert "#define RW_TREE_OPT_GEOMETRIC_DELTA 1" in text
    assert "#define RW_TREE_OPT_LINK_LEAVES 2" in text
    assert (rw.OPT_GEOMETRIC_DELTA, rw.OPT_LINK_LEAVES) == (1, 2)
