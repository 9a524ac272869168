"""Python host side of the B200 tree pipeline, over the C ABI of rw_tree.h.

Mirrors the reference's tree-app surface (ucsc-redwood/redwood-comp,
apps/tree): ``AppData`` with the same buffer names (app_data.hpp:15-158),
``ImStorage`` (cuda/im_storage.cuh:10-42) and ``run_stage1..7``
(cuda/cu_dispatcher.cuh:8-19), plus ``run_pipeline`` (all seven stages fused,
counts on the device) and ``run_host`` (end to end from host memory).

PyTorch only provides device memory and the current stream.  Every stage runs
in the sm_100a kernels of librw_tree.so; there is no CPU fallback, and loading
fails loudly when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

__all__ = [
    "RwTreeError", "lib", "AppData", "ImStorage", "run_stage1", "run_stage2",
    "run_stage3", "run_stage4", "run_stage5", "run_stage6", "run_stage7",
    "run_pipeline", "run_host", "generate_points", "octree_capacity",
    "GEN_APPDATA", "GEN_UNIFORM", "GEN_GAUSSIAN_MIXTURE", "COUNT_UNSET",
]

HERE = os.path.dirname(os.path.abspath(__file__))
_BUILT_LIB = os.path.join(HERE, "librw_tree.so")
# RW_TREE_LIBRARY names another build of the same C ABI (a debug build, say)
LIB_PATH = os.environ.get("RW_TREE_LIBRARY", _BUILT_LIB)

RW_OK, RW_ERR_ARG, RW_ERR_DEGENERATE, RW_ERR_CAPACITY = 0, 1, 2, 3
RW_ERR_CUDA, RW_ERR_TIMEOUT, RW_ERR_NOT_READY, RW_ERR_NO_DEVICE = 4, 5, 6, 7
STATUS_NAMES = {
    0: "RW_OK", 1: "RW_ERR_ARG", 2: "RW_ERR_DEGENERATE", 3: "RW_ERR_CAPACITY",
    4: "RW_ERR_CUDA", 5: "RW_ERR_TIMEOUT", 6: "RW_ERR_NOT_READY",
    7: "RW_ERR_NO_DEVICE",
}
COUNT_UNSET = 0xFFFFFFFF
# options outside the reference contract (rw_tree_im_storage_set_options)
OPT_GEOMETRIC_DELTA, OPT_LINK_LEAVES = 1, 2
GEN_APPDATA, GEN_UNIFORM, GEN_GAUSSIAN_MIXTURE = 0, 1, 2
DEFAULT_SEED = 114514  # app_data.hpp:32

_vp = ctypes.c_void_p


class RwTreeError(RuntimeError):
    """A non-zero rw_status (the reference throws std::runtime_error from
    CUDA_CHECK and from unset-count getters, redwood/cuda/helpers.cuh:12-20,
    app_data.hpp:110-133)."""

    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        msg = f"{where}: {STATUS_NAMES.get(code, code)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


class _AppDataC(ctypes.Structure):
    _fields_ = [
        ("n_input", ctypes.c_uint32), ("oct_capacity", ctypes.c_uint32),
        ("key_bits", ctypes.c_int32), ("min_coord", ctypes.c_float),
        ("range", ctypes.c_float), ("n_unique", ctypes.c_uint32),
        ("n_brt_nodes", ctypes.c_uint32), ("n_octree_nodes", ctypes.c_uint32),
        ("u_input_points", _vp), ("u_morton_keys", _vp), ("u_morton_keys_alt", _vp),
        ("u_edge_count", _vp), ("u_edge_offset", _vp), ("brt_prefix_n", _vp),
        ("brt_has_leaf_left", _vp), ("brt_has_leaf_right", _vp),
        ("brt_left_child", _vp), ("brt_parents", _vp), ("oct_children", _vp),
        ("oct_corner", _vp), ("oct_cell_size", _vp), ("oct_child_node_mask", _vp),
        ("oct_child_leaf_mask", _vp),
    ]


class _BatchBufsC(ctypes.Structure):
    _fields_ = [(name, _vp) for name in (
        "points", "morton_keys", "morton_keys_alt", "edge_count", "edge_offset", "prefix_n",
        "has_leaf_left", "has_leaf_right", "left_child", "parents", "children", "corner",
        "cell_size", "child_node_mask", "child_leaf_mask")]


class _HostOutC(ctypes.Structure):
    _fields_ = [(name, _vp) for name in (
        "sorted_keys", "unique_keys", "prefix_n", "has_leaf_left", "has_leaf_right",
        "left_child", "parents", "edge_count", "edge_offset", "children", "corner",
        "cell_size", "child_node_mask", "child_leaf_mask")]


_LIB = None

EXPORTS = (
    "rw_tree_octree_capacity", "rw_tree_app_data_init", "rw_tree_im_storage_create",
    "rw_tree_im_storage_create_ex", "rw_tree_im_storage_destroy",
    "rw_tree_im_storage_clear", "rw_tree_run_stage1", "rw_tree_run_stage2",
    "rw_tree_run_stage3", "rw_tree_run_stage4", "rw_tree_run_stage5",
    "rw_tree_run_stage6", "rw_tree_run_stage7", "rw_tree_pipeline_enqueue",
    "rw_tree_pipeline_finish", "rw_tree_run_host", "rw_tree_generate_points",
    "rw_tree_last_error", "rw_tree_version", "rw_tree_pipeline_profile",
    "rw_tree_pipeline_kernel_names", "rw_tree_sort_variant_count",
    "rw_tree_sort_variant_info", "rw_tree_im_storage_set_sort_variant",
    "rw_tree_unique_noalloc", "rw_tree_batch_create", "rw_tree_batch_destroy",
    "rw_tree_batch_total_points", "rw_tree_batch_octree_rows", "rw_tree_batch_offsets",
    "rw_tree_batch_set_sort_variant", "rw_tree_batch_enqueue", "rw_tree_batch_graph_launch",
    "rw_tree_batch_finish", "rw_tree_batch_set_classes", "rw_tree_sort_enqueue",
    "rw_tree_sort_profile", "rw_tree_sort_lookback_probe", "rw_tree_im_storage_set_options",
    "rw_tree_batch_set_learned",
    "rw_tree_learned_create", "rw_tree_learned_destroy", "rw_tree_learned_set_params",
    "rw_tree_learned_set_group", "rw_tree_im_storage_set_learned",
    "rw_tree_im_storage_learned_stats", "rw_tree_host_submit", "rw_tree_host_collect",
    "rw_tree_learned_sort", "rw_tree_learned_features", "rw_tree_learned_bucket_counts",
    "rw_tree_mlp_param_count", "rw_tree_mlp_grad", "rw_tree_mlp_adam", "rw_tree_mlp_forward",
)


def lib() -> ctypes.CDLL:
    """The loaded librw_tree.so (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with "
                               "`make -C redwood-comp_b200` (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        L.rw_tree_octree_capacity.restype = ctypes.c_uint32
        L.rw_tree_octree_capacity.argtypes = [ctypes.c_uint32]
        L.rw_tree_app_data_init.restype = None
        L.rw_tree_last_error.restype = ctypes.c_char_p
        L.rw_tree_version.restype = ctypes.c_char_p
        L.rw_tree_pipeline_kernel_names.restype = ctypes.c_char_p
        L.rw_tree_batch_total_points.restype = ctypes.c_uint32
        L.rw_tree_batch_octree_rows.restype = ctypes.c_uint32
        L.rw_tree_generate_points.argtypes = [
            _vp, ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint64, ctypes.c_float,
            ctypes.c_float, ctypes.c_int32, ctypes.c_float, ctypes.c_float]
        _LIB = L
    return _LIB


def _check(rc: int, where: str) -> None:
    if rc != RW_OK:
        raise RwTreeError(rc, where, lib().rw_tree_last_error().decode())


def sort_variants() -> list:
    """The onesweep variant menu: dicts of key_bits, radix_bits, threads,
    keys_per_thread, rank (0 ballot, 1 match.any, 2 smem atomic-or)."""
    out = []
    L = lib()
    v = [ctypes.c_int32() for _ in range(5)]
    for i in range(L.rw_tree_sort_variant_count()):
        _check(L.rw_tree_sort_variant_info(i, *[ctypes.byref(x) for x in v]), "variant_info")
        out.append(dict(index=i, key_bits=v[0].value, radix_bits=v[1].value,
                        threads=v[2].value, keys_per_thread=v[3].value, rank=v[4].value))
    return out


def octree_capacity(n: int) -> int:
    return int(lib().rw_tree_octree_capacity(n))


def generate_points(n: int, kind: int = GEN_APPDATA, seed: int = DEFAULT_SEED,
                    min_coord: float = 0.0, range_: float = 1024.0,
                    n_components: int = 32, sigma_lo: float = 4.0,
                    sigma_hi: float = 40.0, out: Optional[np.ndarray] = None) -> np.ndarray:
    """Seeded [n, 4] float32 points (host memory); see rw_tree_generate_points."""
    pts = out if out is not None else np.empty((n, 4), np.float32)
    assert pts.dtype == np.float32 and pts.shape == (n, 4) and pts.flags.c_contiguous
    _check(lib().rw_tree_generate_points(
        pts.ctypes.data_as(_vp), n, kind, seed, min_coord, range_, n_components,
        sigma_lo, sigma_hi), "generate_points")
    return pts


def _stream_handle(stream) -> _vp:
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return _vp(s.cuda_stream)


class ImStorage:
    """Scratch of one pipeline (the reference's cuda::ImStorage)."""

    def __init__(self, n_input: int, key_bits: int = 32, radix_bits: int = 0):
        self._h = _vp()
        _check(lib().rw_tree_im_storage_create_ex(
            ctypes.c_uint32(n_input), ctypes.c_int32(key_bits), ctypes.c_int32(radix_bits),
            ctypes.byref(self._h)), "ImStorage")
        self.n_input, self.key_bits, self.radix_bits = n_input, key_bits, radix_bits

    @property
    def handle(self) -> _vp:
        return self._h

    def set_options(self, options: int) -> None:
        """OPT_GEOMETRIC_DELTA / OPT_LINK_LEAVES bits (0: the reference's own
        outputs); see rw_tree_im_storage_set_options."""
        _check(lib().rw_tree_im_storage_set_options(self._h, ctypes.c_int32(options)),
               "set_options")

    def set_sort_variant(self, idx: int) -> None:
        _check(lib().rw_tree_im_storage_set_sort_variant(self._h, idx), "set_sort_variant")
        self.sort_variant = idx

    def set_learned(self, learned, mode: int = 0) -> None:
        """Stage 2 sorts with the learned-CDF sort `learned` (a Learned, or
        None for the onesweep sort); 32-bit keys only."""
        _check(lib().rw_tree_im_storage_set_learned(
            self._h, learned._h if learned is not None else None, ctypes.c_int32(mode)),
            "set_learned")
        self.learned = learned

    def learned_stats(self) -> dict:
        st = _LearnedStatsC()
        _check(lib().rw_tree_im_storage_learned_stats(self._h, ctypes.byref(st)), "learned_stats")
        return {"max_bucket": st.max_bucket, "big_buckets": st.big_buckets,
                "fell_back": st.fell_back, "mlp_timeout": st.mlp_timeout}

    def clear(self, stream=None) -> None:
        _check(lib().rw_tree_im_storage_clear(self._h, _stream_handle(stream)), "clearSmem")

    def close(self) -> None:
        if self._h:
            lib().rw_tree_im_storage_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AppData:
    """Device-resident buffers of one point cloud, named as in AppData.

    ``points``: [n, 4] float32 host array; by default the reference's own
    seeded input (mt19937(114514) uniform in [0, 1024), app_data.hpp:32-39).
    """

    min_coord = 0.0
    range = 1024.0

    def __init__(self, n_input: int, key_bits: int = 32,
                 points: Optional[np.ndarray] = None, device: str = "cuda",
                 min_coord: float = 0.0, range_: float = 1024.0,
                 octree_ratio: Optional[float] = None):
        import torch
        if key_bits not in (32, 64):
            raise ValueError("key_bits must be 32 or 64")
        self.n_input = n = int(n_input)
        self.key_bits = key_bits
        self.min_coord, self.range = float(min_coord), float(range_)
        # AppData's floor(0.6f * n) rows (app_data.hpp:13,28) unless a ratio is given
        self.oct_capacity = cap = octree_capacity(n) if octree_ratio is None else \
            int(np.float32(n) * np.float32(octree_ratio))
        kt = torch.int32 if key_bits == 32 else torch.int64
        dev = torch.device(device)
        e = lambda *shape, dtype: torch.zeros(*shape, dtype=dtype, device=dev)
        self.u_input_points = e(n, 4, dtype=torch.float32)
        self.u_morton_keys = e(n, dtype=kt)
        self.u_morton_keys_alt = e(n, dtype=kt)
        self.u_edge_count = e(n, dtype=torch.int32)
        self.u_edge_offset = e(n, dtype=torch.int32)
        self.brt_prefix_n = e(n, dtype=torch.uint8)
        self.brt_has_leaf_left = e(n, dtype=torch.uint8)
        self.brt_has_leaf_right = e(n, dtype=torch.uint8)
        self.brt_left_child = e(n, dtype=torch.int32)
        self.brt_parents = e(n, dtype=torch.int32)
        rows = max(cap, 1)
        self.oct_children = e(rows, 8, dtype=torch.int32)
        self.oct_corner = e(rows, 4, dtype=torch.float32)
        self.oct_cell_size = e(rows, dtype=torch.float32)
        self.oct_child_node_mask = e(rows, dtype=torch.int32)
        self.oct_child_leaf_mask = e(rows, dtype=torch.int32)
        if points is None:
            points = generate_points(n, GEN_APPDATA, DEFAULT_SEED, min_coord, range_)
        self.set_points(points)
        c = _AppDataC()
        lib().rw_tree_app_data_init(ctypes.byref(c), ctypes.c_uint32(n), ctypes.c_int32(key_bits))
        c.min_coord, c.range = self.min_coord, self.range
        c.oct_capacity = cap
        for name, _ in _AppDataC._fields_:
            if hasattr(self, name) and name.startswith(("u_", "brt_", "oct_")) and name != "oct_capacity":
                setattr(c, name, getattr(self, name).data_ptr())
        self._c = c

    # -- data movement ------------------------------------------------------
    def set_points(self, points: np.ndarray) -> None:
        import torch
        pts = np.ascontiguousarray(points, np.float32).reshape(self.n_input, 4)
        self.u_input_points.copy_(torch.from_numpy(pts))

    @property
    def c(self) -> _AppDataC:
        return self._c

    # -- counts (app_data.hpp:108-137) ---------------------------------------
    def get_n_input(self) -> int:
        return self.n_input

    def get_n_unique(self) -> int:
        if self._c.n_unique == COUNT_UNSET:
            raise RuntimeError("n_unique is not set")
        return int(self._c.n_unique)

    def get_n_brt_nodes(self) -> int:
        return self.get_n_unique() - 1

    def get_n_octree_nodes(self) -> int:
        if self._c.n_octree_nodes == COUNT_UNSET:
            raise RuntimeError("n_octree_nodes is not set")
        return int(self._c.n_octree_nodes)

    # -- host views -------------------------------------------------------------
    def _keys_np(self, t) -> np.ndarray:
        a = t.cpu().numpy()
        return a.view(np.uint32 if self.key_bits == 32 else np.uint64)

    def results(self) -> dict:
        """Every output, copied to host and cut to its meaningful length."""
        u = self.get_n_unique()
        b = u - 1
        m = self.get_n_octree_nodes()
        return {
            "sorted_keys": self._keys_np(self.u_morton_keys_alt),
            "unique_keys": self._keys_np(self.u_morton_keys)[:u],
            "n_unique": u,
            "prefix_n": self.brt_prefix_n[:b].cpu().numpy(),
            "has_leaf_left": self.brt_has_leaf_left[:b].cpu().numpy(),
            "has_leaf_right": self.brt_has_leaf_right[:b].cpu().numpy(),
            "left_child": self.brt_left_child[:b].cpu().numpy(),
            "parents": self.brt_parents[:b].cpu().numpy(),
            "edge_count": self.u_edge_count[:b].cpu().numpy(),
            "edge_offset": self.u_edge_offset[:b].cpu().numpy(),
            "n_octree_nodes": m,
            "children": self.oct_children[:m].cpu().numpy(),
            "corner": self.oct_corner[:m].cpu().numpy(),
            "cell_size": self.oct_cell_size[:m].cpu().numpy(),
            "child_node_mask": self.oct_child_node_mask[:m].cpu().numpy(),
            "child_leaf_mask": self.oct_child_leaf_mask[:m].cpu().numpy(),
        }


def _stage(k: int):
    fn_name = f"rw_tree_run_stage{k}"

    def run(app: AppData, im: ImStorage, stream=None) -> None:
        _check(getattr(lib(), fn_name)(ctypes.byref(app.c), im.handle,
                                       _stream_handle(stream)), f"run_stage{k}")

    run.__name__ = f"run_stage{k}"
    run.__doc__ = f"cuda::run_stage{k} (cu_dispatcher.cuh:8-19); synchronous."
    return run


run_stage1, run_stage2, run_stage3, run_stage4, run_stage5, run_stage6, run_stage7 = (
    _stage(k) for k in range(1, 8))


def sort_keys(keys, out, im: ImStorage, stream=None) -> None:
    """Onesweep sort of a device key tensor (int32 for 32-bit keys, int64 for
    64-bit) into `out`, asynchronous on `stream` (rw_tree_sort_enqueue)."""
    c = _AppDataC()
    bits = 32 if keys.element_size() == 4 else 64
    lib().rw_tree_app_data_init(ctypes.byref(c), ctypes.c_uint32(keys.numel()), ctypes.c_int32(bits))
    c.u_morton_keys, c.u_morton_keys_alt = keys.data_ptr(), out.data_ptr()
    _check(lib().rw_tree_sort_enqueue(ctypes.byref(c), im.handle, _stream_handle(stream)),
           "sort_enqueue")


def sort_lookback_probe(app: AppData, im: ImStorage, spin_limit: int, stream=None) -> int:
    """Runs the sort's first pass with its first tile left out, so that every
    other tile's bounded look-back wait runs out (rw_tree_sort_lookback_probe);
    returns the rw_status code (RW_ERR_TIMEOUT when the bound works)."""
    return int(lib().rw_tree_sort_lookback_probe(ctypes.byref(app.c), im.handle,
                                                 ctypes.c_uint32(spin_limit),
                                                 _stream_handle(stream)))


def profile_sort(keys, out, im: ImStorage, reps: int = 5, stream=None) -> dict:
    """Mean device milliseconds of the sort's kernels: histogram, sort_init,
    sort_pass0 .. (rw_tree_sort_profile)."""
    c = _AppDataC()
    bits = 32 if keys.element_size() == 4 else 64
    lib().rw_tree_app_data_init(ctypes.byref(c), ctypes.c_uint32(keys.numel()), ctypes.c_int32(bits))
    c.u_morton_keys, c.u_morton_keys_alt = keys.data_ptr(), out.data_ptr()
    ms = (ctypes.c_float * 64)()
    nk = ctypes.c_int32()
    _check(lib().rw_tree_sort_profile(ctypes.byref(c), im.handle, _stream_handle(stream), reps,
                                      ms, 64, ctypes.byref(nk)), "sort_profile")
    names = ["histogram", "sort_init"] + [f"sort_pass{p}" for p in range(nk.value - 2)]
    return {names[i]: float(ms[i]) for i in range(nk.value)}


def pipeline_enqueue(app: AppData, im: ImStorage, stream=None) -> None:
    _check(lib().rw_tree_pipeline_enqueue(ctypes.byref(app.c), im.handle,
                                          _stream_handle(stream)), "pipeline_enqueue")


def pipeline_finish(app: AppData, im: ImStorage, stream=None) -> None:
    _check(lib().rw_tree_pipeline_finish(ctypes.byref(app.c), im.handle,
                                         _stream_handle(stream)), "pipeline_finish")


def run_pipeline(app: AppData, im: ImStorage, stream=None) -> None:
    """All seven stages, fused, one host synchronisation at the end."""
    pipeline_enqueue(app, im, stream)
    pipeline_finish(app, im, stream)


def profile_pipeline(app: AppData, im: ImStorage, reps: int = 5, stream=None) -> dict:
    """Mean device milliseconds of every kernel of the fused pipeline."""
    ms = (ctypes.c_float * 64)()
    nk = ctypes.c_int32()
    _check(lib().rw_tree_pipeline_profile(ctypes.byref(app.c), im.handle,
                                          _stream_handle(stream), reps, ms, 64,
                                          ctypes.byref(nk)), "pipeline_profile")
    names = lib().rw_tree_pipeline_kernel_names(im.handle).decode().split(",")
    return {names[i]: float(ms[i]) for i in range(nk.value)}


def run_host(app: AppData, im: ImStorage, h_points: np.ndarray,
             out: Optional[dict] = None, stream=None) -> None:
    """End to end from host memory; `out` maps rw_tree_host_out field names to
    preallocated (ideally pinned) host arrays."""
    pts = np.ascontiguousarray(h_points, np.float32)
    ho = _HostOutC()
    keep = []
    for name, arr in (out or {}).items():
        a = arr if isinstance(arr, np.ndarray) else arr.numpy()
        keep.append(a)
        setattr(ho, name, a.ctypes.data)
    _check(lib().rw_tree_run_host(ctypes.byref(app.c), im.handle, pts.ctypes.data_as(_vp),
                                  ctypes.byref(ho), _stream_handle(stream)), "run_host")


def _host_out(out):
    ho = _HostOutC()
    for name, arr in (out or {}).items():
        a = arr if isinstance(arr, np.ndarray) else arr.numpy()
        setattr(ho, name, a.ctypes.data)
    return ho


def host_submit(app: AppData, im: ImStorage, h_points: np.ndarray, stream=None) -> None:
    """Copies the (pinned) host points in and enqueues the pipeline, without
    waiting (rw_tree_host_submit).  h_points must stay alive until `stream`
    has drained."""
    _check(lib().rw_tree_host_submit(ctypes.byref(app.c), im.handle,
                                     h_points.ctypes.data_as(_vp), _stream_handle(stream)),
           "host_submit")


def host_collect(app: AppData, im: ImStorage, out: Optional[dict] = None, stream=None) -> None:
    """Waits for the submitted run's counts and enqueues the copies of `out`'s
    fields (rw_tree_host_collect); they are complete once `stream` has drained."""
    ho = _host_out(out)
    _check(lib().rw_tree_host_collect(ctypes.byref(app.c), im.handle, ctypes.byref(ho),
                                      _stream_handle(stream)), "host_collect")


class Batch:
    """Many clouds through the seven stages with one launch per kernel.

    ``clouds``: list of [n_c, 4] float32 host arrays.  Buffers are device
    tensors concatenated cloud after cloud (the layout of rw_tree.h).
    """

    def __init__(self, clouds, key_bits: int = 32, radix_bits: int = 0,
                 octree_ratio: float = 0.6, device: str = "cuda", tuning="auto"):
        """tuning: "auto" applies the autotuner's table for this key width when
        one exists (tuning/b200_u{32,64}.json), None keeps the default
        variant, a dict is used as the table."""
        import torch
        from . import autotune
        table = autotune.load_table(key_bits) if tuning == "auto" else tuning
        if table and radix_bits == 0:
            radix_bits = int(table["radix_bits"])
        sizes = np.array([c.shape[0] for c in clouds], np.uint32)
        self.n_clouds = len(clouds)
        self.key_bits = key_bits
        self.octree_ratio = octree_ratio
        self._h = _vp()
        _check(lib().rw_tree_batch_create(sizes.ctypes.data_as(_vp), ctypes.c_uint32(len(sizes)),
                                          ctypes.c_int32(key_bits), ctypes.c_int32(radix_bits),
                                          ctypes.c_float(octree_ratio), ctypes.byref(self._h)),
               "Batch")
        L = lib()
        self.n_total = int(L.rw_tree_batch_total_points(self._h))
        self.oct_rows = int(L.rw_tree_batch_octree_rows(self._h))
        self.point_offsets = np.zeros(self.n_clouds + 1, np.uint32)
        self.octree_offsets = np.zeros(self.n_clouds + 1, np.uint32)
        _check(L.rw_tree_batch_offsets(self._h, self.point_offsets.ctypes.data_as(_vp),
                                       self.octree_offsets.ctypes.data_as(_vp)), "offsets")
        n, rows = self.n_total, max(self.oct_rows, 1)
        kt = torch.int32 if key_bits == 32 else torch.int64
        dev = torch.device(device)
        e = lambda *shape, dtype: torch.zeros(*shape, dtype=dtype, device=dev)
        self.points = e(n, 4, dtype=torch.float32)
        self.morton_keys = e(n, dtype=kt)
        self.morton_keys_alt = e(n, dtype=kt)
        self.edge_count = e(n, dtype=torch.int32)
        self.edge_offset = e(n, dtype=torch.int32)
        self.prefix_n = e(n, dtype=torch.uint8)
        self.has_leaf_left = e(n, dtype=torch.uint8)
        self.has_leaf_right = e(n, dtype=torch.uint8)
        self.left_child = e(n, dtype=torch.int32)
        self.parents = e(n, dtype=torch.int32)
        self.children = e(rows, 8, dtype=torch.int32)
        self.corner = e(rows, 4, dtype=torch.float32)
        self.cell_size = e(rows, dtype=torch.float32)
        self.child_node_mask = e(rows, dtype=torch.int32)
        self.child_leaf_mask = e(rows, dtype=torch.int32)
        self.set_points(clouds)
        c = _BatchBufsC()
        for name, _ in _BatchBufsC._fields_:
            setattr(c, name, getattr(self, name).data_ptr())
        self._c = c
        self.n_unique = np.zeros(self.n_clouds, np.uint32)
        self.n_octree_nodes = np.zeros(self.n_clouds, np.uint32)
        self.status = np.zeros(self.n_clouds, np.int32)
        self.tuning = None
        if table and int(table["radix_bits"]) == (radix_bits or 8) and \
                int(table["key_bits"]) == key_bits:
            classes = autotune.class_list(table, sort_variants())
            if classes is not None:
                self.set_classes(classes)
                self.tuning = table

    def capacity(self, c: int) -> int:
        return int(self.octree_offsets[c + 1] - self.octree_offsets[c])

    def set_points(self, clouds) -> None:
        import torch
        host = np.concatenate([np.ascontiguousarray(c, np.float32).reshape(-1, 4) for c in clouds])
        self.points.copy_(torch.from_numpy(host))

    def set_sort_variant(self, idx: int) -> None:
        _check(lib().rw_tree_batch_set_sort_variant(self._h, idx), "batch_set_sort_variant")

    def set_learned(self, learned, mode: int = 0, fallback_im=None) -> None:
        """Stage 2 of every cloud by the learned-CDF sort (32-bit keys;
        rw_tree_batch_set_learned); None restores the batched onesweep sort."""
        self._learned = (learned, fallback_im)  # kept alive while in use
        _check(lib().rw_tree_batch_set_learned(
            self._h, learned._h if learned is not None else None, ctypes.c_int32(mode),
            fallback_im.handle if fallback_im is not None else None), "batch_set_learned")

    def set_classes(self, classes) -> None:
        """classes: [(max_points, variant_index), ...] ascending; the last
        class takes every larger cloud."""
        mx = np.array([c[0] for c in classes], np.uint32)
        var = np.array([c[1] for c in classes], np.int32)
        _check(lib().rw_tree_batch_set_classes(self._h, ctypes.c_uint32(len(classes)),
                                               mx.ctypes.data_as(_vp), var.ctypes.data_as(_vp)),
               "batch_set_classes")

    def enqueue(self, graph: bool = True, stream=None) -> None:
        fn = lib().rw_tree_batch_graph_launch if graph else lib().rw_tree_batch_enqueue
        _check(fn(self._h, ctypes.byref(self._c), _stream_handle(stream)), "batch_enqueue")

    def finish(self, stream=None) -> None:
        _check(lib().rw_tree_batch_finish(
            self._h, _stream_handle(stream), self.n_unique.ctypes.data_as(_vp),
            self.n_octree_nodes.ctypes.data_as(_vp), self.status.ctypes.data_as(_vp)),
            "batch_finish")

    def run(self, graph: bool = True, stream=None) -> None:
        self.enqueue(graph, stream)
        self.finish(stream)

    def results(self, c: int) -> dict:
        """Cloud c's outputs, host copies cut to their meaningful lengths."""
        p0, p1 = int(self.point_offsets[c]), int(self.point_offsets[c + 1])
        r0 = int(self.octree_offsets[c])
        u = int(self.n_unique[c])
        b = u - 1
        m = int(self.n_octree_nodes[c])
        kv = np.uint32 if self.key_bits == 32 else np.uint64
        return {
            "sorted_keys": self.morton_keys_alt[p0:p1].cpu().numpy().view(kv),
            "unique_keys": self.morton_keys[p0:p0 + u].cpu().numpy().view(kv),
            "n_unique": u,
            "prefix_n": self.prefix_n[p0:p0 + b].cpu().numpy(),
            "has_leaf_left": self.has_leaf_left[p0:p0 + b].cpu().numpy(),
            "has_leaf_right": self.has_leaf_right[p0:p0 + b].cpu().numpy(),
            "left_child": self.left_child[p0:p0 + b].cpu().numpy(),
            "parents": self.parents[p0:p0 + b].cpu().numpy(),
            "edge_count": self.edge_count[p0:p0 + b].cpu().numpy(),
            "edge_offset": self.edge_offset[p0:p0 + b].cpu().numpy(),
            "n_octree_nodes": m,
            "children": self.children[r0:r0 + m].cpu().numpy(),
            "corner": self.corner[r0:r0 + m].cpu().numpy(),
            "cell_size": self.cell_size[r0:r0 + m].cpu().numpy(),
            "child_node_mask": self.child_node_mask[r0:r0 + m].cpu().numpy(),
            "child_leaf_mask": self.child_leaf_mask[r0:r0 + m].cpu().numpy(),
        }

    def close(self) -> None:
        if self._h:
            lib().rw_tree_batch_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# learned-CDF bucketed sort and its boundary MLP
# ---------------------------------------------------------------------------

LEARNED_MLP, LEARNED_SAMPLE_QUANTILES = 0, 1
MLP_PARAMS = 5313


class _LearnedStatsC(ctypes.Structure):
    _fields_ = [("max_bucket", ctypes.c_uint32), ("big_buckets", ctypes.c_uint32),
                ("fell_back", ctypes.c_uint32), ("mlp_timeout", ctypes.c_uint32)]


def _dptr(t) -> _vp:
    return _vp(t.data_ptr())


class Learned:
    """Scratch and boundary-MLP parameters of the learned-CDF sort.

    params: "auto" loads the trained table (tuning/cdf_mlp_b200.json) when
    present, None leaves the network unset (sample quantiles only), or a
    float32 array of MLP_PARAMS values."""

    def __init__(self, n_max: int, params="auto", group: int = 4):
        self._h = _vp()
        _check(lib().rw_tree_learned_create(ctypes.c_uint32(n_max), ctypes.byref(self._h)),
               "Learned")
        self.n_max = n_max
        self.params = None
        self.group = group
        if isinstance(params, str) and params == "auto":
            from . import learned as _learned
            params, group = _learned.load_params(with_group=True)
        if params is not None:
            self.set_params(params, group)
        else:
            self.set_group(group)

    def set_params(self, params, group: int | None = None) -> None:
        p = np.ascontiguousarray(params, np.float32).reshape(-1)
        g = self.group if group is None else int(group)
        _check(lib().rw_tree_learned_set_params(self._h, p.ctypes.data_as(_vp),
                                                ctypes.c_int32(p.size), ctypes.c_int32(g)),
               "learned_set_params")
        self.params, self.group = p, g

    def set_group(self, group: int) -> None:
        _check(lib().rw_tree_learned_set_group(self._h, ctypes.c_int32(int(group))),
               "learned_set_group")
        self.group = int(group)

    def sort(self, keys, out=None, mode: int = LEARNED_MLP, fallback_im=None, stream=None):
        """Sorts a device int32 tensor of 32-bit keys; returns (sorted, stats)."""
        import torch
        n = keys.numel()
        out = torch.empty_like(keys) if out is None else out
        st = _LearnedStatsC()
        im = fallback_im.handle if fallback_im is not None else None
        _check(lib().rw_tree_learned_sort(self._h, _dptr(keys), _dptr(out), ctypes.c_uint32(n),
                                          ctypes.c_int32(mode), im, _stream_handle(stream),
                                          ctypes.byref(st)), "learned_sort")
        return out, {"max_bucket": st.max_bucket, "big_buckets": st.big_buckets,
                     "fell_back": st.fell_back, "mlp_timeout": st.mlp_timeout}

    def features(self, keys, stream=None):
        """(MLP inputs [4095, 16] under the current group size, sorted sample
        [65536] as uint32); rows whose context does not fit are zero."""
        n = keys.numel()
        f = np.zeros((4095, 16), np.float32)
        srt = np.zeros(65536, np.uint32)
        _check(lib().rw_tree_learned_features(self._h, _dptr(keys), ctypes.c_uint32(n),
                                              f.ctypes.data_as(_vp), srt.ctypes.data_as(_vp),
                                              _stream_handle(stream)), "learned_features")
        return f, srt

    def bucket_counts(self, keys, mode: int = LEARNED_MLP, stream=None) -> np.ndarray:
        c = np.zeros(4096, np.uint32)
        _check(lib().rw_tree_learned_bucket_counts(self._h, _dptr(keys), ctypes.c_uint32(keys.numel()),
                                                   ctypes.c_int32(mode), c.ctypes.data_as(_vp),
                                                   _stream_handle(stream)), "bucket_counts")
        return c

    def close(self) -> None:
        if self._h:
            lib().rw_tree_learned_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mlp_grad(params, x, t, batch: int, grad=None, loss=None, stream=None):
    """Accumulates d(MSE over `batch`)/d(params) of rows (x, t) into grad
    (device float32 tensors); returns (grad, loss_sum)."""
    import torch
    grad = torch.zeros_like(params) if grad is None else grad
    loss = torch.zeros(1, dtype=torch.float32, device=params.device) if loss is None else loss
    _check(lib().rw_tree_mlp_grad(_dptr(params), _dptr(x), _dptr(t), ctypes.c_uint32(t.numel()),
                                  ctypes.c_uint32(batch), _dptr(grad), _dptr(loss),
                                  _stream_handle(stream)), "mlp_grad")
    return grad, loss


def mlp_adam(params, grad, m, v, lr: float, step: int, beta1=0.9, beta2=0.999, eps=1e-8,
             stream=None) -> None:
    _check(lib().rw_tree_mlp_adam(_dptr(params), _dptr(grad), _dptr(m), _dptr(v),
                                  ctypes.c_float(lr), ctypes.c_float(beta1), ctypes.c_float(beta2),
                                  ctypes.c_float(eps), ctypes.c_int32(step),
                                  _stream_handle(stream)), "mlp_adam")


def mlp_forward(params, x, stream=None):
    import torch
    y = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
    _check(lib().rw_tree_mlp_forward(_dptr(params), _dptr(x), ctypes.c_uint32(x.shape[0]),
                                     _dptr(y), _stream_handle(stream)), "mlp_forward")
    return y
