"""Test infrastructure: Python handles on the two CPU checkers.

* ``Oracle`` - the project's C restatement (``liboracle.so``, tree_oracle.c).
* ``RefTree`` - the reference's own CPU tree code compiled in place
  (``_ref/libref_tree.so``, see Makefile): its point generator
  (apps/tree/app_data.hpp:32-39), its verbatim ``cpu::run_stage1..7``
  (apps/tree/host/host_dispatchers.cpp) and its per-element functions wired
  with the canonical dataflow (ref_driver.cpp).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only to check or to time the reference.  Nothing in the
product imports it.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_tree.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libref_tree_cuda.so")

ORC_OK, ORC_ERR_ARG, ORC_ERR_DEGENERATE, ORC_ERR_CAPACITY = 0, 1, 2, 3

_vp = ctypes.c_void_p


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_vp)


def octree_capacity(n: int) -> int:
    """floor(n * 0.6f) computed in float, as AppData does (app_data.hpp:13,28)."""
    return int(np.float32(n) * np.float32(0.6))


class _OrcTree(ctypes.Structure):
    _fields_ = [
        ("n_input", ctypes.c_uint32),
        ("capacity", ctypes.c_uint32),
        ("key_bits", ctypes.c_int),
        ("min_coord", ctypes.c_float),
        ("range", ctypes.c_float),
        ("points", _vp),
        ("keys", _vp),
        ("keys_alt", _vp),
        ("prefix_n", _vp),
        ("has_leaf_left", _vp),
        ("has_leaf_right", _vp),
        ("left_child", _vp),
        ("parents", _vp),
        ("edge_count", _vp),
        ("edge_offset", _vp),
        ("children", _vp),
        ("corner", _vp),
        ("cell_size", _vp),
        ("child_node_mask", _vp),
        ("child_leaf_mask", _vp),
        ("n_unique", ctypes.c_uint32),
        ("n_brt_nodes", ctypes.c_uint32),
        ("n_octree_nodes", ctypes.c_uint32),
        ("options", ctypes.c_int),
    ]


# Options outside the bit-exact contract with the reference (tree_oracle.h).
OPT_GEOMETRIC_DELTA, OPT_LINK_LEAVES = 1, 2


@dataclass
class TreeResult:
    """Every output array of the tree pipeline plus its counts.

    Arrays hold the full buffer; the meaningful prefixes are [0, n_unique) for
    unique_keys, [0, n_brt_nodes) for the radix-tree and edge arrays and
    [0, n_octree_nodes) for the octree rows.
    """

    key_bits: int
    morton_keys: np.ndarray | None = None  # keys after stage 1
    sorted_keys: np.ndarray | None = None
    unique_keys: np.ndarray | None = None
    prefix_n: np.ndarray | None = None
    has_leaf_left: np.ndarray | None = None
    has_leaf_right: np.ndarray | None = None
    left_child: np.ndarray | None = None
    parents: np.ndarray | None = None
    edge_count: np.ndarray | None = None
    edge_offset: np.ndarray | None = None
    children: np.ndarray | None = None  # [cap, 8]
    corner: np.ndarray | None = None  # [cap, 4]
    cell_size: np.ndarray | None = None
    child_node_mask: np.ndarray | None = None
    child_leaf_mask: np.ndarray | None = None
    n_unique: int = 0
    n_brt_nodes: int = 0
    n_octree_nodes: int = 0
    status: int = 0
    extra: dict = field(default_factory=dict)

    def trimmed(self) -> dict:
        """Outputs cut to their meaningful prefixes (what parity compares)."""
        u, b, m = self.n_unique, self.n_brt_nodes, self.n_octree_nodes
        out = {
            "sorted_keys": self.sorted_keys,
            "unique_keys": self.unique_keys[:u],
            "n_unique": u,
        }
        if self.status == ORC_OK:
            out.update(
                prefix_n=self.prefix_n[:b],
                has_leaf_left=self.has_leaf_left[:b],
                has_leaf_right=self.has_leaf_right[:b],
                left_child=self.left_child[:b],
                parents=self.parents[:b],
                edge_count=self.edge_count[:b],
                edge_offset=self.edge_offset[:b],
                n_octree_nodes=m,
                children=self.children[:m],
                corner=self.corner[:m],
                cell_size=self.cell_size[:m],
                child_node_mask=self.child_node_mask[:m],
                child_leaf_mask=self.child_leaf_mask[:m],
            )
        return out


def _alloc_result(n: int, cap: int, key_bits: int) -> TreeResult:
    kt = np.uint32 if key_bits == 32 else np.uint64
    return TreeResult(
        key_bits=key_bits,
        morton_keys=np.zeros(n, kt),
        sorted_keys=np.zeros(n, kt),
        unique_keys=np.zeros(n, kt),
        prefix_n=np.zeros(n, np.uint8),
        has_leaf_left=np.zeros(n, np.uint8),
        has_leaf_right=np.zeros(n, np.uint8),
        left_child=np.zeros(n, np.int32),
        parents=np.zeros(n, np.int32),
        edge_count=np.zeros(n, np.int32),
        edge_offset=np.zeros(n, np.int32),
        children=np.zeros((max(cap, 1), 8), np.int32),
        corner=np.zeros((max(cap, 1), 4), np.float32),
        cell_size=np.zeros(max(cap, 1), np.float32),
        child_node_mask=np.zeros(max(cap, 1), np.int32),
        child_leaf_mask=np.zeros(max(cap, 1), np.int32),
    )


class Oracle:
    """The C restatement of the tree pipeline (tree_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        lib = ctypes.CDLL(path)
        lib.orc_fnv1a64.restype = ctypes.c_uint64
        lib.orc_capacity.restype = ctypes.c_uint32
        for s in range(1, 8):
            getattr(lib, f"orc_stage{s}").argtypes = [ctypes.POINTER(_OrcTree)]
        self.lib = lib

    def fnv1a64(self, a: np.ndarray) -> int:
        a = np.ascontiguousarray(a)
        return int(self.lib.orc_fnv1a64(_ptr(a), ctypes.c_size_t(a.nbytes)))

    def morton(self, points: np.ndarray, key_bits: int = 32,
               min_coord: float = 0.0, range_: float = 1024.0) -> np.ndarray:
        points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        n = points.shape[0]
        keys = np.zeros(n, np.uint32 if key_bits == 32 else np.uint64)
        self.lib.orc_morton(_ptr(points), _ptr(keys), ctypes.c_uint32(n),
                            ctypes.c_int(key_bits), ctypes.c_float(min_coord),
                            ctypes.c_float(range_))
        return keys

    def generate_points(self, n: int, kind: int, seed: int, min_coord: float = 0.0,
                        range_: float = 1024.0, n_components: int = 32,
                        sigma_lo: float = 4.0, sigma_hi: float = 40.0) -> np.ndarray:
        """The library's counter-based clouds (GEN_UNIFORM = 1,
        GEN_GAUSSIAN_MIXTURE = 2) restated in C, byte for byte: [n, 4] float32."""
        pts = np.zeros((n, 4), np.float32)
        rc = self.lib.orc_generate_points(
            _ptr(pts), ctypes.c_uint64(n), ctypes.c_int(kind), ctypes.c_uint64(seed),
            ctypes.c_float(min_coord), ctypes.c_float(range_), ctypes.c_int(n_components),
            ctypes.c_float(sigma_lo), ctypes.c_float(sigma_hi))
        if rc:
            raise ValueError(f"orc_generate_points: status {rc}")
        return pts

    def sort(self, keys: np.ndarray) -> np.ndarray:
        keys = np.array(keys, copy=True)
        bits = 32 if keys.dtype == np.uint32 else 64
        self.lib.orc_sort(_ptr(keys), ctypes.c_uint32(keys.size), ctypes.c_int(bits))
        return keys

    def run(self, points: np.ndarray, key_bits: int = 32,
            min_coord: float = 0.0, range_: float = 1024.0,
            capacity: int | None = None, options: int = 0) -> TreeResult:
        """Stages 1-7 on `points` ([n,4] float32).  status != 0 stops early.
        `options`: OPT_* bits (0: the reference's own behaviour)."""
        points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        n = points.shape[0]
        cap = octree_capacity(n) if capacity is None else capacity
        r = _alloc_result(n, cap, key_bits)
        t = _OrcTree(
            n_input=n, capacity=cap, key_bits=key_bits, min_coord=min_coord,
            range=range_, points=_ptr(points).value, keys=_ptr(r.unique_keys).value,
            keys_alt=_ptr(r.sorted_keys).value, prefix_n=_ptr(r.prefix_n).value,
            has_leaf_left=_ptr(r.has_leaf_left).value,
            has_leaf_right=_ptr(r.has_leaf_right).value,
            left_child=_ptr(r.left_child).value, parents=_ptr(r.parents).value,
            edge_count=_ptr(r.edge_count).value, edge_offset=_ptr(r.edge_offset).value,
            children=_ptr(r.children).value, corner=_ptr(r.corner).value,
            cell_size=_ptr(r.cell_size).value,
            child_node_mask=_ptr(r.child_node_mask).value,
            child_leaf_mask=_ptr(r.child_leaf_mask).value, options=options)
        tp = ctypes.byref(t)
        status = self.lib.orc_stage1(tp)
        if status == 0:
            r.morton_keys[:] = r.unique_keys
        for s in range(2, 8):
            if status:
                break
            status = getattr(self.lib, f"orc_stage{s}")(tp)
        r.status = status
        r.n_unique, r.n_brt_nodes = t.n_unique, t.n_brt_nodes
        r.n_octree_nodes = t.n_octree_nodes
        return r


class _RefOut(ctypes.Structure):
    _fields_ = [(name, _vp) for name in (
        "keys_after_stage1", "sorted_keys", "unique_keys", "prefix_n",
        "has_leaf_left", "has_leaf_right", "left_child", "parents",
        "edge_count", "edge_offset", "children", "corner", "cell_size",
        "child_node_mask", "child_leaf_mask")] + [
        ("n_unique", ctypes.c_uint32), ("n_brt_nodes", ctypes.c_uint32),
        ("n_octree_nodes", ctypes.c_uint32), ("capacity", ctypes.c_uint32)]


def ref_available(path: str = REF_SO) -> bool:
    return os.path.exists(path)


class RefTree:
    """The reference's own CPU tree code (32-bit keys only)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        lib = ctypes.CDLL(path)
        lib.ref_octree_capacity.restype = ctypes.c_uint32
        lib.ref_hardware_threads.restype = ctypes.c_uint
        self.lib = lib

    def default_points(self, n: int = 640 * 480) -> np.ndarray:
        """AppData's seeded input (mt19937(114514), uniform [0, 1024))."""
        pts = np.zeros((n, 4), np.float32)
        self.lib.ref_default_points(_ptr(pts), ctypes.c_uint32(n))
        return pts

    def hardware_threads(self) -> int:
        return int(self.lib.ref_hardware_threads())

    def verbatim(self, points: np.ndarray, n_threads: int):
        points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        n = points.shape[0]
        keys = np.zeros(n, np.uint32)
        counts = np.zeros(2, np.uint32)
        rc = self.lib.ref_cpu_verbatim(_ptr(points), ctypes.c_uint32(n),
                                       ctypes.c_int(n_threads), _ptr(keys),
                                       _ptr(counts))
        if rc:
            raise RuntimeError(f"ref_cpu_verbatim failed: {rc}")
        return keys, int(counts[0]), int(counts[1])

    def time(self, points: np.ndarray, n_threads: int, iters: int) -> np.ndarray:
        """Wall ms of `iters` verbatim stage 1-7 runs (pipe_main_baseline.cpp)."""
        points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        ms = np.zeros(iters, np.float64)
        rc = self.lib.ref_cpu_time(_ptr(points), ctypes.c_uint32(points.shape[0]),
                                   ctypes.c_int(n_threads), ctypes.c_int(iters),
                                   _ptr(ms))
        if rc:
            raise RuntimeError(f"ref_cpu_time failed: {rc}")
        return ms

    def canonical(self, points: np.ndarray, n_threads: int = 1,
                  link_leaves: bool = False) -> TreeResult:
        """The reference's own per-element functions in the canonical dataflow;
        with link_leaves, its process_link_leaf after stage 7 (status 4 when
        some leaf's walk up the tree would never end on this cloud)."""
        points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        n = points.shape[0]
        cap = int(self.lib.ref_octree_capacity(ctypes.c_uint32(n)))
        r = _alloc_result(n, cap, 32)
        o = _RefOut(
            keys_after_stage1=_ptr(r.morton_keys).value,
            sorted_keys=_ptr(r.sorted_keys).value,
            unique_keys=_ptr(r.unique_keys).value, prefix_n=_ptr(r.prefix_n).value,
            has_leaf_left=_ptr(r.has_leaf_left).value,
            has_leaf_right=_ptr(r.has_leaf_right).value,
            left_child=_ptr(r.left_child).value, parents=_ptr(r.parents).value,
            edge_count=_ptr(r.edge_count).value, edge_offset=_ptr(r.edge_offset).value,
            children=_ptr(r.children).value, corner=_ptr(r.corner).value,
            cell_size=_ptr(r.cell_size).value,
            child_node_mask=_ptr(r.child_node_mask).value,
            child_leaf_mask=_ptr(r.child_leaf_mask).value)
        fn = self.lib.ref_canonical_linked if link_leaves else self.lib.ref_canonical
        rc = fn(_ptr(points), ctypes.c_uint32(n), ctypes.c_int(n_threads), ctypes.byref(o))
        r.status = int(rc)
        r.n_unique, r.n_brt_nodes = o.n_unique, o.n_brt_nodes
        r.n_octree_nodes = o.n_octree_nodes
        return r


def ref_cuda_available(path: str = REF_CUDA_SO) -> bool:
    return os.path.exists(path)


class RefTreeCuda:
    """The reference's own CUDA tree path (cuda::run_stage1..7 compiled for
    sm_100a, _ref/libref_tree_cuda.so, driven by ref_cuda_driver.cu): a timing
    comparison point on the same GPU, not a checker."""

    def __init__(self, path: str = REF_CUDA_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        self.lib = ctypes.CDLL(path)

    def time(self, points: np.ndarray, iters: int) -> dict:
        """Wall ms of `iters` runs (n a multiple of 1024) and what ran."""
        points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        n = points.shape[0]
        ms = np.zeros(iters, np.float64)
        info = np.zeros(7, np.uint32)
        stage_ms = np.zeros(7, np.float64)
        err = ctypes.create_string_buffer(512)
        rc = self.lib.refcu_time(_ptr(points), ctypes.c_uint32(n), ctypes.c_int(iters),
                                 _ptr(ms), _ptr(info), _ptr(stage_ms), err, ctypes.c_int(512))
        if rc:
            raise RuntimeError(f"refcu_time: status {rc} {err.value.decode()}")
        return {"ms": ms.tolist(), "all_stages_ran": bool(info[0]),
                "rows_out_of_range": int(info[1]), "parents_out_of_range": int(info[2]),
                "n_unique": int(info[3]),
                "n_octree_nodes": None if info[4] == 0xFFFFFFFF else int(info[4]),
                "stage4_input_unsorted": bool(info[5]),
                "stage6_did_not_launch": bool(info[6]),
                "stage_ms_last_run": [round(float(x), 4) for x in stage_ms]}


def compare(a: TreeResult, b: TreeResult) -> list[str]:
    """Names of the outputs where two results differ (bit-exact)."""
    ta, tb = a.trimmed(), b.trimmed()
    bad = []
    for k in sorted(set(ta) | set(tb)):
        va, vb = ta.get(k), tb.get(k)
        if isinstance(va, np.ndarray) and isinstance(vb, np.ndarray):
            if va.shape != vb.shape or va.tobytes() != vb.tobytes():
                bad.append(k)
        elif va != vb:
            bad.append(k)
    return bad
