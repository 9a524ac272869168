"""The bound the radix-tree kernel relies on for its in-block far-gap list
(k_radix_tree, csrc/k_tree.cu): for sorted distinct keys, two gaps whose
nearest strictly smaller gap lies beyond the tile's window on the same side
never share a delta, so a tile of 2,048 gaps with a 256-gap halo on each side
holds at most 32 such gaps per side with 30-bit codes (64 with 63-bit codes),
within the 128 entries of the list.  Checked here on the CPU, with plain numpy,
over random, clustered and constructed key sets."""
import numpy as np
import pytest

TILE, HALO, LIST = 2048, 256, 128


def deltas(keys: np.ndarray, bits: int) -> np.ndarray:
    """Length of the common prefix of consecutive keys (any strictly monotone
    function of clz(a ^ b) orders the gaps the same way)."""
    x = (keys[:-1] ^ keys[1:]).astype(np.uint64)
    assert (x > 0).all(), "keys must be distinct"
    length = np.zeros(len(x), np.int64)  # bit length of x, exactly
    for b in range(64):
        length += (x >> np.uint64(b)) > 0
    return bits - length


def nearest_smaller(d: np.ndarray):
    """For every gap: the nearest gap with a strictly smaller delta on the left
    (-1 if none: the wall) and on the right (n if none)."""
    n = len(d)
    left = np.full(n, -1, np.int64)
    right = np.full(n, n, np.int64)
    stack = []
    for g in range(n):
        while stack and d[stack[-1]] >= d[g]:
            stack.pop()
        left[g] = stack[-1] if stack else -1
        stack.append(g)
    stack = []
    for g in range(n - 1, -1, -1):
        while stack and d[stack[-1]] >= d[g]:
            stack.pop()
        right[g] = stack[-1] if stack else n
        stack.append(g)
    return left, right


def far_gaps_per_tile(keys: np.ndarray, bits: int):
    d = deltas(keys, bits)
    n = len(d)
    left, right = nearest_smaller(d)
    # adjacent gaps never share a delta
    assert (d[1:] != d[:-1]).all()
    worst = 0
    for g0 in range(0, n, TILE):
        g1 = min(g0 + TILE, n)
        wlo, whi = g0 - HALO, g0 + TILE + HALO - 1  # the window's first and last gap
        gs = np.arange(g0, g1)
        # a wall (-1 or n) inside the window is found like a smaller gap
        far_l = gs[left[gs] < wlo]
        far_r = gs[right[gs] > whi]
        # the values of one side's far gaps are distinct
        assert len(np.unique(d[far_l])) == len(far_l)
        assert len(np.unique(d[far_r])) == len(far_r)
        worst = max(worst, len(far_l), len(far_r), len(np.union1d(far_l, far_r)))
    return worst


def key_sets(bits: int, n: int, seed: int):
    rng = np.random.default_rng(seed)
    top = 1 << bits
    out = {"uniform": np.unique(rng.integers(0, top, size=n, dtype=np.uint64))}
    centres = rng.integers(0, top, size=8, dtype=np.uint64)
    spread = rng.integers(1 << 8, 1 << 20, size=n, dtype=np.uint64)
    pick = rng.integers(0, 8, size=n)
    cl = np.minimum(centres[pick] + spread, np.uint64(top - 1))
    out["clustered"] = np.unique(cl)
    out["consecutive"] = np.arange(10, 10 + n, dtype=np.uint64)
    # staircases: runs of deep gaps separated by gaps whose deltas climb one
    # level at a time (every level of the code once), repeated at 32 offsets
    steps = []
    for j in range(32):
        k = j << (bits - 5)
        for level in range(bits - 7, 0, -1):
            for _ in range(40):
                k += 1
                steps.append(k)
            k = ((k >> level) + 1) << level
            steps.append(k)
    out["staircase"] = np.unique(np.array(steps, np.uint64))
    return out


@pytest.mark.parametrize("bits,cap", [(30, 32), (63, 64)])
def test_far_gaps_of_a_tile_fit_the_list(bits, cap):
    for seed in (1, 2):
        for name, keys in key_sets(bits, 60_000, seed).items():
            worst = far_gaps_per_tile(keys, bits)
            assert worst <= min(2 * cap, LIST), (bits, name, worst)
            assert worst <= 2 * cap
