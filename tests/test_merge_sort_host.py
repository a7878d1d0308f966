"""The index algebra of the merge sort (stardust_b200/csrc/sd_resort.cu), on the CPU.

Positions sorted by their old row keys, some keys changed, one bit per position
marking at least the changed ones: the merge places every position by counts
alone, and the result must be the stable sort of the new keys, with the new row
table derived from the old one. This states the formulas the kernels evaluate
and checks them against numpy's stable argsort, including marked positions whose
key did not change (bits left over from a step whose merge never ran). The GPU
tests check the kernels themselves against the full radix sort.
"""
import numpy as np
import pytest


def merge_by_counts(old, new, marked, rows):
    """Permutation and new row table by the merge formulas (vectorised)."""
    n = len(old)
    rs_old = np.searchsorted(old, np.arange(rows + 1), side="left")
    below = np.concatenate([[0], np.cumsum(marked)])  # changed_below(x) = below[x]
    ci = np.nonzero(marked)[0]                         # C in position order
    o = np.argsort(new[ci], kind="stable")
    ck, ci = new[ci][o], ci[o]                         # C sorted by key, stable
    c_rows = np.searchsorted(ck, np.arange(rows + 1), side="left")
    perm = np.full(n, -1, np.int64)
    # changed (k, i) at rank r: r + unchanged below the old row start of k, plus the
    # unchanged ones of the old row k below i
    r = np.arange(len(ci))
    lb, ub = rs_old[ck], rs_old[ck + 1]
    m = np.minimum(ub, ci)
    u = (lb - below[lb]) + np.where(ci > lb, (m - lb) - (below[m] - below[lb]), 0)
    perm[r + u] = ci
    # unchanged (k, j): j - changed below j + C with key < k + C with key k below j
    j = np.nonzero(~marked)[0]
    k = new[j]
    before = np.searchsorted(ck * (n + 1) + ci, k * (n + 1) + j)  # C before (k, j)
    perm[j - below[j] + before] = j
    rs_new = rs_old - below[rs_old] + c_rows
    return perm, rs_new


def scene(n, rows, frac, seed, stale=0.0, clustered=False):
    rng = np.random.default_rng(seed)
    old = np.sort(rng.integers(0, rows, n)).astype(np.int64)
    new = old.copy()
    moved = rng.random(n) < frac
    if clustered:
        new[moved] = rows // 2
    else:
        new[moved] = np.clip(old[moved] + rng.choice([-16, -4, -1, 1, 4, 16], moved.sum()), 0, rows - 1)
    marked = (new != old) | (rng.random(n) < stale)
    return old, new, marked


@pytest.mark.parametrize("n,rows,frac,stale,clustered", [
    (1, 16, 1.0, 0.0, False),
    (1000, 16, 0.1, 0.0, False),
    (65536, 256, 0.01, 0.0, False),
    (200_000, 4096, 0.005, 0.0, False),
    (70_000, 1024, 0.3, 0.0, False),
    (5000, 16, 0.0, 0.0, False),          # nothing moved: the identity
    (3000, 64, 1.0, 0.0, False),          # everything moved
    (66_000, 128, 0.05, 0.0, True),       # the changed keys all in one row
    (20_000, 64, 0.02, 0.1, False),       # stale marks on unchanged positions
    (20_000, 64, 0.0, 0.3, False),
])
def test_merge_formulas_give_the_stable_sort(n, rows, frac, stale, clustered):
    old, new, marked = scene(n, rows, frac, n + rows, stale, clustered)
    perm, rs_new = merge_by_counts(old, new, marked, rows)
    ref = np.argsort(new, kind="stable")
    assert np.array_equal(perm, ref)
    assert np.array_equal(rs_new, np.searchsorted(new[ref], np.arange(rows + 1), side="left"))


def test_an_unmarked_change_breaks_the_merge():
    """The marks must cover every changed position: with one left out, the
    unchanged run it sits in is no longer sorted and the formulas place it wrong."""
    old, new, marked = scene(20_000, 64, 0.02, 7)
    i = np.nonzero(marked)[0][len(np.nonzero(marked)[0]) // 2]
    marked[i] = False
    perm, _ = merge_by_counts(old, new, marked, 64)
    assert not np.array_equal(perm, np.argsort(new, kind="stable"))
