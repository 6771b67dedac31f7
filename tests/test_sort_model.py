"""The GFD search's sort (reference_sort and aquicksort in
ap-cloud-cosmology_b200/csrc/gfd.cu), modelled in Python, against the reference's quicksort
(apartition / aquickSort, solver.cpp:600-632, restated here as the oracle restates it in
oracle/apc_oracle.c).

The kernel runs the reference's partition with an explicit stack: it takes the smaller side
first (which bounds the stack) and does not enter a sub-range that starts at or beyond `limit`
(those only permute unwanted positions).  A quicksort's result depends only on the partition
applied to each sub-range, not on the order in which disjoint sub-ranges are taken, so the
first `limit` positions must equal those of the full sort, ties included.  Ties decide which
neighbours enter a stencil, so the model is checked on lists with many equal keys, and the
whole sort tail of searchneighboroctant (octant 0's quicksort, the 1e4^rank penalties, the
final quicksort) against the reference's sequence.  The kernel itself is checked on the GPU
through the bit-exact stencils, cells and fields.
"""
from __future__ import annotations

import random

import pytest


def _partition(a, b, l, r):
    pivot, i, j = a[l], l, r + 1
    while True:
        i += 1
        while i <= r and a[i] <= pivot:
            i += 1
        j -= 1
        while a[j] > pivot:
            j -= 1
        if i >= j:
            break
        a[i], a[j] = a[j], a[i]
        b[i], b[j] = b[j], b[i]
    a[l], a[j] = a[j], a[l]
    b[l], b[j] = b[j], b[l]
    return j


def reference_quicksort(a, b, l, r):
    """aquickSort (solver.cpp:600-613), recursion as the reference takes it."""
    if l < r:
        j = _partition(a, b, l, r)
        reference_quicksort(a, b, l, j - 1)
        reference_quicksort(a, b, j + 1, r)


def kernel_quicksort(a, b, l, r, limit):
    """The kernel's aquicksort: explicit stack, smaller side first, sub-ranges starting at
    or beyond `limit` skipped."""
    stack = []
    while True:
        if l >= r or l >= limit:
            if not stack:
                return
            l, r = stack.pop()
            continue
        j = _partition(a, b, l, r)
        if j - l < r - j:
            stack.append((j + 1, r))
            r = j - 1
        else:
            stack.append((l, j - 1))
            l = j + 1


def reference_tail(d2, idx, nn):
    """searchneighboroctant's sort (solver.cpp:553-569) on the bucket-ordered list: the
    per-octant quicksort at the running offset (only octant 0's run is the octant's own:
    the later calls sort positions of octant 0's zero-filled storage), the penalties, the
    whole-list quicksort."""
    nq = 10 * 17
    tdis = [0.0] * (8 * nq)
    tnb = [0] * (8 * nq)
    k = 0
    for o in range(8):
        for e in range(nn[o]):
            tdis[o * nq + e], tnb[o * nq + e] = d2[k], idx[k]
            k += 1
    dist, neigh = [], []
    k = 0
    for o in range(8):
        reference_quicksort(tdis, tnb, k, k + nn[o] - 1)
        penalty = 1.0
        for e in range(nn[o]):
            neigh.append(tnb[o * nq + e])
            dist.append(penalty * tdis[o * nq + e])
            penalty *= 10000.0
            k += 1
    reference_quicksort(dist, neigh, 0, len(dist) - 1)
    return dist, neigh


def kernel_tail(d2, idx, nn, lm):
    """reference_sort in gfd.cu: octant 0's run, the penalties in place, the list to lm."""
    a, b = list(d2), list(idx)
    kernel_quicksort(a, b, 0, nn[0] - 1, nn[0])
    k = 0
    for o in range(8):
        penalty = 1.0
        for _ in range(nn[o]):
            a[k] = penalty * a[k]
            penalty *= 10000.0
            k += 1
    kernel_quicksort(a, b, 0, len(a) - 1, lm)
    return a, b


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_limited_quicksort_gives_the_reference_order(seed):
    rng = random.Random(seed)
    for _ in range(600):
        n = rng.randint(1, 48)
        pool = rng.choice([[0.0, 1.0, 2.0], [float(v) for v in range(6)], None])
        keys = [rng.choice(pool) if pool else rng.random() for _ in range(n)]
        idx = rng.sample(range(1000), n)
        limit = rng.choice([n, 17, 9, 1, rng.randint(1, 48)])
        ra, rb = list(keys), list(idx)
        reference_quicksort(ra, rb, 0, n - 1)
        ka, kb = list(keys), list(idx)
        kernel_quicksort(ka, kb, 0, n - 1, limit)
        m = min(limit, n)
        assert ka[:m] == ra[:m] and kb[:m] == rb[:m], (keys, idx, limit)


@pytest.mark.parametrize("seed", [4, 5])
def test_sort_tail_gives_the_reference_stencil(seed):
    """Lattice-like squared distances (many exact ties across octants), 17 wanted."""
    rng = random.Random(seed)
    for _ in range(400):
        nn = [rng.randint(0, 6) for _ in range(8)]
        if sum(nn) < 17:
            nn[rng.randrange(8)] += 17 - sum(nn)
        l = sum(nn)
        d2 = [float(rng.choice([1, 2, 3, 4, 5, 6, 8, 9])) for _ in range(l)]
        idx = rng.sample(range(5000), l)
        rd, rn = reference_tail(d2, idx, nn)
        kd, kn = kernel_tail(d2, idx, nn, 17)
        assert kn[:17] == rn[:17] and kd[:17] == rd[:17], (d2, idx, nn)

