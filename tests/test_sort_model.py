"""The pass scheme of the GFD search's warp quicksort (warp_aquicksort in
ap-cloud-cosmology_b200/csrc/gfd.cu), modelled lane by lane in Python, against the
reference's quicksort (apartition / aquickSort, solver.cpp:600-632, restated here as the
oracle restates it in oracle/apc_oracle.c).

The kernel partitions every unsorted sub-range in each pass, using the reference's partition
on each: the scan from the left stops at elements > pivot, the scan from the right at
elements <= pivot, and the pivot takes the crossing point.  A quicksort's result depends only
on the partition applied to each sub-range, not on the order in which disjoint sub-ranges are
taken.  So the first `limit` positions must equal those of the full sort, ties included.  Ties
decide which neighbours enter a stencil, so the model is checked on lists with many equal
keys.  The kernel itself is checked on the GPU through the bit-exact cells and fields.
"""
from __future__ import annotations

import random

import pytest

FULL = 0xFFFFFFFF


def reference_sort(keys, idx):
    """aquickSort over the whole list (solver.cpp:600-632)."""
    a, b = list(keys), list(idx)

    def partition(l, r):
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

    stack = [(0, len(a) - 1)]
    while stack:
        l, r = stack.pop()
        if l < r:
            j = partition(l, r)
            stack += [(l, j - 1), (j + 1, r)]
    return a, b


def _popc(x):
    return bin(x & FULL).count("1")


def _select_bit(mask, k):
    """Position of the k-th set bit from the bottom (the kernel's select_bit)."""
    p, s = 0, 16
    while s:
        c = _popc(mask & ((1 << s) - 1))
        if k >= c:
            k -= c
            mask >>= s
            p += s
        s >>= 1
    return p


def warp_sort_model(keys, idx, n, limit):
    """The kernel's passes over 32 lanes: masks are the warp ballots, list indexing the shuffles."""
    key = list(keys) + [0.0] * (32 - n)
    ix = list(idx) + [0] * (32 - n)
    U = FULL if n >= 32 else (1 << n) - 1
    lim = FULL if limit >= 32 else (1 << limit) - 1
    while True:
        R, E = U & ~(U << 1) & FULL, U & ~(U >> 1)
        U &= ~(R & E & lim)
        R, E = U & ~(U << 1) & FULL, U & ~(U >> 1)
        start, end, active = [0] * 32, [0] * 32, [False] * 32
        for ln in range(32):
            if (U >> ln) & 1:
                start[ln] = (R & ((2 << ln) - 1)).bit_length() - 1
                e = E & ~((1 << ln) - 1)
                end[ln] = (e & -e).bit_length() - 1
                active[ln] = start[ln] < limit and start[ln] < end[ln]
        if not any(active):
            break
        pivot = [key[start[ln]] if active[ln] else key[ln] for ln in range(32)]
        gt = sum(1 << ln for ln in range(32) if active[ln] and ln > start[ln] and key[ln] > pivot[ln])
        le = sum(1 << ln for ln in range(32) if active[ln] and key[ln] <= pivot[ln])
        seg = [((2 << end[ln]) - 1) & ~((1 << start[ln]) - 1) if active[ln] else 0 for ln in range(32)]
        partner = [-1] * 32
        for ln in range(32):
            gts, les = gt & seg[ln], le & seg[ln]
            nle = _popc(les)
            if (gts >> ln) & 1:
                k = _popc(gts & ((1 << ln) - 1))
                if k < nle:
                    sk = _select_bit(les, nle - 1 - k)
                    if sk > ln:
                        partner[ln] = sk
        pb = sum(1 << ln for ln in range(32) if partner[ln] >= 0)
        K = [_popc(pb & seg[ln]) for ln in range(32)]
        for ln in range(32):
            gts, les = gt & seg[ln], le & seg[ln]
            if (les >> ln) & 1:
                k = _popc(les) - 1 - _popc(les & ((1 << ln) - 1))
                if k < K[ln]:
                    partner[ln] = _select_bit(gts, k)
        src = [p if p >= 0 else ln for ln, p in enumerate(partner)]
        key, ix = [key[s] for s in src], [ix[s] for s in src]
        j = list(range(32))
        for ln in range(32):
            if active[ln]:
                gts, les = gt & seg[ln], le & seg[ln]
                nle = _popc(les)
                j[ln] = (les.bit_length() - 1 if K[ln] == 0
                         else max(_select_bit(les, nle - 1 - K[ln]), _select_bit(gts, K[ln] - 1)))
        src2 = [(j[ln] if ln == start[ln] else (start[ln] if ln == j[ln] else ln)) if active[ln] else ln
                for ln in range(32)]
        key, ix = [key[s] for s in src2], [ix[s] for s in src2]
        U &= ~sum(1 << ln for ln in range(32) if active[ln] and ln == j[ln])
    return key[:n], ix[:n]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_all_subrange_passes_give_the_reference_order(seed):
    rng = random.Random(seed)
    for _ in range(600):
        n = rng.randint(1, 32)
        pool = rng.choice([[0.0, 1.0, 2.0], [float(v) for v in range(6)], None])
        keys = [rng.choice(pool) if pool else rng.random() for _ in range(n)]
        idx = rng.sample(range(1000), n)
        limit = rng.choice([n, 17, 9, 1, rng.randint(1, 32)])
        ra, rb = reference_sort(keys, idx)
        ma, mb = warp_sort_model(keys, idx, n, limit)
        m = min(limit, n)
        assert ma[:m] == ra[:m] and mb[:m] == rb[:m], (keys, idx, limit)
